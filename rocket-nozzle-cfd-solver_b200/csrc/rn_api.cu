// rn_api.cu -- the C-ABI of librn.so (declared in include/rn.h).
//
// A handle owns all device memory of one solver instance and one CUDA stream.
// The layout in HBM is the reference's texture layout as plain arrays: a
// 3-slot ring of state planes A and B (float4 per cell, row-major), the
// geometry planes geoA ((Nx+1) x (Nr+1) float4), geoG and geoM (float4 per
// cell), the mask (1 byte per cell), two step-info float4s and two wave-speed
// slots; the spray ring is 2 x 3 planes of 65,536 float4 plus the deposit
// records. rn_step queues 2 kernels per step (stage 1, then stage 2 or stage 2
// fused with the viscous/reaction split step) and 3 more with sprays.
#include <cuda_runtime.h>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <algorithm>
#include <mutex>
#include <vector>
#include "rn.h"
#include "rn_internal.h"

using namespace rn;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(RN_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                              \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call);       \
  } while (0)

constexpr int SPRAY_N = 65536;

}  // namespace

// Shared with rn_static.cu and rn_batch.cu so their errors also reach rn_last_error().
int rn_record_error(int code, const std::string& msg) { return fail(code, msg); }
int rn_record_cuda(cudaError_t e, const char* what) { return cuda_fail(e, what); }

namespace {

void free_buffers(rn_solver* h) {
  if (h->stepGraph) cudaGraphExecDestroy(h->stepGraph);   // its launches name these buffers
  h->stepGraph = nullptr;
  cudaFree(h->SA[0]);   // base of the 6-plane state ring
  for (int s = 0; s < 3; s++) h->SA[s] = h->SB[s] = nullptr;
  cudaFree(h->geoA); cudaFree(h->geoG); cudaFree(h->geoM); cudaFree(h->jw); cudaFree(h->wallRow);
  cudaFree(h->maskP); cudaFree(h->dMaps); cudaFree(h->errFlag);
  h->maskP = nullptr; h->dMaps = nullptr; h->errFlag = nullptr;
  cudaFree(h->mask); cudaFree(h->stepTex); cudaFree(h->wmax); cudaFree(h->dInt);
  cudaFree(h->PA[0]);   // base of the 6-plane parcel ring
  for (int p = 0; p < 2; p++) h->PA[p] = h->PB[p] = h->PC[p] = nullptr;
  cudaFree(h->src); cudaFree(h->tab); cudaFree(h->dep); cudaFree(h->key); cudaFree(h->sortTemp);
  cudaFree(h->acc);
  h->acc = nullptr;
  cudaFree(h->depFlag);
  h->depFlag = nullptr;
  cudaFree(h->depBound);
  h->depBound = nullptr;
  cudaFree(h->liveSteps);
  h->liveSteps = nullptr;
  cudaFree(h->dHS);
  h->dHS = nullptr;
  cudaFree(h->xoff); cudaFree(h->xcell); cudaFree(h->heavy);
  h->xoff = h->xcell = nullptr;
  h->heavy = nullptr;
  h->nHeavy = 0;
  cudaFree(h->mark); cudaFree(h->dRes); cudaFree(h->wallProf); cudaFree(h->derived);
  h->mark = h->markSt = nullptr;
  h->dRes = nullptr;
  h->wallProf = nullptr;
  h->derived = nullptr;
  h->s1last = -1;
  h->maxX = 1;
  h->geoA = h->geoG = h->geoM = h->jw = h->wallRow = nullptr;
  h->mask = nullptr; h->stepTex = nullptr; h->wmax = nullptr; h->dInt = nullptr;
  h->src = h->tab = h->dep = nullptr;
  h->key = h->val = h->keyS = h->valS = nullptr;
  h->sortTemp = nullptr;
}

int spray_reset_dev(rn_solver* h) {
  // PA = (-1, -1, 0, 0), PB = PC = 0 for both ring copies (spray.js:242-254)
  std::vector<float4> dead(SPRAY_N, make_float4(-1.f, -1.f, 0.f, 0.f));
  for (int p = 0; p < 2; p++) {
    CK(cudaMemcpyAsync(h->PA[p], dead.data(), sizeof(float4) * SPRAY_N, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->PB[p], 0, sizeof(float4) * SPRAY_N, h->stream));
    CK(cudaMemsetAsync(h->PC[p], 0, sizeof(float4) * SPRAY_N, h->stream));
  }
  CK(cudaMemsetAsync(h->acc, 0, sizeof(unsigned long long) * 8 * size_t(h->Nx) * h->Nr, h->stream));
  if (h->depBound) CK(cudaMemsetAsync(h->depBound, 0, sizeof(unsigned) * 4, h->stream));
  if (h->liveSteps) CK(cudaMemsetAsync(h->liveSteps, 0, sizeof(unsigned long long), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->head = 0;
  h->scur = 0;
  return RN_OK;
}

int alloc_buffers(rn_solver* h, int Nx, int Nr) {
  if (Nx < 1 || Nr < 1 || (long long)Nx * Nr > (1LL << 28)) return fail(RN_ERR_ARG, "grid size out of range");
  free_buffers(h);
  h->Nx = Nx; h->Nr = Nr;
  const size_t N = size_t(Nx) * Nr, NF = size_t(Nx + 1) * (Nr + 1);
  float4* ring = nullptr;
  cudaError_t e = cudaMalloc(&ring, sizeof(float4) * N * 6);
  if (e != cudaSuccess) return fail(RN_ERR_NOMEM, std::string("state allocation: ") + cudaGetErrorString(e));
  for (int s = 0; s < 3; s++) { h->SA[s] = ring + N * (2 * s); h->SB[s] = ring + N * (2 * s + 1); }
  CK(cudaMemsetAsync(ring, 0, sizeof(float4) * N * 6, h->stream));
  CK(cudaMalloc(&h->geoA, sizeof(float4) * NF));
  CK(cudaMalloc(&h->geoG, sizeof(float4) * N));
  CK(cudaMalloc(&h->geoM, sizeof(float4) * N));
  CK(cudaMalloc(&h->mask, N));
  CK(cudaMalloc(&h->jw, sizeof(float4) * Nx));
  CK(cudaMalloc(&h->wallRow, sizeof(float4) * Nx));
  CK(cudaMalloc(&h->stepTex, sizeof(float4) * 2));
  CK(cudaMalloc(&h->wmax, sizeof(unsigned) * 2));
  CK(cudaMalloc(&h->depFlag, sizeof(unsigned)));
  CK(cudaMalloc(&h->dHS, sizeof(unsigned) * 2));
  CK(cudaMemsetAsync(h->depFlag, 0, sizeof(unsigned), h->stream));
  CK(cudaMalloc(&h->depBound, sizeof(unsigned) * 4));
  CK(cudaMemsetAsync(h->depBound, 0, sizeof(unsigned) * 4, h->stream));
  CK(cudaMalloc(&h->liveSteps, sizeof(unsigned long long)));
  CK(cudaMemsetAsync(h->liveSteps, 0, sizeof(unsigned long long), h->stream));
  CK(cudaMalloc(&h->dInt, sizeof(double) * 16));
  CK(cudaMemsetAsync(h->geoA, 0, sizeof(float4) * NF, h->stream));
  CK(cudaMemsetAsync(h->geoG, 0, sizeof(float4) * N, h->stream));
  CK(cudaMemsetAsync(h->geoM, 0, sizeof(float4) * N, h->stream));
  CK(cudaMemsetAsync(h->mask, 0, N, h->stream));
  CK(cudaMemsetAsync(h->jw, 0, sizeof(float4) * Nx, h->stream));
  CK(cudaMemsetAsync(h->wallRow, 0, sizeof(float4) * Nx, h->stream));
  CK(cudaMemsetAsync(h->stepTex, 0, sizeof(float4) * 2, h->stream));
  CK(cudaMemsetAsync(h->wmax, 0, sizeof(unsigned) * 2, h->stream));
  // halo copies: pitched mask, error word, tensor maps
  h->maskPitch = (Nx + 15) / 16 * 16;
  CK(cudaMalloc(&h->maskP, size_t(h->maskPitch) * Nr));
  CK(cudaMemsetAsync(h->maskP, 0, size_t(h->maskPitch) * Nr, h->stream));
  CK(cudaMalloc(&h->errFlag, sizeof(unsigned)));
  CK(cudaMemsetAsync(h->errFlag, 0, sizeof(unsigned), h->stream));
  CK(cudaMalloc(&h->dMaps, sizeof(TileMaps) * NTILES));
  {
    const int rcm = rn_build_tile_maps(h);
    if (rcm != RN_OK) return rcm;
  }
  // spray ring and deposit records
  float4* pr = nullptr;
  CK(cudaMalloc(&pr, sizeof(float4) * SPRAY_N * 6));
  for (int p = 0; p < 2; p++) {
    h->PA[p] = pr + SPRAY_N * (3 * p);
    h->PB[p] = pr + SPRAY_N * (3 * p + 1);
    h->PC[p] = pr + SPRAY_N * (3 * p + 2);
  }
  CK(cudaMalloc(&h->src, sizeof(float4) * N));
  CK(cudaMemsetAsync(h->src, 0, sizeof(float4) * N, h->stream));
  CK(cudaMalloc(&h->acc, sizeof(unsigned long long) * 8 * N));
  CK(cudaMemsetAsync(h->acc, 0, sizeof(unsigned long long) * 8 * N, h->stream));
  CK(cudaMalloc(&h->tab, sizeof(float4) * 768));
  CK(cudaMemsetAsync(h->tab, 0, sizeof(float4) * 768, h->stream));
  CK(cudaMalloc(&h->dep, sizeof(float4) * SPRAY_N));
  CK(cudaMalloc(&h->key, sizeof(unsigned) * SPRAY_N * 4));
  h->val = h->key + SPRAY_N;
  h->keyS = h->key + 2 * SPRAY_N;
  h->valS = h->key + 3 * SPRAY_N;
  h->sortTempBytes = std::max(kernels_exact.sortTempBytes(int(N)), kernels_fast.sortTempBytes(int(N)));
  CK(cudaMalloc(&h->sortTemp, h->sortTempBytes > 0 ? h->sortTempBytes : 16));
  h->cur = 0; h->stepIdx = 0; h->wslot = 0; h->wvalid = false; h->stepCount = 0;
  h->seed = 1;
  // empty topology (no groups) until a geometry is set
  h->hostMask.assign(N, 0);
  h->hostGeoM.assign(N * 4, 0.0f);
  int rc = rn_build_member_lists(h);
  if (rc != RN_OK) return rc;
  return spray_reset_dev(h);
}

bool valid(rn_solver* h) { return h != nullptr && h->SA[0] != nullptr; }

// cuTensorMapEncodeTiled from the driver (the library links the runtime only).
using EncodeTiledFn = decltype(&cuTensorMapEncodeTiled);
EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

}  // namespace

// The halo copies of a tile shape with PX x PY halo cells: each float4 plane
// as a (4 Nx) x Nr float32 tensor with a (4 PX) x PY box; the mask as an
// Nx x Nr byte tensor (rows maskPitch bytes apart) with an MW x PY box.
// Boxes that reach past the grid read zeros there.
int rn_build_tile_maps(rn_solver* h) {
  const EncodeTiledFn enc = encode_tiled();
  if (!enc) return fail(RN_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the CUDA driver");
  const int Nx = h->Nx, Nr = h->Nr;
  std::vector<TileMaps> maps(NTILES);
  const cuuint32_t estr[2] = {1, 1};
  for (int t = 0; t < NTILES; t++) {
    const int PX = TILE_TX[t] + 4, PY = TILE_TY[t] + 4;
    const cuuint64_t pdim[2] = {cuuint64_t(4) * Nx, cuuint64_t(Nr)};
    const cuuint64_t pstride[1] = {cuuint64_t(16) * Nx};
    const cuuint32_t pbox[2] = {cuuint32_t(4 * PX), cuuint32_t(PY)};
    for (int s = 0; s < 6; s++) {
      CUtensorMap* m = s < 3 ? &maps[t].a[s] : &maps[t].b[s - 3];
      void* base = s < 3 ? static_cast<void*>(h->SA[s]) : static_cast<void*>(h->SB[s - 3]);
      CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, pdim, pstride, pbox, estr,
                       CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                       CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return fail(RN_ERR_CUDA, "cuTensorMapEncodeTiled (state plane) failed: " + std::to_string(r));
    }
    const cuuint64_t mdim[2] = {cuuint64_t(Nx), cuuint64_t(Nr)};
    const cuuint64_t mstride[1] = {cuuint64_t(h->maskPitch)};
    const cuuint32_t mbox[2] = {cuuint32_t(mask_box_width(PX)), cuuint32_t(PY)};
    CUresult r = enc(&maps[t].mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, h->maskP, mdim, mstride, mbox, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(RN_ERR_CUDA, "cuTensorMapEncodeTiled (mask) failed: " + std::to_string(r));
    // the cell geometry planes for shapes that stage them (TILE_WARPS < 32)
    const cuuint32_t gmbox[2] = {cuuint32_t(4 * (TILE_TX[t] + 2)), cuuint32_t(TILE_TY[t] + 2)};
    const cuuint32_t ggbox[2] = {cuuint32_t(4 * TILE_TX[t]), cuuint32_t(TILE_TY[t])};
    r = enc(&maps[t].geoM, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->geoM, pdim, pstride, gmbox, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r == CUDA_SUCCESS)
      r = enc(&maps[t].geoG, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, h->geoG, pdim, pstride, ggbox, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(RN_ERR_CUDA, "cuTensorMapEncodeTiled (geometry) failed: " + std::to_string(r));
  }
  CK(cudaMemcpyAsync(h->dMaps, maps.data(), sizeof(TileMaps) * NTILES, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_mask_refresh(rn_solver* h) {
  CK(cudaMemcpy2DAsync(h->maskP, size_t(h->maskPitch), h->mask, size_t(h->Nx), size_t(h->Nx), size_t(h->Nr),
                       cudaMemcpyDeviceToDevice, h->stream));
  return RN_OK;
}

// Per tile, the cells outside it that belong to a cut-cell group with a cell
// inside it (a sliver merged across the tile edge). Groups are a host plus the
// slaves of its slave mask (geoM.z bits 1/2/4/8, cutcell.js:168-174).
int rn_build_member_lists(rn_solver* h) {
  if (h->stepGraph) cudaGraphExecDestroy(h->stepGraph);   // its launches name the old lists
  h->stepGraph = nullptr;
  const int TX = TILE_TX[h->tile], TY = TILE_TY[h->tile];
  const int Nx = h->Nx, Nr = h->Nr, tx = (Nx + TX - 1) / TX, nT = tx * ((Nr + TY - 1) / TY);
  const uint8_t* mask = h->hostMask.data();
  const float* geoM = h->hostGeoM.data();
  std::vector<std::vector<int>> lists(nT);
  auto tile_of = [&](int k) { return ((k / Nx) / TY) * tx + (k % Nx) / TX; };
  for (int k = 0; k < Nx * Nr; k++) {
    if (mask[k] || geoM[4 * k] != 0.0f || geoM[4 * k + 1] != 0.0f) continue;   // hosts only
    const int sm = int(std::lrint(geoM[4 * k + 2])) & 15;
    if (!sm) continue;
    int mem[5], nm = 0;
    mem[nm++] = k;
    if (sm & 1) mem[nm++] = k - 1;
    if (sm & 2) mem[nm++] = k + 1;
    if (sm & 4) mem[nm++] = k - Nx;
    if (sm & 8) mem[nm++] = k + Nx;
    for (int a = 0; a < nm; a++) {
      const int t = tile_of(mem[a]);
      for (int b = 0; b < nm; b++) {
        if (tile_of(mem[b]) == t) continue;
        std::vector<int>& L = lists[t];
        bool have = false;
        for (int c : L) have |= (c == mem[b]);
        if (!have) L.push_back(mem[b]);
      }
    }
  }
  std::vector<int> off(nT + 1, 0), cells;
  int maxX = 1;
  for (int t = 0; t < nT; t++) {
    off[t + 1] = off[t] + int(lists[t].size());
    maxX = std::max(maxX, int(lists[t].size()));
    cells.insert(cells.end(), lists[t].begin(), lists[t].end());
  }
  if (maxX > MAXX)
    return fail(RN_ERR_ARG, "rn_set_geometry: a tile has " + std::to_string(maxX) + " out-of-tile group members (limit " +
                                std::to_string(MAXX) + ")");
  if (cells.empty()) cells.push_back(0);
  CK(cudaStreamSynchronize(h->stream));
  cudaFree(h->xoff);
  cudaFree(h->xcell);
  h->xoff = h->xcell = nullptr;
  CK(cudaMalloc(&h->xoff, sizeof(int) * (nT + 1)));
  CK(cudaMalloc(&h->xcell, sizeof(int) * cells.size()));
  CK(cudaMemcpyAsync(h->xoff, off.data(), sizeof(int) * (nT + 1), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->xcell, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice, h->stream));
  // tiles whose lists need more shared memory than the common launch holds
  std::vector<int> heavy;
  for (int t = 0; t < nT; t++)
    if (off[t + 1] - off[t] > XSMALL) heavy.push_back(t);
  cudaFree(h->heavy);
  h->heavy = nullptr;
  h->nHeavy = 0;
  if (!heavy.empty()) {
    CK(cudaMalloc(&h->heavy, sizeof(int) * heavy.size()));
    CK(cudaMemcpyAsync(h->heavy, heavy.data(), sizeof(int) * heavy.size(), cudaMemcpyHostToDevice, h->stream));
    h->nHeavy = int(heavy.size());
  }
  CK(cudaStreamSynchronize(h->stream));
  h->maxX = maxX;
  h->hostXoff = off;
  return RN_OK;
}

namespace {

cudaEvent_t prof_event(rn_solver* h) {
  if (!h->evPool.empty()) {
    cudaEvent_t e = h->evPool.back();
    h->evPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
// brackets one kernel launch (or a launch group) with events when profiling
struct ProfScope {
  rn_solver* h;
  int kind;
  cudaEvent_t e0 = nullptr;
  ProfScope(rn_solver* h_, int kind_) : h(h_), kind(kind_) {
    if (h->prof) {
      e0 = prof_event(h);
      record(e0);
    }
  }
  ~ProfScope() {
    if (h->prof && e0) {
      cudaEvent_t e1 = prof_event(h);
      record(e1);
      (h->profCapture ? h->profGraphEv : h->evPending).push_back({kind, {e0, e1}});
    }
  }
  // while a graph is captured for profiling, as an event-record node of it
  void record(cudaEvent_t e) {
    if (h->profCapture) cudaEventRecordWithFlags(e, h->stream, cudaEventRecordExternal);
    else cudaEventRecord(e, h->stream);
  }
};

}  // namespace

// The CFL wave speed of the current state into wmax[wslot] (the value the
// previous step's last kernel would have left there).
int rn_ensure_wave_speed(rn_solver* h) {
  if (h->wvalid) return RN_OK;
  unsigned* w = h->wmax + h->wslot;
  CK(cudaMemsetAsync(w, 0, sizeof(unsigned), h->stream));
  {
    ProfScope ps(h, RN_K_REDUCE);
    h->K->reduce(h->grid(), h->SA[h->cur], h->SB[h->cur], w, h->stream);
  }
  h->launches++;
  h->wvalid = true;
  CK(cudaGetLastError());
  return RN_OK;
}

extern "C" {

const char* rn_last_error(void) { return g_err.c_str(); }

int rn_create(int Nx, int Nr, rn_handle* out) {
  if (!out) return fail(RN_ERR_ARG, "rn_create: out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(RN_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  rn_solver* h = new rn_solver();
  cudaGetDevice(&h->device);
  e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete h; return cuda_fail(e, "cudaStreamCreate"); }
  e = cudaEventCreateWithFlags(&h->asyncEv, cudaEventDisableTiming);
  if (e != cudaSuccess) { cudaStreamDestroy(h->stream); delete h; return cuda_fail(e, "cudaEventCreate"); }
  cudaDeviceGetAttribute(&h->numSMs, cudaDevAttrMultiProcessorCount, h->device);
  {
    // process-wide kernel attributes, once (the solve server creates handles
    // on its worker thread while callers may create their own)
    static std::mutex initMu;
    static bool kernels_ready = false;
    std::lock_guard<std::mutex> lk(initMu);
    if (!kernels_ready) {
      if (kernels_exact.init() != 0 || kernels_fast.init() != 0) {
        cudaEventDestroy(h->asyncEv);
        cudaStreamDestroy(h->stream);
        delete h;
        return fail(RN_ERR_CUDA, "rn_create: cannot size the stage kernels' shared memory");
      }
      kernels_ready = true;
    }
  }
  // default tile shape: 14x16 (compiled for 3 blocks per SM) when the grid's
  // tiles are all resident at 3 per SM at once, else 16x15
  if (Nx > 0 && Nr > 0 && ((Nx + 13) / 14) * ((Nr + 15) / 16) <= 3 * h->numSMs) h->tile = RN_TILE_14x16;
  int rc = alloc_buffers(h, Nx, Nr);
  if (rc != RN_OK) {
    std::string msg = g_err;
    free_buffers(h);
    cudaEventDestroy(h->asyncEv);
    cudaStreamDestroy(h->stream);
    delete h;
    return fail(rc, msg);
  }
  *out = h;
  return RN_OK;
}

int rn_destroy(rn_handle h) {
  if (!h) return RN_OK;
  rn_batch_detach(h);
  cudaStreamSynchronize(h->stream);
  free_buffers(h);
  if (h->copyStream) {
    cudaStreamSynchronize(h->copyStream);
    cudaStreamDestroy(h->copyStream);
    cudaEventDestroy(h->evGathered);
  }
  if (h->pinned) cudaFreeHost(h->pinned);
  if (h->asyncDev) cudaFree(h->asyncDev);
  for (auto& p : h->evPending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
  for (auto e : h->evPool) cudaEventDestroy(e);
  cudaEventDestroy(h->asyncEv);
  if (h->sprayStream) {
    cudaStreamSynchronize(h->sprayStream);
    cudaEventDestroy(h->evSprayFork);
    cudaEventDestroy(h->evSprayJoin);
    cudaStreamDestroy(h->sprayStream);
  }
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaEventDestroy(h->evFork);
    cudaEventDestroy(h->evJoin);
    cudaStreamDestroy(h->side);
  }
  cudaStreamDestroy(h->stream);
  delete h;
  return RN_OK;
}

int rn_resize(rn_handle h, int Nx, int Nr) {
  if (!h) return fail(RN_ERR_ARG, "rn_resize: NULL handle");
  rn_cancel_async(h);
  CK(cudaStreamSynchronize(h->stream));
  return alloc_buffers(h, Nx, Nr);
}

int rn_set_mask(rn_handle h, const uint8_t* mask) {
  if (!valid(h) || !mask) return fail(RN_ERR_ARG, "rn_set_mask: bad argument");
  const size_t N = size_t(h->Nx) * h->Nr;
  std::vector<uint8_t> m(N);
  for (size_t k = 0; k < N; k++) m[k] = mask[k] ? 1 : 0;
  CK(cudaMemcpyAsync(h->mask, m.data(), N, cudaMemcpyHostToDevice, h->stream));
  {
    const int rc = rn_mask_refresh(h);
    if (rc != RN_OK) return rc;
  }
  CK(cudaStreamSynchronize(h->stream));
  h->wvalid = false;
  return RN_OK;
}

int rn_set_geometry(rn_handle h, const uint8_t* mask, const float* geoA, const float* geoG, const float* geoM,
                    const float* jWall) {
  if (!valid(h) || !mask || !geoA || !geoG || !geoM) return fail(RN_ERR_ARG, "rn_set_geometry: bad argument");
  // topology sanity: host offsets are -1, 0, +1 along one axis and point inside the grid
  const int Nx = h->Nx, Nr = h->Nr;
  for (int k = 0; k < Nx * Nr; k++) {
    if (mask[k]) continue;
    float hx = geoM[4 * k], hy = geoM[4 * k + 1];
    int i = k % Nx, j = k / Nx;
    int ix = int(std::lrint(hx)), iy = int(std::lrint(hy));
    if (std::fabs(hx - ix) > 1e-3f || std::fabs(hy - iy) > 1e-3f || std::abs(ix) + std::abs(iy) > 1 || i + ix < 0 ||
        i + ix >= Nx || j + iy < 0 || j + iy >= Nr)
      return fail(RN_ERR_ARG, "rn_set_geometry: geoM host offset of cell " + std::to_string(k) + " is not a neighbour");
    int sm = int(std::lrint(geoM[4 * k + 2])) & 15;
    if (((sm & 1) && i == 0) || ((sm & 2) && i == Nx - 1) || ((sm & 4) && j == 0) || ((sm & 8) && j == Nr - 1))
      return fail(RN_ERR_ARG, "rn_set_geometry: slave bit of cell " + std::to_string(k) + " points outside the grid");
  }
  const size_t N = size_t(Nx) * Nr, NF = size_t(Nx + 1) * (Nr + 1);
  std::vector<uint8_t> oldMask = std::move(h->hostMask);
  std::vector<float> oldGeoM = std::move(h->hostGeoM);
  h->hostMask.resize(N);
  for (size_t k = 0; k < N; k++) h->hostMask[k] = mask[k] ? 1 : 0;
  h->hostGeoM.assign(geoM, geoM + 4 * N);
  int rc = rn_build_member_lists(h);
  if (rc != RN_OK) {
    std::string msg = g_err;
    h->hostMask = std::move(oldMask);
    h->hostGeoM = std::move(oldGeoM);
    rn_build_member_lists(h);
    return fail(rc, msg);
  }
  rc = rn_set_mask(h, mask);
  if (rc != RN_OK) return rc;
  CK(cudaMemcpyAsync(h->geoA, geoA, sizeof(float4) * NF, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->geoG, geoG, sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->geoM, geoM, sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
  if (jWall) CK(cudaMemcpyAsync(h->jw, jWall, sizeof(float4) * Nx, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_get_geometry(rn_handle h, uint8_t* mask, float* geoA, float* geoG, float* geoM, float* jWall) {
  if (!valid(h)) return fail(RN_ERR_ARG, "rn_get_geometry: bad handle");
  const size_t N = size_t(h->Nx) * h->Nr, NF = size_t(h->Nx + 1) * (h->Nr + 1);
  if (mask) CK(cudaMemcpyAsync(mask, h->mask, N, cudaMemcpyDeviceToHost, h->stream));
  if (geoA) CK(cudaMemcpyAsync(geoA, h->geoA, sizeof(float4) * NF, cudaMemcpyDeviceToHost, h->stream));
  if (geoG) CK(cudaMemcpyAsync(geoG, h->geoG, sizeof(float4) * N, cudaMemcpyDeviceToHost, h->stream));
  if (geoM) CK(cudaMemcpyAsync(geoM, h->geoM, sizeof(float4) * N, cudaMemcpyDeviceToHost, h->stream));
  if (jWall) CK(cudaMemcpyAsync(jWall, h->jw, sizeof(float4) * h->Nx, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_set_state(rn_handle h, const float* A, const float* B) {
  if (!valid(h) || !A || !B) return fail(RN_ERR_ARG, "rn_set_state: bad argument");
  const size_t N = size_t(h->Nx) * h->Nr;
  for (int s = 0; s < 3; s++) {
    CK(cudaMemcpyAsync(h->SA[s], A, sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->SB[s], B, sizeof(float4) * N, cudaMemcpyHostToDevice, h->stream));
  }
  CK(cudaMemsetAsync(h->stepTex, 0, sizeof(float4) * 2, h->stream));
  h->cur = 0; h->stepIdx = 0; h->stepCount = 0; h->wvalid = false; h->s1last = -1;
  return spray_reset_dev(h);
}

int rn_get_state(rn_handle h, float* A, float* B) {
  if (!valid(h) || !A || !B) return fail(RN_ERR_ARG, "rn_get_state: bad argument");
  const size_t N = size_t(h->Nx) * h->Nr;
  CK(cudaMemcpyAsync(A, h->SA[h->cur], sizeof(float4) * N, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(B, h->SB[h->cur], sizeof(float4) * N, cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

}  // extern "C"

namespace {
constexpr int STEP_PERIOD = 6;   // 3 ring shifts x 2 step-info parities

// One time step of handle h (the body of step(n, P), solver.js:849-891).
int step_once(rn_solver* h, const rn_params* P) {
  const Grid g = h->grid();
  const bool phys = P->visc || P->chem, inj = P->inj != 0;
  const int s0 = h->cur, s1 = (h->cur + 1) % 3, s2 = (h->cur + 2) % 3;
  unsigned* wIn = h->wmax + h->wslot;
  unsigned* wOut = h->wmax + (1 - h->wslot);
  if (!h->wvalid) {
    int rc = rn_ensure_wave_speed(h);
    if (rc != RN_OK) return rc;
  }
  float4* stPrev = h->stepTex + h->stepIdx;
  float4* stNew = h->stepTex + (1 - h->stepIdx);
  StageArgs a;
  a.g = g;
  a.A = h->SA[s0]; a.B = h->SB[s0]; a.A0 = h->SA[s0]; a.B0 = h->SB[s0];
  a.oA = h->SA[s1]; a.oB = h->SB[s1];
  a.stPrev = stPrev; a.stNew = stNew; a.wIn = wIn; a.wOut = wOut;
  a.finalCfl = 0;
  a.xoff = h->xoff; a.xcell = h->xcell; a.maxX = h->maxX;
  a.slotIn = s0; a.tm = h->dMaps; a.err = h->errFlag;
  {
    ProfScope ps(h, RN_K_STAGE1);
    h->K->stage1(a, *P, h->tile, h->stream);
  }
  h->launches++;
  if (inj) {
    SprayArgs sp;
    sp.g = g;
    sp.A1 = h->SA[s1]; sp.B1 = h->SB[s1];
    sp.PA = h->PA[h->scur]; sp.PB = h->PB[h->scur];
    sp.oPA = h->PA[1 - h->scur]; sp.oPB = h->PB[1 - h->scur]; sp.oPC = h->PC[1 - h->scur];
    sp.tab = h->tab; sp.st = stNew;
    sp.key = h->key; sp.val = h->val; sp.dep = h->dep;
    sp.acc = h->acc + size_t(4) * g.Nx * g.Nr * h->scur;
    sp.depFlag = h->depFlag;
    sp.boundIn = h->depBound + 2 * h->scur;
    sp.boundOut = h->depBound + 2 * (1 - h->scur);
    sp.liveSteps = h->liveSteps;
    sp.head = int(h->head); sp.seed = int(h->seed);
    sp.hs = h->hsOnDevice ? h->dHS : nullptr;
    int launched = 0;
    // The parcel step reads the stage-1 state and writes only the parcel
    // ring and the deposit sums, which stage 2 + the split step do not
    // touch: it runs on a stream of its own, beside them, and the apply
    // waits for it. (Profiling times it on the main stream instead.)
    cudaStream_t ss = h->stream;
    if (!h->prof) {
      if (!h->sprayStream) {
        CK(cudaStreamCreateWithFlags(&h->sprayStream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->evSprayFork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->evSprayJoin, cudaEventDisableTiming));
      }
      CK(cudaEventRecord(h->evSprayFork, h->stream));
      CK(cudaStreamWaitEvent(h->sprayStream, h->evSprayFork, 0));
      ss = h->sprayStream;
    }
    {
      ProfScope ps(h, RN_K_PARCELS);
      if (h->K->spray(sp, *P, h->sortTemp, h->sortTempBytes, h->keyS, h->valS, h->src, ss, &launched) != 0)
        return fail(RN_ERR_CUDA, "rn_step: deposit sort failed");
    }
    if (ss != h->stream) CK(cudaEventRecord(h->evSprayJoin, ss));
    h->launches += launched;
  }
  StageArgs b = a;
  b.A = h->SA[s1]; b.B = h->SB[s1]; b.A0 = h->SA[s0]; b.B0 = h->SB[s0];
  b.oA = h->SA[s2]; b.oB = h->SB[s2];
  b.slotIn = s1;
  b.finalCfl = (!phys && !inj) ? 1 : 0;
  if (phys) {
    // stage 2 + split step in one kernel; its output replaces the stage-2 slot
    PhysArgs p;
    p.g = g;
    p.A1 = h->SA[s1]; p.B1 = h->SB[s1]; p.A2 = h->SA[s2]; p.B2 = h->SB[s2];
    p.oA = h->SA[s2]; p.oB = h->SB[s2];
    p.st = stNew; p.wOut = wOut; p.finalCfl = inj ? 0 : 1;
    p.xoff = h->xoff; p.xcell = h->xcell; p.maxX = h->maxX;
    ProfScope ps(h, RN_K_STAGE2_PHYSICS);
    const int nTiles = int(h->hostXoff.size()) - 1;
    if (h->nHeavy > 0 && nTiles > SPLIT_BLOCKS_PER_SM * h->numSMs) {
      // the few tiles with long member lists on the side stream, at the same time
      if (!h->side) {
        CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming));
      }
      CK(cudaEventRecord(h->evFork, h->stream));
      CK(cudaStreamWaitEvent(h->side, h->evFork, 0));
      h->K->stage2phys(b, p, *P, h->tile, h->heavy, h->nHeavy, false, h->side);
      CK(cudaEventRecord(h->evJoin, h->side));
      h->K->stage2phys(b, p, *P, h->tile, nullptr, h->nHeavy, true, h->stream);
      CK(cudaStreamWaitEvent(h->stream, h->evJoin, 0));
      h->launches++;
    } else {
      h->K->stage2phys(b, p, *P, h->tile, nullptr, 0, false, h->stream);
    }
  } else {
    ProfScope ps(h, RN_K_STAGE2);
    h->K->stage2(b, *P, h->tile, h->stream);
  }
  h->launches++;
  h->cur = s2;
  if (inj) {
    if (!h->prof) CK(cudaStreamWaitEvent(h->stream, h->evSprayJoin, 0));   // the parcel step is done
    const int out = (h->cur + 1) % 3;
    ApplyArgs ap;
    ap.g = g;
    ap.A = h->SA[h->cur]; ap.B = h->SB[h->cur]; ap.src = h->src;
    ap.acc = h->acc + size_t(4) * g.Nx * g.Nr * h->scur;
    ap.accNext = h->acc + size_t(4) * g.Nx * g.Nr * (1 - h->scur);
    ap.boundIn = h->depBound + 2 * h->scur;
    ap.oA = h->SA[out]; ap.oB = h->SB[out];
    ap.wOut = wOut; ap.finalCfl = 1;
    ap.hsNext = h->hsOnDevice ? h->dHS : nullptr;
    {
      ProfScope ps(h, RN_K_APPLY);
      h->K->apply(ap, *P, h->stream);
    }
    h->launches++;
    h->cur = out;
    h->scur = 1 - h->scur;
    h->head = (h->head + 4) % SPRAY_N;
    h->seed = h->seed + 1u;
  }
  h->stepIdx = 1 - h->stepIdx;
  h->wslot = 1 - h->wslot;
  h->wvalid = true;
  h->s1last = s1;
  h->stepCount++;
  return RN_OK;
}

// Whether the handle's 6-step graph can replay the next steps with P: the
// kernels, launch shapes, buffers and parameter block it was captured with.
bool graph_matches(const rn_solver* h, const rn_params* P) {
  return h->stepGraph && h->graphK == h->K && h->graphTile == h->tile && h->graphMaxX == h->maxX &&
         h->graphHeavy == h->nHeavy && h->graphBase == h->SA[0] && h->graphXoff == h->xoff &&
         std::memcmp(&h->graphP, P, sizeof(rn_params)) == 0;
}
void drop_step_graph(rn_solver* h) {
  if (h->stepGraph) cudaGraphExecDestroy(h->stepGraph);
  h->stepGraph = nullptr;
}

// Profiling inside graph replays (rn_profile mode 2, steps without sprays):
// one period of the handle's launches is captured with an event pair around
// each kernel (event-record nodes of the graph) and replayed period by
// period, the pairs read after each replay, so each kernel is timed as it
// runs in the replayed graph (no host launch gaps between the kernels). The
// steps before the first whole period run one by one, timed launch by launch.
int prof_graph_steps(rn_solver* h, const rn_params* P, int n, int& done) {
  while (done < n && !h->wvalid) {
    int rc = step_once(h, P);
    if (rc != RN_OK) return rc;
    done++;
  }
  if (n - done < STEP_PERIOD) return RN_OK;
  if (h->nHeavy > 0 && !h->side) {   // the helper stream exists before the capture
    CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming));
  }
  const int cur = h->cur, stepIdx = h->stepIdx, wslot = h->wslot, s1last = h->s1last;
  const long long stepCount = h->stepCount, launches = h->launches;
  cudaGraph_t gr = nullptr;
  cudaGraphExec_t ex = nullptr;
  h->profGraphEv.clear();
  h->profCapture = true;
  cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
  int rc = RN_OK;
  for (int k = 0; k < STEP_PERIOD && rc == RN_OK && e == cudaSuccess; k++) rc = step_once(h, P);
  cudaError_t e2 = e == cudaSuccess ? cudaStreamEndCapture(h->stream, &gr) : e;
  h->profCapture = false;
  const long long perPeriod = h->launches - launches;
  h->cur = cur; h->stepIdx = stepIdx; h->wslot = wslot; h->s1last = s1last;
  h->stepCount = stepCount; h->launches = launches;
  auto release = [&]() {
    for (auto& p : h->profGraphEv) {
      h->evPool.push_back(p.second.first);
      h->evPool.push_back(p.second.second);
    }
    h->profGraphEv.clear();
    if (ex) cudaGraphExecDestroy(ex);
    if (gr) cudaGraphDestroy(gr);
  };
  if (rc != RN_OK) { release(); return rc; }
  if (e2 != cudaSuccess) { release(); return cuda_fail(e2, "rn_step: profiled graph capture"); }
  e = cudaGraphInstantiate(&ex, gr, 0);
  if (e != cudaSuccess) { ex = nullptr; release(); return cuda_fail(e, "rn_step: profiled graph instantiate"); }
  while (n - done >= STEP_PERIOD) {
    e = cudaGraphLaunch(ex, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    for (auto& p : h->profGraphEv) {
      float t = 0.0f;
      if (e == cudaSuccess) e = cudaEventElapsedTime(&t, p.second.first, p.second.second);
      h->profMs[p.first] += t;
      h->profN[p.first] += 1;
    }
    if (e != cudaSuccess) { release(); return cuda_fail(e, "rn_step: profiled graph replay"); }
    h->s1last = (h->cur + 1 + 2 * (STEP_PERIOD - 1)) % 3;
    h->stepCount += STEP_PERIOD;
    h->launches += perPeriod;
    done += STEP_PERIOD;
  }
  release();
  return RN_OK;
}
}  // namespace

extern "C" {

__global__ void k_set_hs(unsigned* hs, unsigned head, unsigned seed) {
  hs[0] = head;
  hs[1] = seed;
}

int rn_step(rn_handle h, int n, const rn_params* P) {
  if (!valid(h) || !P || n < 0) return fail(RN_ERR_ARG, "rn_step: bad argument");
  if (h->batch) return fail(RN_ERR_STATE, "rn_step: the handle is stepped by a batch");
  const bool inj = P->inj != 0;
  int done = 0;
  // The launch sequence repeats: every 6 steps without sprays (3 ring shifts x
  // 2 step-info parities), every 2 with them (the state ring stays put, the
  // step info, wave-speed slot and parcel ring alternate; the ring head and
  // seed are then read and advanced on the device). Whole periods replay from
  // a CUDA graph captured from the handle's own launches (not while
  // profiling, which brackets each kernel with events).
  const int period = inj ? 2 : STEP_PERIOD;
  auto at_start = [&]() {
    return h->cur == h->graphCur && h->stepIdx == h->graphStepIdx && h->wslot == h->graphWslot &&
           (!inj || h->scur == h->graphScur);
  };
  // (nor when the caller is capturing the handle's stream into a graph of its
  // own: the launches then go into that graph as they are)
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess) cs = cudaStreamCaptureStatusNone;
  if (h->prof == 2 && !inj && cs == cudaStreamCaptureStatusNone && n >= 2 * period) {
    int rc = prof_graph_steps(h, P, n, done);
    if (rc != RN_OK) return rc;
  }
  if (!h->prof && cs == cudaStreamCaptureStatusNone && n >= 2 * period) {
    while (done < n && (!h->wvalid || (graph_matches(h, P) && !at_start()))) {
      int rc = step_once(h, P);
      if (rc != RN_OK) return rc;
      done++;
    }
    if (n - done >= period && !graph_matches(h, P)) {
      drop_step_graph(h);
      if (h->nHeavy > 0 && !h->side) {   // the helper streams exist before the capture
        CK(cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->evFork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->evJoin, cudaEventDisableTiming));
      }
      if (inj && !h->sprayStream) {
        CK(cudaStreamCreateWithFlags(&h->sprayStream, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&h->evSprayFork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->evSprayJoin, cudaEventDisableTiming));
      }
      const int cur = h->cur, stepIdx = h->stepIdx, wslot = h->wslot, s1last = h->s1last, scur = h->scur;
      const uint32_t head = h->head, seed = h->seed;
      const long long stepCount = h->stepCount, launches = h->launches;
      cudaGraph_t gr = nullptr;
      h->hsOnDevice = inj;
      CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
      int rc = RN_OK;
      for (int k = 0; k < period && rc == RN_OK; k++) rc = step_once(h, P);
      cudaError_t e = cudaStreamEndCapture(h->stream, &gr);
      h->hsOnDevice = false;
      const long long perPeriod = h->launches - launches;
      h->cur = cur; h->stepIdx = stepIdx; h->wslot = wslot; h->s1last = s1last; h->scur = scur;
      h->head = head; h->seed = seed;
      h->stepCount = stepCount; h->launches = launches;
      if (rc != RN_OK) { if (gr) cudaGraphDestroy(gr); return rc; }
      if (e != cudaSuccess) { if (gr) cudaGraphDestroy(gr); return cuda_fail(e, "rn_step: graph capture"); }
      e = cudaGraphInstantiate(&h->stepGraph, gr, 0);
      cudaGraphDestroy(gr);
      if (e != cudaSuccess) { h->stepGraph = nullptr; return cuda_fail(e, "rn_step: graph instantiate"); }
      h->graphK = h->K; h->graphTile = h->tile; h->graphMaxX = h->maxX; h->graphHeavy = h->nHeavy;
      h->graphBase = h->SA[0]; h->graphXoff = h->xoff; h->graphP = *P;
      h->graphCur = cur; h->graphStepIdx = stepIdx; h->graphWslot = wslot; h->graphScur = scur;
      h->graphLaunches = perPeriod;
      h->graphPeriod = period;
    }
    if (graph_matches(h, P) && h->graphPeriod == period && h->wvalid && at_start() && n - done >= period) {
      if (inj) {   // the ring head and seed the graph's parcel kernels read
        k_set_hs<<<1, 1, 0, h->stream>>>(h->dHS, h->head, h->seed);
        h->launches++;
      }
      while (n - done >= period) {
        CK(cudaGraphLaunch(h->stepGraph, h->stream));
        // a period leaves the rings, step info and wave-speed slot where they were
        h->s1last = inj ? (h->cur + 1) % 3 : (h->cur + 1 + 2 * (period - 1)) % 3;
        if (inj) {
          h->head = (h->head + 4u * uint32_t(period)) % SPRAY_N;
          h->seed = h->seed + uint32_t(period);
        }
        h->stepCount += period;
        h->launches += h->graphLaunches;
        done += period;
      }
    }
  }
  for (; done < n; done++) {
    int rc = step_once(h, P);
    if (rc != RN_OK) return rc;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "rn_step launch");
  return RN_OK;
}

int rn_rescale_ambient(rn_handle h, float fp, float fT, float du, const rn_params* P) {
  if (!valid(h) || !P) return fail(RN_ERR_ARG, "rn_rescale_ambient: bad argument");
  const int s0 = h->cur, s1 = (h->cur + 1) % 3;
  {
    ProfScope ps(h, RN_K_OTHER);
    h->K->rescale(h->grid(), h->SA[s0], h->SB[s0], h->SA[s1], h->SB[s1], fp, fT, du, *P, h->stream);
  }
  h->launches++;
  h->cur = s1;
  h->wvalid = false;
  h->s1last = -1;
  CK(cudaGetLastError());
  return RN_OK;
}

int rn_draw_wall_row(rn_handle h) {
  if (!valid(h)) return fail(RN_ERR_ARG, "rn_draw_wall_row: bad handle");
  h->K->wallrow(h->grid(), h->SA[h->cur], h->SB[h->cur], h->jw, h->wallRow, h->stream);
  h->launches++;
  CK(cudaGetLastError());
  return RN_OK;
}

}  // extern "C"

namespace {
// device pointer, row pitch (float4) and extent of a named texture
int tex_ptr(rn_solver* h, int tex, const float4** p, int* W, int* H) {
  switch (tex) {
    case RN_TEX_A: *p = h->SA[h->cur]; *W = h->Nx; *H = h->Nr; return RN_OK;
    case RN_TEX_B: *p = h->SB[h->cur]; *W = h->Nx; *H = h->Nr; return RN_OK;
    case RN_TEX_STEPINFO: *p = h->stepTex + h->stepIdx; *W = 1; *H = 1; return RN_OK;
    case RN_TEX_WALLROW: *p = h->wallRow; *W = h->Nx; *H = 1; return RN_OK;
    case RN_TEX_PARCEL_A: *p = h->PA[h->scur]; *W = 256; *H = 256; return RN_OK;
    case RN_TEX_PARCEL_B: *p = h->PB[h->scur]; *W = 256; *H = 256; return RN_OK;
    case RN_TEX_PARCEL_C: *p = h->PC[h->scur]; *W = 256; *H = 256; return RN_OK;
    case RN_TEX_INJECTOR: *p = h->tab; *W = 256; *H = 3; return RN_OK;
    default: return fail(RN_ERR_ARG, "unknown texture " + std::to_string(tex));
  }
}
int queue_rect(rn_solver* h, int tex, int x, int y, int w, int hgt, float* dst) {
  const float4* p;
  int W, H;
  int rc = tex_ptr(h, tex, &p, &W, &H);
  if (rc != RN_OK) return rc;
  if (x < 0 || y < 0 || w < 0 || hgt < 0 || x + w > W || y + hgt > H) return fail(RN_ERR_ARG, "read rectangle out of range");
  if (w == 0 || hgt == 0) return RN_OK;
  CK(cudaMemcpy2DAsync(dst, sizeof(float4) * w, p + size_t(y) * W + x, sizeof(float4) * W, sizeof(float4) * w, hgt,
                       cudaMemcpyDeviceToHost, h->stream));
  return RN_OK;
}
}  // namespace

extern "C" {

int rn_read_rect(rn_handle h, int tex, int x, int y, int w, int hgt, float* out) {
  if (!valid(h) || !out) return fail(RN_ERR_ARG, "rn_read_rect: bad argument");
  int rc = queue_rect(h, tex, x, y, w, hgt, out);
  if (rc != RN_OK) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_read_step_info(rn_handle h, float out[4]) { return rn_read_rect(h, RN_TEX_STEPINFO, 0, 0, 1, 1, out); }

int rn_request_async(rn_handle h, const rn_read_req* reqs, int nreq, int tag) {
  if (!valid(h) || (nreq > 0 && !reqs) || nreq < 0) return fail(RN_ERR_ARG, "rn_request_async: bad argument");
  if (h->asyncBusy) return RN_BUSY;
  // the rectangles are gathered on the device by one kernel into a staging
  // buffer, which then crosses to pinned host memory in one copy
  std::vector<RectCopy> rects;
  size_t total = 0;   // float4 texels
  for (int r = 0; r < nreq; r++) {
    const float4* p;
    int W, H;
    int rc = tex_ptr(h, reqs[r].tex, &p, &W, &H);
    if (rc != RN_OK) return rc;
    const int x = reqs[r].x, y = reqs[r].y, w = reqs[r].w, hg = reqs[r].h;
    if (x < 0 || y < 0 || w < 0 || hg < 0 || x + w > W || y + hg > H)
      return fail(RN_ERR_ARG, "read rectangle out of range");
    if (w > 0 && hg > 0) rects.push_back(RectCopy{p, W, x, y, w, hg, (long long)total});
    total += size_t(w) * hg;
  }
  if (total > h->pinnedCap / 4 || total > h->asyncDevCap) {
    if (h->pinned) cudaFreeHost(h->pinned);
    if (h->asyncDev) cudaFree(h->asyncDev);
    h->pinned = nullptr;
    h->asyncDev = nullptr;
    h->pinnedCap = 0;
    h->asyncDevCap = 0;
    CK(cudaHostAlloc(&h->pinned, sizeof(float4) * (total > 0 ? total : 1), cudaHostAllocDefault));
    h->pinnedCap = 4 * (total > 0 ? total : 1);
    CK(cudaMalloc(&h->asyncDev, sizeof(float4) * (total > 0 ? total : 1)));
    h->asyncDevCap = total > 0 ? total : 1;
  }
  if (!h->copyStream) {
    CK(cudaStreamCreateWithFlags(&h->copyStream, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->evGathered, cudaEventDisableTiming));
  }
  if (!rects.empty()) {
    // the snapshot is taken in stream order; its copy to the host runs on the
    // copy stream, so the steps queued after it do not wait for the copy
    int rc = rn_gather_rects(rects.data(), int(rects.size()), h->asyncDev, h->stream);
    if (rc != RN_OK) return rc;
    h->launches++;
    CK(cudaEventRecord(h->evGathered, h->stream));
    CK(cudaStreamWaitEvent(h->copyStream, h->evGathered, 0));
    CK(cudaMemcpyAsync(h->pinned, h->asyncDev, sizeof(float4) * total, cudaMemcpyDeviceToHost, h->copyStream));
  } else {
    CK(cudaEventRecord(h->evGathered, h->stream));
    CK(cudaStreamWaitEvent(h->copyStream, h->evGathered, 0));
  }
  CK(cudaEventRecord(h->asyncEv, h->copyStream));
  h->asyncBusy = true;
  h->asyncTag = tag;
  h->asyncFloats = 4 * total;
  return RN_OK;
}

int rn_poll_async(rn_handle h, int* tag, float* out, size_t cap_floats) {
  if (!valid(h)) return fail(RN_ERR_ARG, "rn_poll_async: bad handle");
  if (!h->asyncBusy) return fail(RN_ERR_STATE, "rn_poll_async: no read in flight");
  cudaError_t e = cudaEventQuery(h->asyncEv);
  if (e == cudaErrorNotReady) return RN_NOT_READY;
  if (e != cudaSuccess) return cuda_fail(e, "cudaEventQuery");
  if (cap_floats < h->asyncFloats) return fail(RN_ERR_ARG, "rn_poll_async: output buffer too small");
  if (out && h->asyncFloats) std::memcpy(out, h->pinned, sizeof(float) * h->asyncFloats);
  if (tag) *tag = h->asyncTag;
  h->asyncBusy = false;
  return RN_OK;
}

int rn_cancel_async(rn_handle h) {
  if (!h) return RN_OK;
  if (h->asyncBusy) cudaEventSynchronize(h->asyncEv);
  h->asyncBusy = false;
  return RN_OK;
}

int rn_spray_set_injector(rn_handle h, const float* tab) {
  if (!valid(h) || !tab) return fail(RN_ERR_ARG, "rn_spray_set_injector: bad argument");
  CK(cudaMemcpyAsync(h->tab, tab, sizeof(float4) * 768, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_spray_set_parcels(rn_handle h, const float* PA, const float* PB, int head) {
  if (!valid(h) || !PA || !PB) return fail(RN_ERR_ARG, "rn_spray_set_parcels: bad argument");
  CK(cudaMemcpyAsync(h->PA[h->scur], PA, sizeof(float4) * SPRAY_N, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->PB[h->scur], PB, sizeof(float4) * SPRAY_N, cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(h->PC[h->scur], 0, sizeof(float4) * SPRAY_N, h->stream));
  // the deposit bounds of the loaded ring: its largest live mass and speed
  float mMax = 0.0f, vMax = 0.0f;
  for (int k = 0; k < SPRAY_N; k++) {
    const float m = PB[4 * k + 1];
    if (!(m > 0.0f)) continue;
    const float v = std::sqrt(PA[4 * k + 2] * PA[4 * k + 2] + PA[4 * k + 3] * PA[4 * k + 3]);
    if (m < 3.0e38f) mMax = std::max(mMax, m);
    if (v < 3.0e38f) vMax = std::max(vMax, v);
  }
  unsigned hb[4];
  std::memcpy(&hb[0], &mMax, 4);
  std::memcpy(&hb[1], &vMax, 4);
  hb[2] = hb[0];
  hb[3] = hb[1];
  CK(cudaMemcpyAsync(h->depBound, hb, sizeof(hb), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemsetAsync(h->liveSteps, 0, sizeof(unsigned long long), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->head = uint32_t(((head % SPRAY_N) + SPRAY_N) % SPRAY_N);
  return RN_OK;
}

int rn_spray_reset(rn_handle h) {
  if (!valid(h)) return fail(RN_ERR_ARG, "rn_spray_reset: bad handle");
  return spray_reset_dev(h);
}

int rn_spray_parcel_steps(rn_handle h, long long* out) {
  if (!valid(h) || !out) return fail(RN_ERR_ARG, "rn_spray_parcel_steps: bad argument");
  unsigned long long v = 0;
  CK(cudaMemcpyAsync(&v, h->liveSteps, sizeof(v), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  *out = (long long)v;
  return RN_OK;
}

int rn_spray_stats(rn_handle h, double out[4]) {
  if (!valid(h) || !out) return fail(RN_ERR_ARG, "rn_spray_stats: bad argument");
  std::vector<float4> b(SPRAY_N);
  CK(cudaMemcpyAsync(b.data(), h->PB[h->scur], sizeof(float4) * SPRAY_N, cudaMemcpyDeviceToHost, h->stream));
  unsigned flag = 0;
  CK(cudaMemcpyAsync(&flag, h->depFlag, sizeof(unsigned), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (flag) {
    CK(cudaMemsetAsync(h->depFlag, 0, sizeof(unsigned), h->stream));
    return fail(RN_ERR_STATE, "rn_spray_stats: a spray deposit left the fixed-point range of the fast "
                              "precision (a non-finite parcel); the deposits were clamped");
  }
  double f = 0, o = 0, dS = 0;
  long long n = 0;
  for (int k = 0; k < SPRAY_N; k++) {
    double m = b[k].y;
    if (m > 0) {
      n++;
      dS += b[k].x;
      if (b[k].z < 0.5f) f += m; else o += m;
    }
  }
  out[0] = f; out[1] = o; out[2] = double(n); out[3] = n ? dS / double(n) : 0.0;
  return RN_OK;
}

int rn_integrals(rn_handle h, const rn_integral_spec* spec, rn_integrals_out* out) {
  if (!valid(h) || !spec || !out) return fail(RN_ERR_ARG, "rn_integrals: bad argument");
  if (spec->iExit < 0 || spec->iExit + 1 > h->Nx || spec->jExit < 0 || spec->jExit > h->Nr || spec->iThroat < 0 ||
      spec->iThroat >= h->Nx || spec->iChamber < 0 || spec->iChamber >= h->Nx)
    return fail(RN_ERR_ARG, "rn_integrals: column index out of range");
  h->K->integrals(h->grid(), h->SA[h->cur], h->SB[h->cur], h->geoA, *spec, h->stepTex + h->stepIdx, h->dInt,
                   h->stream);
  h->launches++;
  double r[12];
  CK(cudaMemcpyAsync(r, h->dInt, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  out->F = r[0]; out->mdot = r[1]; out->Mw = r[2]; out->pw = r[3]; out->A = r[4];
  out->throat_mdot = r[5]; out->throat_mO = r[6]; out->throat_mF = r[7];
  out->chamber_p = r[8]; out->chamber_T = r[9]; out->dt = r[10]; out->t = r[11];
  return RN_OK;
}

int rn_sync(rn_handle h) {
  if (!h) return fail(RN_ERR_ARG, "rn_sync: NULL handle");
  CK(cudaStreamSynchronize(h->stream));
  if (h->errFlag) {
    unsigned e = 0;
    CK(cudaMemcpy(&e, h->errFlag, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (e) {
      CK(cudaMemset(h->errFlag, 0, sizeof(unsigned)));
      return fail(RN_ERR_CUDA, "rn_sync: a stage kernel's halo copy did not complete; the step's results are invalid");
    }
  }
  if (h->depFlag) {
    unsigned e = 0;
    CK(cudaMemcpy(&e, h->depFlag, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (e) {
      CK(cudaMemset(h->depFlag, 0, sizeof(unsigned)));
      return fail(RN_ERR_STATE, "rn_sync: a spray deposit left the fixed-point range of the fast precision (a "
                                "non-finite parcel); the deposits were clamped");
    }
  }
  return RN_OK;
}

int rn_wait(rn_handle h, int timeout_ms) {
  if (!h) return fail(RN_ERR_ARG, "rn_wait: NULL handle");
  auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(h->stream);
    if (e == cudaSuccess) return RN_OK;
    if (e != cudaErrorNotReady) return cuda_fail(e, "cudaStreamQuery");
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if (ms >= timeout_ms) return RN_NOT_READY;
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

int rn_set_precision(rn_handle h, int mode) {
  if (!h || (mode != RN_PRECISION_FAST && mode != RN_PRECISION_EXACT))
    return fail(RN_ERR_ARG, "rn_set_precision: bad handle or mode");
  h->K = mode == RN_PRECISION_EXACT ? &kernels_exact : &kernels_fast;
  return RN_OK;
}

int rn_set_tile(rn_handle h, int shape) {
  if (!valid(h) || shape < 0 || shape >= NTILES) return fail(RN_ERR_ARG, "rn_set_tile: bad handle or shape");
  if (h->batch) return fail(RN_ERR_STATE, "rn_set_tile: the handle is in a batch");
  if (shape == h->tile) return RN_OK;
  const int old = h->tile;
  h->tile = shape;
  int rc = rn_build_member_lists(h);
  if (rc != RN_OK) {
    std::string msg = g_err;
    h->tile = old;
    rn_build_member_lists(h);
    return fail(rc, msg);
  }
  return RN_OK;
}

int rn_get_tile(rn_handle h, int* shape) {
  if (!h || !shape) return fail(RN_ERR_ARG, "rn_get_tile: bad argument");
  *shape = h->tile;
  return RN_OK;
}

int rn_autotune(rn_handle h, const rn_params* P, int steps, int* chosen) {
  if (!valid(h) || !P || steps < 1) return fail(RN_ERR_ARG, "rn_autotune: bad argument");
  if (h->batch) return fail(RN_ERR_STATE, "rn_autotune: the handle is in a batch");
  // save everything a step changes
  const size_t N = size_t(h->Nx) * h->Nr;
  const size_t stateBytes = sizeof(float4) * N * 6, sprayBytes = sizeof(float4) * SPRAY_N * 6;
  char* save = nullptr;
  CK(cudaMalloc(&save, stateBytes + sprayBytes + sizeof(float4) * 2 + sizeof(unsigned) * 6));
  auto copy_all = [&](bool toSave) -> cudaError_t {
    char* p = save;
    cudaError_t e;
    const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
    e = toSave ? cudaMemcpyAsync(p, h->SA[0], stateBytes, k, h->stream) : cudaMemcpyAsync(h->SA[0], p, stateBytes, k, h->stream);
    if (e != cudaSuccess) return e;
    p += stateBytes;
    e = toSave ? cudaMemcpyAsync(p, h->PA[0], sprayBytes, k, h->stream) : cudaMemcpyAsync(h->PA[0], p, sprayBytes, k, h->stream);
    if (e != cudaSuccess) return e;
    p += sprayBytes;
    e = toSave ? cudaMemcpyAsync(p, h->stepTex, sizeof(float4) * 2, k, h->stream)
               : cudaMemcpyAsync(h->stepTex, p, sizeof(float4) * 2, k, h->stream);
    if (e != cudaSuccess) return e;
    p += sizeof(float4) * 2;
    e = toSave ? cudaMemcpyAsync(p, h->depBound, sizeof(unsigned) * 4, k, h->stream)
               : cudaMemcpyAsync(h->depBound, p, sizeof(unsigned) * 4, k, h->stream);
    if (e != cudaSuccess) return e;
    p += sizeof(unsigned) * 4;
    return toSave ? cudaMemcpyAsync(p, h->wmax, sizeof(unsigned) * 2, k, h->stream)
                  : cudaMemcpyAsync(h->wmax, p, sizeof(unsigned) * 2, k, h->stream);
  };
  const int cur = h->cur, stepIdx = h->stepIdx, wslot = h->wslot, scur = h->scur;
  const bool wvalid = h->wvalid;
  const long long stepCount = h->stepCount, launches = h->launches;
  const uint32_t head = h->head, seed = h->seed;
  const int prof = h->prof;
  h->prof = 0;
  cudaError_t e = copy_all(true);
  int best = h->tile, rc = RN_OK;
  float bestMs = 1e30f;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  for (int shape = 0; shape < NTILES && e == cudaSuccess && rc == RN_OK; shape++) {
    h->tile = shape;
    rc = rn_build_member_lists(h);
    if (rc != RN_OK) { rc = RN_OK; continue; }          // this shape cannot hold the geometry's lists
    rc = rn_step(h, 2, P);                                // warm-up
    if (rc == RN_OK) e = cudaEventRecord(e0, h->stream);
    if (rc == RN_OK && e == cudaSuccess) rc = rn_step(h, steps, P);
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventRecord(e1, h->stream);
    float ms = 0.0f;
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (rc == RN_OK && e == cudaSuccess && ms < bestMs) { bestMs = ms; best = shape; }
    // restore the state the trial advanced
    if (e == cudaSuccess) e = copy_all(false);
    h->cur = cur; h->stepIdx = stepIdx; h->wslot = wslot; h->scur = scur; h->wvalid = wvalid;
    h->stepCount = stepCount; h->head = head; h->seed = seed;
    // the spray's deposit sums start each step at zero whatever parity it has
    if (e == cudaSuccess)
      e = cudaMemsetAsync(h->acc, 0, sizeof(unsigned long long) * 8 * size_t(h->Nx) * h->Nr, h->stream);
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(h->stream);
  cudaFree(save);
  h->launches = launches;
  h->prof = prof;
  h->tile = best;
  int rc2 = rn_build_member_lists(h);
  if (e != cudaSuccess) return cuda_fail(e, "rn_autotune");
  if (rc != RN_OK) return rc;
  if (rc2 != RN_OK) return rc2;
  if (chosen) *chosen = best;
  return RN_OK;
}

int rn_get_precision(rn_handle h, int* mode) {
  if (!h || !mode) return fail(RN_ERR_ARG, "rn_get_precision: bad argument");
  *mode = h->K == &kernels_exact ? RN_PRECISION_EXACT : RN_PRECISION_FAST;
  return RN_OK;
}

int rn_get_stream(rn_handle h, void** stream) {
  if (!h || !stream) return fail(RN_ERR_ARG, "rn_get_stream: bad argument");
  *stream = (void*)h->stream;
  return RN_OK;
}

int rn_profile(rn_handle h, int enable) {
  if (!h || enable < 0 || enable > 2) return fail(RN_ERR_ARG, "rn_profile: bad argument");
  h->prof = enable;
  return RN_OK;
}

int rn_profile_read(rn_handle h, double ms[RN_NKERNELS], long long launches[RN_NKERNELS]) {
  if (!h || !ms || !launches) return fail(RN_ERR_ARG, "rn_profile_read: bad argument");
  CK(cudaStreamSynchronize(h->stream));
  for (auto& p : h->evPending) {
    float t = 0.0f;
    CK(cudaEventElapsedTime(&t, p.second.first, p.second.second));
    h->profMs[p.first] += t;
    h->profN[p.first] += 1;
    h->evPool.push_back(p.second.first);
    h->evPool.push_back(p.second.second);
  }
  h->evPending.clear();
  for (int k = 0; k < RN_NKERNELS; k++) {
    ms[k] = h->profMs[k];
    launches[k] = h->profN[k];
    h->profMs[k] = 0.0;
    h->profN[k] = 0;
  }
  return RN_OK;
}

int rn_kernel_launches(rn_handle h, long long* out) {
  if (!h || !out) return fail(RN_ERR_ARG, "rn_kernel_launches: bad argument");
  *out = h->launches;
  return RN_OK;
}

}  // extern "C"
