// rn_internal.h -- the solver handle and helpers shared by the C-ABI sources
// (rn_api.cu, rn_batch.cu). Not part of the public interface.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <utility>
#include <vector>
#include "rn.h"
#include "rn_kernels.cuh"

// One solver instance: all of its device memory and its stream. The layout in
// HBM is the reference's texture layout as plain arrays (see rn_api.cu).
struct rn_solver {
  int Nx = 0, Nr = 0, device = 0;
  cudaStream_t stream = nullptr;
  float4* SA[3] = {nullptr, nullptr, nullptr};
  float4* SB[3] = {nullptr, nullptr, nullptr};
  int cur = 0;
  float4 *geoA = nullptr, *geoG = nullptr, *geoM = nullptr, *jw = nullptr, *wallRow = nullptr;
  uint8_t* mask = nullptr;
  // the mask again with rows padded to 16 bytes (a tensor map's row stride
  // must be a multiple of 16 bytes), refreshed whenever the mask changes
  uint8_t* maskP = nullptr;
  int maskPitch = 0;
  // tensor maps of the stage kernels' halo copies, one TileMaps per tile shape
  rn::TileMaps* dMaps = nullptr;
  unsigned* errFlag = nullptr;    // set by a stage kernel whose halo copy did not complete in time
  float4* stepTex = nullptr;      // [2]
  unsigned* wmax = nullptr;       // [2]
  unsigned* depFlag = nullptr;    // set when a fast deposit left the fixed-point range
  unsigned* depBound = nullptr;   // [2 step parities] x (largest parcel mass, speed) of the ring, float bits
  unsigned long long* liveSteps = nullptr;   // live parcels summed over the spray steps since the ring was set
  int stepIdx = 0, wslot = 0;
  bool wvalid = false;
  long long stepCount = 0, launches = 0;
  // spray
  float4 *PA[2] = {nullptr, nullptr}, *PB[2] = {nullptr, nullptr}, *PC[2] = {nullptr, nullptr};
  float4 *src = nullptr, *tab = nullptr, *dep = nullptr;
  unsigned *key = nullptr, *val = nullptr, *keyS = nullptr, *valS = nullptr;
  void* sortTemp = nullptr;
  size_t sortTempBytes = 0;
  int scur = 0;
  uint32_t head = 0, seed = 1;
  // asynchronous read-back
  float* pinned = nullptr;
  size_t pinnedCap = 0, asyncFloats = 0;
  cudaEvent_t asyncEv = nullptr;
  unsigned long long* acc = nullptr;   // 2 x N x 4 fixed-point spray deposit sums (by step parity scur)
  float4* asyncDev = nullptr;      // device staging of the gathered rectangles
  size_t asyncDevCap = 0;          // float4 capacity of asyncDev
  cudaStream_t copyStream = nullptr;   // the staging buffer's copy to the host
  cudaEvent_t evGathered = nullptr;
  bool asyncBusy = false;
  int asyncTag = 0;
  double* dInt = nullptr;
  // per-kernel event timing: prof = 1 launch by launch, 2 inside replays of
  // the step graph (profCapture while that graph is captured; its event
  // pairs, read after every replay, in profGraphEv)
  int prof = 0;
  bool profCapture = false;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> profGraphEv;
  std::vector<cudaEvent_t> evPool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> evPending;
  double profMs[RN_NKERNELS] = {0};
  long long profN[RN_NKERNELS] = {0};
  // tile shape of the stage/physics kernels and, per tile, the out-of-tile
  // members of its cut-cell groups (built from host copies of the topology)
  int tile = RN_TILE_16x15;
  int* xoff = nullptr;
  int* xcell = nullptr;
  int maxX = 1;
  std::vector<int> hostXoff;
  // tiles listing more than XSMALL out-of-tile members (own fused launch)
  int* heavy = nullptr;
  int nHeavy = 0;
  int numSMs = 148;
  cudaStream_t side = nullptr;          // runs the heavy tiles' launch beside the main one
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  // the 6-step period of non-spray steps as a CUDA graph, and what it was
  // captured with (rn_step replays it only while all of that still holds)
  cudaGraphExec_t stepGraph = nullptr;
  const void* graphK = nullptr;
  int graphTile = -1, graphMaxX = -1, graphHeavy = -1, graphCur = -1, graphStepIdx = -1, graphWslot = -1;
  const void* graphBase = nullptr;
  const void* graphXoff = nullptr;
  rn_params graphP;
  long long graphLaunches = 0;
  int graphScur = -1, graphPeriod = 0;
  unsigned* dHS = nullptr;   // the spray ring's (head, seed) on the device, for graph-replayed spray steps
  bool hsOnDevice = false;   // step_once launches read and advance dHS (while capturing)
  cudaStream_t sprayStream = nullptr;   // runs the parcel step beside stage 2 + the split step
  cudaEvent_t evSprayFork = nullptr, evSprayJoin = nullptr;
  std::vector<uint8_t> hostMask;
  std::vector<float> hostGeoM;
  // kernels of the selected precision (rn_set_precision)
  const rn::KernelSet* K = &rn::kernels_fast;
  // residual snapshot (A plane + step info) and FP64 scratch (rn_readout.cu)
  float4* mark = nullptr;
  float4* markSt = nullptr;
  double* dRes = nullptr;
  // per-column wall slope, hypot(1, slope) and radius for rn_wall_separation
  double* wallProf = nullptr;
  // derived-field buffer (rn_derived) and the ring slot of the last step's
  // stage-1 state (-1 when no step has run since the state was set)
  float4* derived = nullptr;
  int s1last = -1;
  // the batch this handle is stepped by, if any (rn_batch.cu)
  struct rn_batch_t* batch = nullptr;

  rn::Grid grid() const { return rn::Grid{Nx, Nr, mask, geoA, geoG, geoM}; }
};

// (Re)encode the tensor maps of h's state ring and pitched mask (rn_api.cu).
int rn_build_tile_maps(rn_solver* h);
// Copy h->mask into its row-pitched copy (queued on h->stream).
int rn_mask_refresh(rn_solver* h);
// Record an error for rn_last_error() and return `code`.
int rn_record_error(int code, const std::string& msg);
int rn_record_cuda(cudaError_t e, const char* what);
// (Re)build the per-tile member lists of `h` for its current tile shape.
int rn_build_member_lists(rn_solver* h);
// Make h->wmax[h->wslot] the wave-speed max of the current state if it is not.
int rn_ensure_wave_speed(rn_solver* h);
// Takes h out of its batch, if any (rn_batch.cu).
void rn_batch_detach(rn_solver* h);
// Residual of the current state against the mark, into h->dRes[0..5], and the
// mark itself, queued on `stream` (rn_readout.cu); device bytes they hold.
int rn_residual_launch(rn_solver* h, cudaStream_t stream);
// One rectangle (x, y, w, h) of a W-wide float4 plane, gathered row by row to
// dst + off (rn_readout.cu). Up to RN_GATHER_RECTS per launch.
struct RectCopy {
  const float4* src;
  int W, x, y, w, h;
  long long off;
};
constexpr int RN_GATHER_RECTS = 8;
int rn_gather_rects(const RectCopy* r, int n, float4* dst, cudaStream_t stream);
int rn_residual_mark_on(rn_solver* h, cudaStream_t stream);
size_t rn_residual_bytes(int Nx, int Nr);

#define RN_CK(call)                                            \
  do {                                                         \
    cudaError_t e_ = (call);                                   \
    if (e_ != cudaSuccess) return rn_record_cuda(e_, #call);   \
  } while (0)
