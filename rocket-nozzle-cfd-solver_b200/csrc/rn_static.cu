// rn_static.cu -- FP64 read-out integrals for callers that cannot allocate.
//
// rn_integrals() stages its sums in device memory that the solver handle
// allocated with cudaMalloc. Some callers cannot allocate device memory at the
// moment they need a read-out: a host application that reserves the whole
// device memory budget for its solver instances up front and forbids further
// allocation (allocating later could fail or fragment the reservation), or a
// latency-critical control loop in which cudaMalloc/cudaFree would stall it
// with their implicit synchronisation. rn_integrals_static() computes the
// same read-outs from buffers the caller already owns and keeps its scratch in
// a file-scope __device__ array instead: the per-row terms of up to
// RN_STATIC_MAX_ROWS rows (8 x 4096 doubles = 256 KiB) plus the 12 results.
// Every GPU that loads the library holds this array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents. The kernel writes every slot before it reads it, so nothing needs
// clearing between calls; two calls that overlap on the GPU (on different
// streams, or from different host threads) race on the array.
//
// Host code never dereferences the array's name: on the host it is only a
// stand-in for the symbol. The device address is fetched once per device with
// cudaGetSymbolAddress (with that device current) by the first call made on
// it; make that first call before any stream capture begins on the device.
// The cached address belongs to the module loaded in the device's context: a
// host that calls cudaDeviceReset must not call rn_integrals_static again in
// the same process (the module is reloaded and the old address is stale).
// A call is refused (RN_ERR_ARG) while its stream is being captured, since it
// ends with a blocking read-back.
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "rn.h"

namespace {

constexpr int TERMS = 8;                                    // F, mdot, Mw, pw, A, throat mdot, mO, mF
constexpr int RESULTS = 12;
static __device__ __align__(256) double g_static_scratch[TERMS * RN_STATIC_MAX_ROWS + 16];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
double* g_scratch_ptr[MAX_DEVICES] = {nullptr};

}  // namespace

// records the message rn_last_error() returns (defined with the other entry points)
int rn_record_error(int code, const std::string& msg);

namespace {

int static_fail(int code, const std::string& msg) { return rn_record_error(code, msg); }

struct Neu {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
};

// One block of 256 threads. Phase 1: each row's terms into the scratch rows.
// Phase 2: warp w sums term w over its rows (lane-strided Neumaier sums, then
// the 32 partial pairs in lane order), deterministic for given inputs.
__global__ void __launch_bounds__(256) k_integrals_static(double* scratch, const float4* __restrict__ A,
                                                          const float4* __restrict__ B,
                                                          const float4* __restrict__ geoA,
                                                          const uint8_t* __restrict__ mask, int Nx, int Nr,
                                                          const float4* __restrict__ st, rn_integral_spec sp) {
  __shared__ int jstop;
  __shared__ double ps[TERMS][32], pc[TERMS][32];
  double* rows = scratch;
  double* res = scratch + TERMS * RN_STATIC_MAX_ROWS;
  const int tid = threadIdx.x, W1 = Nx + 1;
  const double PI = 3.14159265358979323846;
  if (tid == 0) jstop = Nr;
  __syncthreads();
  for (int j = tid; j < Nr; j += blockDim.x)          // throat plane ends at its first solid cell
    if (mask[j * Nx + sp.iThroat]) atomicMin(&jstop, j);
  for (int j = tid; j < sp.jExit; j += blockDim.x) {  // exit plane (exitPerformance)
    const int k = j * Nx + sp.iExit;
    float4 a = A[k], b = B[k];
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho, v = (double)a.z / rho;
    double G = (double)b.z, gam = 1.0 + 1.0 / G;
    double p = fmax(((double)a.w - 0.5 * rho * (u * u + v * v)) / G, 1e-9);
    double dA = 2.0 * PI * fabs((double)geoA[j * W1 + sp.iExit + 1].z) * sp.dx * sp.dx;
    double c = sqrt(gam * p / rho);
    double mm = (double)b.x * u * dA;
    rows[0 * RN_STATIC_MAX_ROWS + j] = (rho * u * u + p - sp.pAmb) * dA;
    rows[1 * RN_STATIC_MAX_ROWS + j] = mm;
    rows[2 * RN_STATIC_MAX_ROWS + j] = mm * sqrt(u * u + v * v) / c;
    rows[3 * RN_STATIC_MAX_ROWS + j] = p * dA;
    rows[4 * RN_STATIC_MAX_ROWS + j] = dA;
  }
  __syncthreads();
  const int nthroat = jstop;
  for (int j = tid; j < nthroat; j += blockDim.x) {   // throat plane (chamberPerformance)
    const int k = j * Nx + sp.iThroat;
    float4 a = A[k], b = B[k];
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho;
    double dA = 2.0 * PI * fabs((double)geoA[j * W1 + sp.iThroat].z) * sp.dx * sp.dx;
    rows[5 * RN_STATIC_MAX_ROWS + j] = rho * u * dA;
    rows[6 * RN_STATIC_MAX_ROWS + j] = (double)b.w * u * dA;
    rows[7 * RN_STATIC_MAX_ROWS + j] = (double)b.y * u * dA;
  }
  __syncthreads();
  const int w = tid >> 5, lane = tid & 31;
  if (w < TERMS) {
    const int n = w < 5 ? sp.jExit : nthroat;
    Neu acc;
    for (int j = lane; j < n; j += 32) acc.add(rows[w * RN_STATIC_MAX_ROWS + j]);
    ps[w][lane] = acc.s;
    pc[w][lane] = acc.c;
    __syncwarp();
    if (lane == 0) {
      Neu t;
      for (int l = 0; l < 32; l++) { t.add(ps[w][l]); t.add(pc[w][l]); }
      res[w] = t.s + t.c;
    }
  }
  if (tid == 0) {                                      // chamber probe (cellPrimSI) and step info
    const int kc = sp.iChamber;
    float4 a = A[kc], b = B[kc];
    double G = (double)b.z;
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho, v = (double)a.z / rho;
    double p = fmax(((double)a.w - 0.5 * rho * (u * u + v * v)) / G, 1e-9);
    double Y = fmin(fmax((double)b.x / rho, 0.0), 1.0);
    double Fv = fmax((double)b.y / rho, 0.0), Ov = sp.inj ? fmax((double)b.w / rho, 0.0) : 0.0;
    double Rm = (1.0 - Y) * sp.RaN + Fv * sp.Rs[0] + Ov * sp.Rs[1] + fmax(Y - Fv - Ov, 0.0) * sp.Rs[2];
    res[8] = p;
    res[9] = p / (rho * Rm);
    float4 s = *st;
    res[10] = (double)s.x;
    res[11] = (double)s.z;
  }
}

// The array's device address on the current device, fetched on first use.
int scratch_for_current_device(double** out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return static_fail(RN_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES) return static_fail(RN_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      return static_fail(RN_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return RN_OK;
}

}  // namespace

extern "C" {

int rn_integrals_static(const float* A, const float* B, const float* geoA, const uint8_t* mask, int Nx, int Nr,
                        const float* stepinfo, const rn_integral_spec* spec, rn_integrals_out* out, void* stream) {
  if (!A || !B || !geoA || !mask || !stepinfo || !spec || !out || Nx < 1 || Nr < 1)
    return static_fail(RN_ERR_ARG, "rn_integrals_static: bad argument");
  if (spec->jExit < 0 || spec->jExit > Nr || spec->iExit < 0 || spec->iExit + 1 > Nx || spec->iThroat < 0 ||
      spec->iThroat >= Nx || spec->iChamber < 0 || spec->iChamber >= Nx)
    return static_fail(RN_ERR_ARG, "rn_integrals_static: column index out of range");
  if (Nr > RN_STATIC_MAX_ROWS)
    return static_fail(RN_ERR_ARG, "rn_integrals_static: " + std::to_string(Nr) + " rows exceed the static scratch (" +
                                       std::to_string(RN_STATIC_MAX_ROWS) + " rows); use rn_integrals");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The call ends with a blocking read-back, which a capturing stream cannot
  // take: refuse before anything is queued, so the caller's capture stays valid.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return static_fail(RN_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return static_fail(RN_ERR_ARG, "rn_integrals_static: the stream is being captured; call it outside a capture");
  // An error left by the caller's own earlier work is reported as such, and
  // nothing is launched after it.
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return static_fail(RN_ERR_CUDA, std::string("rn_integrals_static: earlier CUDA error pending: ") +
                                        cudaGetErrorString(e));
  double* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != RN_OK) return rc;
  k_integrals_static<<<1, 256, 0, s>>>(scratch, reinterpret_cast<const float4*>(A), reinterpret_cast<const float4*>(B),
                                       reinterpret_cast<const float4*>(geoA), mask, Nx, Nr,
                                       reinterpret_cast<const float4*>(stepinfo), *spec);
  e = cudaGetLastError();
  if (e != cudaSuccess) return static_fail(RN_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  double r[RESULTS];
  e = cudaMemcpyAsync(r, scratch + TERMS * RN_STATIC_MAX_ROWS, sizeof(r), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return static_fail(RN_ERR_CUDA, std::string("read-back: ") + cudaGetErrorString(e));
  out->F = r[0]; out->mdot = r[1]; out->Mw = r[2]; out->pw = r[3]; out->A = r[4];
  out->throat_mdot = r[5]; out->throat_mO = r[6]; out->throat_mF = r[7];
  out->chamber_p = r[8]; out->chamber_T = r[9]; out->dt = r[10]; out->t = r[11];
  return RN_OK;
}

}  // extern "C"
