// rn_readout.cu -- steady-state residual of a solver handle (declared in rn.h).
//
// No reference counterpart: the reference has no convergence measure (its
// frame loop runs until the user stops it). The residual is the RMS over fluid
// cells of dU/dt for each conserved component of A = (rho, rho u, rho v, E):
//   R_c = sqrt( sum_fluid (A_c - A_c,mark)^2 / N_fluid ) / (t - t_mark)
// evaluated in FP64 from the FP32 planes. rn_residual_mark() snapshots A and
// the step info on the device; one step later rn_residual() gives the L2 norm
// of dU/dt of that step. The sums are deterministic: fixed grid, per-thread
// Neumaier sums in a fixed cell order, a fixed shared-memory tree per block and
// an in-order sum of the block partials.
#include <cuda_runtime.h>
#include <string>
#include "rn.h"
#include "rn_internal.h"

namespace {

constexpr int RES_NT = 256;
constexpr int RES_BLOCKS = 296;   // 2 per SM
constexpr int RES_Q = 5;          // 4 components + fluid-cell count

struct Neu64 {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ double val() const { return s + c; }
};

__global__ void __launch_bounds__(RES_NT) k_residual_partial(const float4* __restrict__ A,
                                                             const float4* __restrict__ M,
                                                             const uint8_t* __restrict__ mask, int N,
                                                             double* __restrict__ part) {
  Neu64 q[4];
  double n = 0.0;
  for (int k = blockIdx.x * RES_NT + threadIdx.x; k < N; k += RES_BLOCKS * RES_NT) {
    if (mask[k]) continue;
    const float4 a = A[k], m = M[k];
    const double d0 = double(a.x) - double(m.x), d1 = double(a.y) - double(m.y);
    const double d2 = double(a.z) - double(m.z), d3 = double(a.w) - double(m.w);
    q[0].add(d0 * d0);
    q[1].add(d1 * d1);
    q[2].add(d2 * d2);
    q[3].add(d3 * d3);
    n += 1.0;
  }
  __shared__ double sh[RES_Q][RES_NT];
  for (int c = 0; c < 4; c++) sh[c][threadIdx.x] = q[c].val();
  sh[4][threadIdx.x] = n;
  __syncthreads();
  for (int w = RES_NT / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
      for (int c = 0; c < RES_Q; c++) sh[c][threadIdx.x] += sh[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x < RES_Q) part[blockIdx.x * RES_Q + threadIdx.x] = sh[threadIdx.x][0];
}

// out = (R_rho, R_rhou, R_rhov, R_E, t - t_mark, fluid cells)
__global__ void k_residual_final(const double* __restrict__ part, const float4* stNow, const float4* stMark,
                                 double* out) {
  if (threadIdx.x >= RES_Q) return;
  Neu64 s;
  for (int b = 0; b < RES_BLOCKS; b++) s.add(part[b * RES_Q + threadIdx.x]);
  const double v = s.val();
  __shared__ double tot[RES_Q];
  tot[threadIdx.x] = v;
  __syncwarp(0x1f);
  if (threadIdx.x == 0) {
    const double span = double(stNow->z) - double(stMark->z);
    const double nf = tot[4];
    for (int c = 0; c < 4; c++) out[c] = (nf > 0.0 && span > 0.0) ? sqrt(tot[c] / nf) / span : 0.0;
    out[4] = span;
    out[5] = nf;
  }
}

}  // namespace

// Queues the residual of h's current state against its mark into h->dRes[0..5]
// on `stream` (the handle's, or a batch's that is ordered after it).
int rn_residual_launch(rn_solver* h, cudaStream_t stream) {
  if (!h->mark) return rn_record_error(RN_ERR_STATE, "rn_residual: no mark (call rn_residual_mark first)");
  const int N = h->Nx * h->Nr;
  k_residual_partial<<<RES_BLOCKS, RES_NT, 0, stream>>>(h->SA[h->cur], h->mark, h->mask, N, h->dRes + 8);
  k_residual_final<<<1, 32, 0, stream>>>(h->dRes + 8, h->stepTex + h->stepIdx, h->markSt, h->dRes);
  h->launches += 2;
  RN_CK(cudaGetLastError());
  return RN_OK;
}

// Snapshot of h's current A plane and step info, queued on `stream`.
int rn_residual_mark_on(rn_solver* h, cudaStream_t stream) {
  const size_t N = size_t(h->Nx) * h->Nr;
  if (!h->mark) {
    RN_CK(cudaMalloc(&h->mark, sizeof(float4) * (N + 1)));
    h->markSt = h->mark + N;
  }
  if (!h->dRes) RN_CK(cudaMalloc(&h->dRes, sizeof(double) * (8 + RES_BLOCKS * RES_Q)));
  RN_CK(cudaMemcpyAsync(h->mark, h->SA[h->cur], sizeof(float4) * N, cudaMemcpyDeviceToDevice, stream));
  RN_CK(cudaMemcpyAsync(h->markSt, h->stepTex + h->stepIdx, sizeof(float4), cudaMemcpyDeviceToDevice, stream));
  return RN_OK;
}

size_t rn_residual_bytes(int Nx, int Nr) {
  return sizeof(float4) * (size_t(Nx) * Nr + 1) + sizeof(double) * (8 + RES_BLOCKS * RES_Q);
}

extern "C" {

int rn_residual_mark(rn_handle h) {
  if (!h || !h->SA[0]) return rn_record_error(RN_ERR_ARG, "rn_residual_mark: bad handle");
  return rn_residual_mark_on(h, h->stream);
}

int rn_residual(rn_handle h, double out[6]) {
  if (!h || !h->SA[0] || !out) return rn_record_error(RN_ERR_ARG, "rn_residual: bad argument");
  int rc = rn_residual_launch(h, h->stream);
  if (rc != RN_OK) return rc;
  RN_CK(cudaMemcpyAsync(out, h->dRes, sizeof(double) * 6, cudaMemcpyDeviceToHost, h->stream));
  RN_CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

}  // extern "C"
