// rn_readout.cu -- device read-outs of a solver handle (declared in rn.h):
// the steady-state residual and the flow-separation point.
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
#include <math.h>
#include <string>
#include <vector>
#include "rn.h"
#include "rn_internal.h"

namespace {

struct RectBatch {
  RectCopy r[RN_GATHER_RECTS];
};
// blockIdx.y = rectangle; threads stride over its w*h texels in row order.
__global__ void k_gather_rects(RectBatch b, float4* __restrict__ dst) {
  const RectCopy& r = b.r[blockIdx.y];
  const int n = r.w * r.h;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int row = k / r.w, col = k - row * r.w;
    dst[r.off + k] = r.src[size_t(r.y + row) * r.W + r.x + col];
  }
}

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

// Gathers the rectangles into dst in launches of up to RN_GATHER_RECTS.
int rn_gather_rects(const RectCopy* r, int n, float4* dst, cudaStream_t stream) {
  for (int b0 = 0; b0 < n; b0 += RN_GATHER_RECTS) {
    RectBatch b;
    const int m = n - b0 < RN_GATHER_RECTS ? n - b0 : RN_GATHER_RECTS;
    int most = 1;
    for (int k = 0; k < m; k++) {
      b.r[k] = r[b0 + k];
      if (r[b0 + k].w * r[b0 + k].h > most) most = r[b0 + k].w * r[b0 + k].h;
    }
    int blocks = (most + 255) / 256;
    if (blocks > 64) blocks = 64;
    k_gather_rects<<<dim3(blocks, m), 256, 0, stream>>>(b, dst);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return rn_record_cuda(e, "k_gather_rects");
  }
  return RN_OK;
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

// --------------------------------------------------------------------------
// Flow-separation read-out on the device (wallSeparation, simsetup.js:352-373):
// one thread walks the near-wall row upstream from the exit, building each
// row entry exactly as FS_WALLROW does (solver.js:665-674), and returns the
// separation column, its pressure ratio and Mach number in FP64. Only the
// scalars cross to the host, not the wall row.
namespace {

__device__ float4 wall_row_entry(const rn::Grid& g, const float4* __restrict__ A, const float4* __restrict__ B,
                                 const float4* __restrict__ jw, int i) {
  int cj = int(jw[i].x);
  cj = min(max(cj, 0), g.Nr - 1);
  rn::Prim q = rn::to_prim(A[cj * g.Nx + i], B[cj * g.Nx + i]);
  return make_float4(q.w.y, q.w.z, q.w.w, rn::sound_speed(q));
}

// prof: per column (slope, hypot(1, slope), R(x_i)); out: found, last, x, frac, eps, pRatio, Msep
__global__ void k_separation(rn::Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                             const float4* __restrict__ jw, const double* __restrict__ prof,
                             rn_separation_spec sp, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int i = sp.iExit, gaps = 0, last = -1;
  for (; i > sp.iThroat + 2 && gaps <= 2; i--) {
    const float4 r = wall_row_entry(g, A, B, jw, i);
    const double u = r.x, v = r.y, c = r.w;
    const double ut = (u + prof[3 * i] * v) / prof[3 * i + 1];
    if (ut < 0.0 || sqrt(u * u + v * v) < 0.6 * c) { last = i; gaps = 0; }
    else if (last >= 0 || sp.iExit - i > 2) gaps++;
  }
  for (int q = 0; q < 8; q++) out[q] = 0.0;
  out[1] = double(last);
  if (last < 0 || sp.iExit - last < 3) return;
  double pSep = INFINITY;
  int kS = last;
  for (int q = last; q >= max(sp.iThroat + 1, last - 30); q--) {
    const double p = wall_row_entry(g, A, B, jw, q).z;
    if (p < pSep) { pSep = p; kS = q; }
  }
  const float4 rs = wall_row_entry(g, A, B, jw, kS);
  const double us = rs.x, vs = rs.y;
  const double Msep = sqrt(us * us + vs * vs) / fmax(double(rs.w), 1e-6);
  out[6] = Msep;
  if (Msep < 1.05) return;
  const double x = (last + 0.5) * sp.dx, R = prof[3 * last + 2];
  out[0] = 1.0;
  out[2] = x;
  out[3] = (x - sp.xt) / (sp.xe - sp.xt);
  out[4] = (R * R) / (sp.Rt * sp.Rt);
  out[5] = pSep * sp.pRef / fmax(sp.paSi, 1e-6);
}

}  // namespace

extern "C" {

int rn_set_wall_profile(rn_handle h, const double* slope, const double* hyp, const double* radius) {
  if (!h || !h->SA[0] || !slope || !hyp || !radius) return rn_record_error(RN_ERR_ARG, "rn_set_wall_profile: bad argument");
  std::vector<double> prof(size_t(h->Nx) * 3);
  for (int i = 0; i < h->Nx; i++) {
    prof[3 * i] = slope[i];
    prof[3 * i + 1] = hyp[i];
    prof[3 * i + 2] = radius[i];
  }
  if (!h->wallProf) RN_CK(cudaMalloc(&h->wallProf, sizeof(double) * prof.size()));
  RN_CK(cudaMemcpyAsync(h->wallProf, prof.data(), sizeof(double) * prof.size(), cudaMemcpyHostToDevice, h->stream));
  RN_CK(cudaStreamSynchronize(h->stream));
  return RN_OK;
}

int rn_wall_separation(rn_handle h, const rn_separation_spec* spec, rn_separation_out* out) {
  if (!h || !h->SA[0] || !spec || !out) return rn_record_error(RN_ERR_ARG, "rn_wall_separation: bad argument");
  if (!h->wallProf) return rn_record_error(RN_ERR_STATE, "rn_wall_separation: no wall profile (rn_set_wall_profile)");
  if (spec->iExit < 0 || spec->iExit >= h->Nx || spec->iThroat < -1 || spec->iThroat >= h->Nx)
    return rn_record_error(RN_ERR_ARG, "rn_wall_separation: column out of range");
  if (!h->dRes) RN_CK(cudaMalloc(&h->dRes, sizeof(double) * (8 + RES_BLOCKS * RES_Q)));
  k_separation<<<1, 32, 0, h->stream>>>(h->grid(), h->SA[h->cur], h->SB[h->cur], h->jw, h->wallProf, *spec, h->dRes);
  h->launches++;
  RN_CK(cudaGetLastError());
  double r[8];
  RN_CK(cudaMemcpyAsync(r, h->dRes, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
  RN_CK(cudaStreamSynchronize(h->stream));
  out->found = r[0] != 0.0;
  out->last = int(r[1]);
  out->x = r[2];
  out->frac = r[3];
  out->eps = r[4];
  out->pRatio = r[5];
  out->Msep = r[6];
  return RN_OK;
}

}  // extern "C"
