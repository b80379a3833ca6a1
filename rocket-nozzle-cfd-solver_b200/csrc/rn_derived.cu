// rn_derived.cu -- derived display fields into a headless device buffer
// (FS_DERIVED, render.js:60-134), declared in rn.h.
//
// The reference renders its fields through a fragment shader into an RGBA32F
// texture that only its display pass reads. Here the same per-cell arithmetic
// writes an Nx x Nr float4 buffer in HBM, (t, Z, normalised T, Mach) per cell,
// which a caller reads back or hands to its own kernels; no graphics API is
// involved. Fields 9 (eddy / laminar viscosity) and 13 (burning rate) read the
// split step's cell data T2 (FS_VCELL, solver.js:458-488); the step kernels
// keep T2 on chip, so this kernel recomputes it from the last step's stage-1
// state at t_new, the inputs the split step used.
#include <cuda_runtime.h>
#include <math.h>
#include <cstring>
#include <string>
#include "rn.h"
#include "rn_internal.h"

namespace {

using rn::Grid;
using rn::Prim;

// P(ivec2 c): clamped to the grid (render.js:73-77)
__device__ Prim prim_at(const Grid& g, const float4* __restrict__ A, const float4* __restrict__ B, int i, int j) {
  i = min(max(i, 0), g.Nx - 1);
  j = min(max(j, 0), g.Nr - 1);
  return rn::to_prim(A[j * g.Nx + i], B[j * g.Nx + i]);
}
// lrho(ivec2 c): log density, mirrored across the axis (render.js:78-82)
__device__ float lrho(const Grid& g, const float4* __restrict__ A, int i, int j) {
  int ci = min(max(i, 0), g.Nx - 1), cj = min(max(j, 0), g.Nr - 1);
  if (j < 0) cj = -j - 1;
  return logf(fmaxf(A[cj * g.Nx + ci].x, 1e-7f));
}
__device__ bool solid_c(const Grid& g, int i, int j) {
  i = min(max(i, 0), g.Nx - 1);
  j = min(max(j, 0), g.Nr - 1);
  return g.mask[j * g.Nx + i] != 0;
}

// T2 of cell (i, j): FS_VCELL on the ghost primitives of the stage-1 state A1/B1 at t
__device__ float4 t2_at(const Grid& g, const float4* __restrict__ A1, const float4* __restrict__ B1, int i, int j,
                        float t, float dt, const rn_params& P) {
  float4 w0, s0, wE, sE, wW, sW, wN, sN, wS, sS;
  rn::ghost_prim(g, A1, B1, i, j, t, P, w0, s0);
  rn::ghost_prim(g, A1, B1, i + 1, j, t, P, wE, sE);
  rn::ghost_prim(g, A1, B1, i - 1, j, t, P, wW, sW);
  rn::ghost_prim(g, A1, B1, i, j + 1, t, P, wN, sN);
  rn::ghost_prim(g, A1, B1, i, j - 1, t, P, wS, sS);
  float4 T1, T2;
  rn::vcell(w0, s0, wE, wW, wN, wS, i, j, g.geoM[j * g.Nx + i].w, dt, P, T1, T2);
  return T2;
}

__global__ void k_derived(Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                          const float4* __restrict__ A1, const float4* __restrict__ B1, const float4* st,
                          rn_derived_spec sp, rn_params P, int haveT2, float4* __restrict__ out) {
  const int i = blockIdx.x * 16 + threadIdx.x, j = blockIdx.y * 16 + threadIdx.y;
  if (i >= g.Nx || j >= g.Nr) return;
  const int k = j * g.Nx + i;
  if (g.mask[k]) {
    out[k] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    return;
  }
  const int F = sp.field;
  const Prim q = prim_at(g, A, B, i, j);
  const float rho = q.w.x, p = q.w.w;
  const float c = rn::sound_speed(q);
  const float spd = rn::len2(q.w.y, q.w.z);
  const float M = spd / c;
  const float Rm = (1.0f - q.s.x) * sp.RaN + q.s.y * sp.Rs[0] + q.s.w * sp.Rs[1] +
                   fmaxf(q.s.x - q.s.y - q.s.w, 0.0f) * sp.Rs[2];
  const float T = p / (rho * Rm) * sp.Tscale[0];
  float v = 0.0f;
  float4 m = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if ((F == 9 || F == 13) && haveT2) m = t2_at(g, A1, B1, i, j, st->z, st->x, P);
  if (F == 0) v = T;
  else if (F == 1) v = M;
  else if (F == 2) {
    // numerical schlieren: |grad ln rho|, ignoring wall neighbours
    const float l0 = lrho(g, A, i, j);
    const float le = solid_c(g, i + 1, j) ? l0 : lrho(g, A, i + 1, j);
    const float lw = solid_c(g, i - 1, j) ? l0 : lrho(g, A, i - 1, j);
    const float ln = solid_c(g, i, j + 1) ? l0 : lrho(g, A, i, j + 1);
    const float ls = (j > 0 && g.mask[(j - 1) * g.Nx + i]) ? l0 : lrho(g, A, i, j - 1);
    const float gr = rn::len2(le - lw, ln - ls) * 0.5f;
    v = 1.0f - expf(-sp.schlGain * gr);
  } else if (F == 3) v = logf(p * 101325.0f) / logf(10.0f);
  else if (F == 4) v = logf(rho * 1.225f) / logf(10.0f);
  else if (F == 5) v = spd * sp.velScale;
  else if (F == 6) {
    const Prim e = prim_at(g, A, B, i + 1, j), w = prim_at(g, A, B, i - 1, j), n = prim_at(g, A, B, i, j + 1);
    float sy = q.w.y;
    if (j > 0) sy = prim_at(g, A, B, i, j - 1).w.y;
    const float om = 0.5f * (e.w.z - w.w.z) - 0.5f * (n.w.y - sy);
    v = fabsf(om) * sp.velScale / sp.dx;
  } else if (F == 7) v = q.s.x;
  else if (F == 9) v = m.w > 0.0f ? logf(fmaxf(m.x / m.w, 1.0f)) / logf(10.0f) : 0.0f;
  else if (F == 10) v = q.s.x > 0.003f ? (q.s.x - q.s.y) / q.s.x : 0.0f;
  else if (F == 11) v = q.s.y;
  else if (F == 12) v = q.s.w;
  else if (F == 13) {
    // burning rate per unit mass on a log scale, same model as the solver
    const float avail = fminf(q.s.y, (q.s.w + 0.233f * fmaxf(1.0f - q.s.x, 0.0f)) / sp.chemV[1]);
    const float kin = sp.chemV[2] * p * expf(-9000.0f / fmaxf(T, 200.0f));
    v = logf(1.0f + 1e5f * avail * fminf(fmaxf(m.z, 4.0f * m.x / rho), kin)) / logf(10.0f);
  } else v = T;
  float t = (v - sp.range[0]) / (sp.range[1] - sp.range[0]);
  if (F == 2) t = v;
  if (F == 6) t = logf(1.0f + 20.0f * fmaxf(v, 0.0f) / sp.range[1]) / logf(21.0f);
  out[k] = make_float4(t, q.s.x, (T - sp.Tscale[2]) / fmaxf(sp.Tscale[1] - sp.Tscale[2], 1.0f), M);
}

}  // namespace

extern "C" {

int rn_derived(rn_handle h, const rn_derived_spec* spec, const rn_params* P, float* out) {
  if (!h || !h->SA[0] || !spec) return rn_record_error(RN_ERR_ARG, "rn_derived: bad argument");
  if (spec->field < 0 || spec->field > 13) return rn_record_error(RN_ERR_ARG, "rn_derived: unknown field");
  const bool needT2 = spec->field == 9 || spec->field == 13;
  if (needT2 && !P) return rn_record_error(RN_ERR_ARG, "rn_derived: fields 9 and 13 need the parameter block");
  const size_t N = size_t(h->Nx) * h->Nr;
  if (!h->derived) RN_CK(cudaMalloc(&h->derived, sizeof(float4) * N));
  rn_params Pz;
  if (P) Pz = *P;
  else std::memset(&Pz, 0, sizeof(Pz));
  const int haveT2 = needT2 && h->s1last >= 0;
  const int s1 = h->s1last >= 0 ? h->s1last : h->cur;
  dim3 grid((h->Nx + 15) / 16, (h->Nr + 15) / 16), block(16, 16);
  k_derived<<<grid, block, 0, h->stream>>>(h->grid(), h->SA[h->cur], h->SB[h->cur], h->SA[s1], h->SB[s1],
                                           h->stepTex + h->stepIdx, *spec, Pz, haveT2, h->derived);
  h->launches++;
  RN_CK(cudaGetLastError());
  if (out) {
    RN_CK(cudaMemcpyAsync(out, h->derived, sizeof(float4) * N, cudaMemcpyDeviceToHost, h->stream));
    RN_CK(cudaStreamSynchronize(h->stream));
  }
  return RN_OK;
}

int rn_derived_buffer(rn_handle h, void** dev) {
  if (!h || !dev) return rn_record_error(RN_ERR_ARG, "rn_derived_buffer: bad argument");
  *dev = h->derived;
  return RN_OK;
}

}  // extern "C"

// --------------------------------------------------------------------------
// Injector table on the device (buildInjectorTable's fill, simsetup.js:181-237):
// the spray elements (a handful, from the injector layout) are weighted into
// the 256-row table by largest remainder, in one thread: the remainders are
// ranked by a stable descending order, as Array.prototype.sort does, and the
// rows are written in element order. Arithmetic in doubles, rows stored as
// float32 like the reference's Float32Array.
namespace {

__global__ void k_injector_table(const rn_injector_element* el, int n, float4* tab) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  constexpr int NROW = 256;
  double total = 0.0;
  for (int e = 0; e < n; e++) total = total + el[e].weight;
  double q[RN_MAX_INJECTOR_ELEMENTS];
  int cnt[RN_MAX_INJECTOR_ELEMENTS], order[RN_MAX_INJECTOR_ELEMENTS];
  int used = 0;
  for (int e = 0; e < n; e++) {
    q[e] = el[e].weight / total * NROW;
    cnt[e] = int(floor(q[e]));
    used += cnt[e];
    order[e] = e;
  }
  // stable insertion sort by descending remainder
  for (int a = 1; a < n; a++) {
    const int v = order[a];
    const double rv = -(q[v] - cnt[v]);
    int b = a - 1;
    while (b >= 0 && -(q[order[b]] - cnt[order[b]]) > rv) {
      order[b + 1] = order[b];
      b--;
    }
    order[b + 1] = v;
  }
  for (int a = 0; a < n && used < NROW; a++) {
    cnt[order[a]]++;
    used++;
  }
  int t = 0;
  for (int e = 0; e < n; e++)
    for (int r = 0; r < cnt[e] && t < NROW; r++, t++) {
      const rn_injector_element& x = el[e];
      tab[t] = make_float4(float(x.x), float(x.r), float(x.angle), float(x.speed));
      tab[NROW + t] = make_float4(float(x.type), float(x.drop), float(x.cone), float(x.width));
      tab[2 * NROW + t] = make_float4(float(x.xi), 0.0f, 0.0f, 0.0f);
    }
  for (; t < NROW; t++) {
    tab[t] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    tab[NROW + t] = tab[t];
    tab[2 * NROW + t] = tab[t];
  }
}

}  // namespace

extern "C" {

int rn_spray_build_injector(rn_handle h, const rn_injector_element* el, int n) {
  if (!h || !h->SA[0] || !el || n < 1 || n > RN_MAX_INJECTOR_ELEMENTS)
    return rn_record_error(RN_ERR_ARG, "rn_spray_build_injector: bad argument or element count");
  rn_injector_element* d = nullptr;
  RN_CK(cudaMalloc(&d, sizeof(rn_injector_element) * n));
  cudaError_t e = cudaMemcpyAsync(d, el, sizeof(rn_injector_element) * n, cudaMemcpyHostToDevice, h->stream);
  if (e == cudaSuccess) {
    k_injector_table<<<1, 32, 0, h->stream>>>(d, n, h->tab);
    h->launches++;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(d);
  if (e != cudaSuccess) return rn_record_cuda(e, "rn_spray_build_injector");
  return RN_OK;
}

}  // extern "C"
