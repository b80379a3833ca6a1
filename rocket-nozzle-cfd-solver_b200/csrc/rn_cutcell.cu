// rn_cutcell.cu -- the cut-cell geometry builder on the device (declared in rn.h).
//
// Restates buildCutGeometry (cutcell.js:14-186) and the geoM post-pass of
// buildSimSetup (simsetup.js:51-63) plus the near-wall row jWall, writing the
// handle's mask / geoA / geoG / geoM / jWall directly: the step that precedes
// every solve runs in a few kernels instead of an O(N x 64) host loop.
//
// Arithmetic is the JavaScript's: doubles, every value the reference keeps in a
// Float32Array rounded to float32 where it does, comparisons in the same order,
// so the topology (mask, host offsets, slave bits) and the float planes are
// bit-identical to the host builder. The inner-wall radius enters as the
// reference's Float32Array table (Rtab) for the column bounds and, at every
// sample abscissa the builder evaluates, as the host's RinAt value (the
// contour can be any host function, e.g. a cavity-modified chamber wall).
//
// Phases: column bounds; per cell maybe-cut flag, volume and meridional area
// (8x8 sub-samples where cut); per face the open area (12 sub-samples where a
// cut or maybe-cut cell touches it); classification and solid faces; the
// sliver merge (two passes in row-major order over the slivers, one thread:
// each decision depends on the earlier ones, as in the reference); solid faces
// again; first-order flags, wall vectors, group sums and slave bits; geoM's
// turbulence length and boundary-layer band; jWall.
#include <cuda_runtime.h>
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>
#include <math.h>
#include <string>
#include <vector>
#include "rn.h"
#include "rn_internal.h"

namespace {

constexpr int SUB = 8, NC = 8, NFS = 12, NS = RN_CUT_SAMPLES;
constexpr double KMERGE = 0.5;

struct CutDev {
  int Nx, Nr, cut, base, nSolids;
  double xeC, twC, xBaseC, bodyC;
  const float* Rtab;
  const double* rin;      // Nx x NS
  const double* solids;   // nSolids x 4
  float* colMin;
  float* colMax;
  uint8_t* mc;            // maybe-cut, Nx*Nr
  uint8_t* isCut;
  uint8_t* solid;
  int* host;
  float *V, *Am, *kap;    // Nx*Nr
  float *Ax, *Ar;         // (Nr+1) x (Nx+1)
};

// fluid(xc, rc) (cutcell.js:36-44); ri = RinAt(xc), read only where xc <= xeC
__device__ bool fluid(const CutDev& c, double xc, double rc, double ri) {
  for (int s = 0; s < c.nSolids; s++) {
    const double* S = c.solids + 4 * s;
    if (xc >= S[0] && xc <= S[1] && rc >= S[2] && rc <= S[3]) return false;
  }
  if (xc <= c.xeC) {
    if (rc >= ri && rc <= ri + c.twC) return false;
    if (c.base && xc < c.xBaseC && rc >= ri && rc < c.bodyC) return false;
  }
  return true;
}
__device__ double rin_at(const CutDev& c, int i, int s) { return c.rin[size_t(i) * NS + s]; }
__device__ bool ov(double a0, double a1, double b0, double b1) { return a0 < b1 && a1 > b0; }

// column range of the inner wall over [i, i+1] (cutcell.js:46-51)
__global__ void k_cols(CutDev c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.Nx) return;
  double mn = 1e9, mx = -1e9;
  bool any = false;
  for (int q = i * SUB; q <= i * SUB + SUB; q++) {
    const double v = c.Rtab[q];
    if (v > -1e8) {
      mn = any ? fmin(mn, v) : v;
      mx = any ? fmax(mx, v) : v;
      any = true;
    }
  }
  c.colMin[i] = any ? float(mn) : 1e9f;
  c.colMax[i] = any ? float(mx) : -1e9f;
}

// maybeCut, V, Am and isCut per cell (cutcell.js:52-82)
__global__ void k_cells(CutDev c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.Nx || j >= c.Nr) return;
  const int k = j * c.Nx + i;
  const double r0 = j, r1 = j + 1;
  bool m = false;
  if (c.cut) {
    const double x0 = i, x1 = i + 1;
    for (int s = 0; s < c.nSolids; s++) {
      const double* S = c.solids + 4 * s;
      if (x0 < S[1] + 1e-6 && x1 > S[0] - 1e-6) m |= ov(r0, r1, S[2] - 1e-6, S[3] + 1e-6);
    }
    if (!(double(c.colMax[i]) < -1e8)) {
      const double mn = c.colMin[i], mx = c.colMax[i];
      m |= ov(r0, r1, mn - 1e-6, mx + 1e-6);
      m |= ov(r0, r1, mn + c.twC - 1e-6, mx + c.twC + 1e-6);
      if (c.xeC >= x0 && c.xeC <= x1) m |= ov(r0, r1, mn, mx + c.twC);
      if (c.base) {
        if (c.xBaseC >= x0 && c.xBaseC <= x1) m |= ov(r0, r1, mn, c.bodyC);
        if (x0 < c.xBaseC) m |= (c.bodyC >= r0 && c.bodyC <= r1);
      }
    }
  }
  const double rcm = j + 0.5;
  const bool fl = fluid(c, i + 0.5, rcm, rin_at(c, i, 1));
  float Am = fl ? 1.0f : 0.0f, V = fl ? float(rcm) : 0.0f;
  uint8_t ic = 0;
  if (m) {
    int am = 0;
    double v = 0.0;
    for (int b = 0; b < NC; b++) {
      const double rc = j + (b + 0.5) / NC;
      for (int a = 0; a < NC; a++)
        if (fluid(c, i + (a + 0.5) / NC, rc, rin_at(c, i, 2 + a))) {
          am++;
          v += rc;
        }
    }
    Am = float(double(am) / (NC * NC));
    V = float(v / (NC * NC));
    ic = (Am > 0.0f && Am < 1.0f) ? 1 : 0;
  }
  c.mc[k] = m;
  c.V[k] = V;
  c.Am[k] = Am;
  c.isCut[k] = ic;
}

// open areas of the x- and r-faces (cutcell.js:84-104); lattice (Nr+1) x (Nx+1)
__global__ void k_faces(CutDev c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int Nx = c.Nx, Nr = c.Nr, W1 = Nx + 1;
  if (i > Nx || j > Nr) return;
  auto cutAt = [&](int ii, int jj) { return ii >= 0 && ii < Nx && jj >= 0 && jj < Nr && c.isCut[jj * Nx + ii]; };
  auto mcAt = [&](int ii, int jj) { return ii >= 0 && ii < Nx && jj >= 0 && jj < Nr && c.mc[jj * Nx + ii]; };
  // x-face at x = i, row j < Nr
  if (j < Nr) {
    bool sel = cutAt(i - 1, j) || cutAt(i, j) || mcAt(min(i, Nx - 1), j) || (i > 0 && mcAt(i - 1, j));
    if (!c.cut) sel = false;
    const double rcm = j + 0.5;
    // RinAt(i): slot 0 of column i, or the last column's slot for x = Nx
    const double ri = i < Nx ? rin_at(c, i, 0) : rin_at(c, Nx - 1, NS - 1);
    float A = fluid(c, double(i), rcm, ri) ? float(rcm) : 0.0f;
    if (sel) {
      double a = 0.0;
      for (int b = 0; b < NFS; b++) {
        const double rc = j + (b + 0.5) / NFS;
        if (fluid(c, double(i), rc, ri)) a += rc;
      }
      A = float(a / NFS);
    }
    c.Ax[j * W1 + i] = A;
  } else {
    c.Ax[j * W1 + i] = 0.0f;
  }
  // r-face at r = j, column i < Nx
  if (i < Nx) {
    bool sel = cutAt(i, j - 1) || cutAt(i, j) || mcAt(i, j) || mcAt(i, j - 1);
    if (!c.cut) sel = false;
    const double jf = j;
    float A = fluid(c, i + 0.5, jf, rin_at(c, i, 1)) ? float(jf) : 0.0f;
    if (sel) {
      int f = 0;
      for (int b = 0; b < NFS; b++)
        if (fluid(c, i + (b + 0.5) / NFS, jf, rin_at(c, i, 10 + b))) f++;
      A = float(double(j * f) / NFS);
    }
    c.Ar[j * W1 + i] = A;
  } else {
    c.Ar[j * W1 + i] = 0.0f;
  }
}

// kappa and the first solid classification (cutcell.js:107-112)
__global__ void k_classify(CutDev c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  if (i >= c.Nx || j >= c.Nr) return;
  const int k = j * c.Nx + i;
  const float kp = float(double(c.V[k]) / (j + 0.5));
  c.kap[k] = kp;
  c.solid[k] = double(kp) < 0.02 ? 1 : 0;   // Float32Array value compared as a double
  c.host[k] = -1;
}

// zero every face of a solid cell (cutcell.js:113-120, 143)
__global__ void k_solid_faces(CutDev c) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int Nx = c.Nx, Nr = c.Nr, W1 = Nx + 1;
  if (i > Nx || j > Nr) return;
  auto sol = [&](int ii, int jj) { return ii >= 0 && ii < Nx && jj >= 0 && jj < Nr && c.solid[jj * Nx + ii]; };
  if (j < Nr && (sol(i - 1, j) || sol(i, j))) c.Ax[j * W1 + i] = 0.0f;
  if (i < Nx && (sol(i, j - 1) || sol(i, j))) c.Ar[j * W1 + i] = 0.0f;
}

// sliver merge (cutcell.js:122-142): two passes over the slivers in row-major
// order, one thread, each decision seeing the earlier ones
__global__ void k_merge(CutDev c, const int* slivers, const int* nSliv) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int Nx = c.Nx, Nr = c.Nr, W1 = Nx + 1, n = *nSliv;
  for (int pas = 0; pas < 2; pas++) {
    for (int q = 0; q < n; q++) {
      const int k = slivers[q], i = k % Nx, j = k / Nx;
      if (c.solid[k] || double(c.kap[k]) >= KMERGE || c.host[k] >= 0) continue;
      int best = -1;
      double bestA = 0.0;
      for (int d = 0; d < 4; d++) {
        int ii = i, jj = j;
        double a;
        if (d == 0) { ii = i - 1; a = double(c.Ax[j * W1 + i]) / (j + 0.5); }
        else if (d == 1) { ii = i + 1; a = double(c.Ax[j * W1 + i + 1]) / (j + 0.5); }
        else if (d == 2) { jj = j - 1; a = j > 0 ? double(c.Ar[j * W1 + i]) / j : 0.0; }
        else { jj = j + 1; a = double(c.Ar[(j + 1) * W1 + i]) / (j + 1); }
        if (ii < 0 || ii >= Nx || jj < 0 || jj >= Nr) continue;
        const int kk = jj * Nx + ii;
        if (c.solid[kk] || double(c.kap[kk]) < KMERGE || c.host[kk] >= 0) continue;
        if (a > bestA + 1e-9) {
          bestA = a;
          best = kk;
        }
      }
      if (best >= 0 && bestA > 0.02) c.host[k] = best;
      else if (pas == 1) c.solid[k] = 1;
    }
  }
}

__global__ void k_sliver_flags(CutDev c, uint8_t* flags) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= c.Nx * c.Nr) return;
  flags[k] = (!c.solid[k] && double(c.kap[k]) < KMERGE) ? 1 : 0;
}

struct OutDev {
  float4* geoA;
  float4* geoG;
  float4* geoM;
  uint8_t* mask;
  float4* jw;
  unsigned* counts;   // nCut, nMerged
  const float* rinCol;
  double dx, xt, xe, Rt;
  int iExit;
};

__device__ bool partial_at(const CutDev& c, int i, int j) {
  if (i < 0 || i >= c.Nx || j < 0 || j >= c.Nr) return false;
  const int k = j * c.Nx + i;
  return !c.solid[k] && (double(c.kap[k]) < 0.98 || c.host[k] >= 0);
}

// geoA with first-order flags (cutcell.js:145-153)
__global__ void k_geoA(CutDev c, OutDev o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int Nx = c.Nx, Nr = c.Nr, W1 = Nx + 1;
  if (i > Nx || j > Nr) return;
  float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (i < Nx && j < Nr) {
    g.x = c.V[j * Nx + i];
    g.y = c.Am[j * Nx + i];
  }
  if (j < Nr) {
    const float a = c.Ax[j * W1 + i];
    g.z = (partial_at(c, i - 1, j) || partial_at(c, i, j)) ? -a : a;
  }
  if (i < Nx) {
    const float a = c.Ar[j * W1 + i];
    g.w = (partial_at(c, i, j - 1) || partial_at(c, i, j)) ? -a : a;
  }
  o.geoA[j * W1 + i] = g;
}

// wall vector of cell k by closure (cutcell.js:155-163)
__device__ void wall_vec(const CutDev& c, int i, int j, float& wx, float& wr) {
  const int W1 = c.Nx + 1, k = j * c.Nx + i;
  wx = float(double(c.Ax[j * W1 + i]) - double(c.Ax[j * W1 + i + 1]));
  wr = float(double(c.Am[k]) - (double(c.Ar[(j + 1) * W1 + i]) - double(c.Ar[j * W1 + i])));
  if (fabs(double(wx)) < 1e-6) wx = 0.0f;
  if (fabs(double(wr)) < 1e-6) wr = 0.0f;
  if (c.solid[k]) { wx = 0.0f; wr = 0.0f; }
}

// group sums, slave bits, geoG and geoM (cutcell.js:165-186), the turbulence
// length and boundary-layer band (simsetup.js:51-63), mask
__global__ void k_groups(CutDev c, OutDev o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
  const int Nx = c.Nx, Nr = c.Nr;
  if (i >= Nx || j >= Nr) return;
  const int k = j * Nx + i;
  const bool sol = c.solid[k] != 0;
  float4 G = make_float4(1.0f, 0.0f, 0.0f, 0.0f), M = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!sol) {
    const int h = c.host[k] >= 0 ? c.host[k] : k;
    const int hi = h % Nx, hj = h / Nx;
    // the group of h in ascending cell order: h-Nx, h-1, h, h+1, h+Nx
    const int nb[5] = {h - Nx, h - 1, h, h + 1, h + Nx};
    const bool okn[5] = {hj > 0, hi > 0, true, hi < Nx - 1, hj < Nr - 1};
    float gv = 0.0f, ga = 0.0f, gx = 0.0f, gr = 0.0f;
    unsigned smask = 0;
    for (int q = 0; q < 5; q++) {
      if (!okn[q]) continue;
      const int m = nb[q];
      const bool member = q == 2 || (c.host[m] == h && !c.solid[m]);
      if (!member) continue;
      float wx, wr;
      wall_vec(c, m % Nx, m / Nx, wx, wr);
      gv = gv + c.V[m];
      ga = ga + c.Am[m];
      gx = gx + wx;
      gr = gr + wr;
      if (q == 0) smask |= 4;
      else if (q == 1) smask |= 1;
      else if (q == 3) smask |= 2;
      else if (q == 4) smask |= 8;
    }
    G = make_float4(gv, ga, gx, gr);
    M = make_float4(float(hi - i), float(hj - j), h == k ? float(smask) : 0.0f, c.kap[k]);
    if (double(c.kap[k]) < 0.98) atomicAdd(o.counts + 0, 1u);   // nCut
    if (c.host[k] >= 0) atomicAdd(o.counts + 1, 1u);            // nMerged
  }
  // turbulence length scale and band flag (simsetup.js:51-63), every cell
  const double CS = 0.17, KAPPA = 0.41;
  const double x = (i + 0.5) * o.dx, Rin = o.rinCol[i], r = (j + 0.5) * o.dx;
  double l = CS;
  if (x <= o.xe && r < Rin) {
    const double s = x > o.xt ? x - o.xt : x;
    const double delta = 0.025 * s + (x > o.xt ? 0.05 * o.Rt : 0.0);
    l = fmax(CS, fmin(KAPPA * (Rin - r), 0.09 * delta) / o.dx);
    if (x > o.xt + 0.5 * o.Rt && Rin - r < fmax(2 * o.dx, delta)) M.z = float(double(M.z) + 16.0);
  }
  M.w = float(l);
  o.geoG[k] = G;
  o.geoM[k] = M;
  o.mask[k] = sol ? 1 : 0;
}

// near-wall fluid row of each column up to the exit plane (simsetup.js:226-231)
__global__ void k_jwall(CutDev c, OutDev o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= c.Nx) return;
  float jv = 0.0f;
  if (i <= o.iExit) {
    int j = min(c.Nr - 1, int(floor(double(o.rinCol[i]) / o.dx)));
    while (j > 0 && (c.solid[j * c.Nx + i] || double(c.kap[j * c.Nx + i]) < 0.5)) j--;
    jv = float(j);
  }
  o.jw[i] = make_float4(jv, 0.0f, 0.0f, 0.0f);
}

}  // namespace

extern "C" {

int rn_build_geometry(rn_handle h, const rn_cut_spec* sp, rn_cut_stats* stats) {
  if (!h || !h->SA[0] || !sp) return rn_record_error(RN_ERR_ARG, "rn_build_geometry: bad argument");
  if (sp->Nx != h->Nx || sp->Nr != h->Nr) return rn_record_error(RN_ERR_ARG, "rn_build_geometry: grid size differs");
  if (!sp->Rtab || !sp->rin || !sp->rinCol || (sp->nSolids > 0 && !sp->solids) || sp->nSolids < 0 ||
      sp->nSolids > 64)
    return rn_record_error(RN_ERR_ARG, "rn_build_geometry: missing table or bad solid count");
  if (sp->iExit < 0 || sp->iExit >= h->Nx) return rn_record_error(RN_ERR_ARG, "rn_build_geometry: iExit out of range");
  const int Nx = h->Nx, Nr = h->Nr, N = Nx * Nr, W1 = Nx + 1, NF = W1 * (Nr + 1);
  cudaStream_t s = h->stream;
  // scratch: one allocation
  const size_t nTab = size_t(Nx) * SUB + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
  const size_t oRtab = take(sizeof(float) * nTab), oRin = take(sizeof(double) * size_t(Nx) * NS);
  const size_t oSol = take(sizeof(double) * 4 * (sp->nSolids + 1)), oRinCol = take(sizeof(float) * Nx);
  const size_t oCol = take(sizeof(float) * 2 * Nx), oU8 = take(size_t(N) * 4), oHost = take(sizeof(int) * N);
  const size_t oF = take(sizeof(float) * 3 * size_t(N)), oFace = take(sizeof(float) * 2 * size_t(NF));
  const size_t oSl = take(sizeof(int) * (size_t(N) + 1)), oCnt = take(sizeof(unsigned) * 4);
  size_t cubBytes = 0;
  cub::DeviceSelect::Flagged(nullptr, cubBytes, thrust::counting_iterator<int>(0), (const uint8_t*)nullptr,
                             (int*)nullptr, (int*)nullptr, N, s);
  const size_t oCub = take(cubBytes + 16);
  char* base = nullptr;
  RN_CK(cudaMalloc(&base, off));
  CutDev c;
  c.Nx = Nx; c.Nr = Nr; c.cut = sp->cut; c.base = sp->base; c.nSolids = sp->nSolids;
  c.xeC = sp->xeC; c.twC = sp->twC; c.xBaseC = sp->xBaseC; c.bodyC = sp->bodyC;
  c.Rtab = reinterpret_cast<float*>(base + oRtab);
  c.rin = reinterpret_cast<double*>(base + oRin);
  c.solids = reinterpret_cast<double*>(base + oSol);
  c.colMin = reinterpret_cast<float*>(base + oCol);
  c.colMax = c.colMin + Nx;
  c.mc = reinterpret_cast<uint8_t*>(base + oU8);
  c.isCut = c.mc + N;
  c.solid = c.isCut + N;
  uint8_t* flags = c.solid + N;
  c.host = reinterpret_cast<int*>(base + oHost);
  c.V = reinterpret_cast<float*>(base + oF);
  c.Am = c.V + N;
  c.kap = c.Am + N;
  c.Ax = reinterpret_cast<float*>(base + oFace);
  c.Ar = c.Ax + NF;
  int* sliv = reinterpret_cast<int*>(base + oSl);
  int* nSliv = sliv + N;
  OutDev o;
  o.geoA = h->geoA; o.geoG = h->geoG; o.geoM = h->geoM; o.mask = h->mask; o.jw = h->jw;
  o.counts = reinterpret_cast<unsigned*>(base + oCnt);
  o.rinCol = reinterpret_cast<float*>(base + oRinCol);
  o.dx = sp->dx; o.xt = sp->xt; o.xe = sp->xe; o.Rt = sp->Rt; o.iExit = sp->iExit;
  cudaError_t e = cudaSuccess;
  auto ck = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  ck(cudaMemcpyAsync((void*)c.Rtab, sp->Rtab, sizeof(float) * nTab, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync((void*)c.rin, sp->rin, sizeof(double) * size_t(Nx) * NS, cudaMemcpyHostToDevice, s));
  if (sp->nSolids > 0)
    ck(cudaMemcpyAsync((void*)c.solids, sp->solids, sizeof(double) * 4 * sp->nSolids, cudaMemcpyHostToDevice, s));
  ck(cudaMemcpyAsync((void*)o.rinCol, sp->rinCol, sizeof(float) * Nx, cudaMemcpyHostToDevice, s));
  ck(cudaMemsetAsync(o.counts, 0, sizeof(unsigned) * 4, s));
  const dim3 b2(32, 8), gC((Nx + 31) / 32, (Nr + 7) / 8), gL((Nx + 32) / 32, (Nr + 8) / 8);
  if (e == cudaSuccess) {
    k_cols<<<(Nx + 127) / 128, 128, 0, s>>>(c);
    k_cells<<<gC, b2, 0, s>>>(c);
    k_faces<<<gL, b2, 0, s>>>(c);
    k_classify<<<gC, b2, 0, s>>>(c);
    k_solid_faces<<<gL, b2, 0, s>>>(c);
    k_sliver_flags<<<(N + 255) / 256, 256, 0, s>>>(c, flags);
    ck(cudaGetLastError());
    size_t cb = cubBytes;
    ck(cub::DeviceSelect::Flagged(base + oCub, cb, thrust::counting_iterator<int>(0), flags, sliv, nSliv, N, s));
    k_merge<<<1, 32, 0, s>>>(c, sliv, nSliv);
    k_solid_faces<<<gL, b2, 0, s>>>(c);
    k_geoA<<<gL, b2, 0, s>>>(c, o);
    k_groups<<<gC, b2, 0, s>>>(c, o);
    k_jwall<<<(Nx + 127) / 128, 128, 0, s>>>(c, o);
    ck(cudaGetLastError());
    h->launches += 11;
  }
  // host copies of the topology for the per-tile member lists
  unsigned cnt[4] = {0, 0, 0, 0};
  std::vector<uint8_t> mask(N);
  std::vector<float4> gm(N);
  if (e == cudaSuccess) {
    ck(cudaMemcpyAsync(mask.data(), h->mask, N, cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(gm.data(), h->geoM, sizeof(float4) * N, cudaMemcpyDeviceToHost, s));
    ck(cudaMemcpyAsync(cnt, o.counts, sizeof(cnt), cudaMemcpyDeviceToHost, s));
    ck(cudaStreamSynchronize(s));
  }
  cudaFree(base);
  if (e != cudaSuccess) return rn_record_cuda(e, "rn_build_geometry");
  h->hostMask = mask;
  h->hostGeoM.resize(size_t(N) * 4);
  std::memcpy(h->hostGeoM.data(), gm.data(), sizeof(float4) * N);
  int rc = rn_build_member_lists(h);
  if (rc != RN_OK) return rc;
  rc = rn_mask_refresh(h);
  if (rc != RN_OK) return rc;
  h->wvalid = false;
  if (stats) {
    stats->nCut = int(cnt[0]);
    stats->nMerged = int(cnt[1]);
  }
  return RN_OK;
}

}  // extern "C"
