// rn_step.cu -- fused time-step kernels for sm_100a.
//
// One SSP-RK2 stage is ONE kernel (k_stage): a block stages the ghost-cell
// primitives of its TX x TY tile plus a 2-cell halo in shared memory
// (FS_PRIM, solver.js:56-126), computes every x- and r-face flux of the tile
// once (makeFluxShader, solver.js:133-259) into shared memory, then updates
// each cell over its merged cut-cell group (FS_UPDATE, solver.js:264-363).
// The reference's 7 full-grid passes per stage (prim, 2 flux, update, CFL
// chain) and its 6 face textures never touch HBM here. Group members that lie
// outside the tile (slivers merged across a tile edge) get their faces from a
// slow path that recomputes them from global memory.
//
// The step's last kernel folds the CFL wave speed of the cells it writes into
// one atomicMax per block (FS_REDUCE1/2, solver.js:368-397); the next step's
// stage-1 kernel turns it into dt in every block and block (0,0) stores the
// step info (FS_STEPINFO, solver.js:398-411). dt never leaves the device.
//
// The viscous/wall/reaction split step is ONE kernel (k_physics): vcell
// (FS_VCELL), the viscous face fluxes (makeViscFluxShader) and FS_SOURCE fused
// per tile, reading the stage-1 primitives (solver.js:940-941).
#include <cuda_runtime.h>
#include "rn_kernels.cuh"

namespace rn {

constexpr int PX = TX + 4, PY = TY + 4;   // primitive tile with a 2-cell halo

// --------------------------------------------------------------------------
// block-wide max of non-negative floats -> one atomicMax on the bit pattern
__device__ __forceinline__ void block_max_to(float w, unsigned* out, float* red) {
  for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = w;
  __syncthreads();
  if (wid == 0) {
    w = lane < (NT / 32) ? red[lane] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, o));
    if (lane == 0 && w > 0.0f) atomicMax(out, __float_as_uint(w));
  }
}

// --------------------------------------------------------------------------
// Slow path: one inviscid face recomputed from global memory.
template <bool DIR_R>
__device__ __noinline__ Flux face_flux_global(const Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                                               int i, int j, float t, const rn_params& P) {
  Flux f;
  f.F = make_float4(0.f, 0.f, 0.f, 0.f);
  f.Y = f.F;
  f.O = 0.0f;
  float4 geo = g.geoA[j * (g.Nx + 1) + i];
  float area = DIR_R ? geo.w : geo.z;
  if (area == 0.0f || (DIR_R && j == 0)) return f;
  const int dx = DIR_R ? 0 : 1, dy = DIR_R ? 1 : 0, tx = DIR_R ? 1 : 0, ty = DIR_R ? 0 : 1;
  float4 w0, b0, w1, b1, w2, b2, w3, b3, sa1, sb1, sa2, sb2, dum;
  ghost_prim(g, A, B, i - 2 * dx, j - 2 * dy, t, P, w0, b0);
  ghost_prim(g, A, B, i - dx, j - dy, t, P, w1, b1);
  ghost_prim(g, A, B, i, j, t, P, w2, b2);
  ghost_prim(g, A, B, i + dx, j + dy, t, P, w3, b3);
  ghost_prim(g, A, B, i - dx + tx, j - dy + ty, t, P, sa1, dum);
  ghost_prim(g, A, B, i - dx - tx, j - dy - ty, t, P, sb1, dum);
  ghost_prim(g, A, B, i + tx, j + ty, t, P, sa2, dum);
  ghost_prim(g, A, B, i - tx, j - ty, t, P, sb2, dum);
  return face_flux<DIR_R>(area, w0, b0, w1, b1, w2, b2, w3, b3, sa1, sb1, sa2, sb2, P);
}

// --------------------------------------------------------------------------
template <int STAGE>
__global__ void __launch_bounds__(NT) k_stage(StageArgs a, rn_params P) {
  __shared__ float4 sW[PY][PX], sWb[PY][PX];
  __shared__ float4 sXF[TY][TX + 1], sXY[TY][TX + 1];
  __shared__ float sXO[TY][TX + 1];
  __shared__ float4 sRF[TY + 1][TX], sRY[TY + 1][TX];
  __shared__ float sRO[TY + 1][TX];
  __shared__ float red[NT / 32];
  const Grid g = a.g;
  const int Nx = g.Nx, Nr = g.Nr, W1 = Nx + 1;
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;

  float dt, t;
  if (STAGE == 1) {
    float4 prev = *a.stPrev;
    float w = fmaxf(P.wFloor, __uint_as_float(*a.wIn));
    dt = fminf(P.cfl / w, P.dtMax);
    if (prev.x > 0.0f) dt = fminf(dt, prev.x * 1.2f);
    t = prev.z;                                   // inlet ramp at t_old
    if (blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) {
      *a.stNew = make_float4(dt, prev.z, prev.z + dt, w);
      *a.wOut = 0u;
    }
  } else {
    float4 st = *a.stNew;
    dt = st.x;
    t = st.z;                                     // inlet ramp at t_new
  }

  // ---- ghost-cell primitives of the tile + 2-cell halo
  for (int k = tid; k < PX * PY; k += NT) {
    int ly = k / PX, lx = k - ly * PX;
    int i = x0 - 2 + lx, j = y0 - 2 + ly;
    float4 W, Wb;
    if (i <= Nx + 1 && j <= Nr + 1) ghost_prim(g, a.A, a.B, i, j, t, P, W, Wb);
    else { W = make_float4(-1.f, 0.f, 0.f, 1.f); Wb = make_float4(0.f, 0.f, 0.f, 0.f); }
    sW[ly][lx] = W;
    sWb[ly][lx] = Wb;
  }
  __syncthreads();

  // ---- face fluxes: x-faces (TX+1) x TY, r-faces TX x (TY+1)
  for (int k = tid; k < TY * (TX + 1); k += NT) {
    int ly = k / (TX + 1), lx = k - ly * (TX + 1);
    int i = x0 + lx, j = y0 + ly;
    Flux f;
    f.F = make_float4(0.f, 0.f, 0.f, 0.f); f.Y = f.F; f.O = 0.f;
    if (i <= Nx && j < Nr) {
      float area = g.geoA[j * W1 + i].z;
      if (area != 0.0f) {
        const int py = ly + 2;
        f = face_flux<false>(area, sW[py][lx], sWb[py][lx], sW[py][lx + 1], sWb[py][lx + 1], sW[py][lx + 2],
                             sWb[py][lx + 2], sW[py][lx + 3], sWb[py][lx + 3], sW[py + 1][lx + 1], sW[py - 1][lx + 1],
                             sW[py + 1][lx + 2], sW[py - 1][lx + 2], P);
      }
    }
    sXF[ly][lx] = f.F; sXY[ly][lx] = f.Y; sXO[ly][lx] = f.O;
  }
  for (int k = tid; k < (TY + 1) * TX; k += NT) {
    int ly = k / TX, lx = k - ly * TX;
    int i = x0 + lx, j = y0 + ly;
    Flux f;
    f.F = make_float4(0.f, 0.f, 0.f, 0.f); f.Y = f.F; f.O = 0.f;
    if (i < Nx && j <= Nr && j != 0) {
      float area = g.geoA[j * W1 + i].w;
      if (area != 0.0f) {
        const int px = lx + 2;
        f = face_flux<true>(area, sW[ly][px], sWb[ly][px], sW[ly + 1][px], sWb[ly + 1][px], sW[ly + 2][px],
                            sWb[ly + 2][px], sW[ly + 3][px], sWb[ly + 3][px], sW[ly + 1][px + 1], sW[ly + 1][px - 1],
                            sW[ly + 2][px + 1], sW[ly + 2][px - 1], P);
      }
    }
    sRF[ly][lx] = f.F; sRY[ly][lx] = f.Y; sRO[ly][lx] = f.O;
  }
  __syncthreads();

  // ---- cut-cell group update (FS_UPDATE)
  const int lx = tid % TX, ly = tid / TX;
  const int i = x0 + lx, j = y0 + ly;
  float wcell = 0.0f;
  if (i < Nx && j < Nr) {
    const int k = j * Nx + i;
    float4 oA, oB;
    bool fluid = !g.mask[k];
    if (!fluid) {
      oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
      oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
    } else {
      float4 gm = g.geoM[k];
      const int Hx = i + iround(gm.x), Hy = j + iround(gm.y), kh = Hy * Nx + Hx;
      float4 gg = g.geoG[k];
      float4 A = a.A[kh], B = a.B[kh];
      Prim q = to_prim(A, B);
      float4 L = make_float4(0.f, 0.f, 0.f, 0.f), LY = L;
      float LO = 0.0f;
      const int sm = iround(g.geoM[kh].z);
      for (int m = 0; m < 5; m++) {
        int cx = Hx, cy = Hy;
        if (m == 1) { if (!(sm & 1)) continue; cx -= 1; }
        else if (m == 2) { if (!(sm & 2)) continue; cx += 1; }
        else if (m == 3) { if (!(sm & 4)) continue; cy -= 1; }
        else if (m == 4) { if (!(sm & 8)) continue; cy += 1; }
        float4 gc = g.geoA[cy * W1 + cx];
        float aw = fabsf(gc.z), ae = fabsf(g.geoA[cy * W1 + cx + 1].z);
        float as_ = fabsf(gc.w), an = fabsf(g.geoA[(cy + 1) * W1 + cx].w);
        const int mx = cx - x0, my = cy - y0;
        Flux fw, fe, fs, fn;
        if (mx >= 0 && mx < TX && my >= 0 && my < TY) {
          fw.F = sXF[my][mx]; fw.Y = sXY[my][mx]; fw.O = sXO[my][mx];
          fe.F = sXF[my][mx + 1]; fe.Y = sXY[my][mx + 1]; fe.O = sXO[my][mx + 1];
          fs.F = sRF[my][mx]; fs.Y = sRY[my][mx]; fs.O = sRO[my][mx];
          fn.F = sRF[my + 1][mx]; fn.Y = sRY[my + 1][mx]; fn.O = sRO[my + 1][mx];
        } else {
          fw = face_flux_global<false>(g, a.A, a.B, cx, cy, t, P);
          fe = face_flux_global<false>(g, a.A, a.B, cx + 1, cy, t, P);
          fs = face_flux_global<true>(g, a.A, a.B, cx, cy, t, P);
          fn = face_flux_global<true>(g, a.A, a.B, cx, cy + 1, t, P);
        }
        sub4(L, ae, fe.F, aw, fw.F);
        sub4(L, an, fn.F, as_, fs.F);
        sub4(LY, ae, fe.Y, aw, fw.Y);
        sub4(LY, an, fn.Y, as_, fs.Y);
        if (P.inj) {
          LO -= ae * fe.O - aw * fw.O;
          LO -= an * fn.O - as_ * fs.O;
        }
      }
      // embedded wall: pressure force along the r-weighted wall vector
      float wl = len2(gg.z, gg.w);
      if (wl > 1e-6f) {
        float nx = gg.z / wl, nr = gg.w / wl;
        float pw = wall_pressure(q, q.w.y * nx + q.w.z * nr);
        L.y -= gg.z * pw;
        L.z -= gg.w * pw;
      }
      L.z += q.w.w * gg.y;                       // axisymmetric source p Am
      float invV = 1.0f / fmaxf(gg.x, 1e-6f);
      float4 LB = make_float4(LY.x, LY.y, LY.z - q.s.z * LY.w, LO);
      float f = dt * invV;
      float4 U, UY;
      if (STAGE == 1) {
        U = make_float4(A.x + f * L.x, A.y + f * L.y, A.z + f * L.z, A.w + f * L.w);
        UY = make_float4(B.x + f * LB.x, B.y + f * LB.y, B.z + f * LB.z, B.w + f * LB.w);
      } else {
        float4 A0 = a.A0[kh], B0 = a.B0[kh];
        U = make_float4(0.5f * (A0.x + A.x + f * L.x), 0.5f * (A0.y + A.y + f * L.y), 0.5f * (A0.z + A.z + f * L.z),
                        0.5f * (A0.w + A.w + f * L.w));
        UY = make_float4(0.5f * (B0.x + B.x + f * LB.x), 0.5f * (B0.y + B.y + f * LB.y),
                         0.5f * (B0.z + B.z + f * LB.z), 0.5f * (B0.w + B.w + f * LB.w));
      }
      float rho = fmaxf(U.x, RHO_MIN);
      float den = fmaxf(U.x, RHO_MIN);
      float vx = U.y / den, vy = U.z / den;
      float sp = len2(vx, vy);
      if (sp > P.vMax) { float s = P.vMax / sp; vx *= s; vy *= s; }
      if (!(rho < 1e30f) || !(vx < 1e30f && vx > -1e30f)) {   // NaN guard
        oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
        oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
      } else {
        float ke = 0.5f * rho * (vx * vx + vy * vy);
        float Gn = clampf(UY.z, P.gamR[0], P.gamR[1]);
        float E = fmaxf(U.w, P_MIN * Gn + ke);
        float Zn = clampf(UY.x, 0.0f, rho);
        oA = make_float4(rho, rho * vx, rho * vy, E);
        float ubar = 0.0f;
        if (P.inj) ubar = clampf(UY.w, 0.0f, rho);
        else if (i == 0) {
          float u0 = a.B[k].w;
          bool on = STAGE == 2 && t > P.bar[2];
          ubar = on ? fminf(u0 + fminf(dt * P.bar[0], 1.0f) * (vx - u0), P.bar[1]) : u0;
        }
        oB = make_float4(Zn, clampf(UY.y, 0.0f, Zn), Gn, ubar);
      }
    }
    a.oA[k] = oA;
    a.oB[k] = oB;
    if (a.finalCfl && fluid) wcell = wave_speed(oA, oB);
  }
  if (a.finalCfl) block_max_to(wcell, a.wOut, red);
}

// --------------------------------------------------------------------------
// Slow path for the physics kernel: one viscous face from global memory.
__device__ __noinline__ void vcell_global(const Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                                          int i, int j, float t, float dt, const rn_params& P, float4& T1, float4& T2) {
  float4 w0, s0, wE, wW, wN, wS, d;
  ghost_prim(g, A, B, i, j, t, P, w0, s0);
  ghost_prim(g, A, B, i + 1, j, t, P, wE, d);
  ghost_prim(g, A, B, i - 1, j, t, P, wW, d);
  ghost_prim(g, A, B, i, j + 1, t, P, wN, d);
  ghost_prim(g, A, B, i, j - 1, t, P, wS, d);
  vcell(w0, s0, wE, wW, wN, wS, i, j, g.geoM[j * g.Nx + i].w, dt, P, T1, T2);
}

template <bool DIR_R>
__device__ __noinline__ void vflux_global(const Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                                          int i, int j, float t, float dt, const rn_params& P, float4& F, float4& FY) {
  F = make_float4(0.f, 0.f, 0.f, 0.f);
  FY = F;
  float4 geo = g.geoA[j * (g.Nx + 1) + i];
  int k1x, k1y;
  if (DIR_R) {
    if (geo.w == 0.0f || j == 0 || j >= g.Nr) return;
    k1x = i; k1y = j - 1;
  } else {
    if (geo.z == 0.0f || i == 0 || i >= g.Nx) return;
    k1x = i - 1; k1y = j;
  }
  float4 w1, s1, w2, s2;
  ghost_prim(g, A, B, k1x, k1y, t, P, w1, s1);
  ghost_prim(g, A, B, i, j, t, P, w2, s2);
  if (w1.x < 0.0f || w2.x < 0.0f) return;
  float4 t1, m1, t2, m2;
  vcell_global(g, A, B, k1x, k1y, t, dt, P, t1, m1);
  vcell_global(g, A, B, i, j, t, dt, P, t2, m2);
  visc_flux<DIR_R>(w1, s1, t1, m1, w2, s2, t2, m2, j, F, FY);
}

// --------------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_physics(PhysArgs a, rn_params P) {
  __shared__ float4 sW[PY][PX], sWb[PY][PX];
  __shared__ float4 sT1[TY + 2][TX + 2], sT2[TY + 2][TX + 2];
  __shared__ float4 sXF[TY][TX + 1], sXY[TY][TX + 1];
  __shared__ float4 sRF[TY + 1][TX], sRY[TY + 1][TX];
  __shared__ float red[NT / 32];
  const Grid g = a.g;
  const int Nx = g.Nx, Nr = g.Nr, W1 = Nx + 1;
  const int tid = threadIdx.x;
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const float4 st = *a.st;
  const float dt = st.x, t = st.z;

  for (int k = tid; k < PX * PY; k += NT) {
    int ly = k / PX, lx = k - ly * PX;
    int i = x0 - 2 + lx, j = y0 - 2 + ly;
    float4 W, Wb;
    if (i <= Nx + 1 && j <= Nr + 1) ghost_prim(g, a.A1, a.B1, i, j, t, P, W, Wb);
    else { W = make_float4(-1.f, 0.f, 0.f, 1.f); Wb = make_float4(0.f, 0.f, 0.f, 0.f); }
    sW[ly][lx] = W;
    sWb[ly][lx] = Wb;
  }
  __syncthreads();
  // vcell over the tile + 1 ring
  for (int k = tid; k < (TX + 2) * (TY + 2); k += NT) {
    int ly = k / (TX + 2), lx = k - ly * (TX + 2);
    int i = x0 - 1 + lx, j = y0 - 1 + ly;
    float4 T1 = make_float4(0.f, 0.f, 0.f, 0.f), T2 = T1;
    if (i >= 0 && i < Nx && j >= 0 && j < Nr) {
      const int px = lx + 1, py = ly + 1;
      vcell(sW[py][px], sWb[py][px], sW[py][px + 1], sW[py][px - 1], sW[py + 1][px], sW[py - 1][px], i, j,
            g.geoM[j * Nx + i].w, dt, P, T1, T2);
    }
    sT1[ly][lx] = T1;
    sT2[ly][lx] = T2;
  }
  __syncthreads();
  if (P.visc) {
    for (int k = tid; k < TY * (TX + 1); k += NT) {
      int ly = k / (TX + 1), lx = k - ly * (TX + 1);
      int i = x0 + lx, j = y0 + ly;
      float4 F = make_float4(0.f, 0.f, 0.f, 0.f), FY = F;
      if (i > 0 && i < Nx && j < Nr && g.geoA[j * W1 + i].z != 0.0f) {
        float4 w1 = sW[ly + 2][lx + 1], w2 = sW[ly + 2][lx + 2];
        if (!(w1.x < 0.0f || w2.x < 0.0f))
          visc_flux<false>(w1, sWb[ly + 2][lx + 1], sT1[ly + 1][lx], sT2[ly + 1][lx], w2, sWb[ly + 2][lx + 2],
                           sT1[ly + 1][lx + 1], sT2[ly + 1][lx + 1], j, F, FY);
      }
      sXF[ly][lx] = F; sXY[ly][lx] = FY;
    }
    for (int k = tid; k < (TY + 1) * TX; k += NT) {
      int ly = k / TX, lx = k - ly * TX;
      int i = x0 + lx, j = y0 + ly;
      float4 F = make_float4(0.f, 0.f, 0.f, 0.f), FY = F;
      if (i < Nx && j > 0 && j < Nr && g.geoA[j * W1 + i].w != 0.0f) {
        float4 w1 = sW[ly + 1][lx + 2], w2 = sW[ly + 2][lx + 2];
        if (!(w1.x < 0.0f || w2.x < 0.0f))
          visc_flux<true>(w1, sWb[ly + 1][lx + 2], sT1[ly][lx + 1], sT2[ly][lx + 1], w2, sWb[ly + 2][lx + 2],
                          sT1[ly + 1][lx + 1], sT2[ly + 1][lx + 1], j, F, FY);
      }
      sRF[ly][lx] = F; sRY[ly][lx] = FY;
    }
  }
  __syncthreads();

  // ---- FS_SOURCE
  const int lx = tid % TX, ly = tid / TX;
  const int i = x0 + lx, j = y0 + ly;
  float wcell = 0.0f;
  if (i < Nx && j < Nr) {
    const int k = j * Nx + i;
    float4 oA, oB;
    bool fluid = !g.mask[k];
    if (!fluid) {
      oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
      oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
    } else {
      float4 gmij = g.geoM[k];
      const int Hx = i + iround(gmij.x), Hy = j + iround(gmij.y), kh = Hy * Nx + Hx;
      float4 gg = g.geoG[k];
      float4 A = a.A2[kh], B = a.B2[kh];
      Prim q = to_prim(A, B);
      float rho = q.w.x, p = q.w.w, G = q.s.z;
      float velx = q.w.y, vely = q.w.z;
      float V = fmaxf(gg.x, 1e-6f);
      float Rm = rmix(q.s, P), Tg = p / (rho * Rm);
      float4 L = make_float4(0.f, 0.f, 0.f, 0.f), LY = L;
      float4 T1h = sT1[Hy - y0 + 1][Hx - x0 + 1], T2h = sT2[Hy - y0 + 1][Hx - x0 + 1];
      if (P.visc) {
        const int sm = iround(g.geoM[kh].z);
        for (int m = 0; m < 5; m++) {
          int cx = Hx, cy = Hy;
          if (m == 1) { if (!(sm & 1)) continue; cx -= 1; }
          else if (m == 2) { if (!(sm & 2)) continue; cx += 1; }
          else if (m == 3) { if (!(sm & 4)) continue; cy -= 1; }
          else if (m == 4) { if (!(sm & 8)) continue; cy += 1; }
          float4 gc = g.geoA[cy * W1 + cx];
          float aw = fabsf(gc.z), ae = fabsf(g.geoA[cy * W1 + cx + 1].z);
          float as_ = fabsf(gc.w), an = fabsf(g.geoA[(cy + 1) * W1 + cx].w);
          const int mx = cx - x0, my = cy - y0;
          float4 fwF, fwY, feF, feY, fsF, fsY, fnF, fnY;
          if (mx >= 0 && mx < TX && my >= 0 && my < TY) {
            fwF = sXF[my][mx]; fwY = sXY[my][mx]; feF = sXF[my][mx + 1]; feY = sXY[my][mx + 1];
            fsF = sRF[my][mx]; fsY = sRY[my][mx]; fnF = sRF[my + 1][mx]; fnY = sRY[my + 1][mx];
          } else {
            vflux_global<false>(g, a.A1, a.B1, cx, cy, t, dt, P, fwF, fwY);
            vflux_global<false>(g, a.A1, a.B1, cx + 1, cy, t, dt, P, feF, feY);
            vflux_global<true>(g, a.A1, a.B1, cx, cy, t, dt, P, fsF, fsY);
            vflux_global<true>(g, a.A1, a.B1, cx, cy + 1, t, dt, P, fnF, fnY);
          }
          sub4(L, ae, feF, aw, fwF);
          sub4(L, an, fnF, as_, fsF);
          sub4(LY, ae, feY, aw, fwY);
          sub4(LY, an, fnY, as_, fsY);
        }
        // axisymmetric hoop stress
        float r = V / fmaxf(gg.y, 1e-6f), vor = vely / r;
        L.z -= T2h.x * (2.0f * vor - 0.6666667f * (T1h.x + T1h.w + vor)) * gg.y;
        // Werner-Wengle wall shear and Reynolds-analogy heat flux
        float wl = len2(gg.z, gg.w);
        if (wl > 1e-6f) {
          float nx = gg.z / wl, nr = gg.w / wl;
          float dn = velx * nx + vely * nr;
          float utx = velx - dn * nx, uty = vely - dn * nr;
          float up = len2(utx, uty);
          float cp = Rm * (G + 1.0f);
          float Taw = Tg + 0.89f * up * up / (2.0f * cp);
          float Ts = fmaxf(Tg + 0.5f * (P.Tw - Tg) + 0.22f * (Taw - Tg), 1e-3f);
          float rs = p / (Rm * Ts), mus = sutherland(Ts * P.gas[2], P);
          float dz = 2.0f * clampf(0.5f * V / wl, 0.25f, 1.0f);
          float nz = mus / (rs * dz);
          float tw = up <= 69.7f * nz ? 2.0f * mus * up / dz
                                      : rs * powf(7.187f * powf(nz, 1.142857f) + 0.13769f * powf(nz, 0.142857f) * up, 1.75f);
          tw = fminf(tw, 0.3f * rho * up * V / fmaxf(wl * dt, 1e-9f));
          if (up > 1e-6f) { L.y -= tw * wl * utx / up; L.z -= tw * wl * uty / up; }
          float qw = tw / fmaxf(up, 1e-4f) * cp * (Taw - P.Tw) * 1.24f;
          float qmax = 0.3f * p * G * V / fmaxf(wl * dt, 1e-9f);
          L.w -= clampf(qw, -qmax, qmax) * wl;
        }
        // shock / boundary-layer interaction on the bit-16 band
        if (sm & 16) {
          float up = len2(velx, vely), Mn = up / sqrtf((1.0f + 1.0f / G) * p / rho);
          if (Mn > 1.0f) {
            float shx = velx / up, shy = vely / up;
            float pd = 0.0f;
            for (int n = 4; n <= 6; n += 2)
              for (int mm = 0; mm <= 1; mm++) {
                int Dx = Hx + int(rintf(float(n) * shx));
                int Dy = Hy + int(floorf(float(n) * shy)) + mm;
                Dx = min(max(Dx, 0), Nx - 1);
                Dy = min(max(Dy, 0), Nr - 1);
                float4 wd, sd;
                interior_prim(g, a.A1, a.B1, Dx, Dy, wd, sd);
                if (wd.x > 0.0f) pd = fmaxf(pd, wd.w);
              }
            float crit = 1.0f + 0.5f * Mn;
            float fsep = smoothstepf(crit, 1.2f * crit, pd / p) * V * rho * up;
            L.y -= fsep * velx;
            L.z -= fsep * vely;
          } else if (velx > 0.0f && p < 1.3f * P.chemK[3]) {
            float fsep = 0.5f * V * rho * up;
            L.y -= fsep * velx;
            L.z -= fsep * vely;
          }
        }
      }
      float invV = dt / V;
      float dO = invV * L.x;
      L.x = 0.0f;
      float4 U = make_float4(A.x + invV * L.x, A.y + invV * L.y, A.z + invV * L.z, A.w + invV * L.w);
      float4 UY = make_float4(B.x + invV * LY.x / 1.0f, B.y + invV * LY.y / 1.0f, B.z + invV * LY.z / rho,
                              B.w + invV * 0.0f / 1.0f);
      if (P.inj) UY.w += dO;
      if (P.chem) {
        float Z = q.s.x, F = q.s.y, O = q.s.w, s = P.chemK[1];
        float avail = P.inj ? fminf(F, (O + 0.233f * fmaxf(1.0f - Z, 0.0f)) / s)
                            : fminf(F, fmaxf(1.0f - Z - s * (Z - F), 0.0f) / s);
        if (avail > 1e-5f) {
          float TK = Tg * P.gas[2];
          float kin = P.chemK[2] * p * expf(-9000.0f / TK) * (1.0f - smoothstepf(P.cap[0], P.cap[1], TK));
          float mixr = P.inj ? fmaxf(T2h.z, 4.0f * T2h.x / rho) : T2h.z;
          float burn = avail * fminf(fminf(mixr, kin) * dt, 0.5f);
          UY.y -= rho * burn;
          if (P.inj) UY.w = fmaxf(UY.w - rho * burn * s, 0.0f);
          U.w += rho * burn * P.chemK[0];
        }
      }
      float rn = fmaxf(U.x, RHO_MIN);
      float vnx = U.y / rn, vny = U.z / rn;
      if (!(rn < 1e30f) || !(vnx < 1e30f && vnx > -1e30f)) {
        oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
        oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
      } else {
        float Gn = clampf(UY.z, P.gamR[0], P.gamR[1]);
        float Zn = clampf(UY.x, 0.0f, rn);
        oA = make_float4(rn, rn * vnx, rn * vny, fmaxf(U.w, P_MIN * Gn + 0.5f * rn * (vnx * vnx + vny * vny)));
        oB = make_float4(Zn, clampf(UY.y, 0.0f, Zn), Gn, P.inj ? clampf(UY.w, 0.0f, rn) : a.B2[k].w);
      }
    }
    a.oA[k] = oA;
    a.oB[k] = oB;
    if (a.finalCfl && fluid) wcell = wave_speed(oA, oB);
  }
  if (a.finalCfl) block_max_to(wcell, a.wOut, red);
}

// --------------------------------------------------------------------------
// stand-alone CFL reduction of a state (first step after setState/rescale)
__global__ void __launch_bounds__(NT) k_reduce(Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                                               unsigned* out) {
  __shared__ float red[NT / 32];
  const int N = g.Nx * g.Nr;
  float w = 0.0f;
  for (int k = blockIdx.x * NT + threadIdx.x; k < N; k += gridDim.x * NT)
    if (!g.mask[k]) w = fmaxf(w, wave_speed(A[k], B[k]));
  block_max_to(w, out, red);
}

// FS_RESCALE (solver.js:418-437)
__global__ void k_rescale(Grid g, const float4* __restrict__ A, const float4* __restrict__ B, float4* oA, float4* oB,
                          float fp, float fT, float du, rn_params P) {
  const int N = g.Nx * g.Nr;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
    float4 a = A[k], b = B[k];
    if (g.mask[k]) {
      oA[k] = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
      oB[k] = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
      continue;
    }
    Prim q = to_prim(a, b);
    float w = 1.0f - smoothstepf(0.0f, 0.03f, q.s.x);
    float rho = q.w.x * mixf(1.0f, fp / fT, w);
    float p = q.w.w * mixf(1.0f, fp, w);
    float vx = q.w.y + du * w, vy = q.w.z + 0.0f;
    oA[k] = make_float4(rho, rho * vx, rho * vy, p * q.s.z + 0.5f * rho * (vx * vx + vy * vy));
    oB[k] = make_float4(rho * q.s.x, rho * q.s.y, q.s.z, b.w);
  }
}

// FS_WALLROW (solver.js:665-674)
__global__ void k_wallrow(Grid g, const float4* __restrict__ A, const float4* __restrict__ B, const float4* jw,
                          float4* row) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= g.Nx) return;
  int cj = int(jw[i].x);
  cj = min(max(cj, 0), g.Nr - 1);
  Prim q = to_prim(A[cj * g.Nx + i], B[cj * g.Nx + i]);
  row[i] = make_float4(q.w.y, q.w.z, q.w.w, sound_speed(q));
}

// --------------------------------------------------------------------------
// FP64 read-outs with Neumaier-compensated sums (one warp per integral).
struct Neu {
  double s = 0.0, c = 0.0;
  __device__ void add(double x) {
    double t = s + x;
    c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  __device__ double val() const { return s + c; }
};
__device__ double warp_sum_exact(Neu n) {
  // combine the lanes' (s, c) pairs in lane order on lane 0: deterministic
  double s = n.s, c = n.c;
  __shared__ double bs[32], bc[32];
  bs[threadIdx.x] = s;
  bc[threadIdx.x] = c;
  __syncwarp();
  double r = 0.0;
  if (threadIdx.x == 0) {
    Neu t;
    for (int l = 0; l < 32; l++) { t.add(bs[l]); t.add(bc[l]); }
    r = t.val();
  }
  __syncwarp();
  return r;
}
__global__ void k_integrals(Grid g, const float4* __restrict__ A, const float4* __restrict__ B,
                            const float4* __restrict__ geoA, rn_integral_spec sp, const float4* st, double* out) {
  const int Nx = g.Nx, W1 = Nx + 1, lane = threadIdx.x;
  const double PI = 3.14159265358979323846;
  Neu F, m, Mw, pw, Ar, tm, tO, tF;
  for (int j = lane; j < sp.jExit; j += 32) {
    const int k = j * Nx + sp.iExit;
    float4 a = A[k], b = B[k];
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho, v = (double)a.z / rho;
    double G = (double)b.z, gam = 1.0 + 1.0 / G;
    double p = fmax(((double)a.w - 0.5 * rho * (u * u + v * v)) / G, 1e-9);
    double dA = 2.0 * PI * fabs((double)geoA[j * W1 + sp.iExit + 1].z) * sp.dx * sp.dx;
    double c = sqrt(gam * p / rho);
    double mm = (double)b.x * u * dA;
    F.add((rho * u * u + p - sp.pAmb) * dA);
    m.add(mm);
    Mw.add(mm * sqrt(u * u + v * v) / c);
    pw.add(p * dA);
    Ar.add(dA);
  }
  // throat plane: stop at the first solid cell (chamberPerformance)
  int jstop = g.Nr;
  for (int j = 0; j < g.Nr; j++)
    if (g.mask[j * Nx + sp.iThroat]) { jstop = j; break; }
  for (int j = lane; j < jstop; j += 32) {
    const int k = j * Nx + sp.iThroat;
    float4 a = A[k], b = B[k];
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho;
    double dA = 2.0 * PI * fabs((double)geoA[j * W1 + sp.iThroat].z) * sp.dx * sp.dx;
    tm.add(rho * u * dA);
    tO.add((double)b.w * u * dA);
    tF.add((double)b.y * u * dA);
  }
  double r[8] = {warp_sum_exact(F), warp_sum_exact(m), warp_sum_exact(Mw), warp_sum_exact(pw),
                 warp_sum_exact(Ar), warp_sum_exact(tm), warp_sum_exact(tO), warp_sum_exact(tF)};
  if (lane == 0) {
    for (int q = 0; q < 8; q++) out[q] = r[q];
    const int kc = sp.iChamber;     // chamber probe at (iChamber, 0)
    float4 a = A[kc], b = B[kc];
    double G = (double)b.z;
    double rho = fmax((double)a.x, 1e-9), u = (double)a.y / rho, v = (double)a.z / rho;
    double p = fmax(((double)a.w - 0.5 * rho * (u * u + v * v)) / G, 1e-9);
    double Y = fmin(fmax((double)b.x / rho, 0.0), 1.0);
    double Fv = fmax((double)b.y / rho, 0.0), Ov = sp.inj ? fmax((double)b.w / rho, 0.0) : 0.0;
    double Rm = (1.0 - Y) * sp.RaN + Fv * sp.Rs[0] + Ov * sp.Rs[1] + fmax(Y - Fv - Ov, 0.0) * sp.Rs[2];
    out[8] = p;
    out[9] = p / (rho * Rm);
    float4 s = *st;
    out[10] = (double)s.x;
    out[11] = (double)s.z;
  }
}

// --------------------------------------------------------------------------
static dim3 tiles(const Grid& g) { return dim3((g.Nx + TX - 1) / TX, (g.Nr + TY - 1) / TY); }

void launch_stage1(const StageArgs& a, const rn_params& P, cudaStream_t s) { k_stage<1><<<tiles(a.g), NT, 0, s>>>(a, P); }
void launch_stage2(const StageArgs& a, const rn_params& P, cudaStream_t s) { k_stage<2><<<tiles(a.g), NT, 0, s>>>(a, P); }
void launch_physics(const PhysArgs& a, const rn_params& P, cudaStream_t s) { k_physics<<<tiles(a.g), NT, 0, s>>>(a, P); }
void launch_reduce(const Grid& g, const float4* A, const float4* B, unsigned* w, cudaStream_t s) {
  int N = g.Nx * g.Nr;
  int blocks = (N + NT - 1) / NT;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_reduce<<<blocks, NT, 0, s>>>(g, A, B, w);
}
void launch_rescale(const Grid& g, const float4* A, const float4* B, float4* oA, float4* oB, float fp, float fT,
                    float du, const rn_params& P, cudaStream_t s) {
  int N = g.Nx * g.Nr;
  k_rescale<<<(N + 255) / 256, 256, 0, s>>>(g, A, B, oA, oB, fp, fT, du, P);
}
void launch_wallrow(const Grid& g, const float4* A, const float4* B, const float4* jw, float4* row, cudaStream_t s) {
  k_wallrow<<<(g.Nx + 127) / 128, 128, 0, s>>>(g, A, B, jw, row);
}
void launch_integrals(const Grid& g, const float4* A, const float4* B, const float4* geoAx, const rn_integral_spec& spec,
                      const float4* st, double* out, cudaStream_t s) {
  k_integrals<<<1, 32, 0, s>>>(g, A, B, geoAx, spec, st, out);
}

}  // namespace rn
