// rn_math.cuh -- per-cell and per-face arithmetic of the time step, sm_100a.
//
// Every function states the reference shader lines it computes
// (source/solver.js, source/spray.js). The kernels in rn_step.cu fuse these
// into tiles; the arithmetic and its operation order are the reference's, so
// that in the exact variant (IEEE division and square root, multiply-add
// contraction off) the fused kernels give the same float32 results as the
// pass-by-pass restatement wherever the math library functions (pow, exp, log,
// sin, cos) agree.
// GLSL max/min are IEEE maxNum/minNum (fmaxf/fminf), what NVIDIA GPUs execute.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "rn.h"

#define RN_DEV __device__ __forceinline__

namespace rn {

constexpr float RHO_MIN = 1e-7f;   // solver.js:27
constexpr float P_MIN = 1e-7f;     // solver.js:28

struct Grid {
  int Nx, Nr;
  const uint8_t* __restrict__ mask;   // Nx*Nr, nonzero = solid
  const float4* __restrict__ geoA;    // (Nx+1)*(Nr+1): (V, Am, Ax west, Ar south), negative area -> first order
  const float4* __restrict__ geoG;    // Nx*Nr: group (V, Am, Wx, Wr)
  const float4* __restrict__ geoM;    // Nx*Nr: (host dx, host dy, slave mask, turbulence length)
};

struct Prim { float4 w, s; };        // w = (rho, u, v, p), s = (Z, F, G, O)   solver.js:29
struct Flux { float4 F, Y; float O; };   // face flux: F(4), (FZ, FF, u_f G_f, u_f), FO

// Division of the time-step arithmetic. The fast variant (RN_FAST) takes
// the hardware's reciprocal-based quotient (div.approx, within 2 ulp for
// divisors of magnitude 2^-126 .. 2^126, which every divisor here is: densities,
// pressures, wave speeds, face areas and volumes, all floored well above
// 2^-126 and far below 2^126); the exact variant divides as IEEE does.
RN_DEV float fdiv(float a, float b) {
#ifdef RN_FAST
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
// Several quotients over one divisor b: over(b)(a) == fdiv(a, b). The fast
// variant forms the reciprocal once and multiplies (fdiv there is a times the
// hardware reciprocal of b); the exact variant divides each time.
struct Over {
  float b, r;
  RN_DEV float operator()(float a) const {
#ifdef RN_FAST
    return a * r;
#else
    return a / b;
#endif
  }
};
RN_DEV Over over(float b) {
  Over o;
  o.b = b;
#ifdef RN_FAST
  o.r = __fdividef(1.0f, b);
#else
  o.r = 0.0f;
#endif
  return o;
}

// Pairs of lanes through Blackwell's packed FP32 instructions (two IEEE
// round-to-nearest operations per instruction, each lane rounding as the
// scalar operation does). madd2 is a*b + c: one fused multiply-add per lane in
// the fast variant, a multiply then an add (scalar) in the exact one.
RN_DEV float2 lo2(float4 v) { return make_float2(v.x, v.y); }
RN_DEV float2 hi2(float4 v) { return make_float2(v.z, v.w); }
RN_DEV float4 cat4(float2 l, float2 h) { return make_float4(l.x, l.y, h.x, h.y); }
RN_DEV float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
RN_DEV float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }   // a + (-b) == a - b
RN_DEV float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
RN_DEV float2 madd2(float2 a, float2 b, float2 c) {
#ifdef RN_FAST
  return __ffma2_rn(a, b, c);
#else
  // scalar lanes: a packed multiply followed by a packed add may be fused,
  // which the exact variant must not do (it is built with -fmad=false)
  return make_float2(c.x + a.x * b.x, c.y + a.y * b.y);
#endif
}
RN_DEV float4 diff4(float4 a, float4 b) { return cat4(sub2(lo2(a), lo2(b)), sub2(hi2(a), hi2(b))); }

RN_DEV float clampf(float x, float a, float b) { return fminf(fmaxf(x, a), b); }
RN_DEV float mixf(float x, float y, float a) { return x * (1.0f - a) + y * a; }
RN_DEV float smoothstepf(float e0, float e1, float x) {
  float t = clampf(fdiv(x - e0, e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
RN_DEV float len2(float a, float b) { return sqrtf(a * a + b * b); }
RN_DEV int iround(float v) { return __float2int_rn(v); }

RN_DEV bool solid_at(const Grid& g, int i, int j) { return g.mask[j * g.Nx + i] != 0; }

// toPrim (solver.js:33-39)
RN_DEV Prim to_prim(float4 a, float4 b) {
  Prim q;
  float rho = fmaxf(a.x, RHO_MIN);
  const Over per_rho = over(rho);
  float vx = per_rho(a.y), vy = per_rho(a.z);
  float G = fmaxf(b.z, 0.5f);
  float p = fmaxf(fdiv(a.w - 0.5f * rho * (vx * vx + vy * vy), G), P_MIN);
  q.w = make_float4(rho, vx, vy, p);
  q.s = make_float4(clampf(per_rho(b.x), 0.0f, 1.0f), clampf(per_rho(b.y), 0.0f, 1.0f), G,
                    clampf(per_rho(b.w), 0.0f, 1.0f));
  return q;
}
// soundSpeed (solver.js:40)
RN_DEV float sound_speed(const Prim& q) { return sqrtf(fdiv((1.0f + fdiv(1.0f, q.s.z)) * q.w.w, q.w.x)); }

// CFL wave speed of one fluid cell (FS_REDUCE1, solver.js:376-379)
RN_DEV float wave_speed(float4 a, float4 b) {
  Prim q = to_prim(a, b);
  return fabsf(q.w.y) + fabsf(q.w.z) + 2.0f * sound_speed(q);
}

// Cells of the grid as ghost_prim_c reads them: solid flag and raw state of
// in-grid cell (i, j). GlobalCells reads the planes in global memory; the
// stage kernels read the tile they staged in shared memory (rn_step.cu).
struct GlobalCells {
  const Grid& g;
  const float4* __restrict__ A;
  const float4* __restrict__ B;
  RN_DEV bool solid(int i, int j) const { return g.mask[j * g.Nx + i] != 0; }
  RN_DEV float4 a(int i, int j) const { return A[j * g.Nx + i]; }
  RN_DEV float4 b(int i, int j) const { return B[j * g.Nx + i]; }
};

// Padded primitive cell (i, j), i in [-2, Nx+1], j in [-2, Nr+1] (FS_PRIM,
// solver.js:56-126). Wall cells come back as W = (-1, 0, 0, 1), Wb = 0.
// t is the time the inlet ramp reads (t_old in stage 1, t_new in stage 2).
// Every cell it reads lies within 2 cells of (i, j), inside the grid.
template <class C>
RN_DEV void ghost_prim_c(int Nx, int Nr, const C& cells, int i, int j, float t, const rn_params& P, float4& W,
                         float4& Wb) {
  bool mir = j < 0;
  if (mir) j = -j - 1;
  Prim q;
  q.w = make_float4(P.amb[0], P.amb[1], P.amb[2], P.amb[3]);
  q.s = make_float4(0.0f, 0.0f, P.inlet[3], 0.0f);
  bool wall = false;
  if (i < 0) {
    if (j < Nr && cells.solid(0, j)) wall = true;
    else if (float(j) + 0.5f < P.RcCells && P.inj) wall = true;
    else if (float(j) + 0.5f < P.RcCells) {
      float f = P.ramp > 0.0f ? smoothstepf(0.0f, P.ramp, t) : 1.0f;
      float P0 = mixf(P.pStart, P.res[0], f);
      float T0 = P.res[1], R = P.res[2], G = P.inlet[2], gg = 1.0f + 1.0f / G;
      float4 a = cells.a(0, j);
      float ubar = fmaxf(cells.b(0, j).w, 0.0f);
      float c0 = sqrtf(gg * R * T0);
      float ui = clampf(a.y / fmaxf(a.x, RHO_MIN), 0.0f, 0.5f * c0);
      float ut = ubar * smoothstepf(1.0f, 2.0f, P0 / fmaxf(P.pStart, 1e-6f));
      float u = mixf(ui, ut, P.inlet[1]);
      float T = T0 - u * u * (gg - 1.0f) / (2.0f * gg * R);
      float p = P0 * powf(T / T0, gg * G);
      q.w = make_float4(p / (R * T), u, 0.0f, p);
      q.s = make_float4(1.0f, 1.0f, G, 0.0f);
    }
  } else if (j >= Nr) {
    int ci = min(i, Nx - 1), cj = Nr - 1;
    if (!cells.solid(ci, cj)) {
      Prim tq = to_prim(cells.a(ci, cj), cells.b(ci, cj));
      float cs = sound_speed(tq);
      if (tq.w.z >= cs) q = tq;
      else if (tq.w.z > 0.0f) { q = tq; q.w.w = P.amb[3]; }
    }
  } else if (i >= Nx) {
    int ci = Nx - 1, cj = j;
    if (!cells.solid(ci, cj)) {
      Prim tq = to_prim(cells.a(ci, cj), cells.b(ci, cj));
      float cs = sound_speed(tq);
      if (tq.w.y >= cs) q = tq;
      else if (tq.w.y > 0.0f) { q = tq; q.w.w = P.amb[3]; }
      else q.w.y = fmaxf(q.w.y, 0.0f);
    }
  } else {
    // the state is loaded with the mask (not after it), so the two loads overlap
    const float4 a = cells.a(i, j), b = cells.b(i, j);
    if (cells.solid(i, j)) wall = true;
    else q = to_prim(a, b);
  }
  if (wall) {
    W = make_float4(-1.0f, 0.0f, 0.0f, 1.0f);
    Wb = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  if (mir) q.w.z = -q.w.z;
  W = q.w;
  Wb = q.s;
}
RN_DEV void ghost_prim(const Grid& g, const float4* __restrict__ A, const float4* __restrict__ B, int i, int j,
                       float t, const rn_params& P, float4& W, float4& Wb) {
  ghost_prim_c(g.Nx, g.Nr, GlobalCells{g, A, B}, i, j, t, P, W, Wb);
}

// Interior cell as the padded texture holds it (wall flag or toPrim).
RN_DEV void interior_prim(const Grid& g, const float4* __restrict__ A, const float4* __restrict__ B, int i, int j,
                          float4& W, float4& Wb) {
  if (solid_at(g, i, j)) {
    W = make_float4(-1.0f, 0.0f, 0.0f, 1.0f);
    Wb = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  } else {
    Prim q = to_prim(A[j * g.Nx + i], B[j * g.Nx + i]);
    W = q.w;
    Wb = q.s;
  }
}

// ---------------------------------------------------------------------------
// Inviscid face flux: MUSCL van Leer + HLLC blended to HLL (makeFluxShader,
// solver.js:133-259). Inputs are the 4 cells along the face normal (padded
// W/Wb values) and the raw W of the 4 transverse sensor cells
// (k1+t, k1-t, ij+t, ij-t).
// 2 max(ab, 0) / den with den = a + b, or 1 where |den| <= 1e-30. For ab <= 0
// the quotient is a zero carrying den's sign, so the division is skipped; the
// result is the same float for every input that is not NaN.
// mix(den, 1, step(abs(den), 1e-30)) is den or 1 exactly for every finite den
// (a select); ab and den come in packed (van_leer4).
RN_DEV float van_leer_of(float ab, float den) {
  den = (1e-30f < fabsf(den)) ? den : 1.0f;
  return ab > 0.0f ? fdiv(2.0f * ab, den) : copysignf(0.0f, den);
}
RN_DEV float van_leer(float a, float b) { return van_leer_of(a * b, a + b); }
#ifdef RN_FAST
// Fast variant of a lane pair: ab > 0 means a and b of one sign, so |den| =
// |a| + |b| >= 2 sqrt(ab) > 1e-30 and the guard never applies; 2 ab / den is
// 2 ab times the hardware reciprocal of den (what fdiv computes), the pair's
// products in one packed multiply. Where ab <= 0 the limiter is a zero (its
// sign, which van_leer_of takes from den, only signs a zero face difference).
RN_DEV float2 van_leer2(float2 ab, float2 den) {
  const float2 q = mul2(add2(ab, ab), make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y)));
  return make_float2(ab.x > 0.0f ? q.x : 0.0f, ab.y > 0.0f ? q.y : 0.0f);
}
#endif
// Componentwise van_leer(a, b) of two float4 slopes.
RN_DEV float4 van_leer4(float4 a, float4 b) {
  const float2 ab0 = mul2(lo2(a), lo2(b)), ab1 = mul2(hi2(a), hi2(b));
  const float2 dn0 = add2(lo2(a), lo2(b)), dn1 = add2(hi2(a), hi2(b));
#ifdef RN_FAST
  return cat4(van_leer2(ab0, dn0), van_leer2(ab1, dn1));
#else
  return make_float4(van_leer_of(ab0.x, dn0.x), van_leer_of(ab0.y, dn0.y), van_leer_of(ab1.x, dn1.x),
                     van_leer_of(ab1.y, dn1.y));
#endif
}
// w + h * d per component (h = +-0.5: the MUSCL face values).
RN_DEV float4 step4(float4 w, float h, float4 d) {
  const float2 hh = make_float2(h, h);
  return cat4(madd2(hh, lo2(d), lo2(w)), madd2(hh, hi2(d), hi2(w)));
}
RN_DEV float jump_ratio(float a, float b) { return fdiv(fabsf(a - b), fminf(a, b)); }

// DIR_R selects the r-direction (normal velocity in .z). One instance of the
// code serves both directions: the fused kernels are large enough that a
// second inlined copy costs more in instruction-cache misses than the
// direction's selects cost in instructions.
RN_DEV Flux face_flux(bool DIR_R, float area, float4 w0, float4 b0, float4 w1, float4 b1, float4 w2, float4 b2,
                      float4 w3, float4 b3, float4 sa1, float4 sb1, float4 sa2, float4 sb2, const rn_params& P) {
  Flux out;
  out.F = make_float4(0.f, 0.f, 0.f, 0.f);
  out.Y = out.F;
  out.O = 0.0f;
  bool s0 = w0.x < 0.0f, s1 = w1.x < 0.0f, s2 = w2.x < 0.0f, s3 = w3.x < 0.0f;
  if (s1 && s2) return out;
  if (DIR_R) {   // face-normal frame: normal velocity in .y
    float t;
    t = w0.y; w0.y = w0.z; w0.z = t;
    t = w1.y; w1.y = w1.z; w1.z = t;
    t = w2.y; w2.y = w2.z; w2.z = t;
    t = w3.y; w3.y = w3.z; w3.z = t;
  }
  float hllw = 0.0f;
  if (P.hllBlend > 0.0f && !(s1 || s2)) {
    float p1 = w1.w, p2 = w2.w;
    float pa1 = sa1.x < 0.0f ? p1 : sa1.w, pb1 = sb1.x < 0.0f ? p1 : sb1.w;
    float pa2 = sa2.x < 0.0f ? p2 : sa2.w, pb2 = sb2.x < 0.0f ? p2 : sb2.w;
    // Smooth pressure (every jump ratio times hllBlend clearly below the 0.15
    // start of the smoothstep) gives hllw = 0 exactly; only test the ratios
    // where a jump is near. The margin (0.1 against 0.15) dwarfs rounding.
    const float hb = P.hllBlend;
    bool smooth = fabsf(pa1 - p1) * hb < 0.1f * fminf(pa1, p1) && fabsf(pb1 - p1) * hb < 0.1f * fminf(pb1, p1) &&
                  fabsf(pa2 - p2) * hb < 0.1f * fminf(pa2, p2) && fabsf(pb2 - p2) * hb < 0.1f * fminf(pb2, p2);
    if (!smooth) {
      float jm = fmaxf(fmaxf(jump_ratio(pa1, p1), jump_ratio(pb1, p1)), fmaxf(jump_ratio(pa2, p2), jump_ratio(pb2, p2)));
      hllw = smoothstepf(0.15f, 0.6f, jm * hb);
    }
  }
  float4 WLw, WLs, WRw, WRs;
  if (s1) { WRw = w2; WRs = b2; WLw = w2; WLw.y = -WLw.y; WLs = b2; }
  else if (s2) { WLw = w1; WLs = b1; WRw = w1; WRw.y = -WRw.y; WRs = b1; }
  else {
    if (s0) { w0 = w1; w0.y = -w0.y; b0 = b1; }
    if (s3) { w3 = w2; w3.y = -w3.y; b3 = b2; }
    WLw = w1; WLs = b1; WRw = w2; WRs = b2;
    if (P.order2 && area > 0.0f) {
      const float4 d12 = diff4(w2, w1);
      const float4 dL = van_leer4(diff4(w1, w0), d12), dR = van_leer4(d12, diff4(w3, w2));
      // w - 0.5 d == w + (-0.5) d in every rounding
      const float4 tL = step4(w1, 0.5f, dL), tR = step4(w2, -0.5f, dR);
      if (tL.x > 0.0f && tL.w > 0.0f && tR.x > 0.0f && tR.w > 0.0f) {
        const float4 e12 = diff4(b2, b1);
        const float4 yL = van_leer4(diff4(b1, b0), e12), yR = van_leer4(e12, diff4(b3, b2));
        const float4 sL = step4(b1, 0.5f, yL), sR = step4(b2, -0.5f, yR);
        WLw = tL;
        WLs = make_float4(clampf(sL.x, 0.0f, 1.0f), clampf(sL.y, 0.0f, 1.0f), clampf(sL.z, 0.5f, 100.0f),
                          clampf(sL.w, 0.0f, 1.0f));
        WRw = tR;
        WRs = make_float4(clampf(sR.x, 0.0f, 1.0f), clampf(sR.y, 0.0f, 1.0f), clampf(sR.z, 0.5f, 100.0f),
                          clampf(sR.w, 0.0f, 1.0f));
      }
    }
  }
  // HLLC (solver.js:211-251)
  float GL = WLs.z, GR = WRs.z;
  float rL = WLw.x, uL = WLw.y, vL = WLw.z, pL = WLw.w;
  float rR = WRw.x, uR = WRw.y, vR = WRw.z, pR = WRw.w;
  const Over per_rL = over(rL), per_rR = over(rR);
  float cL = sqrtf(per_rL((1.0f + fdiv(1.0f, GL)) * pL)), cR = sqrtf(per_rR((1.0f + fdiv(1.0f, GR)) * pR));
  float EL = pL * GL + 0.5f * rL * (uL * uL + vL * vL);
  float ER = pR * GR + 0.5f * rR * (uR * uR + vR * vR);
  float sL = sqrtf(rL), sR = sqrtf(rR);
  const Over per_s = over(sL + sR);
  float uT = per_s(sL * uL + sR * uR);
  float HT = per_s(per_rL(sL * (EL + pL)) + per_rR(sR * (ER + pR)));
  float vT = per_s(sL * vL + sR * vR);
  float GT = per_s(sL * GL + sR * GR);
  float cT = sqrtf(fmaxf(fdiv(HT - 0.5f * (uT * uT + vT * vT), GT), 1e-12f));
  float SL = fminf(uL - cL, uT - cT);
  float SR = fmaxf(uR + cR, uT + cT);
  float mL = rL * uL, mR = rR * uR;
  float FL0 = mL, FL1 = mL * uL + pL, FL2 = mL * vL, FL3 = uL * (EL + pL);
  float FR0 = mR, FR1 = mR * uR + pR, FR2 = mR * vR, FR3 = uR * (ER + pR);
  float YL0 = mL * WLs.x, YL1 = mL * WLs.y, YL2 = mL * WLs.w;
  float YR0 = mR * WRs.x, YR1 = mR * WRs.y, YR2 = mR * WRs.w;
  float F0, F1, F2, F3, Y0, Y1, Y2, uf, Gf;
  if (SL >= 0.0f) { F0 = FL0; F1 = FL1; F2 = FL2; F3 = FL3; Y0 = YL0; Y1 = YL1; Y2 = YL2; uf = uL; Gf = GL; }
  else if (SR <= 0.0f) { F0 = FR0; F1 = FR1; F2 = FR2; F3 = FR3; Y0 = YR0; Y1 = YR1; Y2 = YR2; uf = uR; Gf = GR; }
  else {
    float Ss = fdiv(pR - pL + mL * (SL - uL) - mR * (SR - uR), rL * (SL - uL) - rR * (SR - uR));
    bool left = Ss >= 0.0f;
    float rK = left ? rL : rR, uK = left ? uL : uR, vK = left ? vL : vR, pK = left ? pL : pR;
    float EK = left ? EL : ER, SK = left ? SL : SR;
    float YK0 = left ? WLs.x : WRs.x, YK1 = left ? WLs.y : WRs.y, YK2 = left ? WLs.w : WRs.w;
    float FK0 = left ? FL0 : FR0, FK1 = left ? FL1 : FR1, FK2 = left ? FL2 : FR2, FK3 = left ? FL3 : FR3;
    float FYK0 = left ? YL0 : YR0, FYK1 = left ? YL1 : YR1, FYK2 = left ? YL2 : YR2;
    float UK1 = left ? mL : mR, UK2 = rK * vK;
    const Over per_dS = over(SK - Ss);
    float kk = per_dS(rK * (SK - uK));
    float Us0 = kk * 1.0f, Us1 = kk * Ss, Us2 = kk * vK, Us3 = kk * (fdiv(EK, rK) + (Ss - uK) * (Ss + fdiv(pK, rK * (SK - uK))));
    float C0 = FK0 + SK * (Us0 - rK), C1 = FK1 + SK * (Us1 - UK1), C2 = FK2 + SK * (Us2 - UK2), C3 = FK3 + SK * (Us3 - EK);
    float CY0 = FYK0 + SK * (kk * YK0 - rK * YK0), CY1 = FYK1 + SK * (kk * YK1 - rK * YK1);
    float CY2 = FYK2 + SK * (kk * YK2 - rK * YK2);
    if (hllw != 0.0f) {
      float inv = fdiv(1.0f, SR - SL);
      float SLR = SL * SR;
      float H0 = (SR * FL0 - SL * FR0 + SLR * (rR - rL)) * inv;
      float H1 = (SR * FL1 - SL * FR1 + SLR * (mR - mL)) * inv;
      float H2 = (SR * FL2 - SL * FR2 + SLR * (rR * vR - rL * vL)) * inv;
      float H3 = (SR * FL3 - SL * FR3 + SLR * (ER - EL)) * inv;
      float HY0 = (SR * YL0 - SL * YR0 + SLR * (rR * WRs.x - rL * WLs.x)) * inv;
      float HY1 = (SR * YL1 - SL * YR1 + SLR * (rR * WRs.y - rL * WLs.y)) * inv;
      float HY2 = (SR * YL2 - SL * YR2 + SLR * (rR * WRs.w - rL * WLs.w)) * inv;
      F0 = mixf(C0, H0, hllw); F1 = mixf(C1, H1, hllw); F2 = mixf(C2, H2, hllw); F3 = mixf(C3, H3, hllw);
      Y0 = mixf(CY0, HY0, hllw); Y1 = mixf(CY1, HY1, hllw); Y2 = mixf(CY2, HY2, hllw);
    } else {
      // mix(Fc, Fhll, 0) = Fc + 0 Fhll: the HLL flux only decides the sign of
      // a zero component, so it is not computed where the sensor is quiet
      F0 = C0; F1 = C1; F2 = C2; F3 = C3;
      Y0 = CY0; Y1 = CY1; Y2 = CY2;
    }
    uf = uK + SK * (per_dS(SK - uK) - 1.0f);
    Gf = left ? GL : GR;
  }
  if (DIR_R) { float t = F1; F1 = F2; F2 = t; }    // rotate momentum back to (x, r)
  out.F = make_float4(F0, F1, F2, F3);
  out.Y = make_float4(Y0, Y1, uf * Gf, uf);
  out.O = Y2;
  return out;
}

// wallPressure (solver.js:301-306): slip-wall pressure from the reflected Riemann problem
RN_DEV float wall_pressure(const Prim& q, float un) {
  float g = 1.0f + fdiv(1.0f, q.s.z), p = q.w.w, rho = q.w.x, c = sqrtf(fdiv(g * p, rho));
  if (un > 0.0f) {
    float a = 0.25f * (g + 1.0f) * un;
    return p + rho * un * (a + sqrtf(a * a + c * c));
  }
  float f = fmaxf(1.0f + fdiv(0.5f * (g - 1.0f) * un, c), 0.0f);
  return p * powf(f, fdiv(2.0f * g, g - 1.0f));
}

// member flux accumulation of one group member (memberFlux, solver.js:287-299)
RN_DEV void sub4(float4& L, float ae, float4 fe, float aw, float4 fw) {
  L.x -= ae * fe.x - aw * fw.x;
  L.y -= ae * fe.y - aw * fw.y;
  L.z -= ae * fe.z - aw * fw.z;
  L.w -= ae * fe.w - aw * fw.w;
}

// GLSL_GAS (solver.js:445-450)
RN_DEV float sutherland(float TK, const rn_params& P) { return fdiv(P.gas[3] * 1.458e-6f * TK * sqrtf(TK), TK + 110.4f); }
RN_DEV float rmix(float4 s, const rn_params& P) {
  return (1.0f - s.x) * P.gas[0] + s.y * P.Rs[0] + s.w * P.Rs[1] + fmaxf(s.x - s.y - s.w, 0.0f) * P.Rs[2];
}

// FS_VCELL (solver.js:458-488) for one cell from its padded W/Wb and neighbours.
RN_DEV void vcell(float4 w0, float4 sc, float4 wE, float4 wW, float4 wN, float4 wS, int i, int j, float l, float dt,
                  const rn_params& P, float4& T1, float4& T2) {
  T1 = make_float4(0.f, 0.f, 0.f, 0.f);
  T2 = T1;
  if (w0.x < 0.0f) return;
  float fE = wE.x < 0.0f ? 0.0f : 1.0f, fW = wW.x < 0.0f ? 0.0f : 1.0f;
  float fN = wN.x < 0.0f ? 0.0f : 1.0f, fS = wS.x < 0.0f ? 0.0f : 1.0f;
  float dxn = fmaxf(fE + fW, 1.0f), drn = fmaxf(fN + fS, 1.0f);
  const Over per_dx = over(dxn), per_dr = over(drn);
  float ux = per_dx(fE * (wE.y - w0.y) + fW * (w0.y - wW.y));
  float vx = per_dx(fE * (wE.z - w0.z) + fW * (w0.z - wW.z));
  float ur = per_dr(fN * (wN.y - w0.y) + fS * (w0.y - wS.y));
  float vr = per_dr(fN * (wN.z - w0.z) + fS * (w0.z - wS.z));
  float r = float(j) + 0.5f, vor = fdiv(w0.z, r);
  float div = ux + vr + vor;
  float S2 = 2.0f * (ux * ux + vr * vr + vor * vor) + (ur + vx) * (ur + vx) - 0.6666667f * div * div;
  float om = vx - ur;
  float sens = fdiv(om * om, om * om + div * div + 1e-8f);
  float Smag = sqrtf(fmaxf(S2, 0.0f)) * sens;
  float rho = w0.x, p = w0.w;
  float Rm = rmix(sc, P);
  float mu = sutherland(fdiv(p, rho * Rm) * P.gas[2], P);
  float mut = rho * l * l * Smag;
  if (float(i) < P.chamberNu[1]) mut = fmaxf(mut, rho * P.chamberNu[0]);
  T1 = make_float4(ux, ur, vx, vr);
  T2 = make_float4(fminf(mu + mut, fdiv(0.08f * rho, fmaxf(dt, 1e-9f))), fdiv((sc.z + 1.0f) * p, rho), Smag, mu);
}

// makeViscFluxShader (solver.js:499-536) for one face. (w1, s1, t1, m1) is
// the cell behind the face, (w2, s2, t2, m2) the cell the face belongs to; j
// is the face's row; DIR_R selects the r-direction (one instance for both).
RN_DEV void visc_flux(bool DIR_R, float4 w1, float4 s1, float4 t1, float4 m1, float4 w2, float4 s2, float4 t2,
                      float4 m2, int j, float4& F, float4& FY) {
  float mu = 0.5f * (m1.x + m2.x);
  float uf = 0.5f * (w1.y + w2.y), vf = 0.5f * (w1.z + w2.z);
  float ttx = 0.5f * (t1.x + t2.x), tty = 0.5f * (t1.y + t2.y), ttz = 0.5f * (t1.z + t2.z), ttw = 0.5f * (t1.w + t2.w);
  float r, ux, vx, ur, vr;
  if (DIR_R) { r = fmaxf(float(j), 0.5f); ux = ttx; vx = ttz; ur = w2.y - w1.y; vr = w2.z - w1.z; }
  else { r = float(j) + 0.5f; ux = w2.y - w1.y; vx = w2.z - w1.z; ur = tty; vr = ttw; }
  float div = ux + vr + fdiv(vf, r);
  float txr = mu * (ur + vx);
  float k = mu * 1.25f;
  if (DIR_R) {
    float trr = mu * (2.0f * vr - 0.6666667f * div);
    F = make_float4(-k * (s2.w - s1.w), -txr, -trr, -(uf * txr + vf * trr) - k * (m2.y - m1.y));
  } else {
    float txx = mu * (2.0f * ux - 0.6666667f * div);
    F = make_float4(-k * (s2.w - s1.w), -txx, -txr, -(uf * txx + vf * txr) - k * (m2.y - m1.y));
  }
  FY = make_float4(-k * (s2.x - s1.x), -k * (s2.y - s1.y), -k * (s2.z - s1.z), 0.0f);
}

}  // namespace rn
