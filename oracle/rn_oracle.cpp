// =============================================================================
// rn_oracle.cpp -- CPU oracle for the time-step hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the correctness checker: it is
// loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
// leg, and nothing in the product links, loads or calls it.
//
// What it is: a pass-by-pass restatement, in C++, of the reference's WebGL2
// fragment shaders and of the order in which GPUSolver.step() and
// GPUSpray.step() run them. Each pass keeps the reference's texture layout
// (padded primitive texture, face-flux textures, 3-slot state ring, 2 step-
// info texels, 256x256 parcel textures) so the restatement can be read line
// by line against the GLSL; citations are source/solver.js and source/spray.js
// line numbers of the reference.
//
// Parity status: UNPINNED. The reference runs only as WebGL2 shaders, which
// cannot execute without a graphics stack, and it ships no golden vectors or
// known-answer tests for this path. This oracle is therefore checked against
// the reference by reading, and it is the source of the committed golden
// fixtures (tests/golden/, with their generator).
//
// Arithmetic: template<R> with R = float (the reference's highp FP32) or
// double (the FP64 run of the same scheme). Uniforms are rounded to R exactly
// as gl.uniform*fv rounds JavaScript doubles to float32. GLSL built-ins:
//   max/min -> fmax/fmin (IEEE maxNum, what the reference's GPUs execute),
//   clamp(x,a,b) = min(max(x,a),b), mix(x,y,a) = x*(1-a)+y*a,
//   smoothstep = Hermite t*t*(3-2t) of the clamped ramp, step(e,x) = x<e?0:1.
// Built with -ffp-contract=off so no multiply-add is fused.
// =============================================================================
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>
#include <type_traits>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "rn_oracle.h"

namespace {

constexpr int SPRAY_W = 256, SPRAY_H = 256, SPRAY_N = SPRAY_W * SPRAY_H;   // spray.js:16
constexpr int SPRAY_PER_STEP = 4;                                            // spray.js:17

template <typename R> struct v4 { R x, y, z, w; };
template <typename R> inline v4<R> V4(R x, R y, R z, R w) { return {x, y, z, w}; }

template <typename R> inline R gmax(R a, R b) { return std::fmax(a, b); }
template <typename R> inline R gmin(R a, R b) { return std::fmin(a, b); }
template <typename R> inline R gclamp(R x, R a, R b) { return gmin(gmax(x, a), b); }
template <typename R> inline R gmix(R x, R y, R a) { return x * (R(1) - a) + y * a; }
template <typename R> inline R gsmooth(R e0, R e1, R x) {
  R t = gclamp((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <typename R> inline R glen2(R a, R b) { return std::sqrt(a * a + b * b); }

// Prim: w = (rho, u, v, p), s = (Z, F, G, O)          solver.js:29
template <typename R> struct Prim { v4<R> w, s; };

constexpr float RHO_MIN_F = 1e-7f, P_MIN_F = 1e-7f;  // solver.js:27-28

// Uniform block after the float32 (or FP64) rounding a GL driver applies.
template <typename R> struct U {
  R amb[4], ambCons[4], ambB[4], gamR[2], inlet[4], res[3], gas[4], Rs[3], chemK[4], cap[2];
  R chamberNu[2], bar[3];
  R Tw, cfl, dtMax, wFloor, vMax, hllBlend, ramp, pStart, RcCells, limiter, inj, visc, chem;
  R mhat, tScale, fuel[4], ox[4], eF, eO, Ge, fan;
};

template <typename R> U<R> make_uniforms(const rno_params& p) {
  U<R> u;
  auto cp = [](R* d, const double* s, int n) { for (int k = 0; k < n; k++) d[k] = R(s[k]); };
  cp(u.amb, p.amb, 4); cp(u.ambCons, p.ambCons, 4); cp(u.ambB, p.ambB, 4); cp(u.gamR, p.gamR, 2);
  cp(u.inlet, p.inlet, 4); cp(u.res, p.res, 3); cp(u.gas, p.gas, 4); cp(u.Rs, p.Rs, 3);
  cp(u.chemK, p.chemK, 4); cp(u.cap, p.cap, 2); cp(u.chamberNu, p.chamberNu, 2);
  // uBar = (inlet[0], 1.6*uInlet0, max(ramp, 0)) is formed in JS doubles (solver.js:935)
  u.bar[0] = R(p.inlet[0]); u.bar[1] = R(1.6 * p.uInlet0); u.bar[2] = R(p.ramp > 0 ? p.ramp : 0.0);
  u.Tw = R(p.Tw); u.cfl = R(p.cfl); u.dtMax = R(p.dtMax); u.wFloor = R(p.wFloor); u.vMax = R(p.vMax);
  u.hllBlend = R(p.hllBlend); u.ramp = R(p.ramp); u.pStart = R(p.pStart); u.RcCells = R(p.RcCells);
  u.limiter = R(p.order2 ? 1 : 0); u.inj = R(p.inj ? 1 : 0); u.visc = R(p.visc ? 1 : 0); u.chem = R(p.chem ? 1 : 0);
  u.mhat = R(p.mhat); u.tScale = R(p.tScale); cp(u.fuel, p.fuelVec, 4); cp(u.ox, p.oxVec, 4);
  u.eF = R(p.eF); u.eO = R(p.eO); u.Ge = R(p.Ge);
  u.fan = R(25 * 3.14159265358979323846 / 180);   // spray.js:271
  return u;
}

template <typename R> struct Solver {
  int Nx = 0, Nr = 0;
  // 3-slot state ring (solver.js:766)
  std::vector<R> SA[3], SB[3];
  int cur = 0;
  // flux textures (Nx+1)x(Nr+1) (solver.js:767)
  std::vector<R> FxA, FxB, FxC, FrA, FrB, FrC;
  // padded primitive textures (Nx+4)x(Nr+4) (solver.js:770)
  std::vector<R> W, Wb;
  std::vector<R> T1, T2;       // viscous cell data (solver.js:772)
  R stepTex[2][4];             // (dt, t_old, t_new, w) ping-pong (solver.js:780)
  int stepIdx = 0;
  std::vector<uint8_t> mask;
  std::vector<R> geoA, geoG, geoM, jw, wallRow;
  // spray (spray.js:228-231)
  std::vector<R> PA[2], PB[2], PC[2], src, tab;
  int scur = 0;
  uint32_t head = 0, seed = 1;
  bool sprayReady = false;

  int W1() const { return Nx + 1; }
  int PW() const { return Nx + 4; }

  void resize(int nx, int nr) {
    Nx = nx; Nr = nr;
    size_t N = size_t(Nx) * Nr, NF = size_t(Nx + 1) * (Nr + 1), NP = size_t(Nx + 4) * (Nr + 4);
    for (int s = 0; s < 3; s++) { SA[s].assign(N * 4, R(0)); SB[s].assign(N * 4, R(0)); }
    for (auto* f : {&FxA, &FxB, &FxC, &FrA, &FrB, &FrC}) f->assign(NF * 4, R(0));
    W.assign(NP * 4, R(0)); Wb.assign(NP * 4, R(0));
    T1.assign(N * 4, R(0)); T2.assign(N * 4, R(0));
    std::memset(stepTex, 0, sizeof(stepTex));
    stepIdx = 0; cur = 0;
    mask.assign(N, 0);
    geoA.assign(NF * 4, R(0)); geoG.assign(N * 4, R(0)); geoM.assign(N * 4, R(0));
    jw.assign(size_t(Nx) * 4, R(0)); wallRow.assign(size_t(Nx) * 4, R(0));
    for (int k = 0; k < 2; k++) {
      PA[k].assign(size_t(SPRAY_N) * 4, R(0)); PB[k].assign(size_t(SPRAY_N) * 4, R(0)); PC[k].assign(size_t(SPRAY_N) * 4, R(0));
    }
    src.assign(N * 4, R(0)); tab.assign(256 * 3 * 4, R(0));
    sprayReady = true;
    spray_reset();
  }
  void spray_reset() {                                   // spray.js:242-254
    for (int p = 0; p < 2; p++) {
      std::fill(PA[p].begin(), PA[p].end(), R(0));
      for (int k = 0; k < SPRAY_N; k++) { PA[p][k * 4] = R(-1); PA[p][k * 4 + 1] = R(-1); }
      std::fill(PB[p].begin(), PB[p].end(), R(0));
      std::fill(PC[p].begin(), PC[p].end(), R(0));
    }
    head = 0;
  }

  // ---- texel access (texelFetch)
  v4<R> tex(const std::vector<R>& t, int width, int x, int y) const {
    const R* p = &t[(size_t(y) * width + x) * 4];
    return {p[0], p[1], p[2], p[3]};
  }
  void put(std::vector<R>& t, int width, int x, int y, v4<R> v) {
    R* p = &t[(size_t(y) * width + x) * 4];
    p[0] = v.x; p[1] = v.y; p[2] = v.z; p[3] = v.w;
  }
  bool solidAt(int i, int j) const { return mask[size_t(j) * Nx + i] != 0; }   // solver.js:31

  // solver.js:33-39
  static Prim<R> toPrim(v4<R> a, v4<R> b) {
    const R RHO_MIN = R(RHO_MIN_F), P_MIN = R(P_MIN_F);
    R rho = gmax(a.x, RHO_MIN);
    R vx = a.y / rho, vy = a.z / rho;
    R G = gmax(b.z, R(0.5));
    R p = gmax((a.w - R(0.5) * rho * (vx * vx + vy * vy)) / G, P_MIN);
    Prim<R> q;
    q.w = V4(rho, vx, vy, p);
    q.s = V4(gclamp(b.x / rho, R(0), R(1)), gclamp(b.y / rho, R(0), R(1)), G, gclamp(b.w / rho, R(0), R(1)));
    return q;
  }
  static R soundSpeed(const Prim<R>& q) { return std::sqrt((R(1) + R(1) / q.s.z) * q.w.w / q.w.x); }   // solver.js:40

  // ---------------------------------------------------------------------------
  // FS_PRIM (solver.js:56-126): padded primitive texture with ghost cells.
  void primPass(const std::vector<R>& A, const std::vector<R>& B, const R* st, int timeSel, const U<R>& u) {
    const int Pw = PW();
#pragma omp parallel for schedule(static)
    for (int py = 0; py < Nr + 4; py++) {
      for (int px = 0; px < Nx + 4; px++) {
        int i = px - 2, j = py - 2;
        bool mir = j < 0;
        if (mir) j = -j - 1;
        Prim<R> q;
        q.w = V4(u.amb[0], u.amb[1], u.amb[2], u.amb[3]);
        q.s = V4(R(0), R(0), u.inlet[3], R(0));
        bool wall = false;
        if (i < 0) {
          if (j < Nr && solidAt(0, j)) wall = true;
          else if (R(j) + R(0.5) < u.RcCells && u.inj > R(0.5)) wall = true;
          else if (R(j) + R(0.5) < u.RcCells) {
            R t = timeSel == 1 ? st[1] : st[2];
            R f = u.ramp > R(0) ? gsmooth(R(0), u.ramp, t) : R(1);
            R P0 = gmix(u.pStart, u.res[0], f);
            R T0 = u.res[1], Rg = u.res[2], G = u.inlet[2], g = R(1) + R(1) / G;
            v4<R> a = tex(A, Nx, 0, j);
            R ubar = gmax(tex(B, Nx, 0, j).w, R(0));
            R c0 = std::sqrt(g * Rg * T0);
            R ui = gclamp(a.y / gmax(a.x, R(RHO_MIN_F)), R(0), R(0.5) * c0);
            R ut = ubar * gsmooth(R(1), R(2), P0 / gmax(u.pStart, R(1e-6)));
            R uu = gmix(ui, ut, u.inlet[1]);
            R T = T0 - uu * uu * (g - R(1)) / (R(2) * g * Rg);
            R p = P0 * std::pow(T / T0, g * G);
            q.w = V4(p / (Rg * T), uu, R(0), p);
            q.s = V4(R(1), R(1), G, R(0));
          }
        } else if (j >= Nr) {
          int ci = std::min(i, Nx - 1), cj = Nr - 1;
          if (!solidAt(ci, cj)) {
            Prim<R> t = toPrim(tex(A, Nx, ci, cj), tex(B, Nx, ci, cj));
            R cs = soundSpeed(t);
            if (t.w.z >= cs) q = t;
            else if (t.w.z > R(0)) { q = t; q.w.w = u.amb[3]; }
          }
        } else if (i >= Nx) {
          int ci = Nx - 1, cj = j;
          if (!solidAt(ci, cj)) {
            Prim<R> t = toPrim(tex(A, Nx, ci, cj), tex(B, Nx, ci, cj));
            R cs = soundSpeed(t);
            if (t.w.y >= cs) q = t;
            else if (t.w.y > R(0)) { q = t; q.w.w = u.amb[3]; }
            else q.w.y = gmax(q.w.y, R(0));
          }
        } else {
          if (solidAt(i, j)) wall = true;
          else q = toPrim(tex(A, Nx, i, j), tex(B, Nx, i, j));
        }
        if (wall) {
          put(W, Pw, px, py, V4(R(-1), R(0), R(0), R(1)));
          put(Wb, Pw, px, py, V4(R(0), R(0), R(0), R(0)));
          continue;
        }
        if (mir) q.w.z = -q.w.z;
        put(W, Pw, px, py, q.w);
        put(Wb, Pw, px, py, q.s);
      }
    }
  }

  // ---------------------------------------------------------------------------
  // makeFluxShader (solver.js:133-259): MUSCL van Leer + HLLC/HLL per face.
  Prim<R> cellP(int i, int j, bool& s, bool dirR) const {
    Prim<R> q;
    q.w = tex(W, PW(), i + 2, j + 2);
    q.s = tex(Wb, PW(), i + 2, j + 2);
    s = q.w.x < R(0);
    if (dirR) std::swap(q.w.y, q.w.z);
    return q;
  }
  R pAt(int i, int j, R fb) const { v4<R> w = tex(W, PW(), i + 2, j + 2); return w.x < R(0) ? fb : w.w; }
  static Prim<R> mirrorN(Prim<R> q) { q.w.y = -q.w.y; return q; }
  static R vanLeer1(R a, R b) {
    R ab = a * b, den = a + b;
    den = gmix(den, R(1), (R(1e-30) < std::fabs(den)) ? R(0) : R(1));   // step(abs(den), 1e-30)
    return R(2) * gmax(ab, R(0)) / den;
  }
  static v4<R> vanLeer(v4<R> a, v4<R> b) {
    return V4(vanLeer1(a.x, b.x), vanLeer1(a.y, b.y), vanLeer1(a.z, b.z), vanLeer1(a.w, b.w));
  }
  static R jumpRatio(R a, R b) { return std::fabs(a - b) / gmin(a, b); }

  void fluxFace(int i, int j, bool dirR, const U<R>& u, v4<R>& oF, v4<R>& oFY, v4<R>& oFO) const {
    oF = oFY = oFO = V4(R(0), R(0), R(0), R(0));
    v4<R> geo = tex(geoA, W1(), i, j);
    R area;
    int dx_, dy_, tx, ty;
    if (dirR) {
      area = geo.w;
      if (j == 0 || area == R(0)) return;
      dx_ = 0; dy_ = 1; tx = 1; ty = 0;
    } else {
      area = geo.z;
      if (area == R(0)) return;
      dx_ = 1; dy_ = 0; tx = 0; ty = 1;
    }
    bool s0, s1, s2, s3;
    int k0x = i - 2 * dx_, k0y = j - 2 * dy_, k1x = i - dx_, k1y = j - dy_, k3x = i + dx_, k3y = j + dy_;
    Prim<R> c0 = cellP(k0x, k0y, s0, dirR), c1 = cellP(k1x, k1y, s1, dirR);
    Prim<R> c2 = cellP(i, j, s2, dirR), c3 = cellP(k3x, k3y, s3, dirR);
    if (s1 && s2) return;
    R hllw = R(0);
    if (u.hllBlend > R(0) && !(s1 || s2)) {
      R p1 = c1.w.w, p2 = c2.w.w;
      R jm = gmax(gmax(jumpRatio(pAt(k1x + tx, k1y + ty, p1), p1), jumpRatio(pAt(k1x - tx, k1y - ty, p1), p1)),
                  gmax(jumpRatio(pAt(i + tx, j + ty, p2), p2), jumpRatio(pAt(i - tx, j - ty, p2), p2)));
      hllw = gsmooth(R(0.15), R(0.6), jm * u.hllBlend);
    }
    Prim<R> WL, WR;
    if (s1) { WR = c2; WL = mirrorN(c2); }
    else if (s2) { WL = c1; WR = mirrorN(c1); }
    else {
      if (s0) c0 = mirrorN(c1);
      if (s3) c3 = mirrorN(c2);
      WL = c1; WR = c2;
      if (u.limiter > R(0.5) && area > R(0)) {
        auto sub = [](v4<R> a, v4<R> b) { return V4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); };
        v4<R> dL = vanLeer(sub(c1.w, c0.w), sub(c2.w, c1.w));
        v4<R> dR = vanLeer(sub(c2.w, c1.w), sub(c3.w, c2.w));
        v4<R> yL = vanLeer(sub(c1.s, c0.s), sub(c2.s, c1.s));
        v4<R> yR = vanLeer(sub(c2.s, c1.s), sub(c3.s, c2.s));
        v4<R> tL = V4(c1.w.x + R(0.5) * dL.x, c1.w.y + R(0.5) * dL.y, c1.w.z + R(0.5) * dL.z, c1.w.w + R(0.5) * dL.w);
        v4<R> tR = V4(c2.w.x - R(0.5) * dR.x, c2.w.y - R(0.5) * dR.y, c2.w.z - R(0.5) * dR.z, c2.w.w - R(0.5) * dR.w);
        if (tL.x > R(0) && tL.w > R(0) && tR.x > R(0) && tR.w > R(0)) {
          WL.w = tL;
          WL.s = V4(gclamp(c1.s.x + R(0.5) * yL.x, R(0), R(1)), gclamp(c1.s.y + R(0.5) * yL.y, R(0), R(1)),
                    gclamp(c1.s.z + R(0.5) * yL.z, R(0.5), R(100)), gclamp(c1.s.w + R(0.5) * yL.w, R(0), R(1)));
          WR.w = tR;
          WR.s = V4(gclamp(c2.s.x - R(0.5) * yR.x, R(0), R(1)), gclamp(c2.s.y - R(0.5) * yR.y, R(0), R(1)),
                    gclamp(c2.s.z - R(0.5) * yR.z, R(0.5), R(100)), gclamp(c2.s.w - R(0.5) * yR.w, R(0), R(1)));
        }
      }
    }
    // HLLC blended to HLL by hllw (solver.js:210-251)
    R GL = WL.s.z, GR = WR.s.z;
    R rL = WL.w.x, uL = WL.w.y, vL = WL.w.z, pL = WL.w.w;
    R rR = WR.w.x, uR = WR.w.y, vR = WR.w.z, pR = WR.w.w;
    R cL = std::sqrt((R(1) + R(1) / GL) * pL / rL), cR = std::sqrt((R(1) + R(1) / GR) * pR / rR);
    R EL = pL * GL + R(0.5) * rL * (uL * uL + vL * vL);
    R ER = pR * GR + R(0.5) * rR * (uR * uR + vR * vR);
    R sL = std::sqrt(rL), sR = std::sqrt(rR);
    R uT = (sL * uL + sR * uR) / (sL + sR);
    R HT = (sL * (EL + pL) / rL + sR * (ER + pR) / rR) / (sL + sR);
    R vT = (sL * vL + sR * vR) / (sL + sR);
    R GT = (sL * GL + sR * GR) / (sL + sR);
    R cT = std::sqrt(gmax((HT - R(0.5) * (uT * uT + vT * vT)) / GT, R(1e-12)));
    R SL = gmin(uL - cL, uT - cT);
    R SR = gmax(uR + cR, uT + cT);
    R FL[4] = {rL * uL, rL * uL * uL + pL, rL * uL * vL, uL * (EL + pL)};
    R FR[4] = {rR * uR, rR * uR * uR + pR, rR * uR * vR, uR * (ER + pR)};
    R YLs[3] = {WL.s.x, WL.s.y, WL.s.w}, YRs[3] = {WR.s.x, WR.s.y, WR.s.w};
    R FYL[3], FYR[3];
    for (int c = 0; c < 3; c++) { FYL[c] = rL * uL * YLs[c]; FYR[c] = rR * uR * YRs[c]; }
    R F[4], FY[3], uf, Gf;
    if (SL >= R(0)) { for (int c = 0; c < 4; c++) F[c] = FL[c]; for (int c = 0; c < 3; c++) FY[c] = FYL[c]; uf = uL; Gf = GL; }
    else if (SR <= R(0)) { for (int c = 0; c < 4; c++) F[c] = FR[c]; for (int c = 0; c < 3; c++) FY[c] = FYR[c]; uf = uR; Gf = GR; }
    else {
      R UL[4] = {rL, rL * uL, rL * vL, EL};
      R UR[4] = {rR, rR * uR, rR * vR, ER};
      R inv = R(1) / (SR - SL);
      R Fhll[4], FYhll[3];
      for (int c = 0; c < 4; c++) Fhll[c] = (SR * FL[c] - SL * FR[c] + SL * SR * (UR[c] - UL[c])) * inv;
      for (int c = 0; c < 3; c++) FYhll[c] = (SR * FYL[c] - SL * FYR[c] + SL * SR * (rR * YRs[c] - rL * YLs[c])) * inv;
      R Ss = (pR - pL + rL * uL * (SL - uL) - rR * uR * (SR - uR)) / (rL * (SL - uL) - rR * (SR - uR));
      bool left = Ss >= R(0);
      R rK = left ? rL : rR, uK = left ? uL : uR, vK = left ? vL : vR, pK = left ? pL : pR;
      R EK = left ? EL : ER, SK = left ? SL : SR;
      const R* YK = left ? YLs : YRs;
      const R* FYK = left ? FYL : FYR;
      const R* FK = left ? FL : FR;
      const R* UK = left ? UL : UR;
      R kk = rK * (SK - uK) / (SK - Ss);
      R Us[4] = {kk * R(1), kk * Ss, kk * vK, kk * (EK / rK + (Ss - uK) * (Ss + pK / (rK * (SK - uK))))};
      R Fc[4], FYc[3];
      for (int c = 0; c < 4; c++) Fc[c] = FK[c] + SK * (Us[c] - UK[c]);
      for (int c = 0; c < 3; c++) FYc[c] = FYK[c] + SK * (kk * YK[c] - rK * YK[c]);
      for (int c = 0; c < 4; c++) F[c] = gmix(Fc[c], Fhll[c], hllw);
      for (int c = 0; c < 3; c++) FY[c] = gmix(FYc[c], FYhll[c], hllw);
      uf = uK + SK * ((SK - uK) / (SK - Ss) - R(1));
      Gf = left ? GL : GR;
    }
    if (dirR) std::swap(F[1], F[2]);
    oF = V4(F[0], F[1], F[2], F[3]);
    oFY = V4(FY[0], FY[1], uf * Gf, uf);
    oFO = V4(FY[2], R(0), R(0), R(0));
  }

  void fluxPass(const U<R>& u) {
    const int w1 = W1();
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)                      // x-pass target (Nx+1) x Nr
      for (int i = 0; i <= Nx; i++) {
        v4<R> a, b, c;
        fluxFace(i, j, false, u, a, b, c);
        put(FxA, w1, i, j, a); put(FxB, w1, i, j, b); put(FxC, w1, i, j, c);
      }
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= Nr; j++)                     // r-pass target Nx x (Nr+1)
      for (int i = 0; i < Nx; i++) {
        v4<R> a, b, c;
        fluxFace(i, j, true, u, a, b, c);
        put(FrA, w1, i, j, a); put(FrB, w1, i, j, b); put(FrC, w1, i, j, c);
      }
  }

  // ---------------------------------------------------------------------------
  // FS_UPDATE (solver.js:264-363)
  static void sub4(v4<R>& L, R ae, v4<R> fe, R aw, v4<R> fw) {
    L.x -= ae * fe.x - aw * fw.x; L.y -= ae * fe.y - aw * fw.y;
    L.z -= ae * fe.z - aw * fw.z; L.w -= ae * fe.w - aw * fw.w;
  }
  void memberFlux(int cx, int cy, v4<R>& L, v4<R>& LY, R& LO, bool withO) const {
    const int w1 = W1();
    v4<R> g = tex(geoA, w1, cx, cy);
    R aw = std::fabs(g.z), ae = std::fabs(tex(geoA, w1, cx + 1, cy).z);
    R as_ = std::fabs(g.w), an = std::fabs(tex(geoA, w1, cx, cy + 1).w);
    sub4(L, ae, tex(FxA, w1, cx + 1, cy), aw, tex(FxA, w1, cx, cy));
    sub4(L, an, tex(FrA, w1, cx, cy + 1), as_, tex(FrA, w1, cx, cy));
    sub4(LY, ae, tex(FxB, w1, cx + 1, cy), aw, tex(FxB, w1, cx, cy));
    sub4(LY, an, tex(FrB, w1, cx, cy + 1), as_, tex(FrB, w1, cx, cy));
    if (withO) {
      LO -= ae * tex(FxC, w1, cx + 1, cy).x - aw * tex(FxC, w1, cx, cy).x;
      LO -= an * tex(FrC, w1, cx, cy + 1).x - as_ * tex(FrC, w1, cx, cy).x;
    }
  }
  static R wallPressure(const Prim<R>& q, R un) {
    R g = R(1) + R(1) / q.s.z, p = q.w.w, rho = q.w.x, c = std::sqrt(g * p / rho);
    if (un > R(0)) { R a = R(0.25) * (g + R(1)) * un; return p + rho * un * (a + std::sqrt(a * a + c * c)); }
    R f = gmax(R(1) + R(0.5) * (g - R(1)) * un / c, R(0));
    return p * std::pow(f, R(2) * g / (g - R(1)));
  }
  static int iround(R v) { return int(std::nearbyint(v)); }   // round() of exact integers

  void updatePass(int sIn, int s0, const R* st, int stage, int out, const U<R>& u) {
    const std::vector<R>& A_ = SA[sIn]; const std::vector<R>& B_ = SB[sIn];
    const std::vector<R>& A0_ = SA[s0]; const std::vector<R>& B0_ = SB[s0];
    std::vector<R>& oAv = SA[out]; std::vector<R>& oBv = SB[out];
    const R RHO_MIN = R(RHO_MIN_F), P_MIN = R(P_MIN_F);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        if (solidAt(i, j)) {
          put(oAv, Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(oBv, Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        v4<R> gm = tex(geoM, Nx, i, j);
        int Hx = i + iround(gm.x), Hy = j + iround(gm.y);
        v4<R> gg = tex(geoG, Nx, i, j);
        v4<R> A = tex(A_, Nx, Hx, Hy), B = tex(B_, Nx, Hx, Hy);
        Prim<R> q = toPrim(A, B);
        v4<R> L = V4(R(0), R(0), R(0), R(0)), LY = L;
        R LO = R(0);
        bool wO = u.inj > R(0.5);
        memberFlux(Hx, Hy, L, LY, LO, wO);
        int sm = iround(tex(geoM, Nx, Hx, Hy).z);
        if (sm & 1) memberFlux(Hx - 1, Hy, L, LY, LO, wO);
        if (sm & 2) memberFlux(Hx + 1, Hy, L, LY, LO, wO);
        if (sm & 4) memberFlux(Hx, Hy - 1, L, LY, LO, wO);
        if (sm & 8) memberFlux(Hx, Hy + 1, L, LY, LO, wO);
        R Wx = gg.z, Wr = gg.w;
        R wl = glen2(Wx, Wr);
        if (wl > R(1e-6)) {
          R nx = Wx / wl, nr = Wr / wl;
          R pw = wallPressure(q, q.w.y * nx + q.w.z * nr);
          L.y -= Wx * pw; L.z -= Wr * pw;
        }
        L.z += q.w.w * gg.y;
        R invV = R(1) / gmax(gg.x, R(1e-6));
        R dt = st[0];
        v4<R> LB = V4(LY.x, LY.y, LY.z - q.s.z * LY.w, LO);
        R f = dt * invV;
        v4<R> Uv, UY;
        if (stage == 1) {
          Uv = V4(A.x + f * L.x, A.y + f * L.y, A.z + f * L.z, A.w + f * L.w);
          UY = V4(B.x + f * LB.x, B.y + f * LB.y, B.z + f * LB.z, B.w + f * LB.w);
        } else {
          v4<R> A0 = tex(A0_, Nx, Hx, Hy), B0 = tex(B0_, Nx, Hx, Hy);
          Uv = V4(R(0.5) * (A0.x + A.x + f * L.x), R(0.5) * (A0.y + A.y + f * L.y),
                  R(0.5) * (A0.z + A.z + f * L.z), R(0.5) * (A0.w + A.w + f * L.w));
          UY = V4(R(0.5) * (B0.x + B.x + f * LB.x), R(0.5) * (B0.y + B.y + f * LB.y),
                  R(0.5) * (B0.z + B.z + f * LB.z), R(0.5) * (B0.w + B.w + f * LB.w));
        }
        R rho = gmax(Uv.x, RHO_MIN);
        R den = gmax(Uv.x, RHO_MIN);
        R vx = Uv.y / den, vy = Uv.z / den;
        R sp = glen2(vx, vy);
        if (sp > u.vMax) { R s = u.vMax / sp; vx *= s; vy *= s; }
        if (!(rho < R(1e30)) || !(vx < R(1e30) && vx > R(-1e30))) {
          put(oAv, Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(oBv, Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        R ke = R(0.5) * rho * (vx * vx + vy * vy);
        R Gn = gclamp(UY.z, u.gamR[0], u.gamR[1]);
        R E = gmax(Uv.w, P_MIN * Gn + ke);
        R Zn = gclamp(UY.x, R(0), rho);
        put(oAv, Nx, i, j, V4(rho, rho * vx, rho * vy, E));
        R ubar = R(0);
        if (u.inj > R(0.5)) ubar = gclamp(UY.w, R(0), rho);
        else if (i == 0) {
          R u0 = tex(B_, Nx, i, j).w;
          bool on = stage == 2 && st[2] > u.bar[2];
          ubar = on ? gmin(u0 + gmin(dt * u.bar[0], R(1)) * (vx - u0), u.bar[1]) : u0;
        }
        put(oBv, Nx, i, j, V4(Zn, gclamp(UY.y, R(0), Zn), Gn, ubar));
      }
  }

  // ---------------------------------------------------------------------------
  // FS_REDUCE1/FS_REDUCE2 + FS_STEPINFO (solver.js:368-411). The 4x4 block
  // tree is a max, which is exact and order-free, so one max over all cells.
  void cflPass(int s, const U<R>& u) {
    R wmax = R(0);
    const std::vector<R>& A_ = SA[s]; const std::vector<R>& B_ = SB[s];
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        if (solidAt(i, j)) continue;
        Prim<R> q = toPrim(tex(A_, Nx, i, j), tex(B_, Nx, i, j));
        wmax = gmax(wmax, std::fabs(q.w.y) + std::fabs(q.w.z) + R(2) * soundSpeed(q));
      }
    R w = gmax(u.wFloor, wmax);
    const R* prev = stepTex[stepIdx];
    R dt = gmin(u.cfl / w, u.dtMax);
    if (prev[0] > R(0)) dt = gmin(dt, prev[0] * R(1.2));
    R* o = stepTex[1 - stepIdx];
    R tn = prev[2];
    o[0] = dt; o[1] = tn; o[2] = tn + dt; o[3] = w;
    stepIdx = 1 - stepIdx;
  }

  // ---------------------------------------------------------------------------
  // FS_RESCALE (solver.js:418-437) + rescaleAmbient (998-1010)
  void rescale(R fp, R fT, R du, const U<R>& u) {
    int s0 = cur, s1 = (cur + 1) % 3;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        v4<R> A = tex(SA[s0], Nx, i, j), B = tex(SB[s0], Nx, i, j);
        if (solidAt(i, j)) {
          put(SA[s1], Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(SB[s1], Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        Prim<R> q = toPrim(A, B);
        R w = R(1) - gsmooth(R(0), R(0.03), q.s.x);
        R rho = q.w.x * gmix(R(1), fp / fT, w);
        R p = q.w.w * gmix(R(1), fp, w);
        R vx = q.w.y + du * w, vy = q.w.z + R(0);
        put(SA[s1], Nx, i, j, V4(rho, rho * vx, rho * vy, p * q.s.z + R(0.5) * rho * (vx * vx + vy * vy)));
        put(SB[s1], Nx, i, j, V4(rho * q.s.x, rho * q.s.y, q.s.z, B.w));
      }
    cur = s1;
  }

  // ---------------------------------------------------------------------------
  // GLSL_GAS (solver.js:445-450)
  static R sutherland(R TK, const U<R>& u) { return u.gas[3] * R(1.458e-6) * TK * std::sqrt(TK) / (TK + R(110.4)); }
  static R Rmix(v4<R> s, const U<R>& u) {
    return (R(1) - s.x) * u.gas[0] + s.y * u.Rs[0] + s.w * u.Rs[1] + gmax(s.x - s.y - s.w, R(0)) * u.Rs[2];
  }

  // FS_VCELL (solver.js:451-489)
  void vcellPass(const R* st, const U<R>& u) {
    const int Pw = PW();
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        int cx = i + 2, cy = j + 2;
        v4<R> w0 = tex(W, Pw, cx, cy);
        v4<R> z = V4(R(0), R(0), R(0), R(0));
        put(T1, Nx, i, j, z); put(T2, Nx, i, j, z);
        if (w0.x < R(0)) continue;
        v4<R> wE = tex(W, Pw, cx + 1, cy), wW = tex(W, Pw, cx - 1, cy);
        v4<R> wN = tex(W, Pw, cx, cy + 1), wS = tex(W, Pw, cx, cy - 1);
        R fE = wE.x < R(0) ? R(0) : R(1), fW = wW.x < R(0) ? R(0) : R(1);
        R fN = wN.x < R(0) ? R(0) : R(1), fS = wS.x < R(0) ? R(0) : R(1);
        R dxn = gmax(fE + fW, R(1)), drn = gmax(fN + fS, R(1));
        R gx0 = (fE * (wE.y - w0.y) + fW * (w0.y - wW.y)) / dxn;
        R gx1 = (fE * (wE.z - w0.z) + fW * (w0.z - wW.z)) / dxn;
        R gr0 = (fN * (wN.y - w0.y) + fS * (w0.y - wS.y)) / drn;
        R gr1 = (fN * (wN.z - w0.z) + fS * (w0.z - wS.z)) / drn;
        R ux = gx0, vx = gx1, ur = gr0, vr = gr1;
        R r = R(j) + R(0.5), vor = w0.z / r;
        R div = ux + vr + vor;
        R S2 = R(2) * (ux * ux + vr * vr + vor * vor) + (ur + vx) * (ur + vx) - R(0.6666667) * div * div;
        R om = vx - ur;
        R sens = om * om / (om * om + div * div + R(1e-8));
        R Smag = std::sqrt(gmax(S2, R(0))) * sens;
        v4<R> sc = tex(Wb, Pw, cx, cy);
        R rho = w0.x, p = w0.w;
        R Rm = Rmix(sc, u);
        R mu = sutherland(p / (rho * Rm) * u.gas[2], u);
        R l = tex(geoM, Nx, i, j).w;
        R dt = st[0];
        R mut = rho * l * l * Smag;
        if (R(i) < u.chamberNu[1]) mut = gmax(mut, rho * u.chamberNu[0]);
        put(T1, Nx, i, j, V4(ux, ur, vx, vr));
        put(T2, Nx, i, j, V4(gmin(mu + mut, R(0.08) * rho / gmax(dt, R(1e-9))), (sc.z + R(1)) * p / rho, Smag, mu));
      }
  }

  // makeViscFluxShader (solver.js:490-539)
  void vfluxFace(int i, int j, bool dirR, v4<R>& oF, v4<R>& oFY, v4<R>& oFO) const {
    const int Pw = PW();
    v4<R> z = V4(R(0), R(0), R(0), R(0));
    oF = oFY = oFO = z;
    v4<R> geo = tex(geoA, W1(), i, j);
    int k1x, k1y;
    if (dirR) {
      if (geo.w == R(0) || j == 0 || j >= Nr) return;
      k1x = i; k1y = j - 1;
    } else {
      if (geo.z == R(0) || i == 0 || i >= Nx) return;
      k1x = i - 1; k1y = j;
    }
    v4<R> w1 = tex(W, Pw, k1x + 2, k1y + 2), w2 = tex(W, Pw, i + 2, j + 2);
    if (w1.x < R(0) || w2.x < R(0)) return;
    v4<R> t1 = tex(T1, Nx, k1x, k1y), t2 = tex(T1, Nx, i, j);
    v4<R> m1 = tex(T2, Nx, k1x, k1y), m2 = tex(T2, Nx, i, j);
    v4<R> s1 = tex(Wb, Pw, k1x + 2, k1y + 2), s2 = tex(Wb, Pw, i + 2, j + 2);
    R mu = R(0.5) * (m1.x + m2.x);
    R uf = R(0.5) * (w1.y + w2.y), vf = R(0.5) * (w1.z + w2.z);
    v4<R> tt = V4(R(0.5) * (t1.x + t2.x), R(0.5) * (t1.y + t2.y), R(0.5) * (t1.z + t2.z), R(0.5) * (t1.w + t2.w));
    R r, ux, vx, ur, vr;
    if (dirR) { r = gmax(R(j), R(0.5)); ux = tt.x; vx = tt.z; ur = w2.y - w1.y; vr = w2.z - w1.z; }
    else { r = R(j) + R(0.5); ux = w2.y - w1.y; vx = w2.z - w1.z; ur = tt.y; vr = tt.w; }
    R div = ux + vr + vf / r;
    R txr = mu * (ur + vx);
    R k = mu * R(1.25);
    if (dirR) {
      R trr = mu * (R(2) * vr - R(0.6666667) * div);
      oF = V4(-k * (s2.w - s1.w), -txr, -trr, -(uf * txr + vf * trr) - k * (m2.y - m1.y));
    } else {
      R txx = mu * (R(2) * ux - R(0.6666667) * div);
      oF = V4(-k * (s2.w - s1.w), -txx, -txr, -(uf * txx + vf * txr) - k * (m2.y - m1.y));
    }
    oFY = V4(-k * (s2.x - s1.x), -k * (s2.y - s1.y), -k * (s2.z - s1.z), R(0));
  }
  void vfluxPass() {
    const int w1 = W1();
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i <= Nx; i++) {
        v4<R> a, b, c; vfluxFace(i, j, false, a, b, c);
        put(FxA, w1, i, j, a); put(FxB, w1, i, j, b); put(FxC, w1, i, j, c);
      }
#pragma omp parallel for schedule(static)
    for (int j = 0; j <= Nr; j++)
      for (int i = 0; i < Nx; i++) {
        v4<R> a, b, c; vfluxFace(i, j, true, a, b, c);
        put(FrA, w1, i, j, a); put(FrB, w1, i, j, b); put(FrC, w1, i, j, c);
      }
  }

  // FS_SOURCE (solver.js:540-663)
  void sourcePass(int sIn, const R* st, int out, const U<R>& u) {
    const std::vector<R>& A_ = SA[sIn]; const std::vector<R>& B_ = SB[sIn];
    std::vector<R>& oAv = SA[out]; std::vector<R>& oBv = SB[out];
    const R RHO_MIN = R(RHO_MIN_F), P_MIN = R(P_MIN_F);
    const int Pw = PW();
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        if (solidAt(i, j)) {
          put(oAv, Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(oBv, Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        v4<R> gmij = tex(geoM, Nx, i, j);
        int Hx = i + iround(gmij.x), Hy = j + iround(gmij.y);
        v4<R> gg = tex(geoG, Nx, i, j);
        v4<R> A = tex(A_, Nx, Hx, Hy), B = tex(B_, Nx, Hx, Hy);
        Prim<R> q = toPrim(A, B);
        R rho = q.w.x, p = q.w.w, G = q.s.z;
        R velx = q.w.y, vely = q.w.z;
        R dt = st[0];
        R V = gmax(gg.x, R(1e-6));
        R Rm = Rmix(q.s, u), Tg = p / (rho * Rm);
        v4<R> L = V4(R(0), R(0), R(0), R(0)), LY = L;
        R dummy = R(0);
        v4<R> T1h = tex(T1, Nx, Hx, Hy), T2h = tex(T2, Nx, Hx, Hy);
        if (u.visc > R(0.5)) {
          memberFlux(Hx, Hy, L, LY, dummy, false);
          int sm = iround(tex(geoM, Nx, Hx, Hy).z);
          if (sm & 1) memberFlux(Hx - 1, Hy, L, LY, dummy, false);
          if (sm & 2) memberFlux(Hx + 1, Hy, L, LY, dummy, false);
          if (sm & 4) memberFlux(Hx, Hy - 1, L, LY, dummy, false);
          if (sm & 8) memberFlux(Hx, Hy + 1, L, LY, dummy, false);
          R r = V / gmax(gg.y, R(1e-6)), vor = vely / r;
          L.z -= T2h.x * (R(2) * vor - R(0.6666667) * (T1h.x + T1h.w + vor)) * gg.y;
          R wl = glen2(gg.z, gg.w);
          if (wl > R(1e-6)) {
            R nx = gg.z / wl, nr = gg.w / wl;
            R dn = velx * nx + vely * nr;
            R utx = velx - dn * nx, uty = vely - dn * nr;
            R up = glen2(utx, uty);
            R cp = Rm * (G + R(1));
            R Taw = Tg + R(0.89) * up * up / (R(2) * cp);
            R Ts = gmax(Tg + R(0.5) * (u.Tw - Tg) + R(0.22) * (Taw - Tg), R(1e-3));
            R rs = p / (Rm * Ts), mus = sutherland(Ts * u.gas[2], u);
            R dz = R(2) * gclamp(R(0.5) * V / wl, R(0.25), R(1));
            R nz = mus / (rs * dz);
            R tw = up <= R(69.7) * nz ? R(2) * mus * up / dz
                                      : rs * std::pow(R(7.187) * std::pow(nz, R(1.142857)) + R(0.13769) * std::pow(nz, R(0.142857)) * up, R(1.75));
            tw = gmin(tw, R(0.3) * rho * up * V / gmax(wl * dt, R(1e-9)));
            if (up > R(1e-6)) { L.y -= tw * wl * utx / up; L.z -= tw * wl * uty / up; }
            R qw = tw / gmax(up, R(1e-4)) * cp * (Taw - u.Tw) * R(1.24);
            R qmax = R(0.3) * p * G * V / gmax(wl * dt, R(1e-9));
            L.w -= gclamp(qw, -qmax, qmax) * wl;
          }
          if (sm & 16) {
            R up = glen2(velx, vely), Mn = up / std::sqrt((R(1) + R(1) / G) * p / rho);
            if (Mn > R(1)) {
              R shx = velx / up, shy = vely / up;
              R pd = R(0);
              for (int n = 4; n <= 6; n += 2)
                for (int m = 0; m <= 1; m++) {
                  int Dx = Hx + int(std::nearbyint(R(n) * shx));
                  int Dy = Hy + int(std::floor(R(n) * shy)) + m;
                  Dx = std::min(std::max(Dx, 0), Nx - 1); Dy = std::min(std::max(Dy, 0), Nr - 1);
                  v4<R> wd = tex(W, Pw, Dx + 2, Dy + 2);
                  if (wd.x > R(0)) pd = gmax(pd, wd.w);
                }
              R crit = R(1) + R(0.5) * Mn;
              R f = gsmooth(crit, R(1.2) * crit, pd / p) * V * rho * up;
              L.y -= f * velx; L.z -= f * vely;
            } else if (velx > R(0) && p < R(1.3) * u.chemK[3]) {
              R f = R(0.5) * V * rho * up;
              L.y -= f * velx; L.z -= f * vely;
            }
          }
        }
        R invV = dt / V;
        R dO = invV * L.x;
        L.x = R(0);
        v4<R> Uv = V4(A.x + invV * L.x, A.y + invV * L.y, A.z + invV * L.z, A.w + invV * L.w);
        v4<R> UY = V4(B.x + invV * LY.x / R(1), B.y + invV * LY.y / R(1), B.z + invV * LY.z / rho, B.w + invV * R(0) / R(1));
        if (u.inj > R(0.5)) UY.w += dO;
        if (u.chem > R(0.5)) {
          R Z = q.s.x, F = q.s.y, O = q.s.w, s = u.chemK[1];
          R avail = u.inj > R(0.5) ? gmin(F, (O + R(0.233) * gmax(R(1) - Z, R(0))) / s)
                                   : gmin(F, gmax(R(1) - Z - s * (Z - F), R(0)) / s);
          if (avail > R(1e-5)) {
            R TK = Tg * u.gas[2];
            R kin = u.chemK[2] * p * std::exp(R(-9000) / TK) * (R(1) - gsmooth(u.cap[0], u.cap[1], TK));
            R mixr = u.inj > R(0.5) ? gmax(T2h.z, R(4) * T2h.x / rho) : T2h.z;
            R burn = avail * gmin(gmin(mixr, kin) * dt, R(0.5));
            UY.y -= rho * burn;
            if (u.inj > R(0.5)) UY.w = gmax(UY.w - rho * burn * s, R(0));
            Uv.w += rho * burn * u.chemK[0];
          }
        }
        R rn = gmax(Uv.x, RHO_MIN);
        R vnx = Uv.y / rn, vny = Uv.z / rn;
        if (!(rn < R(1e30)) || !(vnx < R(1e30) && vnx > R(-1e30))) {
          put(oAv, Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(oBv, Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        R Gn = gclamp(UY.z, u.gamR[0], u.gamR[1]);
        R Zn = gclamp(UY.x, R(0), rn);
        put(oAv, Nx, i, j, V4(rn, rn * vnx, rn * vny, gmax(Uv.w, P_MIN * Gn + R(0.5) * rn * (vnx * vnx + vny * vny))));
        put(oBv, Nx, i, j, V4(Zn, gclamp(UY.y, R(0), Zn), Gn, u.inj > R(0.5) ? gclamp(UY.w, R(0), rn) : tex(B_, Nx, i, j).w));
      }
  }

  // FS_WALLROW (solver.js:665-674) + drawWallRow (986-996)
  void drawWallRow() {
    for (int i = 0; i < Nx; i++) {
      int cj = int(tex(jw, Nx, i, 0).x);
      Prim<R> q = toPrim(tex(SA[cur], Nx, i, cj), tex(SB[cur], Nx, i, cj));
      put(wallRow, Nx, i, 0, V4(q.w.y, q.w.z, q.w.w, soundSpeed(q)));
    }
  }

  // ---------------------------------------------------------------------------
  // Spray (spray.js:19-179, step 256-297)
  static uint32_t pcg(uint32_t v) {                                     // spray.js:33
    uint32_t s = v * 747796405u + 2891336453u;
    uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
    return (w >> 22u) ^ w;
  }
  static R rnd(uint32_t a, uint32_t n) { return R(float(pcg(a + n * 7919u) & 0xffffffu)) / R(16777216.0); }   // spray.js:34
  bool wallAt(R x, R y) const {                                          // spray.js:35-39
    int cx = int(std::floor(x)), cy = int(std::floor(y));
    if (cx < 0 || cy < 0 || cx >= Nx || cy >= Nr) return false;
    return tex(W, PW(), cx + 2, cy + 2).x < R(0);
  }
  void sprayUpdate(int from, int to, const R* st, const U<R>& u) {
    const int Pw = PW();
    const R dt = st[0];
#pragma omp parallel for schedule(static)
    for (int idx = 0; idx < SPRAY_N; idx++) {
      v4<R> a = tex(PA[from], SPRAY_W, idx % SPRAY_W, idx / SPRAY_W), b = tex(PB[from], SPRAY_W, idx % SPRAY_W, idx / SPRAY_W);
      int rel = idx - int(head);
      if (rel < 0) rel += SPRAY_N;
      v4<R> oA, oB, oC;
      if (rel < SPRAY_PER_STEP) {
        uint32_t id = uint32_t(idx) ^ (seed * 2654435761u);
        int t = int(rnd(id, 1u) * R(255.999));
        v4<R> e1 = tex(tab, 256, t, 0), e2 = tex(tab, 256, t, 1), e3 = tex(tab, 256, t, 2);
        R ang = e1.z + (rnd(id, 2u) - R(0.5)) * R(2) * e2.z;
        R r = gmax(e1.y + (rnd(id, 3u) - R(0.5)) * e2.w, R(0.05));
        R d = e2.y * std::exp((rnd(id, 4u) - R(0.5)) * R(1.4));
        oA = V4(e1.x, r, e1.w * std::cos(ang), e1.w * std::sin(ang));
        oB = V4(d, u.mhat * dt / R(SPRAY_PER_STEP), e2.x, e3.x);
        oC = b.y > R(0) ? V4(b.y, b.y * a.z, b.y * a.w, R(0)) : V4(R(0), R(0), R(0), R(0));
      } else {
        oA = a; oB = b; oC = V4(R(0), R(0), R(0), R(0));
        if (b.y > R(0)) sprayMove(idx, a, b, dt, u, Pw, oA, oB, oC);
      }
      put(PA[to], SPRAY_W, idx % SPRAY_W, idx / SPRAY_W, oA);
      put(PB[to], SPRAY_W, idx % SPRAY_W, idx / SPRAY_W, oB);
      put(PC[to], SPRAY_W, idx % SPRAY_W, idx / SPRAY_W, oC);
    }
  }
  void sprayMove(int idx, v4<R> a, v4<R> b, R dt, const U<R>& u, int Pw, v4<R>& oA, v4<R>& oB, v4<R>& oC) const {
    int gx = std::min(std::max(int(std::floor(a.x)), 0), Nx - 1);
    int gy = std::min(std::max(int(std::floor(a.y)), 0), Nr - 1);
    v4<R> w = tex(W, Pw, gx + 2, gy + 2);
    if (w.x < R(0)) { oA = V4(a.x + R(1), gmax(a.y - R(0.5), R(0.05)), gmax(a.z, R(0)), a.w); return; }
    const R* pr = b.z < R(0.5) ? u.fuel : u.ox;
    R vx = a.z, vy = a.w;
    R m = b.y, d = b.x, dts = dt * u.tScale;
    R dn = d, mn = m;
    if (w.x > R(0)) {
      v4<R> s = tex(Wb, Pw, gx + 2, gy + 2);
      R rm = (R(1) - s.x) * u.gas[0] + s.y * u.Rs[0] + s.w * u.Rs[1] + gmax(s.x - s.y - s.w, R(0)) * u.Rs[2];
      R T = w.w / (w.x * rm) * u.gas[2];
      R rhoG = w.x * R(1.225), Urel = glen2(w.y - vx, w.z - vy) * R(287.6) + R(1e-3);
      R mu = R(1.458e-6) * T * std::sqrt(T) / (T + R(110.4));
      R Re = rhoG * Urel * d / mu;
      R invTau = R(18) * mu * (R(1) + R(0.15) * std::pow(gmin(Re, R(1000)), R(0.687))) / (pr[0] * d * d);
      R e = std::exp(-dts * invTau);
      vx = w.y + (vx - w.y) * e; vy = w.z + (vy - w.z) * e;
      R cp = rm * R(287.05) * (s.z + R(1));
      R Bs = gmax(cp * (T - pr[1]), R(0)) / pr[2];
      R K = R(8) * (mu / R(0.7)) / pr[0] * std::log(R(1) + Bs) * (R(1) + R(0.27) * std::sqrt(Re));
      R d2 = d * d - K * dts;
      dn = d2 > R(1e-12) ? std::sqrt(d2) : R(0);
      R f = dn / d;
      mn = dn > R(0) ? m * f * f * f : R(0);
      R we = rhoG * Urel * Urel * dn / pr[3];
      if (we > R(12) && dn > R(0)) {
        R dst = R(12) * pr[3] / (rhoG * Urel * Urel);
        R tb = R(3) * dn / Urel * std::sqrt(pr[0] / rhoG);
        dn = gmix(dn, gmax(dst, R(2e-6)), R(1) - std::exp(-dts / tb));
      }
    }
    R xi = b.w;
    if (xi > R(0) && a.x >= xi) {
      uint32_t id = uint32_t(idx) ^ (seed * 2654435761u);
      R sp = glen2(vx, vy), phi = (rnd(id, 5u) - R(0.5)) * R(2) * u.fan;
      vx = sp * std::cos(phi); vy = sp * std::sin(phi);
      dn *= R(0.25); xi = R(0);
    }
    R x = a.x + vx * dt, y = a.y + vy * dt;
    if (y < R(0)) { y = -y; vy = -vy; }
    if (x < R(0)) { x = -x; vx = std::fabs(vx) * R(0.3); }
    if (wallAt(x, y)) {
      bool hx = wallAt(x, a.y), hr = wallAt(a.x, y);
      if (hx) { vx *= R(-0.3); x = a.x; }
      if (hr) { vy *= R(-0.3); y = a.y; }
      if (!hx && !hr) { x = a.x; y = a.y; vx *= R(-0.3); vy *= R(-0.3); }
    }
    R dm = m - mn;
    R dpx = mn * (a.z - vx) + dm * a.z, dpy = mn * (a.w - vy) + dm * a.w;
    oC = V4(dm, dpx, dpy, R(0));
    if (x >= R(Nx) || y >= R(Nr) || mn <= R(0)) {
      oA = V4(R(-1), R(-1), R(0), R(0));
      oB = V4(R(0), R(0), R(0), R(0));
      return;
    }
    oA = V4(x, y, vx, vy);
    oB = V4(dn, mn, b.z, xi);
  }
  // VS_SPRAY_DEP/FS_SPRAY_DEP with ONE,ONE blending (spray.js:125-149, 274-285).
  // GL blends fragments of one pixel in primitive (vertex-id) order, so the
  // sum runs sequentially in parcel-index order.
  void sprayDeposit(int from, int to) {
    std::fill(src.begin(), src.end(), R(0));
    for (int t = 0; t < SPRAY_N; t++) {
      v4<R> a = tex(PA[from], SPRAY_W, t % SPRAY_W, t / SPRAY_W), c = tex(PC[to], SPRAY_W, t % SPRAY_W, t / SPRAY_W);
      if (a.x < R(0) || (c.x == R(0) && c.y == R(0) && c.z == R(0))) continue;
      R type = tex(PB[from], SPRAY_W, t % SPRAY_W, t / SPRAY_W).z;
      int gx = std::min(std::max(int(std::floor(a.x)), 0), Nx - 1);
      int gy = std::min(std::max(int(std::floor(a.y)), 0), Nr - 1);
      v4<R> gm = tex(geoM, Nx, gx, gy);
      gx += iround(gm.x); gy += iround(gm.y);
      R* p = &src[(size_t(gy) * Nx + gx) * 4];
      p[0] = c.x * (R(1) - type) + p[0];
      p[1] = c.x * type + p[1];
      p[2] = c.y + p[2];
      p[3] = c.z + p[3];
    }
  }
  // FS_SPRAY_APPLY (spray.js:150-179)
  void sprayApply(int sIn, int out, const U<R>& u) {
    const std::vector<R>& A_ = SA[sIn]; const std::vector<R>& B_ = SB[sIn];
    std::vector<R>& oAv = SA[out]; std::vector<R>& oBv = SB[out];
    const R RHO_MIN = R(RHO_MIN_F), P_MIN = R(P_MIN_F);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < Nr; j++)
      for (int i = 0; i < Nx; i++) {
        if (solidAt(i, j)) {
          put(oAv, Nx, i, j, V4(u.ambCons[0], u.ambCons[1], u.ambCons[2], u.ambCons[3]));
          put(oBv, Nx, i, j, V4(u.ambB[0], u.ambB[1], u.ambB[2], u.ambB[3]));
          continue;
        }
        v4<R> gm = tex(geoM, Nx, i, j);
        int Hx = i + iround(gm.x), Hy = j + iround(gm.y);
        v4<R> s = tex(src, Nx, Hx, Hy);
        v4<R> A = tex(A_, Nx, Hx, Hy), B = tex(B_, Nx, Hx, Hy);
        R invV = R(1) / gmax(tex(geoG, Nx, i, j).x, R(1e-6));
        R dm = s.x + s.y;
        if (dm == R(0) && s.z == R(0) && s.w == R(0)) { put(oAv, Nx, i, j, A); put(oBv, Nx, i, j, B); continue; }
        R den = gmax(A.x, RHO_MIN);
        R velx = A.y / den, vely = A.z / den;
        R rn = A.x + dm * invV;
        R momx = A.y + s.z * invV, momy = A.z + s.w * invV;
        R E = A.w + (s.x * u.eF + s.y * u.eO + (velx * s.z + vely * s.w)) * invV;
        R phi = gmin(dm * invV / rn, R(1));
        R Gn = gmix(B.z, u.Ge, phi);
        R vnx = momx / rn, vny = momy / rn;
        E = gmax(E, R(0.02) * A.w + R(0.5) * rn * (vnx * vnx + vny * vny) + P_MIN * Gn);
        put(oAv, Nx, i, j, V4(rn, momx, momy, E));
        put(oBv, Nx, i, j, V4(B.x + dm * invV, B.y + s.x * invV, Gn, B.w + s.y * invV));
      }
  }

  // ---------------------------------------------------------------------------
  // GPUSolver.step (solver.js:849-891) + GPUSpray.step (spray.js:256-297)
  void step(int n, const U<R>& u) {
    for (int k = 0; k < n; k++) {
      int s0 = cur, s1 = (cur + 1) % 3, s2 = (cur + 2) % 3;
      cflPass(s0, u);
      const R* st = stepTex[stepIdx];
      primPass(SA[s0], SB[s0], st, 1, u);
      fluxPass(u);
      updatePass(s0, s0, st, 1, s1, u);
      primPass(SA[s1], SB[s1], st, 2, u);
      fluxPass(u);
      updatePass(s1, s0, st, 2, s2, u);
      cur = (cur + 2) % 3;
      if (u.visc > R(0.5) || u.chem > R(0.5)) {
        int out = (cur + 1) % 3;
        vcellPass(st, u);
        if (u.visc > R(0.5)) vfluxPass();
        sourcePass(cur, st, out, u);
        cur = out;
      }
      if (u.inj > R(0.5)) {
        int out = (cur + 1) % 3;
        int from = scur, to = 1 - scur;
        sprayUpdate(from, to, st, u);
        sprayDeposit(from, to);
        sprayApply(cur, out, u);
        cur = out;
        scur = 1 - scur;
        head = (head + SPRAY_PER_STEP) % SPRAY_N;
        seed = seed + 1u;
      }
    }
  }
};

struct Handle {
  int fp64 = 0;
  Solver<float> f;
  Solver<double> d;
};

template <typename R> void load_state(Solver<R>& s, const float* A, const float* B) {
  size_t n = size_t(s.Nx) * s.Nr * 4;
  for (int k = 0; k < 3; k++)
    for (size_t q = 0; q < n; q++) { s.SA[k][q] = R(A[q]); s.SB[k][q] = R(B[q]); }
  std::memset(s.stepTex, 0, sizeof(s.stepTex));
  s.cur = 0; s.stepIdx = 0;
  s.spray_reset();
}
template <typename R> void load_geo(Solver<R>& s, const uint8_t* mask, const float* geoA, const float* geoG,
                                    const float* geoM, const float* jWall) {
  size_t N = size_t(s.Nx) * s.Nr, NF = size_t(s.Nx + 1) * (s.Nr + 1);
  for (size_t k = 0; k < N; k++) s.mask[k] = mask[k] ? 1 : 0;
  for (size_t q = 0; q < NF * 4; q++) s.geoA[q] = R(geoA[q]);
  for (size_t q = 0; q < N * 4; q++) { s.geoG[q] = R(geoG[q]); s.geoM[q] = R(geoM[q]); }
  if (jWall) for (size_t q = 0; q < size_t(s.Nx) * 4; q++) s.jw[q] = R(jWall[q]);
}
template <typename R, typename T> void copy_out(const std::vector<R>& v, T* out) {
  for (size_t q = 0; q < v.size(); q++) out[q] = T(v[q]);
}

}  // namespace

extern "C" {

void* rno_create(int Nx, int Nr, int fp64) {
  Handle* h = new Handle();
  h->fp64 = fp64;
  if (fp64) h->d.resize(Nx, Nr); else h->f.resize(Nx, Nr);
  return h;
}
void rno_destroy(void* hp) { delete static_cast<Handle*>(hp); }

void rno_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

void rno_set_geometry(void* hp, const uint8_t* mask, const float* geoA, const float* geoG, const float* geoM,
                      const float* jWall) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) load_geo(h->d, mask, geoA, geoG, geoM, jWall); else load_geo(h->f, mask, geoA, geoG, geoM, jWall);
}
void rno_set_state(void* hp, const float* A, const float* B) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) load_state(h->d, A, B); else load_state(h->f, A, B);
}
void rno_set_injector(void* hp, const float* tab) {
  Handle* h = static_cast<Handle*>(hp);
  for (int q = 0; q < 256 * 3 * 4; q++) { if (h->fp64) h->d.tab[q] = tab[q]; else h->f.tab[q] = tab[q]; }
}
// a pre-populated parcel ring: PA, PB (65536 x 4 each) into the current slot, PC cleared, ring head
void rno_set_parcels(void* hp, const float* PA, const float* PB, int head) {
  Handle* h = static_cast<Handle*>(hp);
  auto set = [&](auto& s) {
    using R = typename std::decay_t<decltype(s.PA[0])>::value_type;
    for (int q = 0; q < SPRAY_N * 4; q++) {
      s.PA[s.scur][q] = R(PA[q]);
      s.PB[s.scur][q] = R(PB[q]);
      s.PC[s.scur][q] = R(0);
    }
    s.head = uint32_t(((head % SPRAY_N) + SPRAY_N) % SPRAY_N);
  };
  if (h->fp64) set(h->d); else set(h->f);
}
void rno_step(void* hp, int n, const rno_params* p) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) h->d.step(n, make_uniforms<double>(*p)); else h->f.step(n, make_uniforms<float>(*p));
}
void rno_rescale_ambient(void* hp, double fp, double fT, double du, const rno_params* p) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) h->d.rescale(fp, fT, du, make_uniforms<double>(*p));
  else h->f.rescale(float(fp), float(fT), float(du), make_uniforms<float>(*p));
}
// state of the current slot, as double (exact for the FP32 oracle)
void rno_get_state(void* hp, double* A, double* B) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) { copy_out(h->d.SA[h->d.cur], A); copy_out(h->d.SB[h->d.cur], B); }
  else { copy_out(h->f.SA[h->f.cur], A); copy_out(h->f.SB[h->f.cur], B); }
}
void rno_get_step_info(void* hp, double* out4) {
  Handle* h = static_cast<Handle*>(hp);
  for (int c = 0; c < 4; c++) out4[c] = h->fp64 ? h->d.stepTex[h->d.stepIdx][c] : h->f.stepTex[h->f.stepIdx][c];
}
void rno_get_wall_row(void* hp, double* out) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) { h->d.drawWallRow(); copy_out(h->d.wallRow, out); } else { h->f.drawWallRow(); copy_out(h->f.wallRow, out); }
}
// the split step's cell data T2 of the last physics pass (solver.js:458-488), N x 4
void rno_get_t2(void* hp, double* out) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) copy_out(h->d.T2, out); else copy_out(h->f.T2, out);
}
// parcels of the current parcel slot: PA, PB (each 65536 x 4) and PC of that slot
void rno_get_parcels(void* hp, double* PA, double* PB, double* PC) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) { copy_out(h->d.PA[h->d.scur], PA); copy_out(h->d.PB[h->d.scur], PB); copy_out(h->d.PC[h->d.scur], PC); }
  else { copy_out(h->f.PA[h->f.scur], PA); copy_out(h->f.PB[h->f.scur], PB); copy_out(h->f.PC[h->f.scur], PC); }
}
void rno_get_spray_counters(void* hp, uint32_t* head_seed) {
  Handle* h = static_cast<Handle*>(hp);
  head_seed[0] = h->fp64 ? h->d.head : h->f.head;
  head_seed[1] = h->fp64 ? h->d.seed : h->f.seed;
}
// the deposit texture of the last spray step (N x 4)
void rno_get_src(void* hp, double* out) {
  Handle* h = static_cast<Handle*>(hp);
  if (h->fp64) copy_out(h->d.src, out); else copy_out(h->f.src, out);
}

}  // extern "C"
