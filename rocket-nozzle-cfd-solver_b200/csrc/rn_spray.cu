// rn_spray.cu -- spray parcel step with two-way coupling, sm_100a.
//
// k_parcels: one thread per parcel of the 65,536-slot ring (FS_SPRAY_UPDATE,
//   spray.js:19-122): ring spawn from the injector table with the PCG hash,
//   Schiller-Naumann drag, d^2-law evaporation with the Ranz-Marshall factor,
//   We > 12 break-up, impingement fan, wall bounce. It also emits each
//   parcel's deposit record (host-cell key, source vector), i.e. the vertex
//   stage of VS_SPRAY_DEP (spray.js:125-143).
// Deposit: the reference point-sprites every parcel into its cell with ONE,ONE
//   float blending (spray.js:274-285); GL blends the fragments of one pixel in
//   primitive order, so each cell's source is the float sum in parcel-index
//   order. Here the records are sorted by cell with a stable radix sort
//   (parcel index order survives inside a cell) and each cell's run is summed
//   sequentially by one thread: the same order, deterministic, no float atomics.
// k_apply: FS_SPRAY_APPLY (spray.js:150-179) per cell, with the step's CFL
//   epilogue when it is the step's last kernel.
// Fast variant: the deposits go instead into 64-bit fixed-point sums per cell
//   (integer atomics, so the sums do not depend on the order the parcels
//   arrive in: deterministic, with no sort). A component is quantised in
//   steps of 2^-40 of a bound no deposit reaches, after the float product
//   x * 2^40 / bound, so each deposit keeps float precision and the sums hold
//   up to 2^22 bounds. The bounds follow the ring: every parcel step folds the
//   largest mass and speed of the parcels it writes (and the bounds it read)
//   into the next step's pair, so a deposit never exceeds its step's bounds:
//   mass: max(that mass, mhat dtMax / 4), the spawn mass at the largest step;
//   momentum: the mass bound times 4 max(that speed, vMax). A parcel's deposit
//   is at most its mass (evaporated or recycled) and its momentum change at
//   most m (2 |v_old| + |v_new|), with |v_new| <= max(|v_old|, gas speed) and
//   the gas speed of the stage-1 state it reads at most vMax. A deposit beyond
//   64 bounds (only a NaN can reach it) is flagged on the device and reported
//   by rn_spray_stats and rn_sync. The exact variant keeps the sort and the
//   float sum in parcel-index order (and tracks the bounds too, so a handle
//   can switch precision between steps).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include "rn_kernels.cuh"

namespace rn {
namespace RN_VARIANT {

constexpr int SPRAY_N = 65536, SPRAY_PER_STEP = 4;   // 256 x 256 ring, 4 born per step (spray.js:16-17)

// pcg / rnd (spray.js:33-34): 32-bit integer hash, bit-exact with the shader
__device__ __forceinline__ uint32_t pcg(uint32_t v) {
  uint32_t s = v * 747796405u + 2891336453u;
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
__device__ __forceinline__ float rnd(uint32_t a, uint32_t n) {
  return float(pcg(a + n * 7919u) & 0xffffffu) / 16777216.0f;
}
__device__ __forceinline__ bool wall_at(const Grid& g, const float4* A1, const float4* B1, float x, float y) {
  int cx = int(floorf(x)), cy = int(floorf(y));
  if (cx < 0 || cy < 0 || cx >= g.Nx || cy >= g.Nr) return false;
  return g.mask[cy * g.Nx + cx] != 0;          // padded W.x < 0 exactly at solid cells
}

// Fixed-point scales of the deposit sums (fast variant): 2^40 / bound, from
// the step's (mass, speed) bounds b (float bits; 0 for an empty ring).
__device__ __forceinline__ float dep_bound_mass(const rn_params& P, const unsigned* b) {
  return fmaxf(P.mhat * P.dtMax * 0.25f, __uint_as_float(b[0]));
}
__device__ __forceinline__ float dep_scale_mass(const rn_params& P, const unsigned* b) {
  return ldexpf(1.0f / fmaxf(dep_bound_mass(P, b), 1e-30f), 40);
}
__device__ __forceinline__ float dep_scale_mom(const rn_params& P, const unsigned* b) {
  return ldexpf(1.0f / fmaxf(dep_bound_mass(P, b) * 4.0f * fmaxf(fmaxf(P.vMax, __uint_as_float(b[1])), 1.0f), 1e-30f),
                40);
}
// |x * scale| stays below 2^46 (64 bounds) or is clamped there and flagged:
// 65,536 deposits of that size still sum within the 63 bits.
__device__ __forceinline__ unsigned long long to_fixed(float x, float scale, bool& over) {
  constexpr float LIM = 70368744177664.0f;   // 2^46
  float y = x * scale;
  if (!(fabsf(y) < LIM)) {
    over = true;
    y = y < 0.0f ? -LIM : (y > 0.0f ? LIM : 0.0f);   // NaN -> 0
  }
  return (unsigned long long)__float2ll_rn(y);
}
__device__ __forceinline__ float from_fixed(unsigned long long v, float scale) {
  return float(double((long long)v) / double(scale));
}

__global__ void __launch_bounds__(256) k_parcels(SprayArgs a, rn_params P) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= SPRAY_N) return;
  const Grid g = a.g;
  const float dt = a.st->x;
  float4 pa = a.PA[idx], pb = a.PB[idx];
  const int head = a.hs ? int(a.hs[0]) : a.head;
  int rel = idx - head;
  if (rel < 0) rel += SPRAY_N;
  float4 oA, oB, oC;
  const uint32_t seed = a.hs ? a.hs[1] : uint32_t(a.seed);
  if (rel < SPRAY_PER_STEP) {
    // new parcel; whatever the old one still carried goes to the gas
    uint32_t id = uint32_t(idx) ^ (seed * 2654435761u);
    int t = int(rnd(id, 1u) * 255.999f);
    float4 e1 = a.tab[t], e2 = a.tab[256 + t], e3 = a.tab[512 + t];
    float ang = e1.z + (rnd(id, 2u) - 0.5f) * 2.0f * e2.z;
    float r = fmaxf(e1.y + (rnd(id, 3u) - 0.5f) * e2.w, 0.05f);
    float d = e2.y * expf((rnd(id, 4u) - 0.5f) * 1.4f);
    oA = make_float4(e1.x, r, e1.w * cosf(ang), e1.w * sinf(ang));
    oB = make_float4(d, P.mhat * dt / float(SPRAY_PER_STEP), e2.x, e3.x);
    oC = pb.y > 0.0f ? make_float4(pb.y, pb.y * pa.z, pb.y * pa.w, 0.0f) : make_float4(0.f, 0.f, 0.f, 0.f);
  } else {
    oA = pa; oB = pb; oC = make_float4(0.f, 0.f, 0.f, 0.f);
    if (pb.y > 0.0f) {
      int gx = min(max(int(floorf(pa.x)), 0), g.Nx - 1);
      int gy = min(max(int(floorf(pa.y)), 0), g.Nr - 1);
      float4 w, s;
      interior_prim(g, a.A1, a.B1, gx, gy, w, s);
      if (w.x < 0.0f) {
        // born inside solid hardware: walk out into the flow
        oA = make_float4(pa.x + 1.0f, fmaxf(pa.y - 0.5f, 0.05f), fmaxf(pa.z, 0.0f), pa.w);
      } else {
        const float* pr = pb.z < 0.5f ? P.fuel : P.ox;
        float vx = pa.z, vy = pa.w;
        float m = pb.y, d = pb.x, dts = dt * P.tScale;
        float dn = d, mn = m;
        if (w.x > 0.0f) {
          float rm = (1.0f - s.x) * P.gas[0] + s.y * P.Rs[0] + s.w * P.Rs[1] + fmaxf(s.x - s.y - s.w, 0.0f) * P.Rs[2];
          float T = w.w / (w.x * rm) * P.gas[2];
          float rhoG = w.x * 1.225f, Urel = len2(w.y - vx, w.z - vy) * 287.6f + 1e-3f;
          float mu = 1.458e-6f * T * sqrtf(T) / (T + 110.4f);
          float Re = rhoG * Urel * d / mu;
          float invTau = 18.0f * mu * (1.0f + 0.15f * powf(fminf(Re, 1000.0f), 0.687f)) / (pr[0] * d * d);
          float e = expf(-dts * invTau);
          vx = w.y + (vx - w.y) * e;
          vy = w.z + (vy - w.z) * e;
          float cp = rm * 287.05f * (s.z + 1.0f);
          float Bs = fmaxf(cp * (T - pr[1]), 0.0f) / pr[2];
          float K = 8.0f * (mu / 0.7f) / pr[0] * logf(1.0f + Bs) * (1.0f + 0.27f * sqrtf(Re));
          float d2 = d * d - K * dts;
          dn = d2 > 1e-12f ? sqrtf(d2) : 0.0f;
          float f = dn / d;
          mn = dn > 0.0f ? m * f * f * f : 0.0f;
          float we = rhoG * Urel * Urel * dn / pr[3];
          if (we > 12.0f && dn > 0.0f) {
            float dst = 12.0f * pr[3] / (rhoG * Urel * Urel);
            float tb = 3.0f * dn / Urel * sqrtf(pr[0] / rhoG);
            dn = mixf(dn, fmaxf(dst, 2e-6f), 1.0f - expf(-dts / tb));
          }
        }
        float xi = pb.w;
        if (xi > 0.0f && pa.x >= xi) {      // impingement: the jets shatter into a fan
          uint32_t id = uint32_t(idx) ^ (seed * 2654435761u);
          float sp = len2(vx, vy), phi = (rnd(id, 5u) - 0.5f) * 2.0f * P.fan;
          vx = sp * cosf(phi);
          vy = sp * sinf(phi);
          dn *= 0.25f;
          xi = 0.0f;
        }
        float x = pa.x + vx * dt, y = pa.y + vy * dt;
        if (y < 0.0f) { y = -y; vy = -vy; }
        if (x < 0.0f) { x = -x; vx = fabsf(vx) * 0.3f; }
        if (wall_at(g, a.A1, a.B1, x, y)) {
          bool hx = wall_at(g, a.A1, a.B1, x, pa.y), hr = wall_at(g, a.A1, a.B1, pa.x, y);
          if (hx) { vx *= -0.3f; x = pa.x; }
          if (hr) { vy *= -0.3f; y = pa.y; }
          if (!hx && !hr) { x = pa.x; y = pa.y; vx *= -0.3f; vy *= -0.3f; }
        }
        float dm = m - mn;
        oC = make_float4(dm, mn * (pa.z - vx) + dm * pa.z, mn * (pa.w - vy) + dm * pa.w, 0.0f);
        if (x >= float(g.Nx) || y >= float(g.Nr) || mn <= 0.0f) {
          oA = make_float4(-1.0f, -1.0f, 0.0f, 0.0f);
          oB = make_float4(0.f, 0.f, 0.f, 0.f);
        } else {
          oA = make_float4(x, y, vx, vy);
          oB = make_float4(dn, mn, pb.z, xi);
        }
      }
    }
  }
  a.oPA[idx] = oA;
  a.oPB[idx] = oB;
  a.oPC[idx] = oC;
  {
    // the next step's bounds: the largest mass and speed written here (finite
    // values only), folded per block, and this step's bounds (they never shrink)
    // (and, for the parcel-steps counter, how many live parcels it writes)
    __shared__ float bm[8], bv[8];
    __shared__ unsigned bn[8];
    float m = oB.y > 0.0f && oB.y < 3.0e38f ? oB.y : 0.0f;
    float v = oB.y > 0.0f ? len2(oA.z, oA.w) : 0.0f;
    v = v < 3.0e38f ? v : 0.0f;
    unsigned n = __popc(__ballot_sync(0xffffffffu, oB.y > 0.0f));
    for (int o = 16; o > 0; o >>= 1) {
      m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
      v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    if ((threadIdx.x & 31) == 0) { bm[threadIdx.x >> 5] = m; bv[threadIdx.x >> 5] = v; bn[threadIdx.x >> 5] = n; }
    __syncthreads();
    if (threadIdx.x < 32) {
      m = threadIdx.x < 8 ? bm[threadIdx.x] : 0.0f;
      v = threadIdx.x < 8 ? bv[threadIdx.x] : 0.0f;
      n = threadIdx.x < 8 ? bn[threadIdx.x] : 0u;
      for (int o = 16; o > 0; o >>= 1) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        n += __shfl_xor_sync(0xffffffffu, n, o);
      }
      if (threadIdx.x == 0) {
        if (a.liveSteps && n) atomicAdd(a.liveSteps, (unsigned long long)n);
        if (blockIdx.x == 0) {
          m = fmaxf(m, __uint_as_float(a.boundIn[0]));
          v = fmaxf(v, __uint_as_float(a.boundIn[1]));
        }
        if (m > 0.0f) atomicMax(a.boundOut, __float_as_uint(m));
        if (v > 0.0f) atomicMax(a.boundOut + 1, __float_as_uint(v));
      }
    }
  }
  // deposit record (VS_SPRAY_DEP, spray.js:131-141): old position, new source
  const unsigned none = unsigned(g.Nx * g.Nr);
  unsigned key = none;
  float4 dep = make_float4(0.f, 0.f, 0.f, 0.f);
  if (!(pa.x < 0.0f || (oC.x == 0.0f && oC.y == 0.0f && oC.z == 0.0f))) {
    float type = pb.z;
    int gx = min(max(int(floorf(pa.x)), 0), g.Nx - 1);
    int gy = min(max(int(floorf(pa.y)), 0), g.Nr - 1);
    float4 gm = g.geoM[gy * g.Nx + gx];
    gx += iround(gm.x);
    gy += iround(gm.y);
    key = unsigned(gy * g.Nx + gx);
    dep = make_float4(oC.x * (1.0f - type), oC.x * type, oC.y, oC.z);
  }
#ifdef RN_FAST
  if (key != none) {
    const float sm = dep_scale_mass(P, a.boundIn), sp = dep_scale_mom(P, a.boundIn);
    unsigned long long* c = a.acc + 4 * size_t(key);
    bool over = false;
    atomicAdd(c + 0, to_fixed(dep.x, sm, over));
    atomicAdd(c + 1, to_fixed(dep.y, sm, over));
    atomicAdd(c + 2, to_fixed(dep.z, sp, over));
    atomicAdd(c + 3, to_fixed(dep.w, sp, over));
    if (over) atomicOr(a.depFlag, 1u);
  }
#else
  a.key[idx] = key;
  a.val[idx] = unsigned(idx);
  a.dep[idx] = dep;
#endif
}

// one thread per run of equal keys: sum in parcel-index order. The run is read
// 8 records at a time so that their gathers are in flight together; the adds
// stay sequential, in the same order.
__global__ void k_segsum(const unsigned* __restrict__ key, const unsigned* __restrict__ val,
                         const float4* __restrict__ dep, float4* src, unsigned none) {
  constexpr int U = 8;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= SPRAY_N) return;
  const unsigned k = key[q];
  if (k == none || (q > 0 && key[q - 1] == k)) return;
  float sx = 0.f, sy = 0.f, sz = 0.f, sw = 0.f;
  for (int r = q; r < SPRAY_N; r += U) {
    bool in[U];
    float4 d[U];
#pragma unroll
    for (int u = 0; u < U; u++) in[u] = r + u < SPRAY_N && key[r + u] == k;
#pragma unroll
    for (int u = 0; u < U; u++) d[u] = in[u] ? dep[val[r + u]] : make_float4(0.f, 0.f, 0.f, 0.f);
    bool more = true;
#pragma unroll
    for (int u = 0; u < U; u++) {
      more = more && in[u];
      if (more) { sx = d[u].x + sx; sy = d[u].y + sy; sz = d[u].z + sz; sw = d[u].w + sw; }
    }
    if (!more) break;
  }
  src[k] = make_float4(sx, sy, sz, sw);
}

__global__ void __launch_bounds__(256) k_apply(ApplyArgs a, rn_params P) {
  __shared__ float red[8];
  const Grid g = a.g;
  const int N = g.Nx * g.Nr;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  float wcell = 0.0f;
  // the ring head and seed of the next step (GPUSpray.step's bookkeeping,
  // spray.js:295-296), when they live on the device; k_parcels of this step
  // has read them (it runs before this kernel)
  if (a.hsNext && k == 0) {
    a.hsNext[0] = (a.hsNext[0] + unsigned(SPRAY_PER_STEP)) % unsigned(SPRAY_N);
    a.hsNext[1] = a.hsNext[1] + 1u;
  }
  if (k < N) {
    float4 oA, oB;
    bool fluid = !g.mask[k];
    // the next step's deposit sums start at zero (both variants keep this up)
    reinterpret_cast<ulonglong2*>(a.accNext)[2 * k] = make_ulonglong2(0ull, 0ull);
    reinterpret_cast<ulonglong2*>(a.accNext)[2 * k + 1] = make_ulonglong2(0ull, 0ull);
    if (!fluid) {
      oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
      oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
    } else {
      float4 gm = g.geoM[k];
      const int kh = k + iround(gm.y) * g.Nx + iround(gm.x);   // the cell's group host (i + dx, j + dy)
#ifdef RN_FAST
      const ulonglong2* c = reinterpret_cast<const ulonglong2*>(a.acc) + 2 * size_t(kh);
      const ulonglong2 c01 = c[0], c23 = c[1];
      const float sm = dep_scale_mass(P, a.boundIn), sp = dep_scale_mom(P, a.boundIn);
      float4 s = make_float4(from_fixed(c01.x, sm), from_fixed(c01.y, sm), from_fixed(c23.x, sp),
                             from_fixed(c23.y, sp));
#else
      float4 s = a.src[kh];
#endif
      float4 A = a.A[kh], B = a.B[kh];
      float invV = 1.0f / fmaxf(g.geoG[k].x, 1e-6f);
      float dm = s.x + s.y;
      if (dm == 0.0f && s.z == 0.0f && s.w == 0.0f) {
        oA = A; oB = B;
      } else {
        float den = fmaxf(A.x, RHO_MIN);
        float velx = A.y / den, vely = A.z / den;
        float rn = A.x + dm * invV;
        float momx = A.y + s.z * invV, momy = A.z + s.w * invV;
        float E = A.w + (s.x * P.eF + s.y * P.eO + (velx * s.z + vely * s.w)) * invV;
        float phi = fminf(dm * invV / rn, 1.0f);
        float Gn = mixf(B.z, P.Ge, phi);
        float vnx = momx / rn, vny = momy / rn;
        E = fmaxf(E, 0.02f * A.w + 0.5f * rn * (vnx * vnx + vny * vny) + P_MIN * Gn);
        oA = make_float4(rn, momx, momy, E);
        oB = make_float4(B.x + dm * invV, B.y + s.x * invV, Gn, B.w + s.y * invV);
      }
    }
    a.oA[k] = oA;
    a.oB[k] = oB;
    if (a.finalCfl && fluid) wcell = wave_speed(oA, oB);
  }
  if (a.finalCfl) {
    float w = wcell;
    for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = w;
    __syncthreads();
    if (threadIdx.x < 32) {
      w = threadIdx.x < 8 ? red[threadIdx.x] : 0.0f;
      for (int o = 16; o > 0; o >>= 1) w = fmaxf(w, __shfl_xor_sync(0xffffffffu, w, o));
      if (threadIdx.x == 0 && w > 0.0f) atomicMax(a.wOut, __float_as_uint(w));
    }
  }
}

static int key_bits(int Ncells) {
  int b = 1;
  while ((1u << b) <= unsigned(Ncells)) b++;   // keys are 0..Ncells (Ncells = no deposit)
  return b;
}

size_t spray_sort_temp_bytes(int Ncells) {
  size_t bytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, bytes, (const unsigned*)nullptr, (unsigned*)nullptr,
                                  (const unsigned*)nullptr, (unsigned*)nullptr, SPRAY_N, 0, key_bits(Ncells));
  return bytes;
}

int launch_spray(const SprayArgs& a, const rn_params& P, void* sortTemp, size_t sortTempBytes, unsigned* keyOut,
                 unsigned* valOut, float4* src, cudaStream_t s, int* launches) {
  k_parcels<<<SPRAY_N / 256, 256, 0, s>>>(a, P);
#ifdef RN_FAST
  // the deposits are summed in k_parcels itself (fixed point)
  (void)sortTemp; (void)sortTempBytes; (void)keyOut; (void)valOut; (void)src;
  *launches += 1;
#else
  // the deposit records sorted by cell, each cell's run summed in parcel order
  const int Ncells = a.g.Nx * a.g.Nr;
  size_t bytes = sortTempBytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(sortTemp, bytes, a.key, keyOut, a.val, valOut, SPRAY_N, 0,
                                                  key_bits(Ncells), s);
  if (e != cudaSuccess) return -1;
  cudaMemsetAsync(src, 0, sizeof(float4) * size_t(Ncells), s);
  k_segsum<<<SPRAY_N / 256, 256, 0, s>>>(keyOut, valOut, a.dep, src, unsigned(Ncells));
  *launches += 2;   // own kernels: parcels and segsum (the radix sort's kernels are library code)
#endif
  return 0;
}

void launch_apply(const ApplyArgs& a, const rn_params& P, cudaStream_t s) {
  const int N = a.g.Nx * a.g.Nr;
  k_apply<<<(N + 255) / 256, 256, 0, s>>>(a, P);
}

}  // namespace RN_VARIANT
}  // namespace rn
