// rn_step.cu -- fused time-step kernels for sm_100a.
//
// One SSP-RK2 stage is ONE kernel (k_stage): a block stages the ghost-cell
// primitives of its tile plus a 2-cell halo in shared memory (FS_PRIM,
// solver.js:56-126), computes every x- and r-face flux of the tile once
// (makeFluxShader, solver.js:133-259) into shared memory, then updates each
// cell over its merged cut-cell group (FS_UPDATE, solver.js:264-363). The
// reference's 7 full-grid passes per stage (prim, 2 flux, update, CFL chain)
// and its 6 face textures never touch HBM here.
//
// Group members outside the tile (slivers merged across a tile edge) are
// listed per tile at set_geometry (xoff/xcell). For each listed member the
// block adds a 5x5 block of primitives around it to the primitive phase and
// its 4 faces to the face phase: the same loops and the same single instance
// of the face code run them, so blocks along the walls do no serial or
// cold-code work.
//
// The step's last kernel folds the CFL wave speed of the cells it writes into
// one atomicMax per block (FS_REDUCE1/2, solver.js:368-397); the next step's
// stage-1 kernel turns it into dt in every block and the block of tile 0
// stores the step info (FS_STEPINFO, solver.js:398-411). dt never leaves the
// device.
//
// With the viscous/wall/reaction split step, stage 2 and the split step are
// ONE kernel (k_stage2phys): the stage-2 ghost primitives are the ones the
// split step reads (solver.js:940-941), so the block stages them once, keeps
// its stage-2 results in shared memory and runs vcell (FS_VCELL), the viscous
// face fluxes (makeViscFluxShader) and FS_SOURCE on them. Its output goes to
// the ring slot stage 2 alone would write, so no block overwrites the state
// another block's stage-2 update still reads.
//
// Every body is a device function templated on the tile shape; a
// single-instance kernel maps blockIdx to a tile, a batch kernel maps its 1-D
// block index to (instance, tile) through a table and loads the instance's
// buffers and parameter block into shared memory first.
#include <cuda_runtime.h>
#include "rn_kernels.cuh"

namespace rn {
namespace RN_VARIANT {

// Resident warps per SM a tile shape's kernels are compiled for (TILE_WARPS):
// 32 caps them at 64 registers (4 blocks of 256 threads per SM), 24 at 80.
// Measured on B200 with 16x16 tiles (fast precision, G cell-updates/s, caps of
// 8 / 24 / 32 / 40 warps): 64 batched instances 2.24 / 3.05 / 3.44 / 3.04,
// plain 4096x1536 3.33 / 4.55 / 5.52 / 5.65, viscous 512x192 1.71 / 2.24 /
// 2.18 / 1.89. Results are bit-identical across caps.
template <int TX_, int TY_, int NT_, int WARPS_, int ID_>
struct TileT {
  static constexpr int TX = TX_, TY = TY_, NT = NT_, NC = TX * TY;   // NT threads, NC cells (NC <= NT)
  static constexpr int ID = ID_;                                      // index into TILE_* and TileMaps
  static constexpr int MINB = WARPS_ / (NT / 32) > 0 ? WARPS_ / (NT / 32) : 1;
  // Shapes compiled for fewer than 32 warps (more registers per thread) run
  // the fused kernel's stage-2 update and FS_VCELL as one work list, with
  // T1/T2 in shared memory of their own (viscous plume 512x192 with 14x16
  // tiles: 3.00 -> 3.10-3.18 G cell-updates/s). At 4 blocks per SM the extra
  // memory, loop body and live registers cost more than they save (64 batched
  // instances, 16x15: 4.37 -> 4.18 G).
  static constexpr bool WIDE = WARPS_ < 32;
  static constexpr int PX = TX + 4, PY = TY + 4, NPT = PX * PY;   // primitives with a 2-cell halo
  static constexpr int NXF = TY * (TX + 1), NRF = (TY + 1) * TX;  // x- and r-faces of a tile
  static constexpr int TW = TX + 2, NTT = (TX + 2) * (TY + 2);    // vcell ring (tile + 1)
  // halo copy: raw A and B planes (NPT float4 each, B at a 128-byte boundary)
  // and the mask block (PY rows of MW bytes), in float4 slots of shared memory
  static constexpr int MW = mask_box_width(PX);
  static constexpr int NPT8 = (NPT + 7) / 8 * 8;
  static constexpr int MASKF4 = (MW * PY + 127) / 128 * 8;
  static constexpr unsigned HALO_BYTES = 2u * 16u * NPT + unsigned(MW) * PY;
  // WIDE shapes (3 blocks per SM, shared memory to spare) also stage the cell
  // geometry their update and split step read, geoM with a 1-cell ring (the
  // vcell ring's turbulence lengths) and geoG, and keep the raw halo block
  // alive past the face phase: their update reads no global memory for tile
  // cells. STAGED_F4 = the float4 slots these add to the layout.
  static constexpr int NGM = (TX + 2) * (TY + 2), NGM8 = (NGM + 7) / 8 * 8, NGG8 = (NC + 7) / 8 * 8;
  static constexpr unsigned GEO_BYTES = 16u * (NGM + NC);
  static constexpr int STAGED_F4 = WIDE ? 2 * NPT8 + NGM8 + NGG8 : 0;
};
using Tile0 = TileT<TILE_TX[0], TILE_TY[0], TILE_NT[0], TILE_WARPS[0], 0>;
using Tile1 = TileT<TILE_TX[1], TILE_TY[1], TILE_NT[1], TILE_WARPS[1], 1>;
using Tile2 = TileT<TILE_TX[2], TILE_TY[2], TILE_NT[2], TILE_WARPS[2], 2>;
using Tile3 = TileT<TILE_TX[3], TILE_TY[3], TILE_NT[3], TILE_WARPS[3], 3>;
using Tile4 = TileT<TILE_TX[4], TILE_TY[4], TILE_NT[4], TILE_WARPS[4], 4>;
static_assert(Tile0::NC <= Tile0::NT && Tile1::NC <= Tile1::NT && Tile2::NC <= Tile2::NT && Tile3::NC <= Tile3::NT &&
                  Tile4::NC <= Tile4::NT,
              "a thread per cell");
static_assert(4 * Tile3::PX <= 256 && Tile3::MW <= 256 && Tile0::PY <= 256, "copy boxes within 256 elements");

// Polls of the halo copy's mbarrier before a block gives up (each poll waits
// a short hardware-defined time): far beyond any copy, short of a hang.
constexpr unsigned HALO_WAIT_POLLS = 1u << 22;

// --------------------------------------------------------------------------
// block-wide max of non-negative floats -> one atomicMax on the bit pattern
template <int NT>
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

// The dynamic shared memory rounded up to a 128-byte boundary (the halo
// copies' destinations are 128-byte aligned; every layout reserves the slack).
// The rounding is an element offset from the shared array itself, so the
// compiler still knows every derived pointer addresses shared memory (a round
// trip through an integer address would make them generic 64-bit pointers:
// generic loads and two registers per pointer, which spilled).
__device__ __forceinline__ float4* aligned_smem(float4* p) {
  return p + (((128u - (smem_addr(p) & 127u)) & 127u) >> 4);
}

// Shared-memory index of the primitive of cell (mx + dx, my + dy) for listed
// member e: tile cells live in the PX x PY tile array, listed members'
// neighbourhoods in 5x5 blocks after it.
template <class T>
__device__ __forceinline__ int ext_prim(int e, int dx, int dy) {
  return T::NPT + e * 25 + (dy + 2) * 5 + (dx + 2);
}

// Faces of listed member e (slots NXF + NRF + 4e + w, w = W, E, S, N): the
// face position, its direction, whether the reference draws it, and its
// stencil as primitive slots (the 4 cells along the normal c0..c3, the 4
// transverse sensor cells k1+t, k1-t, ij+t, ij-t).
struct FaceSlot {
  int c[4], s[4];
  int i, j;
  bool dirR, valid;
};
template <class T>
__device__ __forceinline__ FaceSlot member_face_slot(int q, const int* xc, int Nx) {
  FaceSlot f;
  const int e = q >> 2, w = q & 3, m = xc[e];
  const int mx = m % Nx, my = m / Nx;
  if (w < 2) {
    const int o = w;                             // face at mx + o
    f.i = mx + o; f.j = my; f.dirR = false; f.valid = true;
    f.c[0] = ext_prim<T>(e, o - 2, 0); f.c[1] = ext_prim<T>(e, o - 1, 0);
    f.c[2] = ext_prim<T>(e, o, 0); f.c[3] = ext_prim<T>(e, o + 1, 0);
    f.s[0] = ext_prim<T>(e, o - 1, 1); f.s[1] = ext_prim<T>(e, o - 1, -1);
    f.s[2] = ext_prim<T>(e, o, 1); f.s[3] = ext_prim<T>(e, o, -1);
  } else {
    const int o = w - 2;                         // face at my + o
    f.i = mx; f.j = my + o; f.dirR = true; f.valid = f.j != 0;
    f.c[0] = ext_prim<T>(e, 0, o - 2); f.c[1] = ext_prim<T>(e, 0, o - 1);
    f.c[2] = ext_prim<T>(e, 0, o); f.c[3] = ext_prim<T>(e, 0, o + 1);
    f.s[0] = ext_prim<T>(e, 1, o - 1); f.s[1] = ext_prim<T>(e, -1, o - 1);
    f.s[2] = ext_prim<T>(e, 1, o); f.s[3] = ext_prim<T>(e, -1, o);
  }
  return f;
}

// The four face slots (W, E, S, N) of group member (cx, cy): tile faces for a
// tile cell (x-face ly*(TX+1)+lx, r-face NXF + ly*TX + lx), else the faces of
// its entry in the tile's member list.
template <class T>
__device__ __forceinline__ void member_faces(int cx, int cy, int x0, int y0, const int* xc, int xn, int Nx,
                                             int& fw, int& fe, int& fs, int& fn) {
  const int mx = cx - x0, my = cy - y0;
  if (unsigned(mx) < unsigned(T::TX) && unsigned(my) < unsigned(T::TY)) {
    fw = my * (T::TX + 1) + mx;
    fe = fw + 1;
    fs = T::NXF + my * T::TX + mx;
    fn = fs + T::TX;
  } else {
    const int mc = cy * Nx + cx;
    int e = 0;
    while (e < xn - 1 && xc[e] != mc) e++;
    fw = T::NXF + T::NRF + 4 * e;
    fe = fw + 1;
    fs = fw + 2;
    fn = fw + 3;
  }
}

// Dynamic shared memory (float4 slots) of the stage kernel for a member list
// of xn cells: 128-byte alignment slack, the mask block, the region that holds
// the raw halo copy and then the face fluxes F, Y, O, the face areas and the
// primitives W, Wb.
template <class T>
__host__ __device__ constexpr int stage_region_t(int xn) {
  return 2 * T::NPT8 > 2 * (T::NXF + T::NRF + 4 * xn) + (T::NXF + T::NRF + 4 * xn + 3) / 4
             ? 2 * T::NPT8
             : 2 * (T::NXF + T::NRF + 4 * xn) + (T::NXF + T::NRF + 4 * xn + 3) / 4;
}
template <class T>
__host__ __device__ constexpr size_t stage_smem_t(int maxX) {
  return sizeof(float4) * (8 + T::MASKF4 + T::STAGED_F4 + stage_region_t<T>(maxX) +
                           (T::NXF + T::NRF + 4 * maxX + 3) / 4 + 2 * (T::NPT + 25 * maxX));
}

// --------------------------------------------------------------------------
// Phases shared by the stage, physics and fused kernels. Each loops its slots
// over the block's threads; the caller puts the barriers between phases.

// Open area of tile x-face k (west face of cell (x0 + lx, y0 + ly)) and tile
// r-face k (south face), as the reference reads them from geoA; 0 where the
// face is not drawn (x: i <= Nx, j < Nr; r: i < Nx, 0 < j <= Nr).
template <class T>
__device__ __forceinline__ float xface_area(const Grid& g, int k, int x0, int y0) {
  const int ly = k / (T::TX + 1), lx = k - ly * (T::TX + 1), i = x0 + lx, j = y0 + ly;
  return (i <= g.Nx && j < g.Nr) ? g.geoA[j * (g.Nx + 1) + i].z : 0.0f;
}
template <class T>
__device__ __forceinline__ float rface_area(const Grid& g, int k, int x0, int y0) {
  const int ly = k / T::TX, lx = k - ly * T::TX, i = x0 + lx, j = y0 + ly;
  return (i < g.Nx && j <= g.Nr && j != 0) ? g.geoA[j * (g.Nx + 1) + i].w : 0.0f;
}
template <class T>
__device__ __forceinline__ float member_face_area(const Grid& g, int q, const int* xc) {
  const FaceSlot s = member_face_slot<T>(q, xc, g.Nx);
  if (!s.valid) return 0.0f;
  const float4* p = g.geoA + (s.j * (g.Nx + 1) + s.i);
  return s.dirR ? p->w : p->z;
}

// Start of a stage kernel's block: thread 0 initialises the halo copy's
// mbarrier and issues the three tiled copies of the tile + 2-cell halo (raw A
// into R, raw B into R + NPT8, the mask block into sMask). The mask box starts
// at the 16-byte boundary at or below the halo's first column.
template <class T>
__device__ __forceinline__ void halo_issue(const TileMaps* tm, int slot, int x0, int y0, float4* R, uint8_t* sMask,
                                           uint64_t* bar) {
  if (threadIdx.x == 0) {
    const TileMaps& M = tm[T::ID];
    mbar_init(bar, 1);
    mbar_expect_tx(bar, T::HALO_BYTES + (T::WIDE ? T::GEO_BYTES : 0u));
    tma_load_2d(R, &M.a[slot], 4 * (x0 - 2), y0 - 2, bar);
    tma_load_2d(R + T::NPT8, &M.b[slot], 4 * (x0 - 2), y0 - 2, bar);
    tma_load_2d(sMask, &M.mask, (x0 - 2) & ~15, y0 - 2, bar);
    if constexpr (T::WIDE) {                     // geoM ring box, then geoG tile box, after the raw block
      tma_load_2d(R + 2 * T::NPT8, &M.geoM, 4 * (x0 - 1), y0 - 1, bar);
      tma_load_2d(R + 2 * T::NPT8 + T::NGM8, &M.geoG, 4 * x0, y0, bar);
    }
  }
}

// Per-cell operands of the update, vcell and split-step phases: from the
// staged boxes where the cell lies in them (WIDE shapes: the raw halo block,
// mask, geoM ring and geoG tile stay in shared memory), else from global
// memory (other shapes, whose raw block the face fluxes overwrite, and listed
// members outside the boxes). The staged values are copies of the same cells.
template <class T>
struct CellSrc {
  const Grid& g;
  const float4* __restrict__ A;     // the stage's input state (the source of the raw block)
  const float4* __restrict__ B;
  const float4* raw;                // raw A at raw[0..NPT), raw B at raw[NPT8..)
  const uint8_t* m;
  int x0, y0, mo;
  __device__ __forceinline__ bool in_halo(int i, int j) const {
    return T::WIDE && unsigned(i - x0 + 2) < unsigned(T::PX) && unsigned(j - y0 + 2) < unsigned(T::PY);
  }
  __device__ __forceinline__ bool in_ring(int i, int j) const {
    return T::WIDE && unsigned(i - x0 + 1) < unsigned(T::TX + 2) && unsigned(j - y0 + 1) < unsigned(T::TY + 2);
  }
  __device__ __forceinline__ bool in_tile(int i, int j) const {
    return T::WIDE && unsigned(i - x0) < unsigned(T::TX) && unsigned(j - y0) < unsigned(T::TY);
  }
  __device__ __forceinline__ int hslot(int i, int j) const { return (j - y0 + 2) * T::PX + (i - x0 + 2); }
  __device__ __forceinline__ bool solid(int i, int j) const {
    return in_halo(i, j) ? m[(j - y0 + 2) * T::MW + mo + (i - x0 + 2)] != 0 : g.mask[j * g.Nx + i] != 0;
  }
  __device__ __forceinline__ float4 a(int i, int j) const { return in_halo(i, j) ? raw[hslot(i, j)] : A[j * g.Nx + i]; }
  __device__ __forceinline__ float4 b(int i, int j) const {
    return in_halo(i, j) ? raw[T::NPT8 + hslot(i, j)] : B[j * g.Nx + i];
  }
  __device__ __forceinline__ float4 gm(int i, int j) const {
    return in_ring(i, j) ? raw[2 * T::NPT8 + (j - y0 + 1) * (T::TX + 2) + (i - x0 + 1)] : g.geoM[j * g.Nx + i];
  }
  __device__ __forceinline__ float4 gg(int i, int j) const {
    return in_tile(i, j) ? raw[2 * T::NPT8 + T::NGM8 + (j - y0) * T::TX + (i - x0)] : g.geoG[j * g.Nx + i];
  }
};
// Every thread waits for the halo copy (after a barrier that published the
// mbarrier's initialisation). False, in every thread, when any thread gave
// up; the block then records the error and leaves.
__device__ __forceinline__ bool halo_wait(uint64_t* bar, unsigned* err) {
  const bool ok = mbar_wait_bounded(bar, HALO_WAIT_POLLS);
  if (__syncthreads_and(ok)) return true;
  if (threadIdx.x == 0 && err) atomicOr(err, 1u);
  return false;
}

// Cells for ghost_prim_c and the interior slots: from the staged halo block
// (raw A, B and mask in shared memory) where the cell lies in it, else from
// global memory (a listed member's neighbourhood outside the block).
template <class T>
struct HaloCells {
  const Grid& g;
  const float4* __restrict__ A;
  const float4* __restrict__ B;
  const float4* rA;
  const float4* rB;
  const uint8_t* m;
  int x0, y0, mo;
  __device__ __forceinline__ bool staged(int i, int j) const {
    return unsigned(i - x0 + 2) < unsigned(T::PX) && unsigned(j - y0 + 2) < unsigned(T::PY);
  }
  __device__ __forceinline__ int slot(int i, int j) const { return (j - y0 + 2) * T::PX + (i - x0 + 2); }
  __device__ __forceinline__ bool solid(int i, int j) const {
    return staged(i, j) ? m[(j - y0 + 2) * T::MW + mo + (i - x0 + 2)] != 0 : g.mask[j * g.Nx + i] != 0;
  }
  __device__ __forceinline__ float4 a(int i, int j) const { return staged(i, j) ? rA[slot(i, j)] : A[j * g.Nx + i]; }
  __device__ __forceinline__ float4 b(int i, int j) const { return staged(i, j) ? rB[slot(i, j)] : B[j * g.Nx + i]; }
};

// FS_PRIM: ghost-cell primitives of the tile + 2-cell halo, then of the listed
// members' 5x5 blocks, in one loop through one instance of the ghost code.
template <class T>
__device__ __forceinline__ void load_prims(const Grid& g, const float4* __restrict__ A, const float4* __restrict__ B,
                                           float t, const rn_params& P, int x0, int y0, const int* xc, int NP,
                                           const float4* R, const uint8_t* sMask, float4* sW, float4* sWb) {
  const int Nx = g.Nx, Nr = g.Nr;
  const int mo = (x0 - 2) - ((x0 - 2) & ~15);
  const HaloCells<T> cells{g, A, B, R, R + T::NPT8, sMask, x0, y0, mo};
  for (int k = threadIdx.x; k < NP; k += T::NT) {
    int i, j, ly = 0, lx = 0;
    if (k < T::NPT) {
      ly = k / T::PX; lx = k - ly * T::PX;
      i = x0 - 2 + lx; j = y0 - 2 + ly;
    } else {                                     // member e's 5x5 block
      const int q = k - T::NPT, e = q / 25, r = q - e * 25, m = xc[e], dy = r / 5;
      i = m % Nx + (r - dy * 5) - 2; j = m / Nx + dy - 2;
    }
    float4 W, Wb;
    if (i >= 0 && i < Nx && j >= 0 && j < Nr) {     // ghost_prim's interior branch
      // a slot of the staged block is its own cell k of it (no lookup)
      const bool own = k < T::NPT;
      const float4 a = own ? R[k] : cells.a(i, j), b = own ? R[T::NPT8 + k] : cells.b(i, j);
      const bool solid = own ? sMask[ly * T::MW + mo + lx] != 0 : cells.solid(i, j);
      if (solid) {
        W = make_float4(-1.0f, 0.0f, 0.0f, 1.0f);
        Wb = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      } else {
        const Prim q = to_prim(a, b);
        W = q.w;
        Wb = q.s;
      }
    } else if (i <= Nx + 1 && j <= Nr + 1) {
      ghost_prim_c(Nx, Nr, cells, i, j, t, P, W, Wb);
    } else {
      W = make_float4(-1.f, 0.f, 0.f, 1.f); Wb = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    sW[k] = W;
    sWb[k] = Wb;
  }
}

// Face areas into sAr: a thread's first x- and r-face (loaded at block start,
// their latency hidden behind the halo copy), the rest of the tile's faces
// (shapes with more faces than threads), then the listed members' faces.
struct FirstAreas {
  float x, r;
};
template <class T>
__device__ __forceinline__ FirstAreas first_areas(const Grid& g, int x0, int y0) {
  FirstAreas f;
  const int tid = threadIdx.x;
  f.x = tid < T::NXF ? xface_area<T>(g, tid, x0, y0) : 0.0f;
  f.r = tid < T::NRF ? rface_area<T>(g, tid, x0, y0) : 0.0f;
  return f;
}
template <class T>
__device__ __forceinline__ void store_areas(const Grid& g, int x0, int y0, const int* xc, int xn, FirstAreas f,
                                            float* sAr) {
  const int tid = threadIdx.x;
  if (tid < T::NXF) sAr[tid] = f.x;
  if (tid < T::NRF) sAr[T::NXF + tid] = f.r;
  if constexpr (T::NXF > T::NT)
    for (int k = tid + T::NT; k < T::NXF; k += T::NT) sAr[k] = xface_area<T>(g, k, x0, y0);
  if constexpr (T::NRF > T::NT)
    for (int k = tid + T::NT; k < T::NRF; k += T::NT) sAr[T::NXF + k] = rface_area<T>(g, k, x0, y0);
  for (int q = tid; q < 4 * xn; q += T::NT) sAr[T::NXF + T::NRF + q] = member_face_area<T>(g, q, xc);
}

// FS_FLUX_X/R: every face of the tile (x-faces, then r-faces) and of its
// listed members in one loop through one instance of the flux code. Face k's
// 4 cells along the normal are primitive slots b, b + d, b + 2d, b + 3d and its
// sensor cells (k1 +- t, ij +- t of makeFluxShader, solver.js:133-259)
// b + d +- t and b + 2d +- t: tile faces have (d, t) = (1, PX) (x) or (PX, 1)
// (r); a listed member's faces live in its 5x5 block, with 5 in place of PX.
// One code path for every face also makes the fast precision's contracted
// multiply-adds round alike in every tile shape.
template <class T>
__device__ __forceinline__ void inviscid_faces(const Grid& g, const rn_params& P, const int* xc, int xn,
                                               const float4* sW, const float4* sWb, float4* sF, float4* sY,
                                               float* sO, const float* sAr) {
  constexpr int NXR = T::NXF + T::NRF;
  for (int k = threadIdx.x; k < NXR + 4 * xn; k += T::NT) {
    int b, d, t;
    bool dirR;
    if (k < T::NXF) {
      const int ly = k / (T::TX + 1), lx = k - ly * (T::TX + 1);
      b = (ly + 2) * T::PX + lx; d = 1; t = T::PX; dirR = false;
    } else if (k < NXR) {
      const int kk = k - T::NXF, ly = kk / T::TX, lx = kk - ly * T::TX;
      b = ly * T::PX + lx + 2; d = T::PX; t = 1; dirR = true;
    } else {                                     // member e's face w (W, E at mx + o; S, N at my + o)
      const int q = k - NXR, e = q >> 2, w = q & 3, o = w & 1;
      dirR = w >= 2;
      b = dirR ? ext_prim<T>(e, 0, o - 2) : ext_prim<T>(e, o - 2, 0);
      d = dirR ? 5 : 1; t = dirR ? 1 : 5;
    }
    Flux f;
    f.F = make_float4(0.f, 0.f, 0.f, 0.f); f.Y = f.F; f.O = 0.f;
    const float area = sAr[k];   // the face's open area, 0 where it is not drawn
    if (area != 0.0f)
      f = face_flux(dirR, area, sW[b], sWb[b], sW[b + d], sWb[b + d], sW[b + 2 * d], sWb[b + 2 * d], sW[b + 3 * d],
                    sWb[b + 3 * d], sW[b + d + t], sW[b + d - t], sW[b + 2 * d + t], sW[b + 2 * d - t], P);
    sF[k] = f.F; sY[k] = f.Y; sO[k] = f.O;
  }
}

// memberFlux (solver.js:287-299) of group member (cx, cy): its four faces'
// fluxes weighted by their open areas (0 on the axis face, whose flux is 0 too).
template <class T, bool WITH_O>
__device__ __forceinline__ void add_member(int cx, int cy, int x0, int y0, const int* xc, int xn, int Nx,
                                           const float4* sF, const float4* sY, const float* sO, const float* sAr,
                                           float4& L, float4& LY, float& LO) {
  int fw, fe, fs, fn;
  member_faces<T>(cx, cy, x0, y0, xc, xn, Nx, fw, fe, fs, fn);
  const float aw = fabsf(sAr[fw]), ae = fabsf(sAr[fe]), as_ = fabsf(sAr[fs]), an = fabsf(sAr[fn]);
  sub4(L, ae, sF[fe], aw, sF[fw]);
  sub4(L, an, sF[fn], as_, sF[fs]);
  sub4(LY, ae, sY[fe], aw, sY[fw]);
  sub4(LY, an, sY[fn], as_, sY[fs]);
  if constexpr (WITH_O) {
    LO -= ae * sO[fe] - aw * sO[fw];
    LO -= an * sO[fn] - as_ * sO[fs];
  }
}
// The group of host (Hx, Hy) with slave mask sm_: the host, then its slaves in
// the reference's member order (slave bits 1, 2, 4, 8 = W, E, S, N), all
// through one call site (bit 0 of the walked mask is the host).
template <class T, bool WITH_O>
__device__ __forceinline__ void group_flux(int Hx, int Hy, int sm_, int x0, int y0, const int* xc, int xn, int Nx,
                                           const float4* sF, const float4* sY, const float* sO, const float* sAr,
                                           float4& L, float4& LY, float& LO) {
  for (int s = ((sm_ & 15) << 1) | 1; s != 0; s &= s - 1) {
    const int bit = __ffs(s) - 1;
    const int cx = Hx + (bit == 1 ? -1 : bit == 2 ? 1 : 0), cy = Hy + (bit == 3 ? -1 : bit == 4 ? 1 : 0);
    add_member<T, WITH_O>(cx, cy, x0, y0, xc, xn, Nx, sF, sY, sO, sAr, L, LY, LO);
  }
}

// FS_UPDATE of cell (i, j) inside the grid: the RK update of its host's
// cut-cell group. Returns whether the cell is fluid.
template <class T, int STAGE>
__device__ __forceinline__ bool update_cell(const StageArgs& a, const CellSrc<T>& cs, const rn_params& P, int i,
                                            int j, float dt, float t, int x0, int y0, const int* xc, int xn,
                                            const float4* sF, const float4* sY, const float* sO, const float* sAr,
                                            float4& oA, float4& oB) {
  const Grid& g = a.g;
  const int Nx = g.Nx;
  const int k = j * Nx + i;
  // the cell's own operands in one round of loads; a slave cell (host kh != k)
  // then loads its host's
  const bool solid = cs.solid(i, j);
  const float4 gm = cs.gm(i, j), gg = cs.gg(i, j);
  float4 A = cs.a(i, j), B = cs.b(i, j), A0 = STAGE == 2 ? a.A0[k] : A, B0 = STAGE == 2 ? a.B0[k] : B;
  if (solid) {
    oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
    oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
    return false;
  }
  const int Hx = i + iround(gm.x), Hy = j + iround(gm.y), kh = Hy * Nx + Hx;
  float ghz = gm.z;
  if (kh != k) {
    A = cs.a(Hx, Hy); B = cs.b(Hx, Hy);
    if (STAGE == 2) { A0 = a.A0[kh]; B0 = a.B0[kh]; }
    ghz = cs.gm(Hx, Hy).z;
  }
  Prim q = to_prim(A, B);
  float4 L = make_float4(0.f, 0.f, 0.f, 0.f), LY = L;
  float LO = 0.0f;
  const int sm_ = iround(ghz);
  if (P.inj) group_flux<T, true>(Hx, Hy, sm_, x0, y0, xc, xn, Nx, sF, sY, sO, sAr, L, LY, LO);
  else group_flux<T, false>(Hx, Hy, sm_, x0, y0, xc, xn, Nx, sF, sY, sO, sAr, L, LY, LO);
  // embedded wall: pressure force along the r-weighted wall vector
  float wl = len2(gg.z, gg.w);
  if (wl > 1e-6f) {
    const Over per_wl = over(wl);
    float nx = per_wl(gg.z), nr = per_wl(gg.w);
    float pw = wall_pressure(q, q.w.y * nx + q.w.z * nr);
    L.y -= gg.z * pw;
    L.z -= gg.w * pw;
  }
  L.z += q.w.w * gg.y;                       // axisymmetric source p Am
  float invV = fdiv(1.0f, fmaxf(gg.x, 1e-6f));
  float4 LB = make_float4(LY.x, LY.y, LY.z - q.s.z * LY.w, LO);
  float f = dt * invV;
  float4 U, UY;
  if (STAGE == 1) {
    U = make_float4(A.x + f * L.x, A.y + f * L.y, A.z + f * L.z, A.w + f * L.w);
    UY = make_float4(B.x + f * LB.x, B.y + f * LB.y, B.z + f * LB.z, B.w + f * LB.w);
  } else {
    U = make_float4(0.5f * (A0.x + A.x + f * L.x), 0.5f * (A0.y + A.y + f * L.y), 0.5f * (A0.z + A.z + f * L.z),
                    0.5f * (A0.w + A.w + f * L.w));
    UY = make_float4(0.5f * (B0.x + B.x + f * LB.x), 0.5f * (B0.y + B.y + f * LB.y),
                     0.5f * (B0.z + B.z + f * LB.z), 0.5f * (B0.w + B.w + f * LB.w));
  }
  float rho = fmaxf(U.x, RHO_MIN);
  const Over per_den = over(fmaxf(U.x, RHO_MIN));
  float vx = per_den(U.y), vy = per_den(U.z);
  float sp = len2(vx, vy);
  if (sp > P.vMax) { float s = fdiv(P.vMax, sp); vx *= s; vy *= s; }
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
      float u0 = cs.b(i, j).w;
      bool on = STAGE == 2 && t > P.bar[2];
      ubar = on ? fminf(u0 + fminf(dt * P.bar[0], 1.0f) * (vx - u0), P.bar[1]) : u0;
    }
    oB = make_float4(Zn, clampf(UY.y, 0.0f, Zn), Gn, ubar);
  }
  return true;
}

// --------------------------------------------------------------------------
// One RK stage on tile (bx, by) = tile index tileId of the instance in `a`.
template <class T, int STAGE>
__device__ __forceinline__ void stage_body(const StageArgs& a, const rn_params& P, int bx, int by, int tileId,
                                           float4* smRaw, float* red, int* xc, uint64_t* bar) {
  constexpr int TX = T::TX, NT = T::NT;
  const Grid& g = a.g;
  const int Nx = g.Nx, Nr = g.Nr;
  const int tid = threadIdx.x;
  const int x0 = bx * TX, y0 = by * T::TY;
  float4* sm = aligned_smem(smRaw);
  uint8_t* sMask = reinterpret_cast<uint8_t*>(sm);
  float4* RAW = sm + T::MASKF4;                 // raw halo block (+ geometry boxes for WIDE shapes)
  float4* R = RAW + T::STAGED_F4;               // face fluxes (other shapes: over the raw block)
  halo_issue<T>(a.tm, a.slotIn, x0, y0, RAW, sMask, bar);
  const FirstAreas fa = first_areas<T>(g, x0, y0);
  const CellSrc<T> cs{g, a.A, a.B, RAW, sMask, x0, y0, (x0 - 2) - ((x0 - 2) & ~15)};
  const int xb = a.xoff[tileId], xn = a.xoff[tileId + 1] - xb;
  const int NP = T::NPT + 25 * xn, NF = T::NXF + T::NRF + 4 * xn;
  float4* sF = R;
  float4* sY = sF + NF;
  float* sO = reinterpret_cast<float*>(sY + NF);
  float* sAr = reinterpret_cast<float*>(R + stage_region_t<T>(xn));
  float4* sW = reinterpret_cast<float4*>(sAr) + (NF + 3) / 4;
  float4* sWb = sW + NP;
  for (int q = tid; q < xn; q += NT) xc[q] = a.xcell[xb + q];

  float dt, t;
  if (STAGE == 1) {
    float4 prev = *a.stPrev;
    float w = fmaxf(P.wFloor, __uint_as_float(*a.wIn));
    dt = fminf(P.cfl / w, P.dtMax);
    if (prev.x > 0.0f) dt = fminf(dt, prev.x * 1.2f);
    t = prev.z;                                   // inlet ramp at t_old
    if (tileId == 0 && tid == 0) {
      *a.stNew = make_float4(dt, prev.z, prev.z + dt, w);
      *a.wOut = 0u;
    }
  } else {
    float4 st = *a.stNew;
    dt = st.x;
    t = st.z;                                     // inlet ramp at t_new
  }
  __syncthreads();
  if (!halo_wait(bar, a.err)) return;
  load_prims<T>(g, a.A, a.B, t, P, x0, y0, xc, NP, RAW, sMask, sW, sWb);
  store_areas<T>(g, x0, y0, xc, xn, fa, sAr);
  __syncthreads();
  inviscid_faces<T>(g, P, xc, xn, sW, sWb, sF, sY, sO, sAr);
  __syncthreads();

  const int i = x0 + tid % TX, j = y0 + tid / TX;
  float wcell = 0.0f;
  if (tid < T::NC && i < Nx && j < Nr) {
    float4 oA, oB;
    const bool fluid = update_cell<T, STAGE>(a, cs, P, i, j, dt, t, x0, y0, xc, xn, sF, sY, sO, sAr, oA, oB);
    const int k = j * Nx + i;
    a.oA[k] = oA;
    a.oB[k] = oB;
    if (a.finalCfl && fluid) wcell = wave_speed(oA, oB);
  }
  if (a.finalCfl) block_max_to<NT>(wcell, a.wOut, red);
}

// --------------------------------------------------------------------------
// FS_VCELL of vcell slot k of the tile + 1 ring (k < NTT) or, after it, of a
// listed member's cell or one of its 4 neighbours (itself, W, E, S, N).
template <class T>
__device__ __forceinline__ void vcell_at(const Grid& g, const CellSrc<T>& cs, const rn_params& P, float dt, int x0,
                                         int y0, const int* xc, int k, const float4* sW, const float4* sWb,
                                         float4* sT1, float4* sT2) {
  const int Nx = g.Nx, Nr = g.Nr;
  int i, j, c, rs;
  if (k < T::NTT) {
    const int ly = k / T::TW, lx = k - ly * T::TW;
    i = x0 - 1 + lx; j = y0 - 1 + ly;
    c = (ly + 1) * T::PX + lx + 1;
    rs = T::PX;
  } else {
    const int q = k - T::NTT, e = q / 5, r = q - e * 5, m = xc[e];
    const int dx = r == 1 ? -1 : r == 2 ? 1 : 0, dy = r == 3 ? -1 : r == 4 ? 1 : 0;
    i = m % Nx + dx; j = m / Nx + dy;
    c = ext_prim<T>(e, dx, dy);
    rs = 5;
  }
  float4 T1 = make_float4(0.f, 0.f, 0.f, 0.f), T2 = T1;
  if (i >= 0 && i < Nx && j >= 0 && j < Nr)
    vcell(sW[c], sWb[c], sW[c + 1], sW[c - 1], sW[c + rs], sW[c - rs], i, j, cs.gm(i, j).w, dt, P, T1, T2);
  sT1[k] = T1;
  sT2[k] = T2;
}

// FS_VFLUX_X/R: every viscous face of the tile and of its listed members in
// one loop through one instance of the flux code (as the inviscid faces):
// primitive slots p1 (behind the face) and p2 (the face's cell), vcell slots
// v1 and v2; zero flux where it is not drawn or a side is a wall.
template <class T>
__device__ __forceinline__ void viscous_faces(const Grid& g, int x0, int y0, const int* xc, int xn, const float4* sW,
                                              const float4* sWb, const float4* sT1, const float4* sT2,
                                              const float* sAr, float4* sF, float4* sY) {
  constexpr int TX = T::TX, PX = T::PX, TW = T::TW, NXR = T::NXF + T::NRF;
  const int Nx = g.Nx, Nr = g.Nr;
  for (int k = threadIdx.x; k < NXR + 4 * xn; k += T::NT) {
    int i, j, p1, p2, v1, v2;
    bool dirR;
    if (k < NXR) {
      dirR = k >= T::NXF;
      // x-face k: row k / (TX + 1); r-face k - NXF: row (k - NXF) / TX (both
      // divisors compile-time constants)
      const int kx = k / (TX + 1), kr = (k - T::NXF) / TX;
      const int ly = dirR ? kr : kx, lx = dirR ? k - T::NXF - kr * TX : k - kx * (TX + 1);
      i = x0 + lx; j = y0 + ly;
      p2 = (ly + 2) * PX + lx + 2; p1 = p2 - (dirR ? PX : 1);
      v2 = (ly + 1) * TW + lx + 1; v1 = v2 - (dirR ? TW : 1);
    } else {                                     // member e's face w (W, E at mx + o; S, N at my + o)
      const int q = k - NXR, e = q >> 2, w = q & 3, o = w & 1, m = xc[e], vb = T::NTT + 5 * e;
      dirR = w >= 2;
      i = m % Nx + (dirR ? 0 : o); j = m / Nx + (dirR ? o : 0);
      p1 = dirR ? ext_prim<T>(e, 0, o - 1) : ext_prim<T>(e, o - 1, 0);
      p2 = p1 + (dirR ? 5 : 1);
      v1 = o ? vb : vb + (dirR ? 3 : 1);
      v2 = o ? vb + (dirR ? 4 : 2) : vb;
    }
    const bool ok = dirR ? (i < Nx && j > 0 && j < Nr) : (i > 0 && i < Nx && j < Nr);
    float4 F = make_float4(0.f, 0.f, 0.f, 0.f), FY = F;
    if (ok) {
      // face k is face k of the inviscid phase, whose open area sAr[k] holds
      // (every face drawn here was drawn there)
      const float area = sAr[k];
      const float4 w1 = sW[p1], w2 = sW[p2];
      if (area != 0.0f && !(w1.x < 0.0f || w2.x < 0.0f))
        visc_flux(dirR, w1, sWb[p1], sT1[v1], sT2[v1], w2, sWb[p2], sT1[v2], sT2[v2], j, F, FY);
    }
    sF[k] = F;
    sY[k] = FY;
  }
}

// FS_SOURCE of cell (i, j) inside the grid. A, B = the stage-2 state of the
// cell's group host; Bw = the cell's own stage-2 B.w. A1/B1 (global) feed
// the separation samples. Returns whether the cell is fluid.
template <class T>
__device__ __forceinline__ bool source_cell(const Grid& g, const CellSrc<T>& cs, const float4* __restrict__ A1,
                                            const float4* __restrict__ B1, const rn_params& P, int i, int j,
                                            float dt, int x0, int y0, const int* xc, int xn, const float4* sF,
                                            const float4* sY, const float* sAr, const float4* sT1,
                                            const float4* sT2, float4 A, float4 B, float Bw, float4& oA,
                                            float4& oB) {
  constexpr int TW = T::TW;
  const int Nx = g.Nx, Nr = g.Nr;
  const int k = j * Nx + i;
  const bool solid = cs.solid(i, j);
  const float4 gmij = cs.gm(i, j), gg = cs.gg(i, j);
  if (solid) {
    oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
    oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
    return false;
  }
  const int Hx = i + iround(gmij.x), Hy = j + iround(gmij.y), kh = Hy * Nx + Hx;
  Prim q = to_prim(A, B);
  float rho = q.w.x, p = q.w.w, G = q.s.z;
  float velx = q.w.y, vely = q.w.z;
  float V = fmaxf(gg.x, 1e-6f);
  float Rm = rmix(q.s, P), Tg = fdiv(p, rho * Rm);
  float4 L = make_float4(0.f, 0.f, 0.f, 0.f), LY = L;
  const int vh = (Hy - y0 + 1) * TW + (Hx - x0 + 1);
  float4 T1h = sT1[vh], T2h = sT2[vh];
  if (P.visc) {
    const int sm_ = iround(kh == k ? gmij.z : cs.gm(Hx, Hy).z);
    float LO = 0.0f;
    group_flux<T, false>(Hx, Hy, sm_, x0, y0, xc, xn, Nx, sF, sY, nullptr, sAr, L, LY, LO);
    // axisymmetric hoop stress
    float r = fdiv(V, fmaxf(gg.y, 1e-6f)), vor = fdiv(vely, r);
    L.z -= T2h.x * (2.0f * vor - 0.6666667f * (T1h.x + T1h.w + vor)) * gg.y;
    // Werner-Wengle wall shear and Reynolds-analogy heat flux
    float wl = len2(gg.z, gg.w);
    if (wl > 1e-6f) {
      const Over per_wl = over(wl);
      float nx = per_wl(gg.z), nr = per_wl(gg.w);
      float dn = velx * nx + vely * nr;
      float utx = velx - dn * nx, uty = vely - dn * nr;
      float up = len2(utx, uty);
      float cp = Rm * (G + 1.0f);
      float Taw = Tg + fdiv(0.89f * up * up, 2.0f * cp);
      float Ts = fmaxf(Tg + 0.5f * (P.Tw - Tg) + 0.22f * (Taw - Tg), 1e-3f);
      float rs = fdiv(p, Rm * Ts), mus = sutherland(Ts * P.gas[2], P);
      float dz = 2.0f * clampf(fdiv(0.5f * V, wl), 0.25f, 1.0f);
      float nz = fdiv(mus, rs * dz);
      float tw = up <= 69.7f * nz ? fdiv(2.0f * mus * up, dz)
                                  : rs * powf(7.187f * powf(nz, 1.142857f) + 0.13769f * powf(nz, 0.142857f) * up, 1.75f);
      tw = fminf(tw, fdiv(0.3f * rho * up * V, fmaxf(wl * dt, 1e-9f)));
      if (up > 1e-6f) { L.y -= fdiv(tw * wl * utx, up); L.z -= fdiv(tw * wl * uty, up); }
      float qw = fdiv(tw, fmaxf(up, 1e-4f)) * cp * (Taw - P.Tw) * 1.24f;
      float qmax = fdiv(0.3f * p * G * V, fmaxf(wl * dt, 1e-9f));
      L.w -= clampf(qw, -qmax, qmax) * wl;
    }
    // shock / boundary-layer interaction on the bit-16 band
    if (sm_ & 16) {
      float up = len2(velx, vely), Mn = fdiv(up, sqrtf(fdiv((1.0f + fdiv(1.0f, G)) * p, rho)));
      if (Mn > 1.0f) {
        float shx = fdiv(velx, up), shy = fdiv(vely, up);
        float pd = 0.0f;
        for (int n = 4; n <= 6; n += 2)
          for (int mm = 0; mm <= 1; mm++) {
            int Dx = Hx + int(rintf(float(n) * shx));
            int Dy = Hy + int(floorf(float(n) * shy)) + mm;
            Dx = min(max(Dx, 0), Nx - 1);
            Dy = min(max(Dy, 0), Nr - 1);
            float4 wd, sd;
            interior_prim(g, A1, B1, Dx, Dy, wd, sd);
            if (wd.x > 0.0f) pd = fmaxf(pd, wd.w);
          }
        float crit = 1.0f + 0.5f * Mn;
        float fsep = smoothstepf(crit, 1.2f * crit, fdiv(pd, p)) * V * rho * up;
        L.y -= fsep * velx;
        L.z -= fsep * vely;
      } else if (velx > 0.0f && p < 1.3f * P.chemK[3]) {
        float fsep = 0.5f * V * rho * up;
        L.y -= fsep * velx;
        L.z -= fsep * vely;
      }
    }
  }
  float invV = fdiv(dt, V);
  float dO = invV * L.x;
  L.x = 0.0f;
  float4 U = make_float4(A.x + invV * L.x, A.y + invV * L.y, A.z + invV * L.z, A.w + invV * L.w);
  float4 UY = make_float4(B.x + invV * LY.x / 1.0f, B.y + invV * LY.y / 1.0f, B.z + fdiv(invV * LY.z, rho),
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
  const Over per_rn = over(rn);
  float vnx = per_rn(U.y), vny = per_rn(U.z);
  if (!(rn < 1e30f) || !(vnx < 1e30f && vnx > -1e30f)) {
    oA = make_float4(P.ambCons[0], P.ambCons[1], P.ambCons[2], P.ambCons[3]);
    oB = make_float4(P.ambB[0], P.ambB[1], P.ambB[2], P.ambB[3]);
  } else {
    float Gn = clampf(UY.z, P.gamR[0], P.gamR[1]);
    float Zn = clampf(UY.x, 0.0f, rn);
    oA = make_float4(rn, rn * vnx, rn * vny, fmaxf(U.w, P_MIN * Gn + 0.5f * rn * (vnx * vnx + vny * vny)));
    oB = make_float4(Zn, clampf(UY.y, 0.0f, Zn), Gn, P.inj ? clampf(UY.w, 0.0f, rn) : Bw);
  }
  return true;
}

// Stage 2 and the split step fused on tile (bx, by): the stage-2 input
// primitives (the stage-1 state at t_new) are exactly what the split step
// reads (solver.js:940-941), so they are staged once; the stage-2 results of
// the tile's cells and of its listed members (every out-of-tile group host a
// tile cell can have) stay in shared memory and feed FS_SOURCE directly.
template <class T>
__host__ __device__ constexpr int fused_region_t(int maxX) {
  // float4 slots of the region that holds first the raw halo copy, then the
  // inviscid faces' F, Y and O, then (T::WIDE) the viscous faces' F and Y,
  // which need less, or the vcell ring's T1/T2 and the viscous faces
  return T::WIDE || (2 * (T::NXF + T::NRF + 4 * maxX) + ((T::NXF + T::NRF + 4 * maxX) + 3) / 4) >
                          (2 * (T::NTT + 5 * maxX) + 2 * (T::NXF + T::NRF + 4 * maxX))
             ? (2 * (T::NXF + T::NRF + 4 * maxX) + ((T::NXF + T::NRF + 4 * maxX) + 3) / 4)
             : (2 * (T::NTT + 5 * maxX) + 2 * (T::NXF + T::NRF + 4 * maxX));
}
template <class T>
__host__ __device__ constexpr int fused_region8_t(int maxX) {
  return (fused_region_t<T>(maxX) > 2 * T::NPT8 ? fused_region_t<T>(maxX) : 2 * T::NPT8);
}
template <class T>
__host__ __device__ constexpr size_t fused_smem_t(int maxX) {
  // alignment slack, mask block, face region, vcell T1/T2 (T::WIDE), stage-2
  // results, face areas, primitives
  return sizeof(float4) * (8 + T::MASKF4 + T::STAGED_F4 + fused_region8_t<T>(maxX) +
                           (T::WIDE ? 2 * (T::NTT + 5 * maxX) : 0) + 2 * (T::NC + maxX) +
                           (T::NXF + T::NRF + 4 * maxX + 3) / 4 + 2 * (T::NPT + 25 * maxX));
}
template <class T>
__device__ __forceinline__ void stage2_physics_body(const StageArgs& a, const PhysArgs& p, const rn_params& P, int bx,
                                                    int by, int tileId, float4* smRaw, float* red, int* xc,
                                                    uint64_t* bar) {
  constexpr int TX = T::TX, NT = T::NT;
  const Grid& g = a.g;
  const int Nx = g.Nx, Nr = g.Nr;
  const int tid = threadIdx.x;
  const int x0 = bx * TX, y0 = by * T::TY;
  float4* sm = aligned_smem(smRaw);
  uint8_t* sMask = reinterpret_cast<uint8_t*>(sm);
  float4* RAW = sm + T::MASKF4;                 // raw halo block (+ geometry boxes for WIDE shapes)
  float4* R = RAW + T::STAGED_F4;               // face region (other shapes: over the raw block)
  halo_issue<T>(a.tm, a.slotIn, x0, y0, RAW, sMask, bar);
  const FirstAreas fa = first_areas<T>(g, x0, y0);
  const CellSrc<T> cs{g, a.A, a.B, RAW, sMask, x0, y0, (x0 - 2) - ((x0 - 2) & ~15)};
  const int xb = a.xoff[tileId], xn = a.xoff[tileId + 1] - xb, xnP = P.visc ? xn : 0;
  const int NP = T::NPT + 25 * xn, NF = T::NXF + T::NRF + 4 * xn;
  const int NV = T::NTT + 5 * xnP;
  float4* sT1 = T::WIDE ? R + fused_region8_t<T>(xn) : R;
  float4* sT2 = sT1 + (T::WIDE ? T::NTT + 5 * xn : NV);
  float4* sA2 = T::WIDE ? sT2 + (T::NTT + 5 * xn) : R + fused_region8_t<T>(xn);
  float4* sB2 = sA2 + T::NC + xn;
  float* sAr = reinterpret_cast<float*>(sB2 + T::NC + xn);   // face areas, kept for FS_SOURCE
  float4* sW = reinterpret_cast<float4*>(sAr) + (NF + 3) / 4;
  float4* sWb = sW + NP;
  for (int q = tid; q < xn; q += NT) xc[q] = a.xcell[xb + q];
  const float4 st = *a.stNew;
  const float dt = st.x, t = st.z;
  __syncthreads();
  if (!halo_wait(bar, a.err)) return;
  load_prims<T>(g, a.A, a.B, t, P, x0, y0, xc, NP, RAW, sMask, sW, sWb);
  store_areas<T>(g, x0, y0, xc, xn, fa, sAr);
  __syncthreads();
  {
    float4* sF = R;
    float4* sY = sF + NF;
    float* sO = reinterpret_cast<float*>(sY + NF);
    inviscid_faces<T>(g, P, xc, xn, sW, sWb, sF, sY, sO, sAr);
    __syncthreads();
    // One flat list (T::WIDE): the stage-2 update of the tile's cells and of
    // its listed members, then FS_VCELL of the vcell slots. FS_VCELL reads only
    // the stage-2 input primitives, so it needs no barrier after the update,
    // and the list fills whole passes of the block. Otherwise FS_VCELL follows
    // in a phase of its own, its T1/T2 taking the faces' place.
    const int NU = T::NC + xn;
    for (int q = tid; q < NU + (T::WIDE ? NV : 0); q += NT) {
      if (q < NU) {                               // a tile cell (q == tid, NC <= NT), then a listed member
        int i, j;
        if (q < T::NC) { i = x0 + q % TX; j = y0 + q / TX; }
        else { const int m = xc[q - T::NC]; i = m % Nx; j = m / Nx; }
        if (i < Nx && j < Nr) {
          float4 oA, oB;
          update_cell<T, 2>(a, cs, P, i, j, dt, t, x0, y0, xc, xn, sF, sY, sO, sAr, oA, oB);
          sA2[q] = oA;
          sB2[q] = oB;
        }
      } else {
        vcell_at<T>(g, cs, P, dt, x0, y0, xc, q - NU, sW, sWb, sT1, sT2);
      }
    }
  }
  __syncthreads();
  const int NFV = T::NXF + T::NRF + 4 * xnP;
  float4* sF = T::WIDE ? R : sT2 + NV;
  float4* sY = sF + NFV;
  if (!T::WIDE) {
    for (int k = tid; k < NV; k += NT) vcell_at<T>(g, cs, P, dt, x0, y0, xc, k, sW, sWb, sT1, sT2);
    __syncthreads();
  }
  if (P.visc) viscous_faces<T>(g, x0, y0, xc, xnP, sW, sWb, sT1, sT2, sAr, sF, sY);
  __syncthreads();

  const int i = x0 + tid % TX, j = y0 + tid / TX;
  float wcell = 0.0f;
  if (tid < T::NC && i < Nx && j < Nr) {
    const int k = j * Nx + i;
    float4 oA, oB, A = make_float4(0.f, 0.f, 0.f, 0.f), B = A;
    float Bw = 0.0f;
    if (!cs.solid(i, j)) {
      float4 gm = cs.gm(i, j);
      const int Hx = i + iround(gm.x), Hy = j + iround(gm.y);
      const int hx = Hx - x0, hy = Hy - y0;
      int s;
      if (unsigned(hx) < unsigned(TX) && unsigned(hy) < unsigned(T::TY)) {
        s = hy * TX + hx;
      } else {
        const int kh = Hy * Nx + Hx;
        int e = 0;
        while (e < xn - 1 && xc[e] != kh) e++;
        s = T::NC + e;
      }
      A = sA2[s];
      B = sB2[s];
      Bw = sB2[tid].w;
    }
    const bool fluid = source_cell<T>(g, cs, p.A1, p.B1, P, i, j, dt, x0, y0, xc, xnP, sF, sY, sAr, sT1, sT2, A, B, Bw,
                                      oA, oB);
    p.oA[k] = oA;
    p.oB[k] = oB;
    if (p.finalCfl && fluid) wcell = wave_speed(oA, oB);
  }
  if (p.finalCfl) block_max_to<NT>(wcell, p.wOut, red);
}

// --------------------------------------------------------------------------
// Single-instance kernels: blockIdx = tile.
template <class T, int STAGE>
__global__ void __launch_bounds__(T::NT, T::MINB) k_stage(StageArgs a, rn_params P) {
  extern __shared__ float4 sm[];
  __shared__ float red[T::NT / 32];
  __shared__ int xc[MAXX];
  __shared__ uint64_t bar;
  stage_body<T, STAGE>(a, P, blockIdx.x, blockIdx.y, blockIdx.y * gridDim.x + blockIdx.x, sm, red, xc, &bar);
}
// heavy == nullptr: one block per tile of the grid, skipping tiles that list
// more than xSmall out-of-tile members (xSmall < 0: none skipped); otherwise
// block b runs tile heavy[b] (the skipped tiles, in a launch of their own with
// the shared memory their lists need).
template <class T>
__global__ void __launch_bounds__(T::NT, T::MINB) k_stage2phys(StageArgs a, PhysArgs p, rn_params P,
                                                               const int* heavy, int xSmall) {
  extern __shared__ float4 sm[];
  __shared__ float red[T::NT / 32];
  __shared__ int xc[MAXX];
  __shared__ uint64_t bar;
  int bx, by, tile;
  if (heavy) {
    const int tilesX = (a.g.Nx + T::TX - 1) / T::TX;
    tile = heavy[blockIdx.x];
    by = tile / tilesX;
    bx = tile - by * tilesX;
  } else {
    bx = blockIdx.x;
    by = blockIdx.y;
    tile = by * gridDim.x + bx;
    if (xSmall >= 0 && a.xoff[tile + 1] - a.xoff[tile] > xSmall) return;
  }
  stage2_physics_body<T>(a, p, P, bx, by, tile, sm, red, xc, &bar);
}

// Batch kernels: block b belongs to instance blockInst[b]; its descriptor
// (buffers, ring position) is staged in shared memory, and thread 0 derives
// the step's kernel arguments from it into shared memory too: the body reads
// each field from there when it needs it, where arguments built in registers
// would stay live across the whole body (and spill). The parameter block is
// read in place from the read-only descriptor array, so the compiler can
// reload a field rather than spill it.
__device__ __forceinline__ void load_inst(const BatchInst* insts, int inst, BatchInst& d) {
  __shared__ int di;
  if (threadIdx.x == 0) di = inst;
  __syncthreads();
  const int* src = reinterpret_cast<const int*>(insts + di);
  int* dst = reinterpret_cast<int*>(&d);
  for (int q = threadIdx.x; q < int(sizeof(BatchInst) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
  __syncthreads();
}
// The step's stage arguments of instance d (stage 1 or 2 + the split step).
__device__ __forceinline__ void batch_stage_args(const BatchInst& d, const BatchPhase& ph, int stage, StageArgs& a) {
  const int s0 = (d.cur0 + ph.shift) % 3, s1 = (s0 + 1) % 3, s2 = (s0 + 2) % 3;
  const int si = d.stepIdx0 ^ ph.par, ws = d.wslot0 ^ ph.par;
  a.g = d.g;
  if (stage == 1) {
    a.A = d.SA[s0]; a.B = d.SB[s0]; a.A0 = d.SA[s0]; a.B0 = d.SB[s0]; a.oA = d.SA[s1]; a.oB = d.SB[s1];
  } else {
    a.A = d.SA[s1]; a.B = d.SB[s1]; a.A0 = d.SA[s0]; a.B0 = d.SB[s0]; a.oA = d.SA[s2]; a.oB = d.SB[s2];
  }
  a.stPrev = d.stepTex + si;
  a.stNew = d.stepTex + (1 - si);
  a.wIn = d.wmax + ws;
  a.wOut = d.wmax + (1 - ws);
  a.finalCfl = ph.finalCfl;
  a.xoff = d.xoff; a.xcell = d.xcell; a.maxX = ph.maxX;
  a.slotIn = stage == 1 ? s0 : s1;
  a.tm = d.tm;
  a.err = d.err;
}
template <class T, int STAGE>
__global__ void __launch_bounds__(T::NT, T::MINB) k_stage_batch(const BatchInst* __restrict__ insts, const int* blockInst, BatchPhase ph) {
  extern __shared__ float4 sm[];
  __shared__ float red[T::NT / 32];
  __shared__ int xc[MAXX];
  __shared__ uint64_t bar;
  __shared__ BatchInst d;
  __shared__ StageArgs a;
  const int inst = blockInst[blockIdx.x];
  if (ph.active && !ph.active[inst]) return;      // a member stopped by rn_batch_run: the whole block
  load_inst(insts, inst, d);
  if (threadIdx.x == 0) batch_stage_args(d, ph, STAGE, a);
  __syncthreads();
  const int local = blockIdx.x - d.firstBlock, by = local / d.tilesX, bx = local - by * d.tilesX;
  stage_body<T, STAGE>(a, insts[inst].P, bx, by, local, sm, red, xc, &bar);
}
template <class T>
__global__ void __launch_bounds__(T::NT, T::MINB) k_stage2phys_batch(const BatchInst* __restrict__ insts, const int* blockInst,
                                                                     BatchPhase ph, const int2* heavy, int xSmall) {
  extern __shared__ float4 sm[];
  __shared__ float red[T::NT / 32];
  __shared__ int xc[MAXX];
  __shared__ uint64_t bar;
  __shared__ BatchInst d;
  __shared__ StageArgs a;
  __shared__ PhysArgs p;
  const int2 hv = heavy ? heavy[blockIdx.x] : make_int2(0, 0);   // (member, tile) of a heavy block
  const int inst = heavy ? hv.x : blockInst[blockIdx.x];
  if (ph.active && !ph.active[inst]) return;      // a member stopped by rn_batch_run: the whole block
  load_inst(insts, inst, d);
  const int local = heavy ? hv.y : blockIdx.x - d.firstBlock, by = local / d.tilesX, bx = local - by * d.tilesX;
  if (!heavy && xSmall >= 0 && d.xoff[local + 1] - d.xoff[local] > xSmall) return;   // in the heavy launch
  if (threadIdx.x == 0) {
    batch_stage_args(d, ph, 2, a);
    a.finalCfl = 0;
    const int s0 = (d.cur0 + ph.shift) % 3, s1 = (s0 + 1) % 3, s2 = (s0 + 2) % 3;
    const int si = d.stepIdx0 ^ ph.par, ws = d.wslot0 ^ ph.par;
    p.g = d.g;
    p.A1 = d.SA[s1]; p.B1 = d.SB[s1]; p.A2 = d.SA[s2]; p.B2 = d.SB[s2]; p.oA = d.SA[s2]; p.oB = d.SB[s2];
    p.st = d.stepTex + (1 - si);
    p.wOut = d.wmax + (1 - ws);
    p.finalCfl = ph.finalCfl;
    p.xoff = d.xoff; p.xcell = d.xcell; p.maxX = ph.maxX;
  }
  __syncthreads();
  stage2_physics_body<T>(a, p, insts[inst].P, bx, by, local, sm, red, xc, &bar);
}

// --------------------------------------------------------------------------
// stand-alone CFL reduction of a state (first step after setState/rescale)
constexpr int RED_NT = 256;
__global__ void __launch_bounds__(RED_NT) k_reduce(Grid g, const float4* __restrict__ A,
                                                   const float4* __restrict__ B, unsigned* out) {
  __shared__ float red[RED_NT / 32];
  const int N = g.Nx * g.Nr;
  float w = 0.0f;
  for (int k = blockIdx.x * RED_NT + threadIdx.x; k < N; k += gridDim.x * RED_NT)
    if (!g.mask[k]) w = fmaxf(w, wave_speed(A[k], B[k]));
  block_max_to<RED_NT>(w, out, red);
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
  __shared__ double bs[32], bc[32];
  bs[threadIdx.x] = n.s;
  bc[threadIdx.x] = n.c;
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
// launchers
template <class T>
static dim3 tiles_of(const Grid& g) {
  return dim3((g.Nx + T::TX - 1) / T::TX, (g.Nr + T::TY - 1) / T::TY);
}

template <class T>
static int init_tile() {
  const int ss = int(stage_smem_t<T>(MAXX)), ps = int(fused_smem_t<T>(MAXX));
  if (cudaFuncSetAttribute(k_stage<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_stage<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_stage2phys<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, ps) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_stage_batch<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss) != cudaSuccess)
    return -1;
  if (cudaFuncSetAttribute(k_stage_batch<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, ss) != cudaSuccess)
    return -1;
  if (cudaFuncSetAttribute(k_stage2phys_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, ps) != cudaSuccess)
    return -1;
  return 0;
}
// Raises the dynamic shared-memory limits of the stage and physics kernels to
// what a member list of MAXX cells needs (process-wide function attributes).
int stage_kernels_init() {
  return (init_tile<Tile0>() == 0 && init_tile<Tile1>() == 0 && init_tile<Tile2>() == 0 && init_tile<Tile3>() == 0 &&
          init_tile<Tile4>() == 0)
             ? 0
             : -1;
}

void launch_stage1(const StageArgs& a, const rn_params& P, int tile, cudaStream_t s) {
  if (tile == 4) k_stage<Tile4, 1><<<tiles_of<Tile4>(a.g), Tile4::NT, stage_smem_t<Tile4>(a.maxX), s>>>(a, P);
  else if (tile == 3) k_stage<Tile3, 1><<<tiles_of<Tile3>(a.g), Tile3::NT, stage_smem_t<Tile3>(a.maxX), s>>>(a, P);
  else if (tile == 2) k_stage<Tile2, 1><<<tiles_of<Tile2>(a.g), Tile2::NT, stage_smem_t<Tile2>(a.maxX), s>>>(a, P);
  else if (tile == 1) k_stage<Tile1, 1><<<tiles_of<Tile1>(a.g), Tile1::NT, stage_smem_t<Tile1>(a.maxX), s>>>(a, P);
  else k_stage<Tile0, 1><<<tiles_of<Tile0>(a.g), Tile0::NT, stage_smem_t<Tile0>(a.maxX), s>>>(a, P);
}
void launch_stage2(const StageArgs& a, const rn_params& P, int tile, cudaStream_t s) {
  if (tile == 4) k_stage<Tile4, 2><<<tiles_of<Tile4>(a.g), Tile4::NT, stage_smem_t<Tile4>(a.maxX), s>>>(a, P);
  else if (tile == 3) k_stage<Tile3, 2><<<tiles_of<Tile3>(a.g), Tile3::NT, stage_smem_t<Tile3>(a.maxX), s>>>(a, P);
  else if (tile == 2) k_stage<Tile2, 2><<<tiles_of<Tile2>(a.g), Tile2::NT, stage_smem_t<Tile2>(a.maxX), s>>>(a, P);
  else if (tile == 1) k_stage<Tile1, 2><<<tiles_of<Tile1>(a.g), Tile1::NT, stage_smem_t<Tile1>(a.maxX), s>>>(a, P);
  else k_stage<Tile0, 2><<<tiles_of<Tile0>(a.g), Tile0::NT, stage_smem_t<Tile0>(a.maxX), s>>>(a, P);
}
// heavy != nullptr: the heavy tiles alone (nHeavy blocks, shared memory for
// their lists); otherwise every tile, with the heavy ones skipped when `skip`
// (they then run in the other launch, on another stream at the same time).
template <class T>
static void stage2phys_t(const StageArgs& a, const PhysArgs& p, const rn_params& P, const int* heavy, int nHeavy,
                         bool skip, cudaStream_t s) {
  if (heavy) {
    k_stage2phys<T><<<nHeavy, T::NT, fused_smem_t<T>(a.maxX), s>>>(a, p, P, heavy, -1);
  } else if (skip) {
    const int xs = a.maxX < XSMALL ? a.maxX : XSMALL;
    k_stage2phys<T><<<tiles_of<T>(a.g), T::NT, fused_smem_t<T>(xs), s>>>(a, p, P, nullptr, XSMALL);
  } else {
    k_stage2phys<T><<<tiles_of<T>(a.g), T::NT, fused_smem_t<T>(a.maxX), s>>>(a, p, P, nullptr, -1);
  }
}
void launch_stage2phys(const StageArgs& a, const PhysArgs& p, const rn_params& P, int tile, const int* heavy,
                       int nHeavy, bool skip, cudaStream_t s) {
  if (tile == 4) stage2phys_t<Tile4>(a, p, P, heavy, nHeavy, skip, s);
  else if (tile == 3) stage2phys_t<Tile3>(a, p, P, heavy, nHeavy, skip, s);
  else if (tile == 2) stage2phys_t<Tile2>(a, p, P, heavy, nHeavy, skip, s);
  else if (tile == 1) stage2phys_t<Tile1>(a, p, P, heavy, nHeavy, skip, s);
  else stage2phys_t<Tile0>(a, p, P, heavy, nHeavy, skip, s);
}
void launch_batch_stage1(const BatchInst* d, const int* bi, int nb, BatchPhase ph, int tile, cudaStream_t s) {
  if (tile == 4) k_stage_batch<Tile4, 1><<<nb, Tile4::NT, stage_smem_t<Tile4>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 3) k_stage_batch<Tile3, 1><<<nb, Tile3::NT, stage_smem_t<Tile3>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 2) k_stage_batch<Tile2, 1><<<nb, Tile2::NT, stage_smem_t<Tile2>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 1) k_stage_batch<Tile1, 1><<<nb, Tile1::NT, stage_smem_t<Tile1>(ph.maxX), s>>>(d, bi, ph);
  else k_stage_batch<Tile0, 1><<<nb, Tile0::NT, stage_smem_t<Tile0>(ph.maxX), s>>>(d, bi, ph);
}
void launch_batch_stage2(const BatchInst* d, const int* bi, int nb, BatchPhase ph, int tile, cudaStream_t s) {
  if (tile == 4) k_stage_batch<Tile4, 2><<<nb, Tile4::NT, stage_smem_t<Tile4>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 3) k_stage_batch<Tile3, 2><<<nb, Tile3::NT, stage_smem_t<Tile3>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 2) k_stage_batch<Tile2, 2><<<nb, Tile2::NT, stage_smem_t<Tile2>(ph.maxX), s>>>(d, bi, ph);
  else if (tile == 1) k_stage_batch<Tile1, 2><<<nb, Tile1::NT, stage_smem_t<Tile1>(ph.maxX), s>>>(d, bi, ph);
  else k_stage_batch<Tile0, 2><<<nb, Tile0::NT, stage_smem_t<Tile0>(ph.maxX), s>>>(d, bi, ph);
}
template <class T>
static void batch_stage2phys_t(const BatchInst* d, const int* bi, int nb, BatchPhase ph, const int2* heavy,
                               int nHeavy, bool skip, cudaStream_t s) {
  if (heavy) {
    k_stage2phys_batch<T><<<nHeavy, T::NT, fused_smem_t<T>(ph.maxX), s>>>(d, bi, ph, heavy, -1);
  } else if (skip) {
    BatchPhase pl = ph;
    pl.maxX = ph.maxX < XSMALL ? ph.maxX : XSMALL;
    k_stage2phys_batch<T><<<nb, T::NT, fused_smem_t<T>(pl.maxX), s>>>(d, bi, pl, nullptr, XSMALL);
  } else {
    k_stage2phys_batch<T><<<nb, T::NT, fused_smem_t<T>(ph.maxX), s>>>(d, bi, ph, nullptr, -1);
  }
}
void launch_batch_stage2phys(const BatchInst* d, const int* bi, int nb, BatchPhase ph, int tile, const int2* heavy,
                             int nHeavy, bool skip, cudaStream_t s) {
  if (tile == 4) batch_stage2phys_t<Tile4>(d, bi, nb, ph, heavy, nHeavy, skip, s);
  else if (tile == 3) batch_stage2phys_t<Tile3>(d, bi, nb, ph, heavy, nHeavy, skip, s);
  else if (tile == 2) batch_stage2phys_t<Tile2>(d, bi, nb, ph, heavy, nHeavy, skip, s);
  else if (tile == 1) batch_stage2phys_t<Tile1>(d, bi, nb, ph, heavy, nHeavy, skip, s);
  else batch_stage2phys_t<Tile0>(d, bi, nb, ph, heavy, nHeavy, skip, s);
}
void launch_reduce(const Grid& g, const float4* A, const float4* B, unsigned* w, cudaStream_t s) {
  int N = g.Nx * g.Nr;
  int blocks = (N + RED_NT - 1) / RED_NT;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_reduce<<<blocks, RED_NT, 0, s>>>(g, A, B, w);
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

}  // namespace RN_VARIANT
}  // namespace rn
