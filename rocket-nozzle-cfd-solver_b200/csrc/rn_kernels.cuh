// rn_kernels.cuh -- kernel argument blocks and the kernel sets shared by the
// step kernels (rn_step.cu), the spray kernels (rn_spray.cu) and the C-ABI
// (rn_api.cu, rn_batch.cu).
#pragma once
#include <cuda_runtime.h>
#include "rn_math.cuh"
#include "rn_tma.cuh"

namespace rn {

// Tile shapes of the stage/physics blocks: TX x TY cells on TILE_NT threads,
// a thread per cell (threads beyond TX*TY idle in the cell phases). 16x15 on
// 256 threads (the default) has 511 faces, so its face phase is exactly two
// passes of the block, where 16x16's 544 faces need a third pass for one warp
// while the other seven wait at the barrier. Measured on B200 (fast
// precision, G cell-updates/s, 16x16 / 16x8 / 16x15 / 32x15): viscous
// 512x192 2.43 / 2.31 / 2.47 / 2.26, viscous 1024x384 3.67 / 3.26 / 4.00 /
// 3.99, plain 4096x1536 5.51 / 5.49 / 5.73 / 5.51, 64 batched instances
// 3.59 / 3.07 / 4.05 / 3.98. (16x16 itself beat 32x8 by 4.5-17 %.) The
// autotuner picks per handle or batch.
// 14x16 spreads a 512x192 grid over 37 x 12 = 444 tiles, 3 per SM on 148 SMs,
// and is compiled for those 3 blocks (24 warps: 80 registers, no spills); the
// others for 32 resident warps (64 registers).
constexpr int NTILES = 5;
constexpr int TILE_TX[NTILES] = {16, 16, 16, 32, 14};
constexpr int TILE_TY[NTILES] = {16, 8, 15, 15, 16};
constexpr int TILE_NT[NTILES] = {256, 128, 256, 512, 256};
constexpr int TILE_WARPS[NTILES] = {32, 32, 32, 32, 24};
// Most out-of-tile group members one tile may list (set_geometry rejects more).
constexpr int MAXX = 64;
// Tiles listing more out-of-tile members than this run the fused stage-2 +
// split-step kernel in a launch of their own, sized for them, so that the
// shared memory of every other block stays within 4 blocks per SM (a 1024x384
// bell has a wall tile with 16; it cost the whole launch a quarter of its
// occupancy).
constexpr int XSMALL = 4;
// The split (a side-stream launch joined back) pays only on grids of many
// waves: more tiles than SPLIT_BLOCKS_PER_SM x SMs. Measured with 16x16 tiles:
// 64 batched instances (36,400 blocks) 3.59 -> 3.97 G cell-updates/s; a lone
// 1024x384 grid (1,536 blocks) 3.67 -> 3.60, so it is not split.
constexpr int SPLIT_BLOCKS_PER_SM = 16;

struct StageArgs {
  Grid g;
  const float4* A;  const float4* B;    // stage input state
  const float4* A0; const float4* B0;   // state at t^n (stage 2)
  float4* oA; float4* oB;               // stage output
  const float4* stPrev;                 // stage 1: step info of the previous step
  float4* stNew;                        // stage 1 writes it, later kernels read it
  const unsigned* wIn;                  // stage 1: max wave speed of the step's input state
  unsigned* wOut;                       // cleared by stage 1, accumulated by the step's last kernel
  int finalCfl;                         // this kernel writes the step's final state
  const int* xoff;                      // per tile: out-of-tile members of its cut-cell groups (CSR)
  const int* xcell;
  int maxX;                             // largest per-tile list (sizes the dynamic shared memory)
  int slotIn;                           // ring slot of (A, B): selects the tensor maps of the halo copy
  const TileMaps* tm;                   // the handle's tensor maps, one TileMaps per tile shape
  unsigned* err;                        // set when a halo copy did not complete in time
};

struct PhysArgs {
  Grid g;
  const float4* A1; const float4* B1;   // stage-1 result (its primitives feed the viscous terms)
  const float4* A2; const float4* B2;   // stage-2 result (slot; the fused kernel keeps it on chip)
  float4* oA; float4* oB;
  const float4* st;
  unsigned* wOut;
  int finalCfl;
  const int* xoff;
  const int* xcell;
  int maxX;
};

struct SprayArgs {
  Grid g;
  const float4* A1; const float4* B1;   // stage-1 state: the gas the parcels see
  const float4* PA; const float4* PB;   // parcels before the step
  float4* oPA; float4* oPB; float4* oPC;
  const float4* tab;                    // 256 x 3 injector table
  const float4* st;
  unsigned* key; unsigned* val; float4* dep;   // deposit records (cell key, parcel index, source)
  unsigned long long* acc;              // fixed-point deposit sums of this step, 4 per cell (fast variant)
  unsigned* depFlag;                    // set when a deposit left the fixed-point range (fast variant)
  const unsigned* boundIn;              // (mass, speed) bounds of the ring this step reads (float bits)
  unsigned* boundOut;                   // the same for the ring it writes: max of boundIn and its parcels
  unsigned long long* liveSteps;        // += live parcels this step writes (parcel-steps counter)
  int head, seed;
  const unsigned* hs;                   // if set: (head, seed) read here instead (graph replay)
};

struct ApplyArgs {
  Grid g;
  const float4* A; const float4* B;
  const float4* src;
  const unsigned long long* acc;        // this step's fixed-point deposit sums (fast variant)
  const unsigned* boundIn;              // the (mass, speed) bounds its deposits were scaled by
  unsigned long long* accNext;          // the next step's, cleared here cell by cell
  float4* oA; float4* oB;
  unsigned* wOut;
  int finalCfl;
  unsigned* hsNext;                     // if set: (head, seed) advanced by one step here (graph replay)
};

// One instance of a batch: its buffers, where it stood in its state ring and
// step-info ping-pong when the batch was (re)built, its first block in the
// batch grid, and its parameter block. The kernels derive the slots of step k
// from (cur0, stepIdx0, wslot0) and the step's BatchPhase.
struct BatchInst {
  Grid g;
  float4* SA[3];
  float4* SB[3];
  float4* stepTex;                      // 2 float4
  unsigned* wmax;                       // 2 slots
  const int* xoff;
  const int* xcell;
  const TileMaps* tm;                   // the member's tensor maps, one TileMaps per tile shape
  unsigned* err;                        // the member's error word (halo copy timeout)
  int cur0, stepIdx0, wslot0;
  int firstBlock, tilesX;
  int pad_;
  rn_params P;
};
struct BatchPhase {
  int shift;                            // ring offset of this step: state slot s0 = (cur0 + shift) % 3
  int par;                              // step parity: stepIdx = stepIdx0 ^ par, wslot = wslot0 ^ par
  int finalCfl;                         // the launched kernel writes the step's final state
  int maxX;
  const int* active;                    // if set: per member, 0 = stopped (its blocks return at once)
};

// The kernels are compiled twice from the same sources (rn_variant.cu):
//   exact -- IEEE division and square root: every float operation rounds as
//            written, so the state matches the CPU oracle bit for bit wherever
//            pow/exp/log/sin/cos agree with the host's libm;
//   fast  -- the hardware's approximate division (div.full) and square root
//            (within 2 ulp, the latitude GLSL highp gives the reference's
//            shaders); agrees with the oracle to ~1e-6 relative L2.
// A solver handle launches through one of the two sets; `tile` selects the
// tile shape (index into TILE_TX/TILE_TY).
struct KernelSet {
  const char* name;
  void (*stage1)(const StageArgs& a, const rn_params& P, int tile, cudaStream_t s);
  void (*stage2)(const StageArgs& a, const rn_params& P, int tile, cudaStream_t s);
  // stage 2 + the viscous/wall/reaction split step in one kernel
  // heavy != nullptr: launch the tiles listing more than XSMALL out-of-tile
  // members (nHeavy of them); else all tiles, skipping those when `skip`
  void (*stage2phys)(const StageArgs& a, const PhysArgs& p, const rn_params& P, int tile, const int* heavy,
                     int nHeavy, bool skip, cudaStream_t s);
  void (*batchStage1)(const BatchInst* d, const int* blockInst, int nblocks, BatchPhase ph, int tile, cudaStream_t s);
  void (*batchStage2)(const BatchInst* d, const int* blockInst, int nblocks, BatchPhase ph, int tile, cudaStream_t s);
  void (*batchStage2Phys)(const BatchInst* d, const int* blockInst, int nblocks, BatchPhase ph, int tile,
                          const int2* heavy, int nHeavy, bool skip, cudaStream_t s);
  void (*reduce)(const Grid& g, const float4* A, const float4* B, unsigned* w, cudaStream_t s);
  void (*rescale)(const Grid& g, const float4* A, const float4* B, float4* oA, float4* oB, float fp, float fT,
                  float du, const rn_params& P, cudaStream_t s);
  void (*wallrow)(const Grid& g, const float4* A, const float4* B, const float4* jw, float4* row, cudaStream_t s);
  void (*integrals)(const Grid& g, const float4* A, const float4* B, const float4* geoAx,
                    const rn_integral_spec& spec, const float4* st, double* out, cudaStream_t s);
  int (*spray)(const SprayArgs& a, const rn_params& P, void* sortTemp, size_t sortTempBytes, unsigned* keyOut,
               unsigned* valOut, float4* src, cudaStream_t s, int* launches);
  void (*apply)(const ApplyArgs& a, const rn_params& P, cudaStream_t s);
  size_t (*sortTempBytes)(int Ncells);
  int (*init)();                    // opts the kernels into the dynamic shared memory they need
};
extern const KernelSet kernels_exact;
extern const KernelSet kernels_fast;

}  // namespace rn
