// rn_batch.cu -- batched stepping of many solver handles (declared in rn.h).
//
// No reference counterpart: the reference runs one grid per browser page
// (solver.js:849-891 steps it). A batch is the serving form of the same step:
// every tile of every member is one block of a single 1-D launch per kernel
// kind, so small grids share the 148 SMs instead of each leaving most of them
// idle, and a step of the whole batch costs 2 launches instead of 2 per
// member.
//
// Each block finds its member in a block->member table and that member's
// descriptor (BatchInst: buffers, ring position, parameter block) in a device
// array. The descriptor's ring position is normalised to the batch's step
// counter, so it stays the same from call to call while the members are only
// stepped by the batch, and the launch sequence repeats with a period of 6
// steps (3 ring shifts x 2 step-info parities). Without sprays that period is
// captured once in a CUDA graph and replayed.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include "rn.h"
#include "rn_internal.h"

using namespace rn;

namespace {
constexpr int PERIOD = 6;
constexpr int SPRAY_N = 65536;

struct Flags {
  int visc = 0, chem = 0, inj = 0;
  bool phys() const { return visc || chem; }
  // how far the state ring turns per step (rn_step's slot bookkeeping): the
  // step's kernels write s1, then s2 (stage 2, or stage 2 fused with the
  // split step); the spray apply writes the slot after s2
  int delta() const { return inj ? 0 : 2; }
  bool operator==(const Flags& o) const { return visc == o.visc && chem == o.chem && inj == o.inj; }
};
Flags flags_of(const rn_params& P) {
  Flags f;
  f.visc = P.visc != 0;
  f.chem = P.chem != 0;
  f.inj = P.inj != 0;
  return f;
}
}  // namespace

struct rn_batch_t {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;           // end of the last rn_batch_step
  cudaEvent_t staged = nullptr;         // the last descriptor upload has read the pinned buffer
  int tile = RN_TILE_16x15;
  Flags flags;
  std::vector<rn_solver*> members;
  std::vector<rn_params> params;
  std::vector<cudaEvent_t> fence;       // per member: its stream's work before a batch step
  int ctr = 0;                          // steps since the descriptors were normalised, mod PERIOD
  // device tables and their host images
  BatchInst* dInst = nullptr;
  size_t instCap = 0;
  int* dBlock = nullptr;
  size_t blockCap = 0;
  BatchInst* hInst = nullptr;           // pinned staging
  size_t hInstCap = 0;
  std::vector<BatchInst> uploaded;      // what dInst holds
  std::vector<int> layout;              // (Nx, Nr) per member the block table was built for
  int nblocks = 0, maxX = 1;
  int2* dHeavy = nullptr;               // (member, tile) of the tiles with long out-of-tile lists
  size_t heavyCap = 0;
  std::vector<int2> heavy;              // what dHeavy holds
  int nHeavy = 0;
  bool split = false;                   // heavy tiles run beside the main launch (see XSMALL)
  int numSMs = 148;
  cudaStream_t side = nullptr;
  cudaEvent_t evFork = nullptr, evJoin = nullptr;
  cudaStream_t sprayStream = nullptr;   // the members' parcel steps, beside stage 2 + the split step
  cudaEvent_t evSprayFork = nullptr, evSprayJoin = nullptr;
  const KernelSet* K = nullptr;
  // the graph of one period
  cudaGraphExec_t graph = nullptr;
  const KernelSet* graphK = nullptr;
  int graphBlocks = -1, graphTile = -1, graphMaxX = -1, graphHeavy = -1;
  Flags graphFlags;
  const int* graphActive = nullptr;
  long long launches = 0;
  // rn_batch_run: per member, whether it still steps (empty outside a run);
  // the same flags on the device, read by the kernels and the gate
  std::vector<char> runActive;
  int* dActive = nullptr;
  double* dTEnd = nullptr;
  int* dGate = nullptr;                 // 2 gate outputs: active count, then the flags
  int* hGate = nullptr;                 // pinned copies of them
  cudaEvent_t evGate[2] = {nullptr, nullptr};   // each copy's arrival
  size_t runCap = 0;
};

namespace {

int bfail(int code, const std::string& msg) { return rn_record_error(code, msg); }
#define BCK(call)                                             \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return rn_record_cuda(e_, #call);  \
  } while (0)

void drop_graph(rn_batch_t* b) {
  if (b->graph) cudaGraphExecDestroy(b->graph);
  b->graph = nullptr;
  b->graphK = nullptr;
  b->graphBlocks = b->graphTile = b->graphMaxX = b->graphHeavy = -1;
}

int index_of(const rn_batch_t* b, const rn_solver* h) {
  for (size_t m = 0; m < b->members.size(); m++)
    if (b->members[m] == h) return int(m);
  return -1;
}

// Normalised ring position of member h at batch step counter ctr: the kernels
// of batch step c use slot (cur0 + c*delta) % 3 and parity stepIdx0 ^ (c & 1).
void normalise(const rn_batch_t* b, const rn_solver* h, int& cur0, int& si0, int& ws0) {
  const int sh = (b->ctr * b->flags.delta()) % 3, par = b->ctr & 1;
  cur0 = (h->cur - sh + 3) % 3;
  si0 = h->stepIdx ^ par;
  ws0 = h->wslot ^ par;
}

// Brings the block table, the descriptors on the device and the members'
// member lists up to date with the handles.
int refresh(rn_batch_t* b) {
  const int nm = int(b->members.size());
  const int TX = TILE_TX[b->tile], TY = TILE_TY[b->tile];
  // block table: rebuilt when a member's grid size changed
  // (members stopped in a run have no blocks: grid size 0 x 0 in the table)
  std::vector<int> layout(2 * nm);
  for (int m = 0; m < nm; m++) {
    const bool on = b->runActive.empty() || b->runActive[m];
    layout[2 * m] = on ? b->members[m]->Nx : 0;
    layout[2 * m + 1] = on ? b->members[m]->Nr : 0;
  }
  std::vector<int> first(nm), tilesX(nm);
  int nb = 0;
  for (int m = 0; m < nm; m++) {
    first[m] = nb;
    tilesX[m] = (b->members[m]->Nx + TX - 1) / TX;
    nb += ((layout[2 * m] + TX - 1) / TX) * ((layout[2 * m + 1] + TY - 1) / TY);
  }
  if (layout != b->layout || nb != b->nblocks) {
    std::vector<int> table(std::max(nb, 1), 0);
    for (int m = 0; m < nm; m++)
      for (int q = first[m]; q < (m + 1 < nm ? first[m + 1] : nb); q++) table[q] = m;
    BCK(cudaStreamSynchronize(b->stream));
    if (size_t(nb) > b->blockCap) {
      cudaFree(b->dBlock);
      b->dBlock = nullptr;
      b->blockCap = 0;
      BCK(cudaMalloc(&b->dBlock, sizeof(int) * size_t(nb)));
      b->blockCap = size_t(nb);
    }
    BCK(cudaMemcpy(b->dBlock, table.data(), sizeof(int) * table.size(), cudaMemcpyHostToDevice));
    b->layout = layout;
    b->nblocks = nb;
  }
  // descriptors: uploaded when one differs from what the device holds
  std::vector<BatchInst> inst(nm);
  int maxX = 1;
  for (int m = 0; m < nm; m++) {
    const rn_solver* h = b->members[m];
    BatchInst& d = inst[m];
    std::memset(&d, 0, sizeof(d));
    d.g = h->grid();
    for (int s = 0; s < 3; s++) {
      d.SA[s] = h->SA[s];
      d.SB[s] = h->SB[s];
    }
    d.stepTex = h->stepTex;
    d.wmax = h->wmax;
    d.tm = h->dMaps;
    d.err = h->errFlag;
    d.xoff = h->xoff;
    d.xcell = h->xcell;
    normalise(b, h, d.cur0, d.stepIdx0, d.wslot0);
    d.firstBlock = first[m];
    d.tilesX = tilesX[m];
    d.P = b->params[m];
    maxX = std::max(maxX, h->maxX);
  }
  b->maxX = maxX;
  // heavy tiles: their own fused launch (see XSMALL)
  std::vector<int2> heavy;
  for (int m = 0; m < nm; m++) {
    if (!b->runActive.empty() && !b->runActive[m]) continue;
    const std::vector<int>& off = b->members[m]->hostXoff;
    for (size_t t = 0; t + 1 < off.size(); t++)
      if (off[t + 1] - off[t] > XSMALL) heavy.push_back(make_int2(m, int(t)));
  }
  const bool heavySame = heavy.size() == b->heavy.size() &&
                         (heavy.empty() || std::memcmp(heavy.data(), b->heavy.data(), sizeof(int2) * heavy.size()) == 0);
  if (!heavySame) {
    BCK(cudaStreamSynchronize(b->stream));
    if (heavy.size() > b->heavyCap) {
      cudaFree(b->dHeavy);
      b->dHeavy = nullptr;
      b->heavyCap = 0;
      BCK(cudaMalloc(&b->dHeavy, sizeof(int2) * heavy.size()));
      b->heavyCap = heavy.size();
      drop_graph(b);
    }
    if (!heavy.empty())
      BCK(cudaMemcpy(b->dHeavy, heavy.data(), sizeof(int2) * heavy.size(), cudaMemcpyHostToDevice));
    b->heavy = heavy;
    b->nHeavy = int(heavy.size());
  }
  b->split = b->nHeavy > 0 && b->nblocks > SPLIT_BLOCKS_PER_SM * b->numSMs;
  const bool same = inst.size() == b->uploaded.size() &&
                    (inst.empty() || std::memcmp(inst.data(), b->uploaded.data(), sizeof(BatchInst) * inst.size()) == 0);
  if (!same && nm > 0) {
    if (size_t(nm) > b->instCap) {
      BCK(cudaStreamSynchronize(b->stream));
      cudaFree(b->dInst);
      b->dInst = nullptr;
      b->instCap = 0;
      BCK(cudaMalloc(&b->dInst, sizeof(BatchInst) * size_t(nm)));
      b->instCap = size_t(nm);
      drop_graph(b);
    }
    if (size_t(nm) > b->hInstCap) {
      BCK(cudaEventSynchronize(b->staged));
      cudaFreeHost(b->hInst);
      b->hInst = nullptr;
      b->hInstCap = 0;
      BCK(cudaHostAlloc(reinterpret_cast<void**>(&b->hInst), sizeof(BatchInst) * size_t(nm), cudaHostAllocDefault));
      b->hInstCap = size_t(nm);
    }
    // the previous upload must have left the pinned buffer before it is reused
    BCK(cudaEventSynchronize(b->staged));
    std::memcpy(b->hInst, inst.data(), sizeof(BatchInst) * size_t(nm));
    BCK(cudaMemcpyAsync(b->dInst, b->hInst, sizeof(BatchInst) * size_t(nm), cudaMemcpyHostToDevice, b->stream));
    BCK(cudaEventRecord(b->staged, b->stream));
    b->uploaded = inst;
  }
  return RN_OK;
}

// The launches of batch step c (counter value at the step) on the batch stream.
// With sprays, the per-member parcel and apply launches go between them.
int launch_step(rn_batch_t* b, int c, bool withSpray) {
  const Flags f = b->flags;
  const int delta = f.delta();
  BatchPhase ph;
  ph.shift = (c * delta) % 3;
  ph.par = c & 1;
  ph.maxX = b->maxX;
  ph.active = b->runActive.empty() ? nullptr : b->dActive;
  const int nb = b->nblocks;
  ph.finalCfl = 0;
  b->K->batchStage1(b->dInst, b->dBlock, nb, ph, b->tile, b->stream);
  b->launches++;
  if (f.inj && withSpray) {
    // GPUSpray.step between the two stages (solver.js:865-871), per member, on
    // a stream of its own: the parcel steps read the stage-1 states and write
    // only the parcel rings and deposit sums, which stage 2 + the split step
    // do not touch; the applies wait for them
    if (!b->sprayStream) {
      BCK(cudaStreamCreateWithFlags(&b->sprayStream, cudaStreamNonBlocking));
      BCK(cudaEventCreateWithFlags(&b->evSprayFork, cudaEventDisableTiming));
      BCK(cudaEventCreateWithFlags(&b->evSprayJoin, cudaEventDisableTiming));
    }
    BCK(cudaEventRecord(b->evSprayFork, b->stream));
    BCK(cudaStreamWaitEvent(b->sprayStream, b->evSprayFork, 0));
    for (size_t m = 0; m < b->members.size(); m++) {
      if (!b->runActive.empty() && !b->runActive[m]) continue;   // stopped in rn_batch_run
      rn_solver* h = b->members[m];
      const BatchInst& d = b->uploaded[m];
      const int s0 = (d.cur0 + ph.shift) % 3, s1 = (s0 + 1) % 3;
      const int si = d.stepIdx0 ^ ph.par;
      SprayArgs sp;
      sp.g = h->grid();
      sp.A1 = h->SA[s1]; sp.B1 = h->SB[s1];
      sp.PA = h->PA[h->scur]; sp.PB = h->PB[h->scur];
      sp.oPA = h->PA[1 - h->scur]; sp.oPB = h->PB[1 - h->scur]; sp.oPC = h->PC[1 - h->scur];
      sp.tab = h->tab; sp.st = h->stepTex + (1 - si);
      sp.key = h->key; sp.val = h->val; sp.dep = h->dep;
      sp.acc = h->acc + size_t(4) * h->Nx * h->Nr * h->scur;
      sp.depFlag = h->depFlag;
      sp.boundIn = h->depBound + 2 * h->scur;
      sp.boundOut = h->depBound + 2 * (1 - h->scur);
      sp.liveSteps = h->liveSteps;
      sp.head = int(h->head); sp.seed = int(h->seed);
      sp.hs = nullptr;
      int launched = 0;
      if (b->K->spray(sp, b->params[m], h->sortTemp, h->sortTempBytes, h->keyS, h->valS, h->src, b->sprayStream,
                      &launched) != 0)
        return bfail(RN_ERR_CUDA, "rn_batch_step: deposit sort failed");
      b->launches += launched;
    }
    BCK(cudaEventRecord(b->evSprayJoin, b->sprayStream));
  }
  ph.finalCfl = f.inj ? 0 : 1;
  if (f.phys()) {
    if (b->split) {
      // the few tiles with long member lists on the side stream, at the same time
      cudaEventRecord(b->evFork, b->stream);
      cudaStreamWaitEvent(b->side, b->evFork, 0);
      b->K->batchStage2Phys(b->dInst, b->dBlock, nb, ph, b->tile, b->dHeavy, b->nHeavy, false, b->side);
      cudaEventRecord(b->evJoin, b->side);
      b->K->batchStage2Phys(b->dInst, b->dBlock, nb, ph, b->tile, nullptr, b->nHeavy, true, b->stream);
      cudaStreamWaitEvent(b->stream, b->evJoin, 0);
      b->launches++;
    } else {
      b->K->batchStage2Phys(b->dInst, b->dBlock, nb, ph, b->tile, nullptr, 0, false, b->stream);
    }
  } else {
    b->K->batchStage2(b->dInst, b->dBlock, nb, ph, b->tile, b->stream);
  }
  b->launches++;
  if (f.inj && withSpray) {
    BCK(cudaStreamWaitEvent(b->stream, b->evSprayJoin, 0));   // the parcel steps are done
    for (size_t m = 0; m < b->members.size(); m++) {
      if (!b->runActive.empty() && !b->runActive[m]) continue;
      rn_solver* h = b->members[m];
      const BatchInst& d = b->uploaded[m];
      const int s0 = (d.cur0 + ph.shift) % 3;
      const int cur = (s0 + 2) % 3, out = (cur + 1) % 3;
      const int ws = d.wslot0 ^ ph.par;
      ApplyArgs ap;
      ap.g = h->grid();
      ap.A = h->SA[cur]; ap.B = h->SB[cur]; ap.src = h->src;
      ap.acc = h->acc + size_t(4) * h->Nx * h->Nr * h->scur;
      ap.accNext = h->acc + size_t(4) * h->Nx * h->Nr * (1 - h->scur);
      ap.boundIn = h->depBound + 2 * h->scur;
      ap.oA = h->SA[out]; ap.oB = h->SB[out];
      ap.wOut = h->wmax + (1 - ws);
      ap.finalCfl = 1;
      ap.hsNext = nullptr;
      b->K->apply(ap, b->params[m], b->stream);
      b->launches++;
      h->scur = 1 - h->scur;
      h->head = (h->head + 4) % SPRAY_N;
      h->seed = h->seed + 1u;
    }
  }
  return RN_OK;
}

int build_graph(rn_batch_t* b) {
  drop_graph(b);
  cudaGraph_t g = nullptr;
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  const long long before = b->launches;
  int rc = RN_OK;
  for (int c = 0; c < PERIOD && rc == RN_OK; c++) rc = launch_step(b, c, false);
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  b->launches = before;   // capturing launches nothing
  if (rc != RN_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return rn_record_cuda(e, "cudaStreamEndCapture");
  e = cudaGraphInstantiate(&b->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    b->graph = nullptr;
    return rn_record_cuda(e, "cudaGraphInstantiate");
  }
  b->graphK = b->K;
  b->graphBlocks = b->nblocks;
  b->graphTile = b->tile;
  b->graphMaxX = b->maxX;
  b->graphHeavy = b->split ? b->nHeavy : 0;
  b->graphFlags = b->flags;
  b->graphActive = b->runActive.empty() ? nullptr : b->dActive;
  return RN_OK;
}

int launches_per_step(const rn_batch_t* b) { return 2 + ((b->flags.phys() && b->split) ? 1 : 0); }

// The launches of n batch steps from the batch counter on (descriptors and
// block table already refreshed): without sprays, up to the start of a period
// step by step, whole periods from the graph, the rest step by step.
int issue_steps(rn_batch_t* b, int n) {
  int done = 0, rc = RN_OK;
  if (b->flags.inj) {
    // parcel heads and seeds change every step: launched step by step
    for (; done < n; done++) {
      rc = launch_step(b, b->ctr, true);
      if (rc != RN_OK) return rc;
      b->ctr = (b->ctr + 1) % PERIOD;
    }
    return RN_OK;
  }
  while (done < n && b->ctr != 0) {
    rc = launch_step(b, b->ctr, false);
    if (rc != RN_OK) return rc;
    b->ctr = (b->ctr + 1) % PERIOD;
    done++;
  }
  if (n - done >= PERIOD) {
    const int* active = b->runActive.empty() ? nullptr : b->dActive;
    if (!b->graph || b->graphK != b->K || b->graphBlocks != b->nblocks || b->graphTile != b->tile ||
        b->graphMaxX != b->maxX || b->graphHeavy != (b->split ? b->nHeavy : 0) || !(b->graphFlags == b->flags) ||
        b->graphActive != active) {
      rc = build_graph(b);
      if (rc != RN_OK) return rc;
    }
    while (n - done >= PERIOD) {
      BCK(cudaGraphLaunch(b->graph, b->stream));
      b->launches += PERIOD * launches_per_step(b);
      done += PERIOD;
    }
  }
  for (; done < n; done++) {
    rc = launch_step(b, b->ctr, false);
    if (rc != RN_OK) return rc;
    b->ctr = (b->ctr + 1) % PERIOD;
  }
  return RN_OK;
}

// A member's host-side bookkeeping after n batch steps, as n calls of rn_step
// would leave it.
void advance(rn_solver* h, long long n, const Flags& f) {
  h->cur = int((h->cur + n * f.delta()) % 3);
  if (n & 1) {
    h->stepIdx = 1 - h->stepIdx;
    h->wslot = 1 - h->wslot;
  }
  h->wvalid = true;
  h->s1last = f.inj ? (h->cur + 1) % 3 : (h->cur + 2) % 3;   // the last step's stage-1 slot
  h->stepCount += n;
}

// Checks the members before the batch step stepping at batch counter c and
// the run's step done (rn_batch_run): a member still stepping stops when its
// simulated time t_new >= tEnd (the step info of its current state) or the run
// reached maxSteps (> 0). out[0] = members still stepping, out[1 + m] = flags.
__global__ void k_batch_gate(const BatchInst* __restrict__ insts, int nm, int par, const double* __restrict__ tEnd,
                             long long done, long long maxSteps, int* active, int* out) {
  __shared__ int count;
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  int mine = 0;
  for (int m = threadIdx.x; m < nm; m += blockDim.x) {
    int on = active[m];
    if (on) {
      const BatchInst& d = insts[m];
      const double t = double(d.stepTex[d.stepIdx0 ^ par].z);
      if (!(t < tEnd[m]) || (maxSteps > 0 && done >= maxSteps)) on = 0;
      active[m] = on;
    }
    out[1 + m] = on;
    mine += on;
  }
  atomicAdd(&count, mine);
  __syncthreads();
  if (threadIdx.x == 0) out[0] = count;
}

// Device buffers of a run over nm members.
int run_buffers(rn_batch_t* b, size_t nm) {
  if (nm <= b->runCap) return RN_OK;
  cudaFree(b->dActive);
  cudaFree(b->dTEnd);
  cudaFree(b->dGate);
  cudaFreeHost(b->hGate);
  b->dActive = nullptr; b->dTEnd = nullptr; b->dGate = nullptr; b->hGate = nullptr;
  b->runCap = 0;
  drop_graph(b);   // a graph may hold the old flags pointer
  BCK(cudaMalloc(&b->dActive, sizeof(int) * nm));
  BCK(cudaMalloc(&b->dTEnd, sizeof(double) * nm));
  BCK(cudaMalloc(&b->dGate, sizeof(int) * 2 * (nm + 1)));
  BCK(cudaHostAlloc(reinterpret_cast<void**>(&b->hGate), sizeof(int) * 2 * (nm + 1), cudaHostAllocDefault));
  for (int q = 0; q < 2; q++)
    if (!b->evGate[q]) BCK(cudaEventCreateWithFlags(&b->evGate[q], cudaEventDisableTiming));
  b->runCap = nm;
  return RN_OK;
}

// Checks the batch's members before a step (rn_batch_step, rn_batch_run) and
// orders their queued work before the batch's kernels.
int prepare(rn_batch_t* b) {
  const KernelSet* K = b->members[0]->K;
  for (rn_solver* h : b->members) {
    if (h->K != K) return bfail(RN_ERR_STATE, "rn_batch_step: members have different precisions");
    if (h->tile != b->tile) return bfail(RN_ERR_STATE, "rn_batch_step: a member's tile shape differs from the batch's");
    if (!h->SA[0]) return bfail(RN_ERR_STATE, "rn_batch_step: a member has no buffers");
  }
  b->K = K;
  // each member's CFL wave speed of its current state, and its queued work,
  // before the batch's kernels
  for (size_t m = 0; m < b->members.size(); m++) {
    rn_solver* h = b->members[m];
    int rc = rn_ensure_wave_speed(h);
    if (rc != RN_OK) return rc;
    BCK(cudaEventRecord(b->fence[m], h->stream));
    BCK(cudaStreamWaitEvent(b->stream, b->fence[m], 0));
  }
  return RN_OK;
}

// Later work of each member waits for the batch.
int release_members(rn_batch_t* b) {
  BCK(cudaEventRecord(b->done, b->stream));
  for (rn_solver* h : b->members) BCK(cudaStreamWaitEvent(h->stream, b->done, 0));
  return RN_OK;
}

}  // namespace

// Removes h from its batch (rn_destroy of a member).
void rn_batch_detach(rn_solver* h) {
  if (h && h->batch) rn_batch_remove(h->batch, h);
}

extern "C" {

int rn_batch_step(rn_batch b, int n) {
  if (!b || n < 0) return bfail(RN_ERR_ARG, "rn_batch_step: bad argument");
  if (b->members.empty() || n == 0) return RN_OK;
  int rc = prepare(b);
  if (rc == RN_OK) rc = refresh(b);
  if (rc == RN_OK) rc = issue_steps(b, n);
  if (rc != RN_OK) return rc;
  BCK(cudaGetLastError());
  for (rn_solver* h : b->members) advance(h, n, b->flags);
  return release_members(b);
}

int rn_batch_run(rn_batch b, const double* t_end, int chunk, long long max_steps, long long* steps) {
  if (!b || !t_end || chunk < 1 || max_steps < 0) return bfail(RN_ERR_ARG, "rn_batch_run: bad argument");
  const size_t nm = b->members.size();
  if (steps)
    for (size_t m = 0; m < nm; m++) steps[m] = 0;
  if (nm == 0) return RN_OK;
  int rc = prepare(b);
  if (rc == RN_OK) rc = run_buffers(b, nm);
  if (rc != RN_OK) return rc;
  std::vector<int> on(nm, 1);
  BCK(cudaMemcpyAsync(b->dTEnd, t_end, sizeof(double) * nm, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->dActive, on.data(), sizeof(int) * nm, cudaMemcpyHostToDevice, b->stream));
  b->runActive.assign(nm, 1);
  auto finish = [&](int code) {
    // outside a run every member steps again; the next step rebuilds the
    // table and the descriptors
    b->runActive.clear();
    b->layout.clear();
    b->uploaded.clear();
    if (code != RN_OK) return code;
    return release_members(b);
  };
  const size_t G = nm + 1;
  long long done = 0;
  // the gate for the steps issued so far (`at` of them), its flags read back
  // into buffer `slot` behind event evGate[slot]
  auto gate = [&](int slot, long long at) -> int {
    k_batch_gate<<<1, 256, 0, b->stream>>>(b->dInst, int(nm), b->ctr & 1, b->dTEnd, at, max_steps, b->dActive,
                                           b->dGate + slot * G);
    b->launches++;
    BCK(cudaMemcpyAsync(b->hGate + slot * G, b->dGate + slot * G, sizeof(int) * G, cudaMemcpyDeviceToHost,
                        b->stream));
    BCK(cudaEventRecord(b->evGate[slot], b->stream));
    return RN_OK;
  };
  // waits for gate buffer `slot`; the members still stepping become runActive
  auto take = [&](int slot, int& count) -> int {
    BCK(cudaEventSynchronize(b->evGate[slot]));
    const int* f = b->hGate + slot * G;
    count = f[0];
    for (size_t m = 0; m < nm; m++) b->runActive[m] = char(f[1 + m] != 0);
    return RN_OK;
  };
  int tableBlocks = 0;
  // the stopped members' blocks leave the table (a new table and graph) once
  // they number an SM's worth and an eighth of it; until then they return at
  // once
  auto compact = [&]() -> int {
    int activeBlocks = 0;
    for (size_t m = 0; m < nm; m++) {
      const rn_solver* h = b->members[m];
      if (b->runActive[m])
        activeBlocks += ((h->Nx + TILE_TX[b->tile] - 1) / TILE_TX[b->tile]) *
                        ((h->Nr + TILE_TY[b->tile] - 1) / TILE_TY[b->tile]);
    }
    const int stoppedBlocks = tableBlocks - activeBlocks;
    if (stoppedBlocks >= b->numSMs && 8 * stoppedBlocks >= tableBlocks) {
      int r = refresh(b);
      if (r != RN_OK) return r;
      tableBlocks = b->nblocks;
    }
    return RN_OK;
  };
  auto chunk_at = [&](long long at) -> int {
    const long long left = max_steps > 0 ? max_steps - at : chunk;
    return int(left < chunk ? (left > 0 ? left : 0) : chunk);
  };
  auto account = [&](int n) {
    for (size_t m = 0; m < nm; m++)
      if (b->runActive[m]) {
        advance(b->members[m], n, b->flags);
        if (steps) steps[m] += n;
      }
  };
  rc = refresh(b);
  tableBlocks = b->nblocks;
  int count = 0;
  if (rc == RN_OK) rc = gate(0, 0);
  if (rc == RN_OK) rc = take(0, count);
  if (b->flags.inj) {
    // with sprays each chunk's per-member parcel launches follow the host's
    // flags, so every chunk waits for the gate before it
    while (rc == RN_OK && count > 0) {
      rc = compact();
      const int n = chunk_at(done);
      if (rc == RN_OK) rc = issue_steps(b, n);
      if (rc != RN_OK) break;
      account(n);
      done += n;
      rc = gate(0, done);
      if (rc == RN_OK) rc = take(0, count);
    }
  } else if (rc == RN_OK && count > 0) {
    // Without sprays the kernels alone read the flags, so the next chunk is
    // queued before the gate ahead of it has been read back: gate j's flags
    // (buffer j & 1) gate chunk j on the device, and the host learns them,
    // and accounts for chunk j, while chunk j runs. The chunk queued after the
    // last member stopped is all early returns.
    rc = compact();
    int n = chunk_at(done);
    if (rc == RN_OK) rc = issue_steps(b, n);
    if (rc == RN_OK) {
      account(n);
      done += n;
      rc = gate(1, done);
    }
    for (int j = 1; rc == RN_OK; j++) {
      n = chunk_at(done);
      if (n > 0) rc = issue_steps(b, n);             // chunk j, ahead of its gate's read-back
      if (rc == RN_OK) rc = gate((j + 1) & 1, done + n);
      if (rc == RN_OK) rc = take(j & 1, count);
      if (rc != RN_OK || count == 0) break;
      account(n);
      done += n;
      rc = compact();
    }
    if (rc == RN_OK) {
      cudaError_t e = cudaStreamSynchronize(b->stream);
      if (e != cudaSuccess) rc = rn_record_cuda(e, "rn_batch_run");
    }
  }
  if (rc == RN_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = rn_record_cuda(e, "rn_batch_run");
  }
  return finish(rc);
}


int rn_batch_create(rn_batch* out) {
  if (!out) return bfail(RN_ERR_ARG, "rn_batch_create: out is NULL");
  *out = nullptr;
  rn_batch_t* b = new rn_batch_t();
  cudaError_t e = cudaGetDevice(&b->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evFork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->evJoin, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, b->device);
  if (e != cudaSuccess) {
    if (b->evJoin) cudaEventDestroy(b->evJoin);
    if (b->evFork) cudaEventDestroy(b->evFork);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->staged) cudaEventDestroy(b->staged);
    if (b->done) cudaEventDestroy(b->done);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return rn_record_cuda(e, "rn_batch_create");
  }
  *out = b;
  return RN_OK;
}

int rn_batch_destroy(rn_batch b) {
  if (!b) return bfail(RN_ERR_ARG, "rn_batch_destroy: NULL batch");
  cudaStreamSynchronize(b->stream);
  for (rn_solver* h : b->members) h->batch = nullptr;
  for (cudaEvent_t e : b->fence) cudaEventDestroy(e);
  drop_graph(b);
  cudaFree(b->dInst);
  cudaFree(b->dBlock);
  cudaFree(b->dHeavy);
  cudaFree(b->dActive);
  cudaFree(b->dTEnd);
  cudaFree(b->dGate);
  cudaFreeHost(b->hGate);
  for (cudaEvent_t e : b->evGate)
    if (e) cudaEventDestroy(e);
  cudaFreeHost(b->hInst);
  cudaEventDestroy(b->staged);
  cudaEventDestroy(b->done);
  cudaStreamSynchronize(b->side);
  cudaEventDestroy(b->evFork);
  cudaEventDestroy(b->evJoin);
  cudaStreamDestroy(b->side);
  if (b->sprayStream) {
    cudaStreamSynchronize(b->sprayStream);
    cudaEventDestroy(b->evSprayFork);
    cudaEventDestroy(b->evSprayJoin);
    cudaStreamDestroy(b->sprayStream);
  }
  cudaStreamDestroy(b->stream);
  delete b;
  return RN_OK;
}

int rn_batch_add(rn_batch b, rn_handle h, const rn_params* P, int* slot) {
  if (!b || !h || !P || !h->SA[0]) return bfail(RN_ERR_ARG, "rn_batch_add: bad argument");
  if (h->batch) return bfail(RN_ERR_STATE, "rn_batch_add: the handle is already in a batch");
  if (h->device != b->device) return bfail(RN_ERR_ARG, "rn_batch_add: the handle is on another device");
  const Flags f = flags_of(*P);
  if (!b->members.empty()) {
    if (!(f == b->flags)) return bfail(RN_ERR_ARG, "rn_batch_add: physics flags (visc, chem, inj) differ from the batch's");
    if (h->K != b->members[0]->K) return bfail(RN_ERR_ARG, "rn_batch_add: precision differs from the batch's");
  }
  if (h->tile != b->tile) {
    int rc = rn_set_tile(h, b->tile);
    if (rc != RN_OK) return rc;
  }
  cudaEvent_t ev = nullptr;
  BCK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  if (b->members.empty()) b->flags = f;
  b->members.push_back(h);
  b->params.push_back(*P);
  b->fence.push_back(ev);
  h->batch = b;
  if (slot) *slot = int(b->members.size()) - 1;
  return RN_OK;
}

int rn_batch_remove(rn_batch b, rn_handle h) {
  if (!b || !h) return bfail(RN_ERR_ARG, "rn_batch_remove: bad argument");
  const int m = index_of(b, h);
  if (m < 0) return bfail(RN_ERR_ARG, "rn_batch_remove: the handle is not in this batch");
  // the handle's later work waits for the batch's queued steps
  cudaEventRecord(b->done, b->stream);
  cudaStreamWaitEvent(h->stream, b->done, 0);
  cudaEventDestroy(b->fence[m]);
  b->members.erase(b->members.begin() + m);
  b->params.erase(b->params.begin() + m);
  b->fence.erase(b->fence.begin() + m);
  h->batch = nullptr;
  return RN_OK;
}

int rn_batch_set_params(rn_batch b, rn_handle h, const rn_params* P) {
  if (!b || !h || !P) return bfail(RN_ERR_ARG, "rn_batch_set_params: bad argument");
  const int m = index_of(b, h);
  if (m < 0) return bfail(RN_ERR_ARG, "rn_batch_set_params: the handle is not in this batch");
  if (!(flags_of(*P) == b->flags) && b->members.size() > 1)
    return bfail(RN_ERR_ARG, "rn_batch_set_params: physics flags (visc, chem, inj) differ from the batch's");
  if (b->members.size() == 1) b->flags = flags_of(*P);
  b->params[m] = *P;
  return RN_OK;
}

int rn_batch_size(rn_batch b, int* members, long long* cells) {
  if (!b) return bfail(RN_ERR_ARG, "rn_batch_size: NULL batch");
  long long c = 0;
  for (const rn_solver* h : b->members) c += (long long)h->Nx * h->Nr;
  if (members) *members = int(b->members.size());
  if (cells) *cells = c;
  return RN_OK;
}

int rn_batch_set_tile(rn_batch b, int shape) {
  if (!b || shape < 0 || shape >= NTILES) return bfail(RN_ERR_ARG, "rn_batch_set_tile: bad argument");
  if (shape == b->tile) return RN_OK;
  BCK(cudaStreamSynchronize(b->stream));
  const int old = b->tile;
  for (size_t m = 0; m < b->members.size(); m++) {
    rn_solver* h = b->members[m];
    h->batch = nullptr;   // rn_set_tile refuses batch members
    int rc = rn_set_tile(h, shape);
    h->batch = b;
    if (rc != RN_OK) {
      std::string msg = rn_last_error();
      for (size_t q = 0; q < m; q++) {
        b->members[q]->batch = nullptr;
        rn_set_tile(b->members[q], old);
        b->members[q]->batch = b;
      }
      return bfail(rc, msg);
    }
  }
  b->tile = shape;
  b->layout.clear();   // block table and descriptors are rebuilt by the next step
  b->uploaded.clear();
  return RN_OK;
}

int rn_batch_autotune(rn_batch b, int steps, int* chosen) {
  if (!b || steps < 1) return bfail(RN_ERR_ARG, "rn_batch_autotune: bad argument");
  if (b->members.empty()) {
    if (chosen) *chosen = b->tile;
    return RN_OK;
  }
  BCK(cudaStreamSynchronize(b->stream));
  // everything a step changes, per member: state ring, step info, wave-speed
  // slots, parcel ring; and the host-side positions
  struct Saved {
    char* buf = nullptr;
    size_t state = 0, spray = 0;
    int cur, stepIdx, wslot, scur;
    bool wvalid;
    long long stepCount;
    uint32_t head, seed;
  };
  const bool inj = b->flags.inj != 0;
  std::vector<Saved> sv(b->members.size());
  auto release = [&]() {
    for (Saved& s : sv) cudaFree(s.buf);
  };
  for (size_t m = 0; m < b->members.size(); m++) {
    rn_solver* h = b->members[m];
    int rc = rn_ensure_wave_speed(h);
    if (rc != RN_OK) { release(); return rc; }
    Saved& s = sv[m];
    s.state = sizeof(float4) * size_t(h->Nx) * h->Nr * 6;
    s.spray = inj ? sizeof(float4) * SPRAY_N * 6 : 0;
    cudaError_t e = cudaMalloc(&s.buf, s.state + s.spray + sizeof(float4) * 2 + sizeof(unsigned) * 2);
    if (e != cudaSuccess) { s.buf = nullptr; release(); return rn_record_cuda(e, "rn_batch_autotune: cudaMalloc"); }
    s.cur = h->cur; s.stepIdx = h->stepIdx; s.wslot = h->wslot; s.scur = h->scur; s.wvalid = h->wvalid;
    s.stepCount = h->stepCount; s.head = h->head; s.seed = h->seed;
  }
  auto copy_all = [&](bool toSave) -> cudaError_t {
    for (size_t m = 0; m < b->members.size(); m++) {
      rn_solver* h = b->members[m];
      Saved& s = sv[m];
      struct { void* dev; size_t n; } parts[4] = {{h->SA[0], s.state}, {h->PA[0], s.spray},
                                                 {h->stepTex, sizeof(float4) * 2}, {h->wmax, sizeof(unsigned) * 2}};
      char* p = s.buf;
      for (auto& q : parts) {
        if (!q.n) continue;
        cudaError_t e = toSave ? cudaMemcpyAsync(p, q.dev, q.n, cudaMemcpyDeviceToDevice, h->stream)
                               : cudaMemcpyAsync(q.dev, p, q.n, cudaMemcpyDeviceToDevice, h->stream);
        if (e != cudaSuccess) return e;
        p += q.n;
      }
      if (!toSave) {
        h->cur = s.cur; h->stepIdx = s.stepIdx; h->wslot = s.wslot; h->scur = s.scur; h->wvalid = s.wvalid;
        h->stepCount = s.stepCount; h->head = s.head; h->seed = s.seed;
        // the spray's deposit sums start each step at zero whatever parity it has
        cudaError_t e = cudaMemsetAsync(h->acc, 0, sizeof(unsigned long long) * 8 * size_t(h->Nx) * h->Nr,
                                        h->stream);
        if (e != cudaSuccess) return e;
      }
    }
    return cudaSuccess;
  };
  const int ctr = b->ctr;
  const long long launches = b->launches;
  const int old = b->tile;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = copy_all(true);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  int best = old, rc = RN_OK;
  float bestMs = 1e30f;
  for (int shape = 0; shape < NTILES && e == cudaSuccess && rc == RN_OK; shape++) {
    if (rn_batch_set_tile(b, shape) != RN_OK) continue;    // a member's lists do not fit this shape
    rc = rn_batch_step(b, PERIOD);                          // warm-up (builds the graph)
    float ms = 0.0f;
    if (rc == RN_OK) e = cudaEventRecord(e0, b->stream);
    if (rc == RN_OK && e == cudaSuccess) rc = rn_batch_step(b, steps);
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
    if (rc == RN_OK && e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (rc == RN_OK && e == cudaSuccess && ms < bestMs) { bestMs = ms; best = shape; }
    // members' streams wait for the batch (rn_batch_step), then restore
    if (e == cudaSuccess) e = copy_all(false);
    b->ctr = ctr;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  for (rn_solver* h : b->members) cudaStreamSynchronize(h->stream);
  release();
  b->launches = launches;
  b->uploaded.clear();
  int rc2 = rn_batch_set_tile(b, best);
  if (e != cudaSuccess) return rn_record_cuda(e, "rn_batch_autotune");
  if (rc != RN_OK) return rc;
  if (rc2 != RN_OK) return rc2;
  if (chosen) *chosen = best;
  return RN_OK;
}

int rn_batch_sync(rn_batch b) {
  if (!b) return bfail(RN_ERR_ARG, "rn_batch_sync: NULL batch");
  BCK(cudaStreamSynchronize(b->stream));
  return RN_OK;
}

int rn_batch_stream(rn_batch b, void** stream) {
  if (!b || !stream) return bfail(RN_ERR_ARG, "rn_batch_stream: bad argument");
  *stream = reinterpret_cast<void*>(b->stream);
  return RN_OK;
}

int rn_batch_kernel_launches(rn_batch b, long long* out) {
  if (!b || !out) return bfail(RN_ERR_ARG, "rn_batch_kernel_launches: bad argument");
  *out = b->launches;
  return RN_OK;
}

}  // extern "C"
