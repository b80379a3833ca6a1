// rn_serve.cu -- the solve server: continuous batching of nozzle solves on one
// GPU (declared in rn.h; no reference counterpart, the reference runs one
// interactive solve per page).
//
// A request carries a whole solve: grid, geometry, initial state, parameter
// block, optional injector table, stop criteria and the read-out columns. The
// caller's thread only copies it into the arrival queue. One worker thread
// owns the device side:
//   admit  -- FIFO: while the head request's device bytes fit in the budget
//             (and the active count is below max_active), create its handle,
//             upload it and add it to the batch of its physics class
//             (visc, chem, inj); classes run on their own streams and overlap;
//   tick   -- every class batch steps check_every steps; one step before the
//             end the members' states are marked, after it their FP64
//             residuals (RMS of dU/dt) and step info are copied back;
//   retire -- a solve whose density residual fell to drop x its first value,
//             whose time reached t_end, or whose step count reached max_steps
//             gets its FP64 read-outs and final state copied out, leaves its
//             batch and frees its memory, which admits the next arrivals.
// A solve steps exactly as it would alone: batch membership does not change a
// cell's arithmetic, so its result is the same in any mix.
// Failures are isolated: a solve whose own work fails (setup, an allocation,
// a non-finite residual) is evicted alone; a class batch whose step fails
// evicts its class; only a broken CUDA context fails everything.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "rn.h"
#include "rn_internal.h"

namespace {

constexpr int SPRAY_N = 65536;

struct Request {
  long long id = 0;
  int Nx = 0, Nr = 0;
  std::vector<uint8_t> mask;
  std::vector<float> geoA, geoG, geoM, jWall, A, B, injTab, parA, parB;
  int parHead = 0;
  rn_params P;
  double drop = 0.0, tEnd = 0.0;
  long long maxSteps = 0;
  rn_integral_spec spec;
  size_t bytes = 0;
  double tSubmit = 0.0;
  int inject = 0;            // RN_INJECT_* armed by rn_serve_inject for this request
};

struct Active {
  Request req;
  rn_solver* h = nullptr;
  int cls = 0;
  long long steps = 0;
  double r0 = -1.0, r = -1.0, t = 0.0, tAdmit = 0.0;
};

struct Done {
  rn_solve_result res;
  std::vector<float> A, B;
};

int class_of(const rn_params& P) { return (P.visc ? 1 : 0) | (P.chem ? 2 : 0) | (P.inj ? 4 : 0); }

}  // namespace

// Device bytes one handle of an Nx x Nr grid holds (rn_api.cu's alloc_buffers,
// the member lists, the residual snapshot and the deposit-sort scratch).
size_t rn_handle_bytes(int Nx, int Nr) {
  const size_t N = size_t(Nx) * Nr, NF = size_t(Nx + 1) * (Nr + 1);
  size_t b = sizeof(float4) * N * 6;                   // state ring
  b += sizeof(float4) * (NF + 2 * N + 2 * Nx);         // geoA, geoG, geoM, jWall, wall row
  b += N;                                              // mask
  b += sizeof(float4) * (2 + SPRAY_N * 7 + N + 768);   // step info, parcel ring + deposits, src, table
  b += sizeof(unsigned) * SPRAY_N * 4 + sizeof(double) * 16;
  b += rn::kernels_fast.sortTempBytes(int(N));
  b += sizeof(int) * (N / 64 + 2) + sizeof(int) * 4096;  // member lists (generous)
  b += rn_residual_bytes(Nx, Nr);
  return (b + (1u << 20)) & ~size_t((1u << 20) - 1);   // allocation granularity slack
}

struct rn_server_t {
  rn_server_opts opts;
  int device = 0;
  std::chrono::steady_clock::time_point t0;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cvWork, cvDone;
  std::deque<Request> queue;
  std::map<long long, Done> done;
  long long nextId = 1;
  bool stop = false;
  int failed = 0;
  std::string failMsg;
  int injectNext = 0;         // armed by rn_serve_inject, taken by the next submit
  long long evicted = 0;      // solves that failed alone
  // worker-side state (read under mu by rn_serve_stats)
  std::vector<Active> active;
  size_t used = 0;
  long long cells = 0;        // grid cells of the active solves
  std::atomic<long long> ticks{0};
  long long admitted = 0, retired = 0;
  std::map<int, rn_batch_t*> batches;
  double* pinned = nullptr;   // per active solve: residual (6 doubles) + step info (2 doubles as 4 floats)
  size_t pinnedCap = 0;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

int sfail(int code, const std::string& msg) { return rn_record_error(code, msg); }

// Creates and uploads the handle of request r and adds it to its class batch.
int admit(rn_server_t* s, Request& r, Active& a) {
  if (r.inject == RN_INJECT_ADMIT) {
    r.inject = 0;
    return sfail(RN_ERR_NOMEM, "injected allocation failure at admission");
  }
  rn_handle h = nullptr;
  int rc = rn_create(r.Nx, r.Nr, &h);
  if (rc != RN_OK) return rc;
  auto bail = [&](int code) {
    rn_destroy(h);
    return code;
  };
  if (s->opts.precision == RN_PRECISION_EXACT && (rc = rn_set_precision(h, RN_PRECISION_EXACT)) != RN_OK) return bail(rc);
  if ((rc = rn_set_geometry(h, r.mask.data(), r.geoA.data(), r.geoG.data(), r.geoM.data(),
                            r.jWall.empty() ? nullptr : r.jWall.data())) != RN_OK)
    return bail(rc);
  if ((rc = rn_set_state(h, r.A.data(), r.B.data())) != RN_OK) return bail(rc);
  if (!r.injTab.empty() && (rc = rn_spray_set_injector(h, r.injTab.data())) != RN_OK) return bail(rc);
  if (!r.parA.empty() && (rc = rn_spray_set_parcels(h, r.parA.data(), r.parB.data(), r.parHead)) != RN_OK)
    return bail(rc);
  const int cls = class_of(r.P);
  rn_batch_t*& b = s->batches[cls];
  if (!b) {
    if ((rc = rn_batch_create(&b)) != RN_OK) return bail(rc);
    if ((rc = rn_batch_set_tile(b, s->opts.tile)) != RN_OK) return bail(rc);
  }
  if ((rc = rn_batch_add(b, h, &r.P, nullptr)) != RN_OK) return bail(rc);
  a.h = h;
  a.cls = cls;
  return RN_OK;
}

// Final read-outs and state of an active solve, then its handle is released.
void retire(rn_server_t* s, Active& a, int status) {
  Done d;
  std::memset(&d.res, 0, sizeof(d.res));
  d.res.status = status;
  d.res.steps = a.steps;
  d.res.t = a.t;
  d.res.residual0 = a.r0;
  d.res.residual = a.r;
  d.res.submit_ms = a.req.tSubmit;
  d.res.admit_ms = a.tAdmit;
  const size_t N = size_t(a.req.Nx) * a.req.Nr;
  d.A.resize(N * 4);
  d.B.resize(N * 4);
  int rc = rn_integrals(a.h, &a.req.spec, &d.res.integrals);
  if (rc == RN_OK) rc = rn_get_state(a.h, d.A.data(), d.B.data());
  if (rc != RN_OK) {
    d.res.status = RN_SOLVE_FAILED;
    d.A.clear();
    d.B.clear();
  }
  rn_batch_t* b = s->batches[a.cls];
  if (b) rn_batch_remove(b, a.h);
  rn_destroy(a.h);
  a.h = nullptr;
  d.res.done_ms = s->now_ms();
  std::lock_guard<std::mutex> lk(s->mu);
  s->used -= a.req.bytes;
  s->cells -= (long long)a.req.Nx * a.req.Nr;
  s->retired++;
  s->done[a.req.id] = std::move(d);
}

// A solve that failed alone: leaves its batch and frees its memory; its
// result carries RN_SOLVE_FAILED and no state.
void evict(rn_server_t* s, Active& a) {
  if (a.h) {
    rn_batch_t* b = s->batches[a.cls];
    if (b) rn_batch_remove(b, a.h);
    rn_destroy(a.h);
    a.h = nullptr;
  }
  Done d;
  std::memset(&d.res, 0, sizeof(d.res));
  d.res.status = RN_SOLVE_FAILED;
  d.res.steps = a.steps;
  d.res.t = a.t;
  d.res.residual0 = a.r0;
  d.res.residual = a.r;
  d.res.submit_ms = a.req.tSubmit;
  d.res.admit_ms = a.tAdmit;
  d.res.done_ms = s->now_ms();
  std::lock_guard<std::mutex> lk(s->mu);
  s->used -= a.req.bytes;
  s->cells -= (long long)a.req.Nx * a.req.Nr;
  s->retired++;
  s->evicted++;
  s->done[a.req.id] = std::move(d);
}

void fail_all(rn_server_t* s, const std::string& msg) {
  for (Active& a : s->active) {
    if (a.h) {
      rn_batch_t* b = s->batches[a.cls];
      if (b) rn_batch_remove(b, a.h);
      rn_destroy(a.h);
    }
    Done d;
    std::memset(&d.res, 0, sizeof(d.res));
    d.res.status = RN_SOLVE_FAILED;
    d.res.steps = a.steps;
    d.res.submit_ms = a.req.tSubmit;
    d.res.admit_ms = a.tAdmit;
    d.res.done_ms = s->now_ms();
    std::lock_guard<std::mutex> lk(s->mu);
    s->done[a.req.id] = std::move(d);
  }
  s->active.clear();
  std::lock_guard<std::mutex> lk(s->mu);
  s->used = 0;
  s->cells = 0;
  s->failed = 1;
  s->failMsg = msg;
  for (Request& r : s->queue) {
    Done d;
    std::memset(&d.res, 0, sizeof(d.res));
    d.res.status = RN_SOLVE_FAILED;
    d.res.submit_ms = r.tSubmit;
    d.res.done_ms = s->now_ms();
    s->done[r.id] = std::move(d);
  }
  s->queue.clear();
}

// One tick: check_every steps of every class batch, residuals of the last step.
// A solve whose own work fails is marked and evicted after the tick, a class
// whose batch step fails has all its solves evicted; the tick itself returns
// an error only when the CUDA context no longer works.
int tick(rn_server_t* s) {
  const int K = std::max(s->opts.check_every, 2);
  const size_t need = s->active.size() * 8;
  if (need > s->pinnedCap) {
    cudaFreeHost(s->pinned);
    s->pinned = nullptr;
    s->pinnedCap = 0;
    RN_CK(cudaHostAlloc(reinterpret_cast<void**>(&s->pinned), sizeof(double) * need * 2, cudaHostAllocDefault));
    s->pinnedCap = need * 2;
  }
  std::vector<char> bad(s->active.size(), 0);
  std::map<int, bool> badClass;
  bool anyBad = false;
  // every class batch queues its K steps before any is waited for
  for (auto& kv : s->batches) {
    rn_batch_t* b = kv.second;
    int members = 0;
    rn_batch_size(b, &members, nullptr);
    if (!members) continue;
    if (rn_batch_step(b, K - 1) != RN_OK) { badClass[kv.first] = anyBad = true; continue; }
    void* st = nullptr;
    rn_batch_stream(b, &st);
    cudaStream_t bs = static_cast<cudaStream_t>(st);
    for (size_t q = 0; q < s->active.size(); q++) {
      Active& a = s->active[q];
      if (a.cls != kv.first) continue;
      if (a.req.inject == RN_INJECT_TICK) {        // host-side injection: fails as an allocation would
        a.req.inject = 0;
        rn_record_error(RN_ERR_NOMEM, "injected allocation failure in a tick");
        bad[q] = anyBad = true;
        continue;
      }
      if (rn_residual_mark_on(a.h, bs) != RN_OK) bad[q] = anyBad = true;
    }
    if (rn_batch_step(b, 1) != RN_OK) { badClass[kv.first] = anyBad = true; continue; }
    for (size_t q = 0; q < s->active.size(); q++) {
      Active& a = s->active[q];
      if (a.cls != kv.first || bad[q]) continue;
      if (rn_residual_launch(a.h, bs) != RN_OK ||
          cudaMemcpyAsync(s->pinned + 8 * q, a.h->dRes, sizeof(double) * 6, cudaMemcpyDeviceToHost, bs) !=
              cudaSuccess ||
          cudaMemcpyAsync(s->pinned + 8 * q + 6, a.h->stepTex + a.h->stepIdx, sizeof(float4), cudaMemcpyDeviceToHost,
                          bs) != cudaSuccess)
        bad[q] = anyBad = true;
    }
  }
  for (auto& kv : s->batches)
    if (rn_batch_sync(kv.second) != RN_OK) badClass[kv.first] = anyBad = true;
  if (anyBad) {
    // a failure that left the context usable is the failing solves' alone
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess && cudaDeviceSynchronize() != cudaSuccess)
      return rn_record_cuda(e, "solve server tick (the CUDA context no longer works)");
  }
  s->ticks++;
  // retire what has converged, run out of time or steps; evict what failed
  std::vector<Active> keep;
  for (size_t q = 0; q < s->active.size(); q++) {
    Active& a = s->active[q];
    if (bad[q] || badClass.count(a.cls)) {
      evict(s, a);
      continue;
    }
    a.steps += K;
    const double* res = s->pinned + 8 * q;
    const float* st = reinterpret_cast<const float*>(s->pinned + 8 * q + 6);
    a.r = res[0];
    a.t = double(st[2]);
    if (!std::isfinite(a.r)) {                      // the solve's state is no longer finite
      evict(s, a);
      continue;
    }
    if (a.r0 < 0.0) a.r0 = a.r;
    int status = -100;
    if (a.req.drop > 0.0 && a.r0 > 0.0 && a.r <= a.req.drop * a.r0 && a.steps > K) status = RN_SOLVE_CONVERGED;
    else if (a.req.tEnd > 0.0 && a.t >= a.req.tEnd) status = RN_SOLVE_TIME;
    else if (a.req.maxSteps > 0 && a.steps >= a.req.maxSteps) status = RN_SOLVE_MAX_STEPS;
    if (status != -100) retire(s, a, status);
    else keep.push_back(std::move(a));
  }
  s->active.swap(keep);
  return RN_OK;
}

void work(rn_server_t* s) {
  cudaSetDevice(s->device);
  for (;;) {
    // admit arrivals that fit
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->active.empty())
        s->cvWork.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->stop) break;
    }
    for (;;) {
      Request r;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->queue.empty()) break;
        Request& head = s->queue.front();
        if (head.bytes > s->opts.hbm_budget) {
          Done d;
          std::memset(&d.res, 0, sizeof(d.res));
          d.res.status = RN_SOLVE_REJECTED;
          d.res.submit_ms = head.tSubmit;
          d.res.done_ms = s->now_ms();
          s->done[head.id] = std::move(d);
          s->queue.pop_front();
          s->cvDone.notify_all();
          continue;
        }
        if (s->used + head.bytes > s->opts.hbm_budget) break;
        if (s->opts.max_active > 0 && int(s->active.size()) >= s->opts.max_active) break;
        const long long hc = (long long)head.Nx * head.Nr;
        if (s->opts.max_active_cells > 0 && !s->active.empty() && s->cells + hc > s->opts.max_active_cells) break;
        r = std::move(head);
        s->queue.pop_front();
        s->used += r.bytes;
        s->cells += hc;
        s->admitted++;
      }
      Active a;
      a.req = std::move(r);
      a.tAdmit = s->now_ms();
      int rc = admit(s, a.req, a);
      if (rc != RN_OK) {
        Done d;
        std::memset(&d.res, 0, sizeof(d.res));
        d.res.status = RN_SOLVE_FAILED;
        d.res.submit_ms = a.req.tSubmit;
        d.res.admit_ms = a.tAdmit;
        d.res.done_ms = s->now_ms();
        std::lock_guard<std::mutex> lk(s->mu);
        s->used -= a.req.bytes;
        s->cells -= (long long)a.req.Nx * a.req.Nr;
        s->evicted++;
        s->done[a.req.id] = std::move(d);
        s->cvDone.notify_all();
        continue;
      }
      s->active.push_back(std::move(a));
    }
    if (s->active.empty()) continue;
    int rc = tick(s);
    if (rc != RN_OK) {
      fail_all(s, std::string("solve server: ") + rn_last_error());
      s->cvDone.notify_all();
      break;
    }
    s->cvDone.notify_all();
  }
}

template <class T>
void copy_in(std::vector<T>& v, const T* p, size_t n) {
  v.assign(p, p + n);
}

}  // namespace

extern "C" {

int rn_server_default_opts(rn_server_opts* o) {
  if (!o) return sfail(RN_ERR_ARG, "rn_server_default_opts: NULL");
  std::memset(o, 0, sizeof(*o));
  o->hbm_budget = 0;
  o->max_active = 0;
  o->check_every = 60;
  o->precision = RN_PRECISION_FAST;
  o->tile = RN_TILE_16x15;
  return RN_OK;
}

int rn_server_create(const rn_server_opts* opts, rn_server* out) {
  if (!out) return sfail(RN_ERR_ARG, "rn_server_create: out is NULL");
  *out = nullptr;
  rn_server_opts o;
  rn_server_default_opts(&o);
  if (opts) o = *opts;
  if (o.check_every < 2 || o.tile < 0 || o.tile >= rn::NTILES ||
      (o.precision != RN_PRECISION_FAST && o.precision != RN_PRECISION_EXACT) || o.max_active < 0 ||
      o.max_active_cells < 0)
    return sfail(RN_ERR_ARG, "rn_server_create: bad options");
  int dev = 0;
  RN_CK(cudaGetDevice(&dev));
  if (o.hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    RN_CK(cudaMemGetInfo(&fr, &tot));
    o.hbm_budget = fr / 10 * 8;
  }
  rn_server_t* s = new rn_server_t();
  s->opts = o;
  s->device = dev;
  s->t0 = std::chrono::steady_clock::now();
  s->worker = std::thread(work, s);
  *out = s;
  return RN_OK;
}

int rn_server_destroy(rn_server s) {
  if (!s) return sfail(RN_ERR_ARG, "rn_server_destroy: NULL server");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cvWork.notify_all();
  s->worker.join();
  cudaSetDevice(s->device);
  for (Active& a : s->active) {
    rn_batch_t* b = s->batches[a.cls];
    if (b) rn_batch_remove(b, a.h);
    rn_destroy(a.h);
  }
  for (auto& kv : s->batches)
    if (kv.second) rn_batch_destroy(kv.second);
  cudaFreeHost(s->pinned);
  delete s;
  return RN_OK;
}

int rn_serve_submit(rn_server s, const rn_solve_request* q, long long* id) {
  if (!s || !q || !id) return sfail(RN_ERR_ARG, "rn_serve_submit: bad argument");
  if (q->Nx < 8 || q->Nr < 8 || !q->mask || !q->geoA || !q->geoG || !q->geoM || !q->A || !q->B)
    return sfail(RN_ERR_ARG, "rn_serve_submit: grid or buffers missing");
  if (q->drop <= 0.0 && q->t_end <= 0.0 && q->max_steps <= 0)
    return sfail(RN_ERR_ARG, "rn_serve_submit: no stop criterion");
  if (q->P.inj && !q->injTab) return sfail(RN_ERR_ARG, "rn_serve_submit: P.inj set without an injector table");
  Request r;
  r.Nx = q->Nx;
  r.Nr = q->Nr;
  const size_t N = size_t(q->Nx) * q->Nr, NF = size_t(q->Nx + 1) * (q->Nr + 1);
  copy_in(r.mask, q->mask, N);
  copy_in(r.geoA, q->geoA, NF * 4);
  copy_in(r.geoG, q->geoG, N * 4);
  copy_in(r.geoM, q->geoM, N * 4);
  if (q->jWall) copy_in(r.jWall, q->jWall, size_t(q->Nx) * 4);
  copy_in(r.A, q->A, N * 4);
  copy_in(r.B, q->B, N * 4);
  if (q->injTab) copy_in(r.injTab, q->injTab, size_t(768) * 4);
  if ((q->parcelsA != nullptr) != (q->parcelsB != nullptr))
    return sfail(RN_ERR_ARG, "rn_serve_submit: parcel ring needs both planes");
  if (q->parcelsA) {
    copy_in(r.parA, q->parcelsA, size_t(SPRAY_N) * 4);
    copy_in(r.parB, q->parcelsB, size_t(SPRAY_N) * 4);
    r.parHead = q->parcelHead;
  }
  r.P = q->P;
  r.drop = q->drop;
  r.tEnd = q->t_end;
  r.maxSteps = q->max_steps;
  r.spec = q->spec;
  r.bytes = rn_handle_bytes(q->Nx, q->Nr);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->failed) return sfail(RN_ERR_STATE, s->failMsg);
    r.inject = s->injectNext;
    s->injectNext = 0;
    r.id = s->nextId++;
    r.tSubmit = s->now_ms();
    *id = r.id;
    s->queue.push_back(std::move(r));
  }
  s->cvWork.notify_all();
  return RN_OK;
}

int rn_serve_poll(rn_server s, long long id, rn_solve_result* res, float* A, float* B) {
  if (!s || !res) return sfail(RN_ERR_ARG, "rn_serve_poll: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->done.find(id);
  if (it == s->done.end()) {
    if (id <= 0 || id >= s->nextId) return sfail(RN_ERR_ARG, "rn_serve_poll: unknown request id");
    return RN_NOT_READY;
  }
  *res = it->second.res;
  if (A && !it->second.A.empty()) std::memcpy(A, it->second.A.data(), sizeof(float) * it->second.A.size());
  if (B && !it->second.B.empty()) std::memcpy(B, it->second.B.data(), sizeof(float) * it->second.B.size());
  s->done.erase(it);
  return RN_OK;
}

int rn_serve_wait(rn_server s, long long id, int timeout_ms, rn_solve_result* res, float* A, float* B) {
  if (!s || !res) return sfail(RN_ERR_ARG, "rn_serve_wait: bad argument");
  {
    std::unique_lock<std::mutex> lk(s->mu);
    if (id <= 0 || id >= s->nextId) return sfail(RN_ERR_ARG, "rn_serve_wait: unknown request id");
    const bool ok = s->cvDone.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)),
                                       [&] { return s->done.count(id) > 0; });
    if (!ok) return RN_NOT_READY;
  }
  return rn_serve_poll(s, id, res, A, B);
}

int rn_serve_stats(rn_server s, rn_serve_status* out) {
  if (!s || !out) return sfail(RN_ERR_ARG, "rn_serve_stats: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out->queued = (long long)s->queue.size();
  out->active = s->admitted - s->retired;
  out->finished = (long long)s->done.size();
  out->bytes_used = (long long)s->used;
  out->bytes_budget = (long long)s->opts.hbm_budget;
  out->ticks = s->ticks.load();
  out->admitted = s->admitted;
  out->failed = s->failed;
  out->evicted = s->evicted;
  return RN_OK;
}

int rn_serve_inject(rn_server s, int where) {
  if (!s || (where != RN_INJECT_ADMIT && where != RN_INJECT_TICK))
    return sfail(RN_ERR_ARG, "rn_serve_inject: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  s->injectNext = where;
  return RN_OK;
}

int rn_solve_bytes(int Nx, int Nr, long long* bytes) {
  if (Nx < 1 || Nr < 1 || !bytes) return sfail(RN_ERR_ARG, "rn_solve_bytes: bad argument");
  *bytes = (long long)rn_handle_bytes(Nx, Nr);
  return RN_OK;
}

}  // extern "C"
