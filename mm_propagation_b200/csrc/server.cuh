// server.cuh — the serving loop behind mmp_server_* (include/mmp.h). Included at the
// end of solver.cu: it builds on the batch machinery there (slot pools are batches
// whose slots are filled and emptied between graph replays).
//
// One worker thread owns the device and never waits for the device as a whole; every
// pool (a batch of solves of one kernel shape: nt, precision, Raman, tableau) runs on
// its own stream and progresses at its own pace:
//   * complete — a pool whose last replay finished (its event has fired) credits its
//                solves with steps_per_tick steps; finished solves are transformed back
//                (getResult) into host memory, their state returns to the stream-ordered
//                memory pool and their slot is emptied; waiters are notified.
//   * admit    — waiting requests, in submission order, join an idle pool of their shape
//                with a free slot (or a new pool) if their device footprint fits the
//                memory budget (first fit: a request that does not fit yet does not block
//                smaller ones behind it). Admission allocates and uploads the solve's
//                state, transforms its initial field, sets its device step limit to its
//                n_steps and computes U for its first stage.
//   * launch   — every idle pool with solves replays its captured steps_per_tick-step
//                graph and records an event. Solves whose step counter reached their
//                limit are skipped by the kernels until they are retired.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

namespace {

struct Request {
  uint64_t id = 0;
  // deep copy of the caller's parameters
  mmp_params p{};
  std::vector<double> beta, fields, raman;
  std::vector<mmp_nz> nz;
  // outcome
  int status = MMP_OK;
  std::string error;  // the failure's text, recorded on the worker thread
  bool done = false;
  uint64_t steps = 0;
  double t_submit = 0, t_start = -1, t_done = -1;
  std::vector<double> result;
  // its device bytes and its contribution to a pool's launch shape, computed once
  // (worker thread only)
  bool sized = false, counted = false;
  size_t need = 0;
  SolveCounts counts;
  // placement while running (worker thread only)
  int pool = -1;
  uint32_t slot = 0;
  uint64_t steps_run = 0;
  size_t bytes = 0;
};

struct Pool {
  mmp_batch* b = nullptr;
  std::vector<Request*> slot_req;  // request in each slot (nullptr = free)
  int used = 0;
  cudaEvent_t done_ev = nullptr;   // recorded after each replay
  bool in_flight = false;
};

}  // namespace

struct mmp_server {
  mmp_server_config cfg{};
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  int device = 0;
  uint64_t next_id = 1;
  std::deque<Request*> waiting;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> requests;
  std::vector<Pool> pools;
  cudaMemPool_t mempool = nullptr;
  uint64_t used_bytes = 0;
  std::chrono::steady_clock::time_point t0;
  int fatal = MMP_OK;  // a CUDA error the worker could not recover from
  std::string fatal_msg;  // its text (the worker's own last-error is thread-local)
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

// Create an empty pool (no solves yet) for the shape of p.
int pool_open(mmp_server* sv, const mmp_params* p, int* index) {
  Tableau tab;
  tableau_for(p, tab);
  mmp_batch* b = new mmp_batch();
  b->capacity = sv->cfg.max_slots;
  b->members.resize(b->capacity);
  b->active.assign(b->capacity, 0);
  b->mempool = sv->mempool;
  int rc = batch_open(b, p, tab);
  if (rc == MMP_OK) rc = upload_desc(b);
  Pool pl;
  if (rc == MMP_OK) {
    cudaError_t e = cudaEventCreateWithFlags(&pl.done_ev, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = fail(MMP_ECUDA, cudaGetErrorString(e));
  }
  if (rc) {
    mmp_batch_destroy(b);
    return rc;
  }
  pl.b = b;
  pl.slot_req.assign(b->capacity, nullptr);
  sv->pools.push_back(pl);
  *index = (int)sv->pools.size() - 1;
  return MMP_OK;
}

// Device bytes the request will hold (state block), from the host setup alone.
size_t footprint(const mmp_params* p) {
  mmp_batch shape;
  shape.fp64 = (p->flags & MMP_F_FP64) != 0;
  shape.raman = p->raman != 0;
  shape.nt = p->nt;
  tableau_for(p, shape.tab);
  Member m;
  host_setup(p, m);
  return member_bytes(&shape, m);
}

// Empty slot `slot` of pool `pl`: state back to the memory pool (stream-ordered).
void clear_slot(Pool& pl, uint32_t slot) {
  mmp_batch* b = pl.b;
  Member& s = b->members[slot];
  dev_free(s.block, b->stream, true);
  dev_free(s.energy);
  s = Member();
  b->active[slot] = 0;
  upload_desc(b);
  batch_shape(b);
}

int admit(mmp_server* sv, Request* r, int pi, uint32_t slot) {
  Pool& pl = sv->pools[pi];
  mmp_batch* b = pl.b;
  int rc = member_init(b, slot, &r->p);
  Member& s = b->members[slot];
  if (rc == MMP_OK) {
    s.desc.step_limit = r->p.n_steps;  // this solve stops at its own step count
    rc = upload_desc(b);
  }
  if (rc == MMP_OK) {
    batch_shape(b);
    rc = launch_row_kernel(b, b->ks, b->ks.prime, (int)s.M, 1, 0, b->d_descs + slot);
  }
  if (rc) {
    if (s.block || b->active[slot]) clear_slot(pl, slot);
    return rc;
  }
  pl.slot_req[slot] = r;
  pl.used += 1;
  r->pool = pi;
  r->slot = slot;
  r->bytes = s.bytes;
  r->t_start = sv->now();
  sv->used_bytes += s.bytes;
  return MMP_OK;
}

// The worker thread's failures are recorded in its own thread-local last-error; the
// text travels with the request (and the fatal error with the server) so that the
// client thread's mmp_server_wait can report it through mmp_last_error.
void set_fatal(mmp_server* sv, int rc) {
  if (rc == MMP_OK || sv->fatal != MMP_OK) return;
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->fatal = rc;
  sv->fatal_msg = g_last_error;
}

void finish(mmp_server* sv, Request* r, int status, std::vector<double>* result, const char* msg = nullptr) {
  std::lock_guard<std::mutex> lk(sv->mu);
  if (result) r->result.swap(*result);
  r->steps = r->steps_run;
  r->status = status;
  if (status) r->error = msg ? msg : (sv->fatal == status && !sv->fatal_msg.empty() ? sv->fatal_msg.c_str()
                                                                                     : g_last_error);
  r->done = true;
  r->t_done = sv->now();
  sv->cv_done.notify_all();
}

// A pool's replay finished: credit its solves, retire the finished ones.
void complete(mmp_server* sv, int pi, int K) {
  Pool& pl = sv->pools[pi];
  pl.in_flight = false;
  for (uint32_t slot = 0; slot < pl.b->capacity; ++slot) {
    Request* r = pl.slot_req[slot];
    if (!r) continue;
    r->steps_run = std::min<uint64_t>(r->steps_run + K, r->p.n_steps);
    if (r->steps_run < r->p.n_steps && sv->fatal == MMP_OK) continue;
    const Member& s = pl.b->members[slot];
    int status = sv->fatal;
    const char* msg = nullptr;
    if (status == MMP_OK) {
      int st = 0;
      cudaError_t e = cudaMemcpy(&st, (char*)s.counters + 3 * sizeof(unsigned long long), sizeof(int),
                                 cudaMemcpyDeviceToHost);
      if (e != cudaSuccess) {
        status = fail(MMP_ECUDA, cudaGetErrorString(e));
      } else if (st & kStatusTimeout) {
        status = MMP_ETIMEOUT;
        msg = "a device-side bounded wait gave up";
      } else if (st & kStatusNonFinite) {
        status = MMP_ENONFINITE;
        msg = "non-finite field values (the solve diverged or its input was not finite)";
      } else if (st & kStatusDrift) {
        status = MMP_EDRIFT;
        msg = "the FP64 energy monitor left the band set by the drift limit";
      }
    }
    std::vector<double> out((size_t)2 * r->p.n_modes * r->p.nt);
    if (status == MMP_OK) status = member_result(pl.b, slot, out.data());
    clear_slot(pl, slot);
    pl.slot_req[slot] = nullptr;
    pl.used -= 1;
    sv->used_bytes -= r->bytes;
    finish(sv, r, status, status == MMP_OK ? &out : nullptr, msg);
  }
}

// Admit what fits from the waiting list. Returns true if anything was admitted or failed.
bool admit_waiting(mmp_server* sv) {
  std::vector<Request*> snapshot;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    snapshot.assign(sv->waiting.begin(), sv->waiting.end());
  }
  bool changed = false;
  for (Request* r : snapshot) {
    int rc = sv->fatal;  // after a device failure every waiting request fails with it
    int pi = -1;
    bool deferred = false;
    if (rc == MMP_OK) {
      for (size_t i = 0; i < sv->pools.size(); ++i) {
        Pool& pl = sv->pools[i];
        // a request joins only a pool where it runs the kernels and tiles it runs alone,
        // so its fields are those of a standalone solve whatever it shares the pool with
        if (pl.used >= (int)pl.b->capacity || !same_shape(pl.b, &r->p)) continue;
        if (!r->counted) {
          r->counts = solve_counts(&r->p);
          r->counted = true;
        }
        if (!joins_same_kernels(pl.b, r->counts)) continue;
        if (pl.in_flight) {
          deferred = true;  // a pool with room is busy: try again after its replay
          continue;
        }
        pi = (int)i;
        break;
      }
      if (pi < 0 && deferred) continue;
      if (!r->sized) {  // host setup once per request, not on every pass over the queue
        r->need = footprint(&r->p);
        r->sized = true;
      }
      const size_t need = r->need;
      if (sv->used_bytes + need > sv->cfg.memory_budget) {
        if (sv->used_bytes != 0) continue;  // first fit: try the next waiting request
        rc = fail(MMP_ENOMEM, "request larger than the server's memory budget");
      }
      if (rc == MMP_OK && pi < 0) rc = pool_open(sv, &r->p, &pi);
    }
    if (rc == MMP_OK) {
      uint32_t slot = 0;
      while (sv->pools[pi].slot_req[slot]) ++slot;
      rc = admit(sv, r, pi, slot);
    }
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      auto it = std::find(sv->waiting.begin(), sv->waiting.end(), r);
      if (it != sv->waiting.end()) sv->waiting.erase(it);
    }
    if (rc) finish(sv, r, rc, nullptr);
    changed = true;
  }
  return changed;
}

void worker_loop(mmp_server* sv) {
  cudaSetDevice(sv->device);
  const int K = (int)sv->cfg.steps_per_tick;
  while (true) {
    bool progressed = false, any_in_flight = false;
    // complete
    for (size_t pi = 0; pi < sv->pools.size(); ++pi) {
      Pool& pl = sv->pools[pi];
      if (!pl.in_flight) continue;
      cudaError_t e = cudaEventQuery(pl.done_ev);
      if (e == cudaErrorNotReady) {
        any_in_flight = true;
        continue;
      }
      if (e != cudaSuccess) set_fatal(sv, fail(MMP_ECUDA, cudaGetErrorString(e)));
      mmp_detail::Range range("mmp.server.complete");
      complete(sv, (int)pi, K);
      progressed = true;
    }
    // admit
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      if (sv->stop) break;
      bool any_used = false;
      for (auto& pl : sv->pools) any_used |= pl.used > 0;
      if (!any_used && sv->waiting.empty()) {
        sv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
    }
    {
      mmp_detail::Range range("mmp.server.admit");
      progressed |= admit_waiting(sv);
    }
    // launch
    for (auto& pl : sv->pools) {
      if (pl.in_flight || pl.used == 0) continue;
      mmp_batch* b = pl.b;
      mmp_detail::Range range("mmp.server.launch");
      int rc = build_graph(b, K);
      if (rc == MMP_OK) {
        cudaError_t e = cudaGraphLaunch(b->graph, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(pl.done_ev, b->stream);
        if (e != cudaSuccess) rc = fail(MMP_ECUDA, cudaGetErrorString(e));
        else g_launches.fetch_add((uint64_t)K * b->kernels_per_step, std::memory_order_relaxed);
      }
      set_fatal(sv, rc);
      if (rc) cudaEventRecord(pl.done_ev, b->stream);  // completes at once; solves fail there
      pl.in_flight = true;
      any_in_flight = true;
      progressed = true;
    }
    if (!progressed && any_in_flight) std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
  for (auto& pl : sv->pools)
    if (pl.in_flight) cudaEventSynchronize(pl.done_ev);
}

void copy_request(const mmp_params* p, Request* r) {
  r->p = *p;
  r->beta.assign(p->dispersion, p->dispersion + (size_t)p->n_modes * p->n_beta);
  r->nz.assign(p->coupling, p->coupling + p->n_nonzeros);
  r->fields.assign(p->initial_fields, p->initial_fields + (size_t)2 * p->n_modes * p->nt);
  if (p->raman && p->raman_response) r->raman.assign(p->raman_response, p->raman_response + p->nt);
  r->p.dispersion = r->beta.data();
  r->p.coupling = r->nz.empty() ? nullptr : r->nz.data();
  r->p.initial_fields = r->fields.data();
  r->p.raman_response = r->raman.empty() ? nullptr : r->raman.data();
  r->p.flags |= MMP_F_NO_MONITORS;  // served solves keep no per-step monitors
}

}  // namespace

extern "C" {

int mmp_server_create(const mmp_server_config* cfg, mmp_server** out) {
  if (!out) return fail(MMP_EINVAL, "out is NULL");
  *out = nullptr;
  std::unique_ptr<mmp_server> sv(new mmp_server());
  if (cfg) sv->cfg = *cfg;
  if (!sv->cfg.max_slots) sv->cfg.max_slots = 64;
  if (!sv->cfg.steps_per_tick) sv->cfg.steps_per_tick = 32;
  CUDA_TRY(cudaGetDevice(&sv->device));
  DeviceRes* res = nullptr;
  int rc = ensure_device(sv->device, &res);
  if (rc) return rc;
  if (!sv->cfg.memory_budget) {
    size_t fr = 0, tot = 0;
    CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    sv->cfg.memory_budget = (uint64_t)(0.8 * (double)fr);
  }
  // the server's own stream-ordered pool; freed blocks stay reserved for reuse
  cudaMemPoolProps props;
  std::memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = sv->device;
  CUDA_TRY(cudaMemPoolCreate(&sv->mempool, &props));
  uint64_t keep = ~0ull;
  CUDA_TRY(cudaMemPoolSetAttribute(sv->mempool, cudaMemPoolAttrReleaseThreshold, &keep));
  sv->t0 = std::chrono::steady_clock::now();
  mmp_server* raw = sv.release();
  raw->worker = std::thread(worker_loop, raw);
  *out = raw;
  return MMP_OK;
}

int mmp_server_submit(mmp_server* sv, const mmp_params* params, uint64_t* id) {
  if (!sv || !id) return fail(MMP_EINVAL, "bad submit arguments");
  std::string why;
  int rc = validate(params, why);
  if (rc) return fail(rc, why);
  std::unique_ptr<Request> r(new Request());
  copy_request(params, r.get());
  r->p.flags |= sv->cfg.flags;
  std::lock_guard<std::mutex> lk(sv->mu);
  r->id = sv->next_id++;
  r->t_submit = sv->now();
  *id = r->id;
  sv->waiting.push_back(r.get());
  sv->requests[r->id] = std::move(r);
  sv->cv_work.notify_one();
  return MMP_OK;
}

int mmp_server_poll(mmp_server* sv, uint64_t id, int* done) {
  if (!sv || !done) return fail(MMP_EINVAL, "bad poll arguments");
  std::lock_guard<std::mutex> lk(sv->mu);
  auto it = sv->requests.find(id);
  if (it == sv->requests.end()) return fail(MMP_EINVAL, "unknown request id");
  *done = it->second->done ? 1 : 0;
  return MMP_OK;
}

int mmp_server_wait(mmp_server* sv, uint64_t id, double timeout_s, double* out, mmp_request_info* info) {
  if (!sv) return fail(MMP_EINVAL, "NULL server");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->requests.find(id);
  if (it == sv->requests.end()) return fail(MMP_EINVAL, "unknown request id");
  Request* r = it->second.get();
  auto ready = [&] { return r->done; };
  if (timeout_s < 0) {
    sv->cv_done.wait(lk, ready);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return fail(MMP_ETIMEOUT, "request not finished within the timeout");
  }
  if (info) {
    info->status = r->status;
    info->n_modes = r->p.n_modes;
    info->nt = r->p.nt;
    info->steps = r->steps;
    info->submit_s = r->t_submit;
    info->start_s = r->t_start;
    info->done_s = r->t_done;
  }
  const int status = r->status;
  if (out && status == MMP_OK) std::memcpy(out, r->result.data(), r->result.size() * sizeof(double));
  const std::string why = status ? "request failed: " + r->error : std::string();
  sv->requests.erase(it);
  if (status) return fail(status, why);
  return MMP_OK;
}

void mmp_server_destroy(mmp_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
    sv->cv_work.notify_all();
  }
  if (sv->worker.joinable()) sv->worker.join();
  cudaSetDevice(sv->device);
  for (auto& pl : sv->pools) {
    if (pl.done_ev) cudaEventDestroy(pl.done_ev);
    mmp_batch_destroy(pl.b);
  }
  if (sv->mempool) cudaMemPoolDestroy(sv->mempool);
  delete sv;
}

}  // extern "C"
