// server.cuh — the serving loop behind mmp_server_* (include/mmp.h). Included at the
// end of solver.cu: it builds on the batch machinery there (slot pools are batches
// whose slots are filled and emptied between graph replays).
//
// One worker thread owns the device:
//   1. admit  — scan the waiting requests in submission order; a request joins a pool
//               of its kernel shape (nt, precision, Raman, tableau) with a free slot, or
//               a new pool, if its device footprint fits the memory budget (first fit:
//               a large request that does not fit yet does not block smaller ones).
//               Admission allocates the solve's state, uploads it, transforms the
//               initial field, sets the solve's device step limit to its n_steps and
//               computes U for its first stage.
//   2. tick   — every pool with solves replays its captured steps_per_tick-step graph
//               on its own stream (pools overlap on the device); solves whose step
//               counter reached their limit are skipped by the kernels.
//   3. retire — finished solves are transformed back (getResult) into host memory,
//               their state is freed and their slot emptied; waiters are notified.
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
  bool done = false;
  uint64_t steps = 0;
  double t_submit = 0, t_start = -1, t_done = -1;
  std::vector<double> result;
  // placement while running
  int pool = -1;
  uint32_t slot = 0;
  uint64_t steps_run = 0;
  size_t bytes = 0;
};

struct Pool {
  mmp_batch* b = nullptr;
  std::vector<Request*> slot_req;  // request in each slot (nullptr = free)
  int used = 0;
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
  uint64_t used_bytes = 0;
  std::chrono::steady_clock::time_point t0;
  int fatal = MMP_OK;  // a CUDA error the worker could not recover from
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

bool pool_matches(const Pool& pl, const mmp_params* p) { return pl.b && same_shape(pl.b, p); }

// Create an empty pool (no solves yet) for the shape of p.
int pool_open(mmp_server* sv, const mmp_params* p, int* index) {
  Tableau tab;
  tableau_for(p, tab);
  mmp_batch* b = new mmp_batch();
  b->capacity = sv->cfg.max_slots;
  b->members.resize(b->capacity);
  b->active.assign(b->capacity, 0);
  int rc = batch_open(b, p, tab);
  if (rc == MMP_OK) rc = upload_desc(b);
  if (rc) {
    mmp_batch_destroy(b);
    return rc;
  }
  Pool pl;
  pl.b = b;
  pl.slot_req.assign(b->capacity, nullptr);
  sv->pools.push_back(pl);
  *index = (int)sv->pools.size() - 1;
  return MMP_OK;
}

// Device bytes the request will hold (state block), from the host setup alone.
size_t footprint(const mmp_batch* shape_of, const mmp_params* p) {
  Member m;
  host_setup(p, m);
  return member_bytes(shape_of, m);
}

int admit(mmp_server* sv, Request* r, int pi, uint32_t slot) {
  Pool& pl = sv->pools[pi];
  mmp_batch* b = pl.b;
  int rc = member_init(b, slot, &r->p);
  if (rc) return rc;
  Member& s = b->members[slot];
  s.desc.step_limit = r->p.n_steps;  // this solve stops at its own step count
  rc = upload_desc(b);
  if (rc) return rc;
  batch_shape(b);
  rc = launch_row_kernel(b, b->ks, b->ks.prime, (int)s.M, 1, 0, b->d_descs + slot);
  if (rc) return rc;
  pl.slot_req[slot] = r;
  pl.used += 1;
  r->pool = pi;
  r->slot = slot;
  r->bytes = s.bytes;
  r->t_start = sv->now();
  sv->used_bytes += s.bytes;
  return MMP_OK;
}

void release(mmp_server* sv, Request* r) {
  Pool& pl = sv->pools[r->pool];
  mmp_batch* b = pl.b;
  Member& s = b->members[r->slot];
  if (s.block) cudaFree(s.block);
  if (s.energy) cudaFree(s.energy);
  s = Member();
  b->active[r->slot] = 0;
  upload_desc(b);
  batch_shape(b);
  pl.slot_req[r->slot] = nullptr;
  pl.used -= 1;
  sv->used_bytes -= r->bytes;
}

void finish(mmp_server* sv, Request* r, int status) {
  std::lock_guard<std::mutex> lk(sv->mu);
  r->status = status;
  r->done = true;
  r->t_done = sv->now();
  sv->cv_done.notify_all();
}

void worker_loop(mmp_server* sv) {
  cudaSetDevice(sv->device);
  const int K = (int)sv->cfg.steps_per_tick;
  while (true) {
    // ---- admit
    std::vector<Request*> batch_in;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      bool any_active = false;
      for (auto& pl : sv->pools) any_active |= pl.used > 0;
      if (!any_active && sv->waiting.empty() && !sv->stop)
        sv->cv_work.wait_for(lk, std::chrono::milliseconds(20));
      if (sv->stop) break;
      batch_in.assign(sv->waiting.begin(), sv->waiting.end());
    }
    for (Request* r : batch_in) {
      int rc = sv->fatal;  // after a device failure every waiting request fails with it
      int pi = -1;
      for (size_t i = 0; rc == MMP_OK && i < sv->pools.size(); ++i)
        if (pool_matches(sv->pools[i], &r->p) && sv->pools[i].used < (int)sv->pools[i].b->capacity) {
          pi = (int)i;
          break;
        }
      if (rc == MMP_OK && pi < 0) rc = pool_open(sv, &r->p, &pi);
      if (rc == MMP_OK) {
        const size_t need = footprint(sv->pools[pi].b, &r->p);
        if (sv->used_bytes + need > sv->cfg.memory_budget) {
          if (sv->used_bytes != 0) continue;  // first fit: try the next waiting request
          rc = fail(MMP_ENOMEM, "request larger than the server's memory budget");
        }
      }
      uint32_t slot = 0;
      bool attempted = false;
      if (rc == MMP_OK) {
        while (sv->pools[pi].slot_req[slot]) ++slot;
        attempted = true;
        rc = admit(sv, r, pi, slot);
      }
      {
        std::lock_guard<std::mutex> lk(sv->mu);
        auto it = std::find(sv->waiting.begin(), sv->waiting.end(), r);
        if (it != sv->waiting.end()) sv->waiting.erase(it);
      }
      if (rc) {
        Pool* pl = attempted ? &sv->pools[pi] : nullptr;
        if (pl && pl->b->members[slot].block && !pl->slot_req[slot]) {  // partly admitted: undo
          Member& s = pl->b->members[slot];
          cudaFree(s.block);
          if (s.energy) cudaFree(s.energy);
          s = Member();
          pl->b->active[slot] = 0;
          upload_desc(pl->b);
          batch_shape(pl->b);
        }
        finish(sv, r, rc);
      }
    }
    // ---- tick: one graph replay per pool with solves, pools on their own streams
    bool ran = false;
    for (auto& pl : sv->pools) {
      if (pl.used == 0) continue;
      mmp_batch* b = pl.b;
      int rc = build_graph(b, K);
      if (rc == MMP_OK) {
        cudaError_t e = cudaGraphLaunch(b->graph, b->stream);
        if (e != cudaSuccess) rc = fail(MMP_ECUDA, cudaGetErrorString(e));
        else g_launches.fetch_add((uint64_t)K * b->kernels_per_step, std::memory_order_relaxed);
      }
      if (rc) {
        sv->fatal = rc;
      }
      ran = true;
    }
    if (!ran) continue;
    // ---- retire
    for (size_t pi = 0; pi < sv->pools.size(); ++pi) {
      Pool& pl = sv->pools[pi];
      if (pl.used == 0) continue;
      cudaError_t e = cudaStreamSynchronize(pl.b->stream);
      if (e != cudaSuccess && sv->fatal == MMP_OK) sv->fatal = fail(MMP_ECUDA, cudaGetErrorString(e));
      for (uint32_t slot = 0; slot < pl.b->capacity; ++slot) {
        Request* r = pl.slot_req[slot];
        if (!r) continue;
        r->steps_run = std::min<uint64_t>(r->steps_run + K, r->p.n_steps);
        if (r->steps_run < r->p.n_steps && sv->fatal == MMP_OK) continue;
        // finished (or the device failed): status bits, then the result
        const Member& s = pl.b->members[slot];
        int st = 0;
        int status = sv->fatal;
        if (status == MMP_OK) {
          cudaError_t e = cudaMemcpy(&st, (char*)s.counters + 3 * sizeof(unsigned long long), sizeof(int),
                                     cudaMemcpyDeviceToHost);
          if (e != cudaSuccess) status = fail(MMP_ECUDA, cudaGetErrorString(e));
          else if (st & kStatusTimeout) status = MMP_ETIMEOUT;
          else if (st & kStatusNonFinite) status = MMP_ENONFINITE;
        }
        std::vector<double> out((size_t)2 * r->p.n_modes * r->p.nt);
        if (status == MMP_OK) status = member_result(pl.b, slot, out.data());
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          r->result.swap(out);
          r->steps = r->steps_run;
        }
        release(sv, r);
        finish(sv, r, status);
      }
    }
  }
}

int copy_request(const mmp_params* p, Request* r) {
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
  return MMP_OK;
}

}  // namespace

extern "C" {

int mmp_server_create(const mmp_server_config* cfg, mmp_server** out) {
  if (!out) return fail(MMP_EINVAL, "out is NULL");
  *out = nullptr;
  mmp_server* sv = new mmp_server();
  if (cfg) sv->cfg = *cfg;
  if (!sv->cfg.max_slots) sv->cfg.max_slots = 64;
  if (!sv->cfg.steps_per_tick) sv->cfg.steps_per_tick = 32;
  cudaError_t e = cudaGetDevice(&sv->device);
  if (e != cudaSuccess) {
    delete sv;
    return fail(MMP_ECUDA, cudaGetErrorString(e));
  }
  DeviceRes* res = nullptr;
  int rc = ensure_device(sv->device, &res);
  if (rc) {
    delete sv;
    return rc;
  }
  if (!sv->cfg.memory_budget) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    sv->cfg.memory_budget = (uint64_t)(0.8 * (double)fr);
  }
  sv->t0 = std::chrono::steady_clock::now();
  sv->worker = std::thread(worker_loop, sv);
  *out = sv;
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
  sv->requests.erase(it);
  if (status) return fail(status, "request failed");
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
  for (auto& pl : sv->pools) mmp_batch_destroy(pl.b);
  delete sv;
}

}  // extern "C"
