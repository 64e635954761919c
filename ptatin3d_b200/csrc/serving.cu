// Solve server: a persistent request loop for independent Stokes solves.
//
// Requests (a whole mesh, coefficients, density, gravity, solver options)
// arrive with p3d_server_submit and are admitted first-in first-out as soon
// as a worker and the HBM they need are free.  A worker solves its request in
// a rolling group (solver_group_run): lock-step FGMRES with every kernel
// launched once for all members.  The group starts with the queued requests
// of the head's shape and options that fit (up to group_max); at the start of
// every restart cycle queued requests of that shape join it, and a member
// leaves -- its solution copied out and its result posted -- as soon as it
// converges, fails, is cancelled or reaches max_it, while the others go on.
// Each of the `max_active` workers runs on its own CUDA streams, with all of
// its solves' state (hierarchy, Krylov bases, captured preconditioner graph)
// resident in device memory; the groups of different workers overlap on the
// device.  Finished solvers go back to a pool keyed by mesh and options, so a
// later request of the same shape reuses the device memory and only uploads
// new coefficients (no cudaMalloc/cudaFree on the hot path).  Idle pooled
// solvers are released, least recently used first, when a request needs
// their memory.
//
// No counterpart in the reference (pTatin3d runs one solve per process); the
// per-request solve is p3d_solver_*.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "p3d_b200.h"
#include "p3d_internal.h"
#include "solver_internal.h"

namespace p3d {

static double wall_ms()
{
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Slot {
  p3d_solver *solver = nullptr;
  int32_t mx = 0, my = 0, mz = 0;
  uint32_t dirichlet = 0;
  p3d_solver_opts opts;
  int64_t bytes = 0;
  double *coords = nullptr, *eta = nullptr, *rho = nullptr, *u = nullptr, *p = nullptr;
  cudaStream_t io = nullptr; // host<->device copies of this slot
  bool busy = false;
  bool ready = false; // created (device memory held)
  uint64_t last_used = 0;
};

struct Pending {
  p3d_request req;
  double t_submit;
};

static bool same_opts(const p3d_solver_opts &a, const p3d_solver_opts &b)
{
  return a.nlevels == b.nlevels && a.cheb_its == b.cheb_its && a.cheb_lo == b.cheb_lo && a.cheb_hi == b.cheb_hi &&
         a.esteig_its == b.esteig_its && a.mg_precision == b.mg_precision && a.restart == b.restart &&
         a.max_it == b.max_it && a.rtol == b.rtol && a.atol == b.atol && a.use_graph == b.use_graph &&
         a.verbose == b.verbose && a.inner_its == b.inner_its && a.coarse_op == b.coarse_op &&
         a.schur_eta == b.schur_eta && a.coarse_eta == b.coarse_eta && a.inner_rtol == b.inner_rtol;
}

static bool same_shape(const Slot &s, const p3d_request &r)
{
  return s.mx == r.mx && s.my == r.my && s.mz == r.mz && s.dirichlet == r.dirichlet && same_opts(s.opts, r.opts);
}

static int64_t request_bytes(const p3d_request &r)
{
  p3d_mesh_desc d;
  if (p3d_mesh_desc_whole(r.mx, r.my, r.mz, r.dirichlet, &d)) return -1;
  int64_t b = 0;
  if (p3d_solver_estimate_bytes(&d, &r.opts, &b)) return -1;
  const int64_t nn = (int64_t)(2 * r.mx + 1) * (2 * r.my + 1) * (2 * r.mz + 1), nel = (int64_t)r.mx * r.my * r.mz;
  return b + 8 * (3 * nn + 27 * nel + 27 * nel + 3 * nn + 4 * nel); // slot buffers
}

static void release_slot(Slot *s)
{
  if (s->solver) p3d_solver_destroy(s->solver);
  for (double *q : {s->coords, s->eta, s->rho, s->u, s->p})
    if (q) cudaFree(q);
  if (s->io) cudaStreamDestroy(s->io);
  s->solver = nullptr;
  s->coords = s->eta = s->rho = s->u = s->p = nullptr;
  s->io = nullptr;
  s->ready = false;
}

static int create_slot(Slot *s, int device)
{
  p3d_mesh_desc d;
  int rc = p3d_mesh_desc_whole(s->mx, s->my, s->mz, s->dirichlet, &d);
  if (!rc) rc = p3d_solver_create(&d, &s->opts, device, &s->solver);
  const size_t nn = (size_t)(2 * s->mx + 1) * (2 * s->my + 1) * (2 * s->mz + 1), nel = (size_t)s->mx * s->my * s->mz;
  if (!rc) rc = dev_alloc((void **)&s->coords, 3 * nn * 8, "request coords");
  if (!rc) rc = dev_alloc((void **)&s->eta, 27 * nel * 8, "request eta");
  if (!rc) rc = dev_alloc((void **)&s->rho, 27 * nel * 8, "request rho");
  if (!rc) rc = dev_alloc((void **)&s->u, 3 * nn * 8, "request u");
  if (!rc) rc = dev_alloc((void **)&s->p, 4 * nel * 8, "request p");
  if (!rc) rc = cuda_check(cudaStreamCreateWithFlags(&s->io, cudaStreamNonBlocking), "request stream");
  if (rc) release_slot(s);
  else s->ready = true;
  return rc;
}

// the request's inputs onto the slot's device buffers, solver set-up and
// right-hand side
static int prepare_request(Slot *s, const p3d_request &r)
{
  const size_t nn = (size_t)(2 * r.mx + 1) * (2 * r.my + 1) * (2 * r.mz + 1), nel = (size_t)r.mx * r.my * r.mz;
  cudaStream_t io = s->io;
  int rc = cuda_check(cudaMemcpyAsync(s->coords, r.coords, 3 * nn * 8, cudaMemcpyHostToDevice, io), "h2d coords");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(s->eta, r.eta, 27 * nel * 8, cudaMemcpyHostToDevice, io), "h2d eta");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(s->rho, r.rho, 27 * nel * 8, cudaMemcpyHostToDevice, io), "h2d rho");
  if (!rc) rc = cuda_check(cudaMemsetAsync(s->u, 0, 3 * nn * 8, io), "zero u");
  if (!rc) rc = cuda_check(cudaMemsetAsync(s->p, 0, 4 * nel * 8, io), "zero p");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(io), "h2d sync");
  if (!rc) rc = solver_setup_nowait(s->solver, s->coords, s->eta); // ordered by the io sync above
  if (!rc) rc = solver_rhs_body_force_nowait(s->solver, s->rho, r.gx, r.gy, r.gz);
  return rc;
}

// the solution back to the request's host arrays
static int finish_request(Slot *s, const p3d_request &r)
{
  const size_t nn = (size_t)(2 * r.mx + 1) * (2 * r.my + 1) * (2 * r.mz + 1), nel = (size_t)r.mx * r.my * r.mz;
  int rc = cuda_check(cudaMemcpyAsync(r.u, s->u, 3 * nn * 8, cudaMemcpyDeviceToHost, s->io), "d2h u");
  if (!rc) rc = cuda_check(cudaMemcpyAsync(r.p, s->p, 4 * nel * 8, cudaMemcpyDeviceToHost, s->io), "d2h p");
  if (!rc) rc = cuda_check(cudaStreamSynchronize(s->io), "d2h sync");
  return rc;
}

// requests that can share grouped launches: one V-cycle per outer iteration
static bool groupable(const p3d_request &r)
{
  return r.opts.inner_its == 0 && r.opts.inner_rtol == 0.0 && r.opts.nlevels >= 2 && r.opts.use_graph;
}

static bool same_group(const p3d_request &a, const p3d_request &b)
{
  return groupable(a) && groupable(b) && a.mx == b.mx && a.my == b.my && a.mz == b.mz && a.dirichlet == b.dirichlet &&
         same_opts(a.opts, b.opts);
}

// an admitted request in the hands of a worker
struct Job {
  Pending pend;
  Slot *slot = nullptr;
  bool fresh = false;
  double t_admit = 0.0;
  std::atomic<int> cancel{0};
};

} // namespace p3d

using namespace p3d;

struct p3d_server {
  int device = 0;
  int64_t budget = 0;
  int max_active = 1;
  int group_max = 8; // requests of one shape solved together by one worker
  int64_t group_elements = 16384; // larger meshes are solved alone
  double overtake_ms = 2000.0;     // see gather()
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> queue;
  std::vector<Slot *> slots;
  std::deque<p3d_result> done;
  std::vector<std::thread> workers;
  bool stopping = false;
  std::vector<std::pair<int64_t, std::atomic<int> *>> running; // tags of the solves in progress, their cancel flags
  int active = 0;
  int64_t bytes = 0, peak = 0;
  uint64_t clock = 0;
  p3d_server_stats st{};
};

namespace p3d {

// Under the lock: pick (or reserve memory for) a slot for the queue head.
// Returns the slot, or nullptr when the head must wait.  `evict` collects idle
// slots to release outside the lock.
static Slot *admit_request(p3d_server *S, const p3d_request &r, std::vector<Slot *> &evict, bool &fresh, bool &too_big)
{
  fresh = false;
  too_big = false;
  for (Slot *s : S->slots)
    if (s->ready && !s->busy && same_shape(*s, r)) return s;
  const int64_t need = request_bytes(r);
  if (need < 0 || need > S->budget) {
    too_big = true;
    return nullptr;
  }
  // release idle slots (least recently used first) until the request fits
  while (S->bytes + need > S->budget) {
    Slot *lru = nullptr;
    for (Slot *s : S->slots)
      if (s->ready && !s->busy && (!lru || s->last_used < lru->last_used)) lru = s;
    if (!lru) return nullptr; // wait for a running solve to finish
    lru->ready = false;
    S->bytes -= lru->bytes;
    S->slots.erase(std::find(S->slots.begin(), S->slots.end(), lru));
    evict.push_back(lru);
  }
  Slot *s = new Slot();
  s->mx = r.mx; s->my = r.my; s->mz = r.mz;
  s->dirichlet = r.dirichlet;
  s->opts = r.opts;
  s->bytes = need;
  S->bytes += need;
  S->peak = std::max(S->peak, S->bytes);
  S->slots.push_back(s);
  fresh = true;
  return s;
}

// Under the lock: the request leaves the queue for a worker (slot chosen)
static Job *take_job(p3d_server *S, std::deque<std::unique_ptr<Job>> &jobs, const Pending &pend, Slot *slot, bool fresh)
{
  jobs.push_back(std::make_unique<Job>());
  Job *jb = jobs.back().get();
  jb->pend = pend;
  jb->slot = slot;
  jb->fresh = fresh;
  jb->t_admit = wall_ms();
  slot->busy = true;
  S->active++;
  S->st.admitted++;
  if (fresh) S->st.solvers_created++;
  else S->st.solvers_reused++;
  S->running.emplace_back(pend.req.tag, &jb->cancel);
  return jb;
}

// Under the lock: the job's result is posted and its slot goes back to the pool
static void post_job(p3d_server *S, Job *jb, int status, int iterations, double rel_residual)
{
  p3d_result res;
  memset(&res, 0, sizeof res);
  const double t = wall_ms();
  res.tag = jb->pend.req.tag;
  res.status = status;
  res.iterations = iterations;
  res.rel_residual = rel_residual;
  res.wait_ms = jb->t_admit - jb->pend.t_submit;
  res.run_ms = t - jb->t_admit;
  res.latency_ms = t - jb->pend.t_submit;
  for (auto it = S->running.begin(); it != S->running.end(); ++it)
    if (it->second == &jb->cancel) { S->running.erase(it); break; }
  Slot *sl = jb->slot;
  sl->busy = false;
  sl->last_used = ++S->clock;
  if (!sl->ready) { // creation failed: give the memory back
    S->bytes -= sl->bytes;
    S->slots.erase(std::find(S->slots.begin(), S->slots.end(), sl));
    delete sl;
  }
  jb->slot = nullptr;
  S->active--;
  S->done.push_back(res);
  S->st.completed++;
  S->cv_done.notify_all();
  S->cv_work.notify_all();
}

// Outside the lock: the job's slot created (if new) and its request set up;
// a cancelled job is not set up
static int start_job(p3d_server *S, Job *jb)
{
  int rc = jb->fresh ? create_slot(jb->slot, S->device) : P3D_OK;
  if (!rc) rc = prepare_request(jb->slot, jb->pend.req);
  if (!rc && jb->cancel.load()) rc = P3D_ERR_CANCELLED;
  return rc;
}

// Under the lock: queued requests that can join a group of `ref`'s shape
// (slots and memory permitting), up to `room`
static int gather(p3d_server *S, const p3d_request &ref, int room, std::deque<std::unique_ptr<Job>> &jobs,
                  std::vector<Job *> &got, std::vector<Slot *> &evict)
{
  int n = 0;
  double t_other = -1.0; // arrival of the oldest queued request of another shape
  for (auto it = S->queue.begin(); it != S->queue.end() && n < room;) {
    if (!same_group(it->req, ref)) {
      if (t_other < 0) t_other = it->t_submit;
      ++it;
      continue;
    }
    // fairness: no request overtakes one of another shape that arrived more
    // than overtake_ms before it (the queue is in arrival order)
    if (t_other >= 0 && it->t_submit - t_other > S->overtake_ms) break;
    bool f = false, big = false;
    Slot *sl = admit_request(S, it->req, evict, f, big);
    if (!sl) break; // no slot or memory for more now
    got.push_back(take_job(S, jobs, *it, sl, f));
    it = S->queue.erase(it);
    n++;
  }
  return n;
}

static void worker(p3d_server *S)
{
  cudaSetDevice(S->device);
  std::unique_lock<std::mutex> lk(S->mu);
  std::deque<std::unique_ptr<Job>> jobs; // this worker's jobs (stable addresses for the cancel flags)
  auto release = [&](std::vector<Slot *> &evict) {
    for (Slot *e : evict) { release_slot(e); delete e; }
    evict.clear();
  };
  for (;;) {
    jobs.clear();
    if (S->queue.empty()) {
      if (S->stopping) return;
      S->cv_work.wait(lk);
      continue;
    }
    std::vector<Slot *> evict;
    bool fresh = false, too_big = false;
    Slot *slot = admit_request(S, S->queue.front().req, evict, fresh, too_big);
    if (!slot && !too_big) {
      if (!evict.empty()) { // memory was given back: release it and look again
        lk.unlock();
        release(evict);
        lk.lock();
        continue;
      }
      S->cv_work.wait(lk);
      continue;
    }
    Pending head = S->queue.front();
    S->queue.pop_front();
    if (too_big) {
      p3d_result res;
      memset(&res, 0, sizeof res);
      res.tag = head.req.tag;
      res.status = P3D_ERR_NOMEM;
      res.wait_ms = res.latency_ms = wall_ms() - head.t_submit;
      S->done.push_back(res);
      S->st.completed++;
      S->cv_done.notify_all();
      continue;
    }
    Job *first = take_job(S, jobs, head, slot, fresh);
    const int gmax = std::min(S->group_max, P3D_GROUP_MAX);
    std::vector<Job *> batch{first};
    const bool group = gmax > 1 && groupable(head.req) &&
                       (int64_t)head.req.mx * head.req.my * head.req.mz <= S->group_elements;
    if (group) gather(S, head.req, gmax - 1, jobs, batch, evict);
    S->cv_work.notify_all(); // the next request may fit as well
    lk.unlock();
    release(evict);
    if (!group) {
      // solved alone
      p3d_solve_stats st;
      memset(&st, 0, sizeof st);
      int rc = start_job(S, first);
      if (!rc) {
        solver_set_cancel_flag(first->slot->solver, &first->cancel);
        rc = solver_solve_nowait(first->slot->solver, first->slot->u, first->slot->p, &st);
        solver_set_cancel_flag(first->slot->solver, nullptr);
        if (rc == P3D_OK || rc == P3D_ERR_NOCONV || rc == P3D_ERR_CANCELLED) {
          const int fr = finish_request(first->slot, first->pend.req);
          if (fr) rc = fr;
        }
      }
      lk.lock();
      post_job(S, first, rc, st.iterations, st.r0 > 0 ? st.rfinal / st.r0 : 0.0);
      continue;
    }
    // a rolling group: members set up here; later arrivals of the shape join
    // at restart boundaries; each member is posted when it leaves
    bool shared = false;
    auto ready_members = [&](const std::vector<Job *> &js, GroupMember *out) -> int {
      int n = 0;
      for (Job *jb : js) {
        const int rc = start_job(S, jb);
        if (rc) {
          std::lock_guard<std::mutex> g(S->mu);
          post_job(S, jb, rc, 0, 0.0);
          continue;
        }
        solver_set_cancel_flag(jb->slot->solver, &jb->cancel);
        out[n].solver = jb->slot->solver;
        out[n].u = jb->slot->u;
        out[n].p = jb->slot->p;
        out[n].tag = jb;
        n++;
      }
      return n;
    };
    GroupHooks hooks;
    hooks.admit = [&](int room, GroupMember *add) -> int {
      std::vector<Job *> got;
      std::vector<Slot *> ev;
      {
        std::lock_guard<std::mutex> g(S->mu);
        gather(S, head.req, room, jobs, got, ev);
      }
      release(ev);
      return got.empty() ? 0 : ready_members(got, add);
    };
    hooks.leave = [&](const GroupMember &m, int status, const p3d_solve_stats &st) {
      Job *jb = static_cast<Job *>(m.tag);
      solver_set_cancel_flag(jb->slot->solver, nullptr);
      int sk = status;
      if (sk == P3D_OK || sk == P3D_ERR_NOCONV || sk == P3D_ERR_CANCELLED) {
        const int fr = finish_request(jb->slot, jb->pend.req);
        if (fr) sk = fr;
      }
      std::lock_guard<std::mutex> g(S->mu);
      if (st.group_members > 1) {
        S->st.grouped++;
        if (!shared) S->st.groups++; // counted before the first shared result is posted
        shared = true;
      }
      post_job(S, jb, sk, st.iterations, st.r0 > 0 ? st.rfinal / st.r0 : 0.0);
    };
    GroupMember mem[P3D_GROUP_MAX];
    const int n = ready_members(batch, mem);
    if (n) solver_group_run(mem, n, gmax, hooks);
    lk.lock();
  }
}

} // namespace p3d

extern "C" {

int p3d_server_create(int device, int64_t hbm_budget_bytes, int32_t max_active, p3d_server **out)
{
  if (!out || hbm_budget_bytes <= 0 || max_active < 1 || max_active > 256)
    return set_error(P3D_ERR_ARG, "server_create: bad arguments");
  *out = nullptr;
  int rc = cuda_check(cudaSetDevice(device), "cudaSetDevice");
  if (rc) return rc;
  p3d_server *S = new p3d_server();
  S->device = device;
  S->budget = hbm_budget_bytes;
  S->max_active = max_active;
  for (int i = 0; i < max_active; i++) S->workers.emplace_back(worker, S);
  *out = S;
  return P3D_OK;
}

int p3d_server_set_group_max(p3d_server *S, int32_t group_max)
{
  if (!S || group_max < 1 || group_max > P3D_GROUP_MAX)
    return set_error(P3D_ERR_ARG, "server_set_group_max: 1..%d", P3D_GROUP_MAX);
  std::lock_guard<std::mutex> g(S->mu);
  S->group_max = group_max;
  return P3D_OK;
}

int p3d_server_set_group_overtake_ms(p3d_server *S, int32_t ms)
{
  if (!S || ms < 0) return set_error(P3D_ERR_ARG, "server_set_group_overtake_ms: bad arguments");
  std::lock_guard<std::mutex> g(S->mu);
  S->overtake_ms = ms;
  return P3D_OK;
}

int p3d_server_set_group_elements(p3d_server *S, int64_t max_elements)
{
  if (!S || max_elements < 0) return set_error(P3D_ERR_ARG, "server_set_group_elements: bad arguments");
  std::lock_guard<std::mutex> g(S->mu);
  S->group_elements = max_elements;
  return P3D_OK;
}

int p3d_server_submit(p3d_server *S, const p3d_request *req)
{
  if (!S || !req || !req->coords || !req->eta || !req->rho || !req->u || !req->p || req->mx < 1 || req->my < 1 ||
      req->mz < 1)
    return set_error(P3D_ERR_ARG, "server_submit: bad request");
  std::lock_guard<std::mutex> g(S->mu);
  if (S->stopping) return set_error(P3D_ERR_STATE, "server_submit: server is shutting down");
  S->queue.push_back(Pending{*req, wall_ms()});
  S->st.submitted++;
  S->cv_work.notify_one();
  return P3D_OK;
}

int p3d_server_poll(p3d_server *S, p3d_result *results, int32_t max_results, int32_t timeout_ms, int32_t *n)
{
  if (!S || !results || !n || max_results < 1) return set_error(P3D_ERR_ARG, "server_poll: bad arguments");
  *n = 0;
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->done.empty() && timeout_ms > 0 &&
      !S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [S] { return !S->done.empty(); }))
    return set_error(P3D_ERR_TIMEOUT, "server_poll: no result within %d ms", (int)timeout_ms);
  int k = 0;
  while (k < max_results && !S->done.empty()) {
    results[k++] = S->done.front();
    S->done.pop_front();
  }
  *n = k;
  return P3D_OK;
}

int p3d_server_cancel(p3d_server *S, int64_t tag)
{
  if (!S) return set_error(P3D_ERR_ARG, "server_cancel: null server");
  std::lock_guard<std::mutex> g(S->mu);
  for (auto it = S->queue.begin(); it != S->queue.end(); ++it)
    if (it->req.tag == tag) {
      p3d_result res;
      memset(&res, 0, sizeof res);
      res.tag = tag;
      res.status = P3D_ERR_CANCELLED;
      res.wait_ms = res.latency_ms = wall_ms() - it->t_submit;
      S->queue.erase(it);
      S->done.push_back(res);
      S->st.completed++;
      S->cv_done.notify_all();
      S->cv_work.notify_all();
      return P3D_OK;
    }
  for (auto &r : S->running)
    if (r.first == tag) {
      r.second->store(1);
      return P3D_OK;
    }
  return set_error(P3D_ERR_ARG, "server_cancel: no queued or running request has tag %lld", (long long)tag);
}

int p3d_server_get_stats(p3d_server *S, p3d_server_stats *st)
{
  if (!S || !st) return set_error(P3D_ERR_ARG, "server_get_stats: null argument");
  std::lock_guard<std::mutex> g(S->mu);
  *st = S->st;
  st->active = S->active;
  st->queued = (int32_t)S->queue.size();
  st->device_bytes = S->bytes;
  st->peak_device_bytes = S->peak;
  return P3D_OK;
}

int p3d_server_destroy(p3d_server *S)
{
  if (!S) return P3D_OK;
  {
    std::lock_guard<std::mutex> g(S->mu);
    S->stopping = true;
  }
  S->cv_work.notify_all();
  for (auto &t : S->workers) t.join();
  cudaSetDevice(S->device);
  for (Slot *s : S->slots) {
    release_slot(s);
    delete s;
  }
  delete S;
  return P3D_OK;
}

} // extern "C"
