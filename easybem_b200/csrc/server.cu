// Continuous-batching solve server (no counterpart in the reference).
//
// A request is one surface mesh with nrhs sets of Dirichlet vertex data g;
// its answer is the Neumann data t solving V t = (1/2 M + K) g for each set.
// Requests pass through four states:
//   queued   -> submitted, waiting for device memory;
//   preparing-> admitted under the memory budget; one of several host worker
//               threads builds the mesh (topology, FP64 Sauter-Schwab near
//               field, preconditioner) and the right-hand sides on the
//               request's own stream, overlapping the solves already running
//               on the GPU (which leave a quarter of the SMs free meanwhile);
//   active   -> its systems joined the shared SolverPool: every step() advances
//               all active systems by one batched GMRES iteration, so requests
//               that arrive later join the running batch as soon as they are
//               prepared and slots (systems) are free;
//   done     -> solutions copied out, latency recorded, Krylov memory and the
//               mesh released (or kept for result reads until release()).
// The budget counts each request's resident mesh data plus the solver's
// Krylov basis and vectors; a request larger than the whole budget is
// rejected at submission.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdlib>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "solver.h"

eb::Mesh* eb_mesh_internal(eb_mesh handle);

namespace eb {

static double now_ms()
{
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Device bytes a mesh keeps resident (geometry, near field, per-apply scratch).
static size_t mesh_resident_bytes(const Mesh* m)
{
  size_t b = 0;
  // the static tables are views into the arena, which is counted once
  const DevBuf* bufs[] = {&m->arena, &m->sl_rowptr, &m->sl_col, &m->sl_val, &m->dl_rowptr,
                          &m->dl_col, &m->dl_val, &m->rec, &m->partial, &m->counter, &m->items, &m->io_t,
                          &m->io_u, &m->io_v, &m->io_q, &m->pc_val};
  for (const DevBuf* d : bufs) b += d->bytes;
  return b;
}

// Estimate before the mesh exists: ~13 near pairs per triangle (SL + DL CSR
// and the pair build), the static tables and the apply scratch.
static size_t estimate_bytes(int nv, int ne, int order, int nrhs, int restart)
{
  Quadrature q;
  make_quadrature(order, &q);
  const size_t Q = q.nt;
  const size_t mesh = (size_t)ne * (13 * (12 + 48) + 400 + Q * (16 + 32 + 8 + 16 + 32 + 3 * 32)) + (size_t)nv * 40;
  const size_t solver = (size_t)nrhs * ne * 8 * (restart + 4) + ((size_t)nrhs + 3) / 4 * ne * (Q * 64 + 160);
  // the symmetric far field's partial slots: kBatchCols outputs per 128-triangle tile and row
  const size_t slots = (size_t)kBatchCols * (((size_t)ne + kTT - 1) / kTT + 1) * ne * 8;
  return mesh + solver + slots;
}

struct Request {
  long long id = 0;
  int nv = 0, ne = 0, order = 4, nrhs = 0;
  std::vector<double> nodes, g;
  std::vector<int> elems;
  std::vector<double> b, x;
  std::vector<SolveStats> stats;
  std::vector<int> sys;
  eb_mesh mesh = nullptr;
  size_t bytes = 0;
  int state = 0;  // 0 queued, 1 preparing, 2 prepared, 3 active, 4 done, 5 failed
  std::string error;
  double t_submit = 0, t_admit = 0, t_active = 0, t_done = 0;
};

class Server {
 public:
  Server(size_t budget, int max_systems, const SolveOptions& o)
      : budget_(budget), max_systems_(max_systems), opt_(o), pool_(o)
  {
    cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking);
    cudaGetDevice(&device_);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device_);
    reserve_sms_ = nsm / 4;
    int nworkers = kPrepWorkers;
    if (const char* e = std::getenv("EASYBEM_PREP_WORKERS")) nworkers = std::max(1, std::min(64, std::atoi(e)));
    for (int k = 0; k < nworkers; k++) workers_.emplace_back([this] { prepare_loop(); });
  }
  ~Server()
  {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& w : workers_) w.join();
    for (auto& kv : reqs_)
      if (kv.second->mesh) eb_mesh_destroy(kv.second->mesh);
    cudaStreamDestroy(stream_);
  }

  int submit(int nv, const double* nodes, int ne, const int* elems, int order, int nrhs, const double* g,
             long long* id)
  {
    if (nv < 3 || ne < 1 || nrhs < 1 || !nodes || !elems || !g) return set_error(EB_ERR_INVALID, "bad request");
    auto r = std::make_shared<Request>();
    r->nv = nv;
    r->ne = ne;
    r->order = order;
    r->nrhs = nrhs;
    r->nodes.assign(nodes, nodes + 3 * (size_t)nv);
    r->elems.assign(elems, elems + 3 * (size_t)ne);
    r->g.assign(g, g + (size_t)nrhs * nv);
    r->bytes = estimate_bytes(nv, ne, order, nrhs, opt_.restart);
    if (r->bytes > budget_)
      return set_error(EB_ERR_NOMEM, "request needs ~" + std::to_string(r->bytes) + " device bytes, budget is " +
                                         std::to_string(budget_));
    r->t_submit = now_ms();
    std::lock_guard<std::mutex> g2(mu_);
    r->id = next_id_++;
    reqs_[r->id] = r;
    queue_.push_back(r);
    *id = r->id;
    admit_locked();
    cv_.notify_all();
    return EB_OK;
  }

  int step(int* nactive, int* nwaiting)
  {
    const double t_enter = now_ms();
    const int rc = step_impl(nactive, nwaiting);
    std::lock_guard<std::mutex> g(mu_);
    n_steps_++;
    t_step_ms_ += now_ms() - t_enter;
    return rc;
  }

  // steps, seconds in step(), batch rebuilds, seconds in them, requests
  // prepared, seconds the preparation workers were busy, of which mesh
  // creation, right-hand sides and preconditioner, mesh creation split into
  // topology, static tables and near field, and the tables' allocation and copy
  void stats(double* out, int n)
  {
    std::lock_guard<std::mutex> g(mu_);
    const double v[14] = {(double)n_steps_, 1e-3 * t_step_ms_, (double)pool_.rebuilds(), pool_.rebuild_seconds(),
                          (double)n_prepared_, 1e-3 * (t_mesh_ms_ + t_rhs_ms_ + t_pc_ms_), 1e-3 * t_mesh_ms_,
                          1e-3 * t_rhs_ms_, 1e-3 * t_pc_ms_, t_setup_s_[0], t_setup_s_[1], t_setup_s_[2],
                          t_setup_s_[3], t_setup_s_[4]};
    for (int k = 0; k < n && k < 14; k++) out[k] = v[k];
  }

 private:
  int step_impl(int* nactive, int* nwaiting)
  {
    cudaSetDevice(device_);
    // join prepared requests (slots permitting)
    {
      std::unique_lock<std::mutex> g(mu_);
      // while meshes are being prepared, the solver's far field leaves a
      // quarter of the SMs to the preparation kernels (near field, right-hand
      // sides, preconditioner), which would otherwise wait for every step
      pool_.set_reserved_sms(preparing_ > 0 || !to_prepare_.empty() ? reserve_sms_ : 0);
      // nothing to run yet but meshes in preparation: wait (bounded) for the
      // first one instead of returning at once, so callers need not spin
      if (active_.empty() && prepared_.empty() && (preparing_ > 0 || !to_prepare_.empty()))
        ready_cv_.wait_for(g, std::chrono::milliseconds(100), [this] {
          return stop_ || !prepared_.empty() || (preparing_ == 0 && to_prepare_.empty());
        });
      for (auto it = prepared_.begin(); it != prepared_.end();) {
        auto r = *it;
        if (active_systems_ + r->nrhs > max_systems_ && active_systems_ > 0) break;
        r->sys.resize(r->nrhs);
        const int rc = pool_.add(eb_mesh_internal(r->mesh), r->nrhs, r->b.data(), r->sys.data());
        if (rc != EB_OK) {
          r->state = 5;
          r->error = last_error();
        } else {
          r->state = 3;
          r->t_active = now_ms();
          active_systems_ += r->nrhs;
          active_.push_back(r);
        }
        it = prepared_.erase(it);
      }
    }
    int n = 0;
    EB_CHECK(pool_.step(stream_, &n));
    // retire finished requests
    std::vector<std::shared_ptr<Request>> finished;
    for (auto it = active_.begin(); it != active_.end();) {
      auto r = *it;
      bool all = true;
      for (int s : r->sys) all &= pool_.done(s);
      if (!all) {
        ++it;
        continue;
      }
      r->x.resize((size_t)r->nrhs * r->ne);
      r->stats.resize(r->nrhs);
      for (int c = 0; c < r->nrhs; c++) {
        EB_CHECK(pool_.result(r->sys[c], r->x.data() + (size_t)c * r->ne, &r->stats[c]));
        EB_CHECK(pool_.remove(r->sys[c]));
      }
      finished.push_back(r);
      it = active_.erase(it);
    }
    {
      std::lock_guard<std::mutex> g(mu_);
      for (auto& r : finished) {
        r->t_done = now_ms();
        r->state = 4;
        active_systems_ -= r->nrhs;
        // the mesh and its budget share are released at once; results stay on the host
        eb_mesh_destroy(r->mesh);
        r->mesh = nullptr;
        used_ -= r->bytes;
        r->nodes.clear();
        r->elems.clear();
        r->g.clear();
        r->b.clear();
      }
      admit_locked();
      if (nactive) *nactive = (int)active_.size();
      if (nwaiting) *nwaiting = (int)(queue_.size() + preparing_ + prepared_.size());
    }
    cv_.notify_all();
    return EB_OK;
  }

 public:
  int poll(long long id, int* state)
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return set_error(EB_ERR_INVALID, "unknown request");
    *state = it->second->state;
    return EB_OK;
  }

  int result(long long id, double* x, eb_solve_stats* stats, double* times_ms)
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return set_error(EB_ERR_INVALID, "unknown request");
    Request& r = *it->second;
    if (r.state == 5) return set_error(EB_ERR_STATE, "request failed: " + r.error);
    if (r.state != 4) return set_error(EB_ERR_STATE, "request not finished");
    if (x) std::copy(r.x.begin(), r.x.end(), x);
    if (stats)
      for (int c = 0; c < r.nrhs; c++)
        stats[c] = eb_solve_stats{r.stats[c].converged, r.stats[c].cycles, r.stats[c].iterations,
                                  r.stats[c].rel_residual};
    if (times_ms) {  // total latency, queue wait, preparation, solve
      times_ms[0] = r.t_done - r.t_submit;
      times_ms[1] = r.t_admit - r.t_submit;
      times_ms[2] = r.t_active - r.t_admit;
      times_ms[3] = r.t_done - r.t_active;
    }
    return EB_OK;
  }

  int release(long long id)
  {
    std::lock_guard<std::mutex> g(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return set_error(EB_ERR_INVALID, "unknown request");
    if (it->second->state < 4) return set_error(EB_ERR_STATE, "request still running");
    reqs_.erase(it);
    return EB_OK;
  }

  void usage(long long* used, long long* budget)
  {
    std::lock_guard<std::mutex> g(mu_);
    if (used) *used = (long long)used_;
    if (budget) *budget = (long long)budget_;
  }

 private:
  // Moves queued requests to preparation while the budget allows (FIFO).
  void admit_locked()
  {
    while (!queue_.empty() && used_ + queue_.front()->bytes <= budget_) {
      auto r = queue_.front();
      queue_.pop_front();
      used_ += r->bytes;
      r->state = 1;
      r->t_admit = now_ms();
      to_prepare_.push_back(r);
    }
  }

  void prepare_loop()
  {
    cudaSetDevice(device_);
    for (;;) {
      std::shared_ptr<Request> r;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [this] { return stop_ || !to_prepare_.empty(); });
        if (stop_) return;
        r = to_prepare_.front();
        to_prepare_.pop_front();
        preparing_++;
      }
      eb_mesh m = nullptr;
      const double t0 = now_ms();
      int rc = eb_mesh_create(r->nv, r->nodes.data(), r->ne, r->elems.data(), r->order, &m);
      // many meshes share each batched launch: a coarser split per mesh keeps
      // the merged work list (and the partial sums) small while still giving
      // every persistent CTA many items
      if (rc == EB_OK) rc = mesh_set_plan(eb_mesh_internal(m), kServeItemsPerSm, 0);
      const double t1 = now_ms();
      std::vector<double> b;
      if (rc == EB_OK) {
        b.resize((size_t)r->nrhs * r->ne);
        rc = eb_dirichlet_rhs_prec(m, opt_.rhs_precision, r->nrhs, r->g.data(), b.data());
      }
      const double t2 = now_ms();
      if (rc == EB_OK && opt_.precond) rc = ensure_near_precond(eb_mesh_internal(m));
      const double t3 = now_ms();
      std::string err = rc == EB_OK ? "" : last_error();
      std::lock_guard<std::mutex> g(mu_);
      preparing_--;
      n_prepared_++;
      if (m)
        for (int k = 0; k < 5; k++) t_setup_s_[k] += eb_mesh_internal(m)->setup_s[k];
      t_mesh_ms_ += t1 - t0;
      t_rhs_ms_ += t2 - t1;
      t_pc_ms_ += t3 - t2;
      ready_cv_.notify_all();  // under the lock: step() sees the new state once it wakes
      if (rc != EB_OK) {
        if (m) eb_mesh_destroy(m);
        r->state = 5;
        r->error = err;
        used_ -= r->bytes;
        r->t_done = now_ms();
        continue;
      }
      // replace the estimate by the measured footprint
      const size_t actual = mesh_resident_bytes(eb_mesh_internal(m)) +
                            (size_t)r->nrhs * pool_.device_bytes_per_system(eb_mesh_internal(m)) +
                            (sym_eligible(eb_mesh_internal(m), true, kBatchCols, 0)
                                 ? sym_slot_bytes(eb_mesh_internal(m)->h, kBatchCols)
                                 : 0);
      used_ = used_ - r->bytes + actual;
      r->bytes = actual;
      r->mesh = m;
      r->b.swap(b);
      r->state = 2;
      prepared_.push_back(r);
    }
  }

  size_t budget_, used_ = 0;
  int max_systems_;
  SolveOptions opt_;
  SolverPool pool_;
  cudaStream_t stream_ = nullptr;
  int device_ = 0;
  std::mutex mu_;
  std::condition_variable cv_;
  std::condition_variable ready_cv_;  // a prepared (or failed) request is ready for step()
  bool stop_ = false;
  static constexpr int kPrepWorkers = 4;      // host threads preparing meshes (EASYBEM_PREP_WORKERS overrides;
                                              // 4, 8 and 16 served the same 4.0-4.2 requests/s: the GPU is the limit)
  static constexpr int kServeItemsPerSm = 4;  // work split of served meshes (see prepare_loop)
  std::vector<std::thread> workers_;
  int reserve_sms_ = 0;
  long long next_id_ = 1;
  int active_systems_ = 0, preparing_ = 0;
  long long n_steps_ = 0, n_prepared_ = 0;
  double t_step_ms_ = 0, t_mesh_ms_ = 0, t_rhs_ms_ = 0, t_pc_ms_ = 0, t_setup_s_[5] = {0, 0, 0, 0, 0};
  std::map<long long, std::shared_ptr<Request>> reqs_;
  std::deque<std::shared_ptr<Request>> queue_, to_prepare_, prepared_;
  std::vector<std::shared_ptr<Request>> active_;
};

}  // namespace eb

struct eb_server_s {
  std::unique_ptr<eb::Server> srv;
};

using eb::set_error;

extern "C" {

int eb_server_create(long long budget_bytes, int max_systems, const eb_solve_options* opt, eb_server* out)
{
  if (!out || budget_bytes <= 0 || max_systems < 1) return set_error(EB_ERR_INVALID, "bad server arguments");
  eb::SolveOptions o;
  if (opt) {
    o.tol = opt->tol;
    o.inner_tol = opt->inner_tol;
    o.restart = opt->restart;
    o.max_cycles = opt->max_cycles;
    o.max_iterations = opt->max_iterations;
    o.inner_precision = opt->inner_precision;
    o.precond = opt->precond;
    o.rhs_precision = opt->rhs_precision;
  }
  if (o.precond != 0 && o.precond != 1) return set_error(EB_ERR_INVALID, "precond must be 0 or 1");
  if (o.rhs_precision != EB_PREC_FP64 && o.rhs_precision != EB_PREC_MIXED)
    return set_error(EB_ERR_INVALID, "rhs_precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  auto s = new eb_server_s();
  s->srv = std::make_unique<eb::Server>((size_t)budget_bytes, max_systems, o);
  *out = s;
  return EB_OK;
}

int eb_server_destroy(eb_server s)
{
  delete s;
  return EB_OK;
}

int eb_server_submit(eb_server s, int nnodes, const double* nodes, int nelems, const int* elems, int order, int nrhs,
                     const double* g, long long* id)
{
  if (!s || !id) return set_error(EB_ERR_INVALID, "null argument");
  return s->srv->submit(nnodes, nodes, nelems, elems, order, nrhs, g, id);
}

int eb_server_step(eb_server s, int* nactive, int* nwaiting)
{
  if (!s) return set_error(EB_ERR_INVALID, "null server");
  return s->srv->step(nactive, nwaiting);
}

int eb_server_poll(eb_server s, long long id, int* state)
{
  if (!s || !state) return set_error(EB_ERR_INVALID, "null argument");
  return s->srv->poll(id, state);
}

int eb_server_result(eb_server s, long long id, double* t, eb_solve_stats* stats, double* times_ms)
{
  if (!s) return set_error(EB_ERR_INVALID, "null server");
  return s->srv->result(id, t, stats, times_ms);
}

int eb_server_release(eb_server s, long long id)
{
  if (!s) return set_error(EB_ERR_INVALID, "null server");
  return s->srv->release(id);
}

int eb_server_usage(eb_server s, long long* used_bytes, long long* budget_bytes)
{
  if (!s) return set_error(EB_ERR_INVALID, "null server");
  s->srv->usage(used_bytes, budget_bytes);
  return EB_OK;
}

int eb_server_stats(eb_server s, double* stats, int n)
{
  if (!s || !stats || n < 0) return set_error(EB_ERR_INVALID, "null argument");
  s->srv->stats(stats, n);
  return EB_OK;
}

}  // extern "C"
