#include "solver.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

namespace eb {

namespace {

constexpr int kRed = 256;  // threads per reduction block

// Deterministic block reduction (fixed tree) of one value per thread.
__device__ double block_sum(double v)
{
  __shared__ double red[kRed];
  red[threadIdx.x] = v;
  __syncthreads();
  for (int w = kRed / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  const double r = red[0];
  __syncthreads();
  return r;
}

struct SysDevK {
  int ne;
  double *basis, *x, *b, *r, *tin, *vout;
  const int *prow, *pcol;
  const double* pval;
};

// y_i = (M v)_i for one row with the near-field-pattern preconditioner
__device__ __forceinline__ double precond_row(const SysDevK& t, const double* v, int i)
{
  double acc = 0.0;
  for (int p = t.prow[i]; p < t.prow[i + 1]; ++p) acc += t.pval[p] * v[t.pcol[p]];
  return acc;
}

// apply input: the refinement residual uses x; an Arnoldi step uses M v_k
// (right preconditioning: GMRES runs on V M, and x = M y)
__global__ void k_load(const SysDevK* T, const int* phase, const int* kk, int want, int from_basis)
{
  const int s = blockIdx.y;
  if (phase[s] != want) return;
  const SysDevK t = T[s];
  const double* src = from_basis ? t.basis + (size_t)kk[s] * t.ne : t.x;
  const bool pc = from_basis && t.pval;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x)
    t.tin[i] = pc ? precond_row(t, src, i) : src[i];
}

__global__ void k_residual(const SysDevK* T, const int* phase, const int* fresh, int want)
{
  const int s = blockIdx.y;
  if (phase[s] != want) return;
  const SysDevK t = T[s];
  const bool f = fresh[s] != 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x)
    t.r[i] = f ? t.b[i] : t.b[i] - t.vout[i];
}

// out[s] = ||vec_s|| with vec = r (which = 0) or the apply output (which = 1)
__global__ void k_norm(const SysDevK* T, const int* phase, int want, int which, double* out)
{
  const int s = blockIdx.x;
  if (phase[s] != want) return;
  const SysDevK t = T[s];
  const double* v = which == 0 ? t.r : t.vout;
  double acc = 0.0;
  for (int i = threadIdx.x; i < t.ne; i += blockDim.x) acc += v[i] * v[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) out[s] = sqrt(acc);
}

// h[s][j] = <basis_j, w> for j <= k[s]
__global__ void k_dots(const SysDevK* T, const int* phase, const int* kk, int m, int want, double* h)
{
  const int s = blockIdx.y, j = blockIdx.x;
  if (phase[s] != want || j > kk[s]) return;
  const SysDevK t = T[s];
  const double* bj = t.basis + (size_t)j * t.ne;
  double acc = 0.0;
  for (int i = threadIdx.x; i < t.ne; i += blockDim.x) acc += bj[i] * t.vout[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) h[(size_t)s * (m + 1) + j] = acc;
}

// w -= sum_{j <= k} h_j basis_j
__global__ void k_update(const SysDevK* T, const int* phase, const int* kk, int m, int want, const double* h)
{
  const int s = blockIdx.y;
  if (phase[s] != want) return;
  const SysDevK t = T[s];
  const int k = kk[s];
  const double* hs = h + (size_t)s * (m + 1);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x) {
    double w = t.vout[i];
    for (int j = 0; j <= k; j++) w -= hs[j] * t.basis[(size_t)j * t.ne + i];
    t.vout[i] = w;
  }
}

__global__ void k_normalize(const SysDevK* T, const int* phase, const int* kk, int m, int want, const double* wn)
{
  const int s = blockIdx.y;
  if (phase[s] != want || kk[s] + 1 > m || !(wn[s] > 0.0)) return;
  const SysDevK t = T[s];
  const double inv = 1.0 / wn[s];
  double* dst = t.basis + (size_t)(kk[s] + 1) * t.ne;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x) dst[i] = t.vout[i] * inv;
}

__global__ void k_start(const SysDevK* T, const int* flag, const double* rn)
{
  const int s = blockIdx.y;
  if (!flag[s]) return;
  const SysDevK t = T[s];
  const double inv = 1.0 / rn[s];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x)
    t.basis[i] = t.r[i] * inv;
}

// x += sum_j y_j v_j, or with the preconditioner z = sum_j y_j v_j (into r,
// free until the next refinement residual) and then x += M z (k_xprecond)
__global__ void k_xupdate(const SysDevK* T, const int* flag, int m, const double* y)
{
  const int s = blockIdx.y;
  const int nk = flag[s];
  if (nk <= 0) return;
  const SysDevK t = T[s];
  const double* ys = y + (size_t)s * m;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int j = 0; j < nk; j++) acc += ys[j] * t.basis[(size_t)j * t.ne + i];
    if (t.pval) t.r[i] = acc;
    else t.x[i] += acc;
  }
}

__global__ void k_xprecond(const SysDevK* T, const int* flag)
{
  const int s = blockIdx.y;
  if (flag[s] <= 0) return;
  const SysDevK t = T[s];
  if (!t.pval) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < t.ne; i += gridDim.x * blockDim.x)
    t.x[i] += precond_row(t, t.r, i);
}

}  // namespace

SolverPool::~SolverPool() = default;

size_t SolverPool::device_bytes_per_system(const Mesh* m) const
{
  return sizeof(double) * (size_t)m->h.ne * (opt_.restart + 1 + 3);
}

int SolverPool::add(Mesh* m, int nrhs, const double* b_host, int* ids)
{
  if (nrhs < 1 || !b_host) return set_error(EB_ERR_INVALID, "need >= 1 right-hand side");
  for (const auto& s : sys_)
    if (s->entry->mesh->h.Q != m->h.Q)
      return set_error(EB_ERR_INVALID, "all meshes of a solve need the same quadrature order");
  if (opt_.precond) EB_CHECK(ensure_near_precond(m));
  const int ne = m->h.ne;
  for (int c0 = 0; c0 < nrhs; c0 += kBatchCols) {
    auto e = std::make_unique<BatchEntry>();
    EB_CHECK(batch_entry_init(e.get(), m));
    for (int c = c0; c < std::min(nrhs, c0 + kBatchCols); c++) {
      auto s = std::make_unique<Sys>();
      s->id = next_id_++;
      s->entry = e.get();
      s->col = c - c0;
      s->ne = ne;
      EB_CHECK(s->basis.alloc(sizeof(double) * (size_t)ne * (opt_.restart + 1)));
      EB_CHECK(s->x.alloc(sizeof(double) * ne));
      EB_CHECK(s->b.alloc(sizeof(double) * ne));
      EB_CHECK(s->r.alloc(sizeof(double) * ne));
      EB_CHECK(memset_sync(s->x.p, 0, sizeof(double) * ne));
      const double* bc = b_host + (size_t)c * ne;
      EB_CHECK(copy_h2d(s->b.p, bc, sizeof(double) * ne));
      double bn = 0.0;
      for (int i = 0; i < ne; i++) bn += bc[i] * bc[i];
      s->bnorm = std::sqrt(bn);
      const int m1 = opt_.restart + 1;
      s->H.assign((size_t)m1 * opt_.restart, 0.0);
      s->cs.assign(opt_.restart, 0.0);
      s->sn.assign(opt_.restart, 0.0);
      s->g.assign(m1, 0.0);
      if (s->bnorm == 0.0) {  // x = 0 solves it
        s->phase = kDone;
        s->converged = true;
        s->rel = 0.0;
      }
      if (ids) ids[c] = s->id;
      sys_.push_back(std::move(s));
    }
    entries_.push_back(std::move(e));
  }
  dirty_ = true;
  return EB_OK;
}

int SolverPool::rebuild()
{
  std::vector<BatchEntry*> ents;
  for (auto& e : entries_) ents.push_back(e.get());
  const int S = (int)sys_.size(), E = (int)ents.size(), m = opt_.restart;
  EB_CHECK(d_eflag_inner_.alloc(sizeof(int) * std::max(E, 1)));
  EB_CHECK(d_eflag_fp64_.alloc(sizeof(int) * std::max(E, 1)));
  int cols = 1;
  for (auto& s : sys_) cols = std::max(cols, s->col + 1);
  EB_CHECK(batch_inner_.build(ents, opt_.inner_precision == EB_PREC_MIXED, cols, d_eflag_inner_.as<int>()));
  // the FP64 residuals take the symmetric kernel on the default engine too
  EB_CHECK(batch_fp64_.build(ents, false, cols, d_eflag_fp64_.as<int>(), 0, true));
  std::vector<SysDev> tab(S);
  for (int s = 0; s < S; s++) {
    Sys& y = *sys_[s];
    const Mesh* mm = y.entry->mesh;
    const bool pc = opt_.precond && mm->pc_val.p;
    tab[s] = SysDev{y.ne, y.basis.as<double>(), y.x.as<double>(), y.b.as<double>(), y.r.as<double>(),
                    y.entry->tin.as<double>() + (size_t)y.col * y.ne, y.entry->vout.as<double>() + (size_t)y.col * y.ne,
                    pc ? mm->sl_rowptr.as<int>() : nullptr, pc ? mm->sl_col.as<int>() : nullptr,
                    pc ? mm->pc_val.as<double>() : nullptr};
  }
  const size_t n1 = std::max(S, 1);
  EB_CHECK(d_tab_.alloc(sizeof(SysDev) * n1));
  if (S) EB_CHECK(copy_h2d(d_tab_.p, tab.data(), sizeof(SysDev) * S));
  EB_CHECK(d_phase_.alloc(sizeof(int) * n1));
  EB_CHECK(d_k_.alloc(sizeof(int) * n1));
  EB_CHECK(d_fresh_.alloc(sizeof(int) * n1));
  EB_CHECK(d_flag_start_.alloc(sizeof(int) * n1));
  EB_CHECK(d_flag_x_.alloc(sizeof(int) * n1));
  EB_CHECK(d_y_.alloc(sizeof(double) * n1 * m));
  EB_CHECK(d_h1_.alloc(sizeof(double) * n1 * (m + 1)));
  EB_CHECK(d_h2_.alloc(sizeof(double) * n1 * (m + 1)));
  EB_CHECK(d_wn_.alloc(sizeof(double) * n1));
  EB_CHECK(d_rn_.alloc(sizeof(double) * n1));
  h1_.assign(n1 * (m + 1), 0.0);
  h2_.assign(n1 * (m + 1), 0.0);
  wn_.assign(n1, 0.0);
  rn_.assign(n1, 0.0);
  phase_.assign(n1, kDone);
  k_.assign(n1, 0);
  fresh_.assign(n1, 0);
  fstart_.assign(n1, 0);
  fx_.assign(n1, 0);
  dirty_ = false;
  return EB_OK;
}

int SolverPool::active() const
{
  int n = 0;
  for (const auto& s : sys_) n += s->phase != kDone;
  return n;
}

bool SolverPool::done(int id) const
{
  for (const auto& s : sys_)
    if (s->id == id) return s->phase == kDone;
  return true;
}

int SolverPool::step(cudaStream_t st, int* nactive)
{
  if (dirty_) {
    const auto t0 = std::chrono::steady_clock::now();
    EB_CHECK(rebuild());
    n_rebuild_++;
    t_rebuild_ += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  const int S = (int)sys_.size(), m = opt_.restart;
  const int E = (int)entries_.size();
  if (S == 0 || active() == 0) {
    if (nactive) *nactive = 0;
    return EB_OK;
  }
  std::vector<int> ef_in(E, 0), ef_64(E, 0);
  bool any_ref = false, any_arn = false, any_apply64 = false;
  int maxne = 1;
  for (int s = 0; s < S; s++) {
    const Sys& y = *sys_[s];
    phase_[s] = y.phase;
    k_[s] = y.k;
    fresh_[s] = y.fresh ? 1 : 0;
    maxne = std::max(maxne, y.ne);
    if (y.phase == kRefine) {
      any_ref = true;
      if (!y.fresh) {
        ef_64[y.entry->index] = 1;
        any_apply64 = true;
      }
    } else if (y.phase == kArnoldi) {
      any_arn = true;
      ef_in[y.entry->index] = 1;
    }
  }
  EB_CUDA(cudaMemcpyAsync(d_phase_.p, phase_.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(d_k_.p, k_.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(d_fresh_.p, fresh_.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(d_eflag_inner_.p, ef_in.data(), sizeof(int) * E, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(d_eflag_fp64_.p, ef_64.data(), sizeof(int) * E, cudaMemcpyHostToDevice, st));
  const SysDevK* T = d_tab_.as<SysDevK>();
  const dim3 eg((maxne + 255) / 256, S);
  if (any_ref) {
    if (any_apply64) {
      k_load<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), kRefine, 0);
      EB_CHECK(batch_fp64_.run_graph(st, reserve_sms_));
    }
    k_residual<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_fresh_.as<int>(), kRefine);
    k_norm<<<S, kRed, 0, st>>>(T, d_phase_.as<int>(), kRefine, 0, d_rn_.as<double>());
  }
  if (any_arn) {
    k_load<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), kArnoldi, 1);
    EB_CHECK(batch_inner_.run_graph(st, reserve_sms_));
    const dim3 dg(m + 1, S);
    k_dots<<<dg, kRed, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), m, kArnoldi, d_h1_.as<double>());
    k_update<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), m, kArnoldi, d_h1_.as<double>());
    k_dots<<<dg, kRed, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), m, kArnoldi, d_h2_.as<double>());
    k_update<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), m, kArnoldi, d_h2_.as<double>());
    k_norm<<<S, kRed, 0, st>>>(T, d_phase_.as<int>(), kArnoldi, 1, d_wn_.as<double>());
    k_normalize<<<eg, 256, 0, st>>>(T, d_phase_.as<int>(), d_k_.as<int>(), m, kArnoldi, d_wn_.as<double>());
  }
  EB_CUDA(cudaGetLastError());
  if (any_ref) EB_CUDA(cudaMemcpyAsync(rn_.data(), d_rn_.p, sizeof(double) * S, cudaMemcpyDeviceToHost, st));
  if (any_arn) {
    EB_CUDA(cudaMemcpyAsync(h1_.data(), d_h1_.p, sizeof(double) * S * (m + 1), cudaMemcpyDeviceToHost, st));
    EB_CUDA(cudaMemcpyAsync(h2_.data(), d_h2_.p, sizeof(double) * S * (m + 1), cudaMemcpyDeviceToHost, st));
    EB_CUDA(cudaMemcpyAsync(wn_.data(), d_wn_.p, sizeof(double) * S, cudaMemcpyDeviceToHost, st));
  }
  EB_CUDA(cudaStreamSynchronize(st));

  // host: refinement decisions and Givens updates
  std::vector<double> y((size_t)S * m, 0.0);
  bool any_start = false, any_x = false;
  for (int s = 0; s < S; s++) {
    Sys& q = *sys_[s];
    fstart_[s] = 0;
    fx_[s] = 0;
    if (q.phase == kRefine) {
      q.fresh = false;
      q.rel = q.bnorm > 0 ? rn_[s] / q.bnorm : 0.0;
      if (q.rel <= opt_.tol) {
        q.phase = kDone;
        q.converged = true;
      } else if (q.cycles >= opt_.max_cycles || q.iterations >= opt_.max_iterations || !(rn_[s] > 0)) {
        q.phase = kDone;
      } else {
        q.beta = rn_[s];
        std::fill(q.g.begin(), q.g.end(), 0.0);
        q.g[0] = q.beta;
        q.k = 0;
        q.phase = kArnoldi;
        fstart_[s] = 1;
        any_start = true;
      }
    } else if (q.phase == kArnoldi) {
      const int k = q.k;
      std::vector<double> h(k + 2);
      for (int j = 0; j <= k; j++) h[j] = h1_[(size_t)s * (m + 1) + j] + h2_[(size_t)s * (m + 1) + j];
      h[k + 1] = wn_[s];
      for (int i = 0; i < k; i++) {  // previous rotations
        const double a = h[i], b = h[i + 1];
        h[i] = q.cs[i] * a + q.sn[i] * b;
        h[i + 1] = -q.sn[i] * a + q.cs[i] * b;
      }
      const double rr = std::hypot(h[k], h[k + 1]);
      const double c = rr > 0 ? h[k] / rr : 1.0, sn = rr > 0 ? h[k + 1] / rr : 0.0;
      q.cs[k] = c;
      q.sn[k] = sn;
      h[k] = rr;
      q.g[k + 1] = -sn * q.g[k];
      q.g[k] = c * q.g[k];
      for (int j = 0; j <= k; j++) q.H[(size_t)j * m + k] = h[j];
      q.k = k + 1;
      q.iterations++;
      // a cycle stops at the inner reduction, or as soon as its estimate
      // already meets the outer target (the next FP64 residual decides)
      const double stop = std::max(opt_.inner_tol * q.beta, 0.5 * opt_.tol * q.bnorm);
      const bool inner_done = std::fabs(q.g[q.k]) <= stop || q.k == m || !(wn_[s] > 0) ||
                              q.iterations >= opt_.max_iterations;
      if (inner_done) {
        // back substitution H(0:k,0:k) y = g(0:k)
        const int n = q.k;
        for (int i = n - 1; i >= 0; i--) {
          double acc = q.g[i];
          for (int j = i + 1; j < n; j++) acc -= q.H[(size_t)i * m + j] * y[(size_t)s * m + j];
          y[(size_t)s * m + i] = q.H[(size_t)i * m + i] != 0.0 ? acc / q.H[(size_t)i * m + i] : 0.0;
        }
        fx_[s] = n;
        any_x = true;
        q.cycles++;
        q.phase = kRefine;
      }
    }
  }
  if (any_x) {
    EB_CUDA(cudaMemcpyAsync(d_y_.p, y.data(), sizeof(double) * S * m, cudaMemcpyHostToDevice, st));
    EB_CUDA(cudaMemcpyAsync(d_flag_x_.p, fx_.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st));
    k_xupdate<<<eg, 256, 0, st>>>(T, d_flag_x_.as<int>(), m, d_y_.as<double>());
    if (opt_.precond) k_xprecond<<<eg, 256, 0, st>>>(T, d_flag_x_.as<int>());
  }
  if (any_start) {
    EB_CUDA(cudaMemcpyAsync(d_flag_start_.p, fstart_.data(), sizeof(int) * S, cudaMemcpyHostToDevice, st));
    k_start<<<eg, 256, 0, st>>>(T, d_flag_start_.as<int>(), d_rn_.as<double>());
  }
  EB_CUDA(cudaGetLastError());
  EB_CUDA(cudaStreamSynchronize(st));
  if (nactive) *nactive = active();
  return EB_OK;
}

int SolverPool::result(int id, double* x_host, SolveStats* stats)
{
  for (auto& s : sys_)
    if (s->id == id) {
      if (x_host) EB_CHECK(copy_d2h(x_host, s->x.p, sizeof(double) * s->ne));
      if (stats) {
        stats->converged = s->converged ? 1 : 0;
        stats->cycles = s->cycles;
        stats->iterations = s->iterations;
        stats->rel_residual = s->rel;
      }
      return EB_OK;
    }
  return set_error(EB_ERR_INVALID, "unknown system id " + std::to_string(id));
}

int SolverPool::remove(int id)
{
  for (size_t k = 0; k < sys_.size(); k++)
    if (sys_[k]->id == id) {
      BatchEntry* e = sys_[k]->entry;
      sys_.erase(sys_.begin() + k);
      bool used = false;
      for (auto& s : sys_) used |= s->entry == e;
      if (!used)
        for (size_t j = 0; j < entries_.size(); j++)
          if (entries_[j].get() == e) {
            entries_.erase(entries_.begin() + j);
            break;
          }
      dirty_ = true;
      return EB_OK;
    }
  return set_error(EB_ERR_INVALID, "unknown system id " + std::to_string(id));
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI

eb::Mesh* eb_mesh_internal(eb_mesh handle);

struct eb_solver_s {
  std::unique_ptr<eb::SolverPool> pool;
  cudaStream_t stream = nullptr;
  std::mutex lock;
};

using eb::set_error;

static eb::SolveOptions to_options(const eb_solve_options* o)
{
  eb::SolveOptions r;
  if (o) {
    r.tol = o->tol;
    r.inner_tol = o->inner_tol;
    r.restart = o->restart;
    r.max_cycles = o->max_cycles;
    r.max_iterations = o->max_iterations;
    r.inner_precision = o->inner_precision;
    r.precond = o->precond;
    r.rhs_precision = o->rhs_precision;
  }
  return r;
}

extern "C" {

void eb_solve_options_default(eb_solve_options* o)
{
  if (!o) return;
  const eb::SolveOptions d;
  o->tol = d.tol;
  o->inner_tol = d.inner_tol;
  o->restart = d.restart;
  o->max_cycles = d.max_cycles;
  o->max_iterations = d.max_iterations;
  o->inner_precision = d.inner_precision;
  o->precond = d.precond;
  o->rhs_precision = d.rhs_precision;
}

int eb_solver_create(const eb_solve_options* opt, eb_solver* out)
{
  if (!out) return set_error(EB_ERR_INVALID, "null output handle");
  const eb::SolveOptions o = to_options(opt);
  if (o.restart < 1 || o.restart > 1000 || !(o.tol > 0) || !(o.inner_tol > 0))
    return set_error(EB_ERR_INVALID, "invalid solve options");
  if (o.inner_precision != EB_PREC_FP64 && o.inner_precision != EB_PREC_MIXED)
    return set_error(EB_ERR_INVALID, "inner precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  if (o.precond != 0 && o.precond != 1) return set_error(EB_ERR_INVALID, "precond must be 0 or 1");
  auto s = new eb_solver_s();
  s->pool = std::make_unique<eb::SolverPool>(o);
  cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete s;
    return set_error(EB_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  *out = s;
  return EB_OK;
}

int eb_solver_destroy(eb_solver s)
{
  if (!s) return EB_OK;
  cudaStreamSynchronize(s->stream);
  s->pool.reset();
  cudaStreamDestroy(s->stream);
  delete s;
  return EB_OK;
}

int eb_solver_add(eb_solver s, eb_mesh mesh, int nrhs, const double* b, int* ids)
{
  if (!s || !mesh) return set_error(EB_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> g(s->lock);
  return s->pool->add(eb_mesh_internal(mesh), nrhs, b, ids);
}

int eb_solver_step(eb_solver s, int* nactive)
{
  if (!s) return set_error(EB_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> g(s->lock);
  return s->pool->step(s->stream, nactive);
}

int eb_solver_done(eb_solver s, int id, int* done)
{
  if (!s || !done) return set_error(EB_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(s->lock);
  *done = s->pool->done(id) ? 1 : 0;
  return EB_OK;
}

int eb_solver_result(eb_solver s, int id, double* x, eb_solve_stats* stats)
{
  if (!s) return set_error(EB_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> g(s->lock);
  eb::SolveStats st;
  EB_CHECK(s->pool->result(id, x, &st));
  if (stats) {
    stats->converged = st.converged;
    stats->cycles = st.cycles;
    stats->iterations = st.iterations;
    stats->rel_residual = st.rel_residual;
  }
  return EB_OK;
}

int eb_solver_remove(eb_solver s, int id)
{
  if (!s) return set_error(EB_ERR_INVALID, "null handle");
  std::lock_guard<std::mutex> g(s->lock);
  return s->pool->remove(id);
}

int eb_solver_bytes_per_system(eb_solver s, eb_mesh mesh, long long* bytes)
{
  if (!s || !mesh || !bytes) return set_error(EB_ERR_INVALID, "null argument");
  *bytes = (long long)s->pool->device_bytes_per_system(eb_mesh_internal(mesh));
  return EB_OK;
}

int eb_solve_sl(int nmesh, const eb_mesh* meshes, const int* nrhs, const double* const* b, double* const* x,
                const eb_solve_options* opt, eb_solve_stats* stats)
{
  if (nmesh < 1 || !meshes || !nrhs || !b || !x) return set_error(EB_ERR_INVALID, "null argument");
  eb_solver s = nullptr;
  EB_CHECK(eb_solver_create(opt, &s));
  std::vector<std::vector<int>> ids(nmesh);
  int rc = EB_OK;
  for (int i = 0; i < nmesh && rc == EB_OK; i++) {
    ids[i].resize(nrhs[i]);
    rc = eb_solver_add(s, meshes[i], nrhs[i], b[i], ids[i].data());
  }
  int nactive = 1;
  while (rc == EB_OK && nactive > 0) rc = eb_solver_step(s, &nactive);
  bool all_conv = true;
  int k = 0;
  for (int i = 0; i < nmesh && rc == EB_OK; i++) {
    const int ne = eb_mesh_internal(meshes[i])->h.ne;
    for (int c = 0; c < nrhs[i] && rc == EB_OK; c++, k++) {
      eb_solve_stats st;
      rc = eb_solver_result(s, ids[i][c], x[i] + (size_t)c * ne, &st);
      if (stats) stats[k] = st;
      all_conv &= st.converged != 0;
    }
  }
  eb_solver_destroy(s);
  if (rc != EB_OK) return rc;
  return all_conv ? EB_OK : set_error(EB_ERR_NOT_CONVERGED, "a system stopped before reaching the tolerance");
}

}  // extern "C"
