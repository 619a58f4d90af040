// GMRES with iterative refinement for the P0 single-layer system V x = b,
// many systems at once.
//
// Not in the reference, whose drivers call SciPy's CG with FP32 GPU
// matvecs (python/examples/laplace3dDirichletGPU.py:64-81). Here every
// system runs restarted GMRES(m) whose matvec is the mixed-precision apply
// (FP32 far field, FP64 near field); the Arnoldi basis, classical Gram-Schmidt
// with reorthogonalisation (CGS2) and the solution update are FP64 on the
// device; each restart cycle ends with the true residual b - V x computed
// with the FP64 apply (iterative refinement), and a system stops when
// ||b - V x|| <= tol ||b|| in that FP64 residual.
//
// All active systems advance in lockstep: one step is one batched apply over
// every mesh that has a system in that phase (see batch.h), followed by
// batched Gram-Schmidt kernels and one small device-to-host copy of the
// Hessenberg column; the Givens rotations run on the host. Systems may be
// added and removed between steps (continuous batching); a system's arithmetic
// does not depend on which other systems share its steps.
#pragma once

#include <memory>
#include <vector>

#include "batch.h"

namespace eb {

struct SolveOptions {
  double tol = 1e-8;        // target ||b - V x|| / ||b|| (FP64 residual)
  double inner_tol = 1e-6;  // GMRES cycle stops at this relative reduction
  int restart = 50;         // Krylov dimension m
  int max_cycles = 40;      // refinement cycles per system
  int max_iterations = 4000;
  int inner_precision = EB_PREC_MIXED;
  int precond = 1;          // 1: near-field sparse approximate inverse (right), 0: none
  int rhs_precision = EB_PREC_FP64;  // served right-hand sides (1/2 M + K) g
};

struct SolveStats {
  int converged = 0, cycles = 0, iterations = 0;
  double rel_residual = 0.0;
};

class SolverPool {
 public:
  explicit SolverPool(const SolveOptions& o) : opt_(o) {}
  ~SolverPool();
  // Adds nrhs systems on mesh m with right-hand sides b ([nrhs][nelems],
  // host); ids receives their ids. All meshes of a pool share one order.
  int add(Mesh* m, int nrhs, const double* b_host, int* ids);
  // One lockstep step of every active system; *nactive = systems still running.
  int step(cudaStream_t st, int* nactive);
  bool done(int id) const;
  // Copies the solution of a finished system to x_host ([nelems]).
  int result(int id, double* x_host, SolveStats* stats);
  // Releases a system (finished or not) and its device memory.
  int remove(int id);
  size_t device_bytes_per_system(const Mesh* m) const;
  int active() const;
  // SMs the batched far field leaves free for other streams (0: none).
  void set_reserved_sms(int n) { reserve_sms_ = n; }
  // Batch rebuilds after membership changes: count and host seconds spent.
  long long rebuilds() const { return n_rebuild_; }
  double rebuild_seconds() const { return t_rebuild_; }

 private:
  enum Phase { kRefine = 0, kArnoldi = 1, kDone = 2 };
  struct Sys {
    int id = -1;
    BatchEntry* entry = nullptr;
    int col = 0, ne = 0;
    DevBuf basis, x, b, r;
    int phase = kRefine;
    bool fresh = true;
    int k = 0, cycles = 0, iterations = 0;
    double bnorm = 0.0, beta = 0.0, rel = 1.0;
    bool converged = false;
    std::vector<double> H, cs, sn, g;
  };
  struct SysDev {
    int ne;
    double *basis, *x, *b, *r, *tin, *vout;
    const int *prow, *pcol;  // right preconditioner M on the near-field pattern (null: none)
    const double* pval;
  };
  int rebuild();
  int upload_control(cudaStream_t st);

  SolveOptions opt_;
  std::vector<std::unique_ptr<Sys>> sys_;  // index = slot
  std::vector<std::unique_ptr<BatchEntry>> entries_;
  Batch batch_inner_, batch_fp64_;
  bool dirty_ = true;
  int next_id_ = 0;
  // device control / reduction buffers
  DevBuf d_tab_, d_phase_, d_k_, d_fresh_, d_flag_start_, d_flag_x_, d_y_, d_h1_, d_h2_, d_wn_, d_rn_;
  DevBuf d_eflag_inner_, d_eflag_fp64_;
  std::vector<double> h1_, h2_, wn_, rn_;
  std::vector<int> phase_, k_, fresh_, fstart_, fx_;
  int reserve_sms_ = 0;
  long long n_rebuild_ = 0;
  double t_rebuild_ = 0.0;
};

}  // namespace eb
