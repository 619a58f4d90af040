// Batched apply: the far field of many meshes and right-hand sides in one
// persistent launch.
//
// Not in the reference, whose GPU path holds a single process-global mesh
// (src/meshTopology.cpp:11-19). An entry is one mesh with up to kBatchCols
// SL right-hand sides (and optionally one DL density); it owns its apply
// scratch and its input/output columns. A Batch merges the work items of all
// entries (largest first, pulled dynamically by the persistent CTAs), so one
// apply over any number of uneven meshes is four launches: batched record
// preparation, a counter reset, the far-field kernel and a batched finalize
// (near field included). Entries can be switched off per apply through a
// device flag without rebuilding the batch, and a built batch can be
// captured once into a CUDA graph and replayed.
#pragma once

#include <memory>
#include <vector>

#include "engine.h"

namespace eb {

constexpr int kBatchCols = 4;  // SL right-hand sides per entry (the NSL = 4 far-field variant)

struct BatchEntry {
  Mesh* mesh = nullptr;
  DevBuf rec, partial;  // apply scratch
  DevBuf tin, vout;     // kBatchCols columns of nelems each (inputs / outputs)
  DevBuf uin, qout;     // DL density [nnodes] and DL output [nelems] (batches with a DL column)
  DevBuf tc_be, tc_charge;  // tensor-core DL operand and charges (tensor-core SL+DL batches)
  DevBuf sym_partial;       // symmetric batches: partial slots (one per tile, row and output)
  int index = -1;       // position in the current batch
};

class Batch {
 public:
  // Builds the launch tables for `entries` (all meshes must share the
  // quadrature order). fp32 selects the mixed-precision far field.
  // nsl: right-hand sides computed per entry (1, 3 or 4; columns beyond an
  // entry's systems carry zeros). nd = 1 adds the double layer (uin -> qout)
  // in the same pass, with nsl 0 or 1 (the fused SL+DL variant). sym_fp64:
  // an FP64 batch inside the library (the solver's residuals) that takes the
  // symmetric kernels when the meshes' engine is the default.
  int build(const std::vector<BatchEntry*>& entries, bool fp32, int nsl, int* d_flags, int nd = 0,
            bool sym_fp64 = false);
  // One apply of all entries whose flag is set (inputs tin, outputs vout).
  // reserve_sms > 0 sizes the persistent far-field grid to leave that many
  // SMs free for kernels of other streams (the far kernel holds every SM it
  // starts on until the whole apply is done).
  int run(cudaStream_t st, int reserve_sms = 0);
  // Captures run() into a CUDA graph on first use (one graph per grid size)
  // and replays it afterwards.
  int run_graph(cudaStream_t st, int reserve_sms = 0);
  void reset_graph();
  ~Batch() { reset_graph(); }

  int nentries() const { return (int)entries_.size(); }
  bool tensor_cores() const { return tc_; }
  bool symmetric() const { return sym_; }
  // EB_ERR_TIMEOUT (flag cleared) if the last tensor-core launch gave up a
  // bounded wait; the batch's stream must be synchronised.
  int check_error();
  long long quad_pairs() const { return quad_pairs_; }

 private:
  std::vector<BatchEntry*> entries_;
  bool fp32_ = true;
  int nsl_ = kBatchCols;
  int nd_ = 0;
  DevBuf desc_, items_, args_, prep_off_, fin_off_, counter_;
  bool tc_ = false;  // far field on the tensor cores (fused FP32 SL+DL, 7-point rule, engine 1 on every mesh)
  DevBuf tc_args_, tc_off_, tc_err_;
  bool sym_ = false;  // symmetric far field (fused FP32 SL+DL, 7-point rule, engine 2 on every mesh)
  int tc_blocks_ = 0;
  int nitems_ = 0, grid_ = 0, occ_ = 1, nsm_ = 148, prep_blocks_ = 0, fin_blocks_ = 0, K_ = 0, Q_ = 0;
  size_t smem_ = 0;
  long long quad_pairs_ = 0;
  // graphs of the full grid [0] and of the reduced grid [1] (reserve_ SMs left free)
  cudaGraph_t graph_[2] = {nullptr, nullptr};
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
  int reserve_ = 0;
};

// Far-field variant width (SL charges) for entries using up to `cols` columns.
int batch_width(int cols);
// Allocates an entry's scratch and columns for mesh m (with_dl: also the DL
// density and output).
int batch_entry_init(BatchEntry* e, Mesh* m, bool with_dl = false);

}  // namespace eb
