#include "batch.h"
#include "farfield_sym.h"
#include "farfield_tc.h"

#include <algorithm>
#include <numeric>
#include <string>

namespace eb {

int batch_entry_init(BatchEntry* e, Mesh* m, bool with_dl)
{
  const HostMesh& h = m->h;
  e->mesh = m;
  // record slots of the widest variant used: 4 SL charges, or SL + DL
  static_assert(rec_slots(kBatchCols, 0) >= rec_slots(1, 1), "entry scratch sized for the SL+DL records");
  EB_CHECK(e->rec.alloc((size_t)h.ne * h.Q * rec_slots(kBatchCols, 0) * sizeof(dq)));
  EB_CHECK(e->partial.alloc(sizeof(double) * (size_t)kBatchCols * m->plan.nsplit * h.nitems));
  EB_CHECK(e->tin.alloc(sizeof(double) * (size_t)kBatchCols * h.ne));
  EB_CHECK(e->vout.alloc(sizeof(double) * (size_t)kBatchCols * h.ne));
  EB_CHECK(memset_sync(e->tin.p, 0, e->tin.bytes));
  if (with_dl) {
    EB_CHECK(e->uin.alloc(sizeof(double) * (size_t)h.nv));
    EB_CHECK(e->qout.alloc(sizeof(double) * (size_t)h.ne));
    EB_CHECK(memset_sync(e->uin.p, 0, e->uin.bytes));
  }
  return EB_OK;
}

void Batch::reset_graph()
{
  for (int k = 0; k < 2; k++) {
    if (exec_[k]) cudaGraphExecDestroy(exec_[k]);
    if (graph_[k]) cudaGraphDestroy(graph_[k]);
    exec_[k] = nullptr;
    graph_[k] = nullptr;
  }
  reserve_ = 0;
}

int batch_width(int cols) { return cols <= 1 ? 1 : (cols <= 3 ? 3 : 4); }

int Batch::build(const std::vector<BatchEntry*>& entries, bool fp32, int nsl, int* d_flags, int nd, bool sym_fp64)
{
  reset_graph();
  entries_ = entries;
  fp32_ = fp32;
  if (nd < 0 || nd > 1 || (nd == 1 && nsl > 1)) return set_error(EB_ERR_INVALID, "a DL batch takes 0 or 1 SL column");
  nd_ = nd;
  nsl_ = nd ? nsl : batch_width(nsl);
  nitems_ = grid_ = prep_blocks_ = fin_blocks_ = 0;
  quad_pairs_ = 0;
  if (entries.empty()) return EB_OK;
  Q_ = entries[0]->mesh->h.Q;
  K_ = entries[0]->mesh->h.K;
  const int n = (int)entries.size();
  tc_ = fp32 && nsl_ == 1 && nd_ == 1;
  for (BatchEntry* be : entries) tc_ = tc_ && tc_eligible(be->mesh, fp32, 1, 1);
  sym_ = !tc_;
  for (BatchEntry* be : entries) sym_ = sym_ && sym_eligible(be->mesh, fp32, nsl_, nd_, sym_fp64);
  std::vector<TcPrepArgs> targs;
  std::vector<int> toff(1, 0);
  std::vector<FarMeshDesc> desc(n);
  std::vector<ApplyArgs> args(n);
  std::vector<int> poff(n + 1, 0), foff(n + 1, 0);
  std::vector<std::pair<long long, WorkItem>> items;
  int src_tile = kTS;
  for (int e = 0; e < n; e++) {
    BatchEntry* be = entries[e];
    be->index = e;
    Mesh* m = be->mesh;
    const HostMesh& h = m->h;
    if (h.Q != Q_) return set_error(EB_ERR_INVALID, "a batch needs one quadrature order for all meshes");
    // the mesh's plan may have changed (finer work split) since the entry was made
    EB_CHECK(be->partial.alloc(sizeof(double) * (size_t)kBatchCols * m->plan.nsplit * h.nitems));
    if (nd_ && !be->uin.p) return set_error(EB_ERR_INVALID, "batch entry without DL columns");
    desc[e] = mesh_far_desc(m, fp32, nsl_, nd_, be->rec.p, be->partial.as<double>());
    desc[e].active = d_flags ? d_flags + e : nullptr;
    if (tc_) {
      EB_CHECK(ensure_tc_static(m));
      EB_CHECK(be->tc_be.alloc(far_tc_operand_bytes(h.ncells)));
      EB_CHECK(be->tc_charge.alloc(far_tc_charge_bytes(h.ncells)));
      desc[e].tc_bd2 = m->tc_bd2.as<float4>();
      desc[e].tc_be = be->tc_be.as<float4>();
      desc[e].tc_charge = be->tc_charge.as<float>();
      targs.push_back(TcPrepArgs{h.ne, h.ncells, be->rec.as<float4>(), m->splane32.as<float4>(),
                                 be->tc_be.as<float4>(), be->tc_charge.as<float>(), desc[e].active});
      toff.push_back(toff.back() + far_tc_prep_blocks(h.ncells));
    }
    std::vector<WorkItem> sym_items;
    int sym_nsplit = 0;
    if (sym_) {  // the mesh's symmetric work list and its own zeroed partial slots
      sym_nsplit = far_sym_items(h.nitems, h.ncells, kSymBatchCellsPerItem, sym_items);
      const size_t bytes = sizeof(double) * (size_t)(nsl_ + nd_) * (size_t)sym_nsplit * h.nitems;
      if (be->sym_partial.bytes < bytes) {  // no zeroing: the finalize reads only written slots
        be->sym_partial.release();
        EB_CHECK(be->sym_partial.alloc(bytes));
      }
      desc[e].partial = be->sym_partial.as<double>();
      desc[e].nsplit = sym_nsplit;
      desc[e].src_tile = kTS;
    }
    src_tile = std::min(src_tile, desc[e].src_tile);
    args[e] = mesh_apply_args(m, fp32, be->rec.p, be->partial.as<double>(), nsl_ ? be->tin.as<double>() : nullptr,
                              h.ne, nd_ ? be->uin.as<double>() : nullptr, nsl_ ? be->vout.as<double>() : nullptr,
                              h.ne, nd_ ? be->qout.as<double>() : nullptr);
    args[e].active = d_flags ? d_flags + e : nullptr;
    if (sym_) {
      args[e].partial = be->sym_partial.as<double>();
      args[e].nsplit = sym_nsplit;
      args[e].sym_cells = far_sym_cells_per_item(kSymBatchCellsPerItem);
    }
    poff[e + 1] = poff[e] + (int)(((long long)h.ne * h.Q + kPrepBlock - 1) / kPrepBlock);
    foff[e + 1] = foff[e] + (h.ne + kFinalizeRows - 1) / kFinalizeRows;
    quad_pairs_ += h.far_quad_pairs;
    for (WorkItem w : sym_ ? sym_items : m->items_host) {
      w.mesh = e;
      const long long tg = std::min(kTT, h.nitems - w.tgt0);
      const long long src = (long long)std::min(h.ne, w.cell1 * kCell) - (long long)w.cell0 * kCell;
      items.push_back({tg * src, w});
    }
  }
  for (auto& d : desc) d.src_tile = src_tile;
  // longest items first: the dynamic queue then ends with the short ones
  std::stable_sort(items.begin(), items.end(),
                   [](const std::pair<long long, WorkItem>& a, const std::pair<long long, WorkItem>& b) {
                     return a.first > b.first;
                   });
  std::vector<WorkItem> flat(items.size());
  for (size_t k = 0; k < items.size(); k++) flat[k] = items[k].second;
  nitems_ = (int)flat.size();
  prep_blocks_ = poff[n];
  fin_blocks_ = foff[n];

  EB_CHECK(desc_.alloc(sizeof(FarMeshDesc) * n));
  EB_CHECK(copy_h2d(desc_.p, desc.data(), sizeof(FarMeshDesc) * n));
  EB_CHECK(args_.alloc(sizeof(ApplyArgs) * n));
  EB_CHECK(copy_h2d(args_.p, args.data(), sizeof(ApplyArgs) * n));
  EB_CHECK(items_.alloc(sizeof(WorkItem) * flat.size()));
  EB_CHECK(copy_h2d(items_.p, flat.data(), sizeof(WorkItem) * flat.size()));
  EB_CHECK(prep_off_.alloc(sizeof(int) * (n + 1)));
  EB_CHECK(copy_h2d(prep_off_.p, poff.data(), sizeof(int) * (n + 1)));
  EB_CHECK(fin_off_.alloc(sizeof(int) * (n + 1)));
  EB_CHECK(copy_h2d(fin_off_.p, foff.data(), sizeof(int) * (n + 1)));
  EB_CHECK(counter_.alloc(sizeof(int)));
  if (tc_) {
    EB_CHECK(tc_args_.alloc(sizeof(TcPrepArgs) * n));
    EB_CHECK(copy_h2d(tc_args_.p, targs.data(), sizeof(TcPrepArgs) * n));
    EB_CHECK(tc_off_.alloc(sizeof(int) * (n + 1)));
    EB_CHECK(copy_h2d(tc_off_.p, toff.data(), sizeof(int) * (n + 1)));
    EB_CHECK(tc_err_.alloc(sizeof(int)));
    EB_CHECK(memset_sync(tc_err_.p, 0, sizeof(int)));
    tc_blocks_ = toff[n];
  }

  smem_ = far_smem_bytes(src_tile, Q_, rec_slots(nsl_, nd_), fp32);
  int occ = far_occupancy(fp32, nsl_, nd_, K_, Q_, smem_);
  if (occ < 1) occ = 1;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  grid_ = std::min(nsm * occ, std::max(1, nitems_));
  occ_ = occ;
  nsm_ = nsm;
  if (tc_) {  // one 256-thread CTA per SM holding all of its tensor memory
    grid_ = std::min(nsm, std::max(1, nitems_));
    occ_ = 1;
  }
  if (sym_) {
    occ_ = std::max(1, far_sym_occupancy(fp32, nsl_, nd_));
    grid_ = std::min(nsm * occ_, std::max(1, nitems_));
  }
  return EB_OK;
}

int Batch::check_error()
{
  if (!tc_ || !tc_err_.p) return EB_OK;
  int flag = 0;
  EB_CHECK(copy_d2h(&flag, tc_err_.p, sizeof(int)));
  if (!flag) return EB_OK;
  EB_CHECK(memset_sync(tc_err_.p, 0, sizeof(int)));
  return set_error(EB_ERR_TIMEOUT, "tensor-core far field: a bounded wait for the tensor cores ran out");
}

int Batch::run(cudaStream_t st, int reserve_sms)
{
  if (entries_.empty()) return EB_OK;
  const int n = (int)entries_.size();
  const int free_sms = std::max(1, nsm_ - std::max(0, reserve_sms));
  const int grid = reserve_sms > 0 ? std::min(grid_, free_sms * occ_) : grid_;
  EB_CUDA(prep_launch_batch(fp32_, nsl_, nd_, args_.as<ApplyArgs>(), prep_off_.as<int>(), n, prep_blocks_, st));
  if (tc_) EB_CUDA(far_tc_prep_dl_batch(tc_args_.as<TcPrepArgs>(), tc_off_.as<int>(), n, tc_blocks_, st));
  EB_CUDA(cudaMemsetAsync(counter_.p, 0, sizeof(int), st));
  if (tc_)
    EB_CUDA(far_tc_launch(desc_.as<FarMeshDesc>(), items_.as<WorkItem>(), nitems_, counter_.as<int>(),
                          tc_err_.as<int>(), grid, st));
  else if (sym_)
    EB_CUDA(far_sym_launch(fp32_, nsl_, nd_, desc_.as<FarMeshDesc>(), items_.as<WorkItem>(), nitems_,
                           counter_.as<int>(), grid, st));
  else
    EB_CUDA(far_launch(fp32_, nsl_, nd_, K_, Q_, desc_.as<FarMeshDesc>(), items_.as<WorkItem>(), nitems_,
                       counter_.as<int>(), smem_, grid, st));
  EB_CUDA(finalize_launch_batch(nsl_, nd_, args_.as<ApplyArgs>(), fin_off_.as<int>(), n, fin_blocks_, st));
  return EB_OK;
}

int Batch::run_graph(cudaStream_t st, int reserve_sms)
{
  if (entries_.empty()) return EB_OK;
  const int k = reserve_sms > 0 ? 1 : 0;
  if (k == 1 && exec_[1] && reserve_sms != reserve_) {  // a different reservation: capture again
    cudaGraphExecDestroy(exec_[1]);
    cudaGraphDestroy(graph_[1]);
    exec_[1] = nullptr;
    graph_[1] = nullptr;
  }
  if (!exec_[k]) {
    EB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = run(st, reserve_sms);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc != EB_OK) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    EB_CUDA(e);
    graph_[k] = g;
    EB_CUDA(cudaGraphInstantiate(&exec_[k], graph_[k], 0));
    if (k == 1) reserve_ = reserve_sms;
  }
  EB_CUDA(cudaGraphLaunch(exec_[k], st));
  return EB_OK;
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI: batched applies over a fixed set of meshes.

eb::Mesh* eb_mesh_internal(eb_mesh handle);

struct eb_batch_s {
  std::vector<std::unique_ptr<eb::BatchEntry>> entries;
  eb::Batch batch;
  eb::DevBuf flags;
  cudaStream_t stream = nullptr;
  int ncols = 1;
  bool sl_dl = false;  // made by eb_batch_create_sl_dl
};

using eb::set_error;

static int batch_create(int nmesh, const eb_mesh* meshes, int ncols, int nd, int precision, eb_batch* out)
{
  if (precision != EB_PREC_FP64 && precision != EB_PREC_MIXED)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  auto b = std::make_unique<eb_batch_s>();
  b->ncols = ncols;
  b->sl_dl = nd > 0;
  std::vector<eb::BatchEntry*> ents;
  int dev = -1;
  for (int i = 0; i < nmesh; i++) {
    if (!meshes[i]) return set_error(EB_ERR_INVALID, "null mesh");
    eb::Mesh* m = eb_mesh_internal(meshes[i]);
    if (dev >= 0 && m->device != dev) return set_error(EB_ERR_INVALID, "a batch needs all meshes on one device");
    dev = m->device;
    EB_CUDA(cudaSetDevice(dev));
    auto e = std::make_unique<eb::BatchEntry>();
    EB_CHECK(eb::batch_entry_init(e.get(), m, nd > 0));
    ents.push_back(e.get());
    b->entries.push_back(std::move(e));
  }
  EB_CHECK(b->flags.alloc(sizeof(int) * nmesh));
  std::vector<int> ones(nmesh, 1);
  EB_CHECK(eb::copy_h2d(b->flags.p, ones.data(), sizeof(int) * nmesh));
  EB_CHECK(b->batch.build(ents, precision == EB_PREC_MIXED, ncols, b->flags.as<int>(), nd));
  EB_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  *out = b.release();
  return EB_OK;
}

extern "C" {

int eb_batch_create(int nmesh, const eb_mesh* meshes, int ncols, int precision, eb_batch* out)
{
  if (!out || nmesh < 1 || !meshes || ncols < 1 || ncols > eb::kBatchCols)
    return set_error(EB_ERR_INVALID, "need >= 1 mesh and 1..4 columns");
  return batch_create(nmesh, meshes, ncols, 0, precision, out);
}

int eb_batch_create_sl_dl(int nmesh, const eb_mesh* meshes, int precision, eb_batch* out)
{
  if (!out || nmesh < 1 || !meshes) return set_error(EB_ERR_INVALID, "need >= 1 mesh");
  return batch_create(nmesh, meshes, 1, 1, precision, out);
}

int eb_batch_destroy(eb_batch b)
{
  if (!b) return EB_OK;
  if (b->stream) {
    cudaStreamSynchronize(b->stream);
    cudaStreamDestroy(b->stream);
  }
  delete b;
  return EB_OK;
}

int eb_batch_apply_sl_dl(eb_batch b, const double* const* d_t, const double* const* d_u, double* const* d_v,
                         double* const* d_q, void* stream)
{
  if (!b || !d_t || !d_u || !d_v || !d_q) return set_error(EB_ERR_INVALID, "null argument");
  if (!b->sl_dl) return set_error(EB_ERR_INVALID, "batch made by eb_batch_create: use eb_batch_apply");
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  for (size_t i = 0; i < b->entries.size(); i++) {
    const eb::BatchEntry& e = *b->entries[i];
    if (!d_t[i] || !d_u[i] || !d_v[i] || !d_q[i]) return set_error(EB_ERR_INVALID, "null vector");
    EB_CUDA(cudaMemcpyAsync(e.tin.p, d_t[i], sizeof(double) * e.mesh->h.ne, cudaMemcpyDeviceToDevice, st));
    EB_CUDA(cudaMemcpyAsync(e.uin.p, d_u[i], sizeof(double) * e.mesh->h.nv, cudaMemcpyDeviceToDevice, st));
  }
  EB_CHECK(b->batch.run_graph(st));
  for (size_t i = 0; i < b->entries.size(); i++) {
    const eb::BatchEntry& e = *b->entries[i];
    EB_CUDA(cudaMemcpyAsync(d_v[i], e.vout.p, sizeof(double) * e.mesh->h.ne, cudaMemcpyDeviceToDevice, st));
    EB_CUDA(cudaMemcpyAsync(d_q[i], e.qout.p, sizeof(double) * e.mesh->h.ne, cudaMemcpyDeviceToDevice, st));
  }
  if (!stream) {
    EB_CUDA(cudaStreamSynchronize(st));
    EB_CHECK(b->batch.check_error());
  }
  return EB_OK;
}

int eb_batch_apply(eb_batch b, const double* const* d_t, double* const* d_v, void* stream)
{
  if (!b || !d_t || !d_v) return set_error(EB_ERR_INVALID, "null argument");
  if (b->sl_dl) return set_error(EB_ERR_INVALID, "batch made by eb_batch_create_sl_dl: use eb_batch_apply_sl_dl");
  cudaStream_t st = stream ? (cudaStream_t)stream : b->stream;
  for (size_t i = 0; i < b->entries.size(); i++) {
    const size_t bytes = sizeof(double) * (size_t)b->ncols * b->entries[i]->mesh->h.ne;
    EB_CUDA(cudaMemcpyAsync(b->entries[i]->tin.p, d_t[i], bytes, cudaMemcpyDeviceToDevice, st));
  }
  EB_CHECK(b->batch.run_graph(st));
  for (size_t i = 0; i < b->entries.size(); i++) {
    const size_t bytes = sizeof(double) * (size_t)b->ncols * b->entries[i]->mesh->h.ne;
    EB_CUDA(cudaMemcpyAsync(d_v[i], b->entries[i]->vout.p, bytes, cudaMemcpyDeviceToDevice, st));
  }
  if (!stream) EB_CUDA(cudaStreamSynchronize(st));
  return EB_OK;
}

int eb_batch_info(eb_batch b, long long* quad_pairs)
{
  if (!b) return set_error(EB_ERR_INVALID, "null batch");
  if (quad_pairs) *quad_pairs = b->batch.quad_pairs();
  return EB_OK;
}

}  // extern "C"
