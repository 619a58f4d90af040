// Single layer with P1 test and trial functions, v = V1 t (t, v at vertices).
//
// Replaces applyGPULaplace3d1Layer(t, v, ansatz=1) (src/BEM3dLaplaceGPU.cu:
// 985-1322 with kernels :82-154, 211-320, 371-442, 491-557). Near pairs use the
// reference's P1 Sauter-Schwab formulas in FP64 (pairs.h), stored once as a
// vertex x vertex CSR; the trial indices come from the trial triangle (the
// reference takes them from the test triangle off the diagonal). The far
// field is the SL tile kernel with the P1-interpolated density as the charge
// (w_b J_j u_h(y_b)) and three outputs per target triangle,
// sum_a w_a phi_k(x_a) acc_a, gathered per vertex by the finalize kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine.h"
#include "pairs.h"

namespace eb {

__global__ void near_p1_kernel(Quadrature q, const double* __restrict__ nodes, const int* __restrict__ elems,
                               const int* __restrict__ pi, const int* __restrict__ pj, int npairs,
                               double* __restrict__ ent)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const int i = pi[p], j = pj[p];
  const int fi[3] = {elems[3 * i], elems[3 * i + 1], elems[3 * i + 2]};
  const int fj[3] = {elems[3 * j], elems[3 * j + 1], elems[3 * j + 2]};
  d3 Pi[3], Pj[3];
  for (int k = 0; k < 3; k++) {
    Pi[k] = mk3(nodes[3 * fi[k]], nodes[3 * fi[k] + 1], nodes[3 * fi[k] + 2]);
    Pj[k] = mk3(nodes[3 * fj[k]], nodes[3 * fj[k] + 1], nodes[3 * fj[k] + 2]);
  }
  const PairGeom g = classify_pair(fi, fj, i == j);
  int oi[3], oj[3];
  p1_local_orders(g, oi, oj);
  double I[9];
  near_pair_values_p1(q, g, Pi, Pj, oi, oj, I);
  for (int k = 0; k < 9; k++) ent[9 * (size_t)p + k] = I[k];
}

__global__ void p1_gather_kernel(const int* __restrict__ cptr, const int* __restrict__ contrib,
                                 const double* __restrict__ ent, int nslots, double* __restrict__ out)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  double acc = 0.0;
  for (int k = cptr[s]; k < cptr[s + 1]; k++) acc += ent[contrib[k]];
  out[s] = acc;
}

// v[a] = sum over (triangle i, local k) at vertex a of J_i/(4 pi) * far_k(i)
//        + sum_b V1near[a][b] t[b]
__global__ void p1_finalize_kernel(int nv, int nchunk, int nsplit, int nitems, const int* __restrict__ vptr,
                                   const int* __restrict__ vlist, const int* __restrict__ iperm,
                                   const dq* __restrict__ trin, const double* __restrict__ partial,
                                   const int* __restrict__ rowptr, const int* __restrict__ col,
                                   const double* __restrict__ val, const double* __restrict__ t,
                                   double* __restrict__ v)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nv) return;
  const size_t stride = (size_t)nsplit * nitems;
  double far = 0.0;
  for (int p = vptr[a]; p < vptr[a + 1]; p++) {
    const int i = vlist[p] >> 2, k = vlist[p] & 3;
    const int s = iperm[i];
    double f = 0.0;
    for (int sp = 0; sp < nsplit; sp++)
      for (int ch = 0; ch < nchunk; ch++) f += partial[k * stride + (size_t)sp * nitems + (size_t)s * nchunk + ch];
    far += trin[s].w * (0.25 / M_PI) * f;
  }
  double nr = 0.0;
  for (int k = rowptr[a]; k < rowptr[a + 1]; k++) nr += val[k] * t[col[k]];
  v[a] = far + nr;
}

static int ensure_p1_near(Mesh* m)
{
  if (m->p1_val.p) return EB_OK;
  const HostMesh& h = m->h;
  const int npairs = (int)h.sl_col.size();
  // entries e = 9p + 3k + l at (test vertex, trial vertex), bucketed by row
  std::vector<int> erow(9 * (size_t)npairs), ecol(9 * (size_t)npairs);
  for (int p = 0; p < npairs; p++) {
    const int i = h.pair_i[p], j = h.sl_col[p];
    const PairGeom g = classify_pair(&h.elems[3 * i], &h.elems[3 * j], i == j);
    int oi[3], oj[3];
    p1_local_orders(g, oi, oj);
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) {
        erow[9 * (size_t)p + 3 * k + l] = h.elems[3 * i + oi[k]];
        ecol[9 * (size_t)p + 3 * k + l] = h.elems[3 * j + oj[l]];
      }
  }
  std::vector<int> rcount(h.nv + 1, 0);
  for (int r : erow) rcount[r + 1]++;
  for (int v = 0; v < h.nv; v++) rcount[v + 1] += rcount[v];
  std::vector<int> byrow(erow.size());
  {
    std::vector<int> fill(rcount.begin(), rcount.end() - 1);
    for (size_t e = 0; e < erow.size(); e++) byrow[fill[erow[e]]++] = (int)e;
  }
  std::vector<int> rowptr(h.nv + 1, 0), cols, cptr(1, 0), contrib;
  contrib.reserve(erow.size());
  for (int a = 0; a < h.nv; a++) {
    std::vector<std::pair<int, int>> es;
    for (int q = rcount[a]; q < rcount[a + 1]; q++) es.push_back({ecol[byrow[q]], byrow[q]});
    std::sort(es.begin(), es.end());
    for (size_t q = 0; q < es.size(); q++) {
      if (q > 0 && es[q].first != es[q - 1].first) cptr.push_back((int)contrib.size());
      if (q == 0 || es[q].first != es[q - 1].first) cols.push_back(es[q].first);
      contrib.push_back(es[q].second);
    }
    if (!es.empty()) cptr.push_back((int)contrib.size());
    rowptr[a + 1] = (int)cols.size();
  }
  DevBuf d_nodes, d_elems, d_pi, d_pj, d_ent, d_cptr, d_contrib;
  auto up = [](DevBuf& b, const void* src, size_t bytes) -> int {
    EB_CHECK(b.alloc(std::max<size_t>(bytes, 16)));
    if (bytes) EB_CHECK(copy_h2d(b.p, src, bytes));
    return EB_OK;
  };
  EB_CHECK(up(d_nodes, h.nodes.data(), sizeof(double) * h.nodes.size()));
  EB_CHECK(up(d_elems, h.elems.data(), sizeof(int) * h.elems.size()));
  EB_CHECK(up(d_pi, h.pair_i.data(), sizeof(int) * h.pair_i.size()));
  EB_CHECK(up(d_pj, h.sl_col.data(), sizeof(int) * h.sl_col.size()));
  EB_CHECK(up(d_cptr, cptr.data(), sizeof(int) * cptr.size()));
  EB_CHECK(up(d_contrib, contrib.data(), sizeof(int) * contrib.size()));
  EB_CHECK(up(m->p1_rowptr, rowptr.data(), sizeof(int) * rowptr.size()));
  EB_CHECK(up(m->p1_col, cols.data(), sizeof(int) * cols.size()));
  EB_CHECK(d_ent.alloc(sizeof(double) * std::max<size_t>(erow.size(), 1)));
  EB_CHECK(m->p1_val.alloc(sizeof(double) * std::max<size_t>(cols.size(), 1)));
  cudaStream_t st = nullptr;
  EB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  if (npairs > 0)
    near_p1_kernel<<<(npairs + 127) / 128, 128, 0, st>>>(h.quad, d_nodes.as<double>(), d_elems.as<int>(),
                                                         d_pi.as<int>(), d_pj.as<int>(), npairs, d_ent.as<double>());
  const int nslots = (int)cols.size();
  if (nslots > 0)
    p1_gather_kernel<<<(nslots + 255) / 256, 256, 0, st>>>(d_cptr.as<int>(), d_contrib.as<int>(), d_ent.as<double>(),
                                                          nslots, m->p1_val.as<double>());
  const cudaError_t e1 = cudaGetLastError();
  const cudaError_t e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  EB_CUDA(e1);
  EB_CUDA(e2);
  return EB_OK;
}

int mesh_apply_sl_p1(Mesh* m, int precision, const double* d_t, double* d_v, cudaStream_t st)
{
  if (!d_t || !d_v) return set_error(EB_ERR_INVALID, "null vector");
  if (precision != EB_PREC_MIXED && precision != EB_PREC_FP64)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  const bool fp32 = precision == EB_PREC_MIXED;
  EB_CHECK(ensure_p1_near(m));
  EB_CHECK(ensure_vertex_lists(m));
  const HostMesh& h = m->h;
  if (!m->rec.p) {
    EB_CHECK(m->rec.alloc((size_t)h.ne * h.Q * kMaxRecSlots * sizeof(dq)));
    EB_CHECK(m->partial.alloc(sizeof(double) * (size_t)kMaxOutputs * m->plan.nsplit * h.nitems));
  }
  Mesh::Variant& var = m->variants[100 + (fp32 ? 1 : 0)];
  if (!var.desc.p) {
    const FarMeshDesc desc = mesh_far_desc(m, fp32, 1, false, m->rec.p, m->partial.as<double>());
    const size_t smem = far_smem_bytes(desc.src_tile, h.Q, rec_slots(1, false), fp32);
    int occ = far_occupancy(fp32, 1, false, h.K, h.Q, smem, true);
    if (occ < 1) occ = 1;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    EB_CHECK(var.desc.alloc(sizeof(FarMeshDesc)));
    EB_CHECK(copy_h2d(var.desc.p, &desc, sizeof desc));
    var.grid = std::min(nsm * occ, std::max(1, m->nitems_work));
    var.smem = smem;
    var.src_tile = desc.src_tile;
  }
  // records: the DL strength slot (w_b J_j u_h(y_b)) is where the single SL
  // charge of the far kernel is read (record slot 1, component 0)
  const ApplyArgs A = mesh_apply_args(m, fp32, m->rec.p, nullptr, nullptr, h.ne, d_t, nullptr, h.ne, nullptr);
  EB_CUDA(prep_launch(fp32, 0, true, A, st));
  EB_CUDA(cudaMemsetAsync(m->counter.p, 0, sizeof(int), st));
  EB_CUDA(far_launch(fp32, 1, false, h.K, h.Q, var.desc.as<FarMeshDesc>(), m->items.as<WorkItem>(), m->nitems_work,
                     m->counter.as<int>(), var.smem, var.grid, st, true));
  p1_finalize_kernel<<<(h.nv + 127) / 128, 128, 0, st>>>(
      h.nv, h.nchunk, m->plan.nsplit, h.nitems, m->vtri_ptr.as<int>(), m->vtri_list.as<int>(), m->iperm.as<int>(),
      m->trin.as<dq>(), m->partial.as<double>(), m->p1_rowptr.as<int>(), m->p1_col.as<int>(), m->p1_val.as<double>(),
      d_t, d_v);
  EB_CUDA(cudaGetLastError());
  return EB_OK;
}

}  // namespace eb
