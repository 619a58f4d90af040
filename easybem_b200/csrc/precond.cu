// Near-field sparse approximate inverse of the P0 single layer, the right
// preconditioner of the GMRES solves (no counterpart in the reference, whose
// drivers call SciPy's CG without a preconditioner,
// python/examples/laplace3dDirichletGPU.py:64-81).
//
// N is the FP64 near-field matrix (the Sauter-Schwab values of all pairs of
// triangles that share a vertex, the CSR the applies already hold). Column j
// of M minimises || N m_j - e_j ||_2 over vectors supported on the
// neighbours J_j of triangle j (its CSR row pattern, the triangles sharing a
// vertex with it); the residual runs over all rows that N couples to J_j.
// With A = N[:, J_j] the normal equations are (A^T A) m = A^T e_j, where
// (A^T A)_ab = <N[:, k_a], N[:, k_b]> are sparse column dot products and
// (A^T e_j)_a = N[j, k_a]. The pattern is symmetric, so M is stored with the
// near-field CSR pattern itself (row i holds M[i, j] for the j sharing a
// vertex with i), and y = M x is one more CSR SpMV.
//
// One warp per column: lane a owns row a of the Gram matrix (|J_j| <= 32;
// columns with larger neighbourhoods, and columns whose Gram matrix is not
// numerically positive definite, fall back to the diagonal M[j, j] = 1 / N[j, j]).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "easybem_gpu.h"
#include "engine.h"

namespace eb {

constexpr int kPcWarps = 4;  // columns per block

__device__ __forceinline__ double sparse_col_dot(const int* __restrict__ rowptr, const int* __restrict__ col,
                                                 const double* __restrict__ val, const int* __restrict__ tpos, int ka,
                                                 int kb)
{
  // column k of N: rows col[p] for p in row k (symmetric pattern), values val[tpos[p]]
  int p = rowptr[ka], pe = rowptr[ka + 1];
  int q = rowptr[kb], qe = rowptr[kb + 1];
  double acc = 0.0;
  while (p < pe && q < qe) {
    const int ia = col[p], ib = col[q];
    if (ia == ib) {
      acc += val[tpos[p]] * val[tpos[q]];
      ++p;
      ++q;
    } else if (ia < ib) {
      ++p;
    } else {
      ++q;
    }
  }
  return acc;
}

__global__ void __launch_bounds__(32 * kPcWarps)
    near_spai_kernel(int ne, const int* __restrict__ rowptr, const int* __restrict__ col,
                     const double* __restrict__ val, const int* __restrict__ tpos, double* __restrict__ mval)
{
  __shared__ double G[kPcWarps][32][33];  // Gram matrix; its lower triangle becomes L in place
  __shared__ double yv[kPcWarps][32];
  __shared__ int ok[kPcWarps];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * kPcWarps + w;
  if (j >= ne) return;  // warp-uniform
  const int rs = rowptr[j], n = rowptr[j + 1] - rs;
  // diagonal position of row j (the coincident pair) for the fallback
  int pd = -1;
  for (int a = lane; a < n; a += 32)
    if (col[rs + a] == j) pd = a;
  for (int o = 16; o > 0; o >>= 1) pd = max(pd, __shfl_xor_sync(0xffffffffu, pd, o));
  auto fallback = [&]() {
    for (int a = lane; a < n; a += 32) mval[tpos[rs + a]] = (a == pd && val[rs + a] != 0.0) ? 1.0 / val[rs + a] : 0.0;
  };
  if (n > 32 || pd < 0) {
    fallback();
    return;
  }
  double (*Gw)[33] = G[w];
  double (*Lw)[33] = G[w];  // L[a][t] (t <= a) overwrites G[a][t]; the upper triangle keeps G
  if (lane < n) {
    const int ka = col[rs + lane];
    for (int b = 0; b <= lane; ++b) {
      const double g = sparse_col_dot(rowptr, col, val, tpos, ka, col[rs + b]);
      Gw[lane][b] = g;
      Gw[b][lane] = g;
    }
  }
  __syncwarp();
  // a small relative shift keeps the factorisation away from round-off breakdown
  double tr = 0.0;
  for (int a = 0; a < n; ++a) tr += Gw[a][a];
  __syncwarp();  // every lane has read the diagonal before lane 0 overwrites it
  double diag[32];
  if (lane == 0)
    for (int a = 0; a < n; ++a) diag[a] = Gw[a][a];
  const double shift = 1e-12 * tr / n;
  if (lane == 0) ok[w] = 1;
  __syncwarp();
  // Cholesky G = L L^T, column by column
  for (int c = 0; c < n; ++c) {
    if (lane == 0) {
      double d = diag[c] + shift;
      for (int t = 0; t < c; ++t) d -= Lw[c][t] * Lw[c][t];
      if (!(d > 0.0)) ok[w] = 0;
      Lw[c][c] = d > 0.0 ? sqrt(d) : 1.0;
    }
    __syncwarp();
    if (lane > c && lane < n) {
      double s = Gw[c][lane];  // = G[lane][c], read from the untouched upper triangle
      for (int t = 0; t < c; ++t) s -= Lw[lane][t] * Lw[c][t];
      Lw[lane][c] = s / Lw[c][c];
    }
    __syncwarp();
  }
  if (!ok[w]) {
    fallback();
    return;
  }
  // L L^T m = r with r_a = N[j, k_a]
  if (lane == 0) {
    for (int a = 0; a < n; ++a) {
      double s = val[rs + a];
      for (int t = 0; t < a; ++t) s -= Lw[a][t] * yv[w][t];
      yv[w][a] = s / Lw[a][a];
    }
    for (int a = n - 1; a >= 0; --a) {
      double s = yv[w][a];
      for (int t = a + 1; t < n; ++t) s -= Lw[t][a] * yv[w][t];
      yv[w][a] = s / Lw[a][a];
    }
  }
  __syncwarp();
  // column j of M goes to row k_a of the stored (row-major) pattern
  if (lane < n) mval[tpos[rs + lane]] = yv[w][lane];
}

// y = M x with M on the near-field pattern (original triangle order)
__global__ void near_spmv_kernel(int ne, const int* __restrict__ rowptr, const int* __restrict__ col,
                                 const double* __restrict__ mval, const double* __restrict__ x, double* __restrict__ y)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  double acc = 0.0;
  for (int p = rowptr[i]; p < rowptr[i + 1]; ++p) acc += mval[p] * x[col[p]];
  y[i] = acc;
}

int ensure_near_precond(Mesh* m)
{
  if (m->pc_val.p) return EB_OK;
  const HostMesh& h = m->h;
  const int nnz = (int)h.sl_col.size();
  // tpos[p] = CSR position of (col, row) for entry p = (row, col)
  std::vector<int> tpos(std::max(nnz, 1), 0);
  for (int i = 0; i < h.ne; i++)
    for (int p = h.sl_rowptr[i]; p < h.sl_rowptr[i + 1]; p++) {
      const int j = h.sl_col[p];
      const int* b = h.sl_col.data() + h.sl_rowptr[j];
      const int* e = h.sl_col.data() + h.sl_rowptr[j + 1];
      const int* f = std::lower_bound(b, e, i);
      if (f == e || *f != i) return set_error(EB_ERR_MESH, "near-field pattern is not symmetric");
      tpos[p] = (int)(f - h.sl_col.data());
    }
  DevBuf pc;
  EB_CHECK(pc.alloc(sizeof(double) * std::max(nnz, 1)));
  cudaStream_t st = nullptr;
  EB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = EB_OK;
  cudaError_t e1 = cudaSuccess;
  {
    TmpBuf d_tpos(st);  // stream-ordered: released without a device-wide wait
    rc = d_tpos.alloc(sizeof(int) * tpos.size());
    if (rc == EB_OK) {
      e1 = cudaMemcpyAsync(d_tpos.p, tpos.data(), sizeof(int) * tpos.size(), cudaMemcpyHostToDevice, st);
      if (e1 == cudaSuccess && h.ne > 0)
        near_spai_kernel<<<(h.ne + kPcWarps - 1) / kPcWarps, 32 * kPcWarps, 0, st>>>(
            h.ne, m->sl_rowptr.as<int>(), m->sl_col.as<int>(), m->sl_val.as<double>(), d_tpos.as<int>(),
            pc.as<double>());
      if (e1 == cudaSuccess) e1 = cudaGetLastError();
    }
  }
  const cudaError_t e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  EB_CHECK(rc);
  EB_CUDA(e1);
  EB_CUDA(e2);
  std::swap(m->pc_val.p, pc.p);
  std::swap(m->pc_val.bytes, pc.bytes);
  return EB_OK;
}

cudaError_t near_precond_apply(const Mesh* m, const double* d_x, double* d_y, cudaStream_t st)
{
  const int ne = m->h.ne;
  near_spmv_kernel<<<(ne + 127) / 128, 128, 0, st>>>(ne, m->sl_rowptr.as<int>(), m->sl_col.as<int>(),
                                                    m->pc_val.as<double>(), d_x, d_y);
  return cudaGetLastError();
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI

eb::Mesh* eb_mesh_internal(eb_mesh handle);

extern "C" int eb_apply_near_precond(eb_mesh mesh, const double* x, double* y)
{
  eb::Mesh* m = eb_mesh_internal(mesh);
  if (!m) return eb::set_error(EB_ERR_INVALID, "null mesh");
  if (!x || !y) return eb::set_error(EB_ERR_INVALID, "null vector");
  EB_CUDA(cudaSetDevice(m->device));
  EB_CHECK(eb::ensure_near_precond(m));
  const size_t bytes = sizeof(double) * m->h.ne;
  eb::DevBuf dx, dy;
  EB_CHECK(dx.alloc(bytes));
  EB_CHECK(dy.alloc(bytes));
  EB_CHECK(eb::copy_h2d(dx.p, x, bytes));
  EB_CUDA(eb::near_precond_apply(m, dx.as<double>(), dy.as<double>(), nullptr));
  EB_CUDA(cudaStreamSynchronize(nullptr));  // the copy below runs on another stream
  EB_CHECK(eb::copy_d2h(y, dy.p, bytes));
  return EB_OK;
}
