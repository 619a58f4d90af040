// Hypersingular operator D (P1 x P1) in the curl form of getLaplace3d
// (src/BEM3dLaplace.cpp:615-637 and :767-771):
//
//   D[a][b] = sum_{i,j} sum_m curl_i^m[k] V(i,j) curl_j^m[l],  a = node(i,k), b = node(j,l)
//
// i.e. D u = sum_m C_m^T V (C_m u) with C_m (nelems x nnodes) the m-th
// Cartesian component of the surface curl of the P1 basis on each triangle.
// The reference GPU entry point applyGPULaplace3dHyperSing is empty
// (src/BEM3dLaplaceGPU.cu:1554-1555); here D u is one curl gather, one SL
// apply with the three curl components as right-hand sides (they share every
// distance evaluation) and one transpose gather per vertex (no atomics, so
// the result is deterministic).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "engine.h"

namespace eb {

// Surface-curl coefficients of the three P1 basis functions of a triangle:
// with e1 = P1 - P0, e2 = P2 - P0, n the unit normal e1 x e2 / |e1 x e2|, the
// metric A = [[e1.e1, e1.e2], [e1.e2, e2.e2]] and b_k = n x e_k, the
// coefficients y = A^{-1} (b_1, b_2) give curl^m = (-y1m - y2m, y1m, y2m).
static void triangle_curls(const d3& P0, const d3& P1, const d3& P2, double* c /* [3][3] m-major */)
{
  const d3 e1 = P1 - P0, e2 = P2 - P0;
  d3 n = cross3(e1, e2);
  n = (1.0 / std::sqrt(dot3(n, n))) * n;
  const double a11 = dot3(e1, e1), a22 = dot3(e2, e2), a12 = dot3(e1, e2);
  const double det = a11 * a22 - a12 * a12;
  const d3 b1 = cross3(n, e1), b2 = cross3(n, e2);
  const double B1[3] = {b1.x, b1.y, b1.z}, B2[3] = {b2.x, b2.y, b2.z};
  for (int m = 0; m < 3; m++) {
    const double y1 = (B1[m] * a22 - B2[m] * a12) / det;
    const double y2 = (a11 * B2[m] - a12 * B1[m]) / det;
    c[3 * m + 0] = -y1 - y2;
    c[3 * m + 1] = y1;
    c[3 * m + 2] = y2;
  }
}

__global__ void curl_gather_kernel(int ne, const int* __restrict__ elems, const double* __restrict__ curl,
                                   const double* __restrict__ u, double* __restrict__ x)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const double u0 = u[elems[3 * i]], u1 = u[elems[3 * i + 1]], u2 = u[elems[3 * i + 2]];
  const double* c = curl + 9 * (size_t)i;
  for (int m = 0; m < 3; m++) x[(size_t)m * ne + i] = c[3 * m] * u0 + c[3 * m + 1] * u1 + c[3 * m + 2] * u2;
}

__global__ void curl_scatter_kernel(int nv, int ne, const int* __restrict__ vptr, const int* __restrict__ vlist,
                                    const double* __restrict__ curl, const double* __restrict__ w,
                                    double* __restrict__ out)
{
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= nv) return;
  double acc = 0.0;
  for (int p = vptr[a]; p < vptr[a + 1]; p++) {
    const int i = vlist[p] >> 2, k = vlist[p] & 3;
    const double* c = curl + 9 * (size_t)i;
    acc += c[k] * w[i] + c[3 + k] * w[(size_t)ne + i] + c[6 + k] * w[2 * (size_t)ne + i];
  }
  out[a] = acc;
}

int ensure_vertex_lists(Mesh* m)
{
  if (m->vtri_ptr.p) return EB_OK;
  const HostMesh& h = m->h;
  // vertex -> (triangle, local index) in ascending triangle order
  std::vector<int> vptr(h.nv + 1, 0), vlist(3 * (size_t)h.ne);
  for (int e = 0; e < 3 * h.ne; e++) vptr[h.elems[e] + 1]++;
  for (int v = 0; v < h.nv; v++) vptr[v + 1] += vptr[v];
  std::vector<int> fill(vptr.begin(), vptr.end() - 1);
  for (int i = 0; i < h.ne; i++)
    for (int k = 0; k < 3; k++) vlist[fill[h.elems[3 * i + k]]++] = (i << 2) | k;
  EB_CHECK(m->vtri_ptr.alloc(sizeof(int) * vptr.size()));
  EB_CHECK(copy_h2d(m->vtri_ptr.p, vptr.data(), sizeof(int) * vptr.size()));
  EB_CHECK(m->vtri_list.alloc(sizeof(int) * vlist.size()));
  EB_CHECK(copy_h2d(m->vtri_list.p, vlist.data(), sizeof(int) * vlist.size()));
  EB_CHECK(m->elems0.alloc(sizeof(int) * h.elems.size()));
  EB_CHECK(copy_h2d(m->elems0.p, h.elems.data(), sizeof(int) * h.elems.size()));
  return EB_OK;
}

static int ensure_curls(Mesh* m)
{
  if (m->curl9.p) return EB_OK;
  EB_CHECK(ensure_vertex_lists(m));
  const HostMesh& h = m->h;
  std::vector<double> curl(9 * (size_t)h.ne);
  for (int i = 0; i < h.ne; i++) {
    const int* f = &h.elems[3 * i];
    d3 P[3];
    for (int k = 0; k < 3; k++) P[k] = mk3(h.nodes[3 * f[k]], h.nodes[3 * f[k] + 1], h.nodes[3 * f[k] + 2]);
    triangle_curls(P[0], P[1], P[2], &curl[9 * (size_t)i]);
  }
  EB_CHECK(m->curl9.alloc(sizeof(double) * curl.size()));
  EB_CHECK(copy_h2d(m->curl9.p, curl.data(), sizeof(double) * curl.size()));
  EB_CHECK(m->hs_x.alloc(sizeof(double) * 3 * (size_t)h.ne));
  EB_CHECK(m->hs_w.alloc(sizeof(double) * 3 * (size_t)h.ne));
  return EB_OK;
}

int mesh_apply_hypersingular(Mesh* m, int precision, const double* d_u, double* d_q, cudaStream_t st)
{
  if (!d_u || !d_q) return set_error(EB_ERR_INVALID, "null vector");
  EB_CHECK(ensure_curls(m));
  const HostMesh& h = m->h;
  const int blk = 128;
  curl_gather_kernel<<<(h.ne + blk - 1) / blk, blk, 0, st>>>(h.ne, m->elems0.as<int>(), m->curl9.as<double>(), d_u,
                                                              m->hs_x.as<double>());
  EB_CUDA(cudaGetLastError());
  EB_CHECK(mesh_apply(m, precision, 3, false, m->hs_x.as<double>(), nullptr, m->hs_w.as<double>(), nullptr, st));
  curl_scatter_kernel<<<(h.nv + blk - 1) / blk, blk, 0, st>>>(h.nv, h.ne, m->vtri_ptr.as<int>(),
                                                               m->vtri_list.as<int>(), m->curl9.as<double>(),
                                                               m->hs_w.as<double>(), d_q);
  EB_CUDA(cudaGetLastError());
  return EB_OK;
}

}  // namespace eb
