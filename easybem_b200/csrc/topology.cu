// Near-pair topology on the device: the CSR lists of triangle pairs that
// share a vertex (the Sauter-Schwab near field) and their double-layer
// vertex columns, the same arrays host_topology (mesh_host.cpp) builds, in
// the same order, for large meshes.
//
// The reference finds adjacency on the host by an O(ne * nedges) edge search
// (src/meshTopology.cpp:22-261) and classifies every pair per matvec
// (src/BEM3dLaplaceGPU.cu:1224-1260). Here: vertex -> triangle incidence by
// atomic counts, an exclusive scan and an atomic fill; then one thread per
// test triangle gathers the triangles of its three vertices, sorts and
// de-duplicates them, and classifies each pair (pairs.h). A first pass counts
// a row's pairs, DL columns and DL entries, scans turn the counts into row
// offsets, and a second pass writes the rows. Sorting within a row makes the
// output independent of the order of the atomic fill, so it equals the host
// arrays bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <climits>
#include <vector>

#include "common.h"
#include "engine.h"
#include "mesh_host.h"
#include "pairs.h"

namespace eb {

namespace {

constexpr int kMaxCand = 48;  // candidate triangles per row (with repeats; valence up to 16); more falls back to the host
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;        // elements per thread of a scan block
constexpr int kScanBlock = kScanThreads * kScanItems;

__global__ void vertex_count_kernel(const int* __restrict__ elems, int ncorner, int* __restrict__ vcount)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncorner) atomicAdd(&vcount[elems[c]], 1);
}

__global__ void vertex_fill_kernel(const int* __restrict__ elems, int ncorner, int* __restrict__ cursor,
                                   int* __restrict__ vtri)
{
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncorner) vtri[atomicAdd(&cursor[elems[c]], 1)] = c / 3;
}

// Exclusive scan of one block of kScanBlock elements: out[k] = sum of in[<k]
// within the block, plus the block's total in sums[blockIdx.x].
__global__ void scan_block_kernel(const int* __restrict__ in, int n, int* __restrict__ out, int* __restrict__ sums)
{
  __shared__ int warp_tot[kScanThreads / 32];
  const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;
  int v[kScanItems], run = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    const int x = v[k];
    v[k] = run;
    run += x;
  }
  // inclusive scan of the thread totals across the warp, then across warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = run;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, d);
    if (lane >= d) incl += y;
  }
  if (lane == 31) warp_tot[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += warp_tot[w];
  const int excl = before + incl - run;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) out[base + k] = excl + v[k];
  if (threadIdx.x == kScanThreads - 1) sums[blockIdx.x] = before + incl;
}

__global__ void scan_add_kernel(int* __restrict__ out, int n, const int* __restrict__ offs)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] += offs[k / kScanBlock];
}

__global__ void copy_total_kernel(const int* __restrict__ in, const int* __restrict__ excl, int n, int* __restrict__ out)
{
  if (threadIdx.x == 0 && blockIdx.x == 0) out[n] = n > 0 ? excl[n - 1] + in[n - 1] : 0;
}

// Lexicographic order of (column, entry) pairs.
__host__ __device__ inline bool less2(int2 a, int2 b) { return a.x < b.x || (a.x == b.x && a.y < b.y); }

// One test triangle's row. FILL = false: counts of the row's pairs (repeated
// triangles excluded), DL vertex columns and DL entries, and in *nuniq the
// candidates including repeats (for the far-field pair count). FILL = true:
// the row written at the scanned offsets. Pairs are in ascending trial index
// and DL entries in ascending (column, entry id) order, as on the host.
// Returns false when the row has more than kMaxCand candidates.
template <bool FILL>
__host__ __device__ inline bool topology_row(int i, const int* __restrict__ elems, const int* __restrict__ vptr,
                                             const int* __restrict__ vtri, int* nuniq, int* nsl_out, int* ndl_out,
                                             int* nde_out, int p0, int g0, int e0, int* __restrict__ sl_col,
                                             int* __restrict__ pair_i, int8_t* __restrict__ pair_kind,
                                             int* __restrict__ dl_col, int* __restrict__ cptr,
                                             int* __restrict__ contrib)
{
  const int fi[3] = {elems[3 * i], elems[3 * i + 1], elems[3 * i + 2]};
  int cand[kMaxCand];
  int nc = 0;
  for (int k = 0; k < 3; ++k) {
    const int v = fi[k];
    for (int p = vptr[v]; p < vptr[v + 1]; ++p) {
      if (nc == kMaxCand) return false;
      cand[nc++] = vtri[p];
    }
  }
  // insertion sort and de-duplication
  for (int a = 1; a < nc; ++a) {
    const int x = cand[a];
    int b = a - 1;
    while (b >= 0 && cand[b] > x) {
      cand[b + 1] = cand[b];
      --b;
    }
    cand[b + 1] = x;
  }
  int nu = 0;
  for (int a = 0; a < nc; ++a)
    if (a == 0 || cand[a] != cand[a - 1]) cand[nu++] = cand[a];
  *nuniq = nu;

  int2 de[3 * kMaxCand];
  int nde = 0, nsl = 0;
  for (int u = 0; u < nu; ++u) {
    const int j = cand[u];
    const int fj[3] = {elems[3 * j], elems[3 * j + 1], elems[3 * j + 2]};
    const PairGeom g = classify_pair(fi, fj, i == j);
    if (g.kind == kPairRepeat) continue;  // a repeated triangle contributes nothing
    const int p = p0 + nsl++;
    if (FILL) {
      sl_col[p] = j;
      pair_i[p] = i;
      pair_kind[p] = (int8_t)g.kind;
    }
    if (g.kind == kPairVertex || g.kind == kPairEdge) {
      int slots[3];
      dl_trial_slots(g, slots);
      for (int k = 0; k < 3; ++k) de[nde++] = make_int2(fj[slots[k]], 3 * p + k);
    }
  }
  for (int a = 1; a < nde; ++a) {
    const int2 x = de[a];
    int b = a - 1;
    while (b >= 0 && less2(x, de[b])) {
      de[b + 1] = de[b];
      --b;
    }
    de[b + 1] = x;
  }
  if (!FILL) {
    int ndl = 0;
    for (int e = 0; e < nde; ++e)
      if (e == 0 || de[e].x != de[e - 1].x) ++ndl;
    *nsl_out = nsl;
    *ndl_out = ndl;
    *nde_out = nde;
    return true;
  }
  // columns, their entries, and each column's end offset in the entry list
  int gcol = g0 - 1;
  for (int e = 0; e < nde; ++e) {
    if (e == 0 || de[e].x != de[e - 1].x) dl_col[++gcol] = de[e].x;
    contrib[e0 + e] = de[e].y;
    if (e == nde - 1 || de[e + 1].x != de[e].x) cptr[gcol + 1] = e0 + e + 1;
  }
  return true;
}

// One test triangle per thread: topology_row, counting (FILL = false) or
// writing at the scanned offsets (FILL = true).
template <bool FILL>
__global__ void __launch_bounds__(128) topology_rows_kernel(
    const int* __restrict__ elems, const int* __restrict__ vptr, const int* __restrict__ vtri, int ne,
    int* __restrict__ slcnt, int* __restrict__ dlcnt, int* __restrict__ ecnt,
    unsigned long long* __restrict__ ncand, int* __restrict__ overflow, const int* __restrict__ slptr,
    const int* __restrict__ dlptr, const int* __restrict__ eptr, int* __restrict__ sl_col, int* __restrict__ pair_i,
    int8_t* __restrict__ pair_kind, int* __restrict__ dl_col, int* __restrict__ cptr, int* __restrict__ contrib)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  int nu = 0, nsl = 0, ndl = 0, nde = 0;
  const bool ok = topology_row<FILL>(i, elems, vptr, vtri, &nu, &nsl, &ndl, &nde, FILL ? slptr[i] : 0,
                                     FILL ? dlptr[i] : 0, FILL ? eptr[i] : 0, sl_col, pair_i, pair_kind, dl_col,
                                     cptr, contrib);
  if (!ok) {
    atomicExch(overflow, 1);
    return;
  }
  if (!FILL) {
    atomicAdd(ncand, (unsigned long long)nu);
    slcnt[i] = nsl;
    dlcnt[i] = ndl;
    ecnt[i] = nde;
  }
}

}  // namespace

namespace {

std::atomic<int> g_device_topology_min{65536};

// out[0..n) = exclusive prefix sums of in[0..n), on st.
int exclusive_scan(const int* in, int* out, int n, cudaStream_t st)
{
  if (n <= 0) return EB_OK;
  const int nb = (n + kScanBlock - 1) / kScanBlock;
  TmpBuf sums(st), offs(st);
  EB_CHECK(sums.alloc(sizeof(int) * nb));
  scan_block_kernel<<<nb, kScanThreads, 0, st>>>(in, n, out, sums.as<int>());
  EB_CUDA(cudaGetLastError());
  if (nb > 1) {
    EB_CHECK(offs.alloc(sizeof(int) * nb));
    EB_CHECK(exclusive_scan(sums.as<int>(), offs.as<int>(), nb, st));
    scan_add_kernel<<<(n + 255) / 256, 256, 0, st>>>(out, n, offs.as<int>());
    EB_CUDA(cudaGetLastError());
  }
  return EB_OK;
}

// ptr[0..n] = row offsets of the counts cnt[0..n).
int row_offsets(const int* cnt, int* ptr, int n, cudaStream_t st)
{
  EB_CHECK(exclusive_scan(cnt, ptr, n, st));
  copy_total_kernel<<<1, 32, 0, st>>>(cnt, ptr, n, ptr);
  EB_CUDA(cudaGetLastError());
  return EB_OK;
}

template <typename T>
int download(std::vector<T>& v, const DevBuf& src, size_t n)
{
  v.resize(n);
  return copy_d2h(v.data(), src.p, sizeof(T) * n);
}

}  // namespace

int device_topology_min() { return g_device_topology_min.load(std::memory_order_relaxed); }

int device_topology(HostMesh* h, bool* done)
{
  *done = false;
  const int ne = h->ne, nv = h->nv;
  cudaStream_t st = nullptr;
  EB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
  } guard{st};
  // outputs (owning, freed at return); scratch is stream-ordered on st
  DevBuf sl_rowptr, dl_rowptr, sl_col, pair_i, pair_kind, dl_col, cptr, contrib;
  long long counts[3] = {0, 0, 0};
  unsigned long long ncand = 0;
  {
    TmpBuf d_elems(st), vcount(st), vptr(st), cursor(st), vtri(st), cnt(st), eptr(st), flags(st);
    EB_CHECK(d_elems.alloc(sizeof(int) * 3 * (size_t)ne));
    // stream-ordered like the scratch it fills (pageable source: staged by the driver)
    EB_CUDA(cudaMemcpyAsync(d_elems.p, h->elems.data(), sizeof(int) * 3 * (size_t)ne, cudaMemcpyHostToDevice, st));
    EB_CHECK(vcount.alloc(sizeof(int) * nv));
    EB_CHECK(vptr.alloc(sizeof(int) * (nv + 1)));
    EB_CHECK(cursor.alloc(sizeof(int) * nv));
    EB_CHECK(vtri.alloc(sizeof(int) * 3 * (size_t)ne));
    EB_CHECK(cnt.alloc(sizeof(int) * 3 * (size_t)ne));   // per row: pairs, DL columns, DL entries
    EB_CHECK(eptr.alloc(sizeof(int) * (ne + 1)));
    EB_CHECK(flags.alloc(16));                            // [0]: candidate count (u64), [2]: overflow
    EB_CHECK(sl_rowptr.alloc(sizeof(int) * (ne + 1)));
    EB_CHECK(dl_rowptr.alloc(sizeof(int) * (ne + 1)));
    const int ncorner = 3 * ne;
    EB_CUDA(cudaMemsetAsync(vcount.p, 0, sizeof(int) * nv, st));
    EB_CUDA(cudaMemsetAsync(flags.p, 0, 16, st));
    vertex_count_kernel<<<(ncorner + 255) / 256, 256, 0, st>>>(d_elems.as<int>(), ncorner, vcount.as<int>());
    EB_CUDA(cudaGetLastError());
    EB_CHECK(row_offsets(vcount.as<int>(), vptr.as<int>(), nv, st));
    EB_CUDA(cudaMemcpyAsync(cursor.p, vptr.p, sizeof(int) * nv, cudaMemcpyDeviceToDevice, st));
    vertex_fill_kernel<<<(ncorner + 255) / 256, 256, 0, st>>>(d_elems.as<int>(), ncorner, cursor.as<int>(),
                                                             vtri.as<int>());
    EB_CUDA(cudaGetLastError());
    int* c_sl = cnt.as<int>();
    int* c_dl = c_sl + ne;
    int* c_e = c_dl + ne;
    auto* d_ncand = reinterpret_cast<unsigned long long*>(flags.p);
    int* d_over = flags.as<int>() + 2;
    const int nb = (ne + 127) / 128;
    topology_rows_kernel<false><<<nb, 128, 0, st>>>(d_elems.as<int>(), vptr.as<int>(), vtri.as<int>(), ne, c_sl, c_dl,
                                                   c_e, d_ncand, d_over, nullptr, nullptr, nullptr, nullptr,
                                                   nullptr, nullptr, nullptr, nullptr, nullptr);
    EB_CUDA(cudaGetLastError());
    EB_CHECK(row_offsets(c_sl, sl_rowptr.as<int>(), ne, st));
    EB_CHECK(row_offsets(c_dl, dl_rowptr.as<int>(), ne, st));
    EB_CHECK(row_offsets(c_e, eptr.as<int>(), ne, st));
    EB_CUDA(cudaStreamSynchronize(st));
    int over = 0;
    EB_CHECK(copy_d2h(&over, d_over, sizeof(int)));
    if (over) return EB_OK;  // a row with more than kMaxCand candidates: the host builds the lists
    EB_CHECK(copy_d2h(&ncand, d_ncand, sizeof(ncand)));
    int tot[3];
    EB_CHECK(copy_d2h(&tot[0], sl_rowptr.as<int>() + ne, sizeof(int)));
    EB_CHECK(copy_d2h(&tot[1], dl_rowptr.as<int>() + ne, sizeof(int)));
    EB_CHECK(copy_d2h(&tot[2], eptr.as<int>() + ne, sizeof(int)));
    for (int k = 0; k < 3; k++) counts[k] = tot[k];
    EB_CHECK(sl_col.alloc(sizeof(int) * std::max(tot[0], 1)));
    EB_CHECK(pair_i.alloc(sizeof(int) * std::max(tot[0], 1)));
    EB_CHECK(pair_kind.alloc(std::max(tot[0], 1)));
    EB_CHECK(dl_col.alloc(sizeof(int) * std::max(tot[1], 1)));
    EB_CHECK(cptr.alloc(sizeof(int) * (tot[1] + 1)));
    EB_CHECK(contrib.alloc(sizeof(int) * std::max(tot[2], 1)));
    EB_CUDA(cudaMemsetAsync(cptr.p, 0, sizeof(int), st));
    topology_rows_kernel<true><<<nb, 128, 0, st>>>(d_elems.as<int>(), vptr.as<int>(), vtri.as<int>(), ne, nullptr,
                                                  nullptr, nullptr, nullptr, d_over, sl_rowptr.as<int>(),
                                                  dl_rowptr.as<int>(), eptr.as<int>(), sl_col.as<int>(),
                                                  pair_i.as<int>(), pair_kind.as<int8_t>(), dl_col.as<int>(),
                                                  cptr.as<int>(), contrib.as<int>());
    EB_CUDA(cudaGetLastError());
  }  // scratch released on st
  EB_CUDA(cudaStreamSynchronize(st));
  EB_CHECK(download(h->sl_rowptr, sl_rowptr, ne + 1));
  EB_CHECK(download(h->sl_col, sl_col, counts[0]));
  EB_CHECK(download(h->pair_i, pair_i, counts[0]));
  EB_CHECK(download(h->pair_kind, pair_kind, counts[0]));
  EB_CHECK(download(h->dl_rowptr, dl_rowptr, ne + 1));
  EB_CHECK(download(h->dl_col, dl_col, counts[1]));
  EB_CHECK(download(h->dl_contrib_ptr, cptr, counts[1] + 1));
  EB_CHECK(download(h->dl_contrib, contrib, counts[2]));
  h->far_quad_pairs = ((long long)ne * ne - (long long)ncand) * (long long)h->Q * h->Q;
  *done = true;
  return EB_OK;
}

}  // namespace eb

int eb_set_device_topology_min(int nelems)
{
  if (nelems < 0) return eb::set_error(EB_ERR_INVALID, "the device-topology threshold must be >= 0");
  eb::g_device_topology_min.store(nelems, std::memory_order_relaxed);
  return EB_OK;
}

int eb_get_device_topology_min(int* nelems)
{
  if (!nelems) return eb::set_error(EB_ERR_INVALID, "null argument");
  *nelems = eb::device_topology_min();
  return EB_OK;
}
