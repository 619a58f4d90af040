// Device-resident mesh, FP64 Sauter-Schwab near field and the apply pipeline
// (prep -> far field -> finalize), plus the C ABI of include/easybem_gpu.h.
#include "engine.h"
#include "farfield_sym.h"
#include "farfield_tc.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iterator>
#include <map>
#include <mutex>
#include <string>

#include "pairs.h"

namespace eb {

static thread_local std::string g_last_error;

int set_error(int status, const std::string& msg)
{
  g_last_error = msg;
  return status;
}

const char* last_error() { return g_last_error.c_str(); }

// ---------------------------------------------------------------------------
// Device memory behind DevBuf: the device's stream-ordered pool, kept warm.
//
// cudaMalloc and cudaFree, called from a thread that prepares a mesh while
// other threads keep the GPU busy, were measured to wait for running kernels
// (cudaFree for the whole device); allocations from a pool that keeps its
// memory (release threshold at the maximum) return in about 0.1 ms. Every
// host thread allocates and frees on its own non-blocking stream per device
// and synchronises after allocating, so a block is usable on any stream at
// once; it is freed only once no queued work uses it (every caller
// synchronises first).

namespace {

constexpr int kPoolDevices = 64;

cudaStream_t pool_stream(int dev)
{
  struct Streams {
    cudaStream_t st[kPoolDevices] = {};
    ~Streams()
    {
      for (int d = 0; d < kPoolDevices; d++)
        if (st[d]) cudaStreamDestroy(st[d]);
    }
  };
  static thread_local Streams s;
  if (dev < 0 || dev >= kPoolDevices) return nullptr;
  if (!s.st[dev]) {
    static std::mutex mu;
    static bool warm[kPoolDevices] = {};
    {
      std::lock_guard<std::mutex> g(mu);
      if (!warm[dev]) {  // keep freed memory in the pool for later allocations
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
          uint64_t thr = UINT64_MAX;
          cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        warm[dev] = true;
      }
    }
    if (cudaStreamCreateWithFlags(&s.st[dev], cudaStreamNonBlocking) != cudaSuccess) s.st[dev] = nullptr;
  }
  return s.st[dev];
}

// Pinned staging memory of the calling thread for set-up copies (freed when
// the thread exits).
constexpr size_t kStageChunk = size_t(16) << 20;

struct Staging {
  void* p = nullptr;
  ~Staging()
  {
    if (p) cudaFreeHost(p);
  }
};

void* staging_buffer()
{
  static thread_local Staging s;
  if (!s.p && cudaMallocHost(&s.p, kStageChunk) != cudaSuccess) {
    cudaGetLastError();
    s.p = nullptr;
  }
  return s.p;
}

}  // namespace

// Set-up copies between pageable host memory and the device: staged through
// the thread's pinned buffer in chunks and issued with cudaMemcpyAsync on the
// thread's non-blocking stream, then waited for. A synchronous cudaMemcpy
// from pageable memory goes through the legacy default stream and the
// driver's own staging; mesh preparation threads that copy while other
// threads keep the GPU busy were measured to spend ~0.3 s per mesh in it.
int copy_h2d(void* dst, const void* src, size_t bytes)
{
  if (bytes == 0) return EB_OK;
  int dev = 0;
  EB_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = pool_stream(dev);
  unsigned char* stage = static_cast<unsigned char*>(staging_buffer());
  if (!st || !stage) return set_error(EB_ERR_CUDA, "cannot create the staging stream or pinned buffer");
  for (size_t off = 0; off < bytes; off += kStageChunk) {
    const size_t n = std::min(kStageChunk, bytes - off);
    std::memcpy(stage, static_cast<const unsigned char*>(src) + off, n);
    EB_CUDA(cudaMemcpyAsync(static_cast<unsigned char*>(dst) + off, stage, n, cudaMemcpyHostToDevice, st));
    EB_CUDA(cudaStreamSynchronize(st));
  }
  return EB_OK;
}

int copy_d2h(void* dst, const void* src, size_t bytes)
{
  if (bytes == 0) return EB_OK;
  int dev = 0;
  EB_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = pool_stream(dev);
  unsigned char* stage = static_cast<unsigned char*>(staging_buffer());
  if (!st || !stage) return set_error(EB_ERR_CUDA, "cannot create the staging stream or pinned buffer");
  for (size_t off = 0; off < bytes; off += kStageChunk) {
    const size_t n = std::min(kStageChunk, bytes - off);
    EB_CUDA(cudaMemcpyAsync(stage, static_cast<const unsigned char*>(src) + off, n, cudaMemcpyDeviceToHost, st));
    EB_CUDA(cudaStreamSynchronize(st));
    std::memcpy(static_cast<unsigned char*>(dst) + off, stage, n);
  }
  return EB_OK;
}

int memset_sync(void* dst, int value, size_t bytes)
{
  if (bytes == 0) return EB_OK;
  int dev = 0;
  EB_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = pool_stream(dev);
  if (!st) return set_error(EB_ERR_CUDA, "cannot create the staging stream");
  EB_CUDA(cudaMemsetAsync(dst, value, bytes, st));
  EB_CUDA(cudaStreamSynchronize(st));
  return EB_OK;
}

void DevBuf::release()
{
  if (p && owns) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    cudaStream_t st = pool_stream(dev);
    if (st) cudaFreeAsync(p, st);
    if (cur != dev) cudaSetDevice(cur);
  }
  p = nullptr;
  bytes = 0;
  owns = true;
}

int DevBuf::alloc(size_t n)
{
  if (n <= bytes && p) return EB_OK;
  release();
  if (n == 0) n = 16;
  cudaGetDevice(&dev);
  cudaStream_t st = pool_stream(dev);
  if (!st) return set_error(EB_ERR_CUDA, "cannot create an allocation stream");
  // the pool grows in steps of at least 1 GiB: each growth costs about as much
  // as a large cudaMalloc, so many small requests should not each pay one
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    if (reserved - used < n + (n >> 3)) {
      void* grow = nullptr;
      const size_t step = std::max<size_t>(n + (n >> 3), size_t(1) << 30);
      if (cudaMallocAsync(&grow, step, st) == cudaSuccess) cudaFreeAsync(grow, st);
      else cudaGetLastError();  // no room for the step: allocate just n below
    }
  }
  cudaError_t e = cudaMallocAsync(&p, n, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    p = nullptr;
    return set_error(e == cudaErrorMemoryAllocation ? EB_ERR_NOMEM : EB_ERR_CUDA,
                     std::string("cudaMallocAsync(") + std::to_string(n) + "): " + cudaGetErrorString(e));
  }
  bytes = n;
  return EB_OK;
}

int devmem_trim(int device)
{
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return EB_OK;
  int cur = 0;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  cudaDeviceSynchronize();
  cudaMemPoolTrimTo(pool, 0);
  cudaSetDevice(cur);
  return EB_OK;
}

size_t devmem_cached_bytes(int device)
{
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return 0;
  uint64_t reserved = 0, used = 0;
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  return reserved > used ? (size_t)(reserved - used) : 0;
}

int TmpBuf::alloc(size_t n)
{
  release();
  if (n == 0) n = 16;
  cudaError_t e = cudaMallocAsync(&p, n, st);
  if (e != cudaSuccess) {
    p = nullptr;
    return set_error(e == cudaErrorMemoryAllocation ? EB_ERR_NOMEM : EB_ERR_CUDA,
                     std::string("cudaMallocAsync(") + std::to_string(n) + "): " + cudaGetErrorString(e));
  }
  bytes = n;
  return EB_OK;
}

template <typename T>
static int upload(DevBuf& b, const std::vector<T>& v)
{
  EB_CHECK(b.alloc(sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty()) EB_CHECK(copy_h2d(b.p, v.data(), sizeof(T) * v.size()));
  return EB_OK;
}

template <typename T>
static int upload(TmpBuf& b, const std::vector<T>& v)
{
  EB_CHECK(b.alloc(sizeof(T) * std::max<size_t>(v.size(), 1)));
  if (!v.empty()) EB_CUDA(cudaMemcpyAsync(b.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, b.st));
  return EB_OK;
}

Mesh::~Mesh()
{
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  if (ev2) cudaEventDestroy(ev2);
}

// ---------------------------------------------------------------------------
// Near field: one thread per near pair computes the FP64 Sauter-Schwab SL
// value and three DL weights; DL weights landing on the same (row, vertex)
// are then summed in ascending pair order.

__global__ void near_values_kernel(Quadrature q, const double* __restrict__ nodes, const int* __restrict__ elems,
                                   const int* __restrict__ pi, const int* __restrict__ pj, int npairs,
                                   double* __restrict__ slv, double* __restrict__ dle)
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
  double s, K[3];
  near_pair_values(q, g, Pi, Pj, &s, K);
  slv[p] = s;
  dle[3 * p] = K[0];
  dle[3 * p + 1] = K[1];
  dle[3 * p + 2] = K[2];
}

__global__ void dl_gather_kernel(const int* __restrict__ cptr, const int* __restrict__ contrib,
                                 const double* __restrict__ dle, int nslots, double* __restrict__ out)
{
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslots) return;
  double acc = 0.0;
  for (int k = cptr[s]; k < cptr[s + 1]; k++) acc += dle[contrib[k]];
  out[s] = acc;
}

// ---------------------------------------------------------------------------

static int build_static(Mesh* m)
{
  HostMesh& h = m->h;
  const int ne = h.ne, Q = h.Q, K = h.K;
  const int ntt = (h.nitems + kTT - 1) / kTT;
  std::vector<float4> pos32((size_t)ne * Q), tgt32((size_t)h.nitems * K), tgtw32((size_t)h.nitems * K);
  std::vector<dq> tgtw64((size_t)h.nitems * K);
  std::vector<dq> pos64((size_t)ne * Q), trin(ne), tgt64((size_t)h.nitems * K), tcent(h.nitems), tnrm(h.nitems),
      ccent(h.ncells), snrm(ne), ttile(ntt), twarp((h.nitems + kWarpItems - 1) / kWarpItems), splane64(ne);
  std::vector<float4> splane32(ne);
  std::vector<double> wjtab((size_t)ne * Q);
  std::vector<int4> svid(ne), tvid(h.nitems);
  std::vector<double> bary(2 * (size_t)Q);
  for (int b = 0; b < Q; b++) {
    bary[2 * b] = h.quad.tx[b];
    bary[2 * b + 1] = h.quad.ty[b];
  }
  auto vertex = [&](int s, int k) {
    const int v = h.elems[3 * h.perm[s] + k];
    return mk3(h.nodes[3 * v], h.nodes[3 * v + 1], h.nodes[3 * v + 2]);
  };
  // cell bounding spheres (centre = mean centroid, radius over all vertices)
  for (int c = 0; c < h.ncells; c++) {
    const d3 cc = mk3(h.cell_center[3 * c], h.cell_center[3 * c + 1], h.cell_center[3 * c + 2]);
    double r2 = 0.0;
    for (int s = c * kCell; s < std::min(ne, (c + 1) * kCell); s++)
      for (int k = 0; k < 3; k++) r2 = std::max(r2, dot3(vertex(s, k) - cc, vertex(s, k) - cc));
    ccent[c] = dq{cc.x, cc.y, cc.z, std::sqrt(r2) * (1.0 + 1e-12)};
  }
  for (int s = 0; s < ne; s++) {
    d3 P[3];
    for (int k = 0; k < 3; k++) P[k] = vertex(s, k);
    const int* f = &h.elems[3 * h.perm[s]];
    const d3 w = P[1] - P[0], z = P[2] - P[0];
    const d3 n = cross3(w, z);
    const double J = std::sqrt(dot3(n, n));
    trin[s] = dq{n.x / J, n.y / J, n.z / J, J};
    const d3 nu = (1.0 / J) * n;
    snrm[s] = dq{nu.x, nu.y, nu.z, dot3(P[0], nu)};
    svid[s] = make_int4(f[0], f[1], f[2], 0);
    const int cell = s / kCell;
    const d3 cc = mk3(ccent[cell].x, ccent[cell].y, ccent[cell].z);
    const double hp = dot3(P[0] - cc, nu);
    splane64[s] = dq{nu.x, nu.y, nu.z, hp};
    splane32[s] = make_float4((float)nu.x, (float)nu.y, (float)nu.z, (float)hp);
    for (int b = 0; b < Q; b++) {
      const d3 y = P[0] + h.quad.tx[b] * w + h.quad.ty[b] * z;
      wjtab[(size_t)s * Q + b] = h.quad.tw[b] * J;
      const d3 yr = y - cc;
      pos64[(size_t)s * Q + b] = dq{-2.0 * yr.x, -2.0 * yr.y, -2.0 * yr.z, dot3(yr, yr)};
      const float fx = (float)yr.x, fy = (float)yr.y, fz = (float)yr.z;
      const double y2 = (double)fx * fx + (double)fy * fy + (double)fz * fz;
      pos32[(size_t)s * Q + b] = make_float4(-2.0f * fx, -2.0f * fy, -2.0f * fz, (float)y2);
    }
    const d3 cen = (1.0 / 3.0) * (P[0] + P[1] + P[2]);
    for (int ch = 0; ch < h.nchunk; ch++) {
      const int item = s * h.nchunk + ch;
      tcent[item] = dq{cen.x, cen.y, cen.z, 0.0};
      tnrm[item] = dq{nu.x, nu.y, nu.z, 0.0};
      tvid[item] = svid[s];
      for (int a = 0; a < K; a++) {
        const int pa = ch * K + a;
        const int pp = std::min(pa, Q - 1);
        const double wa = pa < Q ? h.quad.tw[pp] : 0.0;
        const d3 x = P[0] + h.quad.tx[pp] * w + h.quad.ty[pp] * z;
        const d3 xr = x - cen;
        tgt64[(size_t)item * K + a] = dq{xr.x, xr.y, xr.z, wa};
        tgt32[(size_t)item * K + a] = make_float4((float)xr.x, (float)xr.y, (float)xr.z, (float)wa);
        // P1 test weights w_a (1 - xi - eta, xi, eta) in the triangle's vertex order
        const double ph0 = 1.0 - h.quad.tx[pp] - h.quad.ty[pp], ph1 = h.quad.tx[pp], ph2 = h.quad.ty[pp];
        tgtw64[(size_t)item * K + a] = dq{wa * ph0, wa * ph1, wa * ph2, 0.0};
        tgtw32[(size_t)item * K + a] = make_float4((float)(wa * ph0), (float)(wa * ph1), (float)(wa * ph2), 0.0f);
      }
    }
  }
  // bounding spheres over the triangles of n consecutive target items: per
  // tile of kTT (the tensor-core kernel's test) and per warp of kWarpItems
  // (the CUDA-core kernel's: a tighter sphere leaves fewer cells "near")
  auto item_spheres = [&](int n, std::vector<dq>& out) {
    for (size_t t = 0; t < out.size(); t++) {
      const int i0 = (int)t * n, i1 = std::min(h.nitems, i0 + n);
      d3 c = mk3(0, 0, 0);
      for (int it = i0; it < i1; it++) c = c + mk3(tcent[it].x, tcent[it].y, tcent[it].z);
      c = (1.0 / (i1 - i0)) * c;
      double r2 = 0.0;
      for (int it = i0; it < i1; it++)
        for (int k = 0; k < 3; k++) {
          const d3 v = vertex(it / h.nchunk, k);
          r2 = std::max(r2, dot3(v - c, v - c));
        }
      out[t] = dq{c.x, c.y, c.z, std::sqrt(r2) * (1.0 + 1e-12)};
    }
  };
  item_spheres(kTT, ttile);
  item_spheres(kWarpItems, twarp);
  // how the warp x cell blocks split under the CUDA-core kernel's separation test
  {
    long long fc = 0, nc = 0;
    for (size_t t = 0; t < twarp.size(); t++) {
      const long long nt = std::min<long long>(h.nitems, (long long)(t + 1) * kWarpItems) - (long long)t * kWarpItems;
      for (int c = 0; c < h.ncells; c++) {
        const long long ns = std::min(ne, (c + 1) * kCell) - c * kCell;
        const double dx = ccent[c].x - twarp[t].x, dy = ccent[c].y - twarp[t].y, dz = ccent[c].z - twarp[t].z;
        const double rr = kFarRatio * (ccent[c].w + twarp[t].w);
        (dx * dx + dy * dy + dz * dz > rr * rr ? fc : nc) += nt * ns;
      }
    }
    h.far_cell_tri_pairs = fc;
    h.near_cell_tri_pairs = nc;
  }
  // one allocation and one copy for all static tables (a mesh set-up that
  // runs beside other GPU work pays the per-call latency of the runtime once)
  struct Part {
    DevBuf* dst;
    const void* src;
    size_t bytes;
  };
  auto part = [](DevBuf& d, const auto& v) {
    return Part{&d, (const void*)v.data(), sizeof(v[0]) * v.size()};
  };
  const Part parts[] = {part(m->pos32, pos32),   part(m->pos64, pos64),     part(m->wj, wjtab),
                        part(m->trin, trin),     part(m->svid, svid),       part(m->perm, h.perm),
                        part(m->iperm, h.iperm), part(m->bary, bary),       part(m->tgt32, tgt32),
                        part(m->tgt64, tgt64),   part(m->tgtw32, tgtw32),   part(m->tgtw64, tgtw64),
                        part(m->tcent, tcent),   part(m->tnrm, tnrm),       part(m->snrm, snrm),
                        part(m->tvid, tvid),     part(m->ccent, ccent),     part(m->ttile, ttile),
                        part(m->twarp, twarp),
                        part(m->splane32, splane32), part(m->splane64, splane64)};
  auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t total = 0;
  for (const Part& q : parts) total += align(std::max<size_t>(q.bytes, 16));
  std::vector<unsigned char> staging(total, 0);
  size_t off = 0;
  for (const Part& q : parts) {
    if (q.bytes) std::memcpy(staging.data() + off, q.src, q.bytes);
    off += align(std::max<size_t>(q.bytes, 16));
  }
  const auto ta = std::chrono::steady_clock::now();
  EB_CHECK(m->arena.alloc(total));
  const auto tb = std::chrono::steady_clock::now();
  EB_CHECK(copy_h2d(m->arena.p, staging.data(), total));
  const auto tc = std::chrono::steady_clock::now();
  m->setup_s[3] = std::chrono::duration<double>(tb - ta).count();
  m->setup_s[4] = std::chrono::duration<double>(tc - tb).count();
  off = 0;
  for (const Part& q : parts) {
    const size_t n = align(std::max<size_t>(q.bytes, 16));
    q.dst->view(static_cast<unsigned char*>(m->arena.p) + off, std::max<size_t>(q.bytes, 16));
    off += n;
  }
  return EB_OK;
}

static int build_near(Mesh* m)
{
  HostMesh& h = m->h;
  const int npairs = (int)h.sl_col.size();
  m->npairs = npairs;
  EB_CHECK(upload(m->sl_rowptr, h.sl_rowptr));
  EB_CHECK(upload(m->sl_col, h.sl_col));
  EB_CHECK(upload(m->dl_rowptr, h.dl_rowptr));
  EB_CHECK(upload(m->dl_col, h.dl_col));
  EB_CHECK(m->sl_val.alloc(sizeof(double) * std::max(npairs, 1)));
  const int nslots = (int)h.dl_col.size();
  EB_CHECK(m->dl_val.alloc(sizeof(double) * std::max(nslots, 1)));
  // a private stream with stream-ordered temporaries: mesh set-up overlaps
  // work that other threads run on the GPU and never waits for the device
  cudaStream_t st = nullptr;
  EB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = EB_OK;
  cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
  {
    TmpBuf d_nodes(st), d_elems(st), d_pi(st), d_pj(st), d_dle(st), d_cptr(st), d_contrib(st);
    rc = upload(d_nodes, h.nodes);
    if (rc == EB_OK) rc = upload(d_elems, h.elems);
    if (rc == EB_OK) rc = upload(d_pi, h.pair_i);
    if (rc == EB_OK) rc = upload(d_pj, h.sl_col);
    if (rc == EB_OK) rc = upload(d_cptr, h.dl_contrib_ptr);
    if (rc == EB_OK) rc = upload(d_contrib, h.dl_contrib);
    if (rc == EB_OK) rc = d_dle.alloc(sizeof(double) * 3 * std::max(npairs, 1));
    if (rc == EB_OK) {
      if (npairs > 0)
        near_values_kernel<<<(npairs + 127) / 128, 128, 0, st>>>(h.quad, d_nodes.as<double>(), d_elems.as<int>(),
                                                                 d_pi.as<int>(), d_pj.as<int>(), npairs,
                                                                 m->sl_val.as<double>(), d_dle.as<double>());
      if (nslots > 0)
        dl_gather_kernel<<<(nslots + 255) / 256, 256, 0, st>>>(d_cptr.as<int>(), d_contrib.as<int>(),
                                                              d_dle.as<double>(), nslots, m->dl_val.as<double>());
      e1 = cudaGetLastError();
    }
  }  // temporaries released on st
  e2 = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  EB_CHECK(rc);
  EB_CUDA(e1);
  EB_CUDA(e2);
  return EB_OK;
}

// Source triangles per shared-memory tile for a variant (whole cells when
// they fit; large quadrature rules fall back to smaller tiles).
int src_tile_for(int Q, bool fp32, int nsl, int nd)
{
  const size_t per_tri = far_smem_bytes(1, Q, rec_slots(nsl, nd), fp32);
  const size_t budget = 48 * 1024;
  int ts = (int)std::min<size_t>(kTS, budget / per_tri);
  return std::max(ts, 1);
}

static int build_items(Mesh* m)
{
  HostMesh& h = m->h;
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const int ntt = (h.nitems + kTT - 1) / kTT;
  const int want = nsm * std::max(1, m->plan.items_per_sm);  // work items for balance across persistent CTAs
  int nsplit = std::max(1, std::min(h.ncells, (want + ntt - 1) / ntt));
  const int cells_per = (h.ncells + nsplit - 1) / nsplit;
  nsplit = (h.ncells + cells_per - 1) / cells_per;
  std::vector<WorkItem> items;
  items.reserve((size_t)ntt * nsplit);
  for (int sp = 0; sp < nsplit; sp++)
    for (int t = 0; t < ntt; t++)
      items.push_back(WorkItem{0, t * kTT, sp * cells_per, std::min(h.ncells, (sp + 1) * cells_per), sp});
  m->plan.nsplit = nsplit;
  m->nitems_work = (int)items.size();
  m->items_host = items;
  EB_CHECK(upload(m->items, items));
  EB_CHECK(m->counter.alloc(sizeof(int)));
  return EB_OK;
}

int mesh_set_plan(Mesh* m, int items_per_sm, int tile)
{
  if (items_per_sm < 1 || items_per_sm > 4096 || tile < 0 || tile > kTS)
    return set_error(EB_ERR_INVALID, "plan needs 1 <= items_per_sm <= 4096 and 0 <= tile <= " + std::to_string(kTS));
  // no device-wide synchronisation here: it would break a CUDA graph capture
  // running in another thread; the caller guarantees no work on m is in flight
  m->plan.items_per_sm = items_per_sm;
  m->plan.tile = tile;
  // per-variant descriptors and the scratch sized for the old split go away
  for (auto& v : m->variants) {
    v.desc.release();
    v.grid = 0;
  }
  m->tc_var.desc.release();
  m->tc_var.grid = 0;
  m->sym_var.desc.release();
  m->sym_var.grid = 0;
  m->rec.release();
  m->partial.release();
  return build_items(m);
}

int mesh_create(int nv, const double* nodes, int ne, const int* elems1, int order, Mesh** out)
{
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return set_error(EB_ERR_CUDA, std::string("no CUDA device: ") + cudaGetErrorString(e));
  Mesh* m = new Mesh();
  cudaGetDevice(&m->device);
  using clk = std::chrono::steady_clock;
  const auto t0 = clk::now();
  // large meshes build the near-pair lists on the GPU (host_topology otherwise,
  // and when a row has too many candidates for the device pass)
  const bool dev_topology = ne >= device_topology_min();
  int st = prepare_host_mesh(nv, nodes, ne, elems1, order, &m->h, !dev_topology);
  if (st == EB_OK && dev_topology) {
    bool done = false;
    st = device_topology(&m->h, &done);
    if (st == EB_OK && !done) host_topology(&m->h);
    m->h.topology_on_device = done;
  }
  if (st == EB_OK) tuned_plan_for(m->h, &m->plan.items_per_sm, &m->plan.tile);
  const auto t1 = clk::now();
  if (st == EB_OK) st = build_static(m);
  const auto t2 = clk::now();
  if (st == EB_OK) st = build_near(m);
  const auto t3 = clk::now();
  if (st == EB_OK) st = build_items(m);
  const auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
  m->setup_s[0] = sec(t0, t1);
  m->setup_s[1] = sec(t1, t2);
  m->setup_s[2] = sec(t2, t3);
  if (st != EB_OK) {
    delete m;
    return st;
  }
  *out = m;
  return EB_OK;
}

ApplyArgs mesh_apply_args(const Mesh* m, bool fp32, void* rec, const double* partial, const double* t, int tstride,
                          const double* u, double* v, int vstride, double* q)
{
  const HostMesh& h = m->h;
  ApplyArgs A;
  A.pos = fp32 ? m->pos32.p : m->pos64.p;
  A.wj = m->wj.as<double>();
  A.svid = m->svid.as<int4>();
  A.perm = m->perm.as<int>();
  A.bary = m->bary.as<double>();
  A.t = t;
  A.tstride = tstride;
  A.u = u;
  A.ustride = h.nv;  // DL columns [nd][nnodes]
  A.rec = rec;
  A.ne = h.ne;
  A.Q = h.Q;
  A.nchunk = h.nchunk;
  A.nsplit = m->plan.nsplit;
  A.nitems = h.nitems;
  A.iperm = m->iperm.as<int>();
  A.trin = m->trin.as<dq>();
  A.partial = partial;
  A.sl_rowptr = m->sl_rowptr.as<int>();
  A.sl_col = m->sl_col.as<int>();
  A.sl_val = m->sl_val.as<double>();
  A.dl_rowptr = m->dl_rowptr.as<int>();
  A.dl_col = m->dl_col.as<int>();
  A.dl_val = m->dl_val.as<double>();
  A.v = v;
  A.vstride = vstride;
  A.q = q;
  A.qstride = h.ne;  // DL outputs [nd][nelems]
  A.active = nullptr;
  return A;
}

FarMeshDesc mesh_far_desc(const Mesh* m, bool fp32, int nsl, int nd, void* rec, double* partial)
{
  const HostMesh& h = m->h;
  FarMeshDesc desc;
  desc.tgt32 = m->tgt32.as<float4>();
  desc.tgt64 = m->tgt64.as<dq>();
  desc.tgtw32 = m->tgtw32.as<float4>();
  desc.tgtw64 = m->tgtw64.as<dq>();
  desc.tcent = m->tcent.as<dq>();
  desc.tnrm = m->tnrm.as<dq>();
  desc.snrm = m->snrm.as<dq>();
  desc.splane32 = m->splane32.as<float4>();
  desc.splane64 = m->splane64.as<dq>();
  desc.tvid = m->tvid.as<int4>();
  desc.rec = rec;
  desc.svid = m->svid.as<int4>();
  desc.ccent = m->ccent.as<dq>();
  desc.ttile = m->ttile.as<dq>();
  desc.twarp = m->twarp.as<dq>();
  desc.partial = partial;
  desc.nitems = h.nitems;
  desc.ne = h.ne;
  desc.Q = h.Q;
  desc.nsplit = m->plan.nsplit;
  desc.src_tile = src_tile_for(h.Q, fp32, nsl, nd);
  if (m->plan.tile > 0) desc.src_tile = std::min(desc.src_tile, m->plan.tile);
  // the FP32 far kernel stages source triangles in pairs
  if (fp32) desc.src_tile = std::max(2, desc.src_tile & ~1);
  desc.active = nullptr;
  return desc;
}

size_t sym_slot_bytes(const HostMesh& h, int nout)
{
  const long long nsplit = (h.nitems + kTT - 1) / kTT + 1;  // at most one slot per tile, plus one
  return sizeof(double) * (size_t)nout * (size_t)nsplit * (size_t)h.nitems;
}

bool sym_eligible(const Mesh* m, bool fp32, int nsl, int nd, bool fp64_internal)
{
  // the partial slots take (nsl + nd) ne^2 / 128 * 8 bytes: meshes whose slots
  // would pass kSymMaxSlotBytes keep the ordered-pair kernels (whose slots
  // grow with the work split, not with ne^2)
  const bool engine = (m->plan.engine == 2 && (fp32 || fp64_internal)) || m->plan.engine == 3;
  return engine && far_sym_variant(fp32, nsl, nd) && m->h.Q == kSymRule && m->h.K == kSymRule &&
         m->h.nchunk == 1 && sym_slot_bytes(m->h, nsl + nd) <= kSymMaxSlotBytes;
}

long long mesh_far_slots(const Mesh* m, bool fp32, int nsl, int nd)
{
  if (sym_eligible(m, fp32, nsl, nd)) {
    const int r = far_sym_cells_per_item(kSymCellsPerItem);
    long long n = 0;
    for (int s = 0; s < m->h.ne; s++) n += sym_row_slots(s, m->h.ne, r);
    return n;
  }
  return (long long)m->plan.nsplit * m->h.nitems;
}

// The symmetric far field: work list once per mesh, partial slots for the
// widest variant used so far (grown when a wider one comes; the finalize
// reads only the slots each row's items write, so they need no zeroing), the
// descriptor once per scratch allocation, then the persistent kernel.
static int sym_far_apply(Mesh* m, bool fp32, int nsl, int nd, cudaStream_t st)
{
  const HostMesh& h = m->h;
  if (!m->sym_items.p) {
    m->sym_nsplit = far_sym_items(h.nitems, h.ncells, kSymCellsPerItem, m->sym_items_host);
    m->sym_nitems = (int)m->sym_items_host.size();
    EB_CHECK(upload(m->sym_items, m->sym_items_host));
  }
  const size_t bytes = sizeof(double) * (size_t)(nsl + nd) * (size_t)m->sym_nsplit * h.nitems;
  if (m->sym_partial.bytes < bytes) {
    m->sym_partial.release();
    m->sym_var.desc.release();
    EB_CHECK(m->sym_partial.alloc(bytes));
  }
  if (!m->sym_var.desc.p) {
    FarMeshDesc desc = mesh_far_desc(m, true, 1, 1, m->rec.p, m->sym_partial.as<double>());
    desc.nsplit = m->sym_nsplit;
    desc.src_tile = kTS;
    EB_CHECK(m->sym_var.desc.alloc(sizeof(FarMeshDesc)));
    EB_CHECK(copy_h2d(m->sym_var.desc.p, &desc, sizeof desc));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    m->sym_var.grid = nsm;  // times the kernel's CTAs per SM, per precision below
    m->sym_var.src_tile = kTS;
  }
  const int occ = std::max(1, far_sym_occupancy(fp32, nsl, nd));
  const int grid = std::min(m->sym_var.grid * occ, std::max(1, m->sym_nitems));
  m->sym_var.smem = far_sym_smem_bytes(fp32, nsl, nd);
  EB_CUDA(cudaMemsetAsync(m->counter.p, 0, sizeof(int), st));
  if (m->profile) EB_CUDA(cudaEventRecord(m->ev0, st));
  EB_CUDA(far_sym_launch(fp32, nsl, nd, m->sym_var.desc.as<FarMeshDesc>(), m->sym_items.as<WorkItem>(),
                         m->sym_nitems, m->counter.as<int>(), grid, st));
  m->plan.grid = grid;
  m->tc_used = false;
  m->sym_used = true;
  return EB_OK;
}

bool tc_eligible(const Mesh* m, bool fp32, int nsl, int nd)
{
  return m->plan.engine == 1 && fp32 && nsl == 1 && nd == 1 && m->h.Q == kTcRule && m->h.K == kTcRule;
}

// The tensor-core far field: static operands once per mesh, then per apply
// the DL operand and charges from the records, the persistent kernel.
int ensure_tc_static(Mesh* m)
{
  if (m->tc_static_ready) return EB_OK;
  const HostMesh& h = m->h;
  EB_CHECK(m->tc_bd2.alloc(far_tc_operand_bytes(h.ncells)));
  int dev = 0;
  EB_CUDA(cudaGetDevice(&dev));
  cudaStream_t st = pool_stream(dev);
  if (!st) return set_error(EB_ERR_CUDA, "cannot create the staging stream");
  EB_CUDA(far_tc_prep_static(h.ne, h.ncells, m->pos32.as<float4>(), m->tc_bd2.as<float4>(), st));
  EB_CUDA(cudaStreamSynchronize(st));
  m->tc_static_ready = true;
  return EB_OK;
}

static int tc_far_apply(Mesh* m, cudaStream_t st)
{
  const HostMesh& h = m->h;
  EB_CHECK(ensure_tc_static(m));
  if (!m->tc_err.p) {  // the single-mesh apply's DL operand, charges and error flag
    EB_CHECK(m->tc_be.alloc(far_tc_operand_bytes(h.ncells)));
    EB_CHECK(m->tc_charge.alloc(far_tc_charge_bytes(h.ncells)));
    EB_CHECK(m->tc_err.alloc(sizeof(int)));
    EB_CHECK(memset_sync(m->tc_err.p, 0, sizeof(int)));
  }
  if (!m->tc_var.desc.p) {  // (re)built after a plan change: scratch pointers and split
    FarMeshDesc desc = mesh_far_desc(m, true, 1, 1, m->rec.p, m->partial.as<double>());
    desc.tc_bd2 = m->tc_bd2.as<float4>();
    desc.tc_be = m->tc_be.as<float4>();
    desc.tc_charge = m->tc_charge.as<float>();
    EB_CHECK(m->tc_var.desc.alloc(sizeof(FarMeshDesc)));
    EB_CHECK(copy_h2d(m->tc_var.desc.p, &desc, sizeof desc));
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    m->tc_var.grid = std::min(nsm, std::max(1, m->nitems_work));
  }
  EB_CUDA(far_tc_prep_dl(h.ne, h.ncells, m->rec.as<float4>(), m->splane32.as<float4>(), m->tc_be.as<float4>(),
                         m->tc_charge.as<float>(), st));
  EB_CUDA(cudaMemsetAsync(m->counter.p, 0, sizeof(int), st));
  if (m->profile) EB_CUDA(cudaEventRecord(m->ev0, st));
  EB_CUDA(far_tc_launch(m->tc_var.desc.as<FarMeshDesc>(), m->items.as<WorkItem>(), m->nitems_work,
                        m->counter.as<int>(), m->tc_err.as<int>(), m->tc_var.grid, st));
  m->plan.grid = m->tc_var.grid;
  m->tc_used = true;
  return EB_OK;
}

int mesh_check_far_error(Mesh* m)
{
  if (!m->tc_used || !m->tc_err.p) return EB_OK;
  int flag = 0;
  EB_CHECK(copy_d2h(&flag, m->tc_err.p, sizeof(int)));
  if (!flag) return EB_OK;
  EB_CHECK(memset_sync(m->tc_err.p, 0, sizeof(int)));
  return set_error(EB_ERR_TIMEOUT, "tensor-core far field: a bounded wait for the tensor cores ran out");
}

int mesh_apply(Mesh* m, int precision, int nsl, int nd, const double* d_t, const double* d_u, double* d_v,
               double* d_q, cudaStream_t st)
{
  const bool dl = nd > 0;
  HostMesh& h = m->h;
  const bool fp32 = precision == EB_PREC_MIXED;
  if (precision != EB_PREC_MIXED && precision != EB_PREC_FP64)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  if (!far_variant_supported(nsl, nd)) return set_error(EB_ERR_INVALID, "unsupported operator combination");
  if ((nsl > 0 && (!d_t || !d_v)) || (dl && (!d_u || !d_q))) return set_error(EB_ERR_INVALID, "null vector");
  const int nrec = rec_slots(nsl, nd);
  // Scratch sized once for the largest variant, so device pointers captured
  // in descriptors (and in CUDA graphs) stay valid.
  if (!m->rec.p) {
    EB_CHECK(m->rec.alloc((size_t)h.ne * h.Q * kMaxRecSlots * sizeof(dq)));
    EB_CHECK(m->partial.alloc(sizeof(double) * (size_t)kMaxOutputs * m->plan.nsplit * h.nitems));
  }
  Mesh::Variant& var = m->variants[(fp32 ? 64 : 0) + nsl * 5 + nd];
  if (!var.desc.p) {
    const FarMeshDesc desc = mesh_far_desc(m, fp32, nsl, nd, m->rec.p, m->partial.as<double>());
    const size_t smem = far_smem_bytes(desc.src_tile, h.Q, nrec, fp32);
    int occ = far_occupancy(fp32, nsl, nd, h.K, h.Q, smem);
    if (occ < 1) occ = 1;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    EB_CHECK(var.desc.alloc(sizeof(FarMeshDesc)));
    EB_CHECK(copy_h2d(var.desc.p, &desc, sizeof desc));
    var.grid = std::min(nsm * occ, std::max(1, m->nitems_work));
    var.smem = smem;
    var.src_tile = desc.src_tile;
  }
  const bool sym = sym_eligible(m, fp32, nsl, nd);
  ApplyArgs A = mesh_apply_args(m, fp32, m->rec.p, m->partial.as<double>(), d_t, h.ne, d_u, d_v, h.ne, d_q);
  EB_CUDA(prep_launch(fp32, nsl, nd, A, st));
  if (m->profile && !m->ev0) {
    EB_CUDA(cudaEventCreate(&m->ev0));
    EB_CUDA(cudaEventCreate(&m->ev1));
    EB_CUDA(cudaEventCreate(&m->ev2));
  }
  if (sym) {
    EB_CHECK(sym_far_apply(m, fp32, nsl, nd, st));
    A.partial = m->sym_partial.as<double>();
    A.nsplit = m->sym_nsplit;
    A.sym_cells = far_sym_cells_per_item(kSymCellsPerItem);
  } else if (tc_eligible(m, fp32, nsl, nd)) {
    m->sym_used = false;
    EB_CHECK(tc_far_apply(m, st));
  } else {
    m->sym_used = false;
    EB_CUDA(cudaMemsetAsync(m->counter.p, 0, sizeof(int), st));
    if (m->profile) EB_CUDA(cudaEventRecord(m->ev0, st));
    EB_CUDA(far_launch(fp32, nsl, nd, h.K, h.Q, var.desc.as<FarMeshDesc>(), m->items.as<WorkItem>(), m->nitems_work,
                       m->counter.as<int>(), var.smem, var.grid, st));
    m->plan.grid = var.grid;
    m->tc_used = false;
  }
  m->plan.smem = sym ? m->sym_var.smem : var.smem;
  m->plan.src_tile = sym ? kTS : var.src_tile;
  if (m->profile) EB_CUDA(cudaEventRecord(m->ev1, st));
  EB_CUDA(finalize_launch(nsl, nd, A, st));
  if (m->profile) EB_CUDA(cudaEventRecord(m->ev2, st));
  return EB_OK;
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI

struct eb_mesh_s {
  eb::Mesh* m = nullptr;
  cudaStream_t stream = nullptr;
  std::mutex lock;  // serialises host-buffer calls on one handle
};

using eb::set_error;

eb::Mesh* eb_mesh_internal(eb_mesh handle) { return handle ? handle->m : nullptr; }

extern "C" {

const char* eb_version(void) { return "easybem-b200 0.1"; }
const char* eb_last_error(void) { return eb::last_error(); }

int eb_mesh_create(int nnodes, const double* nodes, int nelems, const int* elems, int order, eb_mesh* out)
{
  if (!out) return set_error(EB_ERR_INVALID, "null output handle");
  *out = nullptr;
  eb::Mesh* m = nullptr;
  int st = eb::mesh_create(nnodes, nodes, nelems, elems, order, &m);
  if (st != EB_OK) return st;
  eb_mesh h = new eb_mesh_s();
  h->m = m;
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    delete h;
    return set_error(EB_ERR_CUDA, std::string("cudaStreamCreate: ") + cudaGetErrorString(e));
  }
  *out = h;
  return EB_OK;
}

int eb_mesh_destroy(eb_mesh mesh)
{
  if (!mesh) return EB_OK;
  cudaSetDevice(mesh->m->device);
  if (mesh->stream) {
    cudaStreamSynchronize(mesh->stream);
    cudaStreamDestroy(mesh->stream);
  }
  delete mesh->m;
  delete mesh;
  return EB_OK;
}

int eb_mesh_info(eb_mesh mesh, int* nnodes, int* nelems, long long* near_pairs, long long* far_quad_pairs)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (nnodes) *nnodes = mesh->m->h.nv;
  if (nelems) *nelems = mesh->m->h.ne;
  if (near_pairs) *near_pairs = mesh->m->npairs;
  if (far_quad_pairs) *far_quad_pairs = mesh->m->h.far_quad_pairs;
  return EB_OK;
}

int eb_release_cached_memory(void)
{
  int n = 0;
  EB_CUDA(cudaGetDeviceCount(&n));
  for (int d = 0; d < n; d++) eb::devmem_trim(d);
  return EB_OK;
}

int eb_cached_memory_bytes(long long* bytes)
{
  if (!bytes) return set_error(EB_ERR_INVALID, "null argument");
  int dev = 0;
  EB_CUDA(cudaGetDevice(&dev));
  *bytes = (long long)eb::devmem_cached_bytes(dev);
  return EB_OK;
}

int eb_mesh_finalize_bytes(eb_mesh mesh, long long* bytes)
{
  if (!mesh || !bytes) return set_error(EB_ERR_INVALID, "null argument");
  const eb::HostMesh& h = mesh->m->h;
  const long long ne = h.ne, sl = (long long)h.sl_col.size(), dl = (long long)h.dl_col.size();
  // per row: CSR row pointers, per entry column + value + gathered density,
  // the far-field partial sums of both outputs, the two outputs
  long long b = 2 * 4 * (ne + 1) + sl * (4 + 8 + 8) + dl * (4 + 8 + 8);
  b += 2 * 8LL * eb::mesh_far_slots(mesh->m, true, 1, 1) + 2 * 8 * ne + 8 * ne /* trin */ + 4 * ne /* iperm */;
  *bytes = b;
  return EB_OK;
}

int eb_mesh_topology_on_device(eb_mesh mesh, int* on_device)
{
  if (!mesh || !on_device) return set_error(EB_ERR_INVALID, "null argument");
  *on_device = mesh->m->h.topology_on_device ? 1 : 0;
  return EB_OK;
}

int eb_mesh_cell_pairs(eb_mesh mesh, long long* far_cell_tri_pairs, long long* near_cell_tri_pairs)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (far_cell_tri_pairs) *far_cell_tri_pairs = mesh->m->h.far_cell_tri_pairs;
  if (near_cell_tri_pairs) *near_cell_tri_pairs = mesh->m->h.near_cell_tri_pairs;
  return EB_OK;
}

int eb_mesh_near_field_bytes(eb_mesh mesh, long long* spmv_bytes, long long* fold_bytes)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null argument");
  const eb::HostMesh& h = mesh->m->h;
  const long long ne = h.ne, sl = (long long)h.sl_col.size(), dl = (long long)h.dl_col.size();
  // the SL and DL near-field SpMVs: row pointers, per entry column + value +
  // gathered density, one FP64 output per row and operator
  if (spmv_bytes) *spmv_bytes = 2 * 4 * (ne + 1) + sl * (4 + 8 + 8) + dl * (4 + 8 + 8) + 2 * 8 * ne;
  // the fold of the far-field partial sums: both outputs' partial slots, the
  // row's normal/area record and its permutation entry
  if (fold_bytes) *fold_bytes = 2 * 8LL * eb::mesh_far_slots(mesh->m, true, 1, 1) + 8 * ne + 4 * ne;
  return EB_OK;
}

int eb_apply_sl_dl_device(eb_mesh mesh, int precision, const double* d_t, const double* d_u, double* d_v,
                          double* d_q, void* stream)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  const bool sl = d_t && d_v;
  const bool dl = d_u && d_q;
  if (!sl && !dl) return set_error(EB_ERR_INVALID, "nothing to apply: pass t/v and/or u/q");
  EB_CUDA(cudaSetDevice(mesh->m->device));
  return eb::mesh_apply(mesh->m, precision, sl ? 1 : 0, dl, d_t, d_u, d_v, d_q, (cudaStream_t)stream);
}

static int host_apply(eb_mesh mesh, int precision, const double* t, const double* u, double* v, double* q)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  std::lock_guard<std::mutex> g(mesh->lock);
  eb::Mesh* m = mesh->m;
  EB_CUDA(cudaSetDevice(m->device));
  const int ne = m->h.ne, nv = m->h.nv;
  const bool sl = t && v, dl = u && q;
  cudaStream_t st = mesh->stream;
  if (sl) {
    EB_CHECK(m->io_t.alloc(sizeof(double) * ne));
    EB_CHECK(m->io_v.alloc(sizeof(double) * ne));
    EB_CUDA(cudaMemcpyAsync(m->io_t.p, t, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  }
  if (dl) {
    EB_CHECK(m->io_u.alloc(sizeof(double) * nv));
    EB_CHECK(m->io_q.alloc(sizeof(double) * std::max(ne, nv)));
    EB_CUDA(cudaMemcpyAsync(m->io_u.p, u, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
  }
  EB_CHECK(eb::mesh_apply(m, precision, sl ? 1 : 0, dl, sl ? m->io_t.as<double>() : nullptr,
                          dl ? m->io_u.as<double>() : nullptr, sl ? m->io_v.as<double>() : nullptr,
                          dl ? m->io_q.as<double>() : nullptr, st));
  if (sl) EB_CUDA(cudaMemcpyAsync(v, m->io_v.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, st));
  if (dl) EB_CUDA(cudaMemcpyAsync(q, m->io_q.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, st));
  EB_CUDA(cudaStreamSynchronize(st));
  return eb::mesh_check_far_error(m);
}

int eb_apply_sl_p0(eb_mesh mesh, int precision, const double* t, double* v)
{
  if (!t || !v) return set_error(EB_ERR_INVALID, "null vector");
  return host_apply(mesh, precision, t, nullptr, v, nullptr);
}

int eb_apply_dl_p1(eb_mesh mesh, int precision, const double* u, double* q)
{
  if (!u || !q) return set_error(EB_ERR_INVALID, "null vector");
  return host_apply(mesh, precision, nullptr, u, nullptr, q);
}

int eb_apply_sl_dl(eb_mesh mesh, int precision, const double* t, const double* u, double* v, double* q)
{
  if (!t || !u || !v || !q) return set_error(EB_ERR_INVALID, "null vector");
  return host_apply(mesh, precision, t, u, v, q);
}

int eb_dirichlet_rhs(eb_mesh mesh, int nrhs, const double* g, double* b)
{
  return eb_dirichlet_rhs_prec(mesh, EB_PREC_FP64, nrhs, g, b);
}

int eb_dirichlet_rhs_prec(eb_mesh mesh, int precision, int nrhs, const double* g, double* b)
{
  if (!mesh || !g || !b || nrhs < 1) return set_error(EB_ERR_INVALID, "null argument");
  if (precision != EB_PREC_FP64 && precision != EB_PREC_MIXED)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  std::lock_guard<std::mutex> lk(mesh->lock);
  eb::Mesh* m = mesh->m;
  EB_CUDA(cudaSetDevice(m->device));
  const eb::HostMesh& h = m->h;
  cudaStream_t st = mesh->stream;
  // K g four data sets per pass (they share every distance and 1/r^3
  // evaluation); a single set, or the last one of an odd group, uses the
  // one-column variant, groups of two or three are padded with zero columns
  constexpr int kCols = 4;
  eb::TmpBuf du(st), dq(st);  // stream-ordered: no device-wide wait when they go
  EB_CHECK(du.alloc(sizeof(double) * kCols * (size_t)h.nv));
  EB_CHECK(dq.alloc(sizeof(double) * kCols * (size_t)h.ne));
  for (int c0 = 0; c0 < nrhs; c0 += kCols) {
    const int nc = std::min(kCols, nrhs - c0);
    const int nd = nc == 1 ? 1 : kCols;
    if (nc < nd) EB_CUDA(cudaMemsetAsync(du.p, 0, sizeof(double) * nd * (size_t)h.nv, st));
    EB_CUDA(cudaMemcpyAsync(du.p, g + (size_t)c0 * h.nv, sizeof(double) * nc * (size_t)h.nv, cudaMemcpyHostToDevice,
                            st));
    EB_CHECK(eb::mesh_apply(m, precision, 0, nd, nullptr, du.as<double>(), nullptr, dq.as<double>(), st));
    EB_CUDA(cudaMemcpyAsync(b + (size_t)c0 * h.ne, dq.p, sizeof(double) * nc * (size_t)h.ne, cudaMemcpyDeviceToHost,
                            st));
  }
  EB_CUDA(cudaStreamSynchronize(st));
  // + (1/2) M g with M[i][node] = J_i / 6 (src/BEM3dLaplace.cpp:469-477)
  for (int i = 0; i < h.ne; i++) {
    const int* f = &h.elems[3 * i];
    const eb::d3 p0 = eb::mk3(h.nodes[3 * f[0]], h.nodes[3 * f[0] + 1], h.nodes[3 * f[0] + 2]);
    const eb::d3 p1 = eb::mk3(h.nodes[3 * f[1]], h.nodes[3 * f[1] + 1], h.nodes[3 * f[1] + 2]);
    const eb::d3 p2 = eb::mk3(h.nodes[3 * f[2]], h.nodes[3 * f[2] + 1], h.nodes[3 * f[2] + 2]);
    const eb::d3 n = eb::cross3(p1 - p0, p2 - p0);
    const double J6 = 0.5 * std::sqrt(eb::dot3(n, n)) / 6.0;
    for (int c = 0; c < nrhs; c++) {
      const double* gc = g + (size_t)c * h.nv;
      b[(size_t)c * h.ne + i] += J6 * (gc[f[0]] + gc[f[1]] + gc[f[2]]);
    }
  }
  return EB_OK;
}

int eb_quadrature(int order, int* nline, double* lx, double* lw, int* ntri, double* tx, double* ty, double* tw)
{
  eb::Quadrature q;
  if (!eb::make_quadrature(order, &q))
    return set_error(EB_ERR_INVALID, "quadrature order must be in 0.." + std::to_string(eb::kMaxOrder));
  if (nline) *nline = q.nl;
  if (ntri) *ntri = q.nt;
  for (int i = 0; i < q.nl; i++) {
    if (lx) lx[i] = q.lx[i];
    if (lw) lw[i] = q.lw[i];
  }
  for (int i = 0; i < q.nt; i++) {
    if (tx) tx[i] = q.tx[i];
    if (ty) ty[i] = q.ty[i];
    if (tw) tw[i] = q.tw[i];
  }
  return EB_OK;
}

int eb_evaluate_potential(eb_mesh mesh, int precision, int npts, const double* pts, const double* t, const double* u,
                          double* out)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (npts < 0 || (npts > 0 && (!pts || !t || !u || !out))) return set_error(EB_ERR_INVALID, "null argument");
  if (npts == 0) return EB_OK;
  std::lock_guard<std::mutex> g(mesh->lock);
  eb::Mesh* m = mesh->m;
  EB_CUDA(cudaSetDevice(m->device));
  cudaStream_t st = mesh->stream;
  const int ne = m->h.ne, nv = m->h.nv;
  EB_CHECK(m->io_t.alloc(sizeof(double) * ne));
  EB_CHECK(m->io_u.alloc(sizeof(double) * nv));
  EB_CHECK(m->io_pts.alloc(sizeof(double) * 3 * (size_t)npts));
  EB_CHECK(m->io_pot.alloc(sizeof(double) * (size_t)npts));
  EB_CUDA(cudaMemcpyAsync(m->io_t.p, t, sizeof(double) * ne, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(m->io_u.p, u, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
  EB_CUDA(cudaMemcpyAsync(m->io_pts.p, pts, sizeof(double) * 3 * (size_t)npts, cudaMemcpyHostToDevice, st));
  EB_CHECK(eb::mesh_evaluate_potential(m, precision, npts, m->io_pts.as<double>(), m->io_t.as<double>(),
                                       m->io_u.as<double>(), m->io_pot.as<double>(), st));
  EB_CUDA(cudaMemcpyAsync(out, m->io_pot.p, sizeof(double) * (size_t)npts, cudaMemcpyDeviceToHost, st));
  EB_CUDA(cudaStreamSynchronize(st));
  return EB_OK;
}

int eb_mesh_set_far_engine(eb_mesh mesh, int engine)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (engine != EB_FAR_CUDA_CORES && engine != EB_FAR_TENSOR_CORES && engine != EB_FAR_SYMMETRIC &&
      engine != EB_FAR_SYMMETRIC_ALL)
    return set_error(EB_ERR_INVALID, "engine must be EB_FAR_CUDA_CORES, EB_FAR_TENSOR_CORES, EB_FAR_SYMMETRIC or "
                                     "EB_FAR_SYMMETRIC_ALL");
  mesh->m->plan.engine = engine;
  return EB_OK;
}

int eb_mesh_get_far_engine(eb_mesh mesh, int precision, int* engine)
{
  if (!mesh || !engine) return set_error(EB_ERR_INVALID, "null argument");
  const bool fp32 = precision == EB_PREC_MIXED;
  *engine = eb::tc_eligible(mesh->m, fp32, 1, 1)    ? EB_FAR_TENSOR_CORES
            : eb::sym_eligible(mesh->m, fp32, 1, 1) ? EB_FAR_SYMMETRIC
                                                    : EB_FAR_CUDA_CORES;
  return EB_OK;
}

int eb_far_engine_costs(int engine, double* mufu_per_pair, double* fma_ops_per_pair, double* tensor_flops_per_pair)
{
  if (engine == EB_FAR_TENSOR_CORES) {
    eb::far_tc_costs(mufu_per_pair, fma_ops_per_pair, tensor_flops_per_pair);
  } else if (engine == EB_FAR_CUDA_CORES) {
    if (mufu_per_pair) *mufu_per_pair = 1.0;
    if (fma_ops_per_pair) *fma_ops_per_pair = 8.0;  // |x-y|^2 1 add + 3 FMA, SL 1 FMA, DL 2 mul + 1 FMA
    if (tensor_flops_per_pair) *tensor_flops_per_pair = 0.0;
  } else if (engine == EB_FAR_SYMMETRIC) {
    // one evaluation per unordered pair, i.e. per two ordered pairs: 1 MUFU,
    // |x-y|^2 1 add + 3 FMA, r^3 2 mul, 1 FMA for the SL sum both rows share,
    // 2 FMA for the DL sums of both rows
    if (mufu_per_pair) *mufu_per_pair = 0.5;
    if (fma_ops_per_pair) *fma_ops_per_pair = 4.5;
    if (tensor_flops_per_pair) *tensor_flops_per_pair = 0.0;
  } else {
    return set_error(EB_ERR_INVALID, "engine must be EB_FAR_CUDA_CORES, EB_FAR_TENSOR_CORES or EB_FAR_SYMMETRIC");
  }
  return EB_OK;
}

int eb_set_profiling(eb_mesh mesh, int on)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  mesh->m->profile = on != 0;
  return EB_OK;
}

int eb_last_kernel_ms(eb_mesh mesh, double* far_ms, double* finalize_ms)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  eb::Mesh* m = mesh->m;
  if (!m->profile || !m->ev0) return set_error(EB_ERR_STATE, "profiling is off or nothing was applied");
  EB_CUDA(cudaEventSynchronize(m->ev2));
  float a = 0.f, b = 0.f;
  EB_CUDA(cudaEventElapsedTime(&a, m->ev0, m->ev1));
  EB_CUDA(cudaEventElapsedTime(&b, m->ev1, m->ev2));
  if (far_ms) *far_ms = a;
  if (finalize_ms) *finalize_ms = b;
  return EB_OK;
}

int eb_apply_sl_p1_device(eb_mesh mesh, int precision, const double* d_t, double* d_v, void* stream)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  EB_CUDA(cudaSetDevice(mesh->m->device));
  return eb::mesh_apply_sl_p1(mesh->m, precision, d_t, d_v, (cudaStream_t)stream);
}

int eb_apply_sl_p1(eb_mesh mesh, int precision, const double* t, double* v)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (!t || !v) return set_error(EB_ERR_INVALID, "null vector");
  std::lock_guard<std::mutex> g(mesh->lock);
  eb::Mesh* m = mesh->m;
  EB_CUDA(cudaSetDevice(m->device));
  const int nv = m->h.nv, ne = m->h.ne;
  cudaStream_t st = mesh->stream;
  EB_CHECK(m->io_u.alloc(sizeof(double) * nv));
  EB_CHECK(m->io_q.alloc(sizeof(double) * std::max(nv, ne)));
  EB_CUDA(cudaMemcpyAsync(m->io_u.p, t, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
  EB_CHECK(eb::mesh_apply_sl_p1(m, precision, m->io_u.as<double>(), m->io_q.as<double>(), st));
  EB_CUDA(cudaMemcpyAsync(v, m->io_q.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
  EB_CUDA(cudaStreamSynchronize(st));
  return EB_OK;
}

int eb_apply_hypersingular_device(eb_mesh mesh, int precision, const double* d_u, double* d_q, void* stream)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  EB_CUDA(cudaSetDevice(mesh->m->device));
  return eb::mesh_apply_hypersingular(mesh->m, precision, d_u, d_q, (cudaStream_t)stream);
}

int eb_apply_hypersingular(eb_mesh mesh, int precision, const double* u, double* q)
{
  if (!mesh) return set_error(EB_ERR_INVALID, "null mesh");
  if (!u || !q) return set_error(EB_ERR_INVALID, "null vector");
  std::lock_guard<std::mutex> g(mesh->lock);
  eb::Mesh* m = mesh->m;
  EB_CUDA(cudaSetDevice(m->device));
  const int nv = m->h.nv;
  cudaStream_t st = mesh->stream;
  EB_CHECK(m->io_u.alloc(sizeof(double) * nv));
  EB_CHECK(m->io_q.alloc(sizeof(double) * std::max(nv, m->h.ne)));
  EB_CUDA(cudaMemcpyAsync(m->io_u.p, u, sizeof(double) * nv, cudaMemcpyHostToDevice, st));
  EB_CHECK(eb::mesh_apply_hypersingular(m, precision, m->io_u.as<double>(), m->io_q.as<double>(), st));
  EB_CUDA(cudaMemcpyAsync(q, m->io_q.p, sizeof(double) * nv, cudaMemcpyDeviceToHost, st));
  EB_CUDA(cudaStreamSynchronize(st));
  return EB_OK;
}

}  // extern "C"
