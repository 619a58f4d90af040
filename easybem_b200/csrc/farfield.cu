// Far-field kernels (see farfield.cuh for the formulation).
#include <cuda_runtime.h>

#include <type_traits>

#include "farfield.cuh"
#include "mesh_host.h"

namespace eb {

// Neumann/Knuth two-sum accumulation: (s, e) holds s + e exactly up to the
// rounding of e.
__device__ __forceinline__ void two_sum_add(float& s, float& e, float x)
{
  const float t = __fadd_rn(s, x);
  const float bp = __fsub_rn(t, s);
  const float err = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp));
  s = t;
  e = __fadd_rn(e, err);
}

__device__ __forceinline__ bool shares_vertex(int4 a, int4 b)
{
  return (a.x == b.x) | (a.x == b.y) | (a.x == b.z) | (a.y == b.x) | (a.y == b.y) | (a.y == b.z) |
         (a.z == b.x) | (a.z == b.y) | (a.z == b.z);
}

template <typename T>
struct Slot;
template <>
struct Slot<float> {
  using type = float4;
};
template <>
struct Slot<double> {
  using type = dq;
};

__device__ __forceinline__ float comp(const float4& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ double comp(const dq& v, int c) { return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w; }
__device__ __forceinline__ float rsq(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }

// One source point against the K target points of an item.
template <typename T, int K, int NSL, bool DL, typename S>
__device__ __forceinline__ void eval_point(const S* __restrict__ r, const T (&x)[K], const T (&y)[K],
                                           const T (&z)[K], T (&sl)[NSL > 0 ? NSL : 1][K], T (&dl)[K])
{
  constexpr int NREC = rec_slots(NSL, DL);
  const S p0 = r[0];
  S p1;
  if constexpr (DL || NSL > 1) p1 = r[1];
#pragma unroll
  for (int a = 0; a < K; ++a) {
    const T dx = x[a] - p0.x, dy = y[a] - p0.y, dz = z[a] - p0.z;
    const T r2 = dx * dx + dy * dy + dz * dz;
    const T inv = rsq(r2);
    if constexpr (NSL >= 1) sl[0][a] += p0.w * inv;
#pragma unroll
    for (int c = 1; c < NSL; ++c) {
      int slot, cc;
      charge_slot(c, DL, &slot, &cc);
      sl[c][a] += comp(slot == 1 ? p1 : r[slot], cc) * inv;
    }
    if constexpr (DL) {
      const T rp = dx * p1.x + dy * p1.y + dz * p1.z;
      const T inv2 = inv * inv;
      dl[a] += (rp * inv2) * inv;
    }
  }
  (void)NREC;
}

// One target item against the source points of triangles [s0, s1) of the
// staged tile: accumulates SL charges (NSL of them) and the DL dipole term.
// Source triangles sharing a vertex with the target triangle are skipped.
template <typename T, int K, int NQ, int NSL, bool DL>
__device__ __forceinline__ void eval_segment(const typename Slot<T>::type* __restrict__ srec,
                                             const int4* __restrict__ svid, int s0, int s1, int nq,
                                             int4 tv, const T (&x)[K], const T (&y)[K], const T (&z)[K],
                                             T (&sl)[NSL > 0 ? NSL : 1][K], T (&dl)[K])
{
  constexpr int NREC = rec_slots(NSL, DL);
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    if (shares_vertex(tv, svid[s])) continue;
    if constexpr (NQ > 0) {
      const typename Slot<T>::type* r = srec + (size_t)s * NQ * NREC;
#pragma unroll
      for (int b = 0; b < NQ; ++b) eval_point<T, K, NSL, DL>(r + b * NREC, x, y, z, sl, dl);
    } else {
      const typename Slot<T>::type* r = srec + (size_t)s * nq * NREC;
#pragma unroll 1
      for (int b = 0; b < nq; ++b) eval_point<T, K, NSL, DL>(r + b * NREC, x, y, z, sl, dl);
    }
  }
}

template <typename T, int K, int NQ, int NSL, bool DL>
__global__ void __launch_bounds__(kTT) far_kernel(const FarMeshDesc* __restrict__ meshes,
                                                  const WorkItem* __restrict__ items, int nitems,
                                                  int* __restrict__ counter)
{
  using S = typename Slot<T>::type;
  constexpr bool F32 = std::is_same<T, float>::value;
  constexpr int NREC = rec_slots(NSL, DL);
  constexpr int NS = NSL > 0 ? NSL : 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kTS];

  S* s_rec = reinterpret_cast<S*>(smem_raw);

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    const int nq = md.Q;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;

    T xt[K], yt[K], zt[K], wt[K];
    double cx = 0.0, cy = 0.0, cz = 0.0;
    if constexpr (F32) {
      const dq c = md.tcent[tsel];
      cx = c.x; cy = c.y; cz = c.z;
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const float4 p = md.tgt32[(size_t)tsel * K + a];
        xt[a] = p.x; yt[a] = p.y; zt[a] = p.z; wt[a] = p.w;
      }
    } else {
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const dq p = md.tgt64[(size_t)tsel * K + a];
        xt[a] = (T)p.x; yt[a] = (T)p.y; zt[a] = (T)p.z; wt[a] = (T)p.w;
      }
    }
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);

    // float-float accumulators (FP32) or plain doubles (FP64) per output
    T acc_hi[NS + 1], acc_lo[NS + 1];
#pragma unroll
    for (int c = 0; c <= NS; ++c) { acc_hi[c] = 0; acc_lo[c] = 0; }

    const int sb = w.cell0 * kCell;
    const int se = min(md.ne, w.cell1 * kCell);
    const int ts = md.src_tile;
    const S* grec = reinterpret_cast<const S*>(md.rec);
    for (int t0 = sb; t0 < se; t0 += ts) {
      const int ns = min(ts, se - t0);
      const S* g = grec + (size_t)t0 * nq * NREC;
      const int nslot = ns * nq * NREC;
      for (int k = threadIdx.x; k < nslot; k += kTT) s_rec[k] = g[k];
      for (int k = threadIdx.x; k < ns; k += kTT) s_vid[k] = md.svid[t0 + k];
      __syncthreads();
      if (active) {
        for (int g0 = 0; g0 < ns;) {
          const int cell = (t0 + g0) / kCell;
          const int g1 = min(ns, (cell + 1) * kCell - t0);
          T xs[K], ys[K], zs[K];
          if constexpr (F32) {
            const dq cc = md.ccent[cell];
            const float ox = (float)(cc.x - cx), oy = (float)(cc.y - cy), oz = (float)(cc.z - cz);
#pragma unroll
            for (int a = 0; a < K; ++a) { xs[a] = xt[a] - ox; ys[a] = yt[a] - oy; zs[a] = zt[a] - oz; }
          } else {
#pragma unroll
            for (int a = 0; a < K; ++a) { xs[a] = xt[a]; ys[a] = yt[a]; zs[a] = zt[a]; }
          }
          T sl[NS][K], dl[K];
#pragma unroll
          for (int a = 0; a < K; ++a) {
            dl[a] = 0;
#pragma unroll
            for (int c = 0; c < NS; ++c) sl[c][a] = 0;
          }
          eval_segment<T, K, NQ, NSL, DL>(s_rec, s_vid, g0, g1, nq, tv, xs, ys, zs, sl, dl);
#pragma unroll
          for (int c = 0; c <= NS; ++c) {
            if (c == NS && !DL) break;
            if (c < NS && NSL == 0) continue;
            T part = 0;
#pragma unroll
            for (int a = 0; a < K; ++a) part += wt[a] * (c < NS ? sl[c][a] : dl[a]);
            if constexpr (F32) two_sum_add(acc_hi[c], acc_lo[c], part);
            else acc_hi[c] += part;
          }
          g0 = g1;
        }
      }
      __syncthreads();
    }
    if (active) {
      const size_t stride = (size_t)md.nsplit * md.nitems;
      double* out = md.partial + (size_t)w.split * md.nitems + ti;
#pragma unroll
      for (int c = 0; c < NSL; ++c) out[c * stride] = (double)acc_hi[c] + (double)acc_lo[c];
      if (DL) out[NSL * stride] = (double)acc_hi[NS] + (double)acc_lo[NS];
    }
  }
}

// Source records for one apply: positions (static) with the per-apply
// charges w_b J_j t_j and dipoles w_b J_j u_h(y_b) n_j.
template <typename T, int NSL, bool DL>
__global__ void prep_kernel(int ne, int Q, const typename Slot<T>::type* __restrict__ pos,
                            const dq* __restrict__ trin, const int4* __restrict__ svid,
                            const int* __restrict__ perm, const double* __restrict__ bary,
                            const double* __restrict__ t, int tstride, const double* __restrict__ u,
                            typename Slot<T>::type* __restrict__ rec)
{
  using S = typename Slot<T>::type;
  constexpr int NREC = rec_slots(NSL, DL);
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)ne * Q) return;
  const int j = (int)(idx / Q), b = (int)(idx % Q);
  const S p = pos[idx];
  const double wj = (double)p.w;  // w_b * J_j (rounded to T in the FP32 table)
  S* r = rec + idx * NREC;
  S s0;
  s0.x = p.x; s0.y = p.y; s0.z = p.z; s0.w = 0;
  const int orig = perm[j];
  if (NSL >= 1) s0.w = (T)(wj * t[orig]);
  r[0] = s0;
  if (DL) {
    const dq n = trin[j];
    const int4 v = svid[j];
    const double e1 = bary[2 * b], e2 = bary[2 * b + 1];
    const double uh = (1.0 - e1 - e2) * u[v.x] + e1 * u[v.y] + e2 * u[v.z];
    const double s = wj * uh;
    S s1;
    s1.x = (T)(s * n.x); s1.y = (T)(s * n.y); s1.z = (T)(s * n.z); s1.w = 0;
    if (NSL >= 2) s1.w = (T)(wj * t[(size_t)tstride + orig]);
    r[1] = s1;
  }
  for (int c = DL ? 2 : 1; c < NSL; ++c) {
    int slot, cc;
    charge_slot(c, DL, &slot, &cc);
    T* rr = reinterpret_cast<T*>(&r[slot]);
    if (cc == 0) { r[slot].x = 0; r[slot].y = 0; r[slot].z = 0; r[slot].w = 0; }
    rr[cc] = (T)(wj * t[(size_t)c * tstride + orig]);
  }
}

// Output rows in original order: sum the partial slots of the triangle's
// items in a fixed order, scale by J_i / (4 pi) and add the FP64 near field.
template <int NSL, bool DL>
__global__ void finalize_kernel(int ne, int nchunk, int nsplit, int nitems, const int* __restrict__ iperm,
                                const dq* __restrict__ trin, const double* __restrict__ partial,
                                const int* __restrict__ sl_rowptr, const int* __restrict__ sl_col,
                                const double* __restrict__ sl_val, const int* __restrict__ dl_rowptr,
                                const int* __restrict__ dl_col, const double* __restrict__ dl_val,
                                const double* __restrict__ t, int tstride, const double* __restrict__ u,
                                double* __restrict__ v, int vstride, double* __restrict__ q)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne) return;
  const int s = iperm[i];
  const double scale = trin[s].w * (0.25 / M_PI);
  const size_t stride = (size_t)nsplit * nitems;
  for (int c = 0; c < NSL; ++c) {
    double far = 0.0;
    for (int sp = 0; sp < nsplit; ++sp)
      for (int ch = 0; ch < nchunk; ++ch) far += partial[c * stride + (size_t)sp * nitems + (size_t)s * nchunk + ch];
    double nr = 0.0;
    for (int k = sl_rowptr[i]; k < sl_rowptr[i + 1]; ++k) nr += sl_val[k] * t[(size_t)c * tstride + sl_col[k]];
    v[(size_t)c * vstride + i] = scale * far + nr;
  }
  if (DL) {
    double far = 0.0;
    for (int sp = 0; sp < nsplit; ++sp)
      for (int ch = 0; ch < nchunk; ++ch) far += partial[NSL * stride + (size_t)sp * nitems + (size_t)s * nchunk + ch];
    double nr = 0.0;
    for (int k = dl_rowptr[i]; k < dl_rowptr[i + 1]; ++k) nr += dl_val[k] * u[dl_col[k]];
    q[i] = scale * far + nr;
  }
}

// ---------------------------------------------------------------------------
// Host-side dispatch over the compiled variants.

struct FarLaunch {
  bool fp32;
  int K, NQ, NSL;
  bool DL;
};

template <typename T, int K, int NQ, int NSL, bool DL>
static cudaError_t launch_far_t(const FarMeshDesc* d_meshes, const WorkItem* d_items, int nitems, int* d_counter,
                                size_t smem, int grid, cudaStream_t st)
{
  auto kern = far_kernel<T, K, NQ, NSL, DL>;
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, kTT, smem, st>>>(d_meshes, d_items, nitems, d_counter);
  return cudaGetLastError();
}

template <typename T, int K, int NQ, int NSL, bool DL>
static int occupancy_t(size_t smem)
{
  int nb = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, far_kernel<T, K, NQ, NSL, DL>, kTT, smem);
  return nb;
}

#define EB_FAR_CASES(X)                                                                                  \
  X(1, 1) X(3, 3) X(4, 4) X(6, 6) X(7, 7) X(8, 0)

#define EB_FAR_DISPATCH(FN, RET, ...)                                                                    \
  {                                                                                                      \
    switch (NSL * 2 + (DL ? 1 : 0)) {                                                                    \
      case 1: return dispatch_k<T, 0, true>(__VA_ARGS__);                                                \
      case 2: return dispatch_k<T, 1, false>(__VA_ARGS__);                                               \
      case 3: return dispatch_k<T, 1, true>(__VA_ARGS__);                                                \
      case 8: return dispatch_k<T, 4, false>(__VA_ARGS__);                                               \
      default: return RET;                                                                               \
    }                                                                                                    \
  }

template <typename T, int NSL, bool DL>
static cudaError_t dispatch_k(int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n, int* dc, size_t smem,
                              int grid, cudaStream_t st)
{
#define X(KK, NQQ) \
  if (K == KK && (NQQ == 0 || Q == NQQ)) return launch_far_t<T, KK, NQQ, NSL, DL>(dm, di, n, dc, smem, grid, st);
  EB_FAR_CASES(X)
#undef X
  return cudaErrorInvalidValue;
}

template <typename T, int NSL, bool DL>
static int dispatch_occ(int K, int Q, size_t smem)
{
#define X(KK, NQQ) \
  if (K == KK && (NQQ == 0 || Q == NQQ)) return occupancy_t<T, KK, NQQ, NSL, DL>(smem);
  EB_FAR_CASES(X)
#undef X
  return 0;
}

template <typename T>
static cudaError_t far_launch_t(int NSL, bool DL, int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n,
                                int* dc, size_t smem, int grid, cudaStream_t st)
{
  switch (NSL * 2 + (DL ? 1 : 0)) {
    case 1: return dispatch_k<T, 0, true>(K, Q, dm, di, n, dc, smem, grid, st);
    case 2: return dispatch_k<T, 1, false>(K, Q, dm, di, n, dc, smem, grid, st);
    case 3: return dispatch_k<T, 1, true>(K, Q, dm, di, n, dc, smem, grid, st);
    case 8: return dispatch_k<T, 4, false>(K, Q, dm, di, n, dc, smem, grid, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename T>
static int far_occ_t(int NSL, bool DL, int K, int Q, size_t smem)
{
  switch (NSL * 2 + (DL ? 1 : 0)) {
    case 1: return dispatch_occ<T, 0, true>(K, Q, smem);
    case 2: return dispatch_occ<T, 1, false>(K, Q, smem);
    case 3: return dispatch_occ<T, 1, true>(K, Q, smem);
    case 8: return dispatch_occ<T, 4, false>(K, Q, smem);
    default: return 0;
  }
}

bool far_variant_supported(int NSL, bool DL)
{
  const int code = NSL * 2 + (DL ? 1 : 0);
  return code == 1 || code == 2 || code == 3 || code == 8;
}

cudaError_t far_launch(bool fp32, int NSL, bool DL, int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n,
                       int* dc, size_t smem, int grid, cudaStream_t st)
{
  return fp32 ? far_launch_t<float>(NSL, DL, K, Q, dm, di, n, dc, smem, grid, st)
              : far_launch_t<double>(NSL, DL, K, Q, dm, di, n, dc, smem, grid, st);
}

int far_occupancy(bool fp32, int NSL, bool DL, int K, int Q, size_t smem)
{
  return fp32 ? far_occ_t<float>(NSL, DL, K, Q, smem) : far_occ_t<double>(NSL, DL, K, Q, smem);
}

template <typename T>
static cudaError_t prep_launch_t(int NSL, bool DL, int ne, int Q, const void* pos, const dq* trin, const int4* svid,
                                 const int* perm, const double* bary, const double* t, int tstride, const double* u,
                                 void* rec, cudaStream_t st)
{
  using S = typename Slot<T>::type;
  const long long n = (long long)ne * Q;
  const int blk = 256;
  const int grid = (int)((n + blk - 1) / blk);
  const S* p = reinterpret_cast<const S*>(pos);
  S* r = reinterpret_cast<S*>(rec);
  switch (NSL * 2 + (DL ? 1 : 0)) {
    case 1: prep_kernel<T, 0, true><<<grid, blk, 0, st>>>(ne, Q, p, trin, svid, perm, bary, t, tstride, u, r); break;
    case 2: prep_kernel<T, 1, false><<<grid, blk, 0, st>>>(ne, Q, p, trin, svid, perm, bary, t, tstride, u, r); break;
    case 3: prep_kernel<T, 1, true><<<grid, blk, 0, st>>>(ne, Q, p, trin, svid, perm, bary, t, tstride, u, r); break;
    case 8: prep_kernel<T, 4, false><<<grid, blk, 0, st>>>(ne, Q, p, trin, svid, perm, bary, t, tstride, u, r); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t prep_launch(bool fp32, int NSL, bool DL, int ne, int Q, const void* pos, const dq* trin, const int4* svid,
                        const int* perm, const double* bary, const double* t, int tstride, const double* u, void* rec,
                        cudaStream_t st)
{
  return fp32 ? prep_launch_t<float>(NSL, DL, ne, Q, pos, trin, svid, perm, bary, t, tstride, u, rec, st)
              : prep_launch_t<double>(NSL, DL, ne, Q, pos, trin, svid, perm, bary, t, tstride, u, rec, st);
}

cudaError_t finalize_launch(int NSL, bool DL, int ne, int nchunk, int nsplit, int nitems, const int* iperm,
                            const dq* trin, const double* partial, const int* sl_rowptr, const int* sl_col,
                            const double* sl_val, const int* dl_rowptr, const int* dl_col, const double* dl_val,
                            const double* t, int tstride, const double* u, double* v, int vstride, double* q,
                            cudaStream_t st)
{
  const int blk = 128, grid = (ne + blk - 1) / blk;
#define FIN(NS, D)                                                                                              \
  finalize_kernel<NS, D><<<grid, blk, 0, st>>>(ne, nchunk, nsplit, nitems, iperm, trin, partial, sl_rowptr,     \
                                               sl_col, sl_val, dl_rowptr, dl_col, dl_val, t, tstride, u, v,    \
                                               vstride, q)
  switch (NSL * 2 + (DL ? 1 : 0)) {
    case 1: FIN(0, true); break;
    case 2: FIN(1, false); break;
    case 3: FIN(1, true); break;
    case 8: FIN(4, false); break;
    default: return cudaErrorInvalidValue;
  }
#undef FIN
  return cudaGetLastError();
}

}  // namespace eb
