// Far-field kernels (see farfield.cuh for the formulation).
#include <cuda_runtime.h>

#include <type_traits>

#include "farfield.cuh"
#include "mesh_host.h"
#include "farfield_eval.cuh"

namespace eb {

// Shape of the FP32 far kernel per variant (measured at the L6 icosphere).
// far_source_pairs: eval_cell_sp over a source-pair tile, or eval_cell_x2
// (target points in pairs). The SL-only variants (1, 3 and 4 right-hand sides)
// share one form, so that a column's sums are the same bits whichever variant
// carries it (the batched solver and the server rely on that); they take
// target pairs unless EB_SP_SL, because the 4-column variant, which the
// batched solves and serving run, fits 3 CTAs per SM in that form (100.7 ms
// against 103.4 ms for source pairs at 2 CTAs; 3 columns 90.5 against 94.6).
// The 8-point four-column DL variant also keeps target pairs (its packed sums
// would spill). far_min_blocks: resident CTAs per SM the registers are capped
// for: 3 for the SL-only variants (no spills), 2 for SL+DL, DL and the
// P1-tested SL (SL+DL at 3 spills: 113.5 against 108.4 ms; DL 101.2 against 99.3).
#ifndef EB_SP_SL
#define EB_SP_SL 0
#endif
#ifndef EB_MINB_SL
#define EB_MINB_SL 3
#endif
template <typename T, int K, int NSL, int ND, bool P1T>
__host__ __device__ constexpr bool far_source_pairs()
{
  return std::is_same<T, float>::value && kFarSourcePairs && !(K >= 8 && ND >= 4) &&
         (ND > 0 || P1T || EB_SP_SL);
}
template <typename T, int NSL, int ND, bool P1T>
__host__ __device__ constexpr int far_min_blocks()
{
  return !std::is_same<T, float>::value ? EB_F64_MINB : ND == 0 && !P1T ? EB_MINB_SL : EB_F32_MINB;
}

// P1T: P1 test functions; the item's three outputs are sum_a w_a phi_k(x_a) acc_a
// (k = 0, 1, 2 in the triangle's vertex order) of the single SL charge.
template <typename T, int K, int NQ, int NSL, int ND, bool P1T>
__global__ void __launch_bounds__(kTT, far_min_blocks<T, NSL, ND, P1T>())
    far_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
               int* __restrict__ counter)
{
  using S = typename Slot<T>::type;
  constexpr bool F32 = std::is_same<T, float>::value;
  constexpr bool SP = far_source_pairs<T, K, NSL, ND, P1T>();
  constexpr bool DL = ND > 0;
  constexpr int NDX = ND > 0 ? ND : 1;
  constexpr int NREC = rec_slots(NSL, ND);
  constexpr int NS = NSL > 0 ? NSL : 1;
  constexpr int NACC = P1T ? 3 : NS + NDX;
  static_assert(!P1T || (NSL == 1 && !DL), "P1 test functions pair with one SL charge");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kTS];
  __shared__ dq s_nrm[DL ? kTS : 1];
  __shared__ S s_plane[DL ? kTS : 1];

  S* s_rec = reinterpret_cast<S*>(smem_raw);

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;  // uniform across the CTA
    const int nq = md.Q;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    // separation test per warp (the warp's items are consecutive in Morton order)
    const dq tile = md.twarp[tsel / kWarpItems];

    // target points relative to the triangle centroid are re-read per cell
    // (L1-resident) rather than held in registers
    double cen[3], nrm[3] = {0.0, 0.0, 0.0};
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
      if constexpr (DL) {
        const dq n = md.tnrm[tsel];
        nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
      }
    }
    auto target = [&](int a, T& px, T& py, T& pz, T& pw) {
      if constexpr (F32) {
        const float4 p = md.tgt32[(size_t)tsel * K + a];
        px = p.x; py = p.y; pz = p.z; pw = p.w;
      } else {
        const dq p = md.tgt64[(size_t)tsel * K + a];
        px = p.x; py = p.y; pz = p.z; pw = p.w;
      }
    };
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);

    // float-float accumulators (FP32) or plain doubles (FP64) per output
    T acc_hi[NACC], acc_lo[NACC];
#pragma unroll
    for (int c = 0; c < NACC; ++c) { acc_hi[c] = 0; acc_lo[c] = 0; }

    const int sb = w.cell0 * kCell;
    const int se = min(md.ne, w.cell1 * kCell);
    // FP32 tiles pair their triangles (an even tile size, at least 2, set by the host)
    const int ts = SP ? (md.src_tile & ~1) : md.src_tile;
    const S* grec = reinterpret_cast<const S*>(md.rec);
    for (int t0 = sb; t0 < se; t0 += ts) {
      const int ns = min(ts, se - t0);
      const S* g = grec + (size_t)t0 * nq * NREC;
      if constexpr (SP) {
        // source-pair layout: record slot (2p, b, k) and (2p+1, b, k) interleaved
        const int per = nq * NREC;
        const int nstage = ((ns + 1) >> 1) * per;
        for (int k = threadIdx.x; k < nstage; k += kTT) {
          const int p = k / per, rem = k - p * per;
          const S a = g[(size_t)(2 * p) * per + rem];
          S c;
          if (2 * p + 1 < ns) c = g[(size_t)(2 * p + 1) * per + rem];
          else c = rem % NREC == 0 ? make_float4(0.f, 0.f, 0.f, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
          s_rec[2 * k] = make_float4(a.x, c.x, a.y, c.y);
          s_rec[2 * k + 1] = make_float4(a.z, c.z, a.w, c.w);
        }
        if ((ns & 1) && threadIdx.x == 0) {
          s_vid[ns] = make_int4(-1, -1, -1, 0);
          if constexpr (DL) {
            s_nrm[ns] = dq{0.0, 0.0, 0.0, 0.0};
            s_plane[ns] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
      } else {
        const int nslot = ns * nq * NREC;
        for (int k = threadIdx.x; k < nslot; k += kTT) s_rec[k] = g[k];
      }
      for (int k = threadIdx.x; k < ns; k += kTT) {
        s_vid[k] = md.svid[t0 + k];
        if constexpr (DL) {
          s_nrm[k] = md.snrm[t0 + k];
          if constexpr (F32) s_plane[k] = md.splane32[t0 + k];
          else s_plane[k] = md.splane64[t0 + k];
        }
      }
      __syncthreads();
      if (active) {
        for (int g0 = 0; g0 < ns;) {
          const int cell = (t0 + g0) / kCell;
          const int g1 = min(ns, (cell + 1) * kCell - t0);
          const dq cc = md.ccent[cell];
          // warp-uniform separation test (the warp's bounding sphere against the cell's)
          const double ddx = cc.x - tile.x, ddy = cc.y - tile.y, ddz = cc.z - tile.z;
          const double rr = kFarRatio * (cc.w + tile.w);
          const bool far = ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
          // targets relative to the cell centre
          const T o[3] = {(T)(cc.x - cen[0]), (T)(cc.y - cen[1]), (T)(cc.z - cen[2])};
          T xs[K], ys[K], zs[K], q2[K];
#pragma unroll
          for (int a = 0; a < K; ++a) {
            T px, py, pz, pw;
            target(a, px, py, pz, pw);
            xs[a] = px - o[0]; ys[a] = py - o[1]; zs[a] = pz - o[2];
            q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
          }
          T sl[NS][K], dl[NDX][K];
#pragma unroll
          for (int a = 0; a < K; ++a) {
#pragma unroll
            for (int c = 0; c < NDX; ++c) dl[c][a] = 0;
#pragma unroll
            for (int c = 0; c < NS; ++c) sl[c][a] = 0;
          }
          if constexpr (SP) {
            if (far)
              eval_cell_sp<K, NQ, NSL, ND, true>(s_rec, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o, cen,
                                                 nrm, sl, dl);
            else
              eval_cell_sp<K, NQ, NSL, ND, false>(s_rec, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o, cen,
                                                  nrm, sl, dl);
          } else if constexpr (F32) {
            const float* sf = reinterpret_cast<const float*>(s_rec);
            if (far)
              eval_cell_x2<K, NQ, NSL, ND, true>(sf, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o, cen,
                                                 nrm, sl, dl);
            else
              eval_cell_x2<K, NQ, NSL, ND, false>(sf, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o, cen,
                                                  nrm, sl, dl);
          } else {
            if (far)
              eval_cell<T, K, NQ, NSL, ND, true>(s_rec, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o,
                                                 cen, nrm, sl, dl);
            else
              eval_cell<T, K, NQ, NSL, ND, false>(s_rec, s_vid, s_nrm, s_plane, g0, g1, nq, tv, xs, ys, zs, q2, o,
                                                  cen, nrm, sl, dl);
          }
          if constexpr (P1T) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
              T part = 0;
#pragma unroll
              for (int a = 0; a < K; ++a) {
                T wk;
                if constexpr (F32) wk = comp(md.tgtw32[(size_t)tsel * K + a], k);
                else wk = comp(md.tgtw64[(size_t)tsel * K + a], k);
                part += wk * sl[0][a];
              }
              if constexpr (F32) two_sum_add(acc_hi[k], acc_lo[k], part);
              else acc_hi[k] += part;
            }
          } else {
            // accumulator c < NS: SL charge c; NS + c: DL column c
#pragma unroll
            for (int c = 0; c < NS + NDX; ++c) {
              if (c >= NS + ND) break;
              if (c < NS && NSL == 0) continue;
              T part = 0;
#pragma unroll
              for (int a = 0; a < K; ++a) {
                T px, py, pz, pw;
                target(a, px, py, pz, pw);
                part += pw * (c < NS ? sl[c][a] : dl[c - NS][a]);
              }
              if constexpr (F32) two_sum_add(acc_hi[c], acc_lo[c], part);
              else acc_hi[c] += part;
            }
          }
          g0 = g1;
        }
      }
      __syncthreads();
    }
    if (active) {
      const size_t stride = (size_t)md.nsplit * md.nitems;
      double* out = md.partial + (size_t)w.split * md.nitems + ti;
      if constexpr (P1T) {
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k * stride] = (double)acc_hi[k] + (double)acc_lo[k];
      } else {
#pragma unroll
        for (int c = 0; c < NSL; ++c) out[c * stride] = (double)acc_hi[c] + (double)acc_lo[c];
#pragma unroll
        for (int c = 0; c < ND; ++c) out[(NSL + c) * stride] = (double)acc_hi[NS + c] + (double)acc_lo[NS + c];
      }
    }
  }
}

// Source records for one apply: positions (static) with the per-apply
// strengths s_c = w_b J_j u_h,c(y_b) (DL column c) and charges
// c_r = w_b J_j t_r[j] (SL).
template <typename T, int NSL, int ND>
__device__ __forceinline__ void prep_point(const ApplyArgs& A, long long idx)
{
  using S = typename Slot<T>::type;
  constexpr int NREC = rec_slots(NSL, ND);
  if (idx >= (long long)A.ne * A.Q || (A.active && *A.active == 0)) return;
  const int j = (int)(idx / A.Q), b = (int)(idx % A.Q);
  const double wj = A.wj[idx];  // w_b * J_j
  const int orig = A.perm[j];
  T vals[4 * NREC];
#pragma unroll
  for (int k = 0; k < 4 * NREC; ++k) vals[k] = 0;
#pragma unroll
  for (int c = 0; c < NSL; ++c)
    vals[4 * charge_slot(c, ND) + charge_comp(c, ND)] = (T)(wj * A.t[(size_t)c * A.tstride + orig]);
  if constexpr (NSL == 1 && ND == 1) {
    // the triangle's SL charge without the point weight, J_j t_j (the
    // symmetric far field factors c_b = w_b J_j t_j)
    vals[6] = (T)(A.trin[j].w * A.t[orig]);
  }
  if constexpr (ND > 0) {
    const int4 v = A.svid[j];
    const double e1 = A.bary[2 * b], e2 = A.bary[2 * b + 1];
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      const double* u = A.u + (size_t)c * A.ustride;
      const double uh = (1.0 - e1 - e2) * u[v.x] + e1 * u[v.y] + e2 * u[v.z];
      vals[4 + c] = (T)(wj * uh);
    }
  }
  S* r = reinterpret_cast<S*>(A.rec) + idx * NREC;
  r[0] = reinterpret_cast<const S*>(A.pos)[idx];
#pragma unroll
  for (int k = 1; k < NREC; ++k) {
    S o;
    o.x = vals[4 * k]; o.y = vals[4 * k + 1]; o.z = vals[4 * k + 2]; o.w = vals[4 * k + 3];
    r[k] = o;
  }
}

// Output rows in sorted (Morton) order, kFinalizeLanes threads per row: the
// lanes take every kFinalizeLanes-th partial slot and CSR entry, then add
// their sums in a fixed shuffle tree (deterministic). Sorted order makes the
// partial-sum reads of neighbouring rows contiguous; the row's original index
// i = perm[s] addresses the near-field CSR and the outputs. Result: far sum
// times J_i / (4 pi) plus the FP64 near field.
//
// The kernel is bound by memory latency, not bandwidth, unless each thread
// keeps several loads in flight: the partial slots are read kFinPipe at a
// time for every output at once, and the CSR columns and values of kFinPipe
// entries are loaded before their densities are gathered. Each lane still
// adds its terms in ascending slot / entry order, so the sums do not depend
// on the grouping.
constexpr int kFinPipe = 4;

__device__ __forceinline__ double lanes_sum(double v)
{
#pragma unroll
  for (int o = 1; o < kFinalizeLanes; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ size_t partial_offset(const ApplyArgs& A, int k)
{
  if (A.nchunk == 1) return (size_t)k * A.nitems;
  const int sp = k / A.nchunk;
  return (size_t)sp * A.nitems + (k - sp * A.nchunk);
}

// nr[c] += sum over the lane's entries of val[k] * x_c[col[k]], c < NC
template <int NC>
__device__ __forceinline__ void near_rows(const int* __restrict__ col, const double* __restrict__ val, int kb, int ke,
                                          const double* __restrict__ x, size_t xstride, int lane, double* nr)
{
  for (int k0 = kb + lane; k0 < ke; k0 += kFinPipe * kFinalizeLanes) {
    int cj[kFinPipe];
    double vj[kFinPipe];
#pragma unroll
    for (int r = 0; r < kFinPipe; ++r) {
      const int k = k0 + r * kFinalizeLanes;
      cj[r] = k < ke ? col[k] : -1;
      vj[r] = k < ke ? val[k] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      double xj[kFinPipe];
#pragma unroll
      for (int r = 0; r < kFinPipe; ++r) xj[r] = cj[r] >= 0 ? x[(size_t)c * xstride + cj[r]] : 0.0;
#pragma unroll
      for (int r = 0; r < kFinPipe; ++r)
        if (cj[r] >= 0) nr[c] += vj[r] * xj[r];
    }
  }
}

template <int NSL, int ND>
__device__ __forceinline__ void finalize_row(const ApplyArgs& A, int row_block)
{
  constexpr int NO = NSL + ND;
  const int lane = threadIdx.x % kFinalizeLanes;
  const int s = row_block * kFinalizeRows + threadIdx.x / kFinalizeLanes;
  // every lane of the warp takes part in the shuffles; rows past the end add zeros
  const bool on = s < A.ne && !(A.active && *A.active == 0);
  double far[NO], nr[NO];
#pragma unroll
  for (int c = 0; c < NO; ++c) far[c] = nr[c] = 0.0;
  int i = 0;
  double scale = 0.0;
  if (on) {
    i = A.perm[s];
    scale = A.trin[s].w * (0.25 / M_PI);
    // far partial sums of row s: slot k of output c at c*stride + offset(k) + s*nchunk
    const size_t stride = (size_t)A.nsplit * A.nitems;
    const double* base = A.partial + (size_t)s * A.nchunk;
    const int nparts = A.sym_cells > 0 ? sym_row_slots(s, A.ne, A.sym_cells) : A.nsplit * A.nchunk;
    int k = lane;
    for (; k + (kFinPipe - 1) * kFinalizeLanes < nparts; k += kFinPipe * kFinalizeLanes) {
      double x[kFinPipe][NO];
#pragma unroll
      for (int r = 0; r < kFinPipe; ++r) {
        const size_t off = partial_offset(A, k + r * kFinalizeLanes);
#pragma unroll
        for (int c = 0; c < NO; ++c) x[r][c] = base[c * stride + off];
      }
#pragma unroll
      for (int r = 0; r < kFinPipe; ++r)
#pragma unroll
        for (int c = 0; c < NO; ++c) far[c] += x[r][c];
    }
    for (; k < nparts; k += kFinalizeLanes) {
      const size_t off = partial_offset(A, k);
#pragma unroll
      for (int c = 0; c < NO; ++c) far[c] += base[c * stride + off];
    }
    // FP64 near field: SL rows gather t, DL rows gather u
    if (NSL > 0) near_rows<NSL>(A.sl_col, A.sl_val, A.sl_rowptr[i], A.sl_rowptr[i + 1], A.t, A.tstride, lane, nr);
    if (ND > 0) near_rows<ND>(A.dl_col, A.dl_val, A.dl_rowptr[i], A.dl_rowptr[i + 1], A.u, A.ustride, lane, nr + NSL);
  }
#pragma unroll
  for (int c = 0; c < NO; ++c) {
    const double f = lanes_sum(far[c]);
    const double n = lanes_sum(nr[c]);
    if (on && lane == 0) {
      if (c < NSL) A.v[(size_t)c * A.vstride + i] = scale * f + n;
      else A.q[(size_t)(c - NSL) * A.qstride + i] = scale * f + n;
    }
  }
}

template <typename T, int NSL, int ND>
__global__ void prep_kernel(ApplyArgs A)
{
  prep_point<T, NSL, ND>(A, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

template <int NSL, int ND>
__global__ void __launch_bounds__(kFinalizeBlock) finalize_kernel(ApplyArgs A)
{
  finalize_row<NSL, ND>(A, blockIdx.x);
}

// Batched forms: block b belongs to entry e with off[e] <= b < off[e+1].
__device__ __forceinline__ int entry_of_block(const int* __restrict__ off, int n, int b)
{
  int lo = 0, hi = n;  // off[lo] <= b < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <typename T, int NSL, int ND>
__global__ void prep_batch_kernel(const ApplyArgs* __restrict__ args, const int* __restrict__ off, int n)
{
  const int e = entry_of_block(off, n, blockIdx.x);
  prep_point<T, NSL, ND>(args[e], (long long)(blockIdx.x - off[e]) * blockDim.x + threadIdx.x);
}

template <int NSL, int ND>
__global__ void finalize_batch_kernel(const ApplyArgs* __restrict__ args, const int* __restrict__ off, int n)
{
  const int e = entry_of_block(off, n, blockIdx.x);
  finalize_row<NSL, ND>(args[e], blockIdx.x - off[e]);
}

// ---------------------------------------------------------------------------
// Host-side dispatch over the compiled variants.

struct FarLaunch {
  bool fp32;
  int K, NQ, NSL;
  int ND;
};

template <typename T, int K, int NQ, int NSL, int ND, bool P1T>
static cudaError_t launch_far_t(const FarMeshDesc* d_meshes, const WorkItem* d_items, int nitems, int* d_counter,
                                size_t smem, int grid, cudaStream_t st)
{
  auto kern = far_kernel<T, K, NQ, NSL, ND, P1T>;
  // the kernel's static shared memory (up to ~4 KB) counts against the same
  // 48 KB default, so opt in above 32 KB of dynamic shared memory
  if (smem > 32 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  kern<<<grid, kTT, smem, st>>>(d_meshes, d_items, nitems, d_counter);
  return cudaGetLastError();
}

template <typename T, int K, int NQ, int NSL, int ND, bool P1T>
static int occupancy_t(size_t smem)
{
  int nb = 0;
  if (smem > 32 * 1024)
    cudaFuncSetAttribute(far_kernel<T, K, NQ, NSL, ND, P1T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, far_kernel<T, K, NQ, NSL, ND, P1T>, kTT, smem);
  return nb;
}

// (points per item K, rule size NQ; NQ = 0: rule size read at run time)
#define EB_FAR_CASES(X) X(1, 1) X(3, 3) X(4, 4) X(6, 6) X(7, 7) X(8, 0)

// Operator variants compiled, (SL charges, DL columns), for record
// preparation, far field and finalize: the fused SL+DL apply, SL alone with
// 1, 3 or 4 right-hand sides, DL alone with 1 or 4 densities (4: the
// Dirichlet right-hand sides of multi-RHS solves); the far field adds the
// P1-test variant (1 charge, no DL).
#define EB_VARIANTS(V) V(0, 1) V(1, 0) V(1, 1) V(3, 0) V(4, 0) V(0, 4)
#define EB_FAR_VARIANTS(V) \
  V(0, 1, false) V(1, 0, false) V(1, 1, false) V(3, 0, false) V(4, 0, false) V(1, 0, true) V(0, 4, false)

template <typename T, int NSL, int ND, bool P1T>
static cudaError_t dispatch_k(int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n, int* dc, size_t smem,
                              int grid, cudaStream_t st)
{
#define X(KK, NQQ)                                    \
  if (K == KK && (NQQ == 0 || Q == NQQ))              \
    return launch_far_t<T, KK, NQQ, NSL, ND, P1T>(dm, di, n, dc, smem, grid, st);
  EB_FAR_CASES(X)
#undef X
  return cudaErrorInvalidValue;
}

template <typename T, int NSL, int ND, bool P1T>
static int dispatch_occ(int K, int Q, size_t smem)
{
#define X(KK, NQQ) \
  if (K == KK && (NQQ == 0 || Q == NQQ)) return occupancy_t<T, KK, NQQ, NSL, ND, P1T>(smem);
  EB_FAR_CASES(X)
#undef X
  return 0;
}

template <typename T>
static cudaError_t far_launch_t(int NSL, int ND, bool P1, int K, int Q, const FarMeshDesc* dm, const WorkItem* di,
                                int n, int* dc, size_t smem, int grid, cudaStream_t st)
{
#define V(NS, D, P) \
  if (NSL == NS && ND == D && P1 == P) return dispatch_k<T, NS, D, P>(K, Q, dm, di, n, dc, smem, grid, st);
  EB_FAR_VARIANTS(V)
#undef V
  return cudaErrorInvalidValue;
}

template <typename T>
static int far_occ_t(int NSL, int ND, bool P1, int K, int Q, size_t smem)
{
#define V(NS, D, P) \
  if (NSL == NS && ND == D && P1 == P) return dispatch_occ<T, NS, D, P>(K, Q, smem);
  EB_FAR_VARIANTS(V)
#undef V
  return 0;
}

bool far_variant_supported(int NSL, int ND)
{
#define V(NS, D) \
  if (NSL == NS && ND == D) return true;
  EB_VARIANTS(V)
#undef V
  return false;
}

cudaError_t far_launch(bool fp32, int NSL, int ND, int K, int Q, const FarMeshDesc* dm, const WorkItem* di, int n,
                       int* dc, size_t smem, int grid, cudaStream_t st, bool p1t)
{
  return fp32 ? far_launch_t<float>(NSL, ND, p1t, K, Q, dm, di, n, dc, smem, grid, st)
              : far_launch_t<double>(NSL, ND, p1t, K, Q, dm, di, n, dc, smem, grid, st);
}

int far_occupancy(bool fp32, int NSL, int ND, int K, int Q, size_t smem, bool p1t)
{
  return fp32 ? far_occ_t<float>(NSL, ND, p1t, K, Q, smem) : far_occ_t<double>(NSL, ND, p1t, K, Q, smem);
}

template <typename T>
static cudaError_t prep_launch_t(int NSL, int ND, const ApplyArgs& A, cudaStream_t st)
{
  const long long n = (long long)A.ne * A.Q;
  const int blk = 256;
  const int grid = (int)((n + blk - 1) / blk);
#define V(NS, D)                                                \
  if (NSL == NS && ND == D) {                                   \
    prep_kernel<T, NS, D><<<grid, blk, 0, st>>>(A);             \
    return cudaGetLastError();                                  \
  }
  EB_VARIANTS(V)
#undef V
  return cudaErrorInvalidValue;
}

cudaError_t prep_launch(bool fp32, int NSL, int ND, const ApplyArgs& A, cudaStream_t st)
{
  return fp32 ? prep_launch_t<float>(NSL, ND, A, st) : prep_launch_t<double>(NSL, ND, A, st);
}

cudaError_t finalize_launch(int NSL, int ND, const ApplyArgs& A, cudaStream_t st)
{
  const int grid = (A.ne + kFinalizeRows - 1) / kFinalizeRows;
#define V(NS, D)                                                \
  if (NSL == NS && ND == D) {                                   \
    finalize_kernel<NS, D><<<grid, kFinalizeBlock, 0, st>>>(A); \
    return cudaGetLastError();                                  \
  }
  EB_VARIANTS(V)
#undef V
  return cudaErrorInvalidValue;
}

template <typename T>
static cudaError_t prep_batch_t(int NSL, int ND, const ApplyArgs* d_args, const int* d_off, int n, int nblocks,
                                cudaStream_t st)
{
#define V(NS, D)                                                                  \
  if (NSL == NS && ND == D) {                                                     \
    prep_batch_kernel<T, NS, D><<<nblocks, kPrepBlock, 0, st>>>(d_args, d_off, n); \
    return cudaGetLastError();                                                    \
  }
  EB_VARIANTS(V)
#undef V
  return cudaErrorInvalidValue;
}

cudaError_t prep_launch_batch(bool fp32, int NSL, int ND, const ApplyArgs* d_args, const int* d_off, int n,
                              int nblocks, cudaStream_t st)
{
  return fp32 ? prep_batch_t<float>(NSL, ND, d_args, d_off, n, nblocks, st)
              : prep_batch_t<double>(NSL, ND, d_args, d_off, n, nblocks, st);
}

cudaError_t finalize_launch_batch(int NSL, int ND, const ApplyArgs* d_args, const int* d_off, int n, int nblocks,
                                  cudaStream_t st)
{
#define V(NS, D)                                                                          \
  if (NSL == NS && ND == D) {                                                             \
    finalize_batch_kernel<NS, D><<<nblocks, kFinalizeBlock, 0, st>>>(d_args, d_off, n);   \
    return cudaGetLastError();                                                            \
  }
  EB_VARIANTS(V)
#undef V
  return cudaErrorInvalidValue;
}

}  // namespace eb
