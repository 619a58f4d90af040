// Potential evaluation off the surface: u(x) = V t - W u (the representation
// formula), as evaluateLaplace3d computes it (src/BEM3dLaplace.cpp:784-843):
//
//   u(x) = sum_j J_j/(4 pi) sum_b w_b [ t_j / |x - y_b| - u_h(y_b) (x - y_b).n_j / |x - y_b|^3 ]
//
// with the triangle rule of the mesh's quadrature index. Each thread owns one
// evaluation point; a block takes 128 points and one chunk of source cells
// staged through shared memory; per-chunk partial sums are added in a fixed
// order by a second kernel (deterministic). The source records are the ones
// the SL+DL apply prepares (charges w_b J_j t_j and strengths w_b J_j u_h);
// (x - y).n_j is the signed distance of x from the plane of triangle j. FP32
// evaluates cell-relative coordinates with per-cell two-sum accumulation.
//
// In FP32 the cell-relative coordinates round to ~6e-8 of the cell radius R;
// for a point closer to a cell than about 2R that error is no longer small
// next to the distances, and near the surface the terms of neighbouring
// triangles cancel on top of it. The FP32 kernel therefore sums every cell
// whose centre lies within kPotNear * R of a point in FP64 (from FP64
// records; a few cells per point near the surface, none away from it).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "engine.h"

namespace eb {

constexpr int kPotThreads = 128;
constexpr double kPotNear = 2.5;  // cells within this many radii of a point are summed in FP64

// One cell's contribution to u(x) in FP64 from FP64 records ([ne*Q][2] dq)
// and planes, (xs, ys, zs) = x relative to the cell centre.
__device__ __noinline__ double pot_cell_fp64(double xs, double ys, double zs, const dq* __restrict__ rec64,
                                             const dq* __restrict__ plane64, int s0, int s1, int Q)
{
  double part = 0.0;
  for (int s = s0; s < s1; ++s) {
    const dq pn = plane64[s];
    const double d = xs * pn.x + (ys * pn.y + (zs * pn.z - pn.w));
    double sl = 0.0, acc = 0.0;
    const dq* r = rec64 + (size_t)s * Q * 2;
    for (int b = 0; b < Q; ++b) {
      const dq p0 = r[2 * b], p1 = r[2 * b + 1];
      const double dx = xs + 0.5 * p0.x, dy = ys + 0.5 * p0.y, dz = zs + 0.5 * p0.z;
      const double inv = rsqrt(dx * dx + dy * dy + dz * dz);
      sl += p1.y * inv;
      acc += (inv * inv) * (p1.x * inv);
    }
    part += sl - d * acc;
  }
  return part;
}

__device__ __forceinline__ void pot_two_sum(float& s, float& e, float x)
{
  const float t = __fadd_rn(s, x);
  const float bp = __fsub_rn(t, s);
  e = __fadd_rn(e, __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp)));
  s = t;
}

template <typename T>
struct PotSlot;
template <>
struct PotSlot<float> {
  using type = float4;
};
template <>
struct PotSlot<double> {
  using type = dq;
};

__device__ __forceinline__ float pot_rsq(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double pot_rsq(double x) { return rsqrt(x); }

// records: 2 slots per source point, slot0 = (-2 y_rel, |y_rel|^2), slot1 = (s, c, ., .)
template <typename T>
__global__ void __launch_bounds__(kPotThreads) potential_kernel(int npts, const double* __restrict__ pts, int ne,
                                                                int Q, int cells_per_chunk, int ts,
                                                                const typename PotSlot<T>::type* __restrict__ rec,
                                                                const typename PotSlot<T>::type* __restrict__ plane,
                                                                const dq* __restrict__ ccent,
                                                                double* __restrict__ partial)
{
  using S = typename PotSlot<T>::type;
  constexpr bool F32 = std::is_same<T, float>::value;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S* s_rec = reinterpret_cast<S*>(smem_raw);
  __shared__ S s_plane[kTS];
  const int i = blockIdx.x * kPotThreads + threadIdx.x;
  const bool active = i < npts;
  const double px = active ? pts[3 * i] : 0.0, py = active ? pts[3 * i + 1] : 0.0, pz = active ? pts[3 * i + 2] : 0.0;
  const int ncells = (ne + kCell - 1) / kCell;
  const int c0 = blockIdx.y * cells_per_chunk, c1 = min(ncells, c0 + cells_per_chunk);
  const int sb = c0 * kCell, se = min(ne, c1 * kCell);
  T hi = 0, lo = 0;
  for (int t0 = sb; t0 < se; t0 += ts) {  // ts <= kTS source triangles per staged tile
    const int ns = min(ts, se - t0);
    for (int k = threadIdx.x; k < ns * Q * 2; k += kPotThreads) s_rec[k] = rec[(size_t)t0 * Q * 2 + k];
    for (int k = threadIdx.x; k < ns; k += kPotThreads) s_plane[k] = plane[t0 + k];
    __syncthreads();
    if (active) {
      for (int g0 = 0; g0 < ns;) {
        const int cell = (t0 + g0) / kCell;
        const int g1 = min(ns, (cell + 1) * kCell - t0);
        const dq cc = ccent[cell];
        const T xs = (T)(px - cc.x), ys = (T)(py - cc.y), zs = (T)(pz - cc.z);
        T part = 0;
        for (int s = g0; s < g1; ++s) {
          const S pn = s_plane[s];
          const T d = xs * pn.x + (ys * pn.y + (zs * pn.z - pn.w));
          T sl = 0, acc = 0;
          const S* r = s_rec + (size_t)s * Q * 2;
          for (int b = 0; b < Q; ++b) {
            const S p0 = r[2 * b], p1 = r[2 * b + 1];
            const T dx = xs + T(0.5) * p0.x, dy = ys + T(0.5) * p0.y, dz = zs + T(0.5) * p0.z;
            const T inv = pot_rsq(dx * dx + dy * dy + dz * dz);
            sl += p1.y * inv;
            acc += (inv * inv) * (p1.x * inv);
          }
          part += sl - d * acc;
        }
        if constexpr (F32) pot_two_sum(hi, lo, part);
        else hi += part;
        g0 = g1;
      }
    }
    __syncthreads();
  }
  if (active) partial[(size_t)blockIdx.y * npts + i] = (double)hi + (double)lo;
}

// FP32 form for sm_100: each thread owns two evaluation points (i and
// i + kPotThreads of the block's 2 * kPotThreads) and evaluates them together
// with packed FFMA2/FMUL2, every source value broadcast to both halves; the
// arithmetic per lane is that of the scalar kernel above.
__global__ void __launch_bounds__(kPotThreads) potential_x2_kernel(int npts, const double* __restrict__ pts, int ne,
                                                                   int Q, int cells_per_chunk, int ts,
                                                                   const float4* __restrict__ rec,
                                                                   const float4* __restrict__ plane,
                                                                   const dq* __restrict__ ccent,
                                                                   const dq* __restrict__ rec64,
                                                                   const dq* __restrict__ plane64,
                                                                   double* __restrict__ partial)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float4* s_rec = reinterpret_cast<float4*>(smem_raw);
  __shared__ float4 s_plane[kTS];
  const int i0 = blockIdx.x * 2 * kPotThreads + threadIdx.x, i1 = i0 + kPotThreads;
  const bool a0 = i0 < npts, a1 = i1 < npts;
  double px[2], py[2], pz[2];
  px[0] = a0 ? pts[3 * i0] : 0.0; py[0] = a0 ? pts[3 * i0 + 1] : 0.0; pz[0] = a0 ? pts[3 * i0 + 2] : 0.0;
  px[1] = a1 ? pts[3 * i1] : px[0]; py[1] = a1 ? pts[3 * i1 + 1] : py[0]; pz[1] = a1 ? pts[3 * i1 + 2] : pz[0];
  const int ncells = (ne + kCell - 1) / kCell;
  const int c0 = blockIdx.y * cells_per_chunk, c1 = min(ncells, c0 + cells_per_chunk);
  const int sb = c0 * kCell, se = min(ne, c1 * kCell);
  const float2 half2 = make_float2(0.5f, 0.5f);
  float hi[2] = {0.f, 0.f}, lo[2] = {0.f, 0.f};
  double near[2] = {0.0, 0.0};  // FP64 sums of the cells close to each point
  for (int t0 = sb; t0 < se; t0 += ts) {  // ts <= kTS source triangles per staged tile
    const int ns = min(ts, se - t0);
    for (int k = threadIdx.x; k < ns * Q * 2; k += kPotThreads) s_rec[k] = rec[(size_t)t0 * Q * 2 + k];
    for (int k = threadIdx.x; k < ns; k += kPotThreads) s_plane[k] = plane[t0 + k];
    __syncthreads();
    if (a0) {
      for (int g0 = 0; g0 < ns;) {
        const int cell = (t0 + g0) / kCell;
        const int g1 = min(ns, (cell + 1) * kCell - t0);
        const dq cc = ccent[cell];
        const float2 X = make_float2((float)(px[0] - cc.x), (float)(px[1] - cc.x));
        const float2 Y = make_float2((float)(py[0] - cc.y), (float)(py[1] - cc.y));
        const float2 Z = make_float2((float)(pz[0] - cc.z), (float)(pz[1] - cc.z));
        float2 part = make_float2(0.f, 0.f);
        for (int s = g0; s < g1; ++s) {
          const float4 pn = s_plane[s];
          const float2 d = __ffma2_rn(X, make_float2(pn.x, pn.x),
                                      __ffma2_rn(Y, make_float2(pn.y, pn.y),
                                                 __ffma2_rn(Z, make_float2(pn.z, pn.z), make_float2(-pn.w, -pn.w))));
          float2 sl = make_float2(0.f, 0.f), acc = make_float2(0.f, 0.f);
          const float4* r = s_rec + (size_t)s * Q * 2;
          for (int b = 0; b < Q; ++b) {
            const float4 p0 = r[2 * b], p1 = r[2 * b + 1];
            const float2 dx = __ffma2_rn(half2, make_float2(p0.x, p0.x), X);
            const float2 dy = __ffma2_rn(half2, make_float2(p0.y, p0.y), Y);
            const float2 dz = __ffma2_rn(half2, make_float2(p0.z, p0.z), Z);
            const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
            const float2 inv = make_float2(pot_rsq(r2.x), pot_rsq(r2.y));
            sl = __ffma2_rn(make_float2(p1.y, p1.y), inv, sl);
            acc = __ffma2_rn(__fmul2_rn(inv, inv), __fmul2_rn(make_float2(p1.x, p1.x), inv), acc);
          }
          part = __fadd2_rn(part, __ffma2_rn(make_float2(-d.x, -d.y), acc, sl));
        }
        const double rn2 = kPotNear * kPotNear * cc.w * cc.w;
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const double ex = px[k] - cc.x, ey = py[k] - cc.y, ez = pz[k] - cc.z;
          const bool close = (k == 0 || a1) && ex * ex + ey * ey + ez * ez < rn2;
          if (close) near[k] += pot_cell_fp64(ex, ey, ez, rec64, plane64, t0 + g0, t0 + g1, Q);
          const float pk = close ? 0.f : (k == 0 ? part.x : part.y);
          pot_two_sum(hi[k], lo[k], pk);
        }
        g0 = g1;
      }
    }
    __syncthreads();
  }
  if (a0) partial[(size_t)blockIdx.y * npts + i0] = (double)hi[0] + (double)lo[0] + near[0];
  if (a1) partial[(size_t)blockIdx.y * npts + i1] = (double)hi[1] + (double)lo[1] + near[1];
}

__global__ void potential_reduce_kernel(int npts, int nchunk, const double* __restrict__ partial,
                                        double* __restrict__ out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npts) return;
  double s = 0.0;
  for (int c = 0; c < nchunk; c++) s += partial[(size_t)c * npts + i];
  out[i] = s * (0.25 / M_PI);
}

int mesh_evaluate_potential(Mesh* m, int precision, int npts, const double* d_pts, const double* d_t,
                            const double* d_u, double* d_out, cudaStream_t st)
{
  const HostMesh& h = m->h;
  const bool fp32 = precision == EB_PREC_MIXED;
  if (precision != EB_PREC_MIXED && precision != EB_PREC_FP64)
    return set_error(EB_ERR_INVALID, "precision must be EB_PREC_FP64 or EB_PREC_MIXED");
  if (npts < 1) return EB_OK;
  // source records of the fused SL+DL variant (slot1 = (s, c))
  if (!m->rec.p) {
    EB_CHECK(m->rec.alloc((size_t)h.ne * h.Q * kMaxRecSlots * sizeof(dq)));
    EB_CHECK(m->partial.alloc(sizeof(double) * (size_t)kMaxOutputs * m->plan.nsplit * h.nitems));
  }
  const ApplyArgs A = mesh_apply_args(m, fp32, m->rec.p, nullptr, d_t, h.ne, d_u, nullptr, h.ne, nullptr);
  EB_CUDA(prep_launch(fp32, 1, true, A, st));
  if (fp32) {  // FP64 records for the cells close to a point
    EB_CHECK(m->pot_rec64.alloc((size_t)h.ne * h.Q * rec_slots(1, 1) * sizeof(dq)));
    const ApplyArgs A64 = mesh_apply_args(m, false, m->pot_rec64.p, nullptr, d_t, h.ne, d_u, nullptr, h.ne, nullptr);
    EB_CUDA(prep_launch(false, 1, true, A64, st));
  }
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  const int per_block = fp32 ? 2 * kPotThreads : kPotThreads;  // the FP32 kernel takes two points per thread
  const int pblocks = (npts + per_block - 1) / per_block;
  int nchunk = std::max(1, std::min(h.ncells, (4 * nsm + pblocks - 1) / pblocks));
  const int cells_per = (h.ncells + nchunk - 1) / nchunk;
  nchunk = (h.ncells + cells_per - 1) / cells_per;
  EB_CHECK(m->pot_partial.alloc(sizeof(double) * (size_t)nchunk * npts));
  // source triangles per staged tile: whole cells' worth up to kTS, fewer
  // for large rules so the tile stays within 48 KB of shared memory
  const size_t per_tri = (size_t)h.Q * 2 * (fp32 ? sizeof(float4) : sizeof(dq));
  const int ts = (int)std::max<size_t>(1, std::min<size_t>(kTS, (48 * 1024) / per_tri));
  const size_t smem = (size_t)ts * per_tri;
  const dim3 grid(pblocks, nchunk);
  if (fp32) {
    auto k = potential_x2_kernel;
    if (smem > 32 * 1024) EB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, kPotThreads, smem, st>>>(npts, d_pts, h.ne, h.Q, cells_per, ts, m->rec.as<float4>(),
                                       m->splane32.as<float4>(), m->ccent.as<dq>(), m->pot_rec64.as<dq>(),
                                       m->splane64.as<dq>(), m->pot_partial.as<double>());
  } else {
    auto k = potential_kernel<double>;
    if (smem > 32 * 1024) EB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<grid, kPotThreads, smem, st>>>(npts, d_pts, h.ne, h.Q, cells_per, ts, m->rec.as<dq>(), m->splane64.as<dq>(),
                                       m->ccent.as<dq>(), m->pot_partial.as<double>());
  }
  EB_CUDA(cudaGetLastError());
  potential_reduce_kernel<<<(npts + 255) / 256, 256, 0, st>>>(npts, nchunk, m->pot_partial.as<double>(), d_out);
  EB_CUDA(cudaGetLastError());
  return EB_OK;
}

}  // namespace eb
