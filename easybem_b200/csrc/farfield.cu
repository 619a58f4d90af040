// Far-field kernels (see farfield.cuh for the formulation).
#include <cuda_runtime.h>

#include <type_traits>

#include "farfield.cuh"
#include "mesh_host.h"

// Launch shape of the far-field kernel: minimum resident CTAs per SM (which
// caps registers per thread) and the unroll depth of the source-point loop.
#ifndef EB_F32_MINB
#define EB_F32_MINB 2
#endif
#ifndef EB_F64_MINB
#define EB_F64_MINB 2
#endif
#ifndef EB_UNROLL_B_F32
#define EB_UNROLL_B_F32 0  // 0: unroll fully when the rule size is a compile-time constant
#endif
#ifndef EB_UNROLL_B_F64
#define EB_UNROLL_B_F64 0  // FP64 variants with at most two outputs; wider ones keep a rolled loop
#endif
#ifndef EB_UNROLL_WIDE_F64
#define EB_UNROLL_WIDE_F64 1  // FP64 variants with three or more outputs
#endif
#ifndef EB_UNROLL_B_X2
#define EB_UNROLL_B_X2 0  // source-point unroll of the packed FP32 form (0: full)
#endif

namespace eb {

constexpr int kUnrollF32 = EB_UNROLL_B_F32;
constexpr int kUnrollF64 = EB_UNROLL_B_F64;
constexpr int kUnrollX2 = EB_UNROLL_B_X2;

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
// One MUFU.RSQ (the argument is a squared distance, never denormal).
__device__ __forceinline__ float rsq(float x)
{
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double rsq(double x) { return rsqrt(x); }

// FP64 1/sqrt: the PTX approximation refined by one Halley step
// (y' = y (1 + e/2 + 3e^2/8), e = 1 - x y^2), cubic convergence.
__device__ __forceinline__ double rsq_f64(double x)
{
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  const double e = fma(-x * y, y, 1.0);
  return fma(y * e, fma(0.375, e, 0.5), y);
}

// One target item (K points) against the source triangles [s0, s1) of one
// cell of the staged tile. Per quadrature-point pair:
//   SL:  sl[c][a] += c_c(b) / r
//   DL:  acc[a]   += s(b) / r^3          (per source triangle)
// and per source triangle dl[a] += d(a, j) * acc[a], where d(a, j) =
// (x_a - y).n_j is the signed distance of x_a from the plane of triangle j
// (the same for every y in it), evaluated as d = (x_a - c_i).(n_j - n_i) +
// (c_i.n_j - P0_j.n_j) with the normal difference and the centroid term formed
// in FP64, so the small normal component is not lost to cancellation
// ((x_a - c_i) enters as the cell-relative point plus the cell offset o).
// FAR: cell well separated from the whole target tile (no vertex mask,
// expanded |x - y|^2, d from the cell-relative plane offset (P0_j - c_cell).n_j
// in the working precision); otherwise the shared-vertex mask and direct
// differences.
template <typename T, int K, int NQ, int NSL, int ND, bool FAR>
__device__ __forceinline__ void eval_cell(const typename Slot<T>::type* __restrict__ srec,
                                          const int4* __restrict__ svid, const dq* __restrict__ snrm,
                                          const typename Slot<T>::type* __restrict__ splane, int s0,
                                          int s1, int nq, int4 tv, const T (&x)[K], const T (&y)[K],
                                          const T (&z)[K], const T (&q2)[K], const T (&o)[3],
                                          const double (&cen)[3], const double (&nrm)[3],
                                          T (&sl)[NSL > 0 ? NSL : 1][K], T (&dl)[ND > 0 ? ND : 1][K])
{
  using S = typename Slot<T>::type;
  constexpr bool DL = ND > 0;
  constexpr int NDX = ND > 0 ? ND : 1;
  constexpr int NREC = rec_slots(NSL, ND);
  // the fully unrolled FP64 loop measured 5 % faster at L6 for SL+DL; with
  // three or more outputs its registers spill, so those variants stay rolled
  constexpr int kUnroll = std::is_same<T, float>::value ? kUnrollF32 : (NSL + ND <= 2 ? kUnrollF64 : EB_UNROLL_WIDE_F64);
  const int nqr = NQ > 0 ? NQ : nq;
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    if constexpr (!FAR) {
      if (shares_vertex(tv, svid[s])) continue;
    }
    const S* r = srec + (size_t)s * nqr * NREC;
    T acc[NDX][K];
#pragma unroll
    for (int a = 0; a < K; ++a)
#pragma unroll
      for (int c = 0; c < NDX; ++c) acc[c][a] = 0;
#pragma unroll(NQ > 0 ? (kUnroll > 0 ? kUnroll : NQ) : 1)
    for (int b = 0; b < nqr; ++b) {
      const S p0 = r[b * NREC];
      const S p1 = r[b * NREC + 1];
#pragma unroll
      for (int a = 0; a < K; ++a) {
        T r2;
        if constexpr (FAR) {
          r2 = x[a] * p0.x + (y[a] * p0.y + (z[a] * p0.z + (q2[a] + p0.w)));
        } else {
          const T dx = x[a] + T(0.5) * p0.x, dy = y[a] + T(0.5) * p0.y, dz = z[a] + T(0.5) * p0.z;
          r2 = dx * dx + dy * dy + dz * dz;
        }
        T inv;
        if constexpr (std::is_same<T, float>::value) inv = rsq(r2);
        else inv = rsq_f64(r2);
#pragma unroll
        for (int c = 0; c < NSL; ++c) {
          const int slot = charge_slot(c, ND);
          sl[c][a] += comp(slot == 1 ? p1 : r[b * NREC + slot], charge_comp(c, ND)) * inv;
        }
        if constexpr (ND == 1) {
          acc[0][a] += (inv * inv) * (p1.x * inv);
        } else if constexpr (ND > 1) {
          const T inv3 = (inv * inv) * inv;
#pragma unroll
          for (int c = 0; c < ND; ++c) acc[c][a] += comp(p1, c) * inv3;
        }
      }
    }
    if constexpr (DL && FAR) {
      // well-separated pair: d = (x_a - c_cell).n_j - (P0_j - c_cell).n_j
      const typename Slot<T>::type pn = splane[s];
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const T d = x[a] * pn.x + (y[a] * pn.y + (z[a] * pn.z - pn.w));
#pragma unroll
        for (int c = 0; c < ND; ++c) dl[c][a] += d * acc[c][a];
      }
    } else if constexpr (DL) {
      // x_a - c_i = (x_a - c_cell) + o with o = c_cell - c_i
      const dq nj = snrm[s];
      const T dnx = (T)(nj.x - nrm[0]), dny = (T)(nj.y - nrm[1]), dnz = (T)(nj.z - nrm[2]);
      const T e = (T)(cen[0] * nj.x + cen[1] * nj.y + cen[2] * nj.z - nj.w) + (o[0] * dnx + (o[1] * dny + o[2] * dnz));
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const T d = x[a] * dnx + (y[a] * dny + (z[a] * dnz + e));
#pragma unroll
        for (int c = 0; c < ND; ++c) dl[c][a] += d * acc[c][a];
      }
    }
  }
}

// Packed FP32 form of eval_cell for sm_100 (FFMA2: two FP32 FMAs per issue).
// Target points are taken in pairs ({x_a, x_a+1}) and every source value is
// broadcast to both halves ({v, v}), so one pair-instruction evaluates one
// source point against two target points. Per source point and target pair:
// 1 FADD2 + 3 FFMA2 for |x - y|^2 (far cells) or 3 FFMA2 + 1 FMUL2 + 2 FFMA2
// (near cells), 2 MUFU.RSQ, 1 FFMA2 per SL charge and 2 FMUL2 + 1 FFMA2 for
// the DL sum; an odd last target point runs the scalar form. Each lane of a
// pair-instruction rounds exactly like the scalar FMA it replaces. The
// FMA-pipe work per quadrature pair is unchanged (FFMA2 occupies the pipe
// for two lanes' worth); the pair form halves the issue slots, which bound
// the scalar loop.
template <int K, int NQ, int NSL, int ND, bool FAR>
__device__ __forceinline__ void eval_cell_x2(const float* __restrict__ srec, const int4* __restrict__ svid,
                                             const dq* __restrict__ snrm, const float4* __restrict__ splane, int s0,
                                             int s1, int nq, int4 tv, const float (&x)[K], const float (&y)[K],
                                             const float (&z)[K], const float (&q2)[K], const float (&o)[3],
                                             const double (&cen)[3], const double (&nrm)[3],
                                             float (&sl)[NSL > 0 ? NSL : 1][K], float (&dl)[ND > 0 ? ND : 1][K])
{
  constexpr bool DL = ND > 0;
  constexpr int NDX = ND > 0 ? ND : 1;
  constexpr int NREC = rec_slots(NSL, ND);
  constexpr int NS = NSL > 0 ? NSL : 1;
  constexpr int KP = K / 2;           // packed target pairs
  constexpr int KP1 = KP > 0 ? KP : 1;
  constexpr bool ODD = (K & 1) != 0;  // last target point runs scalar
  constexpr int PS = 4 * NREC;        // staged floats per source point
  const int nqr = NQ > 0 ? NQ : nq;
  float2 X[KP1], Y[KP1], Z[KP1], W[KP1], SL[NS][KP1], DLp[NDX][KP1];
#pragma unroll
  for (int p = 0; p < KP; ++p) {
    X[p] = make_float2(x[2 * p], x[2 * p + 1]);
    Y[p] = make_float2(y[2 * p], y[2 * p + 1]);
    Z[p] = make_float2(z[2 * p], z[2 * p + 1]);
    W[p] = make_float2(q2[2 * p], q2[2 * p + 1]);
#pragma unroll
    for (int c = 0; c < NDX; ++c) DLp[c][p] = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < NS; ++c) SL[c][p] = make_float2(0.f, 0.f);
  }
  const float2 half2 = make_float2(0.5f, 0.5f);
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    if constexpr (!FAR) {
      if (shares_vertex(tv, svid[s])) continue;
    }
    const float* r = srec + (size_t)s * nqr * PS;
    float2 acc2[NDX][KP1];
    float acc1[NDX];
#pragma unroll
    for (int c = 0; c < NDX; ++c) {
      acc1[c] = 0.f;
#pragma unroll
      for (int p = 0; p < KP; ++p) acc2[c][p] = make_float2(0.f, 0.f);
    }
#pragma unroll(NQ > 0 ? (kUnrollX2 > 0 ? kUnrollX2 : NQ) : 1)
    for (int b = 0; b < nqr; ++b) {
      const float* rb = r + b * PS;
      const float4* rv = reinterpret_cast<const float4*>(rb);
      const float4 p0 = rv[0];
      const float2 px = make_float2(p0.x, p0.x), py = make_float2(p0.y, p0.y);
      const float2 pz = make_float2(p0.z, p0.z), pw = make_float2(p0.w, p0.w);
      float2 ch[NS];
#pragma unroll
      for (int c = 0; c < NSL; ++c) {
        const float v = comp(rv[charge_slot(c, ND)], charge_comp(c, ND));
        ch[c] = make_float2(v, v);
      }
      float2 sd[NDX];
#pragma unroll
      for (int c = 0; c < NDX; ++c) {
        const float v = DL ? comp(rv[1], c) : 0.f;
        sd[c] = make_float2(v, v);
      }
#pragma unroll
      for (int p = 0; p < KP; ++p) {
        float2 r2;
        if constexpr (FAR) {
          r2 = __ffma2_rn(X[p], px, __ffma2_rn(Y[p], py, __ffma2_rn(Z[p], pz, __fadd2_rn(W[p], pw))));
        } else {
          const float2 dx = __ffma2_rn(half2, px, X[p]);
          const float2 dy = __ffma2_rn(half2, py, Y[p]);
          const float2 dz = __ffma2_rn(half2, pz, Z[p]);
          r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
        }
        const float2 inv = make_float2(rsq(r2.x), rsq(r2.y));
#pragma unroll
        for (int c = 0; c < NSL; ++c) SL[c][p] = __ffma2_rn(ch[c], inv, SL[c][p]);
        if constexpr (ND == 1) {
          acc2[0][p] = __ffma2_rn(__fmul2_rn(inv, inv), __fmul2_rn(sd[0], inv), acc2[0][p]);
        } else if constexpr (ND > 1) {
          const float2 inv3 = __fmul2_rn(__fmul2_rn(inv, inv), inv);
#pragma unroll
          for (int c = 0; c < ND; ++c) acc2[c][p] = __ffma2_rn(sd[c], inv3, acc2[c][p]);
        }
      }
      if constexpr (ODD) {
        constexpr int a = K - 1;
        float r2;
        if constexpr (FAR) {
          r2 = x[a] * px.x + (y[a] * py.x + (z[a] * pz.x + (q2[a] + pw.x)));
        } else {
          const float dx = x[a] + 0.5f * px.x, dy = y[a] + 0.5f * py.x, dz = z[a] + 0.5f * pz.x;
          r2 = dx * dx + dy * dy + dz * dz;
        }
        const float inv = rsq(r2);
#pragma unroll
        for (int c = 0; c < NSL; ++c) sl[c][a] += ch[c].x * inv;
        if constexpr (ND == 1) {
          acc1[0] += (inv * inv) * (sd[0].x * inv);
        } else if constexpr (ND > 1) {
          const float inv3 = (inv * inv) * inv;
#pragma unroll
          for (int c = 0; c < ND; ++c) acc1[c] += sd[c].x * inv3;
        }
      }
    }
    if constexpr (DL) {
      // d = signed distance of each target point from the plane of triangle s
      float pnx, pny, pnz, pnw;
      if constexpr (FAR) {
        const float4 pn = splane[s];
        pnx = pn.x; pny = pn.y; pnz = pn.z; pnw = -pn.w;
      } else {
        const dq nj = snrm[s];
        pnx = (float)(nj.x - nrm[0]); pny = (float)(nj.y - nrm[1]); pnz = (float)(nj.z - nrm[2]);
        pnw = (float)(cen[0] * nj.x + cen[1] * nj.y + cen[2] * nj.z - nj.w) + (o[0] * pnx + (o[1] * pny + o[2] * pnz));
      }
      const float2 nx = make_float2(pnx, pnx), ny = make_float2(pny, pny), nz = make_float2(pnz, pnz);
      const float2 nw = make_float2(pnw, pnw);
#pragma unroll
      for (int p = 0; p < KP; ++p) {
        const float2 d = __ffma2_rn(X[p], nx, __ffma2_rn(Y[p], ny, __ffma2_rn(Z[p], nz, nw)));
#pragma unroll
        for (int c = 0; c < ND; ++c) DLp[c][p] = __ffma2_rn(d, acc2[c][p], DLp[c][p]);
      }
      if constexpr (ODD) {
        constexpr int a = K - 1;
        const float d = x[a] * pnx + (y[a] * pny + (z[a] * pnz + pnw));
#pragma unroll
        for (int c = 0; c < ND; ++c) dl[c][a] += d * acc1[c];
      }
    }
  }
#pragma unroll
  for (int p = 0; p < KP; ++p) {
#pragma unroll
    for (int c = 0; c < NS; ++c) {
      sl[c][2 * p] += SL[c][p].x;
      sl[c][2 * p + 1] += SL[c][p].y;
    }
#pragma unroll
    for (int c = 0; c < ND; ++c) {
      dl[c][2 * p] += DLp[c][p].x;
      dl[c][2 * p + 1] += DLp[c][p].y;
    }
  }
}

// P1T: P1 test functions; the item's three outputs are sum_a w_a phi_k(x_a) acc_a
// (k = 0, 1, 2 in the triangle's vertex order) of the single SL charge.
template <typename T, int K, int NQ, int NSL, int ND, bool P1T>
__global__ void __launch_bounds__(kTT, std::is_same<T, float>::value ? EB_F32_MINB : EB_F64_MINB)
    far_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
               int* __restrict__ counter)
{
  using S = typename Slot<T>::type;
  constexpr bool F32 = std::is_same<T, float>::value;
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
    const dq tile = md.ttile[w.tgt0 / kTT];

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
    const int ts = md.src_tile;
    const S* grec = reinterpret_cast<const S*>(md.rec);
    for (int t0 = sb; t0 < se; t0 += ts) {
      const int ns = min(ts, se - t0);
      const S* g = grec + (size_t)t0 * nq * NREC;
      const int nslot = ns * nq * NREC;
      for (int k = threadIdx.x; k < nslot; k += kTT) s_rec[k] = g[k];
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
          // warp-uniform (tile-level) separation test
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
          if constexpr (F32) {
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
    const int nparts = A.nsplit * A.nchunk;
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
