// Device-side evaluation of the far-field quadrature pairs of one cell
// (scalar and packed FFMA2 forms), shared by the CUDA-core far kernel
// (farfield.cu) and the near cells of the tensor-core kernel
// (farfield_tc.cu). See farfield.cuh for the formulation.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "farfield.cuh"

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
#define EB_UNROLL_B_X2 0  // source-point unroll of the packed FP32 forms (0: full)
#endif
#ifndef EB_FAR_SP
#define EB_FAR_SP 1  // FP32 far kernel: 1 pairs source triangles (eval_cell_sp), 0 pairs target points (eval_cell_x2)
#endif

namespace eb {

constexpr int kUnrollF32 = EB_UNROLL_B_F32;
constexpr int kUnrollF64 = EB_UNROLL_B_F64;
constexpr int kUnrollX2 = EB_UNROLL_B_X2;
constexpr bool kFarSourcePairs = EB_FAR_SP != 0;

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

// Source-pair layout of a staged FP32 tile: triangles 2p and 2p+1 of the tile
// share one record of 2 * NREC float4 per quadrature point, in which record
// slot k occupies float4 2k and 2k+1 as (c0, c0', c1, c1') and (c2, c2', c3,
// c3') (unprimed: triangle 2p, primed: 2p+1). An odd last triangle is paired
// with a zero-strength dummy at (-2y, |y|^2) = (0, 0, 0, 1). Component c of
// slot k of both triangles, as one FFMA2 operand:
__device__ __forceinline__ float2 sp_comp(const float4* rv, int slot, int c)
{
  const float4 v = rv[2 * slot + (c >> 1)];
  return (c & 1) ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
}

// eval_cell over a source-pair tile: the two lanes of every FFMA2 are the same
// target point against the same quadrature point of triangles s and s+1, so
// each target value is broadcast once per cell (not per source point), each
// LDS.128 lands in aligned register pairs, and every target point runs packed.
// Per lane the arithmetic and its rounding are those of eval_cell_x2 (far
// cells: expanded |x - y|^2; other cells: direct differences); the SL and DL
// sums of the two lanes are added per cell. Other cells mask a lane whose
// triangle shares a vertex with the target by zeroing its strengths, and add
// 1e-24 to |x - y|^2 so the target triangle's own (zero-strength) points give
// 0 * finite: 1/r = 1e12 and 1/r^3 = 1e36 stay below the FP32 maximum, and the
// term changes no squared distance above 1.7e-17 (points 4e-9 apart). s0 is
// even; s1 - s0 may be odd at the end of the mesh, where the staged dummy
// completes the last pair.
template <int K, int NQ, int NSL, int ND, bool FAR>
__device__ __forceinline__ void eval_cell_sp(const float4* __restrict__ srec, const int4* __restrict__ svid,
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
  const int nqr = NQ > 0 ? NQ : nq;
  float2 X[K], Y[K], Z[K], W[K], SL[NS][K], DLp[NDX][K];
#pragma unroll
  for (int a = 0; a < K; ++a) {
    X[a] = make_float2(x[a], x[a]);
    Y[a] = make_float2(y[a], y[a]);
    Z[a] = make_float2(z[a], z[a]);
    W[a] = make_float2(q2[a], q2[a]);
#pragma unroll
    for (int c = 0; c < NDX; ++c) DLp[c][a] = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < NS; ++c) SL[c][a] = make_float2(0.f, 0.f);
  }
  const float2 half2 = make_float2(0.5f, 0.5f);
  const float2 eps2 = make_float2(1e-24f, 1e-24f);
#pragma unroll 1
  for (int s = s0; s < s1; s += 2) {
    float2 keep = make_float2(1.f, 1.f);
    if constexpr (!FAR) {
      const bool m0 = shares_vertex(tv, svid[s]), m1 = shares_vertex(tv, svid[s + 1]);
      if (m0 && m1) continue;
      keep = make_float2(m0 ? 0.f : 1.f, m1 ? 0.f : 1.f);
    }
    const float4* r = srec + (size_t)(s >> 1) * nqr * NREC * 2;
    float2 acc2[NDX][K];
#pragma unroll
    for (int c = 0; c < NDX; ++c)
#pragma unroll
      for (int a = 0; a < K; ++a) acc2[c][a] = make_float2(0.f, 0.f);
    // four DL columns hold 4 x K packed sums per pair: their loop stays rolled (no spills)
#pragma unroll(NQ > 0 ? (kUnrollX2 > 0 ? kUnrollX2 : (ND >= 4 ? 1 : NQ)) : 1)
    for (int b = 0; b < nqr; ++b) {
      const float4* rv = r + b * NREC * 2;
      const float2 px = sp_comp(rv, 0, 0), py = sp_comp(rv, 0, 1), pz = sp_comp(rv, 0, 2), pw = sp_comp(rv, 0, 3);
      float2 ch[NS], sd[NDX];
#pragma unroll
      for (int c = 0; c < NSL; ++c) {
        ch[c] = sp_comp(rv, charge_slot(c, ND), charge_comp(c, ND));
        if constexpr (!FAR) ch[c] = __fmul2_rn(ch[c], keep);
      }
#pragma unroll
      for (int c = 0; c < ND; ++c) {
        sd[c] = sp_comp(rv, 1 + c / 4, c % 4);
        if constexpr (!FAR) sd[c] = __fmul2_rn(sd[c], keep);
      }
#pragma unroll
      for (int a = 0; a < K; ++a) {
        float2 r2;
        if constexpr (FAR) {
          r2 = __ffma2_rn(X[a], px, __ffma2_rn(Y[a], py, __ffma2_rn(Z[a], pz, __fadd2_rn(W[a], pw))));
        } else {
          const float2 dx = __ffma2_rn(half2, px, X[a]);
          const float2 dy = __ffma2_rn(half2, py, Y[a]);
          const float2 dz = __ffma2_rn(half2, pz, Z[a]);
          r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
        }
        const float2 inv = make_float2(rsq(r2.x), rsq(r2.y));
#pragma unroll
        for (int c = 0; c < NSL; ++c) SL[c][a] = __ffma2_rn(ch[c], inv, SL[c][a]);
        if constexpr (ND == 1) {
          acc2[0][a] = __ffma2_rn(__fmul2_rn(inv, inv), __fmul2_rn(sd[0], inv), acc2[0][a]);
        } else if constexpr (ND > 1) {
          const float2 inv3 = __fmul2_rn(__fmul2_rn(inv, inv), inv);
#pragma unroll
          for (int c = 0; c < ND; ++c) acc2[c][a] = __ffma2_rn(sd[c], inv3, acc2[c][a]);
        }
      }
    }
    if constexpr (DL) {
      // d = signed distance of each target point from the planes of triangles s, s+1
      float2 nx, ny, nz, nw;
      if constexpr (FAR) {
        const float4 p0 = splane[s], p1 = splane[s + 1];
        nx = make_float2(p0.x, p1.x); ny = make_float2(p0.y, p1.y); nz = make_float2(p0.z, p1.z);
        nw = make_float2(-p0.w, -p1.w);
      } else {
        float pn[2][4];
#pragma unroll
        for (int l = 0; l < 2; ++l) {
          const dq nj = snrm[s + l];
          const float dnx = (float)(nj.x - nrm[0]), dny = (float)(nj.y - nrm[1]), dnz = (float)(nj.z - nrm[2]);
          pn[l][0] = dnx; pn[l][1] = dny; pn[l][2] = dnz;
          pn[l][3] = (float)(cen[0] * nj.x + cen[1] * nj.y + cen[2] * nj.z - nj.w) + (o[0] * dnx + (o[1] * dny + o[2] * dnz));
        }
        nx = make_float2(pn[0][0], pn[1][0]); ny = make_float2(pn[0][1], pn[1][1]);
        nz = make_float2(pn[0][2], pn[1][2]); nw = make_float2(pn[0][3], pn[1][3]);
      }
#pragma unroll
      for (int a = 0; a < K; ++a) {
        const float2 d = __ffma2_rn(X[a], nx, __ffma2_rn(Y[a], ny, __ffma2_rn(Z[a], nz, nw)));
#pragma unroll
        for (int c = 0; c < ND; ++c) DLp[c][a] = __ffma2_rn(d, acc2[c][a], DLp[c][a]);
      }
    }
  }
#pragma unroll
  for (int a = 0; a < K; ++a) {
#pragma unroll
    for (int c = 0; c < NSL; ++c) sl[c][a] += SL[c][a].x + SL[c][a].y;
#pragma unroll
    for (int c = 0; c < ND; ++c) dl[c][a] += DLp[c][a].x + DLp[c][a].y;
  }
}

}  // namespace eb
