// Symmetric far field of the fused FP32 SL+DL apply (7-point rule).
//
// The regular quadrature puts the same Q-point rule on the test and on the
// trial triangle (src/BEM3dLaplace.cpp:406-437 evaluates the SL and DL
// integrands of a disjoint pair at the test rule's points x_a and the trial
// rule's points y_b; src/BEM3dLaplaceGPU.cu:445-488 and :775-827 do the same
// per thread). So the kernel values of a point pair, r = 1/|x_a - y_b| and
// r^3, serve both orders of its triangle pair (i, j):
//
//   row i (test i, trial j):  c_b r            + d_j(x_a) s_b r^3
//   row j (test j, trial i):  c_a r            + e_i(y_b) s_a r^3
//
// with c = w J t the SL charges and s = w J u_h the DL strengths of the
// points, d_j(x) = (x - P0_j).n_j the signed distance of x from the plane of
// triangle j and e_i(y) = (y - P0_i).n_i that of y from the plane of i. Each
// unordered pair is evaluated once: one MUFU rsqrt and 9 FMA-pipe lane
// operations (1 add + 3 FMA for |x - y|^2, 2 mul for r^3, 1 FMA for the
// single-layer sum R_a = sum_b w_b r that both rows share, 2 FMA for the
// double-layer sums of the two rows) instead of 2 rsqrt and 16 for the two
// ordered pairs.
//
// Work items of the symmetric plan (tiles of kTT = 128 sorted triangles, cells
// of kCell = 32):
//   * diagonal item of tile T: the tile against its own four cells, every
//     ordered pair (forward only, the CUDA-core kernel's eval_cell_sp);
//     forward sums to partial slot T of its rows;
//   * upper item of tile T: the tile against a range of cells after it; its
//     forward sums go to slot split = T + 1 + r of its target rows, its
//     transposed sums to slot T of its source rows.
// A row of tile T thus receives one slot per earlier tile (their transposed
// sums), slot T and one slot per upper item of its own tile. Every slot is
// written by exactly one item and the finalize adds them in slot order, so
// the result is bitwise reproducible.
//
// The transposed sums of a staged tile are reduced over the CTA's 128 target
// threads through shared memory (one float4 per thread and source-triangle
// pair, added in thread order).
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "farfield.cuh"
#include "farfield_eval.cuh"
#include "farfield_sym.h"
#include "mesh_host.h"

// Source-point unroll of the symmetric pair loop (0: full).
#ifndef EB_SYM_UNROLL_B
#define EB_SYM_UNROLL_B 0
#endif
// Source-point unroll of the FP64 symmetric loop (0: full).
#ifndef EB_SYM_UNROLL_B64
#define EB_SYM_UNROLL_B64 0
#endif
// Source cells per upper work item (even; 256 source triangles by default).
#ifndef EB_SYM_CELLS
#define EB_SYM_CELLS 8
#endif

namespace eb {

namespace {

constexpr int kQ = kSymRule;
constexpr int kUnrollB = EB_SYM_UNROLL_B > 0 ? EB_SYM_UNROLL_B : kQ;
constexpr int kNrec = 2;                     // rec_slots(1, 1): (-2y, |y|^2), (s, c, 0, 0)
constexpr int kPairs = kTS / 2;              // source-triangle pairs per staged tile
constexpr int kRedStride = kPairs + 1;       // float4 per thread row of the reduction buffer (padded)
constexpr size_t kRecBytes = (size_t)kTS * kQ * kNrec * 16;
constexpr size_t kRedBytes = (size_t)kTT * kRedStride * 16;
constexpr int kRed64Stride = kCell + 1;      // double2 per thread row of the FP64 reduction buffer (padded)
constexpr size_t kRec64Bytes = (size_t)kCell * kQ * kNrec * 32;
constexpr size_t kRed64Bytes = (size_t)kTT * kRed64Stride * 16;
constexpr int kUnrollB64 = EB_SYM_UNROLL_B64 > 0 ? EB_SYM_UNROLL_B64 : kQ;
static_assert(kTT == 4 * kCell, "a target tile is four cells");
static_assert(kTS == 2 * kCell, "a staged tile is two cells");
static_assert(kPairs * 4 == kTT, "one reduction output per thread");

__device__ __forceinline__ float2 bcast(float v) { return make_float2(v, v); }


// One target triangle (kQ points, relative to the cell centre) against the
// source triangles [s0, s1) of one cell of the staged pair-interleaved tile,
// both orders of every pair. Forward sums: the single layer as one sum
// already weighted by the target points' rule weights (slw), the double
// layer per target point (dl, as eval_cell_sp); the transposed sums of
// source triangles s, s+1 go to red[s / 2] as (SL s, SL s+1, DL s, DL s+1),
// weighted by the source points' rule weights w_b (the finalize multiplies a
// row by J / 4 pi).
//
// Single layer: both charges factor as c = w J t, so one sum per target
// point, R_a = sum_b w_b / r_ab, serves both rows: row i gets J_j t_j
// sum_a w_a R_a, row j gets sum_a c_a R_a (1 FMA per pair instead of 2).
//
// Far cells: expanded |x - y|^2 and e_i(y) = (y - c).n_i + (c - P0_i).n_i;
// other cells: direct differences, a 1e-24 floor and, per lane, e_i(y) =
// (y - c).(n_i - n_j) + (P0_j.n_j - P0_i.n_i) + c.(n_i - n_j) (exact for y in
// the plane of j; the normal difference keeps e small and accurate for
// nearly coplanar neighbours); lanes whose triangle shares a vertex with the
// target get zero strengths and zero transposed sums.
template <bool FAR>
__device__ __forceinline__ void eval_cell_sym(const float4* __restrict__ srec, const int4* __restrict__ svid,
                                              const dq* __restrict__ snrm, const float4* __restrict__ splane, int s0,
                                              int s1, int4 tv, const float (&x)[kQ], const float (&y)[kQ],
                                              const float (&z)[kQ], const float (&q2)[kQ], const float (&ca)[kQ],
                                              const float (&cd)[kQ], const float (&wq)[kQ], const float (&o)[3],
                                              const double (&cen)[3], const double (&nrm)[3],
                                              const double (&cc)[3], double pin, float& slw, float (&dl)[kQ],
                                              float4* __restrict__ red)
{
  float2 X[kQ], Y[kQ], Z[kQ], W[kQ], DLp[kQ];
  float2 SLW = make_float2(0.f, 0.f);
#pragma unroll
  for (int a = 0; a < kQ; ++a) {
    X[a] = bcast(x[a]);
    Y[a] = bcast(y[a]);
    Z[a] = bcast(z[a]);
    W[a] = bcast(q2[a]);
    DLp[a] = make_float2(0.f, 0.f);
  }
  const float2 half2 = bcast(0.5f);
  const float2 eps2 = bcast(1e-24f);
  // plane of the target triangle seen from the cell centre (far cells)
  float2 EX, EY, EZ, EW;
  if constexpr (FAR) {
    EX = bcast(-0.5f * (float)nrm[0]);
    EY = bcast(-0.5f * (float)nrm[1]);
    EZ = bcast(-0.5f * (float)nrm[2]);
    EW = bcast((float)(cc[0] * nrm[0] + cc[1] * nrm[1] + cc[2] * nrm[2] - pin));
  }
#pragma unroll 1
  for (int s = s0; s < s1; s += 2) {
    float2 keep = make_float2(1.f, 1.f);
    if constexpr (!FAR) {
      const bool m0 = shares_vertex(tv, svid[s]), m1 = shares_vertex(tv, svid[s + 1]);
      if (m0 && m1) {
        red[s >> 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        continue;
      }
      keep = make_float2(m0 ? 0.f : 1.f, m1 ? 0.f : 1.f);
      float e[2][4];
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        const dq nj = snrm[s + l];
        const double dnx = nrm[0] - nj.x, dny = nrm[1] - nj.y, dnz = nrm[2] - nj.z;
        e[l][0] = (float)(-0.5 * dnx);
        e[l][1] = (float)(-0.5 * dny);
        e[l][2] = (float)(-0.5 * dnz);
        e[l][3] = (float)((nj.w - pin) + (cc[0] * dnx + cc[1] * dny + cc[2] * dnz));
      }
      EX = make_float2(e[0][0], e[1][0]);
      EY = make_float2(e[0][1], e[1][1]);
      EZ = make_float2(e[0][2], e[1][2]);
      EW = make_float2(e[0][3], e[1][3]);
    }
    const float4* r = srec + (size_t)(s >> 1) * kQ * kNrec * 2;
    float2 tj = sp_comp(r, 1, 2);  // J_j t_j of both triangles
    if constexpr (!FAR) tj = __fmul2_rn(tj, keep);
    float2 acc2[kQ], R[kQ];
#pragma unroll
    for (int a = 0; a < kQ; ++a) {
      acc2[a] = make_float2(0.f, 0.f);
      R[a] = make_float2(0.f, 0.f);
    }
    float2 Q2 = make_float2(0.f, 0.f);
#pragma unroll(kUnrollB)
    for (int b = 0; b < kQ; ++b) {
      const float4* rv = r + b * kNrec * 2;
      const float2 px = sp_comp(rv, 0, 0), py = sp_comp(rv, 0, 1), pz = sp_comp(rv, 0, 2), pw = sp_comp(rv, 0, 3);
      float2 sd = sp_comp(rv, 1, 0);
      if constexpr (!FAR) sd = __fmul2_rn(sd, keep);
      const float2 wb = bcast(wq[b]);
      float2 td = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
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
        const float2 inv3 = __fmul2_rn(__fmul2_rn(inv, inv), inv);
        R[a] = __ffma2_rn(wb, inv, R[a]);
        acc2[a] = __ffma2_rn(sd, inv3, acc2[a]);
        td.x = fmaf(cd[a], inv3.x, td.x);
        td.y = fmaf(cd[a], inv3.y, td.y);
      }
      // e_i(y_b) for both lanes; y_b - c = -(1/2)(-2 y_b)
      const float2 e = __ffma2_rn(px, EX, __ffma2_rn(py, EY, __ffma2_rn(pz, EZ, EW)));
      Q2 = __ffma2_rn(__fmul2_rn(wb, e), td, Q2);
    }
    // single layer of both rows from R_a
    float2 U = make_float2(0.f, 0.f), S2 = make_float2(0.f, 0.f);
#pragma unroll
    for (int a = 0; a < kQ; ++a) {
      U = __ffma2_rn(bcast(wq[a]), R[a], U);
      S2 = __ffma2_rn(bcast(ca[a]), R[a], S2);
    }
    SLW = __ffma2_rn(tj, U, SLW);
    if constexpr (!FAR) {
      S2 = __fmul2_rn(S2, keep);
      Q2 = __fmul2_rn(Q2, keep);
    }
    red[s >> 1] = make_float4(S2.x, S2.y, Q2.x, Q2.y);
    // forward double layer: d_j(x_a) times the pair's sums (as eval_cell_sp)
    float2 nx, ny, nz, nw;
    if constexpr (FAR) {
      const float4 p0 = splane[s], p1 = splane[s + 1];
      nx = make_float2(p0.x, p1.x);
      ny = make_float2(p0.y, p1.y);
      nz = make_float2(p0.z, p1.z);
      nw = make_float2(-p0.w, -p1.w);
    } else {
      float pn[2][4];
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        const dq nj = snrm[s + l];
        const float dnx = (float)(nj.x - nrm[0]), dny = (float)(nj.y - nrm[1]), dnz = (float)(nj.z - nrm[2]);
        pn[l][0] = dnx;
        pn[l][1] = dny;
        pn[l][2] = dnz;
        pn[l][3] = (float)(cen[0] * nj.x + cen[1] * nj.y + cen[2] * nj.z - nj.w) + (o[0] * dnx + (o[1] * dny + o[2] * dnz));
      }
      nx = make_float2(pn[0][0], pn[1][0]);
      ny = make_float2(pn[0][1], pn[1][1]);
      nz = make_float2(pn[0][2], pn[1][2]);
      nw = make_float2(pn[0][3], pn[1][3]);
    }
#pragma unroll
    for (int a = 0; a < kQ; ++a) {
      const float2 d = __ffma2_rn(X[a], nx, __ffma2_rn(Y[a], ny, __ffma2_rn(Z[a], nz, nw)));
      DLp[a] = __ffma2_rn(d, acc2[a], DLp[a]);
    }
  }
  slw += SLW.x + SLW.y;
#pragma unroll
  for (int a = 0; a < kQ; ++a) dl[a] += DLp[a].x + DLp[a].y;
}

__global__ void __launch_bounds__(kTT, 2)
    far_sym_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
                   int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kTS];
  __shared__ dq s_nrm[kTS];
  __shared__ float4 s_plane[kTS];
  float4* s_rec = reinterpret_cast<float4*>(smem_raw);
  float4* s_red = reinterpret_cast<float4*>(smem_raw + kRecBytes);
  float4* my_red = s_red + threadIdx.x * kRedStride;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;  // uniform across the CTA
    const bool upper = w.cell0 * kCell >= w.tgt0 + kTT;
    const int tslot = w.tgt0 / kTT;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    const dq tile = md.twarp[tsel / kWarpItems];
    double cen[3], nrm[3];
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
      const dq n = md.tnrm[tsel];
      nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
    }
    const double pin = md.snrm[tsel].w;  // P0_i . n_i
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);
    const float4* grec = reinterpret_cast<const float4*>(md.rec);
    float acc_hi[2] = {0.f, 0.f}, acc_lo[2] = {0.f, 0.f};
    const size_t stride = (size_t)md.nsplit * md.nitems;

    const int sb = w.cell0 * kCell;
    const int se = min(md.ne, w.cell1 * kCell);
    for (int t0 = sb; t0 < se; t0 += kTS) {
      const int ns = min(kTS, se - t0);
      {  // stage the tile in the source-pair layout (as the CUDA-core kernel)
        const float4* g = grec + (size_t)t0 * kQ * kNrec;
        constexpr int per = kQ * kNrec;
        const int nstage = ((ns + 1) >> 1) * per;
        for (int k = threadIdx.x; k < nstage; k += kTT) {
          const int p = k / per, rem = k - p * per;
          const float4 a = g[(size_t)(2 * p) * per + rem];
          float4 c;
          if (2 * p + 1 < ns) c = g[(size_t)(2 * p + 1) * per + rem];
          else c = rem % kNrec == 0 ? make_float4(0.f, 0.f, 0.f, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
          s_rec[2 * k] = make_float4(a.x, c.x, a.y, c.y);
          s_rec[2 * k + 1] = make_float4(a.z, c.z, a.w, c.w);
        }
        if ((ns & 1) && threadIdx.x == 0) {
          s_vid[ns] = make_int4(-1, -1, -1, 0);
          s_nrm[ns] = dq{0.0, 0.0, 0.0, 0.0};
          s_plane[ns] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        for (int k = threadIdx.x; k < ns; k += kTT) {
          s_vid[k] = md.svid[t0 + k];
          s_nrm[k] = md.snrm[t0 + k];
          s_plane[k] = md.splane32[t0 + k];
        }
      }
      __syncthreads();
      if (active) {
        for (int g0 = 0; g0 < ns;) {
          const int cell = (t0 + g0) / kCell;
          const int g1 = min(ns, (cell + 1) * kCell - t0);
          const dq ccd = md.ccent[cell];
          const double ddx = ccd.x - tile.x, ddy = ccd.y - tile.y, ddz = ccd.z - tile.z;
          const double rr = kFarRatio * (ccd.w + tile.w);
          const bool far = ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
          const float o[3] = {(float)(ccd.x - cen[0]), (float)(ccd.y - cen[1]), (float)(ccd.z - cen[2])};
          float xs[kQ], ys[kQ], zs[kQ], q2[kQ], wq[kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            const float4 p = md.tgt32[(size_t)tsel * kQ + a];
            xs[a] = p.x - o[0]; ys[a] = p.y - o[1]; zs[a] = p.z - o[2];
            q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
            wq[a] = p.w;
          }
          float sl[kQ], dl[kQ], slw = 0.f;
#pragma unroll
          for (int a = 0; a < kQ; ++a) { sl[a] = 0.f; dl[a] = 0.f; }
          if (upper) {
            float ca[kQ], cd[kQ];
#pragma unroll
            for (int a = 0; a < kQ; ++a) {
              const float4 st = grec[((size_t)tsel * kQ + a) * kNrec + 1];  // (s_a, c_a, 0, 0)
              cd[a] = st.x;
              ca[a] = st.y;
            }
            const double cc[3] = {ccd.x, ccd.y, ccd.z};
            if (far)
              eval_cell_sym<true>(s_rec, s_vid, s_nrm, s_plane, g0, g1, tv, xs, ys, zs, q2, ca, cd, wq, o, cen, nrm,
                                  cc, pin, slw, dl, my_red);
            else
              eval_cell_sym<false>(s_rec, s_vid, s_nrm, s_plane, g0, g1, tv, xs, ys, zs, q2, ca, cd, wq, o, cen,
                                   nrm, cc, pin, slw, dl, my_red);
          } else {
            float slc[1][kQ], dlc[1][kQ];
#pragma unroll
            for (int a = 0; a < kQ; ++a) { slc[0][a] = 0.f; dlc[0][a] = 0.f; }
            if (far)
              eval_cell_sp<kQ, kQ, 1, 1, true>(s_rec, s_vid, s_nrm, s_plane, g0, g1, kQ, tv, xs, ys, zs, q2, o, cen,
                                              nrm, slc, dlc);
            else
              eval_cell_sp<kQ, kQ, 1, 1, false>(s_rec, s_vid, s_nrm, s_plane, g0, g1, kQ, tv, xs, ys, zs, q2, o,
                                               cen, nrm, slc, dlc);
#pragma unroll
            for (int a = 0; a < kQ; ++a) { sl[a] = slc[0][a]; dl[a] = dlc[0][a]; }
          }
          float ps = slw, pd = 0.f;  // slw: the symmetric form's weighted SL sum (0 on the diagonal)
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            ps += wq[a] * sl[a];
            pd += wq[a] * dl[a];
          }
          two_sum_add(acc_hi[0], acc_lo[0], ps);
          two_sum_add(acc_hi[1], acc_lo[1], pd);
          g0 = g1;
        }
      } else if (upper) {
        for (int p = 0; p < kPairs; ++p) my_red[p] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (upper) {
        // transposed sums of the tile's source triangles: thread t adds
        // component t % 4 of pair t / 4 over the 128 target threads in order
        __syncthreads();
        const int p = threadIdx.x >> 2, c = threadIdx.x & 3;
        const int row = t0 + 2 * p + (c & 1);
        if (2 * p + (c & 1) < ns) {
          const float* rf = reinterpret_cast<const float*>(s_red) + p * 4 + c;
          float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
#pragma unroll 8
          for (int t = 0; t < kTT; t += 4) {
            v0 += rf[(t + 0) * kRedStride * 4];
            v1 += rf[(t + 1) * kRedStride * 4];
            v2 += rf[(t + 2) * kRedStride * 4];
            v3 += rf[(t + 3) * kRedStride * 4];
          }
          md.partial[(c >> 1) * stride + (size_t)tslot * md.nitems + row] = (double)((v0 + v1) + (v2 + v3));
        }
      }
      __syncthreads();
    }
    if (active) {
      double* out = md.partial + (size_t)w.split * md.nitems + ti;
      out[0] = (double)acc_hi[0] + (double)acc_lo[0];
      out[stride] = (double)acc_hi[1] + (double)acc_lo[1];
    }
  }
}

// FP64 form of eval_cell_sym (one source triangle at a time, the arithmetic
// of the FP64 ordered-pair kernel's eval_cell, the single layer through
// R_a): the transposed sums of triangle s go to red[s - s0] as (SL, DL).
template <bool FAR>
__device__ __forceinline__ void eval_cell_sym64(const dq* __restrict__ srec, const int4* __restrict__ svid,
                                                const dq* __restrict__ snrm, const dq* __restrict__ splane, int s0,
                                                int s1, int4 tv, const double (&x)[kQ], const double (&y)[kQ],
                                                const double (&z)[kQ], const double (&q2)[kQ],
                                                const double (&ca)[kQ], const double (&cd)[kQ],
                                                const double (&wq)[kQ], const double (&o)[3], const double (&cen)[3],
                                                const double (&nrm)[3], const double (&cc)[3], double pin,
                                                double& slw, double (&dl)[kQ], double2* __restrict__ red)
{
  double ex = 0.0, ey = 0.0, ez = 0.0, ew = 0.0;
  if constexpr (FAR) {
    ex = -0.5 * nrm[0];
    ey = -0.5 * nrm[1];
    ez = -0.5 * nrm[2];
    ew = cc[0] * nrm[0] + cc[1] * nrm[1] + cc[2] * nrm[2] - pin;
  }
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    dq nj;
    if constexpr (!FAR) {
      if (shares_vertex(tv, svid[s])) {
        red[s - s0] = make_double2(0.0, 0.0);
        continue;
      }
      nj = snrm[s];
      const double dnx = nrm[0] - nj.x, dny = nrm[1] - nj.y, dnz = nrm[2] - nj.z;
      ex = -0.5 * dnx;
      ey = -0.5 * dny;
      ez = -0.5 * dnz;
      ew = (nj.w - pin) + (cc[0] * dnx + cc[1] * dny + cc[2] * dnz);
    }
    const dq* r = srec + (size_t)s * kQ * kNrec;
    const double tj = r[1].z;  // J_j t_j
    double acc[kQ], R[kQ];
#pragma unroll
    for (int a = 0; a < kQ; ++a) {
      acc[a] = 0.0;
      R[a] = 0.0;
    }
    double Qt = 0.0;
#pragma unroll(kUnrollB64)
    for (int b = 0; b < kQ; ++b) {
      const dq p0 = r[b * kNrec];
      const dq p1 = r[b * kNrec + 1];  // (s_b, c_b, J_j t_j, 0)
      double td = 0.0;
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
        double r2;
        if constexpr (FAR) {
          r2 = x[a] * p0.x + (y[a] * p0.y + (z[a] * p0.z + (q2[a] + p0.w)));
        } else {
          const double dx = x[a] + 0.5 * p0.x, dy = y[a] + 0.5 * p0.y, dz = z[a] + 0.5 * p0.z;
          r2 = dx * dx + dy * dy + dz * dz;
        }
        const double inv = rsq_f64(r2);
        const double inv3 = (inv * inv) * inv;
        R[a] += wq[b] * inv;
        acc[a] += p1.x * inv3;
        td += cd[a] * inv3;
      }
      const double e = p0.x * ex + (p0.y * ey + (p0.z * ez + ew));
      Qt += (wq[b] * e) * td;
    }
    double U = 0.0, S = 0.0;
#pragma unroll
    for (int a = 0; a < kQ; ++a) {
      U += wq[a] * R[a];
      S += ca[a] * R[a];
    }
    slw += tj * U;
    red[s - s0] = make_double2(S, Qt);
    // forward double layer (as eval_cell)
    if constexpr (FAR) {
      const dq pn = splane[s];
#pragma unroll
      for (int a = 0; a < kQ; ++a) dl[a] += (x[a] * pn.x + (y[a] * pn.y + (z[a] * pn.z - pn.w))) * acc[a];
    } else {
      const double dnx = nj.x - nrm[0], dny = nj.y - nrm[1], dnz = nj.z - nrm[2];
      const double e0 = (cen[0] * nj.x + cen[1] * nj.y + cen[2] * nj.z - nj.w) + (o[0] * dnx + (o[1] * dny + o[2] * dnz));
#pragma unroll
      for (int a = 0; a < kQ; ++a) dl[a] += (x[a] * dnx + (y[a] * dny + (z[a] * dnz + e0))) * acc[a];
    }
  }
}

// FP64 symmetric far field: the FP32 kernel's work list and slots; source
// tiles of one cell (kCell triangles, FP64 records), the transposed sums
// reduced per cell over the 128 target threads in FP64.
__global__ void __launch_bounds__(kTT, 2)
    far_sym64_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
                     int* __restrict__ counter)
{
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kCell];
  __shared__ dq s_nrm[kCell];
  __shared__ dq s_plane[kCell];
  dq* s_rec = reinterpret_cast<dq*>(smem_raw);
  double2* s_red = reinterpret_cast<double2*>(smem_raw + kRec64Bytes);
  double2* my_red = s_red + threadIdx.x * kRed64Stride;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;  // uniform across the CTA
    const bool upper = w.cell0 * kCell >= w.tgt0 + kTT;
    const int tslot = w.tgt0 / kTT;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    const dq tile = md.twarp[tsel / kWarpItems];
    double cen[3], nrm[3];
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
      const dq n = md.tnrm[tsel];
      nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
    }
    const double pin = md.snrm[tsel].w;
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);
    const dq* grec = reinterpret_cast<const dq*>(md.rec);
    double acc_sl = 0.0, acc_dl = 0.0;
    const size_t stride = (size_t)md.nsplit * md.nitems;

    for (int cell = w.cell0; cell < w.cell1; ++cell) {
      const int t0 = cell * kCell;
      const int ns = min(kCell, md.ne - t0);
      {
        const dq* g = grec + (size_t)t0 * kQ * kNrec;
        const int nstage = ns * kQ * kNrec;
        for (int k = threadIdx.x; k < nstage; k += kTT) s_rec[k] = g[k];
        for (int k = threadIdx.x; k < ns; k += kTT) {
          s_vid[k] = md.svid[t0 + k];
          s_nrm[k] = md.snrm[t0 + k];
          s_plane[k] = md.splane64[t0 + k];
        }
      }
      __syncthreads();
      if (active) {
        const dq ccd = md.ccent[cell];
        const double ddx = ccd.x - tile.x, ddy = ccd.y - tile.y, ddz = ccd.z - tile.z;
        const double rr = kFarRatio * (ccd.w + tile.w);
        const bool far = ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
        const double o[3] = {ccd.x - cen[0], ccd.y - cen[1], ccd.z - cen[2]};
        double xs[kQ], ys[kQ], zs[kQ], q2[kQ], wq[kQ];
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          const dq p = md.tgt64[(size_t)tsel * kQ + a];
          xs[a] = p.x - o[0]; ys[a] = p.y - o[1]; zs[a] = p.z - o[2];
          q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
          wq[a] = p.w;
        }
        double sl[kQ], dl[kQ], slw = 0.0;
#pragma unroll
        for (int a = 0; a < kQ; ++a) { sl[a] = 0.0; dl[a] = 0.0; }
        if (upper) {
          double ca[kQ], cd[kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            const dq st = grec[((size_t)tsel * kQ + a) * kNrec + 1];  // (s_a, c_a, 0, 0)
            cd[a] = st.x;
            ca[a] = st.y;
          }
          const double cc[3] = {ccd.x, ccd.y, ccd.z};
          if (far)
            eval_cell_sym64<true>(s_rec, s_vid, s_nrm, s_plane, 0, ns, tv, xs, ys, zs, q2, ca, cd, wq, o, cen, nrm,
                                  cc, pin, slw, dl, my_red);
          else
            eval_cell_sym64<false>(s_rec, s_vid, s_nrm, s_plane, 0, ns, tv, xs, ys, zs, q2, ca, cd, wq, o, cen, nrm,
                                   cc, pin, slw, dl, my_red);
        } else {
          double slc[1][kQ], dlc[1][kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) { slc[0][a] = 0.0; dlc[0][a] = 0.0; }
          if (far)
            eval_cell<double, kQ, kQ, 1, 1, true>(s_rec, s_vid, s_nrm, s_plane, 0, ns, kQ, tv, xs, ys, zs, q2, o, cen,
                                                  nrm, slc, dlc);
          else
            eval_cell<double, kQ, kQ, 1, 1, false>(s_rec, s_vid, s_nrm, s_plane, 0, ns, kQ, tv, xs, ys, zs, q2, o,
                                                   cen, nrm, slc, dlc);
#pragma unroll
          for (int a = 0; a < kQ; ++a) { sl[a] = slc[0][a]; dl[a] = dlc[0][a]; }
        }
        double ps = slw, pd = 0.0;  // slw: the symmetric form's weighted SL sum (0 on the diagonal)
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          ps += wq[a] * sl[a];
          pd += wq[a] * dl[a];
        }
        acc_sl += ps;
        acc_dl += pd;
      } else if (upper) {
        for (int k = 0; k < kCell; ++k) my_red[k] = make_double2(0.0, 0.0);
      }
      if (upper) {
        // thread t < 2 kCell adds output t % 2 of source triangle t / 2 over
        // the 128 target threads in order
        __syncthreads();
        const int k = threadIdx.x >> 1, c = threadIdx.x & 1;
        if (threadIdx.x < 2 * kCell && k < ns) {
          const double* rf = reinterpret_cast<const double*>(s_red) + 2 * k + c;
          double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
#pragma unroll 8
          for (int t = 0; t < kTT; t += 4) {
            v0 += rf[(t + 0) * kRed64Stride * 2];
            v1 += rf[(t + 1) * kRed64Stride * 2];
            v2 += rf[(t + 2) * kRed64Stride * 2];
            v3 += rf[(t + 3) * kRed64Stride * 2];
          }
          md.partial[c * stride + (size_t)tslot * md.nitems + t0 + k] = (v0 + v1) + (v2 + v3);
        }
      }
      __syncthreads();
    }
    if (active) {
      double* out = md.partial + (size_t)w.split * md.nitems + ti;
      out[0] = acc_sl;
      out[stride] = acc_dl;
    }
  }
}

// Single-layer-only symmetric far field with NC right-hand sides (FP32): the
// batched solver's and the single-layer applies' variant. With no double
// layer, each unordered pair costs 1 MUFU rsqrt and 5 FMA-pipe operations
// (|x - y|^2 and R_a += (w_b / w_0) r), whatever NC: the charges of every
// column factor as c = w J t, so the columns differ only in the per-pair
// folds (row i: c_0 sum_a w_a R_a, with c_0 the source's first-point charge;
// row j: sum_a w_0 c_a R_a). Every column runs the same instructions in
// every NC, so a column's sums are the same bits alone or among 3 or 4.
constexpr int kSlPairs = kCell / 2;  // source-triangle pairs per staged cell
template <int NC>
__host__ __device__ constexpr int sl_red_stride() { return kSlPairs * NC + 1; }  // float2 per thread row (odd: conflict-free 8-byte stores)
template <int NC>
__host__ __device__ constexpr size_t sl_smem_bytes()
{
  return (size_t)kSlPairs * kQ * kNrec * 2 * 16 + (size_t)kTT * sl_red_stride<NC>() * 8;
}

template <int NC, bool FAR>
__device__ __forceinline__ void eval_cell_sym_sl(const float4* __restrict__ srec, const int4* __restrict__ svid,
                                                 int s0, int s1, int4 tv, const float (&x)[kQ],
                                                 const float (&y)[kQ], const float (&z)[kQ],
                                                 const float (&q2)[kQ], const float (&cw)[NC][kQ],
                                                 const float (&om)[kQ], const float (&wq)[kQ], float (&slw)[NC],
                                                 float2* __restrict__ red)
{
  float2 X[kQ], Y[kQ], Z[kQ], W[kQ];
#pragma unroll
  for (int a = 0; a < kQ; ++a) {
    X[a] = bcast(x[a]);
    Y[a] = bcast(y[a]);
    Z[a] = bcast(z[a]);
    W[a] = bcast(q2[a]);
  }
  float2 SLW[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) SLW[c] = make_float2(0.f, 0.f);
  const float2 half2 = bcast(0.5f);
  const float2 eps2 = bcast(1e-24f);
#pragma unroll 1
  for (int s = s0; s < s1; s += 2) {
    float2 keep = make_float2(1.f, 1.f);
    if constexpr (!FAR) {
      const bool m0 = shares_vertex(tv, svid[s]), m1 = shares_vertex(tv, svid[s + 1]);
      if (m0 && m1) {
#pragma unroll
        for (int c = 0; c < NC; ++c) red[(s >> 1) * NC + c] = make_float2(0.f, 0.f);
        continue;
      }
      keep = make_float2(m0 ? 0.f : 1.f, m1 ? 0.f : 1.f);
    }
    const float4* r = srec + (size_t)(s >> 1) * kQ * kNrec * 2;
    float2 R[kQ];
#pragma unroll
    for (int a = 0; a < kQ; ++a) R[a] = make_float2(0.f, 0.f);
#pragma unroll
    for (int b = 0; b < kQ; ++b) {
      const float4* rv = r + b * kNrec * 2;
      const float2 px = sp_comp(rv, 0, 0), py = sp_comp(rv, 0, 1), pz = sp_comp(rv, 0, 2), pw = sp_comp(rv, 0, 3);
      const float2 ob = bcast(om[b]);
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
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
        R[a] = __ffma2_rn(ob, inv, R[a]);
      }
    }
    float2 U = make_float2(0.f, 0.f);
#pragma unroll
    for (int a = 0; a < kQ; ++a) U = __ffma2_rn(bcast(wq[a]), R[a], U);
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      float2 c0 = sp_comp(r, 1, c);  // first-point charges of both triangles
      if constexpr (!FAR) c0 = __fmul2_rn(c0, keep);
      SLW[c] = __ffma2_rn(c0, U, SLW[c]);
      float2 S = make_float2(0.f, 0.f);
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
        S.x = fmaf(cw[c][a], R[a].x, S.x);
        S.y = fmaf(cw[c][a], R[a].y, S.y);
      }
      if constexpr (!FAR) S = __fmul2_rn(S, keep);
      red[(s >> 1) * NC + c] = S;
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) slw[c] += SLW[c].x + SLW[c].y;
}

template <int NC>
__global__ void __launch_bounds__(kTT, 2)
    far_sym_sl_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
                      int* __restrict__ counter)
{
  constexpr int kRow = sl_red_stride<NC>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kCell];
  float4* s_rec = reinterpret_cast<float4*>(smem_raw);
  float2* s_red = reinterpret_cast<float2*>(smem_raw + (size_t)kSlPairs * kQ * kNrec * 2 * 16);
  float2* my_red = s_red + threadIdx.x * kRow;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;  // uniform across the CTA
    const bool upper = w.cell0 * kCell >= w.tgt0 + kTT;
    const int tslot = w.tgt0 / kTT;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    const dq tile = md.twarp[tsel / kWarpItems];
    double cen[3];
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
    }
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);
    const float4* grec = reinterpret_cast<const float4*>(md.rec);
    float acc_hi[NC], acc_lo[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) { acc_hi[c] = 0.f; acc_lo[c] = 0.f; }
    const size_t stride = (size_t)md.nsplit * md.nitems;

    for (int cell = w.cell0; cell < w.cell1; ++cell) {
      const int t0 = cell * kCell;
      const int ns = min(kCell, md.ne - t0);
      {  // stage the cell in the source-pair layout
        const float4* g = grec + (size_t)t0 * kQ * kNrec;
        constexpr int per = kQ * kNrec;
        const int nstage = ((ns + 1) >> 1) * per;
        for (int k = threadIdx.x; k < nstage; k += kTT) {
          const int p = k / per, rem = k - p * per;
          const float4 a = g[(size_t)(2 * p) * per + rem];
          float4 c;
          if (2 * p + 1 < ns) c = g[(size_t)(2 * p + 1) * per + rem];
          else c = rem % kNrec == 0 ? make_float4(0.f, 0.f, 0.f, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
          s_rec[2 * k] = make_float4(a.x, c.x, a.y, c.y);
          s_rec[2 * k + 1] = make_float4(a.z, c.z, a.w, c.w);
        }
        if ((ns & 1) && threadIdx.x == 0) s_vid[ns] = make_int4(-1, -1, -1, 0);
        for (int k = threadIdx.x; k < ns; k += kTT) s_vid[k] = md.svid[t0 + k];
      }
      __syncthreads();
      if (active) {
        const dq ccd = md.ccent[cell];
        const double ddx = ccd.x - tile.x, ddy = ccd.y - tile.y, ddz = ccd.z - tile.z;
        const double rr = kFarRatio * (ccd.w + tile.w);
        const bool far = ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
        const float o[3] = {(float)(ccd.x - cen[0]), (float)(ccd.y - cen[1]), (float)(ccd.z - cen[2])};
        float xs[kQ], ys[kQ], zs[kQ], q2[kQ], wq[kQ];
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          const float4 p = md.tgt32[(size_t)tsel * kQ + a];
          xs[a] = p.x - o[0]; ys[a] = p.y - o[1]; zs[a] = p.z - o[2];
          q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
          wq[a] = p.w;
        }
        float part[NC];
        if (upper) {
          float cw[NC][kQ], om[kQ], slw[NC];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            om[a] = wq[a] / wq[0];
            const float4 st = grec[((size_t)tsel * kQ + a) * kNrec + 1];  // the target's charges c_a
#pragma unroll
            for (int c = 0; c < NC; ++c) cw[c][a] = wq[0] * comp(st, c);
          }
#pragma unroll
          for (int c = 0; c < NC; ++c) slw[c] = 0.f;
          if (far)
            eval_cell_sym_sl<NC, true>(s_rec, s_vid, 0, ns, tv, xs, ys, zs, q2, cw, om, wq, slw, my_red);
          else
            eval_cell_sym_sl<NC, false>(s_rec, s_vid, 0, ns, tv, xs, ys, zs, q2, cw, om, wq, slw, my_red);
#pragma unroll
          for (int c = 0; c < NC; ++c) part[c] = slw[c];
        } else {
          const dq* nul = nullptr;
          const double zero3[3] = {0.0, 0.0, 0.0};
          float slc[NC][kQ], dlc[1][kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
#pragma unroll
            for (int c = 0; c < NC; ++c) slc[c][a] = 0.f;
            dlc[0][a] = 0.f;
          }
          if (far)
            eval_cell_sp<kQ, kQ, NC, 0, true>(s_rec, s_vid, nul, nullptr, 0, ns, kQ, tv, xs, ys, zs, q2, o, cen,
                                             zero3, slc, dlc);
          else
            eval_cell_sp<kQ, kQ, NC, 0, false>(s_rec, s_vid, nul, nullptr, 0, ns, kQ, tv, xs, ys, zs, q2, o, cen,
                                              zero3, slc, dlc);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            part[c] = 0.f;
#pragma unroll
            for (int a = 0; a < kQ; ++a) part[c] += wq[a] * slc[c][a];
          }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) two_sum_add(acc_hi[c], acc_lo[c], part[c]);
      } else if (upper) {
        for (int k = 0; k < kSlPairs * NC; ++k) my_red[k] = make_float2(0.f, 0.f);
      }
      if (upper) {
        // thread t < kCell * NC adds column c, triangle 2p + l (t = (p NC + c) 2 + l)
        // of the cell over the 128 target threads in order
        __syncthreads();
        const int pc = threadIdx.x >> 1, l = threadIdx.x & 1;
        const int p = pc / NC, c = pc - p * NC;
        if (threadIdx.x < kCell * NC && 2 * p + l < ns) {
          const float* rf = reinterpret_cast<const float*>(s_red) + 2 * pc + l;
          float v0 = 0.f, v1 = 0.f, v2 = 0.f, v3 = 0.f;
#pragma unroll 8
          for (int t = 0; t < kTT; t += 4) {
            v0 += rf[(t + 0) * kRow * 2];
            v1 += rf[(t + 1) * kRow * 2];
            v2 += rf[(t + 2) * kRow * 2];
            v3 += rf[(t + 3) * kRow * 2];
          }
          md.partial[c * stride + (size_t)tslot * md.nitems + t0 + 2 * p + l] = (double)((v0 + v1) + (v2 + v3));
        }
      }
      __syncthreads();
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < NC; ++c)
        md.partial[c * stride + (size_t)w.split * md.nitems + ti] = (double)acc_hi[c] + (double)acc_lo[c];
    }
  }
}

// FP64 single-layer-only symmetric far field (NC right-hand sides): the
// batched solver's FP64 residual applies. The FP32 form's arithmetic in FP64,
// one source triangle at a time; staged and reduced per half cell (16
// triangles: the transposed buffer holds a double per column and triangle).
constexpr int kSl64Tris = kCell / 2;
template <int NC>
__host__ __device__ constexpr int sl64_red_stride() { return kSl64Tris * NC + 1; }  // doubles per thread row
template <int NC>
__host__ __device__ constexpr size_t sl64_smem_bytes()
{
  return (size_t)kSl64Tris * kQ * kNrec * 32 + (size_t)kTT * sl64_red_stride<NC>() * 8;
}

template <int NC, bool FAR>
__device__ __forceinline__ void eval_cell_sym64_sl(const dq* __restrict__ srec, const int4* __restrict__ svid, int s0,
                                                   int s1, int4 tv, const double (&x)[kQ], const double (&y)[kQ],
                                                   const double (&z)[kQ], const double (&q2)[kQ],
                                                   const double (&cw)[NC][kQ], const double (&om)[kQ],
                                                   const double (&wq)[kQ], double (&slw)[NC],
                                                   double* __restrict__ red)
{
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    if constexpr (!FAR) {
      if (shares_vertex(tv, svid[s])) {
#pragma unroll
        for (int c = 0; c < NC; ++c) red[(s - s0) * NC + c] = 0.0;
        continue;
      }
    }
    const dq* r = srec + (size_t)s * kQ * kNrec;
    double R[kQ];
#pragma unroll
    for (int a = 0; a < kQ; ++a) R[a] = 0.0;
#pragma unroll(kUnrollB64)
    for (int b = 0; b < kQ; ++b) {
      const dq p0 = r[b * kNrec];
#pragma unroll
      for (int a = 0; a < kQ; ++a) {
        double r2;
        if constexpr (FAR) {
          r2 = x[a] * p0.x + (y[a] * p0.y + (z[a] * p0.z + (q2[a] + p0.w)));
        } else {
          const double dx = x[a] + 0.5 * p0.x, dy = y[a] + 0.5 * p0.y, dz = z[a] + 0.5 * p0.z;
          r2 = dx * dx + dy * dy + dz * dz;
        }
        R[a] += om[b] * rsq_f64(r2);
      }
    }
    double U = 0.0;
#pragma unroll
    for (int a = 0; a < kQ; ++a) U += wq[a] * R[a];
    const dq p1 = r[1];  // first-point charges
#pragma unroll
    for (int c = 0; c < NC; ++c) {
      slw[c] += comp(p1, c) * U;
      double S = 0.0;
#pragma unroll
      for (int a = 0; a < kQ; ++a) S += cw[c][a] * R[a];
      red[(s - s0) * NC + c] = S;
    }
  }
}

template <int NC>
__global__ void __launch_bounds__(kTT, 2)
    far_sym64_sl_kernel(const FarMeshDesc* __restrict__ meshes, const WorkItem* __restrict__ items, int nitems,
                        int* __restrict__ counter)
{
  constexpr int kRow = sl64_red_stride<NC>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_item;
  __shared__ int4 s_vid[kSl64Tris];
  dq* s_rec = reinterpret_cast<dq*>(smem_raw);
  double* s_red = reinterpret_cast<double*>(smem_raw + (size_t)kSl64Tris * kQ * kNrec * 32);
  double* my_red = s_red + threadIdx.x * kRow;

  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) break;
    const WorkItem w = items[it];
    const FarMeshDesc md = meshes[w.mesh];
    if (md.active && *md.active == 0) continue;  // uniform across the CTA
    const bool upper = w.cell0 * kCell >= w.tgt0 + kTT;
    const int tslot = w.tgt0 / kTT;
    const int ti = w.tgt0 + threadIdx.x;
    const bool active = ti < md.nitems;
    const int tsel = active ? ti : w.tgt0;
    const dq tile = md.twarp[tsel / kWarpItems];
    double cen[3];
    {
      const dq c = md.tcent[tsel];
      cen[0] = c.x; cen[1] = c.y; cen[2] = c.z;
    }
    const int4 tv = active ? md.tvid[tsel] : make_int4(-1, -1, -1, 0);
    const dq* grec = reinterpret_cast<const dq*>(md.rec);
    double acc[NC];
#pragma unroll
    for (int c = 0; c < NC; ++c) acc[c] = 0.0;
    const size_t stride = (size_t)md.nsplit * md.nitems;

    for (int half = 2 * w.cell0; half < 2 * w.cell1; ++half) {
      const int cell = half >> 1;
      const int t0 = half * kSl64Tris;
      const int ns = min(kSl64Tris, md.ne - t0);
      if (ns <= 0) break;  // uniform: the mesh's last cell has no second half
      {
        const dq* g = grec + (size_t)t0 * kQ * kNrec;
        const int nstage = ns * kQ * kNrec;
        for (int k = threadIdx.x; k < nstage; k += kTT) s_rec[k] = g[k];
        for (int k = threadIdx.x; k < ns; k += kTT) s_vid[k] = md.svid[t0 + k];
      }
      __syncthreads();
      if (active) {
        const dq ccd = md.ccent[cell];
        const double ddx = ccd.x - tile.x, ddy = ccd.y - tile.y, ddz = ccd.z - tile.z;
        const double rr = kFarRatio * (ccd.w + tile.w);
        const bool far = ddx * ddx + ddy * ddy + ddz * ddz > rr * rr;
        const double o[3] = {ccd.x - cen[0], ccd.y - cen[1], ccd.z - cen[2]};
        double xs[kQ], ys[kQ], zs[kQ], q2[kQ], wq[kQ];
#pragma unroll
        for (int a = 0; a < kQ; ++a) {
          const dq p = md.tgt64[(size_t)tsel * kQ + a];
          xs[a] = p.x - o[0]; ys[a] = p.y - o[1]; zs[a] = p.z - o[2];
          q2[a] = xs[a] * xs[a] + ys[a] * ys[a] + zs[a] * zs[a];
          wq[a] = p.w;
        }
        double part[NC];
        if (upper) {
          double cw[NC][kQ], om[kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
            om[a] = wq[a] / wq[0];
            const dq st = grec[((size_t)tsel * kQ + a) * kNrec + 1];  // the target's charges c_a
#pragma unroll
            for (int c = 0; c < NC; ++c) cw[c][a] = wq[0] * comp(st, c);
          }
#pragma unroll
          for (int c = 0; c < NC; ++c) part[c] = 0.0;
          if (far)
            eval_cell_sym64_sl<NC, true>(s_rec, s_vid, 0, ns, tv, xs, ys, zs, q2, cw, om, wq, part, my_red);
          else
            eval_cell_sym64_sl<NC, false>(s_rec, s_vid, 0, ns, tv, xs, ys, zs, q2, cw, om, wq, part, my_red);
        } else {
          const double zero3[3] = {0.0, 0.0, 0.0};
          double slc[NC][kQ], dlc[1][kQ];
#pragma unroll
          for (int a = 0; a < kQ; ++a) {
#pragma unroll
            for (int c = 0; c < NC; ++c) slc[c][a] = 0.0;
            dlc[0][a] = 0.0;
          }
          if (far)
            eval_cell<double, kQ, kQ, NC, 0, true>(s_rec, s_vid, nullptr, nullptr, 0, ns, kQ, tv, xs, ys, zs, q2, o,
                                                   cen, zero3, slc, dlc);
          else
            eval_cell<double, kQ, kQ, NC, 0, false>(s_rec, s_vid, nullptr, nullptr, 0, ns, kQ, tv, xs, ys, zs, q2, o,
                                                    cen, zero3, slc, dlc);
#pragma unroll
          for (int c = 0; c < NC; ++c) {
            part[c] = 0.0;
#pragma unroll
            for (int a = 0; a < kQ; ++a) part[c] += wq[a] * slc[c][a];
          }
        }
#pragma unroll
        for (int c = 0; c < NC; ++c) acc[c] += part[c];
      } else if (upper) {
        for (int k = 0; k < kSl64Tris * NC; ++k) my_red[k] = 0.0;
      }
      if (upper) {
        // thread t < kSl64Tris * NC adds column t % NC of triangle t / NC over
        // the 128 target threads in order
        __syncthreads();
        const int k = threadIdx.x / NC, c = threadIdx.x - k * NC;
        if (threadIdx.x < kSl64Tris * NC && k < ns) {
          const double* rf = s_red + threadIdx.x;
          double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
#pragma unroll 8
          for (int t = 0; t < kTT; t += 4) {
            v0 += rf[(t + 0) * kRow];
            v1 += rf[(t + 1) * kRow];
            v2 += rf[(t + 2) * kRow];
            v3 += rf[(t + 3) * kRow];
          }
          md.partial[c * stride + (size_t)tslot * md.nitems + t0 + k] = (v0 + v1) + (v2 + v3);
        }
      }
      __syncthreads();
    }
    if (active) {
#pragma unroll
      for (int c = 0; c < NC; ++c) md.partial[c * stride + (size_t)w.split * md.nitems + ti] = acc[c];
    }
  }
}

}  // namespace

size_t far_sym_smem_bytes(bool fp32, int nsl, int nd)
{
  if (nd == 0 && fp32) return nsl == 1 ? sl_smem_bytes<1>() : nsl == 3 ? sl_smem_bytes<3>() : sl_smem_bytes<4>();
  if (nd == 0) return nsl == 1 ? sl64_smem_bytes<1>() : nsl == 3 ? sl64_smem_bytes<3>() : sl64_smem_bytes<4>();
  return fp32 ? kRecBytes + kRedBytes : kRec64Bytes + kRed64Bytes;
}

static const void* sym_kernel_fn(bool fp32, int nsl, int nd)
{
  if (nd == 1 && nsl == 1) return fp32 ? (const void*)far_sym_kernel : (const void*)far_sym64_kernel;
  if (nd == 0 && fp32) {
    if (nsl == 1) return (const void*)far_sym_sl_kernel<1>;
    if (nsl == 3) return (const void*)far_sym_sl_kernel<3>;
    if (nsl == 4) return (const void*)far_sym_sl_kernel<4>;
  }
  if (nd == 0 && !fp32) {
    if (nsl == 1) return (const void*)far_sym64_sl_kernel<1>;
    if (nsl == 3) return (const void*)far_sym64_sl_kernel<3>;
    if (nsl == 4) return (const void*)far_sym64_sl_kernel<4>;
  }
  return nullptr;
}

bool far_sym_variant(bool fp32, int nsl, int nd) { return sym_kernel_fn(fp32, nsl, nd) != nullptr; }

cudaError_t far_sym_launch(bool fp32, int nsl, int nd, const FarMeshDesc* dm, const WorkItem* di, int n, int* dc,
                           int grid, cudaStream_t st)
{
  const void* fn = sym_kernel_fn(fp32, nsl, nd);
  if (!fn) return cudaErrorInvalidValue;
  // the attribute is per device: set it on every launch (a host-side call)
  const size_t smem = far_sym_smem_bytes(fp32, nsl, nd);
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  void* args[] = {(void*)&dm, (void*)&di, (void*)&n, (void*)&dc};
  return cudaLaunchKernel(fn, dim3(grid), dim3(kTT), args, smem, st);
}

int far_sym_occupancy(bool fp32, int nsl, int nd)
{
  int occ = 0;
  const void* fn = sym_kernel_fn(fp32, nsl, nd);
  if (!fn) return 0;
  const size_t smem = far_sym_smem_bytes(fp32, nsl, nd);
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, kTT, smem) != cudaSuccess) return 0;
  return occ;
}

int far_sym_cells_per_item(int cells_per_item) { return std::max(2, (cells_per_item > 0 ? cells_per_item : EB_SYM_CELLS) & ~1); }

int far_sym_items(int nitems, int ncells, int cells_per_item, std::vector<WorkItem>& items)
{
  const int ntt = (nitems + kTT - 1) / kTT;
  const int r = far_sym_cells_per_item(cells_per_item);
  items.clear();
  int nsplit = 0;
  std::vector<WorkItem> diag;
  for (int t = 0; t < ntt; t++) {
    const int c0 = t * (kTT / kCell);
    diag.push_back(WorkItem{0, t * kTT, c0, std::min(ncells, c0 + kTT / kCell), t});
    int slot = t + 1;
    for (int c = c0 + kTT / kCell; c < ncells; c += r)
      items.push_back(WorkItem{0, t * kTT, c, std::min(ncells, c + r), slot++});
    nsplit = std::max(nsplit, slot);
  }
  // the larger upper items first, the diagonal ones fill the tail
  std::stable_sort(items.begin(), items.end(), [](const WorkItem& a, const WorkItem& b) {
    return (a.cell1 - a.cell0) > (b.cell1 - b.cell0);
  });
  items.insert(items.end(), diag.begin(), diag.end());
  return nsplit;
}

}  // namespace eb

// ---------------------------------------------------------------------------
// C ABI: the symmetric plan's work list and slot counts (host only).

extern "C" int eb_sym_plan(int nelems, int cells_per_item, int* nitems, int* nslots_max, int* items, int* row_slots)
{
  using namespace eb;
  if (nelems < 1 || cells_per_item < 0) return set_error(EB_ERR_INVALID, "need nelems >= 1 and cells_per_item >= 0");
  const int ncells = (nelems + kCell - 1) / kCell;
  std::vector<WorkItem> list;
  const int nsplit = far_sym_items(nelems, ncells, cells_per_item, list);
  if (nitems) *nitems = (int)list.size();
  if (nslots_max) *nslots_max = nsplit;
  if (items)
    for (size_t k = 0; k < list.size(); k++) {
      items[4 * k] = list[k].tgt0;
      items[4 * k + 1] = list[k].cell0;
      items[4 * k + 2] = list[k].cell1;
      items[4 * k + 3] = list[k].split;
    }
  if (row_slots) {
    const int r = far_sym_cells_per_item(cells_per_item);
    for (int s = 0; s < nelems; s++) row_slots[s] = sym_row_slots(s, nelems, r);
  }
  return EB_OK;
}
