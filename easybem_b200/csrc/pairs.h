// Near-field pair classification and the FP64 Sauter-Schwab integrals.
//
// A pair (test i, trial j) is classified by counting shared vertex ids, with
// the local rotations of getLaplace3d (src/BEM3dLaplace.cpp:692-764):
//   coincident (i == j): u = P1-P0, v = P2-P1 of triangle i;
//   vertex-adjacent: with c the shared local index in i and d in j,
//     u = Pi[c+1]-Pi[c], v = Pi[c+2]-Pi[c+1], w = Pj[d+1]-Pj[d], z = Pj[d+2]-Pj[d+1],
//     DL weights belong to trial vertices (d, d+1, d+2);
//   edge-adjacent: shared local indices (c0,c1) in j ordered so c1 = c0+1 mod 3,
//     u = Pj[c1]-Pj[c0], v = Pi[ri]-Pj[c1], w = Pj[rj]-Pj[c1] (ri, rj the
//     remaining indices), DL weights belong to trial vertices (c0, c1, rj).
// The integrands are the reduced Sauter-Schwab forms of
// src/BEM3dLaplace.cpp:22-148 (single layer) and :195-383 (double layer),
// which the reference GPU kernels repeat in FP32 (src/BEM3dLaplaceGPU.cu:
// 47-79, 157-208, 323-368, 560-772). Here they run in FP64, once per mesh.
#pragma once

#include "common.h"
#include "quadrature.h"

namespace eb {

enum PairKind { kPairNone = -1, kPairSelf = 0, kPairVertex = 1, kPairEdge = 2, kPairRepeat = 3 };

struct PairGeom {
  int kind;
  int ci[2], cj[2];  // shared local indices in i and j (ci[0], cj[0] for the vertex case)
  int ri, rj;        // remaining local index (edge case)
};

// fi, fj: vertex ids of triangles i and j (any consistent base).
__host__ __device__ inline PairGeom classify_pair(const int* fi, const int* fj, bool same)
{
  PairGeom g;
  g.ri = g.rj = 0;
  g.ci[0] = g.ci[1] = g.cj[0] = g.cj[1] = 0;
  if (same) { g.kind = kPairSelf; return g; }
  int nc = 0;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++)
      if (fj[k] == fi[l]) {
        if (nc < 2) { g.ci[nc] = l; g.cj[nc] = k; }
        nc++;
        break;
      }
  if (nc == 2 && g.cj[1] != (g.cj[0] + 1) % 3) {
    int t = g.cj[0]; g.cj[0] = g.cj[1]; g.cj[1] = t;
    t = g.ci[0]; g.ci[0] = g.ci[1]; g.ci[1] = t;
  }
  if (nc == 2) {
    g.ri = 3 - g.ci[0] - g.ci[1];
    g.rj = 3 - g.cj[0] - g.cj[1];
  }
  g.kind = nc == 0 ? kPairNone : (nc == 1 ? kPairVertex : (nc == 2 ? kPairEdge : kPairRepeat));
  return g;
}

// Trial-vertex local indices that receive the three DL weights of a pair.
__host__ __device__ inline void dl_trial_slots(const PairGeom& g, int* s)
{
  if (g.kind == kPairVertex) {
    for (int k = 0; k < 3; k++) s[k] = (g.cj[0] + k) % 3;
  } else if (g.kind == kPairEdge) {
    s[0] = g.cj[0]; s[1] = g.cj[1]; s[2] = g.rj;
  } else {
    s[0] = 0; s[1] = 1; s[2] = 2;
  }
}

#ifdef __CUDACC__
__device__ inline double rnorm(d3 a) { return rsqrt(dot3(a, a)); }
__device__ inline double dlh(d3 a, d3 n)
{
  const double ir = rsqrt(dot3(a, a));
  return dot3(a, n) * ir * ir * ir;
}

// Coincident panels, P0 SL (src/BEM3dLaplace.cpp:22-52).
__device__ inline double ss_sl_self(const Quadrature& q, d3 u, d3 v)
{
  const d3 c = cross3(u, v);
  const d3 uv = u + v;
  double s = 0.0;
  for (int i = 0; i < q.nl; i++) {
    const double e = q.lx[i];
    s += q.lw[i] * (rnorm(e * u + v) + rnorm(e * v + u) + rnorm(e * uv - v));
  }
  return dot3(c, c) * s / (12.0 * M_PI);
}

// Edge-adjacent panels, P0 SL (src/BEM3dLaplace.cpp:55-102).
__device__ inline double ss_sl_edge(const Quadrature& q, d3 u, d3 v, d3 w)
{
  const double jac = sqrt(dot3(cross3(u, v), cross3(u, v))) * sqrt(dot3(cross3(u, w), cross3(u, w)));
  const d3 uw = u + w, uv = u + v;
  double s = 0.0;
  for (int i = 0; i < q.nl; i++) {
    const double e2 = q.lx[i];
    double si = 0.0;
    for (int j = 0; j < q.nl; j++) {
      const double e3 = q.lx[j];
      double f = rnorm(e2 * (e3 * uw - w) + v) + rnorm(v - e2 * (uv + e3 * w)) +
                 rnorm(e2 * (v - e3 * uv) - w) + rnorm(v - e2 * (w + e3 * uv));
      f = e2 * f + rnorm(e2 * uw + e3 * v - w);
      si += q.lw[j] * f;
    }
    s += q.lw[i] * si;
  }
  return jac * s / (24.0 * M_PI);
}

// Vertex-adjacent panels, P0 SL (src/BEM3dLaplace.cpp:105-148).
__device__ inline double ss_sl_vertex(const Quadrature& q, d3 u, d3 v, d3 w, d3 z)
{
  const double jac = sqrt(dot3(cross3(u, v), cross3(u, v))) * sqrt(dot3(cross3(w, z), cross3(w, z)));
  double s = 0.0;
  for (int i = 0; i < q.nl; i++) {
    const double e1 = q.lx[i];
    const d3 a1 = u + e1 * v, b1 = w + e1 * z;
    for (int j = 0; j < q.nl; j++) {
      const double e2 = q.lx[j];
      double sk = 0.0;
      for (int k = 0; k < q.nl; k++) {
        const double e3 = q.lx[k];
        sk += q.lw[k] * (rnorm(a1 - e2 * (w + e3 * z)) + rnorm(b1 - e2 * (u + e3 * v)));
      }
      s += q.lw[i] * q.lw[j] * e2 * sk;
    }
  }
  return jac * s / (12.0 * M_PI);
}

// Moments of the fixed two-point inner rule of the DL integrals:
// a(s) = sum_k w_k p_k (1 - p_k s), b = sum_k w_k p_k^2.
__device__ inline double inner_a(const Quadrature& q, double s)
{
  return q.l2w[0] * q.l2x[0] * (1.0 - q.l2x[0] * s) + q.l2w[1] * q.l2x[1] * (1.0 - q.l2x[1] * s);
}
__device__ inline double inner_b(const Quadrature& q)
{
  return q.l2w[0] * q.l2x[0] * q.l2x[0] + q.l2w[1] * q.l2x[1] * q.l2x[1];
}

// Edge-adjacent panels, DL P0 x P1 (src/BEM3dLaplace.cpp:195-309); n is the
// unit normal of u x w (the trial triangle).
__device__ inline void ss_dl_edge(const Quadrature& q, d3 u, d3 v, d3 w, double* K)
{
  const d3 nt = cross3(u, w);
  const double jt = sqrt(dot3(nt, nt));
  const d3 n = (1.0 / jt) * nt;
  const double jac = sqrt(dot3(cross3(u, v), cross3(u, v))) * jt;
  const double e1 = 0.5, b = inner_b(q), a1 = inner_a(q, 1.0);
  const d3 uw = u + w, uv = u + v;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = 0; i < q.nl; i++) {
    const double e2 = q.lx[i], e12 = e1 * e2;
    for (int j = 0; j < q.nl; j++) {
      const double e3 = q.lx[j], e123 = e12 * e3;
      double h = dlh(e2 * (e3 * uw - w) + v, n);
      double k1 = inner_a(q, 1.0 - e123) * h, k2 = b * (1.0 - e12) * h, k3 = b * e12 * (1.0 - e3) * h;
      h = dlh(v - e2 * (uv + e3 * w), n);
      k1 += a1 * h; k2 += b * (1.0 - e123) * h; k3 += b * e123 * h;
      h = dlh(e2 * (v - e3 * uv) - w, n);
      k1 += a1 * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * h;
      h = dlh(v - e2 * (w + e3 * uv), n);
      k1 += a1 * h; k2 += b * (1.0 - e12) * h; k3 += b * e12 * h;
      k1 *= e2; k2 *= e2; k3 *= e2;
      h = dlh(e2 * uw + e3 * v - w, n);
      k1 += inner_a(q, 1.0 - e12) * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * (1.0 - e2) * h;
      const double ww = q.lw[i] * q.lw[j];
      s1 += ww * k1; s2 += ww * k2; s3 += ww * k3;
    }
  }
  const double f = jac / (4.0 * M_PI);
  K[0] = f * s1; K[1] = f * s2; K[2] = f * s3;
}

// Vertex-adjacent panels, DL P0 x P1 (src/BEM3dLaplace.cpp:312-383); n is
// the unit normal of w x z.
__device__ inline void ss_dl_vertex(const Quadrature& q, d3 u, d3 v, d3 w, d3 z, double* K)
{
  const d3 nt = cross3(w, z);
  const double jt = sqrt(dot3(nt, nt));
  const d3 n = (1.0 / jt) * nt;
  const double jac = sqrt(dot3(cross3(u, v), cross3(u, v))) * jt;
  const double b = inner_b(q), a1 = inner_a(q, 1.0);
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = 0; i < q.nl; i++) {
    const double e1 = q.lx[i];
    const d3 a = u + e1 * v, bb = w + e1 * z;
    for (int j = 0; j < q.nl; j++) {
      const double e2 = q.lx[j];
      for (int k = 0; k < q.nl; k++) {
        const double e3 = q.lx[k];
        double h = dlh(a - e2 * (w + e3 * z), n);
        double k1 = inner_a(q, e2) * h, k2 = b * e2 * (1.0 - e3) * h, k3 = b * e2 * e3 * h;
        h = dlh(e2 * (u + e3 * v) - bb, n);
        k1 += a1 * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * h;
        const double ww = q.lw[i] * q.lw[j] * q.lw[k] * e2;
        s1 += ww * k1; s2 += ww * k2; s3 += ww * k3;
      }
    }
  }
  const double f = jac / (4.0 * M_PI);
  K[0] = f * s1; K[1] = f * s2; K[2] = f * s3;
}

// Near-field entries of pair (i, j): SL value and the three DL weights in the
// order of dl_trial_slots(). P holds the three vertices of each triangle.
__device__ inline void near_pair_values(const Quadrature& q, const PairGeom& g, const d3* Pi,
                                        const d3* Pj, double* sl, double* K)
{
  K[0] = K[1] = K[2] = 0.0;
  *sl = 0.0;
  if (g.kind == kPairSelf) {
    *sl = ss_sl_self(q, Pi[1] - Pi[0], Pi[2] - Pi[1]);
  } else if (g.kind == kPairVertex) {
    const int c = g.ci[0], d = g.cj[0];
    const d3 u = Pi[(c + 1) % 3] - Pi[c], v = Pi[(c + 2) % 3] - Pi[(c + 1) % 3];
    const d3 w = Pj[(d + 1) % 3] - Pj[d], z = Pj[(d + 2) % 3] - Pj[(d + 1) % 3];
    *sl = ss_sl_vertex(q, u, v, w, z);
    ss_dl_vertex(q, u, v, w, z, K);
  } else if (g.kind == kPairEdge) {
    const d3 u = Pj[g.cj[1]] - Pj[g.cj[0]], v = Pi[g.ri] - Pj[g.cj[1]], w = Pj[g.rj] - Pj[g.cj[1]];
    *sl = ss_sl_edge(q, u, v, w);
    ss_dl_edge(q, u, v, w, K);
  }
}

#endif  // __CUDACC__

}  // namespace eb
