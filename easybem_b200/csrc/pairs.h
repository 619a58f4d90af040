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

// ---- P1 x P1 single layer: the reference GPU kernels' Sauter-Schwab forms
// (src/BEM3dLaplaceGPU.cu:82-154, 211-320, 371-442, 491-557) in FP64.
// I[3k+l] couples test basis k and trial basis l in the case's local vertex
// order (p1_local_orders).

__device__ inline void ss_p1_self(const Quadrature& q, d3 u, d3 v, double* I)
{
  double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const d3 uv = u + v;
  for (int i = 0; i < q.nl; i++) {
    const double e = q.lx[i], w = q.lw[i], e2 = e * e;
    double f = w * rnorm(e * u + v);  // D1
    S[0] += f / 30; S[1] += f / 60; S[2] += f / 30; S[3] += f / 60; S[4] += f / 30;
    S[5] += f / 30; S[6] += f / 30; S[7] += f / 30; S[8] += f / 10;
    f = w * rnorm(e * v + u);  // D2
    S[0] += f / 30; S[1] += (2 - e) / 60 * f; S[2] += (1 + e) / 60 * f; S[3] += (2 - e) / 60 * f;
    S[4] += (3 - 3 * e + e2) / 30 * f; S[5] += (1 + e - e2) / 30 * f; S[6] += (1 + e) / 60 * f;
    S[7] += (1 + e - e2) / 30 * f; S[8] += (1 + e + e2) / 30 * f;
    f = w * rnorm(e * uv - v);  // D3
    S[0] += (1 + e + e2) / 30 * f; S[1] += (1 + e) / 60 * f; S[2] += (1 + e - e2) / 30 * f;
    S[3] += (1 + e) / 60 * f; S[4] += f / 30; S[5] += (2 - e) / 60 * f;
    S[6] += (1 + e - e2) / 30 * f; S[7] += (2 - e) / 60 * f; S[8] += (3 - 3 * e + e2) / 30 * f;
  }
  const d3 c = cross3(u, v);
  const double sc = dot3(c, c) / (4.0 * M_PI);
  for (int k = 0; k < 9; k++) I[k] = sc * S[k];
}

__device__ inline void ss_p1_edge(const Quadrature& q, d3 u, d3 v, d3 w, double* I)
{
  double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const d3 uw = u + w, uv = u + v;
  for (int i = 0; i < q.nl; i++)
    for (int j = 0; j < q.nl; j++) {
      const double a = q.lx[i], b = q.lx[j], ww = q.lw[i] * q.lw[j], ab = a * b;
      double f = ww * a * rnorm(a * (b * uw - w) + v);  // D2
      S[0] += (1 + ab) / 60 * f; S[1] += (3 - 2 * a) / 120 * f; S[2] += -a * (b - 1) / 60 * f;
      S[3] += (1 + 2 * ab) / 120 * f; S[4] += (2 - a) / 60 * f; S[5] += -a * (b - 1) / 60 * f;
      S[6] += (1 + 3 * ab) / 60 * f; S[7] += (4 - 3 * a) / 60 * f; S[8] += -a * (b - 1) / 20 * f;
      f = ww * a * rnorm(v - a * (uv + b * w));  // D3
      S[0] += (1 + a) / 60 * f; S[1] += (1.0 / 40 + (4 * a - ab - 3 * a * ab) / 60) * f;
      S[2] += ab * (3 * a + 1) / 60 * f; S[3] += f / 120; S[4] += (2 - ab) / 60 * f; S[5] += ab / 60 * f;
      S[6] += (1 - a) / 60 * f; S[7] += (3 * ab - 4) * (a - 1) / 60 * f; S[8] += -ab * (a - 1) / 20 * f;
      f = ww * a * rnorm(a * (v - b * uv) - w);  // D4
      S[0] += (1 + ab) / 60 * f; S[1] += (1 + 2 * ab) / 120 * f; S[2] += (1 + 3 * ab) / 60 * f;
      S[3] += (3 - 2 * a) / 120 * f; S[4] += (2 - a) / 60 * f; S[5] += (4 - 3 * a) / 60 * f;
      S[6] += -a * (b - 1) / 60 * f; S[7] += -a * (b - 1) / 60 * f; S[8] += -a * (b - 1) / 20 * f;
      f = ww * a * rnorm(v - a * (w + b * uv));  // D5
      S[0] += (1 + ab) / 60 * f; S[1] += (1.0 / 40 + (4 * ab - a - 3 * a * ab) / 60) * f;
      S[2] += a * (1 + 3 * ab) / 60 * f; S[3] += f / 120; S[4] += (2 - a) / 60 * f; S[5] += a / 60 * f;
      S[6] += (1 - ab) / 60 * f; S[7] += (3 * a - 4) * (ab - 1) / 60 * f; S[8] += -a * (ab - 1) / 20 * f;
      f = ww * rnorm(a * uw + b * v - w);  // D1
      S[0] += (1 + a) / 60 * f; S[1] += f / 120; S[2] += (1 - a) / 60 * f;
      S[3] += (1.0 / 40 + (4 * a - 3 * ab - b) / 60) * f; S[4] += (2 - b) / 60 * f;
      S[5] += (3 * b - 4) * (a - 1) / 60 * f; S[6] += b * (3 * a + 1) / 60 * f; S[7] += b / 60 * f;
      S[8] += -b * (a - 1) / 20 * f;
    }
  const double sc = sqrt(dot3(cross3(u, v), cross3(u, v))) * sqrt(dot3(cross3(u, w), cross3(u, w))) / (4.0 * M_PI);
  for (int k = 0; k < 9; k++) I[k] = sc * S[k];
}

__device__ inline void ss_p1_vertex(const Quadrature& q, d3 u, d3 v, d3 w, d3 z, double* I)
{
  double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = 0; i < q.nl; i++)
    for (int j = 0; j < q.nl; j++)
      for (int k = 0; k < q.nl; k++) {
        const double e1 = q.lx[i], e2 = q.lx[j], e3 = q.lx[k];
        const double ww = q.lw[i] * q.lw[j] * q.lw[k] * e2;
        const double a[9] = {1.0 / 12 - e2 / 20,          e2 * e3 / 20,           -e2 * (e3 - 1) / 20,
                             -e1 * (4 * e2 - 5) / 20,     e1 * e2 * e3 / 5,       -e1 * e2 * (e3 - 1) / 5,
                             (4 * e2 - 5) * (e1 - 1) / 20, -e2 * e3 * (e1 - 1) / 5, e2 * (e1 - 1) * (e3 - 1) / 5};
        const double f1 = ww * rnorm(u + e1 * v - e2 * (w + e3 * z));
        const double f2 = ww * rnorm(w + e1 * z - e2 * (u + e3 * v));
        for (int r = 0; r < 3; r++)
          for (int c = 0; c < 3; c++) S[3 * r + c] += a[3 * r + c] * f1 + a[3 * c + r] * f2;
      }
  const double sc = sqrt(dot3(cross3(u, v), cross3(u, v))) * sqrt(dot3(cross3(w, z), cross3(w, z))) / (4.0 * M_PI);
  for (int k = 0; k < 9; k++) I[k] = sc * S[k];
}

// P1 entries of a near pair; oi/oj: local vertex orders (p1_local_orders).
__device__ inline void near_pair_values_p1(const Quadrature& q, const PairGeom& g, const d3* Pi, const d3* Pj,
                                           const int* oi, const int* oj, double* I)
{
  if (g.kind == kPairSelf) {
    ss_p1_self(q, Pi[1] - Pi[0], Pi[2] - Pi[1], I);
  } else if (g.kind == kPairVertex) {
    ss_p1_vertex(q, Pi[oi[1]] - Pi[oi[0]], Pi[oi[2]] - Pi[oi[1]], Pj[oj[1]] - Pj[oj[0]], Pj[oj[2]] - Pj[oj[1]], I);
  } else if (g.kind == kPairEdge) {
    ss_p1_edge(q, Pj[g.cj[1]] - Pj[g.cj[0]], Pi[g.ri] - Pj[g.cj[1]], Pj[g.rj] - Pj[g.cj[1]], I);
  } else {
    for (int k = 0; k < 9; k++) I[k] = 0.0;
  }
}

#endif  // __CUDACC__

// Local vertex orders of the test (oi) and trial (oj) basis functions of the
// P1 near-pair formulas: coincident (0,1,2); vertex-adjacent rotations starting
// at the shared vertex; edge-adjacent (shared c0, shared c1, opposite) in both
// triangles (the reference GPU host code's P1..P3 / Q1..Q3, :1067-1083).
__host__ __device__ inline void p1_local_orders(const PairGeom& g, int* oi, int* oj)
{
  for (int k = 0; k < 3; k++) oi[k] = oj[k] = k;
  if (g.kind == kPairVertex) {
    for (int k = 0; k < 3; k++) {
      oi[k] = (g.ci[0] + k) % 3;
      oj[k] = (g.cj[0] + k) % 3;
    }
  } else if (g.kind == kPairEdge) {
    oi[0] = g.ci[0]; oi[1] = g.ci[1]; oi[2] = g.ri;
    oj[0] = g.cj[0]; oj[1] = g.cj[1]; oj[2] = g.rj;
  }
}

}  // namespace eb
