/*
 * ORACLE — test infrastructure only. A plain-C, FP64 restatement of the
 * reference's CPU Galerkin operators for the Laplace single layer (P0) and
 * double layer (P0 test x P1 trial), used by tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py to check the CUDA path. The product
 * never links or calls this file.
 *
 * Parity is pinned against the reference itself: oracle/_ref/libeasybem_ref.so
 * is compiled from the reference sources by oracle/Makefile, and the tests
 * compare every pair routine and the assembled operators of this port with it
 * (plus committed golden fixtures made from it, tests/golden/make_golden.py).
 *
 * Every function cites the reference routine it restates (paths relative to
 * the reference project root). Quadrature tables are supplied by the caller
 * through orc_set_rules(); the tests feed the reference's own tables.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXL 64
#define ORC_MAXT 79

static int g_nl, g_nt;
static double g_lx[ORC_MAXL], g_lw[ORC_MAXL];
static double g_tx[ORC_MAXT], g_ty[ORC_MAXT], g_tw[ORC_MAXT];
static double g_l2x[2], g_l2w[2];

typedef struct { double x, y, z; } v3;

static inline v3 mk(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 add(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl(double s, v3 a) { return mk(s * a.x, s * a.y, s * a.z); }
static inline double dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b)
{
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline double norm(v3 a) { return sqrt(dot(a, a)); }
static inline double inv_norm(v3 a) { return 1.0 / sqrt(dot(a, a)); }
/* (d . n) / |d|^3, the double-layer kernel numerator over the cube. */
static inline double dl_h(v3 d, v3 n)
{
  double r = norm(d);
  return dot(d, n) / (r * r * r);
}
static inline v3 load(const double *p) { return mk(p[0], p[1], p[2]); }

void orc_set_rules(int nl, const double *lx, const double *lw, int nt, const double *tx,
                   const double *ty, const double *tw, const double *l2x, const double *l2w)
{
  g_nl = nl;
  g_nt = nt;
  memcpy(g_lx, lx, sizeof(double) * nl);
  memcpy(g_lw, lw, sizeof(double) * nl);
  memcpy(g_tx, tx, sizeof(double) * nt);
  memcpy(g_ty, ty, sizeof(double) * nt);
  memcpy(g_tw, tw, sizeof(double) * nt);
  memcpy(g_l2x, l2x, sizeof(double) * 2);
  memcpy(g_l2w, l2w, sizeof(double) * 2);
}

/* Coincident panels, P0 single layer: src/BEM3dLaplace.cpp:22-52. The
 * Sauter-Schwab reduction leaves a 1-D integral of three inverse distances. */
double orc_sl_id(const double *pu, const double *pv)
{
  v3 u = load(pu), v = load(pv);
  v3 c = cross(u, v);
  double s = 0.0;
  for (int i = 0; i < g_nl; i++) {
    double e = g_lx[i];
    double f = inv_norm(add(scl(e, u), v)) + inv_norm(add(scl(e, v), u)) +
               inv_norm(sub(scl(e, add(u, v)), v));
    s += g_lw[i] * f;
  }
  return dot(c, c) * s / M_PI / 12.0;
}

/* Edge-adjacent panels, P0 single layer: src/BEM3dLaplace.cpp:55-102. */
double orc_sl_edge(const double *pu, const double *pv, const double *pw)
{
  v3 u = load(pu), v = load(pv), w = load(pw);
  double jac = norm(cross(u, v)) * norm(cross(u, w));
  v3 uw = add(u, w), uv = add(u, v);
  double s = 0.0;
  for (int i = 0; i < g_nl; i++) {
    double e2 = g_lx[i];
    for (int j = 0; j < g_nl; j++) {
      double e3 = g_lx[j];
      double f = inv_norm(add(scl(e2, sub(scl(e3, uw), w)), v));
      f += inv_norm(add(scl(-e2, add(uv, scl(e3, w))), v));
      f += inv_norm(sub(scl(e2, sub(v, scl(e3, uv))), w));
      f += inv_norm(add(scl(-e2, add(w, scl(e3, uv))), v));
      f *= e2;
      f += inv_norm(sub(add(scl(e2, uw), scl(e3, v)), w));
      s += g_lw[i] * g_lw[j] * f;
    }
  }
  return jac * s / M_PI / 24.0;
}

/* Vertex-adjacent panels, P0 single layer: src/BEM3dLaplace.cpp:105-148. */
double orc_sl_vertex(const double *pu, const double *pv, const double *pw, const double *pz)
{
  v3 u = load(pu), v = load(pv), w = load(pw), z = load(pz);
  double jac = norm(cross(u, v)) * norm(cross(w, z));
  double s = 0.0;
  for (int i = 0; i < g_nl; i++)
    for (int j = 0; j < g_nl; j++)
      for (int k = 0; k < g_nl; k++) {
        double e1 = g_lx[i], e2 = g_lx[j], e3 = g_lx[k];
        double f = inv_norm(sub(add(u, scl(e1, v)), scl(e2, add(w, scl(e3, z)))));
        f += inv_norm(sub(add(w, scl(e1, z)), scl(e2, add(u, scl(e3, v)))));
        s += g_lw[i] * g_lw[j] * g_lw[k] * e2 * f;
      }
  return jac * s / M_PI / 12.0;
}

/* Regular (disjoint) panels, P0 single layer: src/BEM3dLaplace.cpp:151-192. */
double orc_sl_disjoint(const double *pA, const double *pu, const double *pv, const double *pB,
                       const double *pw, const double *pz)
{
  v3 A = load(pA), u = load(pu), v = load(pv), B = load(pB), w = load(pw), z = load(pz);
  double jac = norm(cross(u, v)) * norm(cross(w, z));
  double s = 0.0;
  for (int i = 0; i < g_nt; i++) {
    v3 x = add(A, add(scl(g_tx[i], u), scl(g_ty[i], v)));
    for (int j = 0; j < g_nt; j++) {
      v3 d = sub(sub(sub(x, B), scl(g_tx[j], w)), scl(g_ty[j], z));
      s += g_tw[i] * g_tw[j] * inv_norm(d);
    }
  }
  return jac * s / M_PI / 4.0;
}

/* The two-point inner rule of the double-layer integrals contributes the
 * moments S1 = sum w p and S2 = sum w p^2 (src/BEM3dLaplace.cpp:230-298 write
 * them out term by term). a(s) = sum w p (1 - p s), b = sum w p^2. */
static inline double inner_a(double s)
{
  return g_l2w[0] * g_l2x[0] * (1.0 - g_l2x[0] * s) + g_l2w[1] * g_l2x[1] * (1.0 - g_l2x[1] * s);
}
static inline double inner_b(void)
{
  return g_l2w[0] * g_l2x[0] * g_l2x[0] + g_l2w[1] * g_l2x[1] * g_l2x[1];
}

/* Edge-adjacent panels, double layer (P0 x P1): src/BEM3dLaplace.cpp:195-309.
 * K[0..2] are the weights of the trial-triangle vertices in the order the
 * caller set up (shared c0, shared c1, opposite). */
void orc_dl_edge(const double *pu, const double *pv, const double *pw, double *K)
{
  v3 u = load(pu), v = load(pv), w = load(pw);
  v3 nt = cross(u, w);
  double jt = norm(nt);
  v3 n = scl(1.0 / jt, nt);
  double jac = norm(cross(u, v)) * jt;
  const double e1 = 0.5;
  const double b = inner_b();
  const double a1 = inner_a(1.0); /* sum w p (1 - p) */
  v3 uw = add(u, w), uv = add(u, v);
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = 0; i < g_nl; i++) {
    double e2 = g_lx[i], e12 = e1 * e2;
    for (int j = 0; j < g_nl; j++) {
      double e3 = g_lx[j], e123 = e12 * e3;
      double h = dl_h(add(scl(e2, sub(scl(e3, uw), w)), v), n);
      double k1 = inner_a(1.0 - e123) * h, k2 = b * (1.0 - e12) * h, k3 = b * e12 * (1.0 - e3) * h;
      h = dl_h(add(scl(-e2, add(uv, scl(e3, w))), v), n);
      k1 += a1 * h; k2 += b * (1.0 - e123) * h; k3 += b * e123 * h;
      h = dl_h(sub(scl(e2, sub(v, scl(e3, uv))), w), n);
      k1 += a1 * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * h;
      h = dl_h(add(scl(-e2, add(w, scl(e3, uv))), v), n);
      k1 += a1 * h; k2 += b * (1.0 - e12) * h; k3 += b * e12 * h;
      k1 *= e2; k2 *= e2; k3 *= e2;
      h = dl_h(sub(add(scl(e2, uw), scl(e3, v)), w), n);
      k1 += inner_a(1.0 - e12) * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * (1.0 - e2) * h;
      double ww = g_lw[i] * g_lw[j];
      s1 += ww * k1; s2 += ww * k2; s3 += ww * k3;
    }
  }
  K[0] = jac * s1 / 4.0 / M_PI;
  K[1] = jac * s2 / 4.0 / M_PI;
  K[2] = jac * s3 / 4.0 / M_PI;
}

/* Vertex-adjacent panels, double layer: src/BEM3dLaplace.cpp:312-383. */
void orc_dl_vertex(const double *pu, const double *pv, const double *pw, const double *pz, double *K)
{
  v3 u = load(pu), v = load(pv), w = load(pw), z = load(pz);
  v3 nt = cross(w, z);
  double jt = norm(nt);
  v3 n = scl(1.0 / jt, nt);
  double jac = norm(cross(u, v)) * jt;
  const double b = inner_b();
  const double a1 = inner_a(1.0);
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = 0; i < g_nl; i++)
    for (int j = 0; j < g_nl; j++)
      for (int k = 0; k < g_nl; k++) {
        double e1 = g_lx[i], e2 = g_lx[j], e3 = g_lx[k];
        double h = dl_h(sub(add(u, scl(e1, v)), scl(e2, add(w, scl(e3, z)))), n);
        double k1 = inner_a(e2) * h, k2 = b * e2 * (1.0 - e3) * h, k3 = b * e2 * e3 * h;
        h = dl_h(sub(scl(e2, add(u, scl(e3, v))), add(w, scl(e1, z))), n);
        k1 += a1 * h; k2 += b * (1.0 - e1) * h; k3 += b * e1 * h;
        double ww = g_lw[i] * g_lw[j] * g_lw[k] * e2;
        s1 += ww * k1; s2 += ww * k2; s3 += ww * k3;
      }
  K[0] = jac * s1 / 4.0 / M_PI;
  K[1] = jac * s2 / 4.0 / M_PI;
  K[2] = jac * s3 / 4.0 / M_PI;
}

/* Regular panels, double layer: src/BEM3dLaplace.cpp:386-437. The trial
 * basis is (1 - eta1 - eta2, eta1, eta2) and n the unit normal of the trial
 * triangle w x z. */
void orc_dl_disjoint(const double *pA, const double *pu, const double *pv, const double *pB,
                     const double *pw, const double *pz, double *K)
{
  v3 A = load(pA), u = load(pu), v = load(pv), B = load(pB), w = load(pw), z = load(pz);
  v3 nt = cross(w, z);
  double jt = norm(nt);
  v3 n = scl(1.0 / jt, nt);
  double jac = norm(cross(u, v)) * jt;
  double s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int i = 0; i < g_nt; i++) {
    v3 x = add(A, add(scl(g_tx[i], u), scl(g_ty[i], v)));
    for (int j = 0; j < g_nt; j++) {
      v3 d = sub(sub(sub(x, B), scl(g_tx[j], w)), scl(g_ty[j], z));
      double h = g_tw[i] * g_tw[j] * dl_h(d, n);
      s1 += (1.0 - g_tx[j] - g_ty[j]) * h;
      s2 += g_tx[j] * h;
      s3 += g_ty[j] * h;
    }
  }
  K[0] = jac * s1 / M_PI / 4.0;
  K[1] = jac * s2 / M_PI / 4.0;
  K[2] = jac * s3 / M_PI / 4.0;
}

/* Classification of the pair (test i, trial j) by shared vertices and the
 * local rotations of src/BEM3dLaplace.cpp:692-764. Returns the number of
 * shared vertices (0..3); fills ci/cj (shared local indices, ordered so that
 * cj[1] follows cj[0] cyclically) and ri/rj (the remaining local index). */
static int classify(const int *fi, const int *fj, int *ci, int *cj, int *ri, int *rj)
{
  int nc = 0;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++)
      if (fj[k] == fi[l]) {
        if (nc < 2) { ci[nc] = l; cj[nc] = k; }
        nc++;
        break;
      }
  if (nc == 2 && cj[1] != (cj[0] + 1) % 3) {
    int t = cj[0]; cj[0] = cj[1]; cj[1] = t;
    t = ci[0]; ci[0] = ci[1]; ci[1] = t;
  }
  if (nc == 2) {
    *ri = 3 - ci[0] - ci[1];
    *rj = 3 - cj[0] - cj[1];
  }
  return nc;
}

/* Galerkin entries of one pair: *vij = V(i,j) (P0 SL) and kij[k] the DL weight
 * of trial vertex col[k] (global 0-based vertex ids). Mirrors the switch of
 * getLaplace3d, src/BEM3dLaplace.cpp:641-764 (case 3, a repeated triangle,
 * contributes nothing). Elements are 1-based. */
void orc_pair(const double *nodes, const int *elems, int i, int j, double *vij, double *kij,
              int *col)
{
  const int *fi = elems + 3 * i, *fj = elems + 3 * j;
  v3 Pi[3], Pj[3];
  for (int k = 0; k < 3; k++) {
    Pi[k] = load(nodes + 3 * (fi[k] - 1));
    Pj[k] = load(nodes + 3 * (fj[k] - 1));
  }
  double a[3], b[3], c[3], d[3], A[3], B[3];
  kij[0] = kij[1] = kij[2] = 0.0;
  for (int k = 0; k < 3; k++) col[k] = fj[k] - 1;
  if (i == j) {
    v3 u = sub(Pi[1], Pi[0]), v = sub(Pi[2], Pi[1]);
    memcpy(a, &u, sizeof a); memcpy(b, &v, sizeof b);
    *vij = orc_sl_id(a, b);
    return;
  }
  int ci[2], cj[2], ri = 0, rj = 0;
  int nc = classify(fi, fj, ci, cj, &ri, &rj);
  *vij = 0.0;
  if (nc == 0) {
    v3 u = sub(Pi[1], Pi[0]), v = sub(Pi[2], Pi[0]), w = sub(Pj[1], Pj[0]), z = sub(Pj[2], Pj[0]);
    memcpy(A, &Pi[0], sizeof A); memcpy(B, &Pj[0], sizeof B);
    memcpy(a, &u, sizeof a); memcpy(b, &v, sizeof b); memcpy(c, &w, sizeof c); memcpy(d, &z, sizeof d);
    *vij = orc_sl_disjoint(A, a, b, B, c, d);
    orc_dl_disjoint(A, a, b, B, c, d, kij);
  } else if (nc == 1) {
    int p = ci[0], q = cj[0];
    v3 u = sub(Pi[(p + 1) % 3], Pi[p]), v = sub(Pi[(p + 2) % 3], Pi[(p + 1) % 3]);
    v3 w = sub(Pj[(q + 1) % 3], Pj[q]), z = sub(Pj[(q + 2) % 3], Pj[(q + 1) % 3]);
    memcpy(a, &u, sizeof a); memcpy(b, &v, sizeof b); memcpy(c, &w, sizeof c); memcpy(d, &z, sizeof d);
    *vij = orc_sl_vertex(a, b, c, d);
    orc_dl_vertex(a, b, c, d, kij);
    for (int k = 0; k < 3; k++) col[k] = fj[(q + k) % 3] - 1;
  } else if (nc == 2) {
    v3 u = sub(Pj[cj[1]], Pj[cj[0]]), v = sub(Pi[ri], Pj[cj[1]]), w = sub(Pj[rj], Pj[cj[1]]);
    memcpy(a, &u, sizeof a); memcpy(b, &v, sizeof b); memcpy(c, &w, sizeof c);
    *vij = orc_sl_edge(a, b, c);
    orc_dl_edge(a, b, c, kij);
    col[0] = fj[cj[0]] - 1; col[1] = fj[cj[1]] - 1; col[2] = fj[rj] - 1;
  }
}

/* Matrix-free FP64 apply of selected rows (test triangles rows[r]):
 * v[r] = sum_j V(i,j) t[j], q[r] = sum_j sum_k K(i,j)_k u[col_k]. */
void orc_apply_rows(const double *nodes, int ne, const int *elems, const double *t, const double *u,
                    int nrows, const int *rows, double *v, double *q, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < nrows; r++) {
    int i = rows[r];
    double sv = 0.0, sq = 0.0, vij, kij[3];
    int col[3];
    for (int j = 0; j < ne; j++) {
      orc_pair(nodes, elems, i, j, &vij, kij, col);
      if (t) sv += vij * t[j];
      if (u) sq += kij[0] * u[col[0]] + kij[1] * u[col[1]] + kij[2] * u[col[2]];
    }
    if (v) v[r] = sv;
    if (q) q[r] = sq;
  }
}

/* Dense V (ne x ne, row i = test triangle) and K (ne x nv, row-major). */
void orc_dense(const double *nodes, int nv, int ne, const int *elems, double *V, double *K, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < ne; i++) {
    double vij, kij[3];
    int col[3];
    for (int c = 0; c < nv; c++) K[(size_t)i * nv + c] = 0.0;
    for (int j = 0; j < ne; j++) {
      orc_pair(nodes, elems, i, j, &vij, kij, col);
      V[(size_t)i * ne + j] = vij;
      for (int k = 0; k < 3; k++) K[(size_t)i * nv + col[k]] += kij[k];
    }
  }
}

/* Potential of the single layer of t minus the double layer of u at points
 * (u(x) = V t - W u, the representation formula): src/BEM3dLaplace.cpp:784-843.
 * The triangle rule is the one set by orc_set_rules (index `order`). */
void orc_evaluate(const double *nodes, int ne, const int *elems, int npts, const double *pts,
                  const double *t, const double *u, double *out, int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(static)
  for (int i = 0; i < npts; i++) {
    v3 x = load(pts + 3 * i);
    double acc = 0.0;
    for (int j = 0; j < ne; j++) {
      const int *f = elems + 3 * j;
      v3 A = load(nodes + 3 * (f[0] - 1));
      v3 a = sub(load(nodes + 3 * (f[1] - 1)), A), b = sub(load(nodes + 3 * (f[2] - 1)), A);
      v3 nt = cross(a, b);
      double J = norm(nt);
      v3 n = scl(1.0 / J, nt);
      double u0 = u[f[0] - 1], u1 = u[f[1] - 1], u2 = u[f[2] - 1];
      double s = 0.0;
      for (int k = 0; k < g_nt; k++) {
        v3 d = sub(sub(sub(x, A), scl(g_tx[k], a)), scl(g_ty[k], b));
        double r = norm(d);
        double uh = u0 + (u1 - u0) * g_tx[k] + (u2 - u0) * g_ty[k];
        s += g_tw[k] * (t[j] / r - uh * dot(d, n) / (r * r * r));
      }
      acc += J * s / 4.0 / M_PI;
    }
    out[i] = acc;
  }
}

/* ---- P1 x P1 single layer (no CPU routine in the reference). Restates the
 * reference GPU kernels' Sauter-Schwab formulas in FP64:
 * singleLayer1Laplace3d_idPanels (src/BEM3dLaplaceGPU.cu:82-154),
 * _commonEdge (:211-320), _commonVertex (:371-442), _disjointPanels (:491-557).
 * I[k][l] couples test basis k and trial basis l in each kernel's local vertex
 * order; the host scatter of the reference (:1034-1313) uses the test
 * triangle's vertices for the trial index off the diagonal, which is fixed
 * here (trial indices come from the trial triangle). */
static void p1_self(v3 u, v3 v, double I[3][3])
{
  double S[3][3] = {{0}};
  for (int i = 0; i < g_nl; i++) {
    double e = g_lx[i], w = g_lw[i], e2 = e * e, f;
    f = w * inv_norm(add(scl(e, u), v)); /* D1 */
    S[0][0] += f / 30; S[0][1] += f / 60; S[0][2] += f / 30; S[1][0] += f / 60; S[1][1] += f / 30;
    S[1][2] += f / 30; S[2][0] += f / 30; S[2][1] += f / 30; S[2][2] += f / 10;
    f = w * inv_norm(add(scl(e, v), u)); /* D2 */
    S[0][0] += f / 30; S[0][1] += (2 - e) / 60 * f; S[0][2] += (1 + e) / 60 * f; S[1][0] += (2 - e) / 60 * f;
    S[1][1] += (3 - 3 * e + e2) / 30 * f; S[1][2] += (1 + e - e2) / 30 * f; S[2][0] += (1 + e) / 60 * f;
    S[2][1] += (1 + e - e2) / 30 * f; S[2][2] += (1 + e + e2) / 30 * f;
    f = w * inv_norm(sub(scl(e, add(u, v)), v)); /* D3 */
    S[0][0] += (1 + e + e2) / 30 * f; S[0][1] += (1 + e) / 60 * f; S[0][2] += (1 + e - e2) / 30 * f;
    S[1][0] += (1 + e) / 60 * f; S[1][1] += f / 30; S[1][2] += (2 - e) / 60 * f;
    S[2][0] += (1 + e - e2) / 30 * f; S[2][1] += (2 - e) / 60 * f; S[2][2] += (3 - 3 * e + e2) / 30 * f;
  }
  v3 c = cross(u, v);
  double s = dot(c, c) / 4.0 / M_PI;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++) I[k][l] = s * S[k][l];
}

static void p1_edge(v3 u, v3 v, v3 w, double I[3][3])
{
  double S[3][3] = {{0}};
  v3 uw = add(u, w), uv = add(u, v);
  for (int i = 0; i < g_nl; i++)
    for (int j = 0; j < g_nl; j++) {
      double a = g_lx[i], b = g_lx[j], ww = g_lw[i] * g_lw[j], ab = a * b, f;
      f = ww * a * inv_norm(add(scl(a, sub(scl(b, uw), w)), v)); /* D2 */
      S[0][0] += (1 + ab) / 60 * f; S[0][1] += (3 - 2 * a) / 120 * f; S[0][2] += -a * (b - 1) / 60 * f;
      S[1][0] += (1 + 2 * ab) / 120 * f; S[1][1] += (2 - a) / 60 * f; S[1][2] += -a * (b - 1) / 60 * f;
      S[2][0] += (1 + 3 * ab) / 60 * f; S[2][1] += (4 - 3 * a) / 60 * f; S[2][2] += -a * (b - 1) / 20 * f;
      f = ww * a * inv_norm(add(scl(-a, add(uv, scl(b, w))), v)); /* D3 */
      S[0][0] += (1 + a) / 60 * f; S[0][1] += (1.0 / 40 + (4 * a - ab - 3 * a * ab) / 60) * f;
      S[0][2] += ab * (3 * a + 1) / 60 * f; S[1][0] += f / 120; S[1][1] += (2 - ab) / 60 * f;
      S[1][2] += ab / 60 * f; S[2][0] += (1 - a) / 60 * f; S[2][1] += (3 * ab - 4) * (a - 1) / 60 * f;
      S[2][2] += -ab * (a - 1) / 20 * f;
      f = ww * a * inv_norm(sub(scl(a, sub(v, scl(b, uv))), w)); /* D4 */
      S[0][0] += (1 + ab) / 60 * f; S[0][1] += (1 + 2 * ab) / 120 * f; S[0][2] += (1 + 3 * ab) / 60 * f;
      S[1][0] += (3 - 2 * a) / 120 * f; S[1][1] += (2 - a) / 60 * f; S[1][2] += (4 - 3 * a) / 60 * f;
      S[2][0] += -a * (b - 1) / 60 * f; S[2][1] += -a * (b - 1) / 60 * f; S[2][2] += -a * (b - 1) / 20 * f;
      f = ww * a * inv_norm(add(scl(-a, add(w, scl(b, uv))), v)); /* D5 */
      S[0][0] += (1 + ab) / 60 * f; S[0][1] += (1.0 / 40 + (4 * ab - a - 3 * a * ab) / 60) * f;
      S[0][2] += a * (1 + 3 * ab) / 60 * f; S[1][0] += f / 120; S[1][1] += (2 - a) / 60 * f;
      S[1][2] += a / 60 * f; S[2][0] += (1 - ab) / 60 * f; S[2][1] += (3 * a - 4) * (ab - 1) / 60 * f;
      S[2][2] += -a * (ab - 1) / 20 * f;
      f = ww * inv_norm(sub(add(scl(a, uw), scl(b, v)), w)); /* D1 */
      S[0][0] += (1 + a) / 60 * f; S[0][1] += f / 120; S[0][2] += (1 - a) / 60 * f;
      S[1][0] += (1.0 / 40 + (4 * a - 3 * ab - b) / 60) * f; S[1][1] += (2 - b) / 60 * f;
      S[1][2] += (3 * b - 4) * (a - 1) / 60 * f; S[2][0] += b * (3 * a + 1) / 60 * f; S[2][1] += b / 60 * f;
      S[2][2] += -b * (a - 1) / 20 * f;
    }
  double s = norm(cross(u, v)) * norm(cross(u, w)) / 4.0 / M_PI;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++) I[k][l] = s * S[k][l];
}

static void p1_vertex(v3 u, v3 v, v3 w, v3 z, double I[3][3])
{
  double S[3][3] = {{0}};
  for (int i = 0; i < g_nl; i++)
    for (int j = 0; j < g_nl; j++)
      for (int k = 0; k < g_nl; k++) {
        double e1 = g_lx[i], e2 = g_lx[j], e3 = g_lx[k];
        double ww = g_lw[i] * g_lw[j] * g_lw[k] * e2, f;
        double a11 = 1.0 / 12 - e2 / 20, a12 = e2 * e3 / 20, a13 = -e2 * (e3 - 1) / 20;
        double a21 = -e1 * (4 * e2 - 5) / 20, a22 = e1 * e2 * e3 / 5, a23 = -e1 * e2 * (e3 - 1) / 5;
        double a31 = (4 * e2 - 5) * (e1 - 1) / 20, a32 = -e2 * e3 * (e1 - 1) / 5;
        double a33 = e2 * (e1 - 1) * (e3 - 1) / 5;
        f = ww * inv_norm(sub(add(u, scl(e1, v)), scl(e2, add(w, scl(e3, z)))));
        S[0][0] += a11 * f; S[0][1] += a12 * f; S[0][2] += a13 * f; S[1][0] += a21 * f; S[1][1] += a22 * f;
        S[1][2] += a23 * f; S[2][0] += a31 * f; S[2][1] += a32 * f; S[2][2] += a33 * f;
        f = ww * inv_norm(sub(add(w, scl(e1, z)), scl(e2, add(u, scl(e3, v)))));
        S[0][0] += a11 * f; S[1][0] += a12 * f; S[2][0] += a13 * f; S[0][1] += a21 * f; S[1][1] += a22 * f;
        S[2][1] += a23 * f; S[0][2] += a31 * f; S[1][2] += a32 * f; S[2][2] += a33 * f;
      }
  double s = norm(cross(u, v)) * norm(cross(w, z)) / 4.0 / M_PI;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++) I[k][l] = s * S[k][l];
}

static void p1_disjoint(v3 A, v3 u, v3 v, v3 B, v3 w, v3 z, double I[3][3])
{
  double S[3][3] = {{0}};
  for (int i = 0; i < g_nt; i++) {
    v3 x = add(A, add(scl(g_tx[i], u), scl(g_ty[i], v)));
    double pi[3] = {1 - g_tx[i] - g_ty[i], g_tx[i], g_ty[i]};
    for (int j = 0; j < g_nt; j++) {
      v3 y = add(B, add(scl(g_tx[j], w), scl(g_ty[j], z)));
      double f = g_tw[i] * g_tw[j] * inv_norm(sub(x, y));
      double pj[3] = {1 - g_tx[j] - g_ty[j], g_tx[j], g_ty[j]};
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) S[k][l] += pi[k] * pj[l] * f;
    }
  }
  double s = norm(cross(u, v)) * norm(cross(w, z)) / 4.0 / M_PI;
  for (int k = 0; k < 3; k++)
    for (int l = 0; l < 3; l++) I[k][l] = s * S[k][l];
}

/* P1 entries of pair (test i, trial j): I[k][l] couples vertex ti[k] (0-based)
 * with vertex tj[l]. Returns 0 for a repeated triangle (nothing added). */
int orc_p1_pair(const double *nodes, const int *elems, int i, int j, double *I9, int *ti, int *tj)
{
  const int *fi = elems + 3 * i, *fj = elems + 3 * j;
  v3 Pi[3], Pj[3];
  for (int k = 0; k < 3; k++) {
    Pi[k] = load(nodes + 3 * (fi[k] - 1));
    Pj[k] = load(nodes + 3 * (fj[k] - 1));
  }
  double I[3][3];
  int oi[3] = {0, 1, 2}, oj[3] = {0, 1, 2};
  if (i == j) {
    p1_self(sub(Pi[1], Pi[0]), sub(Pi[2], Pi[1]), I);
  } else {
    int ci[2], cj[2], ri = 0, rj = 0;
    int nc = classify(fi, fj, ci, cj, &ri, &rj);
    if (nc == 0) {
      p1_disjoint(Pi[0], sub(Pi[1], Pi[0]), sub(Pi[2], Pi[0]), Pj[0], sub(Pj[1], Pj[0]), sub(Pj[2], Pj[0]), I);
    } else if (nc == 1) {
      int p = ci[0], q = cj[0];
      for (int k = 0; k < 3; k++) { oi[k] = (p + k) % 3; oj[k] = (q + k) % 3; }
      p1_vertex(sub(Pi[oi[1]], Pi[oi[0]]), sub(Pi[oi[2]], Pi[oi[1]]), sub(Pj[oj[1]], Pj[oj[0]]),
                sub(Pj[oj[2]], Pj[oj[1]]), I);
    } else if (nc == 2) {
      oi[0] = ci[0]; oi[1] = ci[1]; oi[2] = ri;
      oj[0] = cj[0]; oj[1] = cj[1]; oj[2] = rj;
      p1_edge(sub(Pj[cj[1]], Pj[cj[0]]), sub(Pi[ri], Pj[cj[1]]), sub(Pj[rj], Pj[cj[1]]), I);
    } else {
      return 0;
    }
  }
  for (int k = 0; k < 3; k++) {
    ti[k] = fi[oi[k]] - 1;
    tj[k] = fj[oj[k]] - 1;
    for (int l = 0; l < 3; l++) I9[3 * k + l] = I[k][l];
  }
  return 1;
}

/* Dense V1 (nv x nv), row = test vertex. */
void orc_p1_dense(const double *nodes, int nv, int ne, const int *elems, double *V1)
{
  memset(V1, 0, sizeof(double) * (size_t)nv * nv);
  for (int i = 0; i < ne; i++)
    for (int j = 0; j < ne; j++) {
      double I9[9];
      int ti[3], tj[3];
      if (!orc_p1_pair(nodes, elems, i, j, I9, ti, tj)) continue;
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++) V1[(size_t)ti[k] * nv + tj[l]] += I9[3 * k + l];
    }
}
