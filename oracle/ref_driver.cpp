// Test infrastructure only: a C-ABI driver compiled together with the
// reference's own CPU sources (src/BEM3dLaplace.cpp, src/quadrature.cpp,
// src/func.cpp) into oracle/_ref/libeasybem_ref.so by oracle/Makefile.
//
// It exposes the reference's FP64 pair routines (src/BEM3dLaplace.cpp:22-437),
// its dense assembly getLaplace3d (src/BEM3dLaplace.cpp:561-781) and its
// quadrature tables (src/quadrature.cpp:284-305, :1045-1070) to Python via
// ctypes, plus a matrix-free OpenMP apply that classifies triangle pairs the
// way getLaplace3d does (:692-764) and calls the reference pair routines.
// Nothing in the product links this file; only tests, smoke() and the CPU
// baseline leg of bench.py load the resulting library.

#include <cmath>
#include <cstring>
#include <cstdlib>
#include <omp.h>

#include "quadrature.h"
#include "BEM3dLaplace.h"

// Globals defined (non-static) in src/BEM3dLaplace.cpp:12-19.
extern double *qPoints2, *qWeights2;
extern double *qPoints3, *qWeights3;
extern double *qPoints4, *qWeights4;
extern int quadn;
extern double *qPoints, *qWeights;
extern int quadTrin;
extern Point2D *qTriPoints;
extern double *qTriWeights;

// Pair routines exported by src/BEM3dLaplace.cpp:22-437 (no header declares them).
double SingleLayerLaplace3d_idPanels(double *us, double *vs);
double SingleLayerLaplace3d_commonEdge(double *us, double *vs, double *ws);
double SingleLayerLaplace3d_commonVertex(double *us, double *vs, double *ws, double *zs);
double SingleLayerLaplace3d_disjointPanels(double *As, double *us, double *vs,
                                           double *Bs, double *ws, double *zs);
void DoubleLayerLaplace3d_commonEdge(double *us, double *vs, double *ws, double *Kij);
void DoubleLayerLaplace3d_commonVertex(double *us, double *vs, double *ws, double *zs,
                                       double *Kij);
void DoubleLayerLaplace3d_disjointPanels(double *As, double *us, double *vs,
                                         double *Bs, double *ws, double *zs,
                                         double *Kij);

extern "C" {

// Select the quadrature index exactly as getLaplace3d does (:581-592).
void ref_set_order(int order)
{
  quadn = LineQuadratureSizes[order];
  qPoints = LineQuadraturePoints[order];
  qWeights = LineQuadratureWeights[order];
  quadTrin = TriangleQuadratureSizes[order];
  qTriPoints = TriangleQuadraturePoints[order];
  qTriWeights = TriangleQuadratureWeights[order];
  qPoints2 = LineQuadraturePoints[1];
  qWeights2 = LineQuadratureWeights[1];
  qPoints3 = LineQuadraturePoints[2];
  qWeights3 = LineQuadratureWeights[2];
  qPoints4 = LineQuadraturePoints[3];
  qWeights4 = LineQuadratureWeights[3];
}

int ref_line_size(int idx) { return LineQuadratureSizes[idx]; }
int ref_tri_size(int idx) { return TriangleQuadratureSizes[idx]; }

void ref_line_rule(int idx, double *pts, double *wts)
{
  for (int i = 0; i < LineQuadratureSizes[idx]; i++) {
    pts[i] = LineQuadraturePoints[idx][i];
    wts[i] = LineQuadratureWeights[idx][i];
  }
}

void ref_tri_rule(int idx, double *xy, double *wts)
{
  for (int i = 0; i < TriangleQuadratureSizes[idx]; i++) {
    xy[2 * i] = TriangleQuadraturePoints[idx][i].x;
    xy[2 * i + 1] = TriangleQuadraturePoints[idx][i].y;
    wts[i] = TriangleQuadratureWeights[idx][i];
  }
}

double ref_sl_id(double *u, double *v) { return SingleLayerLaplace3d_idPanels(u, v); }
double ref_sl_edge(double *u, double *v, double *w) { return SingleLayerLaplace3d_commonEdge(u, v, w); }
double ref_sl_vertex(double *u, double *v, double *w, double *z)
{ return SingleLayerLaplace3d_commonVertex(u, v, w, z); }
double ref_sl_disjoint(double *A, double *u, double *v, double *B, double *w, double *z)
{ return SingleLayerLaplace3d_disjointPanels(A, u, v, B, w, z); }
void ref_dl_edge(double *u, double *v, double *w, double *K) { DoubleLayerLaplace3d_commonEdge(u, v, w, K); }
void ref_dl_vertex(double *u, double *v, double *w, double *z, double *K)
{ DoubleLayerLaplace3d_commonVertex(u, v, w, z, K); }
void ref_dl_disjoint(double *A, double *u, double *v, double *B, double *w, double *z, double *K)
{ DoubleLayerLaplace3d_disjointPanels(A, u, v, B, w, z, K); }

// Dense FP64 assembly by the reference (row-major C++ layout as written by
// getLaplace3d: V[i*ne+j], K[i+node*ne], D[a+b*np], M[i+node*ne]).
void ref_get_laplace3d(int np, const double *nodes, int ne, const int *elems, int order,
                       double *V, double *K, double *D, double *M)
{
  double *V0 = nullptr, *K0 = nullptr, *D0 = nullptr, *M0 = nullptr;
  getLaplace3d(np, nodes, ne, elems, V0, K0, D0, M0, order);
  std::memcpy(V, V0, sizeof(double) * (size_t)ne * ne);
  std::memcpy(K, K0, sizeof(double) * (size_t)ne * np);
  std::memcpy(D, D0, sizeof(double) * (size_t)np * np);
  std::memcpy(M, M0, sizeof(double) * (size_t)ne * np);
  delete[] V0; delete[] K0; delete[] D0; delete[] M0;
}

void ref_get_mass(int np, const double *nodes, int ne, const int *elems, double *M)
{
  double *M0 = nullptr;
  getLaplace3dMass(np, nodes, ne, elems, M0);
  std::memcpy(M, M0, sizeof(double) * (size_t)ne * np);
  delete[] M0;
}

void ref_evaluate(const double *nodes, int ne, const int *elems, int npts, const double *pts,
                  const double *t, const double *u, int order, double *out)
{
  double *r = nullptr;
  evaluateLaplace3d(nodes, ne, elems, npts, pts, t, u, r, order);
  std::memcpy(out, r, sizeof(double) * npts);
  delete[] r;
}

// Matrix-free FP64 apply of the selected rows: v[r] = sum_j V(i,j) t[j] and
// q[r] = sum_j K(i,:) u for i = rows[r]. Pair classification, local vertex
// rotations and DL scatter follow getLaplace3d (:692-764). The quadrature
// index must have been set with ref_set_order.
void ref_apply_rows(int np, const double *nodes, int ne, const int *elems,
                    const double *t, const double *u, int nrows, const int *rows,
                    double *v, double *q, int nthreads)
{
  (void)np;
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1)
  for (int r = 0; r < nrows; r++) {
    const int i = rows[r];
    int fi[3], fj[3];
    double Pi[3][3], Pj[3][3], a[3], b[3], c[3], d[3], Kij[3];
    for (int k = 0; k < 3; k++) fi[k] = elems[3 * i + k];
    for (int k = 0; k < 3; k++) std::memcpy(Pi[k], nodes + 3 * (fi[k] - 1), 3 * sizeof(double));
    double sv = 0.0, sq = 0.0;
    for (int j = 0; j < ne; j++) {
      if (j == i) {
        for (int k = 0; k < 3; k++) { a[k] = Pi[1][k] - Pi[0][k]; b[k] = Pi[2][k] - Pi[1][k]; }
        sv += SingleLayerLaplace3d_idPanels(a, b) * t[j];
        continue;
      }
      for (int k = 0; k < 3; k++) fj[k] = elems[3 * j + k];
      for (int k = 0; k < 3; k++) std::memcpy(Pj[k], nodes + 3 * (fj[k] - 1), 3 * sizeof(double));
      int ci[2], cj[2], nc = 0;
      for (int k = 0; k < 3; k++)
        for (int l = 0; l < 3; l++)
          if (fj[k] == fi[l]) { if (nc < 2) { ci[nc] = l; cj[nc] = k; } nc++; break; }
      if (nc == 2 && ((cj[0] == 0 && cj[1] == 2) || (cj[0] == 1 && cj[1] == 0) ||
                      (cj[0] == 2 && cj[1] == 1))) {
        int tmp = cj[0]; cj[0] = cj[1]; cj[1] = tmp;
        tmp = ci[0]; ci[0] = ci[1]; ci[1] = tmp;
      }
      if (nc == 0) {
        for (int k = 0; k < 3; k++) {
          a[k] = Pi[1][k] - Pi[0][k]; b[k] = Pi[2][k] - Pi[0][k];
          c[k] = Pj[1][k] - Pj[0][k]; d[k] = Pj[2][k] - Pj[0][k];
        }
        sv += SingleLayerLaplace3d_disjointPanels(Pi[0], a, b, Pj[0], c, d) * t[j];
        DoubleLayerLaplace3d_disjointPanels(Pi[0], a, b, Pj[0], c, d, Kij);
        for (int k = 0; k < 3; k++) sq += Kij[k] * u[fj[k] - 1];
      } else if (nc == 1) {
        for (int k = 0; k < 3; k++) {
          a[k] = Pi[(ci[0] + 1) % 3][k] - Pi[ci[0]][k];
          b[k] = Pi[(ci[0] + 2) % 3][k] - Pi[(ci[0] + 1) % 3][k];
          c[k] = Pj[(cj[0] + 1) % 3][k] - Pj[cj[0]][k];
          d[k] = Pj[(cj[0] + 2) % 3][k] - Pj[(cj[0] + 1) % 3][k];
        }
        sv += SingleLayerLaplace3d_commonVertex(a, b, c, d) * t[j];
        DoubleLayerLaplace3d_commonVertex(a, b, c, d, Kij);
        for (int k = 0; k < 3; k++) sq += Kij[k] * u[fj[(cj[0] + k) % 3] - 1];
      } else if (nc == 2) {
        int ri = 0, rj = 0;
        for (int k = 0; k < 3; k++) {
          if (k != ci[0] && k != ci[1]) ri = k;
          if (k != cj[0] && k != cj[1]) rj = k;
        }
        for (int k = 0; k < 3; k++) {
          a[k] = Pj[cj[1]][k] - Pj[cj[0]][k];
          b[k] = Pi[ri][k] - Pj[cj[1]][k];
          c[k] = Pj[rj][k] - Pj[cj[1]][k];
        }
        sv += SingleLayerLaplace3d_commonEdge(a, b, c) * t[j];
        DoubleLayerLaplace3d_commonEdge(a, b, c, Kij);
        sq += Kij[0] * u[fj[cj[0]] - 1] + Kij[1] * u[fj[cj[1]] - 1] + Kij[2] * u[fj[rj] - 1];
      }
      // nc == 3 (a repeated triangle): getLaplace3d has no case and adds nothing.
    }
    v[r] = sv;
    q[r] = sq;
  }
}

}  // extern "C"
