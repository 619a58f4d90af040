// Quadrature rules indexed the way easybem indexes them: one integer `order`
// selects both the Gauss-Legendre rule on [0,1] used by the Sauter-Schwab
// integrals (src/quadrature.cpp:284-305, sizes {1..12,16,20,24,32,40,48,64})
// and the symmetric triangle rule used for regular pairs
// (src/quadrature.cpp:1045-1070, sizes {1,3,4,6,7,12,...,79}). The default
// order 4 gives 5 line points and the 7-point degree-5 triangle rule.
#pragma once

namespace eb {

constexpr int kMaxLine = 64;
constexpr int kMaxTri = 79;
constexpr int kMaxOrder = 18;  // largest index valid for both tables

struct Quadrature {
  int order;
  int nl;                 // line points
  double lx[kMaxLine];    // Gauss-Legendre nodes on [0,1], ascending
  double lw[kMaxLine];    // weights, summing to 1
  int nt;                 // triangle points
  double tx[kMaxTri];     // reference-triangle coordinates (0,0),(1,0),(0,1)
  double ty[kMaxTri];
  double tw[kMaxTri];     // weights, summing to 1/2
  double l2x[2], l2w[2];  // the fixed 2-point line rule (index 1) of the DL inner integral
};

int line_rule_size(int index);
int tri_rule_size(int index);
// Fills the n-point Gauss-Legendre rule on [0,1] (ascending nodes).
void gauss_legendre01(int n, double* x, double* w);
// Expands triangle rule `index` (0..19) into x, y, w; returns its size.
int triangle_rule(int index, double* x, double* y, double* w);
// Returns false when `order` is outside 0..kMaxOrder.
bool make_quadrature(int order, Quadrature* q);

}  // namespace eb
