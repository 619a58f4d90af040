#include "quadrature.h"

#include <cmath>

#include "tri_rules.h"

namespace eb {

static const int kLineSizes[19] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 16, 20, 24, 32, 40, 48, 64};

int line_rule_size(int index) { return (index >= 0 && index < 19) ? kLineSizes[index] : 0; }

int tri_rule_size(int index)
{
  if (index < 0 || index >= 20) return 0;
  int n = 0;
  for (int o = ebq::kTriOrbitOffset[index]; o < ebq::kTriOrbitOffset[index + 1]; o++)
    n += ebq::kTriOrbits[o].kind == 0 ? 1 : (ebq::kTriOrbits[o].kind == 1 ? 3 : 6);
  return n;
}

// Newton iteration on the Legendre polynomial P_n in extended precision,
// starting from the asymptotic guess cos(pi (i - 1/4) / (n + 1/2)); the nodes
// on [-1,1] are mapped to [0,1] and halved weights returned in ascending order.
void gauss_legendre01(int n, double* x, double* w)
{
  for (int i = 0; i < (n + 1) / 2; i++) {
    long double t = std::cos(M_PI * (i + 0.75L) / (n + 0.5L));
    long double dp = 0.0L;
    for (int it = 0; it < 100; it++) {
      long double p0 = 1.0L, p1 = t;
      for (int k = 2; k <= n; k++) {
        long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = t; p0 = 1.0L; }
      dp = n * (t * p1 - p0) / (t * t - 1.0L);
      long double dt = p1 / dp;
      t -= dt;
      if (std::fabs(dt) < 1e-19L) {
        // one more derivative evaluation at the converged node
        p0 = 1.0L; p1 = t;
        for (int k = 2; k <= n; k++) {
          long double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k;
          p0 = p1;
          p1 = p2;
        }
        if (n == 1) { p1 = t; p0 = 1.0L; }
        dp = n * (t * p1 - p0) / (t * t - 1.0L);
        break;
      }
    }
    if (n == 1) { t = 0.0L; dp = 1.0L; }
    long double wt = 2.0L / ((1.0L - t * t) * dp * dp);
    // t > 0 here: the node (1+t)/2 is in the upper half, its mirror in the lower
    x[n - 1 - i] = (double)((1.0L + t) / 2.0L);
    x[i] = (double)((1.0L - t) / 2.0L);
    w[n - 1 - i] = (double)(wt / 2.0L);
    w[i] = (double)(wt / 2.0L);
  }
  if (n % 2 == 1) x[n / 2] = 0.5;
}

int triangle_rule(int index, double* x, double* y, double* w)
{
  int n = 0;
  for (int o = ebq::kTriOrbitOffset[index]; o < ebq::kTriOrbitOffset[index + 1]; o++) {
    const ebq::TriOrbit& r = ebq::kTriOrbits[o];
    if (r.kind == 0) {
      x[n] = r.p0; y[n] = r.p0; w[n] = r.w; n++;
    } else if (r.kind == 1) {
      const double a = r.p0, c = r.p1;
      const double px[3] = {a, a, c}, py[3] = {a, c, a};
      for (int k = 0; k < 3; k++) { x[n] = px[k]; y[n] = py[k]; w[n] = r.w; n++; }
    } else {
      const double a = r.p0, b = r.p1, c = r.p2;
      const double px[6] = {a, b, c, a, b, c}, py[6] = {b, c, a, c, a, b};
      for (int k = 0; k < 6; k++) { x[n] = px[k]; y[n] = py[k]; w[n] = r.w; n++; }
    }
  }
  return n;
}

bool make_quadrature(int order, Quadrature* q)
{
  if (order < 0 || order > kMaxOrder) return false;
  q->order = order;
  q->nl = kLineSizes[order];
  gauss_legendre01(q->nl, q->lx, q->lw);
  q->nt = triangle_rule(order, q->tx, q->ty, q->tw);
  gauss_legendre01(2, q->l2x, q->l2w);
  return true;
}

}  // namespace eb
