// pg_roots.h -- edge/interface intersection for the enrichment nodes.
//
// The reference locates each enrichment node with a Steffensen iteration started at the edge
// midpoint (tolerance 1e-7 on successive root estimates, at most 25 iterations) and falls back
// to Brent's bracketing method on [0, 1] (tolerance 1e-7 on the bracket, at most 100 iterations)
// when the iteration stalls or leaves the edge (src/Inclusion.cpp:32-121).  The same two
// published methods are written out here so that the enrichment-node coordinates follow the
// same iterate sequence:
//   * Steffensen acceleration: Newton iterates x_{k+1} = x_k - f/f'; from the third iterate on,
//     the reported root is the Aitken delta-squared extrapolation of the last three iterates.
//   * Brent (1973), "Algorithms for Minimization without Derivatives", ch. 4: inverse quadratic
//     / secant steps inside a sign-change bracket, bisection when they are not safe.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define PG_HD __host__ __device__
#else
#define PG_HD
#endif

namespace pg {

PG_HD inline double roots_min(double a, double b) { return a < b ? a : b; }

// f(alpha) and f'(alpha) of the level set along an edge; F provides eval(alpha, &f, &df).  The
// same code runs in the host set-up and in the device preprocessing (pg_prep.cu).
template <class F>
PG_HD double steffensen_then_brent(const F& fn) {
  // --- Steffensen from alpha = 0.5
  double x = 0.5, f, df;
  fn.eval(x, &f, &df);
  double x1 = 0.0, x2 = 0.0;
  int count = 1;
  double root = x, alpha = 0.5, alpha0;
  int iter = 0;
  const int max_iter = 25;
  bool cont = true;
  while (cont && iter < max_iter) {
    iter++;
    if (df == 0.0) {  // the reference would report an error from the solver; the root stays put
      alpha0 = alpha;
      alpha = root;
    } else {
      double xn = x - f / df;
      double fn_, dfn;
      fn.eval(xn, &fn_, &dfn);
      x2 = x1; x1 = x; x = xn; f = fn_; df = dfn;
      if (count >= 3) {
        double u = x1 - x2;
        double v = x - 2.0 * x1 + x2;
        root = (v == 0.0) ? x : x2 - u * u / v;
      } else {
        root = x;
        count++;
      }
      alpha0 = alpha;
      alpha = root;
    }
    // converged when |alpha - alpha0| < 1e-7
    cont = !(alpha == alpha0 || fabs(alpha - alpha0) < 1e-7);
  }
  if (!(iter == max_iter || alpha < 0.0 || alpha > 1.0)) return alpha;

  // --- Brent on [0, 1]
  double a = 0.0, b = 1.0, c, fa, fb, fc, d, e;
  fn.eval(a, &fa, &df);
  fn.eval(b, &fb, &df);
  c = a; fc = fa; d = b - a; e = d;
  double xlo = 0.0, xhi = 1.0;
  iter = 0;
  do {
    iter++;
    if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) { c = a; fc = fa; d = b - a; e = d; }
    if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
    const double tol = 0.5 * 2.220446049250313e-16 * fabs(b);
    const double m = 0.5 * (c - b);
    if (fb == 0.0) { alpha = b; xlo = b; xhi = b; }
    else if (fabs(m) <= tol) {
      alpha = b;
      if (b < c) { xlo = b; xhi = c; } else { xlo = c; xhi = b; }
    } else {
      if (fabs(e) < tol || fabs(fa) <= fabs(fb)) { d = m; e = m; }
      else {
        double p, q, r, ss = fb / fa;
        if (a == c) { p = 2 * m * ss; q = 1 - ss; }
        else {
          q = fa / fc; r = fb / fc;
          p = ss * (2 * m * q * (q - r) - (b - a) * (r - 1));
          q = (q - 1) * (r - 1) * (ss - 1);
        }
        if (p > 0) q = -q; else p = -p;
        if (2 * p < roots_min(3 * m * q - fabs(tol * q), fabs(e * q))) { e = d; d = p / q; }
        else { d = m; e = m; }
      }
      a = b; fa = fb;
      if (fabs(d) > tol) b += d; else b += (m > 0 ? +tol : -tol);
      fn.eval(b, &fb, &df);
      alpha = b;
      if ((fb < 0 && fc < 0) || (fb > 0 && fc > 0)) c = a;
      if (b < c) { xlo = b; xhi = c; } else { xlo = c; xhi = b; }
      fc = (c == a) ? fa : fc;
    }
  } while (!(xlo == xhi || fabs(xlo - xhi) < 1e-7) && iter < 100);
  return alpha;
}

}  // namespace pg
