// pg_setup.cpp -- host-side IGFEM set-up (see pg_setup.h).
//
// Reference steps restated here (paths relative to the PIGFEM source tree):
//   structured mesh ............ src/Mesh.cpp:236-647 (Mesh::generate_mesh), periodic sets 649-760
//   node detection ............. src/Mesh.cpp:2883-2929, src/InclusionCircle.cpp:142-163,
//                                src/InclusionSphere.cpp:156-178
//   cut-case tables ............ src/tri3.cpp:287-441 (Tri3::detection), src/tet4.cpp (Tet4::detection)
//   enrichment nodes ........... src/Mesh.cpp:3103-3252 (Mesh::add_enrichments, serial),
//                                src/Mesh.cpp:3661-3720 (add_enrich_node_to_elem), src/Inclusion.cpp:32-121
//   sub-elements ............... src/elem.cpp:428-558 (generate_integration_elem, transformDetectionCohToReg)
//   quadrature data ............ src/Mesh.cpp:1475-1643 (Mesh::store_shape_functions),
//                                src/elem.cpp:115-139, src/Utilities.cpp:1017-1072 (det / inverse),
//                                src/tri3.cpp:93-208, src/quad4.cpp:65-150, src/Polygon.cpp:51-228,
//                                src/CohEdge2.cpp:55-200, src/CohesiveElem.cpp:140-238
//   DOF numbering .............. src/DofObject.cpp:241-535
//   CSR pattern ................ src/Assembler.cpp:659-679 (every element DOF pair is inserted)
//   linear elastic D ........... src/material_lei.cpp:52-97
#include "pg_setup.h"
#include "pg_roots.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <thread>
#include <set>
#include <sstream>
#include <tuple>
#include <utility>

namespace pg {
namespace {

// Host threads for the set-up's independent loops: PIGFEM_SETUP_THREADS, else the hardware
// concurrency, at most 8.  Results do not depend on the count: every parallel loop writes
// disjoint outputs, and anything order-dependent is laid out from per-chunk counts first.
int setup_threads() {
  static const int n = [] {
    const char* e = std::getenv("PIGFEM_SETUP_THREADS");
    int v = e ? std::atoi(e) : (int)std::thread::hardware_concurrency();
    return std::max(1, std::min(v, 8));
  }();
  return n;
}

// f(chunk, begin, end) over nt contiguous chunks of [0, n), chunk k on its own thread.
template <class F>
void chunked(int n, int nt, F f) {
  if (nt <= 1 || n < 2) { f(0, 0, n); return; }
  std::vector<std::thread> th;
  const int step = (n + nt - 1) / nt;
  for (int k = 0; k < nt; ++k) {
    const int a = std::min(n, k * step), b = std::min(n, a + step);
    th.emplace_back(f, k, a, b);
  }
  for (auto& t : th) t.join();
}

const double kPI = 3.14159265358979323846264338327950;

// ------------------------------------------------------------------ small dense helpers
// det / inverse exactly as the reference's Utilities::det / Utilities::inverse compute them.
double det2(const double J[2][2]) { return J[0][0] * J[1][1] - J[0][1] * J[1][0]; }
double det3(const double J[3][3]) {
  return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) - J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
         J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}
void inv2(const double J[2][2], double R[2][2]) {
  double d = det2(J);
  double s = 1.0 / d;
  R[0][0] = J[1][1] * s; R[1][1] = J[0][0] * s; R[0][1] = (-1.0 * J[0][1]) * s; R[1][0] = (-1.0 * J[1][0]) * s;
}
void inv3(const double J[3][3], double R[3][3]) {
  R[0][0] = J[1][1] * J[2][2] - J[2][1] * J[1][2];
  R[0][1] = -1.0 * (J[0][1] * J[2][2] - J[2][1] * J[0][2]);
  R[0][2] = J[0][1] * J[1][2] - J[1][1] * J[0][2];
  R[1][0] = -1.0 * (J[1][0] * J[2][2] - J[2][0] * J[1][2]);
  R[1][1] = J[0][0] * J[2][2] - J[2][0] * J[0][2];
  R[1][2] = -1.0 * (J[0][0] * J[1][2] - J[1][0] * J[0][2]);
  R[2][0] = J[1][0] * J[2][1] - J[2][0] * J[1][1];
  R[2][1] = -1.0 * (J[0][0] * J[2][1] - J[2][0] * J[0][1]);
  R[2][2] = J[0][0] * J[1][1] - J[1][0] * J[0][1];
  double s = 1.0 / det3(J);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) R[i][j] *= s;
}

// Maps reference-coordinate gradients dNdr (n x dim) through the element geometry (node
// coordinates xs, n x dim) to physical gradients dNdx and the Jacobian determinant
// (Elem::transform_gradients).
void transform_gradients(int dim, int n, const double* dNdr, const double* xs, double* dNdx, double* J) {
  if (dim == 2) {
    double Jac[2][2] = {{0, 0}, {0, 0}};
    for (int a = 0; a < 2; ++a) for (int i = 0; i < 2; ++i) for (int k = 0; k < n; ++k) Jac[a][i] += dNdr[k * 2 + a] * xs[k * 2 + i];
    *J = det2(Jac);
    double R[2][2]; inv2(Jac, R);
    for (int k = 0; k < n; ++k)
      for (int i = 0; i < 2; ++i) dNdx[k * 2 + i] = R[i][0] * dNdr[k * 2 + 0] + R[i][1] * dNdr[k * 2 + 1];
  } else {
    double Jac[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int a = 0; a < 3; ++a) for (int i = 0; i < 3; ++i) for (int k = 0; k < n; ++k) Jac[a][i] += dNdr[k * 3 + a] * xs[k * 3 + i];
    *J = det3(Jac);
    double R[3][3]; inv3(Jac, R);
    for (int k = 0; k < n; ++k)
      for (int i = 0; i < 3; ++i)
        dNdx[k * 3 + i] = R[i][0] * dNdr[k * 3 + 0] + R[i][1] * dNdr[k * 3 + 1] + R[i][2] * dNdr[k * 3 + 2];
  }
}

// ------------------------------------------------------------------ quadrature rules
// Tri3 order 3 (src/tri3.cpp:111-118): the 4-point rule with a negative centroid weight.
const double kTri4[4][3] = {
    {0.333333333333333333333333333333333, 0.333333333333333333333333333333333, -0.281250000000000000000000000000000},
    {0.200000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665},
    {0.200000000000000000000000000000000, 0.600000000000000000000000000000000, 0.260416666666666666666666666666665},
    {0.600000000000000000000000000000000, 0.200000000000000000000000000000000, 0.260416666666666666666666666666665}};
// Tet4 order 3 (src/tet4.cpp:109-118): 5 points, centroid weight -0.8, weights summing to 1.
const double kTet5[5][4] = {{0.25, 0.25, 0.25, -0.8},
                            {0.5, 0.166666666666667, 0.166666666666667, 0.45},
                            {0.166666666666667, 0.166666666666667, 0.166666666666667, 0.45},
                            {0.166666666666667, 0.166666666666667, 0.5, 0.45},
                            {0.166666666666667, 0.5, 0.166666666666667, 0.45}};
// Gauss-Legendre 2-point (edge order 3).
const double kGauss2 = 0.57735026918962576450914878050196;

void tri3_shape(double r, double s, double* N, double* dN) {
  N[0] = 1.0 - r - s; N[1] = r; N[2] = s;
  dN[0] = -1.0; dN[1] = -1.0; dN[2] = 1.0; dN[3] = 0.0; dN[4] = 0.0; dN[5] = 1.0;
}
void quad4_shape(double r, double s, double* N, double* dN) {
  N[0] = 0.25 * (1.0 - r) * (1.0 - s); N[1] = 0.25 * (1.0 + r) * (1.0 - s);
  N[2] = 0.25 * (1.0 + r) * (1.0 + s); N[3] = 0.25 * (1.0 - r) * (1.0 + s);
  dN[0] = -0.25 * (1.0 - s); dN[1] = -0.25 * (1.0 - r);
  dN[2] = 0.25 * (1.0 - s);  dN[3] = -0.25 * (1.0 + r);
  dN[4] = 0.25 * (1.0 + s);  dN[5] = 0.25 * (1.0 + r);
  dN[6] = -0.25 * (1.0 + s); dN[7] = 0.25 * (1.0 - r);
}
// Elem::inverse_map for a quad4 parent (src/elem.cpp:697-765): the parent coordinates of the
// global point g, by Newton steps on x(r, s) = sum_a N_a(r, s) x_a - g from (0, 0), each step
// followed by the reference's residual test (|x - g| < 1e-12 per component, at most 1000 steps).
// On the structured grid's rectangles x is affine in (r, s), so the first step lands on the
// point.  Returns false when the point is outside the parent (Quad4::coords_inside, tolerance
// 1e-12 on the reference square).
bool quad4_inverse(const double* xs, const double* g, double* rs) {
  double r = 0.0, t = 0.0;
  for (int it = 0; it < 1000; ++it) {
    double N[4], dN[8], f[2] = {-g[0], -g[1]}, J[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
    quad4_shape(r, t, N, dN);
    for (int n = 0; n < 4; ++n)
      for (int i = 0; i < 2; ++i) {
        f[i] += N[n] * xs[n * 2 + i];
        for (int a = 0; a < 2; ++a) J[i][a] += dN[n * 2 + a] * xs[n * 2 + i];
      }
    const double det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    if (det == 0.0) return false;
    r -= (J[1][1] * f[0] - J[0][1] * f[1]) / det;
    t -= (-J[1][0] * f[0] + J[0][0] * f[1]) / det;
    quad4_shape(r, t, N, dN);
    double res[2] = {-g[0], -g[1]};
    for (int n = 0; n < 4; ++n) for (int i = 0; i < 2; ++i) res[i] += N[n] * xs[n * 2 + i];
    if (std::fabs(res[0]) < 1e-12 && std::fabs(res[1]) < 1e-12) break;
  }
  rs[0] = r; rs[1] = t;
  const double tol = 1e-12;
  return r >= -1.0 - tol && r <= 1.0 + tol && t >= -1.0 - tol && t <= 1.0 + tol;
}

// Quad4 order 3: tensor product of the 2-point edge rule, qp -> (qp % 2, qp / 2) (src/quad4.cpp:108-127).
void quad4_qp(int qp, double* r, double* s, double* w) {
  const double g[2] = {-kGauss2, kGauss2};
  *r = g[qp % 2]; *s = g[qp / 2]; *w = 1.0 * 1.0;
}

// Polygon (Wachspress over the regular reference polygon), src/Polygon.cpp:51-228.
void poly_points(int nn, double px[], double py[]) {
  for (int n = 0; n < nn; ++n) {
    px[n] = std::cos(2.0 * kPI * (n + 1) / nn);
    py[n] = std::sin(2.0 * kPI * (n + 1) / nn);
  }
}
void poly_tri(int nn, int t, int tri[3]) { tri[0] = nn; tri[1] = t; tri[2] = (t == nn - 1) ? 0 : t + 1; }
// Reached through an Elem* in Mesh::store_shape_functions, so the order is Elem's default 3, not
// Polygon's own default: 4 points (tri3 order 3) on each triangle of the fan.
void poly_qp(int nn, int qp, double* r, double* s, double* w) {
  double px[32], py[32];
  poly_points(nn, px, py);
  px[nn] = 0.0; py[nn] = 0.0;
  const int t = qp / 4, q = qp % 4;
  double tN[3], tdN[6];
  tri3_shape(kTri4[q][0], kTri4[q][1], tN, tdN);
  int tri[3]; poly_tri(nn, t, tri);
  double J0[2][2] = {{0, 0}, {0, 0}};
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j)
      for (int n = 0; n < 3; ++n) J0[i][j] += (i == 0 ? px[tri[n]] : py[tri[n]]) * tdN[n * 2 + j];
  double dJ = J0[0][0] * J0[1][1] - J0[0][1] * J0[1][0];
  *w = dJ * kTri4[q][2];
  double cx = 0.0, cy = 0.0;
  for (int n = 0; n < 3; ++n) { cx += tN[n] * px[tri[n]]; cy += tN[n] * py[tri[n]]; }
  *r = cx; *s = cy;
}
void poly_shape(int nn, double r, double s, double* N, double* dN) {
  double px[33], py[33];
  poly_points(nn, px, py);
  px[nn] = r; py[nn] = s;
  double A[33], dA[33][2], alpha[32], dal[32][2];
  for (int n = 0; n < nn; ++n) {
    int tri[3]; poly_tri(nn, n, tri);
    const double x0 = px[tri[0]], y0 = py[tri[0]], x1 = px[tri[1]], y1 = py[tri[1]], x2 = px[tri[2]], y2 = py[tri[2]];
    A[n + 1] = 0.5 * ((x1 * y2 - y1 * x2) - (x0 * y2 - y0 * x2) + (x0 * y1 - y0 * x1));
    dA[n + 1][0] = 0.5 * (y2 - y1);
    dA[n + 1][1] = 0.5 * (x1 - x2);
  }
  A[0] = A[nn]; dA[0][0] = dA[nn][0]; dA[0][1] = dA[nn][1];
  double sa = 0.0, sd0 = 0.0, sd1 = 0.0;
  for (int n = 0; n < nn; ++n) {
    alpha[n] = 1.0 / (A[n] * A[n + 1]);
    dal[n][0] = -1.0 * alpha[n] * (dA[n][0] / A[n] + dA[n + 1][0] / A[n + 1]);
    dal[n][1] = -1.0 * alpha[n] * (dA[n][1] / A[n] + dA[n + 1][1] / A[n + 1]);
    sa += alpha[n]; sd0 += dal[n][0]; sd1 += dal[n][1];
  }
  for (int n = 0; n < nn; ++n) {
    if (N) N[n] = alpha[n] / sa;
    double Nn = alpha[n] / sa;
    dN[n * 2 + 0] = (dal[n][0] - Nn * sd0) / sa;
    dN[n * 2 + 1] = (dal[n][1] - Nn * sd1) / sa;
  }
}

void tet4_shape(double r, double s, double t, double* N, double* dN) {
  N[0] = 1.0 - r - s - t; N[1] = r; N[2] = s; N[3] = t;
  const double g[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
  for (int i = 0; i < 12; ++i) dN[i] = g[i];
}

// ------------------------------------------------------------------ inclusions
struct Inclusion {
  int dim;
  double c[3], r;
  // Bounding box used by Mesh::detect_node before the exact test.  The sphere's upper z bound is
  // the centre's y coordinate plus r, as the reference writes it (src/InclusionSphere.cpp:158).
  bool in_box(const double* x) const {
    if (dim == 2) return (c[0] - r <= x[0]) && (c[1] - r <= x[1]) && (x[0] <= c[0] + r) && (x[1] <= c[1] + r);
    return (c[0] - r <= x[0]) && (c[1] - r <= x[1]) && (c[2] - r <= x[2]) && (x[0] <= c[0] + r) && (x[1] <= c[1] + r) &&
           (x[2] <= c[1] + r);
  }
  // 0 outside, 1 on the surface (within 1e-12), 2 inside.
  int detect(const double* x) const {
    double val;
    if (dim == 2) {
      double dx = x[0] - c[0], dy = x[1] - c[1];
      val = (std::sqrt(dx * dx + dy * dy) - r) / r;
    } else {
      double gx = x[0] - c[0], gy = x[1] - c[1], gz = x[2] - c[2];
      val = std::pow(gx / r, 2) + std::pow(gy / r, 2) + std::pow(gz / r, 2) - 1.0;
    }
    if (val > 1e-12) return 0;
    if (val < -1e-12) return 2;
    return 1;
  }
  // level set along the edge p0 -> p1 and its derivative (InclusionCircle::int_fdf / InclusionSphere)
  void fdf(const double* p0, const double* p1, double a, double* f, double* df) const {
    if (dim == 2) {
      double g0 = p0[0] + a * (p1[0] - p0[0]) - c[0];
      double g1 = p0[1] + a * (p1[1] - p0[1]) - c[1];
      double d0 = p1[0] - p0[0], d1 = p1[1] - p0[1];
      *f = std::pow(g0 / r, 2) + std::pow(g1 / r, 2) - 1;
      *df = (1 / (r * r)) * 2.0 * (g0 * d0 + g1 * d1);
    } else {
      double g0 = p0[0] + a * (p1[0] - p0[0]) - c[0];
      double g1 = p0[1] + a * (p1[1] - p0[1]) - c[1];
      double g2 = p0[2] + a * (p1[2] - p0[2]) - c[2];
      double d0 = p1[0] - p0[0], d1 = p1[1] - p0[1], d2 = p1[2] - p0[2];
      *f = std::pow(g0 / r, 2) + std::pow(g1 / r, 2) + std::pow(g2 / r, 2) - 1.0;
      *df = (2.0 / (r * r)) * (g0 * d0 + g1 * d1 + g2 * d2);
    }
  }
};

struct EdgeFn {
  const Inclusion* inc;
  const double* p0;
  const double* p1;
  void eval(double a, double* f, double* df) const { inc->fdf(p0, p1, a, f, df); }
};

// ------------------------------------------------------------------ cut-case tables
struct CutCase {
  std::vector<int> cut_edge;   // local edge of each enrichment node
  std::vector<int> incl;       // inclusion of each enrichment node
  std::vector<std::vector<int>> sub;   // sub-element local node lists (parent 0..npe-1, enrichment npe.., mirrors after)
  std::vector<int> sub_mat;    // -1 = the element's own material, k >= 0 = inclusion k's material
  std::vector<std::vector<int>> coh;   // cohesive element local node lists
};

// Tri3::detection (src/tri3.cpp:287-441): node detection values -> cut case (cohesive numbering).
bool tri3_case(const int nd[3], CutCase& cc) {
  const int n0 = nd[0], n1 = nd[1], n2 = nd[2];
  const bool n0e1 = n0 == n1, n0e2 = n0 == n2, n1e2 = n1 == n2;
  std::vector<int> v = {n0, n1, n2};
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  const int nu = (int)v.size();
  if (nu == 1) return false;
  auto M = [](int k) { return k; };  // inclusion index as material selector (-1 = element material)
  if (nu == 2) {
    if (v[0] < 0) {
      if (n1e2) {
        cc.cut_edge = {2, 0}; cc.sub_mat = {M(n0), M(n1)};
        if (n0 < n1) { cc.sub = {{0, 4, 3}, {1, 2, 5, 6}}; cc.coh = {{3, 4, 5, 6}}; }
        else { cc.sub = {{0, 6, 5}, {1, 2, 3, 4}}; cc.coh = {{4, 3, 6, 5}}; }
      } else if (n0e2) {
        cc.cut_edge = {0, 1}; cc.sub_mat = {M(n1), M(n0)};
        if (n1 < n0) { cc.sub = {{1, 4, 3}, {2, 0, 5, 6}}; cc.coh = {{3, 4, 5, 6}}; }
        else { cc.sub = {{1, 6, 5}, {2, 0, 3, 4}}; cc.coh = {{4, 3, 6, 5}}; }
      } else {
        cc.cut_edge = {1, 2}; cc.sub_mat = {M(n2), M(n0)};
        if (n2 < n0) { cc.sub = {{2, 4, 3}, {0, 1, 5, 6}}; cc.coh = {{3, 4, 5, 6}}; }
        else { cc.sub = {{2, 6, 5}, {0, 1, 3, 4}}; cc.coh = {{4, 3, 6, 5}}; }
      }
      cc.incl.assign(cc.cut_edge.size(), v[1]);
    } else {
      if (n1e2) {
        cc.cut_edge = {2, 0, 2, 0}; cc.incl = {n0, n0, n1, n1};
        cc.sub_mat = {M(n0), -1, M(n1)}; cc.sub = {{0, 8, 7}, {4, 6, 5, 3}, {1, 2, 9, 10}};
      } else if (n0e2) {
        cc.cut_edge = {0, 1, 0, 1}; cc.incl = {n1, n1, n2, n2};
        cc.sub_mat = {M(n1), -1, M(n2)}; cc.sub = {{1, 8, 7}, {4, 6, 5, 3}, {2, 0, 9, 10}};
      } else {
        cc.cut_edge = {1, 2, 1, 2}; cc.incl = {n2, n2, n0, n0};
        cc.sub_mat = {M(n2), -1, M(n0)}; cc.sub = {{2, 8, 7}, {4, 6, 5, 3}, {0, 1, 9, 10}};
      }
      cc.coh = {{4, 3, 8, 7}, {5, 6, 9, 10}};
    }
  } else {
    if (v[0] < 0) {
      if (n0 < 0) {
        cc.cut_edge = {1, 0, 2, 1}; cc.incl = {n1, n1, n2, n2};
        cc.sub_mat = {M(n1), -1, M(n2)}; cc.sub = {{1, 7, 8}, {0, 4, 3, 6, 5}, {2, 9, 10}};
      } else if (n1 < 0) {
        cc.cut_edge = {2, 1, 0, 2}; cc.incl = {n2, n2, n0, n0};
        cc.sub_mat = {M(n2), -1, M(n0)}; cc.sub = {{2, 7, 8}, {1, 4, 3, 6, 5}, {0, 9, 10}};
      } else {
        cc.cut_edge = {0, 2, 1, 0}; cc.incl = {n0, n0, n1, n1};
        cc.sub_mat = {M(n0), -1, M(n1)}; cc.sub = {{0, 7, 8}, {2, 4, 3, 6, 5}, {1, 9, 10}};
      }
      cc.coh = {{3, 4, 7, 8}, {5, 6, 9, 10}};
    } else {
      cc.cut_edge = {0, 2, 2, 1, 1, 0}; cc.incl = {n0, n0, n2, n2, n1, n1};
      cc.sub_mat = {M(n0), M(n2), M(n1), -1};
      cc.sub = {{0, 9, 10}, {2, 11, 12}, {1, 13, 14}, {8, 7, 6, 5, 4, 3}};
      cc.coh = {{3, 4, 9, 10}, {5, 6, 11, 12}, {7, 8, 13, 14}};
    }
  }
  return true;
}

// Quad4::detection (src/quad4.cpp:188-497, the cases written with polygonal integration
// elements): node detection values -> cut case (cohesive numbering: enrichment nodes 4.., their
// mirrors after).  Returns 0 uncut, 1 cut, 4 for the layouts the reference stops on (opposite
// nodes sharing a material: "interface highly curved").  Four inclusions on one element leave
// the cohesive list empty, as the reference's branch does.
int quad4_case(const int nd[4], CutCase& cc) {
  const int n0 = nd[0], n1 = nd[1], n2 = nd[2], n3 = nd[3];
  const bool n0e1 = n0 == n1, n0e2 = n0 == n2, n0e3 = n0 == n3, n1e2 = n1 == n2, n1e3 = n1 == n3, n2e3 = n2 == n3;
  std::vector<int> v = {n0, n1, n2, n3};
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  const int nu = (int)v.size();
  if (nu == 1) return 0;
  const int c0 = (int)std::count(nd, nd + 4, v[0]);   // nodes holding the smallest value
  using VV = std::vector<std::vector<int>>;
  auto set = [&](std::vector<int> ce, std::vector<int> inc, VV sub, std::vector<int> mat) {
    cc.cut_edge = ce; cc.incl = inc; cc.sub = sub; cc.sub_mat = mat;
  };
  const VV coh2 = {{4, 5, 8, 9}, {6, 7, 10, 11}};
  const VV coh3 = {{4, 5, 10, 11}, {6, 7, 12, 13}, {8, 9, 14, 15}};
  if (nu == 2) {
    if (v[0] < 0) {
      if (c0 == 1 || c0 == 3) {
        const VV cA = {{4, 5, 6, 7}}, cB = {{5, 4, 7, 6}};
        if (n1e2 && n1e3) {
          cc.cut_edge = {3, 0}; cc.sub_mat = {n0, n2};
          if (n0 < n1) { cc.sub = {{0, 5, 4}, {1, 2, 3, 6, 7}}; cc.coh = cA; } else { cc.sub = {{0, 7, 6}, {1, 2, 3, 4, 5}}; cc.coh = cB; }
        } else if (n0e2 && n0e3) {
          cc.cut_edge = {0, 1}; cc.sub_mat = {n1, n3};
          if (n1 < n0) { cc.sub = {{1, 5, 4}, {2, 3, 0, 6, 7}}; cc.coh = cA; } else { cc.sub = {{1, 7, 6}, {2, 3, 0, 4, 5}}; cc.coh = cB; }
        } else if (n0e1 && n0e3) {
          cc.cut_edge = {1, 2}; cc.sub_mat = {n2, n0};
          if (n2 < n0) { cc.sub = {{2, 5, 4}, {3, 0, 1, 6, 7}}; cc.coh = cA; } else { cc.sub = {{2, 7, 6}, {3, 0, 1, 4, 5}}; cc.coh = cB; }
        } else if (n0e1 && n1e2) {
          cc.cut_edge = {2, 3}; cc.sub_mat = {n3, n1};
          if (n3 < n0) { cc.sub = {{3, 5, 4}, {0, 1, 2, 6, 7}}; cc.coh = cA; } else { cc.sub = {{3, 7, 6}, {0, 1, 2, 4, 5}}; cc.coh = cB; }
        } else return 4;
      } else if (c0 == 2) {
        if (n0e1) {
          cc.cut_edge = {1, 3}; cc.sub_mat = {n0, n2};
          if (n0 < n2) { cc.sub = {{0, 1, 4, 5}, {2, 3, 7, 6}}; cc.coh = {{5, 4, 7, 6}}; }
          else { cc.sub = {{0, 1, 6, 7}, {2, 3, 5, 4}}; cc.coh = {{4, 5, 6, 7}}; }
        } else if (n1e2) {
          cc.cut_edge = {2, 0}; cc.sub_mat = {n0, n1};
          if (n0 < n1) { cc.sub = {{3, 0, 5, 4}, {1, 2, 6, 7}}; cc.coh = {{4, 5, 6, 7}}; }
          else { cc.sub = {{3, 0, 7, 6}, {1, 2, 4, 5}}; cc.coh = {{5, 4, 7, 6}}; }
        } else return 4;
      } else return 4;
      cc.incl.assign(cc.cut_edge.size(), v[1]);
    } else {
      if (c0 == 1 || c0 == 3) {
        if (n1e2 && n1e3) set({0, 3, 3, 0}, {n0, n0, n2, n2}, {{0, 8, 9}, {5, 4, 7, 6}, {1, 2, 3, 10, 11}}, {n0, -1, n2});
        else if (n0e2 && n0e3) set({1, 0, 0, 1}, {n1, n1, n3, n3}, {{1, 8, 9}, {5, 4, 7, 6}, {2, 3, 0, 10, 11}}, {n1, -1, n3});
        else if (n0e1 && n0e3) set({2, 1, 1, 2}, {n2, n2, n0, n0}, {{2, 8, 9}, {5, 4, 7, 6}, {3, 0, 1, 10, 11}}, {n2, -1, n0});
        else if (n0e1 && n1e2) set({3, 2, 2, 3}, {n3, n3, n1, n1}, {{3, 8, 9}, {5, 4, 7, 6}, {0, 1, 2, 10, 11}}, {n3, -1, n1});
        else return 4;
      } else if (c0 == 2) {
        if (n0e1) set({1, 3, 3, 1}, {n0, n0, n2, n2}, {{0, 1, 8, 9}, {5, 4, 7, 6}, {2, 3, 10, 11}}, {n0, -1, n2});
        else if (n1e2) set({2, 0, 0, 2}, {n1, n1, n3, n3}, {{1, 2, 8, 9}, {5, 4, 7, 6}, {3, 0, 10, 11}}, {n1, -1, n3});
        else return 4;
      } else return 4;
      cc.coh = coh2;
    }
  } else if (nu == 3) {
    if (v[0] < 0) {
      if (c0 == 2) {
        if (n0e1) set({3, 2, 2, 1}, {n3, n3, n2, n2}, {{3, 8, 9}, {2, 10, 11}, {0, 1, 7, 6, 5, 4}}, {n3, n2, -1});
        else if (n1e2) set({0, 3, 3, 2}, {n0, n0, n3, n3}, {{0, 8, 9}, {3, 10, 11}, {1, 2, 7, 6, 5, 4}}, {n0, n3, -1});
        else if (n2e3) set({1, 0, 0, 3}, {n1, n1, n0, n0}, {{1, 8, 9}, {0, 10, 11}, {2, 3, 7, 6, 5, 4}}, {n1, n0, -1});
        else if (n0e3) set({2, 1, 1, 0}, {n2, n2, n1, n1}, {{2, 8, 9}, {1, 10, 11}, {3, 0, 7, 6, 5, 4}}, {n2, n1, -1});
        else if (n0e2) set({1, 0, 3, 2}, {n1, n1, n3, n3}, {{1, 8, 9}, {3, 10, 11}, {2, 7, 6, 0, 5, 4}}, {n1, n3, -1});
        else if (n1e3) set({0, 3, 2, 1}, {n0, n0, n2, n2}, {{0, 8, 9}, {2, 10, 11}, {1, 7, 6, 3, 5, 4}}, {n0, n2, -1});
        else return 4;
      } else {
        if (n0e1 && n2 < 0) set({1, 3, 3, 2}, {n0, n0, n3, n3}, {{0, 1, 8, 9}, {3, 10, 11}, {2, 7, 6, 5, 4}}, {n0, n3, -1});
        else if (n0e1 && n3 < 0) set({1, 3, 2, 1}, {n0, n0, n2, n2}, {{0, 1, 8, 9}, {2, 10, 11}, {3, 5, 4, 7, 6}}, {n0, n2, -1});
        else if (n0e1) return 4;
        else if (n1e2 && n3 < 0) set({2, 0, 0, 3}, {n1, n1, n0, n0}, {{1, 2, 8, 9}, {0, 10, 11}, {3, 7, 6, 5, 4}}, {n1, n0, -1});
        else if (n1e2 && n0 < 0) set({2, 0, 3, 2}, {n1, n1, n3, n3}, {{1, 2, 8, 9}, {3, 10, 11}, {0, 5, 4, 7, 6}}, {n1, n3, -1});
        else if (n1e2) return 4;
        else if (n2e3 && n0 < 0) set({3, 1, 1, 0}, {n2, n2, n1, n1}, {{2, 3, 8, 9}, {1, 10, 11}, {0, 7, 6, 5, 4}}, {n2, n1, -1});
        else if (n2e3 && n1 < 0) set({3, 1, 0, 3}, {n2, n2, n0, n0}, {{2, 3, 8, 9}, {0, 10, 11}, {1, 5, 4, 7, 6}}, {n2, n0, -1});
        else if (n2e3) return 4;
        else if (n0e3 && n1 < 0) set({0, 2, 2, 1}, {n3, n3, n2, n2}, {{3, 0, 8, 9}, {2, 10, 11}, {1, 7, 6, 5, 4}}, {n3, n2, -1});
        else if (n0e3 && n2 < 0) set({0, 2, 1, 0}, {n3, n3, n1, n1}, {{3, 0, 8, 9}, {1, 10, 11}, {2, 5, 4, 7, 6}}, {n3, n1, -1});
        else return 4;
      }
      cc.coh = coh2;
    } else {
      if (n0e1) set({1, 3, 3, 2, 2, 1}, {n0, n0, n3, n3, n2, n2}, {{0, 1, 10, 11}, {3, 12, 13}, {2, 14, 15}, {9, 8, 7, 6, 5, 4}}, {n0, n3, n2, -1});
      else if (n1e2) set({2, 0, 0, 3, 3, 2}, {n1, n1, n0, n0, n3, n3}, {{1, 2, 10, 11}, {0, 12, 13}, {3, 14, 15}, {9, 8, 7, 6, 5, 4}}, {n1, n0, n3, -1});
      else if (n2e3) set({3, 1, 1, 0, 0, 3}, {n2, n2, n1, n1, n0, n0}, {{2, 3, 10, 11}, {1, 12, 13}, {0, 14, 15}, {9, 8, 7, 6, 5, 4}}, {n2, n1, n0, -1});
      else if (n0e3) set({0, 2, 2, 1, 1, 0}, {n3, n3, n2, n2, n1, n1}, {{3, 0, 10, 11}, {2, 12, 13}, {1, 14, 15}, {9, 8, 7, 6, 5, 4}}, {n3, n2, n1, -1});
      else return 4;
      cc.coh = coh3;
    }
  } else {
    if (v[0] < 0) {
      if (n0 < 0) set({3, 2, 2, 1, 1, 0}, {n3, n3, n2, n2, n1, n1}, {{3, 10, 11}, {2, 12, 13}, {1, 14, 15}, {0, 9, 8, 7, 6, 5, 4}}, {n3, n2, n1, -1});
      else if (n1 < 0) set({0, 3, 3, 2, 2, 1}, {n0, n0, n3, n3, n2, n2}, {{0, 10, 11}, {3, 12, 13}, {2, 14, 15}, {1, 9, 8, 7, 6, 5, 4}}, {n0, n3, n2, -1});
      else if (n2 < 0) set({1, 0, 0, 3, 3, 2}, {n1, n1, n0, n0, n3, n3}, {{1, 10, 11}, {0, 12, 13}, {3, 14, 15}, {2, 9, 8, 7, 6, 5, 4}}, {n1, n0, n3, -1});
      else set({2, 1, 1, 0, 0, 3}, {n2, n2, n1, n1, n0, n0}, {{2, 10, 11}, {1, 12, 13}, {0, 14, 15}, {3, 9, 8, 7, 6, 5, 4}}, {n2, n1, n0, -1});
      cc.coh = coh3;
    } else {
      set({3, 2, 2, 1, 1, 0, 0, 3}, {n3, n3, n2, n2, n1, n1, n0, n0},
          {{3, 12, 13}, {2, 14, 15}, {1, 16, 17}, {0, 18, 19}, {11, 10, 9, 8, 7, 6, 5, 4}}, {n3, n2, n1, n0, -1});
      cc.coh.clear();
    }
  }
  return 1;
}

// Tet4::partitionPrism (src/tet4.cpp:776-873): a prism (l[0..2] bottom, l[3..5] top) split into
// three tets.  g holds the global ids of the parent nodes among the prism's nodes and the local
// ids of its enrichment nodes; bottom_known selects the rule keyed on nodes 0-2, otherwise the one
// keyed on nodes 0 and 3 plus the smallest enrichment id (with the reference's comparison of
// g[3] < g[5] in the second test kept as written).
bool tet4_partition_prism(const std::vector<int>& l, const long long g[6], bool bottom_known,
                          std::vector<std::vector<int>>& out) {
  auto T = [&](int a, int b, int c, int d) { out.push_back({l[a], l[b], l[c], l[d]}); };
  if (bottom_known) {
    if (g[0] < g[1] && g[0] < g[2]) {
      if (g[1] < g[2]) { T(0, 1, 2, 5); T(0, 1, 5, 4); T(0, 4, 5, 3); }
      else { T(0, 1, 2, 4); T(0, 4, 2, 5); T(0, 4, 5, 3); }
    } else if (g[1] < g[0] && g[1] < g[2]) {
      if (g[0] < g[2]) { T(0, 1, 2, 5); T(0, 1, 5, 3); T(1, 5, 3, 4); }
      else { T(0, 1, 2, 3); T(1, 2, 3, 5); T(1, 5, 3, 4); }
    } else if (g[2] < g[0] && g[2] < g[1]) {
      if (g[0] < g[1]) { T(0, 1, 2, 4); T(0, 4, 2, 3); T(2, 3, 4, 5); }
      else { T(0, 1, 2, 3); T(1, 2, 3, 4); T(2, 3, 4, 5); }
    } else {
      return false;
    }
    return true;
  }
  int min_enrich = 0;
  if (g[1] < g[2] && g[1] < g[4] && g[1] < g[5]) min_enrich = 1;
  else if (g[2] < g[1] && g[2] < g[4] && g[3] < g[5]) min_enrich = 2;
  else if (g[4] < g[1] && g[4] < g[2] && g[4] < g[5]) min_enrich = 4;
  else if (g[5] < g[1] && g[5] < g[2] && g[5] < g[4]) min_enrich = 5;
  const bool a = (min_enrich == 1 || min_enrich == 5);
  if (g[0] < g[3]) {
    if (a) { T(0, 1, 2, 5); T(0, 1, 5, 4); T(0, 4, 5, 3); }
    else { T(0, 1, 2, 4); T(0, 4, 2, 5); T(0, 4, 5, 3); }
  } else if (g[3] < g[0]) {
    if (a) { T(0, 1, 2, 3); T(1, 2, 3, 5); T(1, 5, 3, 4); }
    else { T(0, 1, 2, 3); T(1, 2, 3, 4); T(2, 3, 4, 5); }
  } else {
    return false;
  }
  return true;
}

// Tet4::detection (src/tet4.cpp:228-675), the prism-based cases, followed by decomposePrisms
// (src/tet4.cpp:682-773): node detection values and the parent's global node ids -> cut case in
// the cohesive numbering (parent 0-3, enrichment 4.., mirrors after).  Returns 0 when uncut, 1
// when cut, or a status code with `err` set for the cases the reference cannot process: more than
// two distinct values (it exits), two different spheres (its branches are empty or exit), and
// separations its tables do not list (it exits).  The cohesive quad of a 2-2 split is not split
// into triangles: decomposePrisms tests the number of cohesive elements, not their node count.
int tet4_case(const int nd[4], const long long gid[4], CutCase& cc, std::string& err) {
  const int n0 = nd[0], n1 = nd[1], n2 = nd[2], n3 = nd[3];
  const bool n0e1 = n0 == n1, n0e2 = n0 == n2, n0e3 = n0 == n3, n1e2 = n1 == n2, n1e3 = n1 == n3, n2e3 = n2 == n3;
  std::vector<int> v = {n0, n1, n2, n3};
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  if (v.size() == 1) return 0;
  if (v.size() > 2) { err = "a tet4 element is cut by more than one interface (src/tet4.cpp:259-264)"; return 4; }
  if (v[0] >= 0) { err = "a tet4 element has nodes in two different inclusions (src/tet4.cpp:568-611)"; return 4; }
  const int cnt = (int)std::count(nd, nd + 4, v[0]);
  std::vector<std::vector<int>> sub;
  std::vector<int> sub_mat;
  if (cnt == 1 || cnt == 3) {
    // one node separated: a tet at that node and a prism, a CohTri3 between them
    int sep, oth;
    if (n1e2 && n1e3) { sep = 0; oth = 1; cc.cut_edge = {0, 3, 2}; }
    else if (n0e2 && n0e3) { sep = 1; oth = 0; cc.cut_edge = {0, 1, 4}; }
    else if (n0e1 && n0e3) { sep = 2; oth = 0; cc.cut_edge = {1, 2, 5}; }
    else if (n0e1 && n1e2) { sep = 3; oth = 1; cc.cut_edge = {3, 4, 5}; }
    else { err = "tet4 element with one node separated in an unlisted way (src/tet4.cpp:522-523)"; return 4; }
    static const int kBase[4][3] = {{1, 3, 2}, {0, 2, 3}, {1, 0, 3}, {0, 1, 2}};
    const int* b = kBase[sep];
    // the material of the prism: the reference indexes mats with n1 for nodes 0, 2, 3 separated
    // and with n0 for node 1 separated -- in every case a node on the prism side
    sub_mat = {nd[sep], nd[oth]};
    if (nd[sep] < nd[oth]) { sub = {{4, 5, 6, sep}, {b[0], b[1], b[2], 7, 8, 9}}; cc.coh = {{4, 6, 5, 7, 9, 8}}; }
    else { sub = {{7, 8, 9, sep}, {b[0], b[1], b[2], 4, 5, 6}}; cc.coh = {{4, 5, 6, 7, 8, 9}}; }
  } else {
    // two and two: an edge cut off, two prisms, a CohQuad4 between them
    int pa, pb;  // the materials come from nodes pa (first prism) and pb (second prism)
    bool lo;     // the reference's ordering test for choosing the '-' side
    if (n0e1 && n2e3 && !n0e2) { cc.cut_edge = {1, 2, 3, 4}; pa = 0; pb = 2; lo = n0 < n2;
      if (lo) sub = {{0, 5, 6, 1, 4, 7}, {2, 9, 8, 3, 10, 11}}; else sub = {{0, 9, 10, 1, 8, 11}, {2, 5, 4, 3, 6, 7}}; }
    else if (n1e2 && n0e3 && !n0e1) { cc.cut_edge = {2, 0, 4, 5}; pa = 1; pb = 0; lo = n1 < n3;
      if (lo) sub = {{1, 5, 6, 2, 4, 7}, {0, 9, 8, 3, 10, 11}}; else sub = {{1, 9, 10, 2, 8, 11}, {0, 5, 4, 3, 6, 7}}; }
    else if (n0e2 && n1e3 && !n0e1) { cc.cut_edge = {0, 1, 5, 3}; pa = 2; pb = 1; lo = n0 < n1;
      if (lo) sub = {{2, 5, 6, 0, 4, 7}, {1, 9, 8, 3, 10, 11}}; else sub = {{2, 9, 10, 0, 8, 11}, {1, 5, 4, 3, 6, 7}}; }
    else { err = "tet4 element with two nodes separated in an unlisted way (src/tet4.cpp:553-554)"; return 4; }
    sub_mat = {nd[pa], nd[pb]};
    cc.coh = lo ? std::vector<std::vector<int>>{{4, 5, 6, 7, 8, 9, 10, 11}}
                : std::vector<std::vector<int>>{{7, 6, 5, 4, 11, 10, 9, 8}};
  }
  cc.incl.assign(cc.cut_edge.size(), v[1]);
  // decomposePrisms: every prism becomes three tets with the prism's material
  cc.sub.clear();
  cc.sub_mat.clear();
  for (size_t i = 0; i < sub.size(); ++i) {
    if (sub[i].size() != 6) { cc.sub.push_back(sub[i]); cc.sub_mat.push_back(sub_mat[i]); continue; }
    long long g[6];
    int n_known = 0;
    for (int q = 0; q < 6; ++q) {
      const int l = sub[i][q];
      if (l < 4) { g[q] = gid[l]; ++n_known; }
      else g[q] = l;
    }
    std::vector<std::vector<int>> tets;
    if (!tet4_partition_prism(sub[i], g, n_known != 2, tets)) {
      err = "impossible prism decomposition (src/tet4.cpp:829, 868)";
      return 4;
    }
    for (auto& t : tets) { cc.sub.push_back(t); cc.sub_mat.push_back(sub_mat[i]); }
  }
  return 1;
}

const int kTriEdge[3][2] = {{0, 1}, {1, 2}, {2, 0}};
const int kQuadEdge[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
const int kTetEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};

}  // namespace

// The DOF nodes' adjacency (element, local node) in element order, their sorted distinct
// neighbours and the CSR pattern of the four blocks (Solver::preallocate_matrix with
// populate_local_neighbors, src/Solver.cpp:426-490, 772-896: every DOF pair of every element).
int build_pattern(Setup& s) {
  const int dim = s.dim;
  auto elem_n = [&](int e) {
    const int c = s.cut_of[e];
    return c < 0 ? s.npe : s.cut_node_off[c + 1] - s.cut_node_off[c];
  };
  auto elem_node = [&](int e, int a) {
    const int c = s.cut_of[e];
    return c < 0 ? s.conn[(size_t)e * s.npe + a] : s.cut_nodes[s.cut_node_off[c] + a];
  };
  // Adjacency of every DOF node in element order (element, local node) and its sorted distinct
  // neighbours.  Elements are split into contiguous chunks; each chunk counts its entries per DOF
  // node, the counts place every chunk's entries after the earlier chunks' (so each node's list
  // stays in element order), and the chunks fill their places in parallel.
  for (int e = 0; e < s.ne; ++e)
    if (elem_n(e) > 32) { s.error = "element with more than 32 nodes"; return 8; }
  const int nt = setup_threads();
  std::vector<std::vector<long long>> cadj(nt, std::vector<long long>(s.n_dn, 0)), cnb(nt, std::vector<long long>(s.n_dn, 0));
  chunked(s.ne, nt, [&](int k, int e0, int e1) {
    for (int e = e0; e < e1; ++e) {
      const int m = elem_n(e);
      for (int a = 0; a < m; ++a) {
        const int da = s.node_dn[elem_node(e, a)];
        cadj[k][da] += 1;
        cnb[k][da] += m;
      }
    }
  });
  std::vector<long long> adj_off(s.n_dn + 1, 0), nb_off(s.n_dn + 1, 0);
  for (int a = 0; a < s.n_dn; ++a) {
    long long ta = adj_off[a], tb = nb_off[a];
    for (int k = 0; k < nt; ++k) {
      const long long ca = cadj[k][a], cb = cnb[k][a];
      cadj[k][a] = ta; cnb[k][a] = tb;   // the chunk's first place for this node
      ta += ca; tb += cb;
    }
    adj_off[a + 1] = ta; nb_off[a + 1] = tb;
  }
  if (adj_off[s.n_dn] > 2147483647LL || nb_off[s.n_dn] > 2147483647LL) { s.error = "mesh too large"; return 2; }
  s.dn_adj.assign((size_t)adj_off[s.n_dn], 0);
  std::vector<int> nb_all((size_t)nb_off[s.n_dn]);
  chunked(s.ne, nt, [&](int k, int e0, int e1) {
    for (int e = e0; e < e1; ++e) {
      const int m = elem_n(e);
      for (int a = 0; a < m; ++a) {
        const int da = s.node_dn[elem_node(e, a)];
        s.dn_adj[(size_t)cadj[k][da]++] = e * 32 + a;
        long long& p = cnb[k][da];
        for (int b = 0; b < m; ++b) nb_all[(size_t)p++] = s.node_dn[elem_node(e, b)];
      }
    }
  });
  s.dn_adj_off.resize(s.n_dn + 1);
  for (int a = 0; a <= s.n_dn; ++a) s.dn_adj_off[a] = (int)adj_off[a];
  std::vector<int> nb_cnt(s.n_dn);
  chunked(s.n_dn, nt, [&](int, int a0, int a1) {
    for (int a = a0; a < a1; ++a) {
      int* b = nb_all.data() + nb_off[a];
      int* e = nb_all.data() + nb_off[a + 1];
      std::sort(b, e);
      nb_cnt[a] = (int)(std::unique(b, e) - b);
    }
  });
  s.dn_nbr_off.assign(s.n_dn + 1, 0);
  for (int a = 0; a < s.n_dn; ++a) s.dn_nbr_off[a + 1] = s.dn_nbr_off[a] + nb_cnt[a];
  s.dn_nbr.resize(s.dn_nbr_off[s.n_dn]);
  chunked(s.n_dn, nt, [&](int, int a0, int a1) {
    for (int a = a0; a < a1; ++a)
      std::copy(nb_all.begin() + nb_off[a], nb_all.begin() + nb_off[a] + nb_cnt[a], s.dn_nbr.begin() + s.dn_nbr_off[a]);
  });
  // CSR of the four blocks; rows in DOF order follow DOF-node order.
  s.nrows[0] = s.n_free; s.ncols[0] = s.n_free;
  s.nrows[1] = s.n_free; s.ncols[1] = s.n_const;
  s.nrows[2] = s.n_const; s.ncols[2] = s.n_free;
  s.nrows[3] = s.n_const; s.ncols[3] = s.n_const;
  for (int b = 0; b < 4; ++b) { s.rp[b].assign(s.nrows[b] + 1, 0); s.ci[b].clear(); }
  // row lengths (each DOF node writes only its own rows' entries)
  chunked(s.n_dn, nt, [&](int, int a0, int a1) {
  for (int a = a0; a < a1; ++a) {
    const int na = s.dn_node[a];
    int cf = 0, cp = 0;
    for (int k = s.dn_nbr_off[a]; k < s.dn_nbr_off[a + 1]; ++k) {
      const int nbn = s.dn_node[s.dn_nbr[k]];
      for (int q = 0; q < dim; ++q) { if (s.node_dof[(size_t)nbn * dim + q] < s.n_free) cf++; else cp++; }
    }
    for (int q = 0; q < dim; ++q) {
      const int g = s.node_dof[(size_t)na * dim + q];
      if (g < s.n_free) { s.rp[0][g + 1] = cf; s.rp[1][g + 1] = cp; }
      else { s.rp[2][g - s.n_free + 1] = cf; s.rp[3][g - s.n_free + 1] = cp; }
    }
  }
  });
  for (int b = 0; b < 4; ++b) for (int r = 0; r < s.nrows[b]; ++r) s.rp[b][r + 1] += s.rp[b][r];
  for (int b = 0; b < 4; ++b) s.ci[b].assign(s.rp[b][s.nrows[b]], -1);
  chunked(s.n_dn, nt, [&](int, int a0, int a1) {
  for (int a = a0; a < a1; ++a) {
    const int na = s.dn_node[a];
    for (int q = 0; q < dim; ++q) {
      const int g = s.node_dof[(size_t)na * dim + q];
      const bool rf = g < s.n_free;
      int pf = rf ? s.rp[0][g] : s.rp[2][g - s.n_free];
      int pp = rf ? s.rp[1][g] : s.rp[3][g - s.n_free];
      int* cif = rf ? s.ci[0].data() : s.ci[2].data();
      int* cip = rf ? s.ci[1].data() : s.ci[3].data();
      for (int k = s.dn_nbr_off[a]; k < s.dn_nbr_off[a + 1]; ++k) {
        const int nbn = s.dn_node[s.dn_nbr[k]];
        for (int q2 = 0; q2 < dim; ++q2) {
          const int g2 = s.node_dof[(size_t)nbn * dim + q2];
          if (g2 < s.n_free) cif[pf++] = g2; else cip[pp++] = g2 - s.n_free;
        }
      }
    }
  }
  });
  return 0;
}

int build_setup(const ProblemDesc& d, Setup& s, const PrepResult* pr) {
  s = Setup();
  if (pr && !pr->valid) pr = nullptr;
  s.desc = d;
  s.etype = d.elem_type;
  s.dim = (d.elem_type == TET4) ? 3 : 2;
  s.npe = (d.elem_type == TRI3) ? 3 : 4;
  s.cohesive = d.coh_law != COH_NONE;
  const int dim = s.dim;

  // ---------------- materials (material_lei.cpp:52-97); D is latched per material by dimension
  s.nvoigt = (dim == 2) ? 3 : 6;
  const double Es[2] = {d.E_matrix, d.E_fiber}, nus[2] = {d.nu_matrix, d.nu_fiber};
  for (int m = 0; m < 2; ++m) {
    double* D = s.D[m];
    for (int i = 0; i < 36; ++i) D[i] = 0.0;
    const double E = Es[m], nu = nus[m];
    if (dim == 2) {
      if (d.plane_strain) {
        double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
        D[0] = coef * (1.0 - nu); D[1] = coef * nu; D[3] = coef * nu; D[4] = coef * (1.0 - nu);
        D[8] = coef * (1.0 - 2.0 * nu) / 2.0;
      } else {
        double coef = E / (1.0 - nu * nu);
        D[0] = coef; D[1] = coef * nu; D[3] = coef * nu; D[4] = coef; D[8] = coef * (1.0 - nu) / 2.0;
      }
    } else {
      double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
      for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) D[i * 6 + j] = coef * (i == j ? (1.0 - nu) : nu);
      for (int i = 3; i < 6; ++i) D[i * 6 + i] = coef * (1.0 - 2.0 * nu) / 2;
    }
  }

  // ---------------- D sensitivities (src/material_lei.cpp:101-227): E, lambda, mu and K scale the
  // D pattern by coefficients of nu; nu has its own expressions
  for (int m = 0; m < 2; ++m) {
    const double E = Es[m], nu = nus[m];
    for (int p = 0; p < 5; ++p) for (int i = 0; i < 36; ++i) s.dD[m][p][i] = 0.0;
    double coefs[4];
    if (dim == 2 && !d.plane_strain) {
      coefs[0] = 1.0 / (1.0 - nu * nu); coefs[1] = (1.0 - 2.0 * nu) / (nu * (1.0 - nu));
      coefs[2] = 2.0 / (1.0 - nu); coefs[3] = 3.0 * (1.0 - 2.0 * nu) / (1.0 - nu * nu);
    } else {
      coefs[0] = 1.0 / ((1.0 + nu) * (1.0 - 2.0 * nu)); coefs[1] = 1.0 / nu;
      coefs[2] = 2.0 / (1.0 - 2.0 * nu); coefs[3] = 3.0 / (1.0 + nu);
    }
    for (int p = 0; p < 4; ++p) {
      double* Q = s.dD[m][p];
      const double c = coefs[p];
      if (dim == 2) {
        if (d.plane_strain) { Q[0] = c * (1.0 - nu); Q[1] = c * nu; Q[3] = c * nu; Q[4] = c * (1.0 - nu); Q[8] = c * (1.0 - 2.0 * nu) / 2.0; }
        else { Q[0] = c; Q[1] = c * nu; Q[3] = c * nu; Q[4] = c; Q[8] = c * (1.0 - nu) / 2.0; }
      } else {
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i * 6 + j] = (i == j) ? c * (1.0 - nu) : c * nu;
        for (int i = 3; i < 6; ++i) Q[i * 6 + i] = c * (1.0 - 2.0 * nu) / 2;
      }
    }
    double* Q = s.dD[m][4];
    if (dim == 2 && !d.plane_strain) {
      const double coef = E / (1.0 - nu * nu), dcoef = 2.0 * E * nu / std::pow(1.0 - nu * nu, 2);
      Q[0] = dcoef; Q[1] = dcoef * nu + coef; Q[3] = dcoef * nu + coef; Q[4] = dcoef;
      Q[8] = dcoef * (1.0 - nu) / 2.0 - 0.5 * coef;
    } else {
      const double coef = E / ((1.0 + nu) * (1.0 - 2.0 * nu));
      const double dcoef = E * (1.0 + 4.0 * nu) / std::pow(1.0 - nu - 2.0 * nu * nu, 2);
      if (dim == 2) {
        Q[0] = dcoef * (1.0 - nu) - coef; Q[1] = dcoef * nu + coef; Q[3] = dcoef * nu + coef; Q[4] = dcoef * (1.0 - nu) - coef;
        Q[8] = dcoef * (1.0 - 2.0 * nu) / 2.0 - coef;
      } else {
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i * 6 + j] = (i == j) ? dcoef * (1.0 - nu) - coef : dcoef * nu + coef;
        for (int i = 3; i < 6; ++i) Q[i * 6 + i] = dcoef * (1.0 - 2.0 * nu) / 2.0 - coef;
      }
    }
  }

  // ---------------- bounding plies: LinearElasticTransverselyIsotropicMaterial::computeLinearDmat
  // (src/material_leti.cpp:52-128): fibers along x, E3 = E2, G13 = G12, nu13 = nu12,
  // nu23 = E2 / (2 G23) - 1; the expressions and their order as the reference writes them
  // (the plane-stress branch included).
  {
    double* D = s.D[2];
    for (int i = 0; i < 36; ++i) D[i] = 0.0;
    if (d.ply_frac > 0.0) {
      const double E1 = d.ply[0], E2 = d.ply[1], G12 = d.ply[2], G23 = d.ply[3], nu12 = d.ply[4];
      if (!(E1 > 0 && E2 > 0 && G12 > 0 && G23 > 0) || d.ply_frac >= 0.5) {
        s.error = "bounding plies need E1, E2, G12, G23 > 0 and a fraction below 0.5";
        return 2;
      }
      const double E3 = E2, G13 = G12, nu13 = nu12, nu23 = E2 / (2.0 * G23) - 1.0;
      const double delta = 1.0 - 2.0 * (E3 / E1) * nu12 * nu13 * nu23 - (E3 / E1) * nu13 * nu13 - (E3 / E2) * nu23 * nu23 -
                           (E2 / E1) * nu12 * nu12;
      const double C11 = E1 * (1.0 - (E3 / E2) * nu23 * nu23) / delta;
      const double C22 = E2 * (1.0 - (E3 / E1) * nu13 * nu13) / delta;
      const double C33 = E3 * (1.0 - (E2 / E1) * nu12 * nu12) / delta;
      const double C12 = (E2 * nu12 + E3 * nu13 * nu23) / delta;
      const double C13 = E3 * (nu12 * nu23 + nu13) / delta;
      const double C23 = (E3 / E1) * (E1 * nu23 + E2 * nu12 * nu13) / delta;
      const double C44 = G23, C55 = G13, C66 = G12;
      if (dim == 2) {
        if (d.plane_strain) { D[0] = C11; D[1] = C12; D[3] = C12; D[4] = C22; D[8] = C66; }
        else { D[0] = C11 - C13 / C33; D[1] = C12 - C23 / C33; D[3] = C12 - C23 / C33; D[4] = C22 - C23 / C33; D[8] = C66; }
      } else {
        D[0] = C11; D[1] = C12; D[2] = C13;
        D[6] = C12; D[7] = C22; D[8] = C23;
        D[12] = C13; D[13] = C23; D[14] = C33;
        D[21] = C44; D[28] = C55; D[35] = C66;
      }
    }
  }

  // ---------------- cohesive law constants
  s.coh.law = d.coh_law;
  switch (d.coh_law) {
    // Mesh::add_material stores a copy made by each law's copy(); the bilinear copy passes ALPHA as
    // sqrt(alpha) (src/Material_BilinearCohesiveNU.cpp:37 with set_alpha storing its argument,
    // :493-499), so the mesh's bilinear laws use alpha = sqrt(50); the Xu-Needleman copy passes Q
    // as sqrt(q) (src/Material_XNCohesiveNU.cpp:35, set_q :384-390).
    case COH_BL: case COH_BLNU:
      s.coh.sigma_c = d.coh[0]; s.coh.delta_c1 = d.coh[1]; s.coh.delta_c2 = d.coh[2];
      s.coh.alpha = std::sqrt(50.0);
      s.coh.nvar = (d.coh_law == COH_BL) ? 1 : 0; break;
    case COH_XN: case COH_XNNU:
      s.coh.sigma_c = d.coh[0]; s.coh.delta_cn = d.coh[1]; s.coh.delta_ct = d.coh[2]; s.coh.q = std::sqrt(d.coh[3]);
      s.coh.nvar = (d.coh_law == COH_XN) ? 2 : 0; break;
    case COH_OP: case COH_OPNU: case COH_OPAUG: case COH_OPNUAUG:
      s.coh.sigma_c = d.coh[0]; s.coh.delta_c = d.coh[1]; s.coh.beta2 = d.coh[2] * d.coh[2];
      s.coh.nvar = (d.coh_law == COH_OP || d.coh_law == COH_OPAUG) ? 1 : 0; break;
    // The trilinear copies pass ALPHA as sqrt(alpha) too (src/Material_TrilinearCohesiveNU.cpp:40,
    // src/Material_SmoothedTrilinearCohesiveNU.cpp:40; set_alpha stores its argument), and the
    // setters stop the reference on parameters out of order (set_dc1 .. set_dc3, set_sc).
    case COH_TL: case COH_TLNU: case COH_STL: case COH_STLNU:
      s.coh.sigma_c = d.coh[0]; s.coh.delta_c1 = d.coh[1]; s.coh.delta_c2 = d.coh[2]; s.coh.delta_c3 = d.coh[3];
      if (!(d.coh[0] > 0 && d.coh[1] > 0 && d.coh[2] >= d.coh[1] && d.coh[3] >= d.coh[2])) {
        s.error = "trilinear cohesive law needs sigma_c > 0 and 0 < delta_c1 <= delta_c2 <= delta_c3";
        return 2;
      }
      s.coh.alpha = std::sqrt(50.0);
      s.coh.nvar = (d.coh_law == COH_TL || d.coh_law == COH_STL) ? 1 : 0; break;
    case COH_NONE: break;
    default: s.error = "unknown cohesive law"; return 2;
  }

  // ---------------- structured mesh (Mesh::generate_mesh)
  const int Nx = d.n[0], Ny = d.n[1], Nz = (dim == 3) ? d.n[2] : 0;
  if (Nx <= 0 || Ny <= 0 || (dim == 3 && Nz <= 0)) { s.error = "grid counts must be positive"; return 2; }
  for (int q = 0; q < dim; ++q)
    if (!(d.hi[q] > d.lo[q])) { s.error = "domain box must have hi > lo in every direction"; return 2; }
  if (d.incl.size() % (dim + 1) != 0) { s.error = "inclusion array has a partial record"; return 2; }
  for (size_t f = 0; f < d.incl.size() / (dim + 1); ++f) {
    const double r = d.incl[f * (dim + 1) + dim];
    if (!(r > 0.0) || !std::isfinite(r)) { s.error = "inclusion radius must be positive and finite"; return 2; }
  }
  const double hx = (d.hi[0] - d.lo[0]) / Nx, hy = (d.hi[1] - d.lo[1]) / Ny;
  const double hz = (dim == 3) ? (d.hi[2] - d.lo[2]) / Nz : 0.0;
  const long long nstd_ll = (long long)(Nx + 1) * (Ny + 1) * (Nz + 1);
  if (nstd_ll > 400000000LL) { s.error = "mesh too large"; return 2; }
  s.n_std = (int)nstd_ll;
  std::vector<double> X3((size_t)s.n_std * 3);  // 3-component copy used by the geometric tests
  for (int k = 0; k <= Nz; ++k)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i) {
        size_t id = (size_t)i + (size_t)j * (Nx + 1) + (size_t)k * (Nx + 1) * (Ny + 1);
        X3[id * 3 + 0] = d.lo[0] + i * hx;
        X3[id * 3 + 1] = d.lo[1] + j * hy;
        X3[id * 3 + 2] = (dim == 3 ? d.lo[2] : 0.0) + k * hz;
      }
  auto nid = [&](int i, int j, int k) { return i + j * (Nx + 1) + k * (Nx + 1) * (Ny + 1); };
  if (d.elem_type == TRI3) {
    s.ne = 2 * Nx * Ny;
    s.conn.resize((size_t)s.ne * 3);
    size_t e = 0;
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i) {
        int c[6];
        if ((i + j) % 2 == 0) {
          c[0] = nid(i, j, 0); c[1] = nid(i + 1, j, 0); c[2] = nid(i + 1, j + 1, 0);
          c[3] = nid(i, j, 0); c[4] = nid(i + 1, j + 1, 0); c[5] = nid(i, j + 1, 0);
        } else {
          c[0] = nid(i, j, 0); c[1] = nid(i + 1, j, 0); c[2] = nid(i, j + 1, 0);
          c[3] = nid(i + 1, j, 0); c[4] = nid(i + 1, j + 1, 0); c[5] = nid(i, j + 1, 0);
        }
        for (int t = 0; t < 6; ++t) s.conn[e * 3 + t] = c[t];
        e += 2;
      }
  } else if (d.elem_type == QUAD4) {
    s.ne = Nx * Ny;
    s.conn.resize((size_t)s.ne * 4);
    size_t e = 0;
    for (int j = 0; j < Ny; ++j)
      for (int i = 0; i < Nx; ++i, ++e) {
        s.conn[e * 4 + 0] = nid(i, j, 0); s.conn[e * 4 + 1] = nid(i + 1, j, 0);
        s.conn[e * 4 + 2] = nid(i + 1, j + 1, 0); s.conn[e * 4 + 3] = nid(i, j + 1, 0);
      }
  } else {
    s.ne = 6 * Nx * Ny * Nz;
    s.conn.resize((size_t)s.ne * 4);
    size_t e = 0;
    for (int k = 0; k < Nz; ++k)
      for (int j = 0; j < Ny; ++j)
        for (int i = 0; i < Nx; ++i) {
          const int n0 = nid(i, j, k), n1 = nid(i + 1, j, k), n2 = nid(i + 1, j + 1, k), n3 = nid(i, j + 1, k);
          const int n4 = nid(i, j, k + 1), n5 = nid(i + 1, j, k + 1), n6 = nid(i + 1, j + 1, k + 1), n7 = nid(i, j + 1, k + 1);
          const int tets[6][4] = {{n0, n2, n3, n6}, {n0, n3, n7, n6}, {n0, n7, n4, n6},
                                  {n0, n5, n6, n4}, {n1, n5, n6, n0}, {n1, n6, n2, n0}};
          for (int t = 0; t < 6; ++t, ++e)
            for (int q = 0; q < 4; ++q) s.conn[e * 4 + q] = tets[t][q];
        }
  }
  s.elem_mat.assign(s.ne, 0);
  s.cut_of.assign(s.ne, -1);

  // periodic DOF owners (Mesh::build_periodic_nodesets: the primary is the lowest id of a set)
  s.dnode.resize(s.n_std);
  for (int k = 0; k <= Nz; ++k)
    for (int j = 0; j <= Ny; ++j)
      for (int i = 0; i <= Nx; ++i) {
        int id = nid(i, j, k);
        s.dnode[id] = d.subscale ? nid(i % Nx, j % Ny, (dim == 3) ? (k % Nz) : 0) : id;
      }

  // ---------------- inclusions and node detection (Mesh::detect_node)
  std::vector<Inclusion> incs;
  const int stride = dim + 1;
  for (size_t i = 0; i + stride <= d.incl.size(); i += stride) {
    Inclusion in;
    in.dim = dim;
    in.c[0] = d.incl[i]; in.c[1] = d.incl[i + 1]; in.c[2] = (dim == 3) ? d.incl[i + 2] : 0.0;
    in.r = d.incl[i + dim];
    incs.push_back(in);
  }
  const int ninc = (int)incs.size();
  s.node_detect.assign(s.n_std, -1);
  if (pr) {
    // from the device pass; a node on a surface is reported with the inclusion the host loop
    // meets first for it
    if ((int)pr->node_detect.size() != s.n_std) { s.error = "internal: device detection size"; return 6; }
    s.node_detect = pr->node_detect;
    if (pr->surface_node >= 0) {
      const int n = pr->surface_node;
      int j = ninc - 1;
      for (; j >= 0; --j) if (incs[j].in_box(&X3[(size_t)n * 3]) && incs[j].detect(&X3[(size_t)n * 3]) != 0) break;
      std::ostringstream os;
      os << "node " << n << " lies on the surface of inclusion " << j << " (the reference stops here: src/Mesh.cpp:2904-2911)";
      s.error = os.str();
      return 3;
    }
  } else {
    // nodes in parallel chunks; the first node on a surface (in node order) is the one reported
    const int ntd = setup_threads();
    std::vector<std::pair<int, int>> on_surface(ntd, {-1, -1});
    chunked(s.n_std, ntd, [&](int k, int n0, int n1) {
      for (int n = n0; n < n1; ++n) {
        const double* x = &X3[(size_t)n * 3];
        int res = -1;
        for (int j = ninc - 1; j >= 0; --j) {
          if (!incs[j].in_box(x)) continue;
          int r = incs[j].detect(x);
          if (r == 0) continue;
          if (r == 1) { on_surface[k] = {n, j}; return; }
          res = j;
          break;
        }
        s.node_detect[n] = res;
      }
    });
    for (const auto& f : on_surface)
      if (f.first >= 0) {
        std::ostringstream os;
        os << "node " << f.first << " lies on the surface of inclusion " << f.second
           << " (the reference stops here: src/Mesh.cpp:2904-2911)";
        s.error = os.str();
        return 3;
      }
  }

  // ---------------- bounding plies (Tests/Main.cpp:262-289): an element whose nodes all lie at or
  // above top = hi_y - f (hi_y - lo_y), or all at or below bottom = lo_y + f (hi_y - lo_y), takes
  // the ply material.  This precedes detection, as in the reference (Mesh::detection reads the
  // element's material as the one of its matrix-side sub-elements, Mesh.cpp:2988, and gives an
  // element wholly inside an inclusion the inclusion's material, Mesh.cpp:2999-3005).
  if (d.ply_frac > 0.0) {
    const double span = d.hi[1] - d.lo[1];
    const double top = d.hi[1] - span * d.ply_frac, bottom = d.lo[1] + span * d.ply_frac;
    for (int e = 0; e < s.ne; ++e) {
      bool in_top = true, in_bottom = true;
      for (int q = 0; q < s.npe; ++q) {
        const double y = X3[(size_t)s.conn[(size_t)e * s.npe + q] * 3 + 1];
        if (y < top) in_top = false;
        if (y > bottom) in_bottom = false;
      }
      if (in_top || in_bottom) s.elem_mat[e] = 2;
    }
  }

  // ---------------- element detection (Tri3::detection / Tet4::detection)
  std::vector<CutCase> cases;
  std::vector<int> cut_elems;
  if (pr && (int)pr->elem_flag.size() != s.ne) { s.error = "internal: device element pass size"; return 6; }
  for (int e = 0; e < s.ne; ++e) {
    if (pr && pr->elem_flag[e] != 2) {   // the device's all-equal test
      if (pr->elem_flag[e] == 1) s.elem_mat[e] = 1;
      continue;
    }
    int nd[4];
    for (int q = 0; q < s.npe; ++q) nd[q] = s.node_detect[s.conn[(size_t)e * s.npe + q]];
    bool all_same = true;
    for (int q = 1; q < s.npe; ++q) all_same &= (nd[q] == nd[0]);
    if (all_same) {
      if (nd[0] != -1) s.elem_mat[e] = 1;  // entirely inside a fiber
      continue;
    }
    CutCase cc;
    bool cut = false;
    if (d.elem_type == TRI3) cut = tri3_case(nd, cc);
    else if (d.elem_type == TET4) {
      long long gid[4];
      for (int q = 0; q < 4; ++q) gid[q] = s.conn[(size_t)e * 4 + q];
      std::string why;
      const int rc = tet4_case(nd, gid, cc, why);
      if (rc > 1) {
        std::ostringstream os;
        os << "element " << e << ": " << why;
        s.error = os.str();
        return rc;
      }
      cut = rc == 1;
    } else if (d.elem_type == QUAD4) {
      const int rc = quad4_case(nd, cc);
      if (rc == 4) {
        std::ostringstream os;
        os << "element " << e << ": quad4 element cut in a manner the reference stops on (opposite nodes share a "
           << "material: interface highly curved, src/quad4.cpp:333-336)";
        s.error = os.str();
        return 4;
      }
      cut = rc == 1;
    } else { s.error = "element type has no cut-case table here"; return 4; }
    if (!cut) continue;
    s.cut_of[e] = (int)cut_elems.size();
    cut_elems.push_back(e);
    cases.push_back(cc);
  }
  s.ncut = (int)cut_elems.size();
  s.cut_elem = cut_elems;

  // ---------------- enrichment nodes (Mesh::add_enrichments, serial)
  const int (*emap)[2] = (d.elem_type == TRI3) ? kTriEdge : (d.elem_type == QUAD4 ? kQuadEdge : kTetEdge);
  std::set<std::tuple<int, int, int>> cut_edges;  // (min node, max node, inclusion), ordered as std::set<pair<vector,id>>
  const bool dev_edges = pr && pr->edges_valid;
  for (int c = 0; c < s.ncut && !dev_edges; ++c) {
    const int e = cut_elems[c];
    const CutCase& cc = cases[c];
    for (size_t i = 0; i < cc.cut_edge.size(); ++i) {
      int a = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i]][0]], b = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i]][1]];
      if (a > b) std::swap(a, b);
      cut_edges.insert(std::make_tuple(a, b, cc.incl[i]));
    }
  }
  const int n_init = dev_edges ? (int)pr->enr_incl.size() : (int)cut_edges.size();
  s.n_enr_initial = n_init;
  s.n_enr = s.cohesive ? 2 * n_init : n_init;
  std::map<std::tuple<int, int, int>, int> edge_index;
  std::vector<double> XE((size_t)s.n_enr * 3);
  s.enr_edge.resize((size_t)s.n_enr * 2);
  s.enr_incl.resize(s.n_enr);
  if (dev_edges) {
    // the device's enrichment nodes, already in the set's order, and their intersection points
    if (pr->no_sign_change >= 0) {
      const int k = pr->no_sign_change;
      std::ostringstream os;
      os << "no sign change of inclusion " << pr->enr_incl[k] << " on edge " << pr->enr_edge[2 * k] << "-"
         << pr->enr_edge[2 * k + 1] << " (src/Inclusion.cpp:38-39)";
      s.error = os.str();
      return 5;
    }
    for (int k = 0; k < n_init; ++k) {
      for (int q = 0; q < 3; ++q) XE[(size_t)k * 3 + q] = pr->XE[(size_t)k * 3 + q];
      s.enr_edge[(size_t)k * 2] = pr->enr_edge[2 * k]; s.enr_edge[(size_t)k * 2 + 1] = pr->enr_edge[2 * k + 1];
      s.enr_incl[k] = pr->enr_incl[k];
      edge_index[std::make_tuple(pr->enr_edge[2 * k], pr->enr_edge[2 * k + 1], pr->enr_incl[k])] = k;
    }
  } else {
    int k = 0;
    for (const auto& t : cut_edges) {
      const int a = std::get<0>(t), b = std::get<1>(t), inc = std::get<2>(t);
      const double* p0 = &X3[(size_t)a * 3];
      const double* p1 = &X3[(size_t)b * 3];
      double fa, fb, dfa;
      incs[inc].fdf(p0, p1, 0.0, &fa, &dfa);
      incs[inc].fdf(p0, p1, 1.0, &fb, &dfa);
      if (fa * fb >= 0) {
        std::ostringstream os;
        os << "no sign change of inclusion " << inc << " on edge " << a << "-" << b << " (src/Inclusion.cpp:38-39)";
        s.error = os.str();
        return 5;
      }
      EdgeFn fn{&incs[inc], p0, p1};
      double alpha = steffensen_then_brent(fn);
      for (int q = 0; q < 3; ++q) XE[(size_t)k * 3 + q] = p0[q] + alpha * (p1[q] - p0[q]);
      s.enr_edge[(size_t)k * 2] = a; s.enr_edge[(size_t)k * 2 + 1] = b; s.enr_incl[k] = inc;
      edge_index[t] = k;
      ++k;
    }
  }
  {
    if (s.cohesive)
      for (int m = 0; m < n_init; ++m) {
        for (int q = 0; q < 3; ++q) XE[(size_t)(m + n_init) * 3 + q] = XE[(size_t)m * 3 + q];
        s.enr_edge[(size_t)(m + n_init) * 2] = s.enr_edge[(size_t)m * 2];
        s.enr_edge[(size_t)(m + n_init) * 2 + 1] = s.enr_edge[(size_t)m * 2 + 1];
        s.enr_incl[m + n_init] = s.enr_incl[m];
      }
  }
  const int n_nodes = s.n_std + s.n_enr;
  s.X.resize((size_t)n_nodes * dim);
  for (int n = 0; n < s.n_std; ++n) for (int q = 0; q < dim; ++q) s.X[(size_t)n * dim + q] = X3[(size_t)n * 3 + q];
  for (int n = 0; n < s.n_enr; ++n) for (int q = 0; q < dim; ++q) s.X[(size_t)(s.n_std + n) * dim + q] = XE[(size_t)n * 3 + q];
  for (int n = 0; n < s.n_enr; ++n) s.dnode.push_back(s.n_std + n);
  auto X3of = [&](int node) -> const double* {
    return node < s.n_std ? &X3[(size_t)node * 3] : &XE[(size_t)(node - s.n_std) * 3];
  };

  // ---------------- per cut element: nodes, sub-elements, quadrature data
  // The cut elements are independent: contiguous chunks of them run in parallel, each appending
  // to its own accumulator with chunk-local offsets, and the chunks are then concatenated in
  // order (offsets shifted by the earlier chunks' sizes), which gives exactly the arrays of one
  // pass over the cut elements.
  struct CutAcc {
    std::vector<int> cut_nodes, cut_node_off, sub_type, sub_mat, sub_nodes, sub_node_off, qp_mat, qp_grad_off,
        sub_qp_off, cut_sub_off, cut_qp_off, coh_nh, coh_local_off, coh_local, cqp_isv, coh_qp_off, cut_coh_off;
    std::vector<double> qp_wgt, qp_grad, cqp_N, cqp_R, cqp_wgt;
    int n_isv = 0;
    std::string error;
    int rc = 0;
  };
  const int ntc = setup_threads();
  std::vector<CutAcc> accs(std::max(1, ntc));
  auto cut_chunk = [&](int k, int c0, int c1) {
    CutAcc& A = accs[k];
    for (int c = c0; c < c1; ++c) {
      const int e = cut_elems[c];
      CutCase cc = cases[c];
      const int ncut_e = (int)cc.cut_edge.size();
      const int n_en = s.cohesive ? 2 * ncut_e : ncut_e;
      // transformDetectionCohToReg: fold mirror indices back when the mesh is not cohesive
      if (!s.cohesive) {
        for (auto& sub : cc.sub)
          for (int& v : sub)
            if (v >= s.npe + ncut_e) v -= ncut_e;
        cc.coh.clear();
      }
      // enrichment node of each slot (add_enrich_node_to_elem)
      std::vector<int> slot(n_en, -1);
      for (int i = 0; i < ncut_e; ++i) {
        int a = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i]][0]], b = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i]][1]];
        if (a > b) std::swap(a, b);
        auto it = edge_index.find(std::make_tuple(a, b, cc.incl[i]));
        if (it == edge_index.end()) { A.error = "internal: cut edge without enrichment node"; A.rc = 6; return; }
        // first cut-edge entry with this (edge, inclusion) takes the node
        int first = i;
        for (int i2 = 0; i2 < i; ++i2) {
          int a2 = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i2]][0]], b2 = s.conn[(size_t)e * s.npe + emap[cc.cut_edge[i2]][1]];
          if (a2 > b2) std::swap(a2, b2);
          if (a2 == a && b2 == b && cc.incl[i2] == cc.incl[i]) { first = i2; break; }
        }
        if (first != i) { A.error = "internal: repeated (edge, inclusion) in one element"; A.rc = 6; return; }
        slot[i] = s.n_std + it->second;
        if (s.cohesive) slot[i + ncut_e] = s.n_std + it->second + n_init;
      }
      // element node list: parent nodes then enrichment slots
      std::vector<int> enodes;
      for (int q = 0; q < s.npe; ++q) enodes.push_back(s.conn[(size_t)e * s.npe + q]);
      for (int q = 0; q < n_en; ++q) enodes.push_back(slot[q]);
      const int nall = (int)enodes.size();
      for (int v : enodes) A.cut_nodes.push_back(v);
      A.cut_node_off.push_back((int)A.cut_nodes.size());

      // parent gradients: constant for the affine tri3 / tet4 parents; for a quad4 parent at each
      // point, from the inverse map of the point's global coordinates (src/Mesh.cpp:1564-1580)
      const bool quad_parent = d.elem_type == QUAD4;
      double pxs[4 * 3], pdNdr[4 * 3], pdNdx[4 * 3], pN[4], pJ;
      for (int q = 0; q < s.npe; ++q) for (int k = 0; k < dim; ++k) pxs[q * dim + k] = X3of(enodes[q])[k];
      if (!quad_parent) {
        if (dim == 2) tri3_shape(0.0, 0.0, pN, pdNdr);
        else tet4_shape(0.0, 0.0, 0.0, pN, pdNdr);
        transform_gradients(dim, s.npe, pdNdr, pxs, pdNdx, &pJ);
      }

      for (size_t ie = 0; ie < cc.sub.size(); ++ie) {
        const std::vector<int>& sub = cc.sub[ie];
        const int nsn = (int)sub.size();
        int stype;
        if (dim == 2) stype = (nsn == 3) ? SUB_TRI3 : (nsn == 4 ? SUB_QUAD4 : SUB_POLYGON);
        else stype = (nsn == 4) ? SUB_TET4 : (nsn == 6 ? SUB_PRISM6 : SUB_HEX8);
        const int mat = (cc.sub_mat[ie] < 0) ? s.elem_mat[e] : 1;
        A.sub_type.push_back(stype);
        A.sub_mat.push_back(mat);
        std::vector<int> gsub(nsn);
        double sx[32 * 3];
        for (int q = 0; q < nsn; ++q) {
          gsub[q] = enodes[sub[q]];
          A.sub_nodes.push_back(gsub[q]);
          for (int k = 0; k < dim; ++k) sx[q * dim + k] = X3of(gsub[q])[k];
        }
        A.sub_node_off.push_back((int)A.sub_nodes.size());
        int nqp = 0;
        if (stype == SUB_TRI3) nqp = 4;
        else if (stype == SUB_QUAD4) nqp = 4;
        else if (stype == SUB_POLYGON) nqp = 4 * nsn;
        else if (stype == SUB_TET4) nqp = 5;
        else { A.error = "prism6 / hex8 sub-elements do not occur after the prism decomposition"; A.rc = 6; return; }
        for (int qp = 0; qp < nqp; ++qp) {
          double r, t, w, cN[32], cdN[96], cdNdx[96], cJ;
          if (stype == SUB_TRI3) { r = kTri4[qp][0]; t = kTri4[qp][1]; w = kTri4[qp][2]; tri3_shape(r, t, cN, cdN); }
          else if (stype == SUB_QUAD4) { quad4_qp(qp, &r, &t, &w); quad4_shape(r, t, cN, cdN); }
          else if (stype == SUB_POLYGON) { poly_qp(nsn, qp, &r, &t, &w); poly_shape(nsn, r, t, cN, cdN); }
          else { w = kTet5[qp][3]; tet4_shape(kTet5[qp][0], kTet5[qp][1], kTet5[qp][2], cN, cdN); }
          transform_gradients(dim, nsn, cdN, sx, cdNdx, &cJ);
          if (cJ < 0.0) { A.error = "negative sub-element Jacobian (src/Mesh.cpp:1561)"; A.rc = 7; return; }
          if (quad_parent) {
            double gx[2] = {0.0, 0.0}, rs[2];
            for (int q = 0; q < nsn; ++q) for (int k = 0; k < 2; ++k) gx[k] += sx[q * 2 + k] * cN[q];
            if (!quad4_inverse(pxs, gx, rs)) { A.error = "bad inverse map of a quad4 parent (src/Mesh.cpp:1572)"; A.rc = 7; return; }
            quad4_shape(rs[0], rs[1], pN, pdNdr);
            transform_gradients(2, 4, pdNdr, pxs, pdNdx, &pJ);
          }
          A.qp_wgt.push_back(cJ * w);
          A.qp_mat.push_back(mat);
          // gradients over the element's nodes: parent gradients, then the child gradient of the
          // sub-element node that is each enrichment node (zero when the sub-element lacks it)
          for (int q = 0; q < s.npe; ++q) for (int k = 0; k < dim; ++k) A.qp_grad.push_back(pdNdx[q * dim + k]);
          for (int en = 0; en < n_en; ++en) {
            const int id = enodes[s.npe + en];
            int found = -1;
            for (int q = 0; q < nsn; ++q) if (gsub[q] == id) { found = q; break; }
            for (int k = 0; k < dim; ++k) A.qp_grad.push_back(found >= 0 ? 1.0 * cdNdx[found * dim + k] : 0.0);
          }
          A.qp_grad_off.push_back((int)A.qp_grad.size());
        }
        A.sub_qp_off.push_back((int)A.qp_wgt.size());
      }
      A.cut_sub_off.push_back((int)A.sub_type.size());
      A.cut_qp_off.push_back((int)A.qp_wgt.size());

      // cohesive elements (CohEdge2, 2-point Gauss; rotation from the '-' side nodes)
      for (size_t ce = 0; ce < cc.coh.size(); ++ce) {
        const std::vector<int>& cl = cc.coh[ce];
        const int nh = (int)cl.size() / 2;
        A.coh_nh.push_back(nh);
        for (int v : cl) A.coh_local.push_back(v);
        A.coh_local_off.push_back((int)A.coh_local.size());
        if (dim == 3) {
          // CohTri3 (4-point tri rule, src/CohTri3.cpp:70-84) or CohQuad4 (2 x 2 Gauss, qp -> (qp % 2,
          // qp / 2), src/CohQuad4.cpp:55-70); rotation rows (dx/dr, dx/ds, their cross product)
          // normalised, from the '-' side nodes (CohesiveElem::compute_rotation_general).
          const int nq = 4;
          for (int qp = 0; qp < nq; ++qp) {
            double r, t, w, N[4], dN[8];
            if (nh == 3) { r = kTri4[qp][0]; t = kTri4[qp][1]; w = kTri4[qp][2]; tri3_shape(r, t, N, dN); }
            else if (nh == 4) { quad4_qp(qp, &r, &t, &w); quad4_shape(r, t, N, dN); }
            else { A.error = "internal: 3D cohesive element with an unexpected node count"; A.rc = 6; return; }
            double Jac[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
            for (int n = 0; n < nh; ++n) {
              const double* xn = X3of(enodes[cl[n]]);
              for (int a = 0; a < 2; ++a) for (int i = 0; i < 3; ++i) Jac[a][i] += dN[n * 2 + a] * xn[i];
            }
            double nrm[3];
            nrm[0] = Jac[0][1] * Jac[1][2] - Jac[0][2] * Jac[1][1];
            nrm[1] = -(Jac[0][0] * Jac[1][2] - Jac[0][2] * Jac[1][0]);
            nrm[2] = Jac[0][0] * Jac[1][1] - Jac[0][1] * Jac[1][0];
            double mag[2];
            for (int a = 0; a < 2; ++a) {
              double dd = 0.0;
              for (int i = 0; i < 3; ++i) dd += Jac[a][i] * Jac[a][i];
              mag[a] = std::sqrt(dd);
            }
            double nn = 0.0;
            for (int i = 0; i < 3; ++i) nn += nrm[i] * nrm[i];
            const double dA = std::sqrt(nn);
            for (int n = 0; n < nh; ++n) A.cqp_N.push_back(N[n] * 1.0);
            for (int a = 0; a < 2; ++a) for (int i = 0; i < 3; ++i) A.cqp_R.push_back(Jac[a][i] / mag[a]);
            for (int i = 0; i < 3; ++i) A.cqp_R.push_back(nrm[i] / dA);
            A.cqp_wgt.push_back(dA * w);
            A.cqp_isv.push_back(A.n_isv);
            A.n_isv += s.coh.nvar;
          }
          A.coh_qp_off.push_back((int)A.cqp_wgt.size());
          continue;
        }
        for (int qp = 0; qp < 2; ++qp) {
          const double xi = (qp == 0) ? -kGauss2 : kGauss2;
          const double w = 1.0;
          const double N0 = 0.5 * (1.0 - xi), N1 = 0.5 * (1 + xi);
          const double* x0 = X3of(enodes[cl[0]]);
          const double* x1 = X3of(enodes[cl[1]]);
          double Jac[2] = {0.0, 0.0};
          for (int i = 0; i < 2; ++i) { Jac[i] += -0.5 * x0[i]; Jac[i] += 0.5 * x1[i]; }
          const double nrm[2] = {-Jac[1], Jac[0]};
          const double mag = std::sqrt(Jac[0] * Jac[0] + Jac[1] * Jac[1]);
          const double dA = std::sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1]);
          A.cqp_N.push_back(N0 * 1.0);
          A.cqp_N.push_back(N1 * 1.0);
          A.cqp_R.push_back(Jac[0] / mag); A.cqp_R.push_back(Jac[1] / mag);
          A.cqp_R.push_back(nrm[0] / dA);  A.cqp_R.push_back(nrm[1] / dA);
          A.cqp_wgt.push_back(dA * w);
          A.cqp_isv.push_back(A.n_isv);
          A.n_isv += s.coh.nvar;
        }
        A.coh_qp_off.push_back((int)A.cqp_wgt.size());
      }
      A.cut_coh_off.push_back((int)A.coh_nh.size());
    }
  };
  chunked(s.ncut, ntc, cut_chunk);
  for (const CutAcc& A : accs)
    if (A.rc) { s.error = A.error; return A.rc; }
  // Concatenation: every chunk's slice of each array starts after the earlier chunks' slices;
  // offset arrays (one entry per item after a leading 0) are shifted by the earlier chunks' sizes
  // of the array they index.  The chunks copy their slices in parallel.
  struct Slice { size_t cut_nodes, sub_type, sub_nodes, qp_wgt, qp_grad, coh_nh, coh_local, cqp_wgt, cqp_N, cqp_R;
                 size_t ncut, nsub, nqp, ncoh; int isv; };
  std::vector<Slice> at(accs.size() + 1, Slice{0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0});
  for (size_t k = 0; k < accs.size(); ++k) {
    const CutAcc& A = accs[k];
    Slice n = at[k];
    n.cut_nodes += A.cut_nodes.size(); n.sub_type += A.sub_type.size(); n.sub_nodes += A.sub_nodes.size();
    n.qp_wgt += A.qp_wgt.size(); n.qp_grad += A.qp_grad.size(); n.coh_nh += A.coh_nh.size();
    n.coh_local += A.coh_local.size(); n.cqp_wgt += A.cqp_wgt.size(); n.cqp_N += A.cqp_N.size(); n.cqp_R += A.cqp_R.size();
    n.ncut += A.cut_node_off.size(); n.nsub += A.sub_node_off.size(); n.nqp += A.qp_grad_off.size(); n.ncoh += A.coh_qp_off.size();
    n.isv += A.n_isv;
    at[k + 1] = n;
  }
  const Slice& T = at[accs.size()];
  if (T.qp_grad > 2147483647ULL || T.cqp_R > 2147483647ULL) { s.error = "cut-element tables beyond 2^31 entries"; return 2; }
  s.cut_nodes.resize(T.cut_nodes); s.sub_type.resize(T.sub_type); s.sub_mat.resize(T.sub_type);
  s.sub_nodes.resize(T.sub_nodes); s.qp_wgt.resize(T.qp_wgt); s.qp_mat.resize(T.qp_wgt); s.qp_grad.resize(T.qp_grad);
  s.coh_nh.resize(T.coh_nh); s.coh_local.resize(T.coh_local); s.cqp_wgt.resize(T.cqp_wgt); s.cqp_isv.resize(T.cqp_wgt);
  s.cqp_N.resize(T.cqp_N); s.cqp_R.resize(T.cqp_R);
  s.cut_node_off.assign(T.ncut + 1, 0); s.cut_sub_off.assign(T.ncut + 1, 0); s.cut_qp_off.assign(T.ncut + 1, 0);
  s.cut_coh_off.assign(T.ncut + 1, 0);
  s.sub_node_off.assign(T.nsub + 1, 0); s.sub_qp_off.assign(T.nsub + 1, 0);
  s.qp_grad_off.assign(T.nqp + 1, 0);
  s.coh_local_off.assign(T.ncoh + 1, 0); s.coh_qp_off.assign(T.ncoh + 1, 0);
  const int isv0 = s.n_isv;
  chunked((int)accs.size(), (int)accs.size(), [&](int, int k0, int k1) {
    for (int k = k0; k < k1; ++k) {
      const CutAcc& A = accs[k];
      const Slice& o = at[k];
      auto put = [](std::vector<int>& dst, size_t pos, const std::vector<int>& src, long long base) {
        for (size_t i = 0; i < src.size(); ++i) dst[pos + i] = (int)(base + src[i]);
      };
      put(s.cut_node_off, 1 + o.ncut, A.cut_node_off, (long long)o.cut_nodes);
      put(s.cut_sub_off, 1 + o.ncut, A.cut_sub_off, (long long)o.sub_type);
      put(s.cut_qp_off, 1 + o.ncut, A.cut_qp_off, (long long)o.qp_wgt);
      put(s.cut_coh_off, 1 + o.ncut, A.cut_coh_off, (long long)o.coh_nh);
      put(s.sub_node_off, 1 + o.nsub, A.sub_node_off, (long long)o.sub_nodes);
      put(s.sub_qp_off, 1 + o.nsub, A.sub_qp_off, (long long)o.qp_wgt);
      put(s.qp_grad_off, 1 + o.nqp, A.qp_grad_off, (long long)o.qp_grad);
      put(s.coh_local_off, 1 + o.ncoh, A.coh_local_off, (long long)o.coh_local);
      put(s.coh_qp_off, 1 + o.ncoh, A.coh_qp_off, (long long)o.cqp_wgt);
      put(s.cqp_isv, o.cqp_wgt, A.cqp_isv, (long long)isv0 + o.isv);
      std::copy(A.cut_nodes.begin(), A.cut_nodes.end(), s.cut_nodes.begin() + o.cut_nodes);
      std::copy(A.sub_type.begin(), A.sub_type.end(), s.sub_type.begin() + o.sub_type);
      std::copy(A.sub_mat.begin(), A.sub_mat.end(), s.sub_mat.begin() + o.sub_type);
      std::copy(A.sub_nodes.begin(), A.sub_nodes.end(), s.sub_nodes.begin() + o.sub_nodes);
      std::copy(A.qp_wgt.begin(), A.qp_wgt.end(), s.qp_wgt.begin() + o.qp_wgt);
      std::copy(A.qp_mat.begin(), A.qp_mat.end(), s.qp_mat.begin() + o.qp_wgt);
      std::copy(A.qp_grad.begin(), A.qp_grad.end(), s.qp_grad.begin() + o.qp_grad);
      std::copy(A.coh_nh.begin(), A.coh_nh.end(), s.coh_nh.begin() + o.coh_nh);
      std::copy(A.coh_local.begin(), A.coh_local.end(), s.coh_local.begin() + o.coh_local);
      std::copy(A.cqp_wgt.begin(), A.cqp_wgt.end(), s.cqp_wgt.begin() + o.cqp_wgt);
      std::copy(A.cqp_N.begin(), A.cqp_N.end(), s.cqp_N.begin() + o.cqp_N);
      std::copy(A.cqp_R.begin(), A.cqp_R.end(), s.cqp_R.begin() + o.cqp_R);
    }
  });
  s.n_isv += T.isv;

  // ---------------- DOF numbering (DofObject::set_local_owned_normal_dofs / _enrich_dofs)
  // Dirichlet conditions as Tests/Main.cpp:549-581 applies them.
  if (pr) {
    // the standard nodes' numbers from the device pass (free index, or -1 - constrained index);
    // enrichment DOFs follow the standard free ones, constrained DOFs come after all free ones
    if (pr->std_dof.size() != (size_t)s.n_std * dim) { s.error = "internal: device DOF numbering size"; return 6; }
    int nfree_std = 0, nconst_ = 0;
    for (size_t i = 0; i < pr->std_dof.size(); ++i) {
      const int v = pr->std_dof[i];
      if (v >= 0) nfree_std = std::max(nfree_std, v + 1);
      else nconst_ = std::max(nconst_, -v);
    }
    const int nfree = nfree_std + s.n_enr * dim;
    s.n_free = nfree; s.n_const = nconst_;
    s.node_dof.assign((size_t)n_nodes * dim, -1);
    for (size_t i = 0; i < pr->std_dof.size(); ++i) {
      const int v = pr->std_dof[i];
      s.node_dof[i] = v >= 0 ? v : nfree + (-1 - v);
    }
    for (int n = 0; n < s.n_enr; ++n)
      for (int q = 0; q < dim; ++q) s.node_dof[(size_t)(s.n_std + n) * dim + q] = nfree_std + n * dim + q;
    s.dirichlet.assign(nconst_, 0.0);
    if (!d.subscale) {
      const double app = (d.hi[0] - d.lo[0]) * d.app_strain;
      for (int k = 0; k <= Nz; ++k)
        for (int j = 0; j <= Ny; ++j) s.dirichlet[s.node_dof[(size_t)nid(Nx, j, k) * dim] - nfree] = app;
    }
  } else {
  std::vector<std::vector<std::pair<bool, double>>> bc(s.n_std, std::vector<std::pair<bool, double>>(dim, {false, 0.0}));
  if (d.subscale) {
    for (int q = 0; q < dim; ++q) bc[0][q] = {true, 0.0};
  } else {
    const double app = (d.hi[0] - d.lo[0]) * d.app_strain;
    for (int k = 0; k <= Nz; ++k)
      for (int j = 0; j <= Ny; ++j) {
        bc[nid(Nx, j, k)][0] = {true, app};
        bc[nid(0, j, k)][0] = {true, 0.0};
      }
    for (int q = 0; q < dim; ++q) bc[0][q] = {true, 0.0};
  }
  int nfree = 0, nconst_ = 0;
  for (int n = 0; n < s.n_std; ++n)
    if (s.dnode[n] == n) for (int q = 0; q < dim; ++q) { if (bc[n][q].first) nconst_++; else nfree++; }
  nfree += s.n_enr * dim;
  s.n_free = nfree; s.n_const = nconst_;
  s.node_dof.assign((size_t)n_nodes * dim, -1);
  s.dirichlet.assign(nconst_, 0.0);
  {
    int f = 0, p = 0;
    for (int n = 0; n < s.n_std; ++n) {
      if (s.dnode[n] != n) continue;
      for (int q = 0; q < dim; ++q) {
        if (bc[n][q].first) { s.node_dof[(size_t)n * dim + q] = nfree + p; s.dirichlet[p] = bc[n][q].second; ++p; }
        else s.node_dof[(size_t)n * dim + q] = f++;
      }
    }
    for (int n = 0; n < s.n_enr; ++n)
      for (int q = 0; q < dim; ++q) s.node_dof[(size_t)(s.n_std + n) * dim + q] = f++;
    for (int n = 0; n < s.n_std; ++n)
      if (s.dnode[n] != n)
        for (int q = 0; q < dim; ++q) s.node_dof[(size_t)n * dim + q] = s.node_dof[(size_t)s.dnode[n] * dim + q];
  }
  }

  // ---------------- DOF nodes, adjacency and the CSR pattern
  s.node_dn.assign(n_nodes, -1);
  for (int n = 0; n < n_nodes; ++n)
    if (s.dnode[n] == n) { s.node_dn[n] = s.n_dn++; s.dn_node.push_back(n); }
  for (int n = 0; n < n_nodes; ++n) s.node_dn[n] = s.node_dn[s.dnode[n]];
  if (pr && pr->pattern_on_device) return 0;   // the caller forms the adjacency and the pattern
  return build_pattern(s);

}

}  // namespace pg
