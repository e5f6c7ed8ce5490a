// Oracle (test infrastructure only): an FP64 CPU restatement of Forcesmith's
// objective-evaluation path.  Only tests/, the smoke check and bench.py's
// cpu_baseline leg load it, and only as the checker or the timed CPU
// baseline — never as part of the product path.
//
// Parity pinning: the reference cannot be built here (Eigen, Boost, oneTBB,
// ddx missing; GCC >= 14 required), so this restatement is pinned against the
// reference's own unit-test known answers (tests/test_oracle_pins.py, which
// re-expresses tests/unit/test_spline.cpp, test_neighbor_list.cpp,
// test_boundary_conditions.cpp, test_eam_force.cpp, test_stiweb_force.cpp,
// test_adp_force.cpp and test_param_jacobian.cpp of the reference).
//
// Every function cites the reference file:line it follows.  Floating-point
// operation order follows the reference's scalar expressions, compiled with
// -ffp-contract=off (ISO C++ mode, as the reference's CMAKE_CXX_EXTENSIONS
// OFF implies).
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

namespace orc {

using Vec3 = std::array<double, 3>;

inline Vec3 operator+(const Vec3 &a, const Vec3 &b) {
  return {a[0] + b[0], a[1] + b[1], a[2] + b[2]};
}
inline Vec3 operator-(const Vec3 &a, const Vec3 &b) {
  return {a[0] - b[0], a[1] - b[1], a[2] - b[2]};
}
inline Vec3 operator*(double s, const Vec3 &a) {
  return {s * a[0], s * a[1], s * a[2]};
}
inline double dot(const Vec3 &a, const Vec3 &b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
// Eigen squaredNorm of a 3-vector: ((x² + y²) + z²).
inline double sqnorm(const Vec3 &a) {
  return a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
}
inline double norm(const Vec3 &a) { return std::sqrt(sqnorm(a)); }

struct Mat3 {
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double operator()(int r, int c) const { return m[r][c]; }
  double &operator()(int r, int c) { return m[r][c]; }
};

inline Vec3 mul(const Mat3 &A, const Vec3 &v) {
  Vec3 o;
  for (int r = 0; r < 3; ++r)
    o[r] = A(r, 0) * v[0] + A(r, 1) * v[1] + A(r, 2) * v[2];
  return o;
}

// 3×3 determinant by the first-row cofactor expansion used by Eigen 3.4's
// fixed-size determinant (third-party; restated algorithm).
inline double det3(const Mat3 &m) {
  auto h = [&](int a, int b, int c) {
    return m(0, a) * (m(1, b) * m(2, c) - m(1, c) * m(2, b));
  };
  return h(0, 1, 2) - h(1, 0, 2) + h(2, 0, 1);
}

// 3×3 inverse by the adjugate, with det from the first cofactor column, as
// Eigen 3.4's compute_inverse<…,3> does (third-party; restated algorithm).
inline Mat3 inverse3(const Mat3 &m) {
  auto cof = [&](int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
    const int j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m(i1, j1) * m(i2, j2) - m(i1, j2) * m(i2, j1);
  };
  const double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
  const double det = c00 * m(0, 0) + c10 * m(1, 0) + c20 * m(2, 0);
  const double invdet = 1.0 / det;
  Mat3 r;
  r(0, 0) = c00 * invdet;
  r(0, 1) = c10 * invdet;
  r(0, 2) = c20 * invdet;
  r(1, 0) = cof(0, 1) * invdet;
  r(1, 1) = cof(1, 1) * invdet;
  r(1, 2) = cof(2, 1) * invdet;
  r(2, 0) = cof(0, 2) * invdet;
  r(2, 1) = cof(1, 2) * invdet;
  r(2, 2) = cof(2, 2) * invdet;
  return r;
}

// PeriodicBC (include/forcesmith/core/boundary_conditions.hpp:9-50).
struct PBC {
  Mat3 box, inv;
  double volume = 1.0;
  void set(const Mat3 &b) {
    box = b;
    const double det = det3(b);
    bool finite = std::isfinite(det);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        finite = finite && std::isfinite(b(r, c));
    if (finite && det != 0.0) {
      inv = inverse3(b);
    } else {
      inv = Mat3{};
      inv(0, 0) = inv(1, 1) = inv(2, 2) = 1.0;
    }
    volume = std::isfinite(det) ? std::abs(det) : 0.0;
  }
  // wrap = box·(f − floor f), f = inv·r  (boundary_conditions.hpp:11-17,38-40)
  Vec3 wrap(const Vec3 &r) const {
    Vec3 f = mul(inv, r);
    for (double &x : f) x = x - std::floor(x);
    return mul(box, f);
  }
  Vec3 col(int c) const { return {box(0, c), box(1, c), box(2, c)}; }
};

// ---------------------------------------------------------------------------
// Makima spline (src/potentials/spline.cpp, include/forcesmith/potentials/spline.hpp)
// ---------------------------------------------------------------------------

// upper_bound − 1, clamped to [0, n−2] (spline.cpp:18-30).
inline std::size_t locate_interval(const std::vector<double> &x, double r) {
  const std::size_t n = x.size();
  std::size_t i =
      static_cast<std::size_t>(std::upper_bound(x.begin(), x.end(), r) - x.begin());
  if (i > 0) --i;
  if (i > n - 2) i = n - 2;
  return i;
}

// One makima weight |u − v| + |u + v| / 2 (spline.cpp:58-59).
inline double mk_w(double u, double v) {
  return std::abs(u - v) + std::abs(u + v) / 2;
}

struct Spline {
  std::vector<double> x, y, s; // s empty when n < 4 (piecewise linear)
  std::vector<uint8_t> fixed;

  Spline() = default;
  Spline(std::vector<double> xs, std::vector<double> ys)
      : x(std::move(xs)), y(std::move(ys)), fixed(x.size(), 0) {
    recompute_slopes();
  }
  static Spline uniform(double rmin, double rmax, const double *yv, int n) {
    // potential_reader.cpp:178-182: x_k = rmin + k·h, h = (rmax−rmin)/(n−1)
    std::vector<double> xs(n);
    const double h = (rmax - rmin) / static_cast<double>(n - 1);
    for (int k = 0; k < n; ++k) xs[k] = rmin + static_cast<double>(k) * h;
    return Spline(std::move(xs), std::vector<double>(yv, yv + n));
  }
  std::size_t n() const { return x.size(); }
  double rmin() const { return x.front(); }
  double rmax() const { return x.back(); }

  // recompute_slopes_ (spline.cpp:43-103), same expressions and order.
  void recompute_slopes() {
    const std::size_t n = x.size();
    if (n < 4) {
      s.clear();
      return;
    }
    s.assign(n, 0.0);
    double m2 = (y[3] - y[2]) / (x[3] - x[2]);
    double m1 = (y[2] - y[1]) / (x[2] - x[1]);
    double m0 = (y[1] - y[0]) / (x[1] - x[0]);
    double mm1 = 2 * m0 - m1;
    double mm2 = 2 * mm1 - m0;
    double w1 = std::abs(m1 - m0) + std::abs(m1 + m0) / 2;
    double w2 = std::abs(mm1 - mm2) + std::abs(mm1 + mm2) / 2;
    s[0] = (w1 * mm1 + w2 * m0) / (w1 + w2);
    if (std::isnan(s[0])) s[0] = 0;
    w1 = std::abs(m2 - m1) + std::abs(m2 + m1) / 2;
    w2 = std::abs(m0 - mm1) + std::abs(m0 + mm1) / 2;
    s[1] = (w1 * m0 + w2 * m1) / (w1 + w2);
    if (std::isnan(s[1])) s[1] = 0;
    for (std::size_t i = 2; i < n - 2; ++i) {
      double mim2 = (y[i - 1] - y[i - 2]) / (x[i - 1] - x[i - 2]);
      double mim1 = (y[i] - y[i - 1]) / (x[i] - x[i - 1]);
      double mi = (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
      double mip1 = (y[i + 2] - y[i + 1]) / (x[i + 2] - x[i + 1]);
      w1 = std::abs(mip1 - mi) + std::abs(mip1 + mi) / 2;
      w2 = std::abs(mim1 - mim2) + std::abs(mim1 + mim2) / 2;
      s[i] = (w1 * mim1 + w2 * mi) / (w1 + w2);
      if (std::isnan(s[i])) s[i] = 0;
    }
    double mnm4 = (y[n - 3] - y[n - 4]) / (x[n - 3] - x[n - 4]);
    double mnm3 = (y[n - 2] - y[n - 3]) / (x[n - 2] - x[n - 3]);
    double mnm2 = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
    double mnm1 = 2 * mnm2 - mnm3;
    double mn = 2 * mnm1 - mnm2;
    w1 = std::abs(mnm1 - mnm2) + std::abs(mnm1 + mnm2) / 2;
    w2 = std::abs(mnm3 - mnm4) + std::abs(mnm3 + mnm4) / 2;
    s[n - 2] = (w1 * mnm3 + w2 * mnm2) / (w1 + w2);
    if (std::isnan(s[n - 2])) s[n - 2] = 0;
    w1 = std::abs(mn - mnm1) + std::abs(mn + mnm1) / 2;
    w2 = std::abs(mnm2 - mnm3) + std::abs(mnm2 + mnm3) / 2;
    s[n - 1] = (w1 * mnm2 + w2 * mnm1) / (w1 + w2);
    if (std::isnan(s[n - 1])) s[n - 1] = 0;
  }

  // Hermite value kExpr (spline.cpp:130-135), evaluated as written.
  double hermite_eval(std::size_t i, double r) const {
    const double x0 = x[i], dx = x[i + 1] - x[i];
    const double t = (r - x0) / dx;
    const double omt = 1.0 - t;
    return omt * omt * (y[i] * (1.0 + 2.0 * t) + s[i] * (r - x0)) +
           t * t * (y[i + 1] * (3.0 - 2.0 * t) + dx * s[i + 1] * (t - 1.0));
  }
  // d/dr of kExpr.
  double hermite_deriv(std::size_t i, double r) const {
    const double x0 = x[i], dx = x[i + 1] - x[i];
    const double t = (r - x0) / dx;
    const double omt = 1.0 - t;
    const double A = y[i] * (1.0 + 2.0 * t) + s[i] * (r - x0);
    const double B = y[i + 1] * (3.0 - 2.0 * t) + dx * s[i + 1] * (t - 1.0);
    return -2.0 * omt / dx * A + omt * omt * (2.0 * y[i] / dx + s[i]) +
           2.0 * t / dx * B + t * t * (-2.0 * y[i + 1] / dx + s[i + 1]);
  }

  // eval / deriv (spline.cpp:215-252).
  double eval(double r) const {
    const std::size_t n = x.size();
    if (r <= x.front()) {
      const double slope = (y[1] - y[0]) / (x[1] - x[0]);
      return y.front() + slope * (r - x.front());
    } else if (r >= x.back()) {
      const double slope = (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
      return y.back() + slope * (r - x.back());
    } else if (s.empty()) {
      const std::size_t i = locate_interval(x, r);
      const double t = (r - x[i]) / (x[i + 1] - x[i]);
      return y[i] + t * (y[i + 1] - y[i]);
    }
    return hermite_eval(locate_interval(x, r), r);
  }
  double deriv(double r) const {
    const std::size_t n = x.size();
    if (r <= x.front()) {
      return (y[1] - y[0]) / (x[1] - x[0]);
    } else if (r >= x.back()) {
      return (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]);
    } else if (s.empty()) {
      const std::size_t i = locate_interval(x, r);
      return (y[i + 1] - y[i]) / (x[i + 1] - x[i]);
    }
    return hermite_deriv(locate_interval(x, r), r);
  }
  // Second derivative of the same branch (0 on linear branches).
  double deriv2(double r) const {
    if (r <= x.front() || r >= x.back() || s.empty()) return 0.0;
    const std::size_t i = locate_interval(x, r);
    const double dx = x[i + 1] - x[i];
    const double t = (r - x[i]) / dx;
    return (-6.0 * (1.0 - 2.0 * t) / (dx * dx)) * y[i] +
           (6.0 * (1.0 - 2.0 * t) / (dx * dx)) * y[i + 1] +
           ((-4.0 + 6.0 * t) / dx) * s[i] + ((6.0 * t - 2.0) / dx) * s[i + 1];
  }
};

// The fit-time site cache (spline.cpp:281-324; spline.hpp:47-98,111-125):
// per distance, the interval and the Hermite value/derivative basis, so that
// v and dv are 4-term dot products with (y_i, y_{i+1}, s_i, s_{i+1}).
struct Site {
  uint8_t linear = 1;
  uint32_t i = 0;
  double off = 0, inv_dx = 0;
  double v0 = 0, v1 = 0, vs0 = 0, vs1 = 0;
  double d0 = 0, d1 = 0, ds0 = 0, ds1 = 0;
};

inline Site prepare_site(const Spline &sp, double r) {
  const std::size_t n = sp.n();
  Site st;
  if (r <= sp.x.front()) {
    st.linear = 1;
    st.i = 0;
  } else if (r >= sp.x.back()) {
    st.linear = 1;
    st.i = static_cast<uint32_t>(n - 2);
  } else if (sp.s.empty()) {
    st.linear = 1;
    st.i = static_cast<uint32_t>(locate_interval(sp.x, r));
  } else {
    st.linear = 0;
    st.i = static_cast<uint32_t>(locate_interval(sp.x, r));
  }
  const std::size_t i = st.i;
  const double dx = sp.x[i + 1] - sp.x[i];
  st.inv_dx = 1.0 / dx;
  st.off = r - sp.x[i];
  if (!st.linear) {
    // ∂kExpr/∂(y0,y1,s0,s1) and ∂²kExpr/∂r∂(y0,y1,s0,s1).
    const double t = (r - sp.x[i]) / dx;
    const double omt = 1.0 - t;
    st.v0 = omt * omt * (1.0 + 2.0 * t);
    st.v1 = t * t * (3.0 - 2.0 * t);
    st.vs0 = omt * omt * (r - sp.x[i]);
    st.vs1 = t * t * dx * (t - 1.0);
    st.d0 = -6.0 * t * omt / dx;
    st.d1 = 6.0 * t * omt / dx;
    st.ds0 = omt * (1.0 - 3.0 * t);
    st.ds1 = t * (3.0 * t - 2.0);
  }
  return st;
}

// eval_at / deriv_at (spline.hpp:47-81).
inline double eval_at(const Spline &sp, const Site &st) {
  const std::size_t i = st.i;
  if (st.linear) return sp.y[i] + st.off * st.inv_dx * (sp.y[i + 1] - sp.y[i]);
  return st.v0 * sp.y[i] + st.v1 * sp.y[i + 1] + st.vs0 * sp.s[i] +
         st.vs1 * sp.s[i + 1];
}
inline double deriv_at(const Spline &sp, const Site &st) {
  const std::size_t i = st.i;
  if (st.linear) return (sp.y[i + 1] - sp.y[i]) * st.inv_dx;
  return st.d0 * sp.y[i] + st.d1 * sp.y[i + 1] + st.ds0 * sp.s[i] +
         st.ds1 * sp.s[i + 1];
}

// ---------------------------------------------------------------------------
// Knot derivatives of the makima spline (no reference counterpart: the
// reference differentiates splines by central differences,
// forcesmith_functor.cpp:279-286).  ∂s_k/∂y follows the branch of every |·|
// (sign(0) = 0, the central-difference limit) and NaN→0 gives 0.
// ---------------------------------------------------------------------------

// Dense ∂s/∂y (n × n); fine for the ≤ 64-knot fitted tables.
inline std::vector<double> slope_jacobian(const Spline &sp) {
  const std::size_t n = sp.n();
  std::vector<double> J(n * n, 0.0);
  if (n < 4) return J;
  const auto &x = sp.x;
  const auto &y = sp.y;
  // secant q as (value, coefficient on y_q, coefficient on y_{q+1})
  auto sec = [&](std::size_t q) { return (y[q + 1] - y[q]) / (x[q + 1] - x[q]); };
  auto sgn = [](double v) { return v > 0 ? 1.0 : (v < 0 ? -1.0 : 0.0); };
  // A "p" is a linear combination of secants: value + gradient over y.
  struct P {
    double v = 0;
    std::vector<double> g;
  };
  auto P_sec = [&](std::size_t q) {
    P p;
    p.v = sec(q);
    p.g.assign(n, 0.0);
    const double ih = 1.0 / (x[q + 1] - x[q]);
    p.g[q] -= ih;
    p.g[q + 1] += ih;
    return p;
  };
  auto lin = [&](double a, const P &pa, double b, const P &pb) {
    P p;
    p.v = a * pa.v + b * pb.v;
    p.g.assign(n, 0.0);
    for (std::size_t k = 0; k < n; ++k) p.g[k] = a * pa.g[k] + b * pb.g[k];
    return p;
  };
  // s = (w1·p2 + w2·p3)/(w1 + w2), w1 = W(p4,p3), w2 = W(p2,p1)
  auto slope_row = [&](std::size_t k, const P &p1, const P &p2, const P &p3,
                       const P &p4) {
    const double w1 = mk_w(p4.v, p3.v), w2 = mk_w(p2.v, p1.v);
    const double W = w1 + w2;
    double *row = &J[k * n];
    const double s = (w1 * p2.v + w2 * p3.v) / W;
    if (std::isnan(s) || W == 0.0) return; // NaN → 0 branch: zero gradient
    const double ds_dw1 = (p2.v - s) / W, ds_dw2 = (p3.v - s) / W;
    const double ds_dp2 = w1 / W, ds_dp3 = w2 / W;
    const double dw1_dp4 = sgn(p4.v - p3.v) + 0.5 * sgn(p4.v + p3.v);
    const double dw1_dp3 = -sgn(p4.v - p3.v) + 0.5 * sgn(p4.v + p3.v);
    const double dw2_dp2 = sgn(p2.v - p1.v) + 0.5 * sgn(p2.v + p1.v);
    const double dw2_dp1 = -sgn(p2.v - p1.v) + 0.5 * sgn(p2.v + p1.v);
    const double c1 = ds_dw2 * dw2_dp1;
    const double c2 = ds_dp2 + ds_dw2 * dw2_dp2;
    const double c3 = ds_dp3 + ds_dw1 * dw1_dp3;
    const double c4 = ds_dw1 * dw1_dp4;
    for (std::size_t q = 0; q < n; ++q)
      row[q] = c1 * p1.g[q] + c2 * p2.g[q] + c3 * p3.g[q] + c4 * p4.g[q];
  };
  const P m0 = P_sec(0), m1 = P_sec(1), m2 = P_sec(2);
  const P mm1 = lin(2, m0, -1, m1);  // 2 m0 − m1
  const P mm2 = lin(2, mm1, -1, m0); // 2 mm1 − m0
  slope_row(0, mm2, mm1, m0, m1);
  slope_row(1, mm1, m0, m1, m2);
  for (std::size_t i = 2; i < n - 2; ++i)
    slope_row(i, P_sec(i - 2), P_sec(i - 1), P_sec(i), P_sec(i + 1));
  const P mnm4 = P_sec(n - 4), mnm3 = P_sec(n - 3), mnm2 = P_sec(n - 2);
  const P mnm1 = lin(2, mnm2, -1, mnm3);
  const P mn = lin(2, mnm1, -1, mnm2);
  slope_row(n - 2, mnm4, mnm3, mnm2, mnm1);
  slope_row(n - 1, mnm3, mnm2, mnm1, mn);
  return J;
}

// ∂v/∂y and ∂v'/∂y of the spline at r (dense, length n), following the same
// branch as eval / deriv.  dS = slope_jacobian(sp) (n × n, row k = ∂s_k/∂y).
inline void spline_param_grad(const Spline &sp, const std::vector<double> &dS,
                              double r, double *gv, double *gd, double *gdd = nullptr) {
  const std::size_t n = sp.n();
  std::fill(gv, gv + n, 0.0);
  std::fill(gd, gd + n, 0.0);
  if (gdd) std::fill(gdd, gdd + n, 0.0);
  const auto &x = sp.x;
  auto linear_seg = [&](std::size_t a, std::size_t b, double xa) {
    const double ih = 1.0 / (x[b] - x[a]);
    const double u = (r - xa) * ih;
    gv[a] += 1.0 - u;
    gv[b] += u;
    gd[a] -= ih;
    gd[b] += ih;
  };
  if (r <= x.front()) {
    // y0 + (y1−y0)/h·(r − x0)
    const double ih = 1.0 / (x[1] - x[0]);
    const double u = (r - x[0]) * ih;
    gv[0] += 1.0 - u;
    gv[1] += u;
    gd[0] -= ih;
    gd[1] += ih;
    return;
  }
  if (r >= x.back()) {
    const double ih = 1.0 / (x[n - 1] - x[n - 2]);
    const double u = (r - x[n - 1]) * ih;
    gv[n - 1] += 1.0 + u;
    gv[n - 2] -= u;
    gd[n - 1] += ih;
    gd[n - 2] -= ih;
    return;
  }
  const std::size_t i = locate_interval(x, r);
  if (sp.s.empty()) {
    linear_seg(i, i + 1, x[i]);
    return;
  }
  const Site st = prepare_site(sp, r);
  gv[i] += st.v0;
  gv[i + 1] += st.v1;
  gd[i] += st.d0;
  gd[i + 1] += st.d1;
  const double dx = x[i + 1] - x[i];
  const double t = (r - x[i]) / dx;
  const double e0 = -6.0 * (1.0 - 2.0 * t) / (dx * dx);
  const double e1 = 6.0 * (1.0 - 2.0 * t) / (dx * dx);
  const double es0 = (-4.0 + 6.0 * t) / dx, es1 = (6.0 * t - 2.0) / dx;
  if (gdd) {
    gdd[i] += e0;
    gdd[i + 1] += e1;
  }
  for (std::size_t q = 0; q < n; ++q) {
    const double a = dS[i * n + q], b = dS[(i + 1) * n + q];
    gv[q] += st.vs0 * a + st.vs1 * b;
    gd[q] += st.ds0 * a + st.ds1 * b;
    if (gdd) gdd[q] += es0 * a + es1 * b;
  }
}

// ---------------------------------------------------------------------------
// Analytic forms (include/forcesmith/potentials/analytic_potential.hpp:304-780)
// evaluated with forward-mode hyper-dual numbers: value, ∂/∂r, ∂²/∂r²,
// ∂/∂θ_k and ∂²/∂r∂θ_k are exact (the reference derives the same partials
// symbolically with ddx).
// ---------------------------------------------------------------------------

struct HD { // a + b ε1 + c ε2 + d ε1ε2, ε² = 0
  double a = 0, b = 0, c = 0, d = 0;
  HD() = default;
  HD(double v) : a(v) {}
  HD(double a_, double b_, double c_, double d_) : a(a_), b(b_), c(c_), d(d_) {}
};
inline HD operator+(HD x, HD y) { return {x.a + y.a, x.b + y.b, x.c + y.c, x.d + y.d}; }
inline HD operator-(HD x, HD y) { return {x.a - y.a, x.b - y.b, x.c - y.c, x.d - y.d}; }
inline HD operator-(HD x) { return {-x.a, -x.b, -x.c, -x.d}; }
inline HD operator*(HD x, HD y) {
  return {x.a * y.a, x.a * y.b + x.b * y.a, x.a * y.c + x.c * y.a,
          x.a * y.d + x.b * y.c + x.c * y.b + x.d * y.a};
}
// f(x) lifted: f(a) + f'(a)(bε1 + cε2 + dε1ε2) + f''(a) b c ε1ε2
inline HD lift(HD x, double f, double f1, double f2) {
  return {f, f1 * x.b, f1 * x.c, f1 * x.d + f2 * x.b * x.c};
}
inline HD recip(HD x) {
  const double i = 1.0 / x.a;
  return lift(x, i, -i * i, 2.0 * i * i * i);
}
inline HD operator/(HD x, HD y) { return x * recip(y); }
inline HD hexp(HD x) {
  const double e = std::exp(x.a);
  return lift(x, e, e, e);
}
inline HD hsqrt(HD x) {
  const double s = std::sqrt(x.a);
  return lift(x, s, 0.5 / s, -0.25 / (s * x.a));
}
inline HD hlog(HD x) { return lift(x, std::log(x.a), 1.0 / x.a, -1.0 / (x.a * x.a)); }
inline HD hcos(HD x) { return lift(x, std::cos(x.a), -std::sin(x.a), -std::cos(x.a)); }
// min / max: the selected operand, derivatives included (ties take x)
inline HD hmin(HD x, HD y) { return x.a <= y.a ? x : y; }
inline HD hmax(HD x, HD y) { return x.a >= y.a ? x : y; }
// x^p for a variable exponent: the value is std::pow, so a negative base with
// an integral exponent keeps its value; ln x enters only through the
// exponent's own derivative parts.
inline HD hpow(HD x, HD p) {
  const double v = std::pow(x.a, p.a);
  const double fx = p.a * std::pow(x.a, p.a - 1.0);
  const double fxx = p.a * (p.a - 1.0) * std::pow(x.a, p.a - 2.0);
  HD o{v, fx * x.b, fx * x.c, fx * x.d + fxx * x.b * x.c};
  if (p.b != 0.0 || p.c != 0.0 || p.d != 0.0) {
    const double L = std::log(x.a);
    const double fp = v * L, fpp = v * L * L, fxp = std::pow(x.a, p.a - 1.0) * (1.0 + p.a * L);
    o.b += fp * p.b;
    o.c += fp * p.c;
    o.d += fp * p.d + fxp * (x.b * p.c + p.b * x.c) + fpp * p.b * p.c;
  }
  return o;
}
inline HD hpowc(HD x, double p) {
  const double v = std::pow(x.a, p);
  return lift(x, v, p * std::pow(x.a, p - 1.0), p * (p - 1.0) * std::pow(x.a, p - 2.0));
}

// Parameters per form: ids 0-11 as restated first, then the rest of the
// reference's AnalyticForms list (analytic_potential.hpp:801-806).
inline int form_nparams(int form) {
  static const int np[] = {2, 3, 2, 2, 2, 3, 2, 3, 3, 1, 3, 5,            // 0-11
                           4, 6, 6, 7, 5, 7, 5, 6, 5, 6, 2,               // 12-22
                           11, 2, 16, 9, 12, 2, 5, 3, 4, 3, 7};           // 23-33
  return (form >= 0 && form < 34) ? np[form] : -1;
}

// cosine_cutoff (analytic_potential.hpp:142-145)
inline HD cos_cut(HD r, HD lo, HD hi) {
  const double pi = 3.14159265358979323846;
  return HD(0.5) + HD(0.5) * hcos(HD(pi) * (hmin(hmax(r, lo), hi) - lo) / (hi - lo));
}
// switching_factor (analytic_potential.hpp:147-151): u⁴/(1 + u⁴), u = min((r − r0)/h, 0)
inline HD sw_factor(HD r, HD r0, HD h) {
  const HD u = hmin((r - r0) / h, HD(0.0));
  const HD u4 = (u * u) * (u * u);
  return u4 / (HD(1.0) + u4);
}

// Every form's expression (analytic_potential.hpp:304-780), over hyper-duals.
// rmax is the table's upper gate bound (the `_sc` forms' switching point).
inline HD form_expr(int form, const HD *p, HD r, double rmax) {
  switch (form) {
  case 0: { // LennardJones 4ε(sr6² − sr6)
    HD sr6 = hpowc(p[1] / r, 6.0);
    return HD(4.0) * p[0] * (sr6 * sr6 - sr6);
  }
  case 1: { // Morse
    HD e = hexp(-p[1] * (r - p[2]));
    return p[0] * (HD(1.0) - e) * (HD(1.0) - e) - p[0];
  }
  case 2: return p[0] * hexp(-p[1] * r);                 // ExpDecay
  case 3: return p[0] * hsqrt(r / p[1]);                 // SqrtFunc
  case 4: return p[0] / hpow(r, p[1]);                   // PowerDecay
  case 5: return p[0] * hexp(-p[1] * (r - p[2]));        // MexpDecay
  case 6: return p[0] * (r - p[1]) * (r - p[1]);         // Harmonic
  case 7: return p[0] * hexp(-p[1] * r) + p[2];          // ExpPlus
  case 8: return p[0] * r * r + p[1] * r + p[2];         // Parabola
  case 9: return p[0] + HD(0.0) * r;                     // ConstFunc
  case 10: { // Buckingham
    HD x = (p[1] * p[1]) / (r * r);
    return p[0] * hexp(-r / p[1]) - p[2] * x * x * x;
  }
  case 11: { // Born
    HD r2 = r * r;
    HD r6 = r2 * r2 * r2;
    return p[0] * hexp((p[2] - r) / p[1]) - p[3] / r6 + p[4] / (r6 * r2);
  }
  case 12: // Universal {E0, a, b, c}
    return p[0] * (p[2] / (p[2] - p[1]) * hpow(r, p[1]) - p[1] / (p[2] - p[1]) * hpow(r, p[2])) + p[3] * r;
  case 13: // Eopp {A, n, B, m, k, phi}
    return p[0] / hpow(r, p[1]) + (p[2] / hpow(r, p[3])) * hcos(p[4] * r + p[5]);
  case 14: // EoppExp {A, B, C, m, k, phi}
    return p[0] * hexp(-p[1] * r) + (p[2] / hpow(r, p[3])) * hcos(p[4] * r + p[5]);
  case 15: // Meopp {A, n, B, m, k, phi, r0}
    return p[0] / hpow(r - p[6], p[1]) + (p[2] / hpow(r, p[3])) * hcos(p[4] * r + p[5]);
  case 16: { // GenLJ {A, n, m, r0, B}
    HD x = r / p[3];
    return p[0] / (p[2] - p[1]) * (p[2] * hpow(x, -p[1]) - p[1] * hpow(x, -p[2])) + p[4];
  }
  case 17: { // DoubleMorse {D1, a1, r1, D2, a2, r2, C}
    HD e1 = hexp(-p[1] * (r - p[2])), e2 = hexp(-p[4] * (r - p[5]));
    return p[0] * ((HD(1.0) - e1) * (HD(1.0) - e1) - HD(1.0)) +
           p[3] * ((HD(1.0) - e2) * (HD(1.0) - e2) - HD(1.0)) + p[6];
  }
  case 18: { // DoubleExp {A, B, r1, C, r2}
    HD dr = r - p[2];
    return p[0] * hexp(-p[1] * dr * dr) + hexp(-p[3] * (r - p[4]));
  }
  case 19: { // Mishin {A, B, C, r0, n, d}
    HD z = r - p[3];
    HD e = hexp(-p[5] * z);
    return p[0] * hpow(z, p[4]) * e * (HD(1.0) + p[1] * e) + p[2];
  }
  case 20: { // Poly5 {a0..a4}
    HD s1 = r - HD(1.0);
    HD s2 = s1 * s1;
    return p[0] + HD(0.5) * p[1] * s2 + p[2] * s1 * s2 + p[3] * s2 * s2 + p[4] * s2 * s2 * s1;
  }
  case 21: // StiwWeb2 {A, B, p, q, delta, rc}
    return (p[0] * hpow(r, -p[2]) - p[1] * hpow(r, -p[3])) * hexp(p[4] / (r - p[5]));
  case 22: // StiwWeb3 {gamma, a}
    return hexp(p[0] / (r - p[1]));
  case 23: // TersoffPot {A, B, lambda, mu, beta, n, c, d, h, R, S}
    return cos_cut(r, p[9], p[10]) * (p[0] * hexp(-p[2] * r) - p[1] * hexp(-p[3] * r));
  case 24: return p[0] * hexp(-p[1] * r);                // TersoffMix {chi, omega}
  case 25: { // TersoffModPot {A, B, lambda, mu, beta, n, c, d, h, R, S, c1..c5}
    HD r2 = r * r, r3 = r2 * r, r4 = r3 * r, r5 = r4 * r;
    return cos_cut(r, p[9], p[10]) * (p[0] * hexp(-p[2] * r) - p[1] * hexp(-p[3] * r)) *
           (HD(1.0) + p[11] * r + p[12] * r2 + p[13] * r3 + p[14] * r4 + p[15] * r5);
  }
  case 26: { // Kawamura {A..I}
    HD s1 = p[5] + p[6], t = p[3] + p[4];
    return p[0] * p[1] / r + p[2] * s1 * hexp((t - r) / s1) - p[7] * p[8] / hpowc(r, 6.0);
  }
  case 27: { // KawamuraMix {A..L}
    HD s1 = p[5] + p[6], t = p[3] + p[4], w = r - p[11];
    return p[0] * p[1] / r + p[2] * s1 * hexp((t - r) / s1) - p[7] * p[8] / hpowc(r, 6.0) +
           p[2] * p[9] * (hexp(HD(-2.0) * p[10] * w) - HD(2.0) * hexp(-p[10] * w));
  }
  case 28: return hpow(p[0] / r, p[1]);                  // Softshell {A, n}
  case 29: { // Strmm {A, B, C, D, E}
    HD s1 = r - p[4];
    return HD(2.0) * p[0] * hexp(-p[1] / HD(2.0) * s1) - p[2] * (HD(1.0) + p[3] * s1) * hexp(-p[3] * s1);
  }
  case 30: case 31: case 32: case 33: { // SmoothCutoff<LJ, Morse, ExpDecay, Eopp>: base × switch(r, rmax, h)
    static const int base_form[4] = {0, 1, 2, 13};
    const int b = base_form[form - 30];
    const int nb = form_nparams(b);
    return form_expr(b, p, r, rmax) * sw_factor(r, HD(rmax), p[nb]);
  }
  }
  return HD(0.0);
}

// StiwWeb2 / StiwWeb3 are exactly zero past their cut-off, or where the
// exponent would underflow (StiwWeb2::outside, analytic_potential.hpp:587-590).
// The partials there are zero as well: the reference's generic param_grad
// would differentiate the expression past rc (exp of a positive power).
inline bool form_outside(int form, const double *params, double r) {
  if (form == 21 || form == 22) {
    const int k = form == 21 ? 5 : 1;
    const double d = r - params[k];
    return d >= 0.0 || params[k - 1] / d < -708.0;
  }
  return false;
}

struct FormEval {
  double v = 0, d = 0, d2 = 0;
  double g[16] = {0}, dg[16] = {0}; // ∂v/∂θ_k, ∂²v/∂r∂θ_k
};

inline FormEval form_eval(int form, const double *params, int np, double r,
                          bool with_grad, double rmax = 0.0) {
  FormEval out;
  if (form_outside(form, params, r)) return out;
  HD p[16];
  for (int k = 0; k < np; ++k) p[k] = HD(params[k]);
  {
    HD rr(r, 1.0, 1.0, 0.0); // ε1 = ε2 = dr → d = ∂²/∂r²
    HD f = form_expr(form, p, rr, rmax);
    out.v = f.a;
    out.d = f.b;
    out.d2 = f.d;
  }
  if (with_grad) {
    for (int k = 0; k < np; ++k) {
      HD q[16];
      for (int m = 0; m < np; ++m) q[m] = HD(params[m]);
      q[k] = HD(params[k], 0.0, 1.0, 0.0); // ε2 = dθ_k
      HD rr(r, 1.0, 0.0, 0.0);             // ε1 = dr
      HD f = form_expr(form, q, rr, rmax);
      out.g[k] = f.c;
      out.dg[k] = f.d;
    }
  }
  return out;
}

} // namespace orc
