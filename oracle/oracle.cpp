// Oracle (test infrastructure only; see oracle_core.hpp for the header rules).
//
// A handle-based C ABI (`orc_*`) that mirrors the product's `fs_gpu_*` calls,
// so that every parity test drives both implementations with the same calls
// on the same inputs.  Parallelism: OpenMP over configurations, as the
// reference's std::execution::par over configs
// (src/optimization/forcesmith_functor.cpp:43).
#include "oracle_core.hpp"

#include "../include/forcesmith_gpu.h"

#include <omp.h>

#include <cstdio>
#include <memory>
#include <random>

namespace orc {

constexpr double kDummyWeight = 100.0; // force_calculator_concept.hpp:85
constexpr int kVoigt[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}}; // voigt.hpp:9-12

// pair_ordinal (include/forcesmith/force/potential_table.hpp:31-37)
inline int pair_ordinal(int a, int b, int nt) {
  if (a > b) std::swap(a, b);
  return a * nt - a * (a - 1) / 2 + (b - a);
}

// One radial table: a SplinePotential or an AnalyticForm
// (radial_potential.hpp:94-215 erases the same two).
struct Table {
  int kind = FS_TABLE_SPLINE, form = 0, n = 0;
  double rmin = 0, rmax = 0;
  std::vector<double> v;
  std::vector<uint8_t> fixed;
  std::vector<double> lo, hi;
  Spline sp;
  std::vector<double> dS; // ∂s/∂y for splines
  std::vector<int> free_idx;

  void init(const fs_table &t) {
    kind = t.kind;
    form = t.form;
    n = t.n;
    rmin = t.rmin;
    rmax = t.rmax;
    v.assign(t.values, t.values + n);
    fixed.assign(n, 0);
    lo.assign(n, -std::numeric_limits<double>::infinity());
    hi.assign(n, std::numeric_limits<double>::infinity());
    for (int k = 0; k < n; ++k) {
      if (t.fixed) fixed[k] = t.fixed[k] ? 1 : 0;
      // splines are NoBounds (spline.hpp:23); analytic params carry min/max
      if (kind != FS_TABLE_SPLINE) {
        if (t.lower) lo[k] = t.lower[k];
        if (t.upper) hi[k] = t.upper[k];
      }
    }
    free_idx.clear();
    for (int k = 0; k < n; ++k)
      if (!fixed[k]) free_idx.push_back(k);
    refresh();
  }
  void refresh() {
    if (kind == FS_TABLE_SPLINE) {
      sp = Spline::uniform(rmin, rmax, v.data(), n);
      dS = slope_jacobian(sp);
    }
  }
  int param_count() const { return static_cast<int>(free_idx.size()); }
  std::pair<double, double> span() const {
    if (kind == FS_TABLE_SPLINE) return {sp.x.front(), sp.x.back()};
    return {rmin, rmax};
  }
  bool in_range(double r) const { // closed gate (force_calculator_concept.hpp:94-98)
    auto [a, b] = span();
    return r >= a && r <= b;
  }
  double eval(double r) const {
    return kind == FS_TABLE_SPLINE ? sp.eval(r) : form_eval(form, v.data(), n, r, false, rmax).v;
  }
  double deriv(double r) const {
    return kind == FS_TABLE_SPLINE ? sp.deriv(r) : form_eval(form, v.data(), n, r, false, rmax).d;
  }
  double deriv2(double r) const {
    return kind == FS_TABLE_SPLINE ? sp.deriv2(r) : form_eval(form, v.data(), n, r, false, rmax).d2;
  }
  // ∂v/∂θ, ∂v'/∂θ (and ∂v''/∂θ for splines) over the FREE parameters.
  void grad(double r, double *gv, double *gd, double *gdd = nullptr) const {
    thread_local std::vector<double> bv, bd, bdd;
    bv.assign(n, 0.0);
    bd.assign(n, 0.0);
    bdd.assign(n, 0.0);
    if (kind == FS_TABLE_SPLINE) {
      spline_param_grad(sp, dS, r, bv.data(), bd.data(), gdd ? bdd.data() : nullptr);
    } else {
      FormEval f = form_eval(form, v.data(), n, r, true, rmax);
      for (int k = 0; k < n; ++k) {
        bv[k] = f.g[k];
        bd[k] = f.dg[k];
        bdd[k] = 0.0;
      }
    }
    for (std::size_t q = 0; q < free_idx.size(); ++q) {
      gv[q] = bv[free_idx[q]];
      gd[q] = bd[free_idx[q]];
      if (gdd) gdd[q] = bdd[free_idx[q]];
    }
  }
};

struct Config {
  int natoms = 0;
  int64_t atom0 = 0;
  PBC pbc;
  double ref_energy = 0;
  double ref_stress[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};

// Per-config calculator outputs (the Configuration's calc_* fields,
// include/forcesmith/core/atom.hpp:84-93).
struct Out {
  std::vector<Vec3> force;
  double energy = 0, limit = 0;
  double stress[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
};

struct State {
  std::vector<Config> cfgs;
  std::vector<Vec3> pos, ref_force;
  std::vector<int> type;
  int64_t natoms_total = 0;
  // neighbour CSR (global atom index → pairs); j is config-local
  std::vector<int64_t> nb_start;
  std::vector<int32_t> nb_j;
  std::vector<int8_t> nb_img;
  std::vector<Vec3> nb_d;
  double rcut_built = -1;
  // model
  bool have_model = false;
  int family = 0, ntypes = 1;
  std::vector<Table> tables;
  // global parameters (GlobalParam, force_calculator_concept.hpp:21-44):
  // values, fixed flags, links (global, table, slot)
  std::vector<double> gval;
  std::vector<uint8_t> gfixed;
  std::vector<std::array<int, 3>> links;
  // spline sites per pair per role (φ, g_j, g_i, u, w); −1 = not cached
  std::vector<Site> site[5];
  std::vector<uint8_t> site_ok[5];
  std::string err;
  int threads = 0;
};

inline int npair_of(int nt) { return nt * (nt + 1) / 2; }

int expected_tables(int family, int nt) {
  const int np = npair_of(nt);
  switch (family) {
  case FS_FAMILY_PAIR: return np;
  case FS_FAMILY_EAM: return np + 2 * nt;
  case FS_FAMILY_ADP: return 3 * np + 2 * nt;
  case FS_FAMILY_SW: return np + 1;
  case FS_FAMILY_TERSOFF: return np;
  case FS_FAMILY_ANGULAR: return 2 * np + nt;
  case FS_FAMILY_ACSF: return 1 + nt;
  case FS_FAMILY_LMBTR: return 1 + nt;
  }
  return -1;
}

double max_cutoff(const State &S) {
  // TableParams::max_cutoff (force_calculator_concept.hpp:210-221): max span
  // end over RADIAL tables (embedding is not radial).  SW: max(a1, a2)
  // (stiweb_force.cpp:234-239).
  double m = 0.0;
  const int nt = S.ntypes, np = npair_of(nt);
  if (S.family == FS_FAMILY_SW) {
    for (int p = 0; p < np; ++p)
      m = std::max(m, std::max(S.tables[p].v[5], S.tables[p].v[7]));
    return m;
  }
  if (S.family == FS_FAMILY_ACSF) return S.tables[0].v[0]; // descriptor_cutoff (acsf.hpp:73)
  if (S.family == FS_FAMILY_LMBTR) return S.tables[0].v[0]; // descriptor_cutoff (lmbtr.hpp:47)
  if (S.family == FS_FAMILY_TERSOFF) { // max S over pair slots (tersoff_force.cpp:259-265)
    for (int p = 0; p < np; ++p) m = std::max(m, S.tables[p].v[10]);
    return m;
  }
  for (int t = 0; t < static_cast<int>(S.tables.size()); ++t) {
    const bool embedding = (S.family == FS_FAMILY_EAM || S.family == FS_FAMILY_ADP) &&
                           t >= np + nt && t < np + 2 * nt;
    const bool angular = S.family == FS_FAMILY_ANGULAR && t >= 2 * np; // cos θ, not radial
    if (!embedding && !angular) m = std::max(m, S.tables[t].span().second);
  }
  return m;
}

// build_periodic (src/core/neighbor_list.cpp:59-92): full list, images
// ix∈[−sx,sx] with sx = ceil(rc·‖row_x(inv_box)‖), keep iff ‖d‖² ≤ rc²,
// skip only i==j in the home image; order i, j, (ix, iy, iz).
void build_neighbors(State &S, double rcut) {
  const int64_t N = S.natoms_total;
  std::vector<std::vector<int32_t>> jl(N);
  std::vector<std::vector<int8_t>> il(N);
  std::vector<std::vector<Vec3>> dl(N);
  const double rcut2 = rcut * rcut;
#pragma omp parallel for schedule(dynamic)
  for (int c = 0; c < static_cast<int>(S.cfgs.size()); ++c) {
    const Config &cf = S.cfgs[c];
    if (!(rcut > 0.0 && std::isfinite(rcut))) continue;
    const Vec3 a = cf.pbc.col(0), b = cf.pbc.col(1), cc = cf.pbc.col(2);
    auto shells = [&](int axis) {
      const Vec3 row = {cf.pbc.inv(axis, 0), cf.pbc.inv(axis, 1), cf.pbc.inv(axis, 2)};
      const double w = norm(row);
      if (!std::isfinite(w) || w <= 0.0) return 0;
      return static_cast<int>(std::ceil(rcut * w));
    };
    const int sx = shells(0), sy = shells(1), sz = shells(2);
    std::vector<Vec3> wpos(cf.natoms);
    for (int i = 0; i < cf.natoms; ++i) wpos[i] = cf.pbc.wrap(S.pos[cf.atom0 + i]);
    for (int i = 0; i < cf.natoms; ++i) {
      auto &J = jl[cf.atom0 + i];
      auto &I = il[cf.atom0 + i];
      auto &D = dl[cf.atom0 + i];
      for (int j = 0; j < cf.natoms; ++j) {
        const Vec3 base = wpos[j] - wpos[i];
        for (int ix = -sx; ix <= sx; ++ix)
          for (int iy = -sy; iy <= sy; ++iy)
            for (int iz = -sz; iz <= sz; ++iz) {
              if (i == j && ix == 0 && iy == 0 && iz == 0) continue;
              // base + ix·a + iy·b + iz·c, left to right
              Vec3 d;
              for (int k = 0; k < 3; ++k)
                d[k] = ((base[k] + static_cast<double>(ix) * a[k]) +
                        static_cast<double>(iy) * b[k]) +
                       static_cast<double>(iz) * cc[k];
              if (sqnorm(d) > rcut2) continue;
              J.push_back(j);
              I.push_back(static_cast<int8_t>(ix));
              I.push_back(static_cast<int8_t>(iy));
              I.push_back(static_cast<int8_t>(iz));
              D.push_back(d);
            }
      }
    }
  }
  S.nb_start.assign(N + 1, 0);
  for (int64_t i = 0; i < N; ++i) S.nb_start[i + 1] = S.nb_start[i] + jl[i].size();
  const int64_t P = S.nb_start[N];
  S.nb_j.resize(P);
  S.nb_img.resize(3 * P);
  S.nb_d.resize(P);
  for (int64_t i = 0; i < N; ++i) {
    std::copy(jl[i].begin(), jl[i].end(), S.nb_j.begin() + S.nb_start[i]);
    std::copy(il[i].begin(), il[i].end(), S.nb_img.begin() + 3 * S.nb_start[i]);
    std::copy(dl[i].begin(), dl[i].end(), S.nb_d.begin() + S.nb_start[i]);
  }
  S.rcut_built = rcut;
}

// Table accessors by role.
struct Roles {
  int np, nt;
  int pair(int ti, int tj) const { return pair_ordinal(ti, tj, nt); }
  int dens(int t) const { return np + t; }
  int emb(int t) const { return np + nt + t; }
  int dip(int ti, int tj) const { return np + 2 * nt + pair_ordinal(ti, tj, nt); }
  int quad(int ti, int tj) const { return 2 * np + 2 * nt + pair_ordinal(ti, tj, nt); }
};

// prepare(): prime the spline sites of every bond (eam_force.cpp:281-296,
// pair_force.cpp:62-74, adp_force.cpp:387-406).  Only in-range distances of
// spline tables are cached (kernels.hpp:14-17 prime_site).
void prime_sites(State &S) {
  const int64_t P = S.nb_j.size();
  for (auto &v : S.site) v.assign(P, Site{});
  for (auto &v : S.site_ok) v.assign(P, 0);
  if (S.family == FS_FAMILY_SW || S.family == FS_FAMILY_TERSOFF || S.family == FS_FAMILY_ANGULAR ||
      S.family == FS_FAMILY_ACSF || S.family == FS_FAMILY_LMBTR)
    return;
  const Roles R{npair_of(S.ntypes), S.ntypes};
#pragma omp parallel for schedule(dynamic)
  for (int c = 0; c < static_cast<int>(S.cfgs.size()); ++c) {
    const Config &cf = S.cfgs[c];
    for (int i = 0; i < cf.natoms; ++i) {
      const int64_t gi = cf.atom0 + i;
      const int ti = S.type[gi];
      for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
        const int tj = S.type[cf.atom0 + S.nb_j[p]];
        const double r = norm(S.nb_d[p]);
        int role_tab[5] = {R.pair(ti, tj), -1, -1, -1, -1};
        if (S.family == FS_FAMILY_EAM || S.family == FS_FAMILY_ADP) {
          role_tab[1] = R.dens(ti);
          role_tab[2] = R.dens(tj);
        }
        if (S.family == FS_FAMILY_ADP) {
          role_tab[3] = R.dip(ti, tj);
          role_tab[4] = R.quad(ti, tj);
        }
        for (int role = 0; role < 5; ++role) {
          const int t = role_tab[role];
          if (t < 0) continue;
          const Table &T = S.tables[t];
          if (T.kind == FS_TABLE_SPLINE && T.in_range(r)) {
            S.site[role][p] = prepare_site(T.sp, r);
            S.site_ok[role][p] = 1;
          }
        }
      }
    }
  }
}

enum { kPhi = 0, kGi = 1, kGj = 2, kDip = 3, kQuad = 4 };

inline double gated_eval(const State &S, int role, int64_t p, const Table &T, double r) {
  if (S.site_ok[role][p]) return eval_at(T.sp, S.site[role][p]);
  return T.in_range(r) ? T.eval(r) : 0.0;
}
inline double gated_deriv(const State &S, int role, int64_t p, const Table &T, double r) {
  if (S.site_ok[role][p]) return deriv_at(T.sp, S.site[role][p]);
  return T.in_range(r) ? T.deriv(r) : 0.0;
}

// clamp_embedding (include/forcesmith/force/kernels.hpp:19-31)
inline double clamp_rho(const Table &emb, double rho, double &limit) {
  auto [b, e] = emb.span();
  if (rho > e) {
    const double d = rho - e;
    limit += kDummyWeight * 10.0 * d * d;
    return e;
  } else if (rho < b) {
    const double d = b - rho;
    limit += kDummyWeight * 10.0 * d * d;
    return b;
  }
  return rho;
}

inline void acc_pair(Out &o, Vec3 &Fi, const Vec3 &d, const Vec3 &f, double e) {
  // accumulate_pair (kernels.hpp:33-38)
  Fi = Fi + f;
  o.energy += 0.5 * e;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) o.stress[a][b] -= (0.5 * d[a]) * f[b];
}

// EAMForceCalculator::eval_forces (src/force/eam_force.cpp:45-102)
void eval_eam(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const Roles R{npair_of(S.ntypes), S.ntypes};
  const int n = cf.natoms;
  std::vector<double> rho(n, 0.0), gradF(n, 0.0);
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const double r = norm(S.nb_d[p]);
      const int tj = S.type[cf.atom0 + S.nb_j[p]];
      rho[i] += gated_eval(S, kGj, p, S.tables[R.dens(tj)], r);
    }
  }
  for (int i = 0; i < n; ++i) {
    const Table &emb = S.tables[R.emb(S.type[cf.atom0 + i])];
    rho[i] = clamp_rho(emb, rho[i], o.limit);
    o.energy += emb.eval(rho[i]);
    gradF[i] = emb.deriv(rho[i]);
  }
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const int j = S.nb_j[p];
      const int tj = S.type[cf.atom0 + j];
      const double inv_r = 1.0 / r;
      const Table &phi_t = S.tables[R.pair(ti, tj)];
      const double phi = gated_eval(S, kPhi, p, phi_t, r);
      const double dphi = gated_deriv(S, kPhi, p, phi_t, r);
      const double drho_j = gated_deriv(S, kGj, p, S.tables[R.dens(tj)], r);
      const double drho_i = gated_deriv(S, kGi, p, S.tables[R.dens(ti)], r);
      const double fscale = (dphi + gradF[i] * drho_j + gradF[j] * drho_i) * inv_r;
      acc_pair(o, o.force[i], d, fscale * d, phi);
    }
  }
}

// PairForceCalculator::eval_forces (src/force/pair_force.cpp:21-60): the gate
// is the HALF-OPEN [rmin, rmax) of make_pair_bond (:28).
void eval_pair(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const Roles R{npair_of(S.ntypes), S.ntypes};
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const Table &T = S.tables[R.pair(ti, S.type[cf.atom0 + S.nb_j[p]])];
      auto [rmin, rmax] = T.span();
      if (r < rmin || r >= rmax) continue;
      double phi, dphi;
      if (S.site_ok[kPhi][p]) {
        phi = eval_at(T.sp, S.site[kPhi][p]);
        dphi = deriv_at(T.sp, S.site[kPhi][p]);
      } else {
        phi = T.eval(r);
        dphi = T.deriv(r);
      }
      acc_pair(o, o.force[i], d, (dphi * (1.0 / r)) * d, phi);
    }
  }
}

using Sym = double[3][3];
inline double quad_nu(const double M[3][3], const Vec3 &d) {
  // d·(M d) − |d|²/3 · tr M (adp_force.hpp:63-66)
  Vec3 Md = {M[0][0] * d[0] + M[0][1] * d[1] + M[0][2] * d[2],
             M[1][0] * d[0] + M[1][1] * d[1] + M[1][2] * d[2],
             M[2][0] * d[0] + M[2][1] * d[1] + M[2][2] * d[2]};
  return dot(d, Md) - sqnorm(d) / 3.0 * (M[0][0] + M[1][1] + M[2][2]);
}
inline Vec3 quad_xi(const double M[3][3], const Vec3 &d) {
  // M d − (tr M / 3) d (adp_force.hpp:67-69)
  const double tr = (M[0][0] + M[1][1] + M[2][2]) / 3.0;
  return {M[0][0] * d[0] + M[0][1] * d[1] + M[0][2] * d[2] - tr * d[0],
          M[1][0] * d[0] + M[1][1] * d[1] + M[1][2] * d[2] - tr * d[1],
          M[2][0] * d[0] + M[2][1] * d[1] + M[2][2] * d[2] - tr * d[2]};
}

// ADPForceCalculator::eval_forces (src/force/adp_force.cpp:73-135)
void eval_adp(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const Roles R{npair_of(S.ntypes), S.ntypes};
  const int n = cf.natoms;
  std::vector<double> rho(n, 0.0), gradF(n, 0.0);
  std::vector<Vec3> mu(n, Vec3{0, 0, 0});
  std::vector<std::array<double, 9>> lam(n);
  for (auto &l : lam) l.fill(0.0);
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    double rr = 0.0;
    Vec3 m = {0, 0, 0};
    double L[9] = {0};
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const int tj = S.type[cf.atom0 + S.nb_j[p]];
      rr += gated_eval(S, kGj, p, S.tables[R.dens(tj)], r);
      m = m + gated_eval(S, kDip, p, S.tables[R.dip(ti, tj)], r) * d;
      const double w = gated_eval(S, kQuad, p, S.tables[R.quad(ti, tj)], r);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) L[3 * a + b] += w * (d[a] * d[b]);
    }
    rho[i] += rr;
    mu[i] = mu[i] + m;
    for (int k = 0; k < 9; ++k) lam[i][k] += L[k];
  }
  double energy = 0.0;
  for (int i = 0; i < n; ++i) {
    const Table &emb = S.tables[R.emb(S.type[cf.atom0 + i])];
    rho[i] = clamp_rho(emb, rho[i], o.limit);
    double e = emb.eval(rho[i]);
    gradF[i] = emb.deriv(rho[i]);
    e += 0.5 * sqnorm(mu[i]);
    const double tr = lam[i][0] + lam[i][4] + lam[i][8];
    double sq = 0.0;
    for (int k = 0; k < 9; ++k) sq += lam[i][k] * lam[i][k];
    e += 0.5 * (sq - tr * tr / 3.0);
    energy += e;
  }
  o.energy += energy;
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    double Li[3][3], Lj[3][3];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) Li[a][b] = lam[i][3 * a + b];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const double inv_r = 1.0 / r;
      const int j = S.nb_j[p];
      const int tj = S.type[cf.atom0 + j];
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) Lj[a][b] = lam[j][3 * a + b];
      Vec3 f = {0, 0, 0};
      // add_eam_force (:31-43)
      const Table &phi_t = S.tables[R.pair(ti, tj)];
      const double phi = gated_eval(S, kPhi, p, phi_t, r);
      const double dphi = gated_deriv(S, kPhi, p, phi_t, r);
      const double drho_j = gated_deriv(S, kGj, p, S.tables[R.dens(tj)], r);
      const double drho_i = gated_deriv(S, kGi, p, S.tables[R.dens(ti)], r);
      f = f + ((dphi + gradF[i] * drho_j + gradF[j] * drho_i) * inv_r) * d;
      // add_dipole_force (:45-54)
      const Table &ut = S.tables[R.dip(ti, tj)];
      const double u = gated_eval(S, kDip, p, ut, r);
      const double du = gated_deriv(S, kDip, p, ut, r);
      const double dot_i = dot(mu[i], d), dot_j = dot(mu[j], d);
      f = f + (du * inv_r * (dot_i - dot_j)) * d + u * (mu[i] - mu[j]);
      // add_quadrupole_force (:56-65)
      const Table &wt = S.tables[R.quad(ti, tj)];
      const double w = gated_eval(S, kQuad, p, wt, r);
      const double dw = gated_deriv(S, kQuad, p, wt, r);
      const double nu = quad_nu(Li, d) + quad_nu(Lj, d);
      const Vec3 xi = quad_xi(Li, d) + quad_xi(Lj, d);
      f = f + (dw * inv_r * nu) * d + (2.0 * w) * xi;
      acc_pair(o, o.force[i], d, f, phi);
    }
  }
}

// Stillinger–Weber (src/force/stiweb_force.cpp:24-54,241-271)
struct SWP {
  double A, B, p, q, delta, a1, gamma, a2;
};
inline SWP swp(const Table &t) {
  return {t.v[0], t.v[1], t.v[2], t.v[3], t.v[4], t.v[5], t.v[6], t.v[7]};
}
inline void v2_dv2(double r, const SWP &p, double &v2, double &dv2) {
  v2 = dv2 = 0.0;
  if (r >= p.a1) return;
  const double d = r - p.a1;
  const double e = std::exp(p.delta / d);
  if (e == 0.0) return;
  const double rp = std::pow(r, -p.p);
  const double rq = std::pow(r, -p.q);
  const double poly = p.A * rp - p.B * rq;
  const double dpoly = -p.A * p.p * std::pow(r, -p.p - 1.0) + p.B * p.q * std::pow(r, -p.q - 1.0);
  v2 = poly * e;
  dv2 = dpoly * e + poly * e * (-p.delta / (d * d));
}
inline void h_dh(double r, const SWP &p, double &h, double &dh) {
  h = dh = 0.0;
  if (r >= p.a2) return;
  const double d = r - p.a2;
  h = std::exp(p.gamma / d);
  if (h == 0.0) return;
  dh = h * (-p.gamma / (d * d));
}

void eval_sw(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes, np = npair_of(nt);
  const Table &lam = S.tables[np];
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const SWP P = swp(S.tables[pair_ordinal(ti, S.type[cf.atom0 + S.nb_j[p]], nt)]);
      double v2, dv2;
      v2_dv2(r, P, v2, dv2);
      acc_pair(o, o.force[i], d, (dv2 / r) * d, v2);
    }
  }
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    const int64_t s0 = S.nb_start[gi], s1 = S.nb_start[gi + 1];
    for (int64_t pj = s0; pj < s1; ++pj) {
      const Vec3 &d1 = S.nb_d[pj];
      const double r1 = norm(d1);
      if (r1 < 1e-14) continue;
      const int j = S.nb_j[pj];
      const int tj = S.type[cf.atom0 + j];
      double h1, dh1;
      h_dh(r1, swp(S.tables[pair_ordinal(ti, tj, nt)]), h1, dh1);
      if (h1 == 0.0 && dh1 == 0.0) continue;
      const double inv_r1 = 1.0 / r1;
      for (int64_t pk = pj + 1; pk < s1; ++pk) {
        const Vec3 &d2 = S.nb_d[pk];
        const double r2 = norm(d2);
        if (r2 < 1e-14) continue;
        const int k = S.nb_j[pk];
        const int tk = S.type[cf.atom0 + k];
        double h2, dh2;
        h_dh(r2, swp(S.tables[pair_ordinal(ti, tk, nt)]), h2, dh2);
        if (h2 == 0.0 && dh2 == 0.0) continue;
        const double inv_r2 = 1.0 / r2;
        const double lambda = lam.v[ti * np + pair_ordinal(tj, tk, nt)];
        // add_angular (:138-144)
        const double cth = dot(d1, d2) * inv_r1 * inv_r2;
        const double cp13 = cth + 1.0 / 3.0;
        const double w = lambda * cp13 * cp13;
        const double dw = 2.0 * lambda * cp13;
        o.energy += h1 * h2 * w;
        // three_body_forces (kernels.hpp:44-58)
        const double inv_r1r2 = inv_r1 * inv_r2;
        const double Aa = cth * inv_r1 * inv_r1 - inv_r1r2;
        const double Bb = cth * inv_r2 * inv_r2 - inv_r1r2;
        const double g = w, dg = dw;
        const Vec3 fi = (dh1 * inv_r1 * h2 * g) * d1 + (h1 * dh2 * inv_r2 * g) * d2 -
                        (h1 * h2 * dg) * (Aa * d1 + Bb * d2);
        const Vec3 fj = -1.0 * ((dh1 * inv_r1 * h2 * g) * d1) -
                        (h1 * h2 * dg) * (inv_r1r2 * d2 - (cth * inv_r1 * inv_r1) * d1);
        const Vec3 fk = -1.0 * ((h1 * dh2 * inv_r2 * g) * d2) -
                        (h1 * h2 * dg) * (inv_r1r2 * d1 - (cth * inv_r2 * inv_r2) * d2);
        // accumulate_triplet (kernels.hpp:60-68)
        o.force[i] = o.force[i] + fi;
        o.force[j] = o.force[j] + fj;
        o.force[k] = o.force[k] + fk;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) o.stress[a][b] += d1[a] * fj[b];
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) o.stress[a][b] += d2[a] * fk[b];
      }
    }
  }
}

// Tersoff (src/force/tersoff_force.cpp).  Per directed bond i→j with the
// (t_i, t_j) parameters p: f_c, V_R = A e^{−λr}, V_A = B e^{−μr} (make_bond
// :85-101); ζ_ij = Σ_{k≠j} ω_ik f_c(r_ik) g_ij(cos θ_ijk) with the (t_i, t_k)
// cutoff and ω (add_zeta :103-128); b = (1 + (βζ)^n)^{−1/2n} (bond_order
// :63-70); E += ½ f_c (V_R − b V_A) and the radial pair force on i, −on j
// (accumulate_pair :135-151); then the ζ-gradient forces on i, j, k with
// P = ½ f_c V_A ∂b/∂ζ (accumulate_three_body :153-206).
constexpr double kPi = 3.14159265358979323846; // std::numbers::pi
struct TsP {
  double A, B, lam, mu, beta, n, c, d, h, R, S, omega;
};
inline TsP tsp(const Table &t) {
  return {t.v[0], t.v[1], t.v[2], t.v[3], t.v[4], t.v[5], t.v[6], t.v[7], t.v[8], t.v[9], t.v[10], t.v[11]};
}
// fc_val / dfc_val (:26-43)
inline double ts_fc(double r, double R, double S) {
  if (r <= R) return 1.0;
  if (r >= S) return 0.0;
  return 0.5 + 0.5 * std::cos(kPi * (r - R) / (S - R));
}
inline double ts_dfc(double r, double R, double S) {
  if (r <= R || r >= S) return 0.0;
  return -0.5 * kPi / (S - R) * std::sin(kPi * (r - R) / (S - R));
}
// g_val / dg_val (:45-61)
inline double ts_g(double c, const TsP &p) {
  const double c2 = p.c * p.c, d2 = p.d * p.d, hc = p.h - c;
  return 1.0 + c2 / d2 - c2 / (d2 + hc * hc);
}
inline double ts_dg(double c, const TsP &p) {
  const double c2 = p.c * p.c, d2 = p.d * p.d, hc = p.h - c;
  const double den = d2 + hc * hc;
  return -2.0 * c2 * hc / (den * den);
}
// bond_order / dbond_dzeta (:63-83)
inline double ts_b(double zeta, const TsP &p) {
  if (zeta == 0.0) return 1.0;
  return std::pow(1.0 + std::pow(p.beta * zeta, p.n), -0.5 / p.n);
}
inline double ts_db(double zeta, const TsP &p) {
  if (zeta == 0.0) return 0.0;
  const double bzn = std::pow(p.beta * zeta, p.n);
  const double b = std::pow(1.0 + bzn, -0.5 / p.n);
  return -0.5 * b * bzn / (zeta * (1.0 + bzn));
}

void eval_tersoff(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes, np = npair_of(nt);
  std::vector<TsP> P(np);
  for (int s = 0; s < np; ++s) P[s] = tsp(S.tables[s]);
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    const int64_t s0 = S.nb_start[gi], s1 = S.nb_start[gi + 1];
    for (int64_t pj = s0; pj < s1; ++pj) {
      const Vec3 &d1 = S.nb_d[pj];
      const double r1 = norm(d1);
      const int j = S.nb_j[pj];
      const TsP &p = P[pair_ordinal(ti, S.type[cf.atom0 + j], nt)];
      if (r1 < 1e-14) continue;
      const double fc = ts_fc(r1, p.R, p.S), dfc = ts_dfc(r1, p.R, p.S);
      if (fc == 0.0 && dfc == 0.0) continue;
      const double VR = p.A * std::exp(-p.lam * r1), VA = p.B * std::exp(-p.mu * r1);
      const double VRp = -p.lam * VR, VAp = -p.mu * VA;
      double zeta = 0.0;
      for (int64_t pk = s0; pk < s1; ++pk) {
        if (pk == pj) continue;
        const Vec3 &d2 = S.nb_d[pk];
        const double r2 = norm(d2);
        if (r2 < 1e-14) continue;
        const TsP &q = P[pair_ordinal(ti, S.type[cf.atom0 + S.nb_j[pk]], nt)];
        const double fck = ts_fc(r2, q.R, q.S);
        if (fck == 0.0) continue;
        const double cth = dot(d1, d2) / (r1 * r2);
        zeta += q.omega * fck * ts_g(cth, p);
      }
      const double b = ts_b(zeta, p);
      o.energy += 0.5 * fc * (VR - b * VA);
      const double pc = 0.5 * (dfc * (VR - b * VA) + fc * (VRp - b * VAp)) / r1;
      const Vec3 Fp = pc * d1;
      o.force[i] = o.force[i] + Fp;
      o.force[j] = o.force[j] - Fp;
      for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb) o.stress[a][bb] += 0.5 * d1[a] * (-Fp[bb]);
      if (zeta == 0.0) continue;
      const double Pz = 0.5 * fc * VA * ts_db(zeta, p);
      const double inv_r1 = 1.0 / r1;
      for (int64_t pk = s0; pk < s1; ++pk) {
        if (pk == pj) continue;
        const Vec3 &d2 = S.nb_d[pk];
        const double r2 = norm(d2);
        if (r2 < 1e-14) continue;
        const int k = S.nb_j[pk];
        const TsP &q = P[pair_ordinal(ti, S.type[cf.atom0 + k], nt)];
        const double fck = ts_fc(r2, q.R, q.S), dfck = ts_dfc(r2, q.R, q.S);
        if (fck == 0.0 && dfck == 0.0) continue;
        const double inv_r2 = 1.0 / r2;
        const double cth = dot(d1, d2) * inv_r1 * inv_r2;
        const double gv = ts_g(cth, p), dgv = ts_dg(cth, p);
        const double Ac = cth * inv_r1 * inv_r1 - inv_r1 * inv_r2;
        const double Bc = cth * inv_r2 * inv_r2 - inv_r1 * inv_r2;
        const double w = q.omega;
        const Vec3 dzi = w * ((-dfck * inv_r2 * gv) * d2 + (fck * dgv) * (Ac * d1 + Bc * d2));
        const Vec3 dzj = (w * fck * dgv) * ((inv_r1 * inv_r2) * d2 - (cth * inv_r1 * inv_r1) * d1);
        const Vec3 dzk =
            w * ((dfck * inv_r2 * gv) * d2 + (fck * dgv) * ((inv_r1 * inv_r2) * d1 - (cth * inv_r2 * inv_r2) * d2));
        const Vec3 Fi = Pz * dzi, Fj = Pz * dzj, Fk = Pz * dzk;
        o.force[i] = o.force[i] + Fi;
        o.force[j] = o.force[j] + Fj;
        o.force[k] = o.force[k] + Fk;
        for (int a = 0; a < 3; ++a)
          for (int bb = 0; bb < 3; ++bb) o.stress[a][bb] += d1[a] * Fj[bb] + d2[a] * Fk[bb];
      }
    }
  }
}

// Angular (src/force/angular_force.cpp:13-88): the pair term φ_{t_i t_j}
// (½ per directed pair, accumulate_pair kernels.hpp:33-38) plus, per central
// atom i and neighbour pair j < k, f_{t_i t_j}(r_ij) f_{t_i t_k}(r_ik)
// g_{t_i}(cos θ) with three_body_forces / accumulate_triplet
// (kernels.hpp:44-68).  φ and f are gated to their closed spans
// (force_calculator_concept.hpp:94-98); g is evaluated ungated.
void eval_angular(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes, np = npair_of(nt);
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const Table &T = S.tables[pair_ordinal(ti, S.type[cf.atom0 + S.nb_j[p]], nt)];
      if (!T.in_range(r)) continue;
      const double phi = T.eval(r), dphi = T.deriv(r);
      acc_pair(o, o.force[i], d, (dphi / r) * d, phi);
    }
  }
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    const Table &G = S.tables[2 * np + ti];
    const int64_t s0 = S.nb_start[gi], s1 = S.nb_start[gi + 1];
    for (int64_t pj = s0; pj < s1; ++pj) {
      const Vec3 &d1 = S.nb_d[pj];
      const double r1 = norm(d1);
      if (r1 < 1e-14) continue;
      const double inv_r1 = 1.0 / r1;
      const int j = S.nb_j[pj];
      const Table &Rj = S.tables[np + pair_ordinal(ti, S.type[cf.atom0 + j], nt)];
      if (!Rj.in_range(r1)) continue;
      const double f1 = Rj.eval(r1), df1 = Rj.deriv(r1);
      for (int64_t pk = pj + 1; pk < s1; ++pk) {
        const Vec3 &d2 = S.nb_d[pk];
        const double r2 = norm(d2);
        if (r2 < 1e-14) continue;
        const double inv_r2 = 1.0 / r2;
        const int k = S.nb_j[pk];
        const Table &Rk = S.tables[np + pair_ordinal(ti, S.type[cf.atom0 + k], nt)];
        if (!Rk.in_range(r2)) continue;
        const double f2 = Rk.eval(r2), df2 = Rk.deriv(r2);
        const double cth = dot(d1, d2) * inv_r1 * inv_r2;
        const double g = G.eval(cth), dg = G.deriv(cth);
        o.energy += f1 * f2 * g;
        const double inv_r1r2 = inv_r1 * inv_r2;
        const double Aa = cth * inv_r1 * inv_r1 - inv_r1r2;
        const double Bb = cth * inv_r2 * inv_r2 - inv_r1r2;
        const Vec3 fi = (df1 * inv_r1 * f2 * g) * d1 + (f1 * df2 * inv_r2 * g) * d2 -
                        (f1 * f2 * dg) * (Aa * d1 + Bb * d2);
        const Vec3 fj = -1.0 * ((df1 * inv_r1 * f2 * g) * d1) -
                        (f1 * f2 * dg) * (inv_r1r2 * d2 - (cth * inv_r1 * inv_r1) * d1);
        const Vec3 fk = -1.0 * ((f1 * df2 * inv_r2 * g) * d2) -
                        (f1 * f2 * dg) * (inv_r1r2 * d1 - (cth * inv_r2 * inv_r2) * d2);
        o.force[i] = o.force[i] + fi;
        o.force[j] = o.force[j] + fj;
        o.force[k] = o.force[k] + fk;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) o.stress[a][b] += d1[a] * fj[b] + d2[a] * fk[b];
      }
    }
  }
}

// ACSF descriptors (src/force/acsf.cpp) with a linear energy head per
// species (LinearHead, src/force/ml_force.cpp:11-47), evaluated as
// MLBase::eval_forces (include/forcesmith/force/ml_force.hpp): E_i = b + w·D_i;
// F_i −= (∂D_i/∂r_i)ᵀ w, F_j −= (∂D_i/∂r_j)ᵀ w, σ += d_ij ⊗ F_j part
// (accumulate_atom_forces).  The head gradient w is constant, so each term's
// descriptor gradient is weighted by its coefficient as it is formed.
struct AcsfSpec {
  double rcut;
  int g1, n2, n3, n4, n5;
  const double *p2, *p3, *p4, *p5; // (eta, rs), kappa, (eta, zeta, lambda) ×2
  explicit AcsfSpec(const double *v)
      : rcut(v[0]), g1(static_cast<int>(v[1])), n2(static_cast<int>(v[2])), n3(static_cast<int>(v[3])),
        n4(static_cast<int>(v[4])), n5(static_cast<int>(v[5])) {
    p2 = v + 6;
    p3 = p2 + 2 * n2;
    p4 = p3 + n3;
    p5 = p4 + 3 * n4;
  }
  // AcsfLayout (acsf.hpp:23-46): blocks G1..G3 per species, G4, G5 per pair
  int index(int block, int chan, int t, int nt) const {
    const int P = nt * (nt + 1) / 2;
    const int cnt[5] = {g1, n2, n3, n4, n5}, nch[5] = {nt, nt, nt, P, P};
    int base = 0;
    for (int b = 0; b < block; ++b) base += cnt[b] * nch[b];
    return base + chan * cnt[block] + t;
  }
};
// number of values an ACSF table must have (−1 if the counts are invalid)
int acsf_values(const double *v, int n) {
  if (n < 6) return -1;
  for (int k = 1; k < 6; ++k)
    if (v[k] < 0 || v[k] != std::floor(v[k])) return -1;
  return 6 + 2 * static_cast<int>(v[2]) + static_cast<int>(v[3]) + 3 * static_cast<int>(v[4]) +
         3 * static_cast<int>(v[5]);
}
int acsf_size(const AcsfSpec &A, int nt) {
  return nt * (A.g1 + A.n2 + A.n3) + nt * (nt + 1) / 2 * (A.n4 + A.n5);
}
// cutoff (acsf.cpp:15-23)
inline void acsf_fc(double r, double rc, double &fc, double &fcp) {
  if (r >= rc) {
    fc = fcp = 0.0;
    return;
  }
  const double x = kPi * r / rc;
  fc = 0.5 * (1.0 + std::cos(x));
  fcp = -0.5 * kPi / rc * std::sin(x);
}

// Per-species effective head {w ⊙ inv_std, b − Σ w·inv_std·mean}: the linear
// head of standardized descriptors (D − mean) ⊙ inv_std (ml_force.hpp:607-623)
// as a head of raw descriptors; without standardization tables, the head.
std::vector<double> acsf_head(const State &S, int t, int Sz) {
  const std::vector<double> &w = S.tables[1 + t].v;
  if (static_cast<int>(S.tables.size()) != 1 + 2 * S.ntypes) return w;
  const std::vector<double> &st = S.tables[1 + S.ntypes + t].v; // mean[S], inv_std[S]
  std::vector<double> h(Sz + 1);
  double b = w[Sz];
  for (int k = 0; k < Sz; ++k) {
    h[k] = w[k] * st[Sz + k];
    b -= h[k] * st[k];
  }
  h[Sz] = b;
  return h;
}

void eval_acsf(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes;
  const AcsfSpec A(S.tables[0].v.data());
  const int Sz = acsf_size(A, nt);
  std::vector<std::vector<double>> heads(nt);
  for (int t = 0; t < nt; ++t) heads[t] = acsf_head(S, t, Sz);
  struct Nb {
    int64_t p; // the entry in the atom's neighbour list
    Vec3 d, rh;
    double r, fc, fcp;
    int s;
  };
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    const double *w = heads[ti].data();
    const int64_t s0 = S.nb_start[gi], s1 = S.nb_start[gi + 1];
    std::vector<Nb> nb; // collect_neighbors (acsf.cpp:84-99): 1e-14 ≤ r < rcut
    for (int64_t p = s0; p < s1; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14 || r >= A.rcut) continue;
      Nb n{p, d, (1.0 / r) * d, r, 0.0, 0.0, S.type[cf.atom0 + S.nb_j[p]]};
      acsf_fc(r, A.rcut, n.fc, n.fcp);
      nb.push_back(n);
    }
    std::vector<Vec3> gw(s1 - s0, Vec3{0, 0, 0}); // (∂D_i/∂r_j)ᵀ w per neighbour entry
    Vec3 gself{0, 0, 0};
    double e = w[Sz];
    // accumulate_radial (acsf.cpp:101-131) with scatter_radial (:25-30)
    auto radial = [&](const Nb &n, int idx, double g, double dg) {
      e += w[idx] * g;
      gw[n.p - s0] = gw[n.p - s0] + (w[idx] * dg) * n.rh;
      gself = gself - (w[idx] * dg) * n.rh;
    };
    for (const Nb &n : nb) {
      for (int t = 0; t < A.g1; ++t) radial(n, A.index(0, n.s, t, nt), n.fc, n.fcp);
      for (int t = 0; t < A.n2; ++t) {
        const double eta = A.p2[2 * t], rs = A.p2[2 * t + 1], dr = n.r - rs;
        const double gauss = std::exp(-eta * dr * dr);
        radial(n, A.index(1, n.s, t, nt), gauss * n.fc, gauss * (-2.0 * eta * dr * n.fc + n.fcp));
      }
      for (int t = 0; t < A.n3; ++t) {
        const double k = A.p3[t], cc = std::cos(k * n.r), ss = std::sin(k * n.r);
        radial(n, A.index(2, n.s, t, nt), cc * n.fc, -k * ss * n.fc + cc * n.fcp);
      }
    }
    // accumulate_angular (acsf.cpp:133-183) with scatter_angular (:43-79)
    if (A.n4 + A.n5 > 0)
      for (size_t a = 0; a < nb.size(); ++a)
        for (size_t b = a + 1; b < nb.size(); ++b) {
          const Nb &J = nb[a], &K = nb[b];
          const double costh = std::clamp(dot(J.d, K.d) / (J.r * K.r), -1.0, 1.0);
          const Vec3 djk = K.d - J.d;
          const double rjk = norm(djk);
          const Vec3 rjk_h = rjk > 1e-14 ? (1.0 / rjk) * djk : Vec3{0, 0, 0};
          double fcjk, fcpjk;
          acsf_fc(rjk, A.rcut, fcjk, fcpjk);
          const Vec3 dcj = (1.0 / J.r) * (K.rh - costh * J.rh), dck = (1.0 / K.r) * (J.rh - costh * K.rh);
          const int po = pair_ordinal(J.s, K.s, nt);
          auto angular = [&](int idx, double eta, double zeta, double lambda, bool with_jk) {
            const double Aa = 1.0 + lambda * costh;
            if (Aa <= 1e-12) return;
            const double C = std::pow(2.0, 1.0 - zeta), ang = std::pow(Aa, zeta);
            const double dang = zeta * std::pow(Aa, zeta - 1.0) * lambda;
            const double rsum = J.r * J.r + K.r * K.r + (with_jk ? rjk * rjk : 0.0);
            const double rad = std::exp(-eta * rsum);
            const double fjk = with_jk ? fcjk : 1.0;
            const double fcs = J.fc * K.fc * fjk;
            e += w[idx] * (C * ang * rad * fcs);
            const double drij = rad * (-2.0 * eta * J.r), drik = rad * (-2.0 * eta * K.r);
            const double drjk = with_jk ? rad * (-2.0 * eta * rjk) : 0.0;
            const double dfij = J.fcp * K.fc * fjk, dfik = J.fc * K.fcp * fjk;
            const double dfjk = with_jk ? J.fc * K.fc * fcpjk : 0.0;
            const double cij = C * ang * (drij * fcs + rad * dfij), cik = C * ang * (drik * fcs + rad * dfik);
            const double cjk = C * ang * (drjk * fcs + rad * dfjk), ccos = C * rad * fcs * dang;
            const Vec3 gj = cij * J.rh - cjk * rjk_h + ccos * dcj;
            const Vec3 gk = cik * K.rh + cjk * rjk_h + ccos * dck;
            gw[J.p - s0] = gw[J.p - s0] + w[idx] * gj;
            gw[K.p - s0] = gw[K.p - s0] + w[idx] * gk;
            gself = gself - w[idx] * (gj + gk);
          };
          for (int t = 0; t < A.n4; ++t)
            angular(A.index(3, po, t, nt), A.p4[3 * t], A.p4[3 * t + 1], A.p4[3 * t + 2], true);
          for (int t = 0; t < A.n5; ++t)
            angular(A.index(4, po, t, nt), A.p5[3 * t], A.p5[3 * t + 1], A.p5[3 * t + 2], false);
        }
    // energy and accumulate_atom_forces
    o.energy += e;
    o.force[i] = o.force[i] - gself;
    for (int64_t p = s0; p < s1; ++p) {
      const Vec3 fj = -1.0 * gw[p - s0];
      const int j = S.nb_j[p];
      o.force[j] = o.force[j] + fj;
      for (int a = 0; a < 3; ++a)
        for (int bb = 0; bb < 3; ++bb) o.stress[a][bb] += S.nb_d[p][a] * fj[bb];
    }
  }
}

// Descriptor values of atom i of configuration c (ACSF::get_descriptor,
// acsf.cpp:84-196, values only) into D[Sz].
void acsf_values_of(const State &S, int c, int i, double *D) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes;
  const AcsfSpec A(S.tables[0].v.data());
  const int Sz = acsf_size(A, nt);
  std::fill(D, D + Sz, 0.0);
  const int64_t gi = cf.atom0 + i;
  struct Nb {
    Vec3 d;
    double r, fc;
    int s;
  };
  std::vector<Nb> nb;
  for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
    const Vec3 &d = S.nb_d[p];
    const double r = norm(d);
    if (r < 1e-14 || r >= A.rcut) continue;
    double fc, fcp;
    acsf_fc(r, A.rcut, fc, fcp);
    nb.push_back({d, r, fc, S.type[cf.atom0 + S.nb_j[p]]});
  }
  for (const Nb &n : nb) {
    for (int t = 0; t < A.g1; ++t) D[A.index(0, n.s, t, nt)] += n.fc;
    for (int t = 0; t < A.n2; ++t) {
      const double dr = n.r - A.p2[2 * t + 1];
      D[A.index(1, n.s, t, nt)] += std::exp(-A.p2[2 * t] * dr * dr) * n.fc;
    }
    for (int t = 0; t < A.n3; ++t) D[A.index(2, n.s, t, nt)] += std::cos(A.p3[t] * n.r) * n.fc;
  }
  for (size_t a = 0; a < nb.size(); ++a)
    for (size_t b = a + 1; b < nb.size(); ++b) {
      const Nb &J = nb[a], &K = nb[b];
      const double costh = std::clamp(dot(J.d, K.d) / (J.r * K.r), -1.0, 1.0);
      const double rjk = norm(K.d - J.d);
      double fcjk, fcpjk;
      acsf_fc(rjk, A.rcut, fcjk, fcpjk);
      const int po = pair_ordinal(J.s, K.s, nt);
      auto g = [&](double eta, double zeta, double lambda, bool with_jk) {
        const double Aa = 1.0 + lambda * costh;
        if (Aa <= 1e-12) return 0.0;
        const double rsum = J.r * J.r + K.r * K.r + (with_jk ? rjk * rjk : 0.0);
        return std::pow(2.0, 1.0 - zeta) * std::pow(Aa, zeta) * std::exp(-eta * rsum) * J.fc * K.fc *
               (with_jk ? fcjk : 1.0);
      };
      for (int t = 0; t < A.n4; ++t)
        D[A.index(3, po, t, nt)] += g(A.p4[3 * t], A.p4[3 * t + 1], A.p4[3 * t + 2], true);
      for (int t = 0; t < A.n5; ++t)
        D[A.index(4, po, t, nt)] += g(A.p5[3 * t], A.p5[3 * t + 1], A.p5[3 * t + 2], false);
    }
}

// LMBTR descriptors (src/force/lmbtr.cpp) with a linear energy head per
// species, evaluated as MLBase::eval_forces (ml_force.hpp:462-480).  LMBTR
// has no analytic descriptor gradient (analytic_grads() is false,
// lmbtr.hpp:48), so MLBase::descriptor_with_grad (ml_force.hpp:544-572)
// forms it by central differences, h = 1e-4, moving one neighbour-list
// displacement component at a time and recomputing the whole descriptor.
struct LmbtrGrid {
  int n;
  double min, max, sigma;
};
struct LmbtrSpec {
  double rcut, ws;
  bool normalize;
  LmbtrGrid k2, k3; // n == 0: the term is absent
  explicit LmbtrSpec(const double *v)
      : rcut(v[0]), ws(v[1]), normalize(v[2] != 0.0),
        k2{static_cast<int>(v[3]), v[4], v[5], v[6]}, k3{static_cast<int>(v[7]), v[8], v[9], v[10]} {}
};
inline int lmbtr_size(const LmbtrSpec &L, int nt) { return nt * L.k2.n + nt * (nt + 1) / 2 * L.k3.n; }
// 11 values, counts non-negative integers, at least one term, positive
// rcut, weight scale and widths of the present terms
bool lmbtr_valid(const double *v, int n) {
  if (n != 11 || !(v[0] > 0.0) || !(v[1] > 0.0)) return false;
  for (int k : {3, 7})
    if (v[k] < 0 || v[k] != std::floor(v[k]) || (v[k] > 0 && !(v[k + 3] > 0.0))) return false;
  return v[3] + v[7] > 0;
}

// broaden (lmbtr.cpp:31-55): a Gaussian of width sigma at geom, scaled by
// w / (sigma sqrt(2π)), added to the grid bins within 5 sigma; successive
// bins by the constant-ratio recurrence of make_kernel (lmbtr.cpp:21-29).
void lmbtr_broaden(double *block, const LmbtrGrid &g, double geom, double w) {
  const double inv = 1.0 / (g.sigma * std::sqrt(2.0 * kPi)), s2 = 2.0 * g.sigma * g.sigma;
  const double a = w * inv;
  if (g.n <= 1) {
    const double dx = g.min - geom;
    block[0] += a * std::exp(-dx * dx / s2);
    return;
  }
  const double step = (g.max - g.min) / (g.n - 1), ratio = std::exp(-2.0 * step * step / s2);
  const double center = (geom - g.min) / step, rad = 5.0 * g.sigma / step;
  const int b0 = std::max(0, static_cast<int>(std::ceil(center - rad)));
  const int b1 = std::min(g.n - 1, static_cast<int>(std::floor(center + rad)));
  if (b0 > b1) return;
  const double dx0 = g.min + static_cast<double>(b0) * step - geom;
  double f = std::exp(-dx0 * dx0 / s2), u = std::exp(-(2.0 * dx0 * step + step * step) / s2);
  for (int b = b0; b <= b1; ++b) {
    block[b] += a * f;
    f *= u;
    u *= ratio;
  }
}

// get_descriptor (lmbtr.cpp:64-121) of one atom from its neighbour-list
// displacements d[0..n) and species s[0..n): neighbours with 1e-14 ≤ r < rcut
// (descriptor_neighbor, ml_force.hpp:85-97), the k2 term per neighbour, the
// k3 term per neighbour pair j < k in list order, then the L2 normalisation.
void lmbtr_descriptor(const LmbtrSpec &L, int nt, const Vec3 *d, const int *s, int n, double *D) {
  const int Sz = lmbtr_size(L, nt), base3 = nt * L.k2.n;
  std::fill(D, D + Sz, 0.0);
  struct Nb {
    double r;
    Vec3 d;
    int s;
  };
  std::vector<Nb> nb;
  for (int p = 0; p < n; ++p) {
    const double r = norm(d[p]);
    if (r < 1e-14 || r >= L.rcut) continue;
    nb.push_back({r, d[p], s[p]});
  }
  if (L.k2.n > 0)
    for (const Nb &j : nb) lmbtr_broaden(D + j.s * L.k2.n, L.k2, j.r, std::exp(-j.r / L.ws));
  if (L.k3.n > 0)
    for (size_t a = 0; a < nb.size(); ++a)
      for (size_t b = a + 1; b < nb.size(); ++b) {
        const Nb &J = nb[a], &K = nb[b];
        const double costh = std::clamp(dot(J.d, K.d) / (J.r * K.r), -1.0, 1.0);
        const double rjk = norm(K.d - J.d);
        const double w = std::exp(-(J.r + K.r + rjk) / L.ws);
        lmbtr_broaden(D + base3 + pair_ordinal(J.s, K.s, nt) * L.k3.n, L.k3, costh, w);
      }
  if (L.normalize) {
    double ss = 0.0;
    for (int k = 0; k < Sz; ++k) ss += D[k] * D[k];
    const double nrm = std::sqrt(ss);
    if (nrm > 1e-300)
      for (int k = 0; k < Sz; ++k) D[k] /= nrm;
  }
}

// Atom i's neighbour-list displacements and species.
void lmbtr_env(const State &S, int c, int i, std::vector<Vec3> &d, std::vector<int> &s) {
  const Config &cf = S.cfgs[c];
  const int64_t gi = cf.atom0 + i;
  d.clear();
  s.clear();
  for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
    d.push_back(S.nb_d[p]);
    s.push_back(S.type[cf.atom0 + S.nb_j[p]]);
  }
}

void lmbtr_values_of(const State &S, int c, int i, double *D) {
  std::vector<Vec3> d;
  std::vector<int> s;
  lmbtr_env(S, c, i, d, s);
  lmbtr_descriptor(LmbtrSpec(S.tables[0].v.data()), S.ntypes, d.data(), s.data(), static_cast<int>(d.size()), D);
}

void eval_lmbtr(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  const int nt = S.ntypes;
  const LmbtrSpec L(S.tables[0].v.data());
  const int Sz = lmbtr_size(L, nt);
  std::vector<std::vector<double>> heads(nt);
  for (int t = 0; t < nt; ++t) heads[t] = acsf_head(S, t, Sz); // standardization folded in
  constexpr double h = 1e-4; // descriptor_with_grad (ml_force.hpp:553)
  // per atom: its energy and, per neighbour-list entry, (∂D/∂d)ᵀ w; formed
  // in parallel over the atoms, summed below in atom order
  std::vector<double> ea(cf.natoms);
  std::vector<std::vector<Vec3>> gwa(cf.natoms);
#pragma omp parallel for schedule(dynamic) if (!omp_in_parallel())
  for (int i = 0; i < cf.natoms; ++i) {
    std::vector<Vec3> d;
    std::vector<int> s;
    std::vector<double> D(Sz), Dp(Sz), Dm(Sz);
    const int64_t gi = cf.atom0 + i;
    const double *w = heads[S.type[gi]].data();
    lmbtr_env(S, c, i, d, s);
    const int n = static_cast<int>(d.size());
    lmbtr_descriptor(L, nt, d.data(), s.data(), n, D.data());
    double e = w[Sz];
    for (int k = 0; k < Sz; ++k) e += w[k] * D[k];
    ea[i] = e;
    // grad_neigh by central differences, contracted with dE/dD = w
    gwa[i].assign(n, Vec3{0, 0, 0});
    for (int p = 0; p < n; ++p)
      for (int a = 0; a < 3; ++a) {
        const double x0 = d[p][a];
        d[p][a] = x0 + h;
        lmbtr_descriptor(L, nt, d.data(), s.data(), n, Dp.data());
        d[p][a] = x0 - h;
        lmbtr_descriptor(L, nt, d.data(), s.data(), n, Dm.data());
        d[p][a] = x0;
        double t = 0.0;
        for (int k = 0; k < Sz; ++k) t += w[k] * ((Dp[k] - Dm[k]) / (2.0 * h));
        gwa[i][p][a] = t;
      }
  }
  // accumulate_atom_forces (ml_force.hpp:595-605)
  for (int i = 0; i < cf.natoms; ++i) {
    const int64_t gi = cf.atom0 + i;
    o.energy += ea[i];
    for (size_t p = 0; p < gwa[i].size(); ++p) {
      const Vec3 &gw = gwa[i][p];
      const Vec3 fj = -1.0 * gw;
      o.force[i] = o.force[i] + gw; // −grad_selfᵀ w, grad_self = −Σ grad_neigh
      const int64_t q = S.nb_start[gi] + static_cast<int64_t>(p);
      const int j = S.nb_j[q];
      o.force[j] = o.force[j] + fj;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) o.stress[a][b] += S.nb_d[q][a] * fj[b];
    }
  }
}

// with_eval_scope (include/forcesmith/force/eval_scope.hpp:13-31): zero,
// run the kernel, σ /= V.
void eval_config(const State &S, int c, Out &o) {
  const Config &cf = S.cfgs[c];
  o.force.assign(cf.natoms, Vec3{0, 0, 0});
  o.energy = o.limit = 0.0;
  for (auto &row : o.stress) row[0] = row[1] = row[2] = 0.0;
  switch (S.family) {
  case FS_FAMILY_EAM: eval_eam(S, c, o); break;
  case FS_FAMILY_PAIR: eval_pair(S, c, o); break;
  case FS_FAMILY_ADP: eval_adp(S, c, o); break;
  case FS_FAMILY_SW: eval_sw(S, c, o); break;
  case FS_FAMILY_TERSOFF: eval_tersoff(S, c, o); break;
  case FS_FAMILY_ANGULAR: eval_angular(S, c, o); break;
  case FS_FAMILY_ACSF: eval_acsf(S, c, o); break;
  case FS_FAMILY_LMBTR: eval_lmbtr(S, c, o); break;
  }
  const double V = cf.pbc.volume;
  for (auto &row : o.stress)
    for (double &v : row) v /= V;
}

int64_t config_rows(const Config &cf, double w_s) {
  return 3 * cf.natoms + 2 + (w_s > 0.0 ? 6 : 0); // residual_layout.hpp:18-22
}

// write_config_residuals (residual_layout.hpp:37-54)
int64_t write_residuals(const State &S, int c, const Out &o, double w_e, double w_s,
                        double *F, int64_t row) {
  const Config &cf = S.cfgs[c];
  for (int i = 0; i < cf.natoms; ++i)
    for (int a = 0; a < 3; ++a) F[row++] = o.force[i][a] - S.ref_force[cf.atom0 + i][a];
  F[row++] = w_e * (o.energy - cf.ref_energy);
  if (w_s > 0.0)
    for (auto &vv : kVoigt)
      F[row++] = w_s * (o.stress[vv[0]][vv[1]] - cf.ref_stress[vv[0]][vv[1]]);
  F[row++] = o.limit;
  return row;
}

// TableParams (force_calculator_concept.hpp:171-208): tables in order, then
// the free globals; scatter broadcasts each global to its links (:225-229).
int param_count(const State &S) {
  int D = 0;
  for (const Table &t : S.tables) D += t.param_count();
  for (uint8_t f : S.gfixed) D += f ? 0 : 1;
  return D;
}
void gather(const State &S, double *x) {
  int o = 0;
  for (const Table &t : S.tables)
    for (int k : t.free_idx) x[o++] = t.v[k];
  for (std::size_t g = 0; g < S.gval.size(); ++g)
    if (!S.gfixed[g]) x[o++] = S.gval[g];
}
void broadcast_globals(State &S) {
  for (const auto &lk : S.links) S.tables[lk[1]].v[lk[2]] = S.gval[lk[0]];
}
void scatter(State &S, const double *x) {
  int o = 0;
  for (Table &t : S.tables)
    for (int k : t.free_idx) t.v[k] = x[o++];
  for (std::size_t g = 0; g < S.gval.size(); ++g)
    if (!S.gfixed[g]) S.gval[g] = x[o++];
  broadcast_globals(S);
  for (Table &t : S.tables) t.refresh();
}

std::vector<int64_t> row_offsets(const State &S, double w_s) {
  std::vector<int64_t> ro(S.cfgs.size() + 1, 0);
  for (std::size_t c = 0; c < S.cfgs.size(); ++c) ro[c + 1] = ro[c] + config_rows(S.cfgs[c], w_s);
  return ro;
}

void residual(const State &S, double w_e, double w_s, double *F,
              const std::vector<int64_t> &ro, std::vector<Out> *keep = nullptr) {
  const int nc = static_cast<int>(S.cfgs.size());
  if (keep) keep->resize(nc);
  if (S.family == FS_FAMILY_LMBTR) { // parallel over each configuration's atoms instead (eval_lmbtr)
    Out o;
    for (int c = 0; c < nc; ++c) {
      Out &oo = keep ? (*keep)[c] : o;
      eval_config(S, c, oo);
      write_residuals(S, c, oo, w_e, w_s, F, ro[c]);
    }
    return;
  }
#pragma omp parallel
  {
    Out o;
#pragma omp for schedule(dynamic)
    for (int c = 0; c < nc; ++c) {
      Out &oo = keep ? (*keep)[c] : o;
      eval_config(S, c, oo);
      write_residuals(S, c, oo, w_e, w_s, F, ro[c]);
    }
  }
}

// Column offsets of every table in the parameter vector (table_columns,
// include/forcesmith/force/param_jacobian.hpp:18-41).
std::vector<int> table_cols(const State &S) {
  std::vector<int> col(S.tables.size() + 1, 0);
  for (std::size_t t = 0; t < S.tables.size(); ++t) col[t + 1] = col[t] + S.tables[t].param_count();
  return col;
}

// Analytic parameter Jacobian for EAM (src/force/eam_force.cpp:108-279) and
// Pair (src/force/pair_force.cpp:80-111), with param_grad/dderiv_dparam
// generalised to spline knots (Table::grad).  Writes rows [row0, …) of the
// column-major m × D matrix J (leading dimension m).
void add_force_column(double *J, int64_t m, int64_t atom_row, int64_t rE, int64_t rS,
                      int col, const Vec3 &d, const Vec3 &df, double denergy, double w_e,
                      double w_s, double inv_V) {
  // param_jacobian.hpp:91-109
  double *Jc = J + static_cast<int64_t>(col) * m;
  for (int a = 0; a < 3; ++a) Jc[atom_row + a] += df[a];
  if (denergy != 0.0) Jc[rE] += w_e * denergy;
  if (rS >= 0)
    for (int v = 0; v < 6; ++v) Jc[rS + v] -= w_s * 0.5 * d[kVoigt[v][0]] * df[kVoigt[v][1]] * inv_V;
}

void jacobian_eam_config(const State &S, int c, double w_e, double w_s, double *J, int64_t m,
                         int64_t row0, const std::vector<int> &col) {
  const Config &cf = S.cfgs[c];
  const Roles R{npair_of(S.ntypes), S.ntypes};
  const int n = cf.natoms;
  const int64_t rE = row0 + 3 * n;
  const int64_t rS = w_s > 0.0 ? rE + 1 : -1;
  const int64_t rL = rE + 1 + (w_s > 0.0 ? 6 : 0);
  const double inv_V = 1.0 / cf.pbc.volume;
  const int nt = S.ntypes;
  const int dens0 = col[R.dens(0)], ndens = col[R.dens(nt - 1) + 1] - dens0;
  const int emb0 = col[R.emb(0)], nemb = col[R.emb(nt - 1) + 1] - emb0;
  std::vector<double> rho(n, 0.0), drho(static_cast<std::size_t>(n) * ndens, 0.0);
  std::vector<double> gv(4096), gd(4096), gdd(4096);
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const double r = norm(S.nb_d[p]);
      const int tj = S.type[cf.atom0 + S.nb_j[p]];
      const Table &g = S.tables[R.dens(tj)];
      if (!g.in_range(r)) continue;
      rho[i] += g.eval(r);
      const int np_ = g.param_count();
      if (np_ == 0) continue;
      g.grad(r, gv.data(), gd.data());
      const int base = col[R.dens(tj)] - dens0;
      for (int k = 0; k < np_; ++k) drho[static_cast<std::size_t>(i) * ndens + base + k] += gv[k];
    }
  }
  std::vector<double> gradF(n), curvF(n), dgrad(static_cast<std::size_t>(n) * nemb, 0.0);
  for (int i = 0; i < n; ++i) {
    const int ti = S.type[cf.atom0 + i];
    const Table &emb = S.tables[R.emb(ti)];
    auto [b, e] = emb.span();
    double rb = rho[i], over = 0.0;
    if (rb > e) {
      over = 2.0 * kDummyWeight * 10.0 * (rb - e);
      rb = e;
    } else if (rb < b) {
      over = -2.0 * kDummyWeight * 10.0 * (b - rb);
      rb = b;
    }
    const bool clamped = over != 0.0;
    gradF[i] = emb.deriv(rb);
    curvF[i] = emb.deriv2(rb);
    const int ne = emb.param_count();
    if (ne > 0) {
      emb.grad(rb, gv.data(), gd.data());
      for (int k = 0; k < ne; ++k) {
        J[static_cast<int64_t>(col[R.emb(ti)] + k) * m + rE] += w_e * gv[k];
        dgrad[static_cast<std::size_t>(i) * nemb + (col[R.emb(ti)] - emb0) + k] = gd[k];
      }
    }
    for (int mm = 0; mm < ndens; ++mm) {
      const double dd = drho[static_cast<std::size_t>(i) * ndens + mm];
      if (dd == 0.0) continue;
      if (clamped)
        J[static_cast<int64_t>(dens0 + mm) * m + rL] += over * dd;
      else
        J[static_cast<int64_t>(dens0 + mm) * m + rE] += w_e * gradF[i] * dd;
    }
    if (clamped)
      std::fill(drho.begin() + static_cast<std::size_t>(i) * ndens,
                drho.begin() + static_cast<std::size_t>(i + 1) * ndens, 0.0);
    rho[i] = rb;
  }
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    const int64_t arow = row0 + 3 * i;
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const int j = S.nb_j[p];
      const int tj = S.type[cf.atom0 + j];
      const double inv_r = 1.0 / r;
      const int pt = R.pair(ti, tj);
      const Table &phi_t = S.tables[pt];
      if (phi_t.in_range(r) && phi_t.param_count() > 0) {
        phi_t.grad(r, gv.data(), gd.data());
        for (int k = 0; k < phi_t.param_count(); ++k)
          add_force_column(J, m, arow, rE, rS, col[pt] + k, d, (gd[k] * inv_r) * d,
                           0.5 * gv[k], w_e, w_s, inv_V);
      }
      const Table &gj = S.tables[R.dens(tj)];
      const Table &gi_t = S.tables[R.dens(ti)];
      const bool gj_in = gj.in_range(r), gi_in = gi_t.in_range(r);
      const double dg_j = gj_in ? gj.deriv(r) : 0.0;
      const double dg_i = gi_in ? gi_t.deriv(r) : 0.0;
      if (gj_in && gj.param_count() > 0) {
        gj.grad(r, gv.data(), gd.data());
        for (int k = 0; k < gj.param_count(); ++k)
          add_force_column(J, m, arow, rE, rS, col[R.dens(tj)] + k, d,
                           (gradF[i] * gd[k] * inv_r) * d, 0.0, w_e, w_s, inv_V);
      }
      if (gi_in && gi_t.param_count() > 0) {
        gi_t.grad(r, gv.data(), gd.data());
        for (int k = 0; k < gi_t.param_count(); ++k)
          add_force_column(J, m, arow, rE, rS, col[R.dens(ti)] + k, d,
                           (gradF[j] * gd[k] * inv_r) * d, 0.0, w_e, w_s, inv_V);
      }
      for (int mm = 0; mm < ndens; ++mm) {
        const double chain = curvF[i] * drho[static_cast<std::size_t>(i) * ndens + mm] * dg_j +
                             curvF[j] * drho[static_cast<std::size_t>(j) * ndens + mm] * dg_i;
        if (chain != 0.0)
          add_force_column(J, m, arow, rE, rS, dens0 + mm, d, (chain * inv_r) * d, 0.0, w_e,
                           w_s, inv_V);
      }
      for (int mm = 0; mm < nemb; ++mm) {
        const double chain = dgrad[static_cast<std::size_t>(i) * nemb + mm] * dg_j +
                             dgrad[static_cast<std::size_t>(j) * nemb + mm] * dg_i;
        if (chain != 0.0)
          add_force_column(J, m, arow, rE, rS, emb0 + mm, d, (chain * inv_r) * d, 0.0, w_e,
                           w_s, inv_V);
      }
    }
  }
}

void jacobian_pair_config(const State &S, int c, double w_e, double w_s, double *J, int64_t m,
                          int64_t row0, const std::vector<int> &col) {
  const Config &cf = S.cfgs[c];
  const Roles R{npair_of(S.ntypes), S.ntypes};
  const int n = cf.natoms;
  const int64_t rE = row0 + 3 * n;
  const int64_t rS = w_s > 0.0 ? rE + 1 : -1;
  const double inv_V = 1.0 / cf.pbc.volume;
  std::vector<double> gv(4096), gd(4096);
  for (int i = 0; i < n; ++i) {
    const int64_t gi = cf.atom0 + i;
    const int ti = S.type[gi];
    for (int64_t p = S.nb_start[gi]; p < S.nb_start[gi + 1]; ++p) {
      const Vec3 &d = S.nb_d[p];
      const double r = norm(d);
      if (r < 1e-14) continue;
      const int pt = R.pair(ti, S.type[cf.atom0 + S.nb_j[p]]);
      const Table &T = S.tables[pt];
      auto [rmin, rmax] = T.span();
      if (r < rmin || r >= rmax || T.param_count() == 0) continue;
      T.grad(r, gv.data(), gd.data());
      for (int k = 0; k < T.param_count(); ++k)
        add_force_column(J, m, row0 + 3 * i, rE, rS, col[pt] + k, d, (gd[k] * (1.0 / r)) * d,
                         0.5 * gv[k], w_e, w_s, inv_V);
    }
  }
}

// ---------------------------------------------------------------------------
// Dense FP64 helpers for the solver steps.
// ---------------------------------------------------------------------------

// In-place Cholesky A = L Lᵀ (lower), returns false if not SPD.
bool cholesky(std::vector<double> &A, int n) {
  for (int j = 0; j < n; ++j) {
    double s = A[j * n + j];
    for (int k = 0; k < j; ++k) s -= A[j * n + k] * A[j * n + k];
    if (!(s > 0.0)) return false;
    const double l = std::sqrt(s);
    A[j * n + j] = l;
    for (int i = j + 1; i < n; ++i) {
      double t = A[i * n + j];
      for (int k = 0; k < j; ++k) t -= A[i * n + k] * A[j * n + k];
      A[i * n + j] = t / l;
    }
  }
  return true;
}
void chol_solve(const std::vector<double> &L, int n, double *b) {
  for (int i = 0; i < n; ++i) {
    double s = b[i];
    for (int k = 0; k < i; ++k) s -= L[i * n + k] * b[k];
    b[i] = s / L[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double s = b[i];
    for (int k = i + 1; k < n; ++k) s -= L[k * n + i] * b[k];
    b[i] = s / L[i * n + i];
  }
}

} // namespace orc

using namespace orc;

struct orc_state {
  State S;
};

extern "C" {

int orc_create(orc_state **out) {
  if (!out) return FS_ERR_ARG;
  *out = new orc_state();
  return FS_OK;
}
int orc_destroy(orc_state *h) {
  delete h;
  return FS_OK;
}
int orc_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}
int orc_max_threads() { return omp_get_max_threads(); }

int orc_upload_configs(orc_state *h, int32_t n_cfg, const int32_t *natoms, const double *box9,
                       const double *pos, const int32_t *type, const double *ref_force,
                       const double *ref_energy, const double *ref_stress9) {
  if (!h || n_cfg < 0 || !natoms || !box9 || !pos || !type) return FS_ERR_ARG;
  State &S = h->S;
  S.cfgs.assign(n_cfg, Config{});
  int64_t off = 0;
  for (int c = 0; c < n_cfg; ++c) {
    Config &cf = S.cfgs[c];
    cf.natoms = natoms[c];
    cf.atom0 = off;
    off += natoms[c];
    Mat3 b;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) b(r, k) = box9[9 * c + 3 * r + k];
    cf.pbc.set(b);
    cf.ref_energy = ref_energy ? ref_energy[c] : 0.0;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) cf.ref_stress[r][k] = ref_stress9 ? ref_stress9[9 * c + 3 * r + k] : 0.0;
  }
  S.natoms_total = off;
  S.pos.resize(off);
  S.ref_force.resize(off);
  S.type.resize(off);
  for (int64_t i = 0; i < off; ++i) {
    S.pos[i] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    S.ref_force[i] = ref_force ? Vec3{ref_force[3 * i], ref_force[3 * i + 1], ref_force[3 * i + 2]}
                               : Vec3{0, 0, 0};
    S.type[i] = type[i];
  }
  S.rcut_built = -1;
  return FS_OK;
}

int orc_set_references(orc_state *h, const double *ref_force, const double *ref_energy,
                       const double *ref_stress9) {
  if (!h) return FS_ERR_ARG;
  State &S = h->S;
  for (int64_t i = 0; i < S.natoms_total; ++i)
    S.ref_force[i] = ref_force ? Vec3{ref_force[3 * i], ref_force[3 * i + 1], ref_force[3 * i + 2]}
                               : Vec3{0, 0, 0};
  for (std::size_t c = 0; c < S.cfgs.size(); ++c) {
    S.cfgs[c].ref_energy = ref_energy ? ref_energy[c] : 0.0;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k)
        S.cfgs[c].ref_stress[r][k] = ref_stress9 ? ref_stress9[9 * c + 3 * r + k] : 0.0;
  }
  return FS_OK;
}

int orc_set_model(orc_state *h, const fs_model *m) {
  if (!h || !m || m->ntypes < 1) return FS_ERR_ARG;
  const bool ml = m->family == FS_FAMILY_ACSF || m->family == FS_FAMILY_LMBTR;
  const bool acsf_std = ml && m->n_tables == 1 + 2 * m->ntypes;
  if (expected_tables(m->family, m->ntypes) != m->n_tables && !acsf_std) return FS_ERR_ARG;
  State &S = h->S;
  S.family = m->family;
  S.ntypes = m->ntypes;
  S.tables.assign(m->n_tables, Table{});
  for (int t = 0; t < m->n_tables; ++t) {
    const fs_table &ft = m->tables[t];
    if (ft.n < 1 || !ft.values) return FS_ERR_ARG;
    if (ft.kind == FS_TABLE_SPLINE && (ft.n < 2 || !(ft.rmax > ft.rmin))) return FS_ERR_ARG;
    if (ft.kind == FS_TABLE_ANALYTIC && form_nparams(ft.form) != ft.n) return FS_ERR_ARG;
    if ((m->family == FS_FAMILY_TERSOFF) != (ft.kind == FS_TABLE_TERSOFF)) return FS_ERR_ARG;
    if (ml) {
      const bool lm = m->family == FS_FAMILY_LMBTR;
      const int want = t == 0 ? (lm ? FS_TABLE_LMBTR : FS_TABLE_ACSF)
                              : t <= m->ntypes ? FS_TABLE_LINEAR_HEAD : FS_TABLE_STANDARDIZATION;
      if (ft.kind != want) return FS_ERR_ARG;
      if (t == 0 && !lm && acsf_values(ft.values, ft.n) != ft.n) return FS_ERR_ARG;
      if (t == 0 && lm && !lmbtr_valid(ft.values, ft.n)) return FS_ERR_ARG;
      const int Sz = t == 0 ? 0
                     : lm   ? lmbtr_size(LmbtrSpec(m->tables[0].values), m->ntypes)
                            : acsf_size(AcsfSpec(m->tables[0].values), m->ntypes);
      if (t > 0 && t <= m->ntypes && ft.n != Sz + 1) return FS_ERR_ARG;
      if (t > m->ntypes) { // standardization: 2S values, none of them free
        if (ft.n != 2 * Sz) return FS_ERR_ARG;
        for (int k = 0; k < ft.n; ++k)
          if (!ft.fixed || !ft.fixed[k]) return FS_ERR_ARG;
      }
    }
    if (ft.kind == FS_TABLE_TERSOFF && ft.n != 12) return FS_ERR_ARG;
    S.tables[t].init(ft);
  }
  // globals: pair and EAM only, links on analytic parameters; a linked
  // parameter is fixed and takes the global's value (finalize_globals)
  S.gval.assign(m->global_values, m->global_values + std::max(m->n_globals, 0));
  S.gfixed.assign(S.gval.size(), 0);
  S.links.clear();
  if (m->n_globals > 0 && S.family != FS_FAMILY_EAM && S.family != FS_FAMILY_PAIR) return FS_ERR_ARG;
  for (std::size_t g = 0; g < S.gval.size(); ++g) S.gfixed[g] = m->global_fixed && m->global_fixed[g] ? 1 : 0;
  for (int l = 0; l < m->n_links; ++l) {
    const int g = m->link_global[l], t = m->link_table[l], k = m->link_param[l];
    if (g < 0 || g >= m->n_globals || t < 0 || t >= m->n_tables) return FS_ERR_ARG;
    Table &tb = S.tables[t];
    if (tb.kind != FS_TABLE_ANALYTIC || k < 0 || k >= tb.n) return FS_ERR_ARG;
    tb.fixed[k] = 1;
    tb.lo[k] = -std::numeric_limits<double>::infinity();
    tb.hi[k] = std::numeric_limits<double>::infinity();
    S.links.push_back({g, t, k});
  }
  for (Table &tb : S.tables) {
    tb.free_idx.clear();
    for (int k = 0; k < tb.n; ++k)
      if (!tb.fixed[k]) tb.free_idx.push_back(k);
  }
  broadcast_globals(S);
  for (Table &tb : S.tables) tb.refresh();
  S.have_model = true;
  S.rcut_built = -1;
  return FS_OK;
}

int orc_prepare(orc_state *h) {
  if (!h || !h->S.have_model) return FS_ERR_STATE;
  for (const auto t : h->S.type)
    if (t < 0 || t >= h->S.ntypes) return FS_ERR_ARG; // species slot outside the model
  build_neighbors(h->S, max_cutoff(h->S));
  prime_sites(h->S);
  return FS_OK;
}

int orc_num_pairs(orc_state *h, int64_t *np) {
  if (!h || !np) return FS_ERR_ARG;
  *np = static_cast<int64_t>(h->S.nb_j.size());
  return FS_OK;
}
int orc_get_neighbor_counts(orc_state *h, int32_t *counts) {
  if (!h || !counts) return FS_ERR_ARG;
  for (int64_t i = 0; i < h->S.natoms_total; ++i)
    counts[i] = static_cast<int32_t>(h->S.nb_start[i + 1] - h->S.nb_start[i]);
  return FS_OK;
}
int orc_get_neighbors(orc_state *h, int32_t *j, int8_t *img3, double *d3) {
  if (!h) return FS_ERR_ARG;
  const State &S = h->S;
  if (j) std::copy(S.nb_j.begin(), S.nb_j.end(), j);
  if (img3) std::copy(S.nb_img.begin(), S.nb_img.end(), img3);
  if (d3)
    for (std::size_t p = 0; p < S.nb_d.size(); ++p)
      for (int k = 0; k < 3; ++k) d3[3 * p + k] = S.nb_d[p][k];
  return FS_OK;
}

int orc_param_count(orc_state *h, int32_t *D) {
  if (!h || !D) return FS_ERR_ARG;
  *D = param_count(h->S);
  return FS_OK;
}
int orc_gather_params(orc_state *h, double *x) {
  if (!h || !x) return FS_ERR_ARG;
  gather(h->S, x);
  return FS_OK;
}
int orc_gather_bounds(orc_state *h, double *lo, double *hi) {
  if (!h || !lo || !hi) return FS_ERR_ARG;
  int o = 0;
  for (const Table &t : h->S.tables)
    for (int k : t.free_idx) {
      lo[o] = t.lo[k];
      hi[o] = t.hi[k];
      ++o;
    }
  for (std::size_t g = 0; g < h->S.gval.size(); ++g) // build_globals keeps no min/max
    if (!h->S.gfixed[g]) {
      lo[o] = -std::numeric_limits<double>::infinity();
      hi[o] = std::numeric_limits<double>::infinity();
      ++o;
    }
  return FS_OK;
}
int orc_set_params(orc_state *h, const double *x, int32_t D) {
  if (!h || !x || D != param_count(h->S)) return FS_ERR_ARG;
  scatter(h->S, x);
  // with_eval_scope rebuilds the lists whenever the cutoff changes
  // (eval_scope.hpp:13-20); pairs beyond a shorter cutoff contribute zero, so
  // only a longer one needs new lists.
  if (h->S.rcut_built >= 0 && max_cutoff(h->S) > h->S.rcut_built) {
    build_neighbors(h->S, max_cutoff(h->S));
    prime_sites(h->S);
  }
  return FS_OK;
}
int orc_residual_count(orc_state *h, double w_s, int64_t *m) {
  if (!h || !m) return FS_ERR_ARG;
  *m = row_offsets(h->S, w_s).back();
  return FS_OK;
}

int orc_eval(orc_state *h, double w_e, double w_s, double *F, double *forces, double *energy,
             double *stress9, double *limit, double *obj) {
  if (!h) return FS_ERR_ARG;
  State &S = h->S;
  if (S.rcut_built < 0) return FS_ERR_STATE;
  const auto ro = row_offsets(S, w_s);
  std::vector<double> Fl(F ? 0 : ro.back());
  double *Fp = F ? F : Fl.data();
  std::vector<Out> outs;
  residual(S, w_e, w_s, Fp, ro, &outs);
  for (std::size_t c = 0; c < S.cfgs.size(); ++c) {
    const Config &cf = S.cfgs[c];
    if (forces)
      for (int i = 0; i < cf.natoms; ++i)
        for (int a = 0; a < 3; ++a) forces[3 * (cf.atom0 + i) + a] = outs[c].force[i][a];
    if (energy) energy[c] = outs[c].energy;
    if (limit) limit[c] = outs[c].limit;
    if (stress9)
      for (int r = 0; r < 3; ++r)
        for (int k = 0; k < 3; ++k) stress9[9 * c + 3 * r + k] = outs[c].stress[r][k];
  }
  if (obj) {
    double s = 0.0;
    for (int64_t r = 0; r < ro.back(); ++r) s += Fp[r] * Fp[r];
    *obj = s;
  }
  return FS_OK;
}

// opt::fd_jacobian (include/forcesmith/optimization/fd_jacobian.hpp:37-49):
// central differences, h = 1e-5, x restored by the same add/subtract
// sequence.  Columns [c0, c1) only (c1 < 0: all) so that a bounded sample can
// be timed; J is column-major m × D.
int orc_eval_jacobian_fd(orc_state *h, double w_e, double w_s, double *J, int32_t c0, int32_t c1) {
  if (!h || !J) return FS_ERR_ARG;
  State &S = h->S;
  if (S.rcut_built < 0) return FS_ERR_STATE;
  const int D = param_count(S);
  if (c1 < 0 || c1 > D) c1 = D;
  const auto ro = row_offsets(S, w_s);
  const int64_t m = ro.back();
  std::vector<double> x(D), xp, fp(m), fm(m);
  gather(S, x.data());
  xp = x;
  const double hh = 1e-5;
  auto scatter_fit = [&](const double *xx) {
    scatter(S, xx);
    if (max_cutoff(S) > S.rcut_built) {
      build_neighbors(S, max_cutoff(S));
      prime_sites(S);
    }
  };
  for (int j = c0; j < c1; ++j) {
    xp[j] += hh;
    scatter_fit(xp.data());
    residual(S, w_e, w_s, fp.data(), ro);
    xp[j] -= 2.0 * hh;
    scatter_fit(xp.data());
    residual(S, w_e, w_s, fm.data(), ro);
    xp[j] += hh;
    double *col = J + static_cast<int64_t>(j) * m;
    for (int64_t r = 0; r < m; ++r) col[r] = (fp[r] - fm[r]) / (2.0 * hh);
  }
  scatter(S, x.data());
  return FS_OK;
}

// Analytic Jacobian restatement (EAM, Pair).  J column-major m × D.
int orc_eval_jacobian_analytic(orc_state *h, double w_e, double w_s, double *J) {
  if (!h || !J) return FS_ERR_ARG;
  State &S = h->S;
  if (S.rcut_built < 0) return FS_ERR_STATE;
  if (S.family != FS_FAMILY_EAM && S.family != FS_FAMILY_PAIR) return FS_ERR_UNSUPPORTED;
  for (uint8_t f : S.gfixed) // analytic_jacobian_available (param_jacobian.hpp:44-57)
    if (!f) return FS_ERR_UNSUPPORTED;
  const auto ro = row_offsets(S, w_s);
  const int64_t m = ro.back();
  const int D = param_count(S);
  std::fill(J, J + m * D, 0.0);
  const auto col = table_cols(S);
#pragma omp parallel for schedule(dynamic)
  for (int c = 0; c < static_cast<int>(S.cfgs.size()); ++c) {
    if (S.family == FS_FAMILY_EAM)
      jacobian_eam_config(S, c, w_e, w_s, J, m, ro[c], col);
    else
      jacobian_pair_config(S, c, w_e, w_s, J, m, ro[c], col);
  }
  return FS_OK;
}

// Batched objective ‖F(x_k)‖² (BoostDESolver's cost, solver.cpp:143-146).
int orc_eval_population(orc_state *h, double w_e, double w_s, const double *xs, int32_t NP,
                        double *obj) {
  if (!h || !xs || !obj) return FS_ERR_ARG;
  State &S = h->S;
  const int D = param_count(S);
  const auto ro = row_offsets(S, w_s);
  std::vector<double> x0(D), F(ro.back());
  gather(S, x0.data());
  for (int k = 0; k < NP; ++k) {
    scatter(S, xs + static_cast<int64_t>(k) * D);
    residual(S, w_e, w_s, F.data(), ro);
    double s = 0.0;
    for (double v : F) s += v * v;
    obj[k] = s;
  }
  scatter(S, x0.data());
  return FS_OK;
}

// Descriptor values of atom i of configuration c (ACSF or LMBTR models).
int orc_descriptor(orc_state *h, int32_t c, int32_t i, double *D) {
  if (!h || !D) return FS_ERR_ARG;
  State &S = h->S;
  if (!S.have_model || S.rcut_built < 0) return FS_ERR_STATE;
  if (c < 0 || c >= static_cast<int>(S.cfgs.size()) || i < 0 || i >= S.cfgs[c].natoms) return FS_ERR_ARG;
  if (S.family == FS_FAMILY_LMBTR)
    lmbtr_values_of(S, c, i, D);
  else if (S.family == FS_FAMILY_ACSF)
    acsf_values_of(S, c, i, D);
  else
    return FS_ERR_STATE;
  return FS_OK;
}

// JᵀJ and Jᵀr from a column-major J (FP64).
int orc_acsf_standardization(orc_state *h, double *mean, double *inv_std, int64_t *count) {
  if (!h || !mean || !inv_std || !count) return FS_ERR_ARG;
  State &S = h->S;
  const bool lm = S.family == FS_FAMILY_LMBTR;
  if (!S.have_model || (S.family != FS_FAMILY_ACSF && !lm) || S.rcut_built < 0) return FS_ERR_STATE;
  const int nt = S.ntypes;
  const int Sz = lm ? lmbtr_size(LmbtrSpec(S.tables[0].v.data()), nt) : acsf_size(AcsfSpec(S.tables[0].v.data()), nt);
  // MLBase::compute_standardization (ml_force.hpp:644-688), atoms in order
  std::vector<double> sum(static_cast<size_t>(nt) * Sz, 0.0), sq(sum.size(), 0.0), D(Sz);
  std::vector<int64_t> n(nt, 0);
  for (int c = 0; c < static_cast<int>(S.cfgs.size()); ++c)
    for (int i = 0; i < S.cfgs[c].natoms; ++i) {
      if (lm)
        lmbtr_values_of(S, c, i, D.data());
      else
        acsf_values_of(S, c, i, D.data());
      const int t = S.type[S.cfgs[c].atom0 + i];
      for (int k = 0; k < Sz; ++k) {
        sum[static_cast<size_t>(t) * Sz + k] += D[k];
        sq[static_cast<size_t>(t) * Sz + k] += D[k] * D[k];
      }
      ++n[t];
    }
  for (int t = 0; t < nt; ++t) {
    count[t] = n[t];
    for (int k = 0; k < Sz; ++k) {
      const size_t q = static_cast<size_t>(t) * Sz + k;
      if (n[t] == 0) {
        mean[q] = 0.0;
        inv_std[q] = 1.0;
        continue;
      }
      const double mu = sum[q] / static_cast<double>(n[t]);
      const double var = sq[q] / static_cast<double>(n[t]) - mu * mu;
      mean[q] = mu;
      inv_std[q] = var > 1e-12 ? 1.0 / std::sqrt(var) : 0.0;
    }
  }
  return FS_OK;
}

int orc_normal_equations(const double *J, const double *F, int64_t m, int32_t D, double *JtJ,
                         double *Jtr) {
  if (!J || !F) return FS_ERR_ARG;
#pragma omp parallel for schedule(dynamic)
  for (int a = 0; a < D; ++a) {
    const double *ca = J + static_cast<int64_t>(a) * m;
    if (Jtr) {
      double s = 0.0;
      for (int64_t r = 0; r < m; ++r) s += ca[r] * F[r];
      Jtr[a] = s;
    }
    if (JtJ)
      for (int b = 0; b <= a; ++b) {
        const double *cb = J + static_cast<int64_t>(b) * m;
        double s = 0.0;
        for (int64_t r = 0; r < m; ++r) s += ca[r] * cb[r];
        JtJ[a * D + b] = JtJ[b * D + a] = s;
      }
  }
  return FS_OK;
}

// Damped normal-equation step (JᵀJ + λ·diag) dx = −Jᵀr, FP64 Cholesky.
int orc_lm_step(const double *JtJ, const double *Jtr, int32_t D, double lambda, int32_t mode,
                double *dx) {
  std::vector<double> A(JtJ, JtJ + static_cast<int64_t>(D) * D);
  // Marquardt scaling by diag(JᵀJ), with 1 where a column is zero (MINPACK's rule)
  for (int i = 0; i < D; ++i) {
    const double dii = JtJ[i * D + i];
    A[i * D + i] += lambda * (mode == 1 ? (dii > 0.0 ? dii : 1.0) : 1.0);
  }
  if (!cholesky(A, D)) return FS_ERR_NUMERIC;
  for (int i = 0; i < D; ++i) dx[i] = -Jtr[i];
  chol_solve(A, D, dx);
  return FS_OK;
}

// NormalEquationsSolver (src/optimization/solver.cpp:242-266):
// λ = ridge > 0 ? ridge : 1e-8·max(mean diag, 1); x −= (AᵀA + λI)⁻¹ Aᵀb.
int orc_lsq_step(const double *JtJ, const double *Jtr, int32_t D, double ridge, double *dx) {
  double lambda = ridge;
  if (lambda <= 0.0) {
    double mean = 0.0;
    for (int i = 0; i < D; ++i) mean += JtJ[i * D + i];
    mean /= D;
    lambda = 1e-8 * std::max(mean, 1.0);
  }
  return orc_lm_step(JtJ, Jtr, D, lambda, 0, dx);
}

// Unit-level probes used by the pin tests.
int orc_spline_eval(const double *x, const double *y, int32_t n, double r, double *out6) {
  if (!x || !y || n < 2 || !out6) return FS_ERR_ARG;
  Spline sp(std::vector<double>(x, x + n), std::vector<double>(y, y + n));
  const Site st = prepare_site(sp, r);
  out6[0] = sp.eval(r);
  out6[1] = sp.deriv(r);
  out6[2] = eval_at(sp, st);
  out6[3] = deriv_at(sp, st);
  out6[4] = sp.deriv2(r);
  out6[5] = static_cast<double>(st.i);
  return FS_OK;
}
int orc_spline_slopes(const double *x, const double *y, int32_t n, double *s) {
  if (!x || !y || n < 2 || !s) return FS_ERR_ARG;
  Spline sp(std::vector<double>(x, x + n), std::vector<double>(y, y + n));
  for (int k = 0; k < n; ++k) s[k] = sp.s.empty() ? 0.0 : sp.s[k];
  return FS_OK;
}
int orc_spline_grad(const double *x, const double *y, int32_t n, double r, double *gv, double *gd,
                    double *gdd) {
  if (!x || !y || n < 2) return FS_ERR_ARG;
  Spline sp(std::vector<double>(x, x + n), std::vector<double>(y, y + n));
  const auto dS = slope_jacobian(sp);
  spline_param_grad(sp, dS, r, gv, gd, gdd);
  return FS_OK;
}
int orc_form_eval(int32_t form, const double *params, int32_t np, double r, double *out3,
                  double *g, double *dg, double rmax) {
  if (form_nparams(form) != np || !params || !out3) return FS_ERR_ARG;
  FormEval f = form_eval(form, params, np, r, g || dg, rmax);
  out3[0] = f.v;
  out3[1] = f.d;
  out3[2] = f.d2;
  for (int k = 0; k < np; ++k) {
    if (g) g[k] = f.g[k];
    if (dg) dg[k] = f.dg[k];
  }
  return FS_OK;
}
int orc_pbc(const double *box9, const double *r3, double *wrapped3, double *volume,
            double *inv9) {
  Mat3 b;
  for (int r = 0; r < 3; ++r)
    for (int k = 0; k < 3; ++k) b(r, k) = box9[3 * r + k];
  PBC p;
  p.set(b);
  if (wrapped3 && r3) {
    const Vec3 w = p.wrap({r3[0], r3[1], r3[2]});
    for (int k = 0; k < 3; ++k) wrapped3[k] = w[k];
  }
  if (volume) *volume = p.volume;
  if (inv9)
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) inv9[3 * r + k] = p.inv(r, k);
  return FS_OK;
}

} // extern "C"
