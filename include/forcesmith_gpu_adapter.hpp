// forcesmith_gpu_adapter.hpp — Forcesmith's extension points implemented on
// the B200 library (forcesmith_gpu.h): a force calculator the reference's
// ForceCalculator accepts, and solvers that satisfy its CSolver.
//
//   GpuForceCalculator  CForceCalculator + the cache hooks of the erased
//                       ForceCalculator (include/forcesmith/force/
//                       force_calculator_concept.hpp:286-304,
//                       force_calculator.hpp:62-159)
//   GpuLMSolver         CSolver (include/forcesmith/optimization/solver.hpp:13-26)
//                       in place of EigenLMSolver (src/optimization/solver.cpp:67-85)
//   GpuDESolver         CSolver in place of BoostDESolver (solver.cpp:113-155)
//
// How the reference drives a calculator, and how this one answers:
//   - models are copied by value (forcesmith_functor.cpp:116,178): every copy
//     shares one device context through a shared_ptr and keeps its own
//     parameter vector (scatter_params);
//   - prepare(configs) runs once, single-threaded (forcesmith_functor.cpp:217):
//     one SoA upload of every configuration; neighbour lists are built on
//     the device;
//   - eval_forces(cfg, c) is called concurrently from TBB workers, one
//     configuration each (forcesmith_functor.cpp:43-51): the first call after
//     a parameter change evaluates the whole batch in one launch, under the
//     shared mutex; every call then copies its configuration's slice;
//   - with has_cache() and has_param_jacobian() true the functor asks for J
//     one configuration at a time (df_cached_analytic,
//     forcesmith_functor.cpp:111-132): the first call evaluates residual +
//     Jacobian on the device, and each call copies its configuration's row
//     block into the column-major fjac (fs_gpu_copy_jacobian_rows).
//
// Inside the Forcesmith tree, define FORCESMITH_GPU_ADAPTER_USE_REFERENCE_HEADERS
// and include the reference's headers first; otherwise forcesmith_shim.hpp
// restates the few types used here.
#pragma once

#ifndef FORCESMITH_GPU_ADAPTER_USE_REFERENCE_HEADERS
#include "forcesmith_shim.hpp"
#endif
#include "forcesmith_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <memory>
#include <mutex>
#include <span>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>
#include <vector>

namespace forcesmith {

// A device call that failed, with the library's message.
class GpuError : public std::runtime_error {
public:
  int status;
  GpuError(int code, const std::string &what) : std::runtime_error(what), status(code) {}
};

inline void gpu_check(fs_gpu *h, int rc, const char *what) {
  if (rc == FS_OK) return;
  char buf[512] = {0};
  if (h) fs_gpu_last_error(h, buf, sizeof buf);
  throw GpuError(rc, std::string(what) + ": status " + std::to_string(rc) + ": " + buf);
}

// A table of a model, owned (the fs_table of the ABI only points).
struct GpuTable {
  int kind = FS_TABLE_SPLINE, form = 0;
  double rmin = 0.0, rmax = 0.0;
  std::vector<double> values;
  std::vector<uint8_t> fixed;       // empty: every value free
  std::vector<double> lower, upper; // empty: unbounded
};

// A global parameter (GlobalParam, force_calculator_concept.hpp:21-44): its
// value, fixed flag and links (table in model order, parameter slot).  Pair
// and EAM models only; a free global's column follows the tables' columns.
struct GpuGlobal {
  double value = 0.0;
  bool fixed = false;
  std::vector<std::pair<int, int>> links;
};

// A model in the reference's gather order (force_calculator_concept.hpp:171-284).
struct GpuModel {
  int family = FS_FAMILY_EAM;
  int ntypes = 1;
  std::vector<GpuTable> tables;
  std::vector<GpuGlobal> globals;
};

namespace gpu_detail {

// The ABI view of a model (pointers into `m`, valid while `m` lives).
struct ModelView {
  std::vector<fs_table> t;
  std::vector<double> gv;
  std::vector<uint8_t> gf;
  std::vector<int32_t> lg, lt, lp;
  fs_model m{};
  explicit ModelView(const GpuModel &g) : t(g.tables.size()) {
    for (std::size_t k = 0; k < g.globals.size(); ++k) {
      gv.push_back(g.globals[k].value);
      gf.push_back(g.globals[k].fixed ? 1 : 0);
      for (const auto &[tab, slot] : g.globals[k].links) {
        lg.push_back(static_cast<int32_t>(k));
        lt.push_back(tab);
        lp.push_back(slot);
      }
    }
    for (std::size_t k = 0; k < g.tables.size(); ++k) {
      const GpuTable &s = g.tables[k];
      fs_table &d = t[k];
      d.kind = s.kind;
      d.form = s.form;
      d.n = static_cast<int32_t>(s.values.size());
      d.reserved = 0;
      d.rmin = s.rmin;
      d.rmax = s.rmax;
      d.values = s.values.data();
      d.fixed = s.fixed.empty() ? nullptr : s.fixed.data();
      d.lower = s.lower.empty() ? nullptr : s.lower.data();
      d.upper = s.upper.empty() ? nullptr : s.upper.data();
    }
    m.family = g.family;
    m.ntypes = g.ntypes;
    m.n_tables = static_cast<int32_t>(t.size());
    m.reserved = 0;
    m.tables = t.data();
    m.n_globals = static_cast<int32_t>(gv.size());
    m.n_links = static_cast<int32_t>(lg.size());
    m.global_values = gv.empty() ? nullptr : gv.data();
    m.global_fixed = gf.empty() ? nullptr : gf.data();
    m.link_global = lg.empty() ? nullptr : lg.data();
    m.link_table = lt.empty() ? nullptr : lt.data();
    m.link_param = lp.empty() ? nullptr : lp.data();
  }
};

// SoA arrays of configurations as fs_gpu_upload_configs takes them.
struct Batch {
  std::vector<int32_t> natoms, type;
  std::vector<double> box9, pos, ref_force, ref_energy, ref_stress9;
  template <class Cfgs> explicit Batch(const Cfgs &cfgs) {
    for (const Configuration &cfg : cfgs) {
      const auto *pbc = std::get_if<PeriodicBC>(&cfg.bc);
      if (!pbc) throw GpuError(FS_ERR_UNSUPPORTED, "GpuForceCalculator: periodic configurations only");
      natoms.push_back(static_cast<int32_t>(cfg.atoms.size()));
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) box9.push_back(pbc->box()(a, b));
      for (const Atom &at : cfg.atoms) {
        for (int a = 0; a < 3; ++a) pos.push_back(at.pos[a]);
        for (int a = 0; a < 3; ++a) ref_force.push_back(at.ref.force[a]);
        type.push_back(static_cast<int32_t>(static_cast<std::size_t>(at.type)));
      }
      ref_energy.push_back(cfg.ref.energy);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) ref_stress9.push_back(cfg.ref.stress(a, b));
    }
  }
  int upload(fs_gpu *h) const {
    return fs_gpu_upload_configs(h, static_cast<int32_t>(natoms.size()), natoms.data(), box9.data(), pos.data(),
                                 type.data(), ref_force.data(), ref_energy.data(), ref_stress9.data());
  }
};

} // namespace gpu_detail

// Device, precision and residual weights of a GpuForceCalculator.
struct GpuOptions {
  int device = 0;
  int precision = FS_PREC_FP32; // FS_PREC_FP32: FP32 compute, FP64 sums
  double w_e = 1.0, w_s = 0.0;  // weights of fs_gpu_eval's residual rows
};

// The force calculator.  Copies share the device context; each copy keeps
// the parameter vector its scatter_params last set.
class GpuForceCalculator {
public:
  using Options = GpuOptions;

  std::size_t ntypes = 1;

  explicit GpuForceCalculator(GpuModel model, Options opt = Options()) : s_(std::make_shared<Shared>()) {
    s_->opt = opt;
    s_->model = std::move(model);
    ntypes = static_cast<std::size_t>(s_->model.ntypes);
    s_->h = create(opt);
    const gpu_detail::ModelView v(s_->model);
    gpu_check(s_->h, fs_gpu_set_model(s_->h, &v.m), "fs_gpu_set_model");
    int32_t D = 0;
    gpu_check(s_->h, fs_gpu_param_count(s_->h, &D), "fs_gpu_param_count");
    x_.resize(static_cast<std::size_t>(D));
    gpu_check(s_->h, fs_gpu_gather_params(s_->h, x_.data()), "fs_gpu_gather_params");
  }

  // ---- CFittable (core/fit_params.hpp) -------------------------------------
  std::size_t param_count() const { return x_.size(); }
  void gather_params(VectorXd &v, std::size_t off) const {
    std::copy(x_.begin(), x_.end(), v.data() + off);
  }
  void scatter_params(const VectorXd &v, std::size_t off) {
    std::copy(v.data() + off, v.data() + off + x_.size(), x_.begin());
  }
  void gather_bounds(VectorXd &lo, VectorXd &hi, std::size_t off) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    gpu_check(s_->h, fs_gpu_gather_bounds(s_->h, lo.data() + off, hi.data() + off), "fs_gpu_gather_bounds");
  }

  // ---- CForceCalculator -----------------------------------------------------
  double max_cutoff() const {
    std::lock_guard<std::mutex> lock(s_->mu);
    double rc = 0.0;
    gpu_check(s_->h, fs_gpu_max_cutoff(s_->h, &rc), "fs_gpu_max_cutoff");
    return rc;
  }

  // Every configuration the functor will evaluate, in order; the cache index
  // c of eval_forces(cfg, c) and eval_cached_jacobian(c, …) is the position.
  void prepare(std::span<Configuration> cfgs) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    const gpu_detail::Batch b(cfgs);
    gpu_check(s_->h, b.upload(s_->h), "fs_gpu_upload_configs");
    gpu_check(s_->h, fs_gpu_prepare(s_->h), "fs_gpu_prepare");
    s_->natoms = b.natoms;
    s_->atom0.assign(b.natoms.size() + 1, 0);
    for (std::size_t c = 0; c < b.natoms.size(); ++c) s_->atom0[c + 1] = s_->atom0[c] + b.natoms[c];
    const std::size_t n = static_cast<std::size_t>(s_->atom0.back());
    s_->forces.assign(3 * n, 0.0);
    s_->energy.assign(b.natoms.size(), 0.0);
    s_->stress9.assign(9 * b.natoms.size(), 0.0);
    s_->limit.assign(b.natoms.size(), 0.0);
    s_->have_eval = s_->have_jac = false;
  }

  // Configuration c of prepare()'s span: the batch at this copy's parameters
  // (evaluated by the first call after they change), then c's slice.
  void eval_forces(Configuration &cfg, std::size_t c) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    ensure_batch();
    if (c >= s_->natoms.size() || cfg.atoms.size() != static_cast<std::size_t>(s_->natoms[c]))
      throw GpuError(FS_ERR_ARG, "GpuForceCalculator::eval_forces: configuration " + std::to_string(c) +
                                     " does not match prepare()'s");
    const int64_t a0 = s_->atom0[c];
    for (std::size_t i = 0; i < cfg.atoms.size(); ++i)
      for (int a = 0; a < 3; ++a) cfg.atoms[i].calc_force[a] = s_->forces[3 * (a0 + i) + a];
    cfg.calc_energy = s_->energy[c];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) cfg.calc_stress(a, b) = s_->stress9[9 * c + 3 * a + b]; // already / V
    cfg.calc_limit = s_->limit[c];
  }

  // A configuration on its own (force::evaluate, src/force/evaluate.cpp:5-20):
  // a second context of the same device holds just this configuration.
  void eval_forces(Configuration &cfg) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    if (!s_->solo) {
      s_->solo = create(s_->opt);
      const gpu_detail::ModelView v(s_->model);
      gpu_check(s_->solo, fs_gpu_set_model(s_->solo, &v.m), "fs_gpu_set_model");
    }
    const std::vector<Configuration> one{cfg};
    const gpu_detail::Batch b(one);
    fs_gpu *h = s_->solo;
    gpu_check(h, b.upload(h), "fs_gpu_upload_configs");
    gpu_check(h, fs_gpu_set_params(h, x_.data(), static_cast<int32_t>(x_.size())), "fs_gpu_set_params");
    gpu_check(h, fs_gpu_prepare(h), "fs_gpu_prepare");
    std::vector<double> f(3 * cfg.atoms.size()), s9(9);
    double e = 0.0, lim = 0.0;
    gpu_check(h, fs_gpu_eval(h, s_->opt.w_e, s_->opt.w_s, nullptr, f.data(), &e, s9.data(), &lim, nullptr),
              "fs_gpu_eval");
    for (std::size_t i = 0; i < cfg.atoms.size(); ++i)
      for (int a = 0; a < 3; ++a) cfg.atoms[i].calc_force[a] = f[3 * i + a];
    cfg.calc_energy = e;
    for (int a = 0; a < 3; ++a)
      for (int k = 0; k < 3; ++k) cfg.calc_stress(a, k) = s9[3 * a + k];
    cfg.calc_limit = lim;
  }

  // ---- the cache hooks of the erased ForceCalculator ----------------------
  bool has_cache() const { return true; }
  bool has_param_jacobian() const { return true; }
  bool has_standardization() const { return false; }
  std::vector<std::size_t> head_param_counts() const { return {x_.size()}; }

  void eval_cached(std::size_t c, std::span<Vec3> forces, double &energy, SymTens &stress) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    ensure_batch();
    const int64_t a0 = s_->atom0[c];
    for (std::size_t i = 0; i < forces.size(); ++i)
      for (int a = 0; a < 3; ++a) forces[i][a] = s_->forces[3 * (a0 + i) + a];
    energy = s_->energy[c];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) stress(a, b) = s_->stress9[9 * c + 3 * a + b];
  }

  // Configuration c's rows of ∂(residual)/∂x into fjac rows [row0, …) and
  // columns [col_off[0], …): the rows write_config_residuals lays out
  // (3N forces, energy, 6 stress if w_s > 0, limit; residual_layout.hpp:37-54).
  void eval_cached_jacobian(std::size_t c, int row0, const std::vector<int> &col_off, double w_e, double w_s,
                            MatrixXd &fjac) const {
    std::lock_guard<std::mutex> lock(s_->mu);
    ensure_jacobian(w_e, w_s);
    const int64_t extra = 2 + (w_s > 0.0 ? 6 : 0);
    const int64_t dev_row0 = 3 * s_->atom0[c] + static_cast<int64_t>(c) * extra;
    const int64_t rows = 3 * static_cast<int64_t>(s_->natoms[c]) + extra;
    const int64_t col0 = col_off.empty() ? 0 : col_off[0];
    if (row0 < 0 || row0 + rows > fjac.rows() || col0 + static_cast<int64_t>(x_.size()) > fjac.cols())
      throw GpuError(FS_ERR_ARG, "GpuForceCalculator::eval_cached_jacobian: block outside fjac");
    gpu_check(s_->h,
              fs_gpu_copy_jacobian_rows(s_->h, dev_row0, rows, fjac.data() + row0 + col0 * fjac.rows(), fjac.rows()),
              "fs_gpu_copy_jacobian_rows");
  }

  // The device context of every copy, for device-native solvers.
  fs_gpu *handle() const { return s_->h; }
  std::mutex &mutex() const { return s_->mu; }
  const std::vector<double> &params() const { return x_; }

private:
  struct Shared {
    fs_gpu *h = nullptr, *solo = nullptr;
    Options opt;
    GpuModel model;
    std::mutex mu;
    std::vector<int32_t> natoms;
    std::vector<int64_t> atom0;
    std::vector<double> x_eval, forces, energy, stress9, limit;
    bool have_eval = false;
    std::vector<double> x_jac;
    double we_jac = 0.0, ws_jac = -1.0;
    bool have_jac = false;
    ~Shared() {
      if (solo) fs_gpu_destroy(solo);
      if (h) fs_gpu_destroy(h);
    }
  };
  std::shared_ptr<Shared> s_;
  std::vector<double> x_;

  static fs_gpu *create(const Options &o) {
    fs_gpu_opts fo{o.device, o.precision, 0, 0};
    fs_gpu *h = nullptr;
    gpu_check(nullptr, fs_gpu_create(&fo, &h), "fs_gpu_create");
    return h;
  }
  void set_params_locked() const {
    gpu_check(s_->h, fs_gpu_set_params(s_->h, x_.data(), static_cast<int32_t>(x_.size())), "fs_gpu_set_params");
  }
  void ensure_batch() const {
    if (s_->have_eval && s_->x_eval == x_) return;
    set_params_locked();
    gpu_check(s_->h,
              fs_gpu_eval(s_->h, s_->opt.w_e, s_->opt.w_s, nullptr, s_->forces.data(), s_->energy.data(),
                          s_->stress9.data(), s_->limit.data(), nullptr),
              "fs_gpu_eval");
    s_->x_eval = x_;
    s_->have_eval = true;
  }
  void ensure_jacobian(double w_e, double w_s) const {
    if (s_->have_jac && s_->x_jac == x_ && s_->we_jac == w_e && s_->ws_jac == w_s) return;
    set_params_locked();
    gpu_check(s_->h, fs_gpu_eval_jacobian_async(s_->h, w_e, w_s), "fs_gpu_eval_jacobian_async");
    s_->x_jac = x_;
    s_->we_jac = w_e;
    s_->ws_jac = w_s;
    s_->have_jac = true;
  }
};

// Levenberg–Marquardt on the device, for a GpuForceCalculator: the residual,
// J, JᵀJ and Jᵀr stay on the GPU; a step reads back D-sized vectors.  The
// arithmetic is that of forcesmith_b200/solvers.py's LMSolver: per
// iteration one residual + Jacobian evaluation, three damped FP64 Cholesky
// steps (λ·{¼, 1, 4}) whose objectives are evaluated together, the best
// step with a positive gain ratio ρ taken, λ updated by Nielsen's rule
// λ·max(⅓, 1 − (2ρ − 1)³), λ ×16 and a retry when none decreases the
// objective.  λ₀ = τ·max diag(JᵀJ).  Termination and the returned status
// follow Eigen's LevenbergMarquardt (solver.cpp:67-85): 1 relative reduction
// below ftol, 2 relative step below xtol (also returned after max_iter
// iterations, as the reference does), 3 both, 5 more than 100·max_iter + 100
// objective evaluations.  The ResidualFn / JacobianFn arguments of the
// CSolver signature are not called: the calculator bound at construction is
// the objective.
struct GpuLMSolver {
  const GpuForceCalculator *calc = nullptr;
  int max_iter = 500;
  double xtol = 1e-7, ftol = 1e-7, tau = 1e-3;
  double w_e = 1.0, w_s = 0.0;
  // filled by minimize
  mutable int iterations = 0, nfev = 0;
  mutable std::vector<double> objective_history;

  bool honors_bounds() const { return false; }
  bool one_shot() const { return false; }

  int minimize(VectorXd &xv, ResidualFn, JacobianFn, int, const VectorXd &, const VectorXd &) const {
    if (!calc) throw GpuError(FS_ERR_STATE, "GpuLMSolver: no GpuForceCalculator bound");
    std::lock_guard<std::mutex> lock(calc->mutex());
    fs_gpu *h = calc->handle();
    const int D = static_cast<int>(xv.size());
    iterations = nfev = 0;
    objective_history.clear();
    if (D == 0) return 0; // ImproperInputParameters
    std::vector<double> x(xv.data(), xv.data() + D), JtJ(static_cast<std::size_t>(D) * D), g(D);
    const int maxfev = std::max(max_iter, 1) * 100 + 100;
    const double factors[3] = {0.25, 1.0, 4.0};
    double lam = -1.0;
    int status = -1;
    for (int it = 0; it < max_iter && status < 0; ++it) {
      gpu_check(h, fs_gpu_set_params(h, x.data(), D), "fs_gpu_set_params");
      double obj = 0.0;
      gpu_check(h, fs_gpu_eval_jacobian(h, w_e, w_s, nullptr, nullptr, JtJ.data(), g.data(), &obj),
                "fs_gpu_eval_jacobian");
      ++nfev;
      if (it == 0) objective_history.push_back(obj);
      if (lam < 0.0) {
        double dmax = 1e-300;
        for (int k = 0; k < D; ++k) dmax = std::max(dmax, JtJ[static_cast<std::size_t>(k) * D + k]);
        lam = tau * dmax;
      }
      bool accepted = false;
      while (!accepted && status < 0) {
        std::vector<std::vector<double>> steps(3, std::vector<double>(D));
        std::vector<double> trials(3 * static_cast<std::size_t>(D)), objs(3);
        for (int k = 0; k < 3; ++k) {
          gpu_check(h, fs_gpu_lm_step(h, lam * factors[k], 0, steps[k].data()), "fs_gpu_lm_step");
          for (int q = 0; q < D; ++q) trials[static_cast<std::size_t>(k) * D + q] = x[q] + steps[k][q];
        }
        trial_objectives(h, trials, D, objs);
        nfev += 3;
        int best = -1;
        double best_rho = 0.0;
        for (int k = 0; k < 3; ++k) {
          const double l = lam * factors[k];
          double gs = 0.0, ss = 0.0;
          for (int q = 0; q < D; ++q) {
            gs += g[q] * steps[k][q];
            ss += steps[k][q] * steps[k][q];
          }
          const double pred = -gs + l * ss;
          const double rho = pred > 0.0 ? (obj - objs[k]) / pred : -1.0;
          if (std::isfinite(objs[k]) && rho > 0.0 && (best < 0 || objs[k] < objs[best])) {
            best = k;
            best_rho = rho;
          }
        }
        if (best >= 0) {
          accepted = true;
          const double l = lam * factors[best];
          double gs = 0.0, ss = 0.0, xx = 0.0;
          for (int q = 0; q < D; ++q) {
            gs += g[q] * steps[best][q];
            ss += steps[best][q] * steps[best][q];
            x[q] += steps[best][q];
            xx += x[q] * x[q];
          }
          const double pred = -gs + l * ss, o = objs[best];
          const double act_rel = obj > 0.0 ? (obj - o) / obj : 0.0, pred_rel = obj > 0.0 ? pred / obj : 0.0;
          obj = o;
          const double u = 2.0 * best_rho - 1.0;
          lam = l * std::max(1.0 / 3.0, 1.0 - u * u * u);
          objective_history.push_back(obj);
          const bool f_conv = std::abs(act_rel) <= ftol && pred_rel <= ftol && best_rho <= 2.0;
          const bool x_conv = std::sqrt(ss) <= xtol * std::sqrt(xx);
          if (f_conv && x_conv) status = 3;
          else if (f_conv) status = 1;
          else if (x_conv) status = 2;
        } else {
          lam *= 16.0;
          if (lam > 1e16) status = 2; // no decrease along any damped step
        }
        if (nfev >= maxfev && status < 0) status = 5;
      }
      iterations = it + 1;
    }
    if (status < 0) status = 2; // still running after max_iter: the reference returns 2
    std::copy(x.begin(), x.end(), xv.data());
    gpu_check(h, fs_gpu_set_params(h, x.data(), D), "fs_gpu_set_params");
    return status;
  }

private:
  // ‖F(x_k)‖² of each trial: one population launch where the family has one
  // (EAM / pair splines), else one residual evaluation per trial.
  void trial_objectives(fs_gpu *h, const std::vector<double> &xs, int D, std::vector<double> &objs) const {
    const int n = static_cast<int>(objs.size());
    const int rc = fs_gpu_eval_population(h, w_e, w_s, xs.data(), n, objs.data());
    if (rc == FS_OK) return;
    if (rc != FS_ERR_UNSUPPORTED) gpu_check(h, rc, "fs_gpu_eval_population");
    for (int k = 0; k < n; ++k) {
      gpu_check(h, fs_gpu_set_params(h, xs.data() + static_cast<std::size_t>(k) * D, D), "fs_gpu_set_params");
      gpu_check(h, fs_gpu_eval(h, w_e, w_s, nullptr, nullptr, nullptr, nullptr, nullptr, &objs[k]), "fs_gpu_eval");
    }
  }
};

// Differential evolution on the device (fs_gpu_de_*), for a GpuForceCalculator:
// BoostDESolver's knobs (NP = 15·D by default, F = 0.65, CR = 0.5, seed,
// max_generations) and its search box (solver.cpp:118-124): a finite bound is
// kept, an infinite one becomes x ∓ max(2|x|, 5e-4).  The result is the
// best member after max_generations; status 0.
struct GpuDESolver {
  const GpuForceCalculator *calc = nullptr;
  int NP = 0; // 0: 15·D
  double mutation = 0.65, crossover = 0.5;
  uint64_t seed = 42;
  int max_generations = 200;
  double w_e = 1.0, w_s = 0.0;
  mutable double best_objective = 0.0;

  bool honors_bounds() const { return true; }
  bool one_shot() const { return false; }

  int minimize(VectorXd &xv, ResidualFn, JacobianFn, int, const VectorXd &lower, const VectorXd &upper) const {
    if (!calc) throw GpuError(FS_ERR_STATE, "GpuDESolver: no GpuForceCalculator bound");
    std::lock_guard<std::mutex> lock(calc->mutex());
    fs_gpu *h = calc->handle();
    const int D = static_cast<int>(xv.size());
    std::vector<double> lo(D), hi(D), x(xv.data(), xv.data() + D);
    for (int k = 0; k < D; ++k) {
      const double half = std::max(2.0 * std::abs(x[k]), 5e-4);
      const double l = k < lower.size() ? lower[k] : -std::numeric_limits<double>::infinity();
      const double u = k < upper.size() ? upper[k] : std::numeric_limits<double>::infinity();
      lo[k] = std::isfinite(l) ? l : x[k] - half;
      hi[k] = std::isfinite(u) ? u : x[k] + half;
      x[k] = std::clamp(x[k], lo[k], hi[k]); // member 0 starts at the clamped guess
    }
    fs_de_opts o{};
    o.NP = NP > 0 ? NP : 15 * D;
    o.mutation = mutation;
    o.crossover = crossover;
    o.seed = seed;
    o.w_e = w_e;
    o.w_s = w_s;
    gpu_check(h, fs_gpu_de_init(h, &o, lo.data(), hi.data(), x.data()), "fs_gpu_de_init");
    gpu_check(h, fs_gpu_de_run(h, max_generations, 1, &best_objective, x.data(), nullptr), "fs_gpu_de_run");
    std::copy(x.begin(), x.end(), xv.data());
    gpu_check(h, fs_gpu_set_params(h, x.data(), D), "fs_gpu_set_params");
    return 0;
  }
};

} // namespace forcesmith
