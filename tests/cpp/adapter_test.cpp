// Drives forcesmith_gpu_adapter.hpp the way Forcesmith's functor and solvers
// drive a force calculator (src/optimization/forcesmith_functor.cpp:35-57,
// 111-132): prepare() once, then eval_forces(cfg, c) and
// eval_cached_jacobian(c, …) from several threads at once, one configuration
// per call, then a GpuLMSolver fit and a GpuDESolver run.  Reads a case written by
// tests/test_gpu_cpp_adapter.py and writes what it computed for the test to
// check against the oracle.
//
//   adapter_test <case.bin> <out.bin>
//
// case.bin (little-endian): int32 n_cfg, family, ntypes, n_tables, precision,
// threads, lm_iters, de_generations; per configuration int32 natoms, 9 doubles box (row-major,
// columns = lattice vectors), per atom int32 type + 3 doubles position + 3
// doubles reference force, double reference energy, 9 doubles reference
// stress; per table int32 kind, form, n, doubles rmin, rmax, n values; doubles
// w_e, w_s; int32 D; D doubles x (the evaluation point).
// out.bin: doubles forces (3 per atom), energy, stress9 and limit per
// configuration; the M × D column-major J; the forces, energy and stress9 of
// configuration 0 evaluated on its own; then int32 status, iterations,
// n_history, doubles history, D doubles x after the fit; then the DE run's
// best objective and its D doubles x.
#include "forcesmith_gpu_adapter.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <thread>

using namespace forcesmith;

namespace {

struct Reader {
  std::ifstream f;
  explicit Reader(const char *path) : f(path, std::ios::binary) {
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
  }
  template <class T> T get() {
    T v{};
    f.read(reinterpret_cast<char *>(&v), sizeof v);
    if (!f) throw std::runtime_error("case file truncated");
    return v;
  }
};

struct Writer {
  std::ofstream f;
  explicit Writer(const char *path) : f(path, std::ios::binary) {}
  template <class T> void put(T v) { f.write(reinterpret_cast<const char *>(&v), sizeof v); }
};

} // namespace

int main(int argc, char **argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s case.bin out.bin\n", argv[0]);
    return 2;
  }
  try {
    Reader in(argv[1]);
    const int n_cfg = in.get<int32_t>(), family = in.get<int32_t>(), ntypes = in.get<int32_t>();
    const int n_tables = in.get<int32_t>(), precision = in.get<int32_t>(), threads = in.get<int32_t>();
    const int lm_iters = in.get<int32_t>(), de_generations = in.get<int32_t>();
    std::vector<Configuration> cfgs(n_cfg);
    for (Configuration &cfg : cfgs) {
      const int n = in.get<int32_t>();
      Mat3 box;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) box(a, b) = in.get<double>();
      cfg.bc = PeriodicBC(box);
      cfg.atoms.resize(n);
      for (Atom &at : cfg.atoms) {
        at.type = Species(static_cast<std::size_t>(in.get<int32_t>()));
        for (int a = 0; a < 3; ++a) at.pos[a] = in.get<double>();
        for (int a = 0; a < 3; ++a) at.ref.force[a] = in.get<double>();
      }
      cfg.ref.energy = in.get<double>();
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) cfg.ref.stress(a, b) = in.get<double>();
    }
    GpuModel model;
    model.family = family;
    model.ntypes = ntypes;
    for (int t = 0; t < n_tables; ++t) {
      GpuTable tb;
      tb.kind = in.get<int32_t>();
      tb.form = in.get<int32_t>();
      const int n = in.get<int32_t>();
      tb.rmin = in.get<double>();
      tb.rmax = in.get<double>();
      for (int k = 0; k < n; ++k) tb.values.push_back(in.get<double>());
      model.tables.push_back(std::move(tb));
    }
    const double w_e = in.get<double>(), w_s = in.get<double>();
    const int D = in.get<int32_t>();
    VectorXd x(D);
    for (int k = 0; k < D; ++k) x[k] = in.get<double>();

    GpuOptions opt;
    opt.precision = precision;
    opt.w_e = w_e;
    opt.w_s = w_s;
    GpuForceCalculator proto(model, opt);
    if (static_cast<int>(proto.param_count()) != D) throw std::runtime_error("parameter count mismatch");
    proto.prepare(std::span<Configuration>(cfgs));
    GpuForceCalculator calc = proto; // the functor works on a copy of the model
    calc.scatter_params(x, 0);

    // eval_forces(cfg, c), concurrently, one configuration per call
    {
      std::vector<std::thread> pool;
      for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
          for (int c = t; c < n_cfg; c += threads) calc.eval_forces(cfgs[c], static_cast<std::size_t>(c));
        });
      for (std::thread &th : pool) th.join();
    }
    // eval_cached_jacobian(c, row0, col_off, …), concurrently
    std::vector<int> row0(n_cfg + 1, 0);
    for (int c = 0; c < n_cfg; ++c)
      row0[c + 1] = row0[c] + 3 * static_cast<int>(cfgs[c].atoms.size()) + 2 + (w_s > 0.0 ? 6 : 0);
    MatrixXd fjac(row0[n_cfg], D);
    const std::vector<int> col_off{0, D};
    {
      std::vector<std::thread> pool;
      for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
          for (int c = t; c < n_cfg; c += threads)
            calc.eval_cached_jacobian(static_cast<std::size_t>(c), row0[c], col_off, w_e, w_s, fjac);
        });
      for (std::thread &th : pool) th.join();
    }
    Configuration solo = cfgs[0];
    calc.eval_forces(solo);

    Writer out(argv[2]);
    for (const Configuration &cfg : cfgs)
      for (const Atom &at : cfg.atoms)
        for (int a = 0; a < 3; ++a) out.put<double>(at.calc_force[a]);
    for (const Configuration &cfg : cfgs) {
      out.put<double>(cfg.calc_energy);
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) out.put<double>(cfg.calc_stress(a, b));
      out.put<double>(cfg.calc_limit);
    }
    for (std::ptrdiff_t k = 0; k < fjac.rows() * fjac.cols(); ++k) out.put<double>(fjac.data()[k]);
    for (const Atom &at : solo.atoms)
      for (int a = 0; a < 3; ++a) out.put<double>(at.calc_force[a]);
    out.put<double>(solo.calc_energy);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) out.put<double>(solo.calc_stress(a, b));

    // a device LM fit from x
    GpuLMSolver lm;
    lm.calc = &calc;
    lm.max_iter = lm_iters;
    lm.w_e = w_e;
    lm.w_s = w_s;
    VectorXd xfit = x, none;
    const int status = lm.minimize(xfit, nullptr, nullptr, static_cast<int>(fjac.rows()), none, none);
    out.put<int32_t>(status);
    out.put<int32_t>(lm.iterations);
    out.put<int32_t>(static_cast<int32_t>(lm.objective_history.size()));
    for (double o : lm.objective_history) out.put<double>(o);
    for (int k = 0; k < D; ++k) out.put<double>(xfit[k]);

    // a device DE run from x (NP = 15·D, seed 42, no bounds: the box rule)
    GpuDESolver de;
    de.calc = &calc;
    de.max_generations = de_generations;
    de.w_e = w_e;
    de.w_s = w_s;
    VectorXd xde = x;
    de.minimize(xde, nullptr, nullptr, static_cast<int>(fjac.rows()), none, none);
    out.put<double>(de.best_objective);
    for (int k = 0; k < D; ++k) out.put<double>(xde[k]);
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "adapter_test: %s\n", e.what());
    return 1;
  }
}
