// forcesmith_shim.hpp — the part of Forcesmith's C++ data model and extension
// points that the GPU adapter (forcesmith_gpu_adapter.hpp) touches, restated
// with the reference's names and member layout but without Eigen or Boost.
//
// The reference's own headers need Eigen 3.4, Boost and oneTBB; this header
// lets the adapter and its test program compile and run without them.  Inside
// the Forcesmith tree the adapter includes the real headers instead; every
// name it uses below exists there with the same meaning:
//
//   Vec3, Mat3, SymTens        include/forcesmith/core/types.hpp:16-18
//                              (Eigen::Vector3d / Matrix3d: operator()/[])
//   Species, Atom,             include/forcesmith/core/species.hpp:23-43,
//   Configuration              include/forcesmith/core/atom.hpp:44-100
//   PeriodicBC, InfiniteBC,    include/forcesmith/core/boundary_conditions.hpp:9-66
//   BoundaryConditions
//   ResidualFn, JacobianFn     include/forcesmith/optimization/solver.hpp:13-16
//   Eigen::VectorXd / MatrixXd column-major dense storage (data(), rows(),
//                              cols(), size())
#pragma once

#include <array>
#include <cmath>
#include <cstddef>
#include <functional>
#include <string>
#include <variant>
#include <vector>

namespace forcesmith {

// Eigen::VectorXd: a dense column of doubles.
class VectorXd {
  std::vector<double> v_;

public:
  VectorXd() = default;
  explicit VectorXd(std::ptrdiff_t n, double fill = 0.0) : v_(static_cast<std::size_t>(n), fill) {}
  double *data() { return v_.data(); }
  const double *data() const { return v_.data(); }
  std::ptrdiff_t size() const { return static_cast<std::ptrdiff_t>(v_.size()); }
  void resize(std::ptrdiff_t n) { v_.assign(static_cast<std::size_t>(n), 0.0); }
  double &operator[](std::ptrdiff_t i) { return v_[static_cast<std::size_t>(i)]; }
  double operator[](std::ptrdiff_t i) const { return v_[static_cast<std::size_t>(i)]; }
  double &operator()(std::ptrdiff_t i) { return v_[static_cast<std::size_t>(i)]; }
  double operator()(std::ptrdiff_t i) const { return v_[static_cast<std::size_t>(i)]; }
  double squaredNorm() const {
    double s = 0.0;
    for (double x : v_) s += x * x;
    return s;
  }
};

// Eigen::MatrixXd: dense, column-major (element (i, j) at data()[i + j·rows()]).
class MatrixXd {
  std::ptrdiff_t r_ = 0, c_ = 0;
  std::vector<double> v_;

public:
  MatrixXd() = default;
  MatrixXd(std::ptrdiff_t r, std::ptrdiff_t c) : r_(r), c_(c), v_(static_cast<std::size_t>(r * c), 0.0) {}
  void resize(std::ptrdiff_t r, std::ptrdiff_t c) {
    r_ = r;
    c_ = c;
    v_.assign(static_cast<std::size_t>(r * c), 0.0);
  }
  double *data() { return v_.data(); }
  const double *data() const { return v_.data(); }
  std::ptrdiff_t rows() const { return r_; }
  std::ptrdiff_t cols() const { return c_; }
  double &operator()(std::ptrdiff_t i, std::ptrdiff_t j) { return v_[static_cast<std::size_t>(i + j * r_)]; }
  double operator()(std::ptrdiff_t i, std::ptrdiff_t j) const { return v_[static_cast<std::size_t>(i + j * r_)]; }
};

// Eigen::Vector3d / Matrix3d
struct Vec3 {
  double d[3] = {0.0, 0.0, 0.0};
  double &operator[](int a) { return d[a]; }
  double operator[](int a) const { return d[a]; }
  double &operator()(int a) { return d[a]; }
  double operator()(int a) const { return d[a]; }
  static Vec3 Zero() { return Vec3{}; }
};
struct Mat3 {
  double m[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  double &operator()(int a, int b) { return m[a][b]; }
  double operator()(int a, int b) const { return m[a][b]; }
  static Mat3 Zero() { return Mat3{}; }
  static Mat3 Identity() {
    Mat3 I;
    I.m[0][0] = I.m[1][1] = I.m[2][2] = 1.0;
    return I;
  }
};
using SymTens = Mat3;

// core/species.hpp: the compact slot `index` indexes the potential tables
struct Species {
  std::string symbol;
  std::size_t Z = 0;
  double mass_amu = 0.0;
  std::size_t index = 0;
  Species() = default;
  Species(std::size_t i) : index(i) {}
  operator std::size_t() const { return index; }
};

// core/boundary_conditions.hpp: the box's COLUMNS are the lattice vectors
class PeriodicBC {
  Mat3 box_ = Mat3::Identity();

public:
  explicit PeriodicBC(const Mat3 &box) : box_(box) {}
  const Mat3 &box() const { return box_; }
};
class InfiniteBC {
  double volume_ = 1.0;

public:
  explicit InfiniteBC(double volume = 1.0) : volume_(volume) {}
  double volume() const { return volume_; }
};
using BoundaryConditions = std::variant<PeriodicBC, InfiniteBC>;

// core/atom.hpp
struct Atom {
  Species type{};
  Vec3 pos = Vec3::Zero();
  struct Reference {
    Vec3 force = Vec3::Zero();
  } ref;
  Vec3 calc_force = Vec3::Zero();
};

struct Configuration {
  std::vector<Atom> atoms;
  BoundaryConditions bc = PeriodicBC(Mat3::Identity());
  std::string name;
  struct Reference {
    double energy = 0.0;
    SymTens stress = SymTens::Zero();
  } ref;
  double weight = 1.0;
  double calc_energy = 0.0;
  SymTens calc_stress = SymTens::Zero();
  double calc_limit = 0.0;
};

// optimization/solver.hpp
using ResidualFn = std::function<VectorXd(const VectorXd &)>;
using JacobianFn = std::function<void(const VectorXd &, MatrixXd &)>;

} // namespace forcesmith
