// Seeded synthetic configurations with the shapes of the benchmark workloads
// (fcc Al, random ternary packings, diamond Si).  Deterministic across
// machines: a splitmix64 counter RNG and explicit Box–Muller, no <random>
// distributions (whose output is implementation-defined).
//
// Layout of every output matches fs_gpu_upload_configs: box9 is row-major with
// the lattice vectors as COLUMNS; positions are Cartesian, 3 per atom.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  double normal() {
    double u1 = uniform();
    if (u1 < 1e-300) u1 = 1e-300;
    const double u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

void mat_vec(const double *M, const double *v, double *o) {
  for (int r = 0; r < 3; ++r) o[r] = M[3 * r] * v[0] + M[3 * r + 1] * v[1] + M[3 * r + 2] * v[2];
}

// Minimum-image distance² in a cubic-then-strained box, via fractional coords.
double min_image_d2(const double *box, const double *f1, const double *f2) {
  double df[3];
  for (int k = 0; k < 3; ++k) {
    df[k] = f2[k] - f1[k];
    df[k] -= std::round(df[k]);
  }
  double d[3];
  mat_vec(box, df, d);
  return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
}

} // namespace

extern "C" {

// fcc lattice, ncell³ conventional cells (4·ncell³ atoms), lattice constant a,
// isotropic strain factor U[s_lo, s_hi], Gaussian displacement σ per
// coordinate.  One species (slot 0).
int fs_synth_fcc(int32_t n_cfg, int32_t ncell, double a, double sigma, double s_lo, double s_hi,
                 uint64_t seed, int32_t *natoms, double *box9, double *pos, int32_t *type) {
  const int n = 4 * ncell * ncell * ncell;
  const double basis[4][3] = {{0, 0, 0}, {0.5, 0.5, 0}, {0.5, 0, 0.5}, {0, 0.5, 0.5}};
  int64_t off = 0;
  for (int c = 0; c < n_cfg; ++c) {
    Rng rng(seed + 1000003ull * c);
    const double s = rng.uniform(s_lo, s_hi);
    const double L = a * ncell * s;
    natoms[c] = n;
    double *B = box9 + 9 * c;
    std::memset(B, 0, 9 * sizeof(double));
    B[0] = B[4] = B[8] = L;
    for (int ix = 0; ix < ncell; ++ix)
      for (int iy = 0; iy < ncell; ++iy)
        for (int iz = 0; iz < ncell; ++iz)
          for (int b = 0; b < 4; ++b) {
            double *p = pos + 3 * off;
            p[0] = (ix + basis[b][0]) * a * s + sigma * rng.normal();
            p[1] = (iy + basis[b][1]) * a * s + sigma * rng.normal();
            p[2] = (iz + basis[b][2]) * a * s + sigma * rng.normal();
            type[off] = 0;
            ++off;
          }
  }
  return 0;
}

// Diamond lattice (8 atoms per conventional cell), cells chosen per config
// from cell_choices[0..n_choices); volumetric strain U[v_lo, v_hi] applied
// as a linear factor ∛v; Gaussian displacement σ.  natoms[c] = 8·m³.
int fs_synth_diamond(int32_t n_cfg, const int32_t *cell_choices, int32_t n_choices, double a,
                     double sigma, double v_lo, double v_hi, uint64_t seed, int32_t *natoms,
                     double *box9, double *pos, int32_t *type, int64_t pos_capacity) {
  const double basis[8][3] = {{0, 0, 0},       {0, 0.5, 0.5},     {0.5, 0, 0.5},
                              {0.5, 0.5, 0},   {0.25, 0.25, 0.25}, {0.25, 0.75, 0.75},
                              {0.75, 0.25, 0.75}, {0.75, 0.75, 0.25}};
  int64_t off = 0;
  for (int c = 0; c < n_cfg; ++c) {
    Rng rng(seed + 7919ull * c);
    const int m = cell_choices[rng.next() % static_cast<uint64_t>(n_choices)];
    const double s = std::cbrt(rng.uniform(v_lo, v_hi));
    const int n = 8 * m * m * m;
    if (off + n > pos_capacity) return -1;
    natoms[c] = n;
    double *B = box9 + 9 * c;
    std::memset(B, 0, 9 * sizeof(double));
    B[0] = B[4] = B[8] = a * m * s;
    for (int ix = 0; ix < m; ++ix)
      for (int iy = 0; iy < m; ++iy)
        for (int iz = 0; iz < m; ++iz)
          for (int b = 0; b < 8; ++b) {
            double *p = pos + 3 * off;
            p[0] = (ix + basis[b][0]) * a * s + sigma * rng.normal();
            p[1] = (iy + basis[b][1]) * a * s + sigma * rng.normal();
            p[2] = (iz + basis[b][2]) * a * s + sigma * rng.normal();
            type[off] = 0;
            ++off;
          }
  }
  return 0;
}

// Random sequential packing: natoms[c] given, cubic box of side
// (N/density)^{1/3}, points inserted uniformly with minimum-image distance ≥
// dmin, then an affine random symmetric strain ε (entries U[−strain, strain])
// applied to box and positions.  Species i.i.d. with probabilities prob[nt]
// (slot order).  Returns −(c+1) if config c cannot be packed.
int fs_synth_packing(int32_t n_cfg, const int32_t *natoms, double density, double dmin,
                     double strain, const double *prob, int32_t nt, uint64_t seed, double *box9,
                     double *pos, int32_t *type) {
  int64_t off = 0;
  const double d2min = dmin * dmin;
  for (int c = 0; c < n_cfg; ++c) {
    Rng rng(seed + 104729ull * c);
    const int n = natoms[c];
    const double L = std::cbrt(n / density);
    double cube[9] = {L, 0, 0, 0, L, 0, 0, 0, L};
    std::vector<double> frac(3 * static_cast<size_t>(n));
    // cell grid over the cube (cell side >= dmin) so that an insertion test
    // only visits the 27 surrounding cells
    const int nc = static_cast<int>(std::floor(L / dmin));
    const bool grid = nc >= 3;
    std::vector<std::vector<int>> cells(grid ? nc * nc * nc : 1);
    auto cell_of = [&](const double *f, int *ci) {
      for (int k = 0; k < 3; ++k) {
        ci[k] = static_cast<int>(f[k] * nc);
        if (ci[k] >= nc) ci[k] = nc - 1;
        if (ci[k] < 0) ci[k] = 0;
      }
    };
    int placed = 0;
    int64_t tries = 0;
    const int64_t max_tries = 200000000;
    while (placed < n) {
      if (++tries > max_tries) return -(c + 1);
      double f[3] = {rng.uniform(), rng.uniform(), rng.uniform()};
      bool ok = true;
      if (grid) {
        int ci[3];
        cell_of(f, ci);
        for (int dx = -1; dx <= 1 && ok; ++dx)
          for (int dy = -1; dy <= 1 && ok; ++dy)
            for (int dz = -1; dz <= 1 && ok; ++dz) {
              const int x = (ci[0] + dx + nc) % nc, y = (ci[1] + dy + nc) % nc,
                        z = (ci[2] + dz + nc) % nc;
              for (int k : cells[(x * nc + y) * nc + z])
                if (min_image_d2(cube, &frac[3 * k], f) < d2min) {
                  ok = false;
                  break;
                }
            }
      } else {
        for (int k = 0; k < placed && ok; ++k)
          if (min_image_d2(cube, &frac[3 * k], f) < d2min) ok = false;
      }
      if (!ok) continue;
      std::memcpy(&frac[3 * placed], f, sizeof f);
      if (grid) {
        int ci[3];
        cell_of(f, ci);
        cells[(ci[0] * nc + ci[1]) * nc + ci[2]].push_back(placed);
      }
      ++placed;
    }
    double eps[3][3];
    for (int r = 0; r < 3; ++r)
      for (int k = r; k < 3; ++k) eps[r][k] = eps[k][r] = rng.uniform(-strain, strain);
    double *B = box9 + 9 * c;
    for (int r = 0; r < 3; ++r)
      for (int k = 0; k < 3; ++k) B[3 * r + k] = ((r == k ? 1.0 : 0.0) + eps[r][k]) * L;
    for (int i = 0; i < n; ++i) {
      mat_vec(B, &frac[3 * i], pos + 3 * (off + i));
      double u = rng.uniform(), acc = 0.0;
      int t = nt - 1;
      for (int s = 0; s < nt; ++s) {
        acc += prob[s];
        if (u < acc) {
          t = s;
          break;
        }
      }
      type[off + i] = t;
    }
    off += n;
  }
  return 0;
}

// Uniform integers in [lo, hi] (atom counts of the uneven workloads).
int fs_synth_counts(int32_t n, int32_t lo, int32_t hi, uint64_t seed, int32_t *out) {
  Rng rng(seed);
  for (int i = 0; i < n; ++i)
    out[i] = lo + static_cast<int32_t>(rng.next() % static_cast<uint64_t>(hi - lo + 1));
  return 0;
}

// Uniform doubles in [lo, hi) (knot perturbations, DE populations).
int fs_synth_uniform(int64_t n, double lo, double hi, uint64_t seed, double *out) {
  Rng rng(seed);
  for (int64_t i = 0; i < n; ++i) out[i] = rng.uniform(lo, hi);
  return 0;
}

} // extern "C"
