// Internal declarations shared by the translation units of
// libforcesmith_b200.so (the fs_gpu context, device table layout, launchers).
#pragma once

#include "forcesmith_gpu.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

namespace fsg {

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
struct Status {
  int code = FS_OK;
  std::string msg;
};

#define FS_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);             \
      return FS_ERR_CUDA;                                                      \
    }                                                                          \
  } while (0)

#define FS_TRY(expr)                                                           \
  do {                                                                         \
    int rc_ = (expr);                                                          \
    if (rc_ != FS_OK) return rc_;                                              \
  } while (0)

// ---------------------------------------------------------------------------
// Device table layout.
//
// A spline of n knots is stored as n+1 "extended segments": e = 0 is the
// linear extrapolation below x0, e = 1..n-1 the interior cubic (or linear,
// n < 4) pieces, e = n the linear extrapolation above x_{n-1}.  Segment e
// holds the power-basis coefficients a[0..3] in t = (r - origin_e)/h, the
// knot-derivative block G[4][6] = ∂a_k/∂y_{ws+q}, and its window start ws.
// ---------------------------------------------------------------------------
constexpr int kWin = 6;      // knots a segment depends on (makima: 6)
constexpr int kMaxTables = 64;
constexpr int kMaxSegs = 4096;

struct TableDesc {
  int kind;    // fs_table_kind
  int form;    // fs_form (analytic)
  int n;       // knots / parameters
  int seg0;    // first extended segment (splines)
  int cmap0;   // first entry of the knot/param → column map
  int pv0;     // first value in the parameter-value array
  int pad0, pad1;
  double x0, h, inv_h, xmax; // spline grid (x0, spacing, 1/h, last knot)
  double rmin, rmax;         // gate span
};

// Per-config geometry on the device.
struct CfgDev {
  int atom0;      // first atom (global)
  int natoms;
  int pair0;      // first pair (global) of the config
  int sx, sy, sz; // image shells
  double box[9];  // row-major, lattice vectors as columns
  double inv[9];
  double volume;
  double ref_energy;
  double ref_stress[9];
};

// ---------------------------------------------------------------------------
// The context behind the opaque fs_gpu handle.
// ---------------------------------------------------------------------------
template <class X> struct DBuf {
  X *p = nullptr;
  size_t n = 0;
};

struct HostTable {
  int kind = 0, form = 0, n = 0;
  double rmin = 0, rmax = 0;
  std::vector<double> v, lo, hi;
  std::vector<uint8_t> fixed;
  std::vector<int> cols; // column per value (-1 if fixed)
};

} // namespace fsg

namespace fsg {
struct DeState;
void de_free(DeState *s);
struct Mlp;
void mlp_free(Mlp *s);
struct Surrogate;
void surrogate_free(Surrogate *s);
} // namespace fsg

struct fs_gpu {
  int device = 0;
  int precision = FS_PREC_FP32;
  int lanes_per_atom = 0;
  cudaStream_t stream = nullptr;
  // side stream of a Jacobian step: the residual runs there beside the
  // per-atom Jacobian pass; the force-row pass waits for ev_join
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool join_pending = false;
  std::string err;

  // configs (host)
  int n_cfg = 0;
  int64_t n_atoms = 0;
  int max_natoms = 0;
  std::vector<int32_t> natoms;
  std::vector<int64_t> atom0;
  std::vector<fsg::CfgDev> cfg_host;
  // configs (device)
  fsg::CfgDev *d_cfg = nullptr;
  double *d_pos = nullptr;       // raw positions, 3 per atom
  double *d_wpos = nullptr;      // wrapped positions, 3 per atom
  int32_t *d_type = nullptr;
  double *d_ref_force = nullptr; // 3 per atom

  // neighbours
  double rcut_built = -1.0;
  int64_t n_pairs = 0;
  int32_t *d_nb_start = nullptr; // n_atoms + 1 (global pair offsets)
  uint32_t *d_nb_pack = nullptr; // j_local (20 bits) | image index (12 bits)
  int32_t *d_nb_count = nullptr; // per atom
  // 3-body work: the largest count of directed pairs + neighbour pairs (j < k)
  // of one configuration, and the configurations ordered by that count,
  // heaviest first (launch order of the per-configuration 3-body kernels)
  int64_t max_cfg_work = 0;
  int max_list = -1; // the longest neighbour list (LMBTR warp slices); −1: not yet counted
  int32_t *d_cfg_by_work = nullptr;

  // model
  bool have_model = false;
  int family = 0, ntypes = 1;
  std::vector<fsg::HostTable> tables;
  int D = 0;                // free parameters
  // global parameters: values and columns (−1 fixed); shared_cols when a
  // free global has links, i.e. several values share one column
  std::vector<double> global_val;
  std::vector<int> global_col;
  bool shared_cols = false;
  std::vector<fsg::TableDesc> desc;
  int n_segs = 0, n_cmap = 0, n_vals = 0;
  fsg::TableDesc *d_desc = nullptr;
  int32_t *d_cmap = nullptr;     // knot/param → column (-1 fixed)
  double *d_vals = nullptr;      // all table values (FP64, current params)
  // segment tables in the working precision (FP32 or FP64)
  void *d_seg_a = nullptr;       // [n_segs][4]
  void *d_seg_g = nullptr;       // [n_segs][4][kWin]
  int32_t *d_seg_ws = nullptr;   // [n_segs]
  double *d_x = nullptr;         // current parameter vector (D)
  bool params_dirty = true;
  int32_t *d_spl = nullptr;      // indices of the spline tables (segment setup)
  int n_spl = 0;
  // pinned host staging: parameter values going up, normal equations coming
  // back (one DMA each, no pageable staging); vals_ev marks the last upload
  double *h_vals_pin = nullptr, *h_ne_pin = nullptr;
  size_t h_vals_pin_n = 0, h_ne_pin_n = 0;
  cudaEvent_t vals_ev = nullptr;

  // evaluation buffers
  int64_t rows_alloc = 0;
  double *d_F = nullptr;         // residual (rows)
  double *d_forces = nullptr;    // 3 per atom
  double *d_energy = nullptr, *d_stress9 = nullptr, *d_limit = nullptr;
  double *d_obj_part = nullptr;  // per config
  double *d_obj = nullptr;       // scalar
  // Jacobian buffers
  int64_t jac_alloc = 0;         // elements of J
  void *d_J = nullptr;           // J, FP32 or FP64; rows rounded up to 32 (rows ≥ M are zero)
  int64_t ldj = 0;               // column-major: the padded row count; row-major: the row stride (≥ D)
  bool j_rowmajor = false;       // row-major J (FP32 EAM / pair Jacobians feeding the tensor-core JᵀJ)
  double *d_jx = nullptr;        // FP64 column-major staging of an exported row block of J
  size_t jx_alloc = 0;
  void *d_an = nullptr;          // analytic-table Jacobian: column table and per-atom scratch
  size_t an_alloc = 0;
  double *d_jtr_part = nullptr;  // per-config Jᵀr partials (FP64)
  size_t jtr_part_alloc = 0;
  double *d_half_part = nullptr; // force-row pass with two CTAs per configuration: their sums
  size_t half_part_alloc = 0;
  double *d_fd_scratch = nullptr; // central-difference Jacobian: base and perturbed residuals
  size_t fd_scratch_alloc = 0;
  int32_t *d_err = nullptr;      // device error word (bounded waits that gave up)
  double *d_JtJ = nullptr;       // D × D
  double *d_Jtr = nullptr;       // D
  double *d_gram_part = nullptr; // split partials
  size_t gram_part_alloc = 0;
  // per-atom Jacobian scratch
  void *d_atom_scalars = nullptr; // [n_atoms][4]: gradF, curvF, (ws as float), over
  void *d_drho = nullptr;         // [n_atoms][ndens]
  void *d_dgd = nullptr;          // [n_atoms][kWin]
  int32_t *d_wsF = nullptr;       // [n_atoms]
  int64_t atom_scratch_alloc = 0;
  // population kernel on a knot grid shared by the pair and density tables:
  // each atom's in-gate pairs sorted by (neighbour species, segment of the
  // grid), built once per neighbour list and grid (pair_runs.cuh)
  float4 *d_run_a = nullptr;      // [pair]: u_x, u_y, u_z, t  (pair slots of the neighbour list)
  int2 *d_run_b = nullptr;        // [pair]: packed neighbour entry, key = (species << 8) | segment
  int32_t *d_run_cnt = nullptr;   // [atom]: in-gate pairs
  float *d_run_r = nullptr;       // [pair]: FP64 length rounded to FP32
  bool runs_valid = false;        // built for the current neighbour lists and model grid
  double last_ws = -1.0, last_we = 0.0;
  bool jac_valid = false;

  // LM solve scratch
  double *d_chol = nullptr;
  int chol_D = 0;
  int max_type = 0;
  double *d_dx = nullptr;
  int32_t *d_flag = nullptr;

  // live per-phase timing (CUDA events on `stream`) and kernel launch count
  std::vector<cudaEvent_t> prof_ev; // prof_slots × (kPhases + 1)
  int prof_slots = 0, prof_used = 0;
  int64_t launches = 0;

  // population scratch
  void *d_pop_seg_a = nullptr;   // per-trial segments | per-(trial, config) Σ rows² | config order
  int64_t pop_alloc = 0;
  int *d_pop_spl = nullptr;      // spline table indices
  int pop_spl_count = 0;
  double *d_pop_vals = nullptr;
  double *d_pop_obj = nullptr;

  // schedules chosen by fs_gpu_autotune (0: built-in choice)
  int tuned_lpa = 0;       // residual lanes per atom
  int tuned_k2_warps = 0;  // warps per CTA of the Jacobian force-row kernel
  int tuned_pop_waves = 0; // CTA waves of the FP32 population kernel

  // device differential evolution (population.cu) and its surrogate (mlp.cu)
  fsg::DeState *de = nullptr;
  fsg::Mlp *mlp = nullptr;
  fsg::Surrogate *sur = nullptr;
};

namespace fsg {

int set_error(fs_gpu *h, int code, const std::string &m);
// fs_gpu_eval_population_noalloc's cached scratch address of a device: dropped
// when a context is created there, so a later first call looks it up again.
void noalloc_forget(int device);
// stream sync + the device error word of bounded waits
int sync_checked(fs_gpu *h);

// Phases of one residual + Jacobian evaluation, timed with CUDA events
// when profiling is on: residual, per-atom Jacobian, force/stress rows,
// normal-equation products.
constexpr int kPhases = 4;
enum { kPhResidual = 0, kPhJacAtoms = 1, kPhJacForces = 2, kPhGram = 3 };
inline void mark(fs_gpu *h, int boundary) {
  if (h->prof_slots > 0 && h->prof_used < h->prof_slots)
    cudaEventRecord(h->prof_ev[h->prof_used * (kPhases + 1) + boundary], h->stream);
}

// neighbour.cu
int build_neighbors(fs_gpu *h, double rcut);

// pair_runs.cu: each atom's pairs sorted by (neighbour species, segment) on
// the knot grid shared by the pair and density tables
constexpr int kRunMaxT = 4;  // species
constexpr int kRunMaxN = 64; // knots of the shared grid
constexpr int kRunKeyBits = 8; // run key = (neighbour species << 8) | segment (segments ≤ kRunMaxN)
struct RunGrid {
  double x0, xmax, inv_h;
  int n;
};
bool pair_runs_grid(const fs_gpu *h, RunGrid *g);
int build_pair_runs(fs_gpu *h); // after every neighbour build (no-op without a shared grid)

// tables.cu
int upload_tables(fs_gpu *h);          // structure + values (after set_model)
int upload_values(fs_gpu *h);          // values only (after set_params), asynchronous
int ensure_pinned(fs_gpu *h, double **buf, size_t *cap, size_t n);
int refresh_segments(fs_gpu *h);       // recompute segment data from d_vals
int spline_segments_fp64(fs_gpu *h, const double *d_x1, double4 *seg); // FP64 segments at x (n_segs)
double model_max_cutoff(const fs_gpu *h);

// eam.cu / pair
int eval_residual(fs_gpu *h, double w_e, double w_s);
int eval_jacobian(fs_gpu *h, double w_e, double w_s);

// gram.cu
// ACSF: per-species descriptor mean and 1/σ over the uploaded atoms (acsf.cu)
int acsf_standardization(fs_gpu *h, double *mean, double *inv_std, int64_t *count);
int gram(fs_gpu *h, int64_t m, double *JtJ_dev, double *Jtr_dev);
int gram_tc(fs_gpu *h, int64_t m, double *JtJ_dev); // tcgen05 (FP32 J)
// JᵀJ paths: D ≤ kGramSmallD a row-slab kernel over the upper triangle;
// else FP32 with D ≤ 256 the tensor cores (the only reader of a row-major J);
// else 64 × 64 CUDA-core tiles
constexpr int kGramSmallD = 48;
inline bool gram_on_tensor_cores(int precision, int D) {
  return precision == FS_PREC_FP32 && D > kGramSmallD && D <= 256;
}

// solve.cu
int lm_solve(fs_gpu *h, double lambda, int mode, double *dx_host);

// population.cu / eam.cu
int eval_population(fs_gpu *h, double w_e, double w_s, const double *xs, int NP, double *obj);
int eval_population_device(fs_gpu *h, double w_e, double w_s, const double *d_xs, int NP, double *d_obj);

// mlp.cu
int64_t mlp_param_count(int D);
int mlp_create(fs_gpu *h, int D, uint64_t seed, float lr, Mlp **out);
int mlp_set_params(fs_gpu *h, Mlp *s, const float *host_params);
int mlp_get(fs_gpu *h, Mlp *s, const float *dev_flat, float *host_params);
float *mlp_param_ptr(Mlp *s);
float *mlp_grad_ptr(Mlp *s);
float *mlp_rows_x(Mlp *s); // FP32 features, row-major D, capacity mlp_capacity rows
float *mlp_rows_t(Mlp *s); // FP32 targets
float *mlp_rows_y(Mlp *s); // FP32 predictions
float *mlp_loss_ptr(Mlp *s);
int mlp_capacity(Mlp *s);
int mlp_reserve(fs_gpu *h, Mlp *s, int rows);
int mlp_forward_dev(fs_gpu *h, Mlp *s, int rows);
int mlp_gradient_dev(fs_gpu *h, Mlp *s, int rows);
int mlp_adam_dev(fs_gpu *h, Mlp *s);

inline int64_t rows_of(const fs_gpu *h, double w_s) {
  return 3 * h->n_atoms + static_cast<int64_t>(h->n_cfg) * (2 + (w_s > 0.0 ? 6 : 0));
}

inline int npair_of(int nt) { return nt * (nt + 1) / 2; }

} // namespace fsg
