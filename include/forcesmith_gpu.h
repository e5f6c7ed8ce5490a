/*
 * forcesmith_gpu.h — C ABI of the B200 objective-evaluation path.
 *
 * This is the drop-in boundary between Forcesmith's C++ host code and the
 * sm_100a kernels.  Every entry point is `extern "C"`, takes plain pointers
 * and sizes, returns an int status (FS_OK == 0, negative on error) and never
 * throws.  Host pointers are ordinary pageable or pinned memory; the library
 * owns every device allocation behind the opaque `fs_gpu` handle.
 *
 * Each entry point replaces one interface of the reference's CPU path
 * (paths are relative to the Forcesmith source tree):
 *
 *   fs_gpu_upload_configs      Forcesmith::add_configuration / the per-config
 *                              `Configuration` data model
 *                              (include/forcesmith/core/atom.hpp:38-100,
 *                               src/io/config_reader.cpp:58-130)
 *   fs_gpu_set_model           Forcesmith::seed_force_model + the calculator
 *                              tables (include/forcesmith/api/forcesmith.hpp:125,
 *                               include/forcesmith/force/eam_force.hpp:24-32,
 *                               pair_force.hpp:27-29, adp_force.hpp:34-54,
 *                               stiweb_force.hpp:19-62)
 *   fs_gpu_prepare             CForceCalculator::prepare → build_all_neighbor_lists
 *                              (src/core/neighbor_list.cpp:105-147,
 *                               src/force/eam_force.cpp:281-296)
 *   fs_gpu_get_neighbor_counts / fs_gpu_get_neighbors
 *                              the integer neighbour sets of build_periodic
 *                              (src/core/neighbor_list.cpp:59-92)
 *   fs_gpu_param_count / fs_gpu_gather_params / fs_gpu_gather_bounds /
 *   fs_gpu_set_params          CFittable param_count / gather_params /
 *                              gather_bounds / scatter_params, table order
 *                              (include/forcesmith/force/force_calculator_concept.hpp:171-208,
 *                               src/force/stiweb_force.cpp:169-195,
 *                               src/potentials/spline.cpp:191-203)
 *   fs_gpu_residual_count      opt::count_residuals
 *                              (include/forcesmith/optimization/residual_layout.hpp:18-31)
 *   fs_gpu_eval                ForcesmithFunctor::operator() → eval_into:
 *                              scatter + eval_forces per config + write_config_residuals
 *                              (src/optimization/forcesmith_functor.cpp:35-57,221-231)
 *                              and force::evaluate / Forcesmith::evaluate_all
 *                              (src/force/evaluate.cpp:5-20, src/api/forcesmith.cpp:587-614)
 *   fs_gpu_eval_jacobian       ForcesmithFunctor::df (src/optimization/forcesmith_functor.cpp:252-292)
 *                              — the analytic chain rule of write_param_jacobian
 *                              (src/force/eam_force.cpp:108-279, pair_force.cpp:80-111)
 *                              extended to spline knots, in place of opt::fd_jacobian
 *                              (include/forcesmith/optimization/fd_jacobian.hpp:37-49);
 *                              plus the JᵀJ / Jᵀr products that
 *                              NormalEquationsSolver and LM consume
 *                              (src/optimization/solver.cpp:242-266)
 *   fs_gpu_copy_jacobian_rows  the per-configuration block of fjac that
 *                              CForceCalculator::eval_cached_jacobian fills
 *                              (include/forcesmith/force/force_calculator_concept.hpp:62-67,
 *                               src/optimization/forcesmith_functor.cpp:111-132)
 *   fs_gpu_max_cutoff          CForceCalculator::max_cutoff
 *                              (include/forcesmith/force/force_calculator_concept.hpp:210-225,288-292)
 *   fs_gpu_tabulate            RadialPotential::eval / deriv as the model writers
 *                              sample them (src/io/output_writer.cpp:22-40,266-310)
 *   fs_gpu_lm_step / fs_gpu_lsq_step
 *                              the LM / lsq step of EigenLMSolver and
 *                              NormalEquationsSolver (src/optimization/solver.cpp:67-85,242-266)
 *   fs_gpu_eval_population[_noalloc]
 *                              many parameter vectors' objectives in one launch
 *                              (the inner loop of BoostDESolver and of the LM trials)
 *   fs_gpu_de_*                BoostDESolver's population evaluation
 *                              (src/optimization/solver.cpp:113-155)
 *   fs_gpu_surrogate_*         (no reference counterpart: the learned
 *                              pre-screen of DE trial vectors)
 *   fs_gpu_check_bounded_wait  (no reference counterpart: a device wait that
 *                              gives up and reports, for failure detection)
 *
 * include/forcesmith_gpu_adapter.hpp wraps these in C++ classes that satisfy
 * the reference's CForceCalculator and CSolver concepts.
 */
#ifndef FORCESMITH_GPU_H
#define FORCESMITH_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  FS_OK = 0,
  FS_ERR_ARG = -1,         /* bad argument (null handle, size mismatch …)   */
  FS_ERR_CUDA = -2,        /* a CUDA runtime call failed                    */
  FS_ERR_STATE = -3,       /* call out of order (no configs / no model …)   */
  FS_ERR_UNSUPPORTED = -4, /* valid input this build does not handle        */
  FS_ERR_NOMEM = -5,       /* device allocation failed                      */
  FS_ERR_DEVICE = -6,      /* a kernel reported an error word               */
  FS_ERR_NUMERIC = -7      /* non-finite result / failed factorisation      */
};

/* ---- model description ------------------------------------------------- */
enum fs_family {
  FS_FAMILY_PAIR = 0, /* tables: pair[npair]                                */
  FS_FAMILY_EAM = 1,  /* tables: pair[npair], density[nt], embedding[nt]    */
  FS_FAMILY_ADP = 2,  /* tables: EAM + dipole[npair], quadrupole[npair]     */
  FS_FAMILY_SW = 3,   /* tables: sw[npair] (8 params each), lambda[1]       */
  FS_FAMILY_TERSOFF = 4, /* tables: tersoff[npair] (12 params each)        */
  FS_FAMILY_ANGULAR = 5, /* tables: pair[npair], radial[npair], angular[nt]:
                            spline or analytic (angular_force.hpp:15-33)   */
  FS_FAMILY_ACSF = 6,    /* tables: acsf[1] (descriptor), head[nt] (linear
                            energy head per species) (acsf.hpp:48-86,
                            ml_force.hpp LinearHead), and optionally
                            standardization[nt] (MLBase mean_ / inv_std_,
                            ml_force.hpp:194-199)                          */
  FS_FAMILY_LMBTR = 7    /* tables: lmbtr[1] (descriptor), head[nt], and
                            optionally standardization[nt], as for ACSF
                            (include/forcesmith/potentials/lmbtr.hpp:40-63) */
};

enum fs_table_kind {
  FS_TABLE_SPLINE = 0,   /* uniform-grid makima spline: n knot values       */
  FS_TABLE_ANALYTIC = 1, /* closed form `form` with n parameters            */
  FS_TABLE_SW = 2,       /* SWParams {A,B,p,q,delta,a1,gamma,a2}, n == 8    */
  FS_TABLE_LAMBDA = 3,   /* SW triplet strengths, n == nt * npair           */
  FS_TABLE_TERSOFF = 4,  /* TersoffParams {A,B,lambda,mu,beta,n,c,d,h,R,S,omega},
                            n == 12 (include/forcesmith/force/tersoff_force.hpp:17-31;
                            gather order tersoff_force.cpp:14-25)          */
  FS_TABLE_ACSF = 5,     /* ACSF symmetry functions, all values fixed:
                            {rcut, nG1, nG2, nG3, nG4, nG5,
                             (eta, rs) × nG2, kappa × nG3,
                             (eta, zeta, lambda) × nG4, (eta, zeta, lambda) × nG5};
                            descriptor size S = nt(nG1 + nG2 + nG3)
                            + npair(nG4 + nG5) (AcsfLayout, acsf.hpp:23-33) */
  FS_TABLE_LINEAR_HEAD = 6, /* E_i = w·D_i + b: {w[S], b}, n == S + 1; the
                            bias is fixed unless `fixed` says otherwise    */
  FS_TABLE_STANDARDIZATION = 7, /* per species, all values fixed: {mean[S],
                            inv_std[S]}, n == 2S; the head then sees
                            (D − mean) ⊙ inv_std (ml_force.hpp:607-623);
                            mean 0 and inv_std 1 leave D unchanged        */
  FS_TABLE_LMBTR = 8     /* LMBTR descriptor, all values fixed:
                            {rcut, weight_scale, normalize (0/1),
                             n2, min2, max2, sigma2, n3, min3, max3, sigma3};
                            a term with n = 0 is absent; descriptor size
                            S = nt·n2 + npair·n3 (LmbtrLayout, lmbtr.hpp:13-38) */
};

/* Analytic radial forms (include/forcesmith/potentials/analytic_potential.hpp). */
enum fs_form {
  FS_FORM_LJ = 0,          /* 4ε((σ/r)^12 − (σ/r)^6)             {eps,sigma} */
  FS_FORM_MORSE = 1,       /* De(1−e^{−a(r−re)})² − De           {De,a,re}   */
  FS_FORM_EXP_DECAY = 2,   /* A e^{−Br}                          {A,B}       */
  FS_FORM_SQRT = 3,        /* A sqrt(r/B)                        {A,B}       */
  FS_FORM_POWER_DECAY = 4, /* A / r^n                            {A,n}       */
  FS_FORM_MEXP_DECAY = 5,  /* A e^{−B(r−r0)}                     {A,B,r0}    */
  FS_FORM_HARMONIC = 6,    /* k (r−r0)²                          {k,r0}      */
  FS_FORM_EXP_PLUS = 7,    /* A e^{−Br} + C                      {A,B,C}     */
  FS_FORM_PARABOLA = 8,    /* A r² + B r + C                     {A,B,C}     */
  FS_FORM_CONST = 9,       /* C                                  {C}         */
  FS_FORM_BUCKINGHAM = 10, /* A e^{−r/ρ} − C (ρ²/r²)³            {A,rho,C}   */
  FS_FORM_BORN = 11,       /* A e^{(C−r)/B} − D/r^6 + E/r^8      {A,B,C,D,E} */
  FS_FORM_UNIVERSAL = 12,  /* E0(b/(b−a) r^a − a/(b−a) r^b) + c r {E0,a,b,c} */
  FS_FORM_EOPP = 13,       /* A/r^n + B/r^m cos(k r + φ)   {A,n,B,m,k,phi}   */
  FS_FORM_EOPP_EXP = 14,   /* A e^{−Br} + C/r^m cos(k r + φ) {A,B,C,m,k,phi} */
  FS_FORM_MEOPP = 15,      /* A/(r−r0)^n + B/r^m cos(k r + φ) {…,r0}        */
  FS_FORM_GEN_LJ = 16,     /* A/(m−n)(m x^{−n} − n x^{−m}) + B, x = r/r0
                                                           {A,n,m,r0,B}      */
  FS_FORM_DOUBLE_MORSE = 17, /* Σ D_k((1−e_k)² − 1) + C {D1,a1,r1,D2,a2,r2,C} */
  FS_FORM_DOUBLE_EXP = 18, /* A e^{−B(r−r1)²} + e^{−C(r−r2)}  {A,B,r1,C,r2}   */
  FS_FORM_MISHIN = 19,     /* A z^n e^{−dz}(1 + B e^{−dz}) + C, z = r − r0
                                                           {A,B,C,r0,n,d}    */
  FS_FORM_POLY5 = 20,      /* a0 + ½a1 s² + a2 s³ + a3 s⁴ + a4 s⁵, s = r − 1 */
  FS_FORM_STIWEB2 = 21,    /* (A r^{−p} − B r^{−q}) e^{δ/(r−rc)}, 0 past rc
                                                           {A,B,p,q,delta,rc}*/
  FS_FORM_STIWEB3 = 22,    /* e^{γ/(r−a)}, 0 past a             {gamma,a}  */
  FS_FORM_TERSOFF = 23,    /* fc(r)(A e^{−λr} − B e^{−μr})
                              {A,B,lambda,mu,beta,n,c,d,h,R,S}               */
  FS_FORM_TERSOFF_MIX = 24, /* χ e^{−ωr}                         {chi,omega} */
  FS_FORM_TERSOFF_MOD = 25, /* Tersoff × (1 + c1 r + … + c5 r⁵), 16 params  */
  FS_FORM_KAWAMURA = 26,   /* AB/r + C(F+G) e^{(D+E−r)/(F+G)} − HI/r⁶ {A..I} */
  FS_FORM_KAWAMURA_MIX = 27, /* Kawamura + CJ(e^{−2K(r−L)} − 2e^{−K(r−L)}) {A..L} */
  FS_FORM_SOFTSHELL = 28,  /* (A/r)^n                              {A,n}      */
  FS_FORM_STRMM = 29,      /* 2A e^{−B s/2} − C(1 + D s) e^{−D s}, s = r − E */
  FS_FORM_LJ_SC = 30,      /* LJ × switch(r; rmax, h)          {eps,sigma,h} */
  FS_FORM_MORSE_SC = 31,   /* Morse × switch                    {De,a,re,h}  */
  FS_FORM_EXP_DECAY_SC = 32, /* ExpDecay × switch                  {A,B,h}   */
  FS_FORM_EOPP_SC = 33,    /* Eopp × switch                     {…,h}        */
  FS_FORM_COUNT = 34
};
/* switch(r; rmax, h) = u⁴/(1 + u⁴), u = min((r − rmax)/h, 0), with rmax the
 * table's upper gate bound (SmoothCutoff, analytic_potential.hpp:782-793);
 * fc is the cosine cutoff between R and S (analytic_potential.hpp:142-145).
 * The order is the reference's AnalyticForms list (analytic_potential.hpp:801-806)
 * after the first twelve. */

typedef struct fs_table {
  int32_t kind;          /* fs_table_kind                                   */
  int32_t form;          /* fs_form for FS_TABLE_ANALYTIC, else ignored     */
  int32_t n;             /* knots / parameters                              */
  int32_t reserved;
  double rmin, rmax;     /* knot domain (spline) or gate span (analytic)    */
  const double *values;  /* knot values y[n] or parameters[n]               */
  const uint8_t *fixed;  /* nullable: 1 = value is fixed (takes no column)  */
  const double *lower;   /* nullable: per-value lower bound (−inf if null)  */
  const double *upper;   /* nullable: per-value upper bound (+inf if null)  */
} fs_table;

typedef struct fs_model {
  int32_t family;   /* fs_family                                            */
  int32_t ntypes;   /* species slots (Z-sorted)                             */
  int32_t n_tables; /* must equal the family's table count                  */
  int32_t reserved;
  const fs_table *tables; /* in the reference's gather order                */
  /* Global parameters (GlobalParam, force_calculator_concept.hpp:21-44;
   * pair and EAM families, analytic tables): n_globals values and fixed
   * flags (nullable: all free), and n_links links (global, table in model
   * order, parameter slot).  A linked parameter is fixed in its table and
   * takes the global's value (finalize_globals, :235-242); a free global's
   * column follows every table column, in global order (:171-208).  The
   * global's own min/max are not kept (build_globals reads only value and
   * fixed, force_model_reader.cpp:64-75): its bounds are ±inf.  Zero
   * everything for a model without globals. */
  int32_t n_globals;
  int32_t n_links;
  const double *global_values;
  const uint8_t *global_fixed;
  const int32_t *link_global;
  const int32_t *link_table;
  const int32_t *link_param;
} fs_model;

/* ---- context ----------------------------------------------------------- */
enum fs_precision { FS_PREC_FP32 = 0, FS_PREC_FP64 = 1 };

typedef struct fs_gpu_opts {
  int32_t device;         /* CUDA ordinal                                  */
  int32_t precision;      /* fs_precision: FP32 compute + FP64 sums, or FP64 */
  int32_t lanes_per_atom; /* 0 = autotuned schedule, else 8 / 16 / 32      */
  int32_t reserved;
} fs_gpu_opts;

typedef struct fs_gpu fs_gpu;

int fs_gpu_create(const fs_gpu_opts *opts, fs_gpu **out);
int fs_gpu_destroy(fs_gpu *h);
/* Copies the last error message (NUL-terminated, truncated) into buf. */
int fs_gpu_last_error(const fs_gpu *h, char *buf, size_t size);
/* The CUDA stream every launch of this context is enqueued on. */
int fs_gpu_get_stream(fs_gpu *h, void **stream);

/*
 * Configurations, concatenated.  box9 is row-major 3×3 per config whose
 * COLUMNS are the lattice vectors X, Y, Z (config_reader.cpp:58-68).
 * pos / ref_force: 3 doubles per atom.  type: species slot per atom.
 * ref_stress9: row-major 3×3 per config.  ref_* may be NULL (zeros).
 */
int fs_gpu_upload_configs(fs_gpu *h, int32_t n_cfg, const int32_t *natoms,
                          const double *box9, const double *pos,
                          const int32_t *type, const double *ref_force,
                          const double *ref_energy, const double *ref_stress9);
/* Replace only the reference labels (same shapes as the upload). */
int fs_gpu_set_references(fs_gpu *h, const double *ref_force,
                          const double *ref_energy, const double *ref_stress9);

int fs_gpu_set_model(fs_gpu *h, const fs_model *model);
/* Builds the device neighbour lists at the model's max cutoff: device cell
 * lists (slabs at least the cutoff wide per lattice direction), the
 * reference's FP64 distance test on every candidate, then each atom's list
 * sorted into the reference's order.  For an FP32 EAM model whose pair and
 * density tables share one knot grid it also sorts each atom's pairs by
 * (neighbour species, segment) for the population kernel. */
int fs_gpu_prepare(fs_gpu *h);

int fs_gpu_num_pairs(fs_gpu *h, int64_t *n_pairs);
/* counts[total_atoms]; neighbours in the reference order (i, then j, then
 * image ix, iy, iz lexicographic): j is the config-local atom index,
 * img3 holds (ix, iy, iz) per pair. */
int fs_gpu_get_neighbor_counts(fs_gpu *h, int32_t *counts);
int fs_gpu_get_neighbors(fs_gpu *h, int32_t *j, int8_t *img3);

int fs_gpu_param_count(fs_gpu *h, int32_t *D);
int fs_gpu_gather_params(fs_gpu *h, double *x);
int fs_gpu_gather_bounds(fs_gpu *h, double *lo, double *hi);
int fs_gpu_set_params(fs_gpu *h, const double *x, int32_t D);

/* The model's interaction cut-off: CForceCalculator::max_cutoff
 * (force_calculator_concept.hpp:210-221; SW: max(a1, a2), stiweb_force.cpp:234-239). */
int fs_gpu_max_cutoff(fs_gpu *h, double *rc);

/* Value and d/dr of radial table `table` (model order; a spline or analytic
 * table) at the current parameters, at n points r[]: what the reference's
 * writers sample with RadialPotential::eval / deriv (output_writer.cpp:22-40,
 * 266-310).  Always FP64, whatever the context precision; a spline outside
 * its knot span gives its linear extension.  Other table kinds: FS_ERR_ARG.
 * Needs a model only (no configurations). */
int fs_gpu_tabulate(fs_gpu *h, int32_t table, int32_t n, const double *r, double *value, double *deriv);

/* rows = Σ_c 3N_c + 2 + (w_s > 0 ? 6 : 0)  (residual_layout.hpp:18-31) */
int fs_gpu_residual_count(fs_gpu *h, double w_s, int64_t *m);

/*
 * One residual evaluation over every configuration at the current params.
 * Every output is nullable.  F[m]: residual vector in the reference's row
 * order.  forces[3·Ntot], energy[n_cfg], stress9[9·n_cfg] (already /V),
 * limit[n_cfg]: the calculator outputs.  obj: ‖F‖² (FP64 sum).
 */
int fs_gpu_eval(fs_gpu *h, double w_e, double w_s, double *F, double *forces,
                double *energy, double *stress9, double *limit, double *obj);

/*
 * Residual + Jacobian.  J is column-major m × D (Eigen's fjac layout) in
 * FP64; JtJ is D × D and Jtr is D (FP64 accumulation).  Every output is
 * nullable; with J == NULL the Jacobian stays on the device.
 */
int fs_gpu_eval_jacobian(fs_gpu *h, double w_e, double w_s, double *F,
                         double *J, double *JtJ, double *Jtr, double *obj);

/*
 * Rows [row0, row0 + nrows) of the last evaluated Jacobian, FP64, into a
 * host column-major block: element (row0 + r, c) goes to J[c·ldJ + r]
 * (ldJ ≥ nrows).  With J = fjac.data() + row0 and ldJ = m this fills one
 * configuration's row block of Eigen's column-major `fjac`, as
 * ForceCalculator::eval_cached_jacobian does per configuration
 * (include/forcesmith/force/force_calculator.hpp:62-159, called from
 * df_cached_analytic, src/optimization/forcesmith_functor.cpp:111-132).
 * The widening to FP64 and the transpose run on the device.  Synchronous.
 */
int fs_gpu_copy_jacobian_rows(fs_gpu *h, int64_t row0, int64_t nrows, double *J, int64_t ldJ);

/* Device-resident variant: enqueues residual + Jacobian + JᵀJ + Jᵀr on the
 * context stream and returns without synchronising.  Results stay on the
 * device (fetch them with fs_gpu_fetch_normal_equations). */
int fs_gpu_eval_jacobian_async(fs_gpu *h, double w_e, double w_s);
int fs_gpu_fetch_normal_equations(fs_gpu *h, double *JtJ, double *Jtr,
                                  double *obj);

/*
 * Damped Gauss–Newton step from the last eval_jacobian:
 * solve (JᵀJ + λ·diag) dx = −Jᵀr by FP64 Cholesky on the device.
 * mode 0: diag = I (Levenberg); mode 1: diag = diag(JᵀJ) (Marquardt).
 */
int fs_gpu_lm_step(fs_gpu *h, double lambda, int32_t mode, double *dx);
/* NormalEquationsSolver step: λ = ridge > 0 ? ridge : 1e-8·max(mean diag,1);
 * dx = −(JᵀJ + λI)⁻¹ Jᵀr. */
int fs_gpu_lsq_step(fs_gpu *h, double ridge, double *dx);

/* ACSF and LMBTR models: per-species descriptor mean and 1/σ over every atom of the
 * uploaded configurations (MLBase::compute_standardization,
 * ml_force.hpp:644-688): σ² = E[D²] − E[D]², inv_std = σ² > 1e-12 ? 1/σ : 0.
 * mean, inv_std: nt × S (species-major); count: atoms per species (nt).
 * Descriptors are formed in the context precision, sums in FP64.  A model
 * with standardization tables is standardized by them; these statistics are
 * what such tables hold after the reference's prepare(). */
int fs_gpu_acsf_standardization(fs_gpu *h, double *mean, double *inv_std, int64_t *count);

/* Copies [JᵀJ (D·D), Jᵀr (D), ‖F‖² (1)] as FP64 into a caller-owned DEVICE
 * buffer, ordered on the context stream (for a collective over ranks). */
int fs_gpu_copy_normal_equations(fs_gpu *h, void *dst_device);

/*
 * Instrumentation.  With profiling on, every eval_jacobian records CUDA
 * events on the context stream between its phases (residual, per-atom
 * Jacobian, force/stress rows, JᵀJ/Jᵀr), for up to max_steps calls.
 * fs_gpu_phase_times synchronises, returns the summed milliseconds per phase
 * and the number of recorded calls, and resets.  fs_gpu_launch_count is the
 * number of kernels this context has launched.
 */
int fs_gpu_set_profiling(fs_gpu *h, int32_t max_steps);
int fs_gpu_phase_times(fs_gpu *h, double *ms, int32_t n, int32_t *steps);
int fs_gpu_launch_count(fs_gpu *h, int64_t *count);

/*
 * Failure detection (no reference counterpart: the reference has no device
 * waits).  Every wait inside this library's kernels has a cycle budget
 * (about 2 s); a wait that runs out sets the context's device error word,
 * the kernel returns, and the next synchronising call returns
 * FS_ERR_DEVICE, after which the context stays usable.
 * fs_gpu_check_bounded_wait exercises that path: one CTA waits, with a
 * budget of `cycles` (1 … 4e9) and the kernels' own wait routine, on a
 * barrier phase that never completes and has no copy or MMA bound to it.
 * It returns FS_ERR_DEVICE when the wait gave up and reported, as designed.
 *
 * Non-finite input: fs_gpu_set_params refuses a vector with a NaN or
 * infinite entry (FS_ERR_NUMERIC; the model keeps its previous values).
 * The population entry points evaluate rows as given: a non-finite entry
 * reaches the objective through the spline segments it enters (as in the
 * reference), so its row's objective turns non-finite when a pair reaches
 * them, and other rows are unaffected.  fs_gpu_lm_step refuses λ < 0
 * (FS_ERR_ARG) and returns FS_ERR_NUMERIC when JᵀJ + λ·diag is not
 * positive definite.
 */
int fs_gpu_check_bounded_wait(fs_gpu *h, int64_t cycles);

/* sizeof of the ABI's structs as this library was compiled, in the order
 * fs_table, fs_model, fs_gpu_opts, fs_tune_report, fs_de_opts,
 * fs_surrogate_opts, into sizes[0..n): a binding compares them with its own
 * declarations when it loads the library, so that a stale build fails at
 * load rather than writing past a caller's struct.  Returns the count. */
int fs_gpu_abi_sizes(int64_t *sizes, int32_t n);

/*
 * Batched objective: obj[k] = ‖F(x_k)‖² for NP parameter vectors xs[NP·D]
 * (row-major), all configurations, one launch.  The DE population kernel.
 */
int fs_gpu_eval_population(fs_gpu *h, double w_e, double w_s, const double *xs,
                           int32_t NP, double *obj);

/*
 * Schedule autotuner (no reference counterpart: the CPU path has no launch
 * shapes).  Times, on this context's configurations and model, the residual
 * kernel's lanes per atom (4, 8, 16, 32; skipped when fs_gpu_opts fixed it),
 * the Jacobian force-row kernel's warps per CTA (8 … 4) and, in FP32, the
 * population kernel's CTA waves (2, 4, 8), and keeps the fastest for every
 * later call of this context.  Results differ between schedules only in the
 * summation order of their sums.  Milliseconds per candidate are reported
 * (0 where a candidate was not timed).
 */
typedef struct fs_tune_report {
    int32_t lanes_per_atom, k2_warps, pop_waves, reserved;
    double residual_ms[4];    /* lanes 4, 8, 16, 32 */
    double jacobian_ms[5];    /* warps 11, 10, 8, 6, 4 (infinite: not tried) */
    double population_ms[3];  /* waves 2, 4, 8 */
} fs_tune_report;

int fs_gpu_autotune(fs_gpu *h, double w_e, double w_s, fs_tune_report *report);

/*
 * fs_gpu_eval_population_noalloc — the batched objective of
 * fs_gpu_eval_population for callers that cannot allocate device memory.
 * No counterpart in the reference (its DE evaluates trials one at a time on
 * the CPU).
 *
 * Who needs it: a host that has handed all of the GPU's memory to its own
 * pool and forbids further cudaMalloc, or a latency-critical loop that must
 * not call cudaMalloc / cudaFree because they can synchronise the device.
 * This call allocates nothing and frees nothing: the caller passes device
 * buffers xs_dev (NP × D doubles, row-major) and obj_dev (NP doubles) on the
 * context's GPU, and the kernels' scratch (per-trial spline segments and
 * per-(trial, configuration) partial sums) lives in one fixed 8 MiB device
 * array inside the library, which every GPU that loads the library holds
 * until the process exits.  NP whose scratch would exceed 8 MiB is rejected
 * with FS_ERR_ARG and a message giving the largest NP that fits (about 1000
 * trials for 500 configurations of a 12-table EAM model in FP32).
 *
 * Results equal fs_gpu_eval_population's (same kernels; configurations are
 * taken heaviest first, in the order the context keeps from its neighbour
 * lists, with the autotuned CTA waves).  The call is
 * asynchronous on the context's stream (fs_gpu_get_stream): obj_dev is ready
 * once that stream reaches it.  The context must have been prepared
 * (fs_gpu_prepare) with its configurations and model; EAM or pair family,
 * spline tables.
 *
 * The first call on each GPU looks up the array's device address (a
 * runtime query, no allocation); make that first call before any stream
 * capture.  fs_gpu_create drops the looked-up address of its device, so
 * after a cudaDeviceReset (which invalidates every existing context) the
 * first call of a newly created context looks it up again.  All calls in the process share the one array and it keeps the
 * previous call's contents; every byte a call reads it has written first,
 * so nothing needs clearing, but two calls whose kernels overlap on the
 * same GPU (two contexts, two streams) race on it — serialise them.
 */
int fs_gpu_eval_population_noalloc(fs_gpu *h, double w_e, double w_s,
                                   const double *xs_dev, int32_t NP,
                                   double *obj_dev);

/*
 * Differential evolution on the device — replaces BoostDESolver::solve
 * (src/optimization/solver.cpp:113-155; DEParams: NP, mutation F, crossover
 * CR, seed, max_generations).  DE/rand/1/bin with box clamping and greedy
 * selection; a generation is trial construction, the batched objective
 * (fs_gpu_eval_population's kernels) and selection, captured once as a CUDA
 * graph and replayed when use_graph != 0.  Random numbers are a counter hash
 * of (seed, generation, member), so a run is reproducible for a given seed;
 * it does not reproduce Boost.Math's random stream.
 *
 * fs_gpu_de_init: population member 0 = clamp(x0) when x0 != NULL, the rest
 * uniform in [lo, hi]; evaluates the initial population.  Any later
 * fs_gpu_upload_configs / fs_gpu_set_model discards the DE state.
 * fs_gpu_de_run: `generations` more generations; writes the best objective
 * and vector, and when history != NULL the best objective after each
 * generation (recorded on the device, copied back once at the end).
 * fs_gpu_de_population: copies the population (NP·D) and its objectives.
 */
typedef struct fs_de_opts {
    int32_t NP;        /* population size, >= 4 */
    int32_t reserved;
    double mutation;   /* F  (reference default 0.65) */
    double crossover;  /* CR (reference default 0.5)  */
    uint64_t seed;
    double w_e, w_s;   /* energy / stress weights of the objective */
} fs_de_opts;

int fs_gpu_de_init(fs_gpu *h, const fs_de_opts *opts, const double *lo,
                   const double *hi, const double *x0);
int fs_gpu_de_run(fs_gpu *h, int32_t generations, int32_t use_graph,
                  double *best_obj, double *best_x, double *history);
int fs_gpu_de_population(fs_gpu *h, double *pop, double *obj);

/*
 * Surrogate-screened DE (no reference counterpart: the reference evaluates
 * every DE trial exactly).  A BF16 MLP  D → 256 → 256 → 1  (GELU, FP32
 * accumulation, tcgen05 tensor cores) is trained with Adam on the log of
 * every exact objective the run computes.  After `warm_generations` plain
 * generations, each generation draws `screen` candidate trials per member,
 * the model ranks them, and only each member's best-ranked candidate is
 * evaluated exactly; the exact objective alone decides acceptance.  Every
 * round(1/holdout)-th archive row is held out of training; when the model's
 * Spearman correlation on the newest held-out rows (at most 2048) is below
 * `gate`, the next generation is plain DE.  D ≤ 256.
 *
 * fs_gpu_surrogate_init: (re)creates the model (uniform ±1/√fan-in weights
 * from `seed`, zero biases) and an empty archive for the current model's D.
 * fs_gpu_de_run_screened: like fs_gpu_de_run (after fs_gpu_de_init); rho and
 * screened (nullable, `generations` entries) report the gate's correlation
 * and whether each generation was screened.
 *
 * Model access (tests and tools): parameters are FP32 in the order
 * W1 [256 × D] row-major, b1 [256], W2 [256 × 256], b2 [256], w3 [256],
 * b3 [1].  Inputs x are FP32 rows of D features (the DE run uses
 * 2(x − lo)/(hi − lo) − 1); loss = mean (y − t)²; gradient rows >= 8 and a
 * multiple of 8.
 */
typedef struct fs_surrogate_opts {
    int32_t screen;               /* candidates per member (4)                  */
    int32_t warm_generations;     /* plain generations before screening (5)     */
    int32_t batch;                /* training batch, multiple of 8 (512)        */
    int32_t steps_per_generation; /* Adam steps after each generation (32)      */
    double lr;                    /* Adam learning rate (1e-3)                  */
    double gate;                  /* Spearman threshold (0.8)                   */
    double holdout;               /* held-out fraction of the archive (0.1)     */
    uint64_t seed;
    int64_t archive_rows;         /* archive capacity, 0 = every evaluation     */
} fs_surrogate_opts;

int fs_gpu_surrogate_init(fs_gpu *h, const fs_surrogate_opts *opts);
int fs_gpu_de_run_screened(fs_gpu *h, int32_t generations, double *best_obj,
                           double *best_x, double *history, double *rho,
                           int32_t *screened);
int fs_gpu_surrogate_param_count(fs_gpu *h, int64_t *n);
int fs_gpu_surrogate_get_params(fs_gpu *h, float *params);
int fs_gpu_surrogate_set_params(fs_gpu *h, const float *params);
int fs_gpu_surrogate_predict(fs_gpu *h, const float *x, int32_t rows, float *y);
int fs_gpu_surrogate_gradient(fs_gpu *h, const float *x, const float *t,
                              int32_t rows, float *grad, float *loss);
int fs_gpu_surrogate_train(fs_gpu *h, const float *x, const float *t,
                           int32_t rows, int32_t steps, float *loss);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* FORCESMITH_GPU_H */
