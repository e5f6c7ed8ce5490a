// The C ABI of include/forcesmith_gpu.h: context lifecycle, configuration
// and model upload, parameter scatter, and the evaluate entry points.
#include "forms_dev.cuh"
#include "internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

using namespace fsg;

namespace fsg {

int set_error(fs_gpu *h, int code, const std::string &m) {
  if (h) h->err = m;
  return code;
}

namespace {

template <class X> int dalloc(fs_gpu *h, X **p, size_t n) {
  if (*p) {
    cudaFree(*p);
    *p = nullptr;
  }
  if (n == 0) return FS_OK;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), n * sizeof(X));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_error(h, FS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  return FS_OK;
}

template <class X> void dfree(X *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// 3×3 inverse by the adjugate with the determinant taken from the first
// cofactor column (the order Eigen 3.4 uses for fixed 3×3 inverses, which
// the reference's PeriodicBC::set_box calls, boundary_conditions.hpp:19-28).
void inverse3(const double *m, double *r) {
  auto M = [&](int i, int j) { return m[3 * i + j]; };
  auto cof = [&](int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return M(i1, j1) * M(i2, j2) - M(i1, j2) * M(i2, j1);
  };
  const double c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
  const double det = c00 * M(0, 0) + c10 * M(1, 0) + c20 * M(2, 0);
  const double id = 1.0 / det;
  r[0] = c00 * id;
  r[1] = c10 * id;
  r[2] = c20 * id;
  r[3] = cof(0, 1) * id;
  r[4] = cof(1, 1) * id;
  r[5] = cof(2, 1) * id;
  r[6] = cof(0, 2) * id;
  r[7] = cof(1, 2) * id;
  r[8] = cof(2, 2) * id;
}

double det3(const double *m) {
  auto M = [&](int i, int j) { return m[3 * i + j]; };
  auto hh = [&](int a, int b, int c) { return M(0, a) * (M(1, b) * M(2, c) - M(1, c) * M(2, b)); };
  return hh(0, 1, 2) - hh(1, 0, 2) + hh(2, 0, 1);
}

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

int ensure_eval_buffers(fs_gpu *h, double w_s) {
  const int64_t rows = rows_of(h, 1.0); // the larger layout (with stress rows)
  (void)w_s;
  if (h->rows_alloc < rows) {
    FS_TRY(dalloc(h, &h->d_F, rows));
    h->rows_alloc = rows;
  }
  if (!h->d_forces) {
    FS_TRY(dalloc(h, &h->d_forces, 3 * h->n_atoms));
    FS_TRY(dalloc(h, &h->d_energy, h->n_cfg));
    FS_TRY(dalloc(h, &h->d_stress9, 9 * static_cast<size_t>(h->n_cfg)));
    FS_TRY(dalloc(h, &h->d_limit, h->n_cfg));
    FS_TRY(dalloc(h, &h->d_obj_part, h->n_cfg));
    FS_TRY(dalloc(h, &h->d_obj, 1));
  }
  return FS_OK;
}

void free_configs(fs_gpu *h) {
  dfree(h->d_cfg);
  dfree(h->d_pos);
  dfree(h->d_wpos);
  dfree(h->d_type);
  dfree(h->d_ref_force);
  dfree(h->d_nb_start);
  dfree(h->d_nb_pack);
  dfree(h->d_nb_count);
  dfree(h->d_cfg_by_work);
  h->max_cfg_work = 0;
  dfree(h->d_run_a);
  dfree(h->d_run_b);
  dfree(h->d_run_cnt);
  dfree(h->d_run_r);
  h->runs_valid = false;
  h->max_list = -1;
  dfree(h->d_F);
  dfree(h->d_forces);
  dfree(h->d_energy);
  dfree(h->d_stress9);
  dfree(h->d_limit);
  dfree(h->d_obj_part);
  dfree(h->d_obj);
  dfree(h->d_pop_seg_a);
  h->pop_alloc = 0;
  fsg::de_free(h->de);
  h->de = nullptr;
  fsg::surrogate_free(h->sur);
  h->sur = nullptr;
  h->rows_alloc = 0;
  h->rcut_built = -1.0;
  h->n_pairs = 0;
  h->jac_valid = false;
}

void free_jacobian(fs_gpu *h) {
  dfree(h->d_J);
  dfree(h->d_JtJ);
  dfree(h->d_Jtr);
  dfree(h->d_gram_part);
  dfree(h->d_jtr_part);
  h->jtr_part_alloc = 0;
  dfree(h->d_half_part);
  h->half_part_alloc = 0;
  dfree(h->d_fd_scratch);
  h->fd_scratch_alloc = 0;
  dfree(h->d_atom_scalars);
  dfree(h->d_drho);
  dfree(h->d_dgd);
  dfree(h->d_wsF);
  dfree(h->d_jx);
  h->jx_alloc = 0;
  dfree(h->d_an);
  h->an_alloc = 0;
  h->jac_alloc = 0;
  h->gram_part_alloc = 0;
  h->atom_scratch_alloc = 0;
  h->jac_valid = false;
}

int sync(fs_gpu *h) {
  cudaError_t e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return set_error(h, FS_ERR_CUDA, std::string("kernel: ") + cudaGetErrorString(e));
  if (h->d_err) { // a bounded device wait gave up
    int32_t flag = 0;
    cudaMemcpy(&flag, h->d_err, sizeof(int32_t), cudaMemcpyDeviceToHost);
    if (flag) {
      cudaMemset(h->d_err, 0, sizeof(int32_t));
      return set_error(h, FS_ERR_DEVICE, "a device-side wait timed out (results discarded)");
    }
  }
  return FS_OK;
}

int ensure_params(fs_gpu *h) {
  if (h->params_dirty) {
    FS_TRY(refresh_segments(h));
    h->params_dirty = false;
  }
  return FS_OK;
}

int check_ready(fs_gpu *h) {
  if (!h) return FS_ERR_ARG;
  if (h->n_cfg == 0) return set_error(h, FS_ERR_STATE, "no configurations uploaded");
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "no model set");
  if (h->rcut_built < 0) return set_error(h, FS_ERR_STATE, "fs_gpu_prepare not called");
  return FS_OK;
}

} // namespace

int sync_checked(fs_gpu *h) { return sync(h); }

} // namespace fsg

extern "C" {

int fs_gpu_create(const fs_gpu_opts *opts, fs_gpu **out) {
  if (!out) return FS_ERR_ARG;
  *out = nullptr;
  fs_gpu *h = new fs_gpu();
  if (opts) {
    h->device = opts->device;
    h->precision = opts->precision;
    h->lanes_per_atom = opts->lanes_per_atom;
  }
  if (h->precision != FS_PREC_FP32 && h->precision != FS_PREC_FP64) {
    delete h;
    return FS_ERR_ARG;
  }
  if (h->lanes_per_atom != 0 && h->lanes_per_atom != 4 && h->lanes_per_atom != 8 &&
      h->lanes_per_atom != 16 && h->lanes_per_atom != 32) {
    delete h;
    return FS_ERR_ARG;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || h->device < 0 || h->device >= ndev) {
    delete h;
    return FS_ERR_CUDA;
  }
  if (cudaSetDevice(h->device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->vals_ev, cudaEventDisableTiming) != cudaSuccess) {
    if (h->stream) cudaStreamDestroy(h->stream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->vals_ev) cudaEventDestroy(h->vals_ev);
    delete h;
    return FS_ERR_CUDA;
  }
  fsg::noalloc_forget(h->device);
  *out = h;
  return FS_OK;
}

int fs_gpu_destroy(fs_gpu *h) {
  if (!h) return FS_OK;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_configs(h);
  free_jacobian(h);
  dfree(h->d_desc);
  dfree(h->d_cmap);
  dfree(h->d_vals);
  dfree(h->d_seg_a);
  dfree(h->d_seg_g);
  dfree(h->d_seg_ws);
  dfree(h->d_spl);
  if (h->h_vals_pin) cudaFreeHost(h->h_vals_pin);
  if (h->h_ne_pin) cudaFreeHost(h->h_ne_pin);
  if (h->vals_ev) cudaEventDestroy(h->vals_ev);
  dfree(h->d_x);
  dfree(h->d_chol);
  dfree(h->d_dx);
  dfree(h->d_flag);
  fsg::mlp_free(h->mlp);
  h->mlp = nullptr;
  dfree(h->d_pop_spl);
  dfree(h->d_pop_vals);
  dfree(h->d_pop_obj);
  dfree(h->d_err);
  for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
  if (h->side) {
    cudaStreamSynchronize(h->side);
    cudaStreamDestroy(h->side);
    cudaEventDestroy(h->ev_fork);
    cudaEventDestroy(h->ev_join);
  }
  cudaStreamDestroy(h->stream);
  delete h;
  return FS_OK;
}

int fs_gpu_last_error(const fs_gpu *h, char *buf, size_t size) {
  if (!h || !buf || size == 0) return FS_ERR_ARG;
  const size_t n = std::min(size - 1, h->err.size());
  std::memcpy(buf, h->err.data(), n);
  buf[n] = '\0';
  return FS_OK;
}

int fs_gpu_get_stream(fs_gpu *h, void **stream) {
  if (!h || !stream) return FS_ERR_ARG;
  *stream = reinterpret_cast<void *>(h->stream);
  return FS_OK;
}

int fs_gpu_upload_configs(fs_gpu *h, int32_t n_cfg, const int32_t *natoms, const double *box9,
                          const double *pos, const int32_t *type, const double *ref_force,
                          const double *ref_energy, const double *ref_stress9) {
  if (!h || n_cfg <= 0 || !natoms || !box9 || !pos || !type)
    return set_error(h, FS_ERR_ARG, "upload_configs: null input or n_cfg <= 0");
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  free_configs(h);
  free_jacobian(h);
  h->n_cfg = n_cfg;
  h->natoms.assign(natoms, natoms + n_cfg);
  h->atom0.assign(n_cfg, 0);
  h->cfg_host.assign(n_cfg, CfgDev{});
  int64_t off = 0;
  int maxn = 0;
  for (int c = 0; c < n_cfg; ++c) {
    if (natoms[c] < 0 || natoms[c] > (1 << 20) - 1)
      return set_error(h, FS_ERR_ARG, "upload_configs: natoms out of range");
    h->atom0[c] = off;
    CfgDev &cd = h->cfg_host[c];
    cd.atom0 = static_cast<int>(off);
    cd.natoms = natoms[c];
    for (int k = 0; k < 9; ++k) cd.box[k] = box9[9 * c + k];
    const double det = det3(cd.box);
    bool finite = std::isfinite(det);
    for (int k = 0; k < 9; ++k) finite = finite && std::isfinite(cd.box[k]);
    if (finite && det != 0.0) {
      inverse3(cd.box, cd.inv);
    } else {
      for (int k = 0; k < 9; ++k) cd.inv[k] = (k % 4 == 0) ? 1.0 : 0.0;
    }
    cd.volume = std::isfinite(det) ? std::abs(det) : 0.0;
    cd.ref_energy = ref_energy ? ref_energy[c] : 0.0;
    for (int k = 0; k < 9; ++k) cd.ref_stress[k] = ref_stress9 ? ref_stress9[9 * c + k] : 0.0;
    off += natoms[c];
    maxn = std::max(maxn, natoms[c]);
  }
  if (off > std::numeric_limits<int32_t>::max() / 4)
    return set_error(h, FS_ERR_UNSUPPORTED, "upload_configs: too many atoms");
  h->n_atoms = off;
  h->max_natoms = maxn;
  h->max_type = 0;
  for (int64_t i = 0; i < off; ++i) {
    if (type[i] < 0 || type[i] > 255) return set_error(h, FS_ERR_ARG, "upload_configs: bad type");
    h->max_type = std::max(h->max_type, static_cast<int>(type[i]));
  }
  FS_TRY(dalloc(h, &h->d_cfg, n_cfg));
  FS_TRY(dalloc(h, &h->d_pos, 3 * off));
  FS_TRY(dalloc(h, &h->d_wpos, 3 * off));
  FS_TRY(dalloc(h, &h->d_type, off));
  FS_TRY(dalloc(h, &h->d_ref_force, 3 * off));
  FS_CUDA(cudaMemcpyAsync(h->d_pos, pos, 3 * off * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(h->d_type, type, off * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
  if (ref_force)
    FS_CUDA(cudaMemcpyAsync(h->d_ref_force, ref_force, 3 * off * sizeof(double),
                            cudaMemcpyHostToDevice, h->stream));
  else
    FS_CUDA(cudaMemsetAsync(h->d_ref_force, 0, 3 * off * sizeof(double), h->stream));
  FS_CUDA(cudaMemcpyAsync(h->d_cfg, h->cfg_host.data(), n_cfg * sizeof(CfgDev),
                          cudaMemcpyHostToDevice, h->stream));
  FS_TRY(sync(h));
  return FS_OK;
}

int fs_gpu_set_references(fs_gpu *h, const double *ref_force, const double *ref_energy,
                          const double *ref_stress9) {
  if (!h || h->n_cfg == 0) return FS_ERR_STATE;
  cudaSetDevice(h->device);
  for (int c = 0; c < h->n_cfg; ++c) {
    h->cfg_host[c].ref_energy = ref_energy ? ref_energy[c] : 0.0;
    for (int k = 0; k < 9; ++k) h->cfg_host[c].ref_stress[k] = ref_stress9 ? ref_stress9[9 * c + k] : 0.0;
  }
  if (ref_force)
    FS_CUDA(cudaMemcpyAsync(h->d_ref_force, ref_force, 3 * h->n_atoms * sizeof(double),
                            cudaMemcpyHostToDevice, h->stream));
  else
    FS_CUDA(cudaMemsetAsync(h->d_ref_force, 0, 3 * h->n_atoms * sizeof(double), h->stream));
  // pair0 lives in cfg_host too; re-upload the whole array
  FS_CUDA(cudaMemcpyAsync(h->d_cfg, h->cfg_host.data(), h->n_cfg * sizeof(CfgDev),
                          cudaMemcpyHostToDevice, h->stream));
  return sync(h);
}

int fs_gpu_set_model(fs_gpu *h, const fs_model *m) {
  if (!h || !m) return FS_ERR_ARG;
  if (m->ntypes < 1 || m->ntypes > 16) return set_error(h, FS_ERR_ARG, "set_model: ntypes out of range");
  // ACSF and LMBTR models may carry standardization tables after the heads
  const bool ml_fam = m->family == FS_FAMILY_ACSF || m->family == FS_FAMILY_LMBTR;
  const bool acsf_std = ml_fam && m->n_tables == 1 + 2 * m->ntypes;
  if ((expected_tables(m->family, m->ntypes) != m->n_tables && !acsf_std) || !m->tables)
    return set_error(h, FS_ERR_ARG, "set_model: table count does not match the family");
  const int np = npair_of(m->ntypes);
  // global parameters: links (table, slot) → global
  const int ng = m->n_globals, nl = m->n_links;
  if (ng < 0 || nl < 0 || (ng > 0 && !m->global_values) ||
      (nl > 0 && (!m->link_global || !m->link_table || !m->link_param)))
    return set_error(h, FS_ERR_ARG, "set_model: malformed global parameter arrays");
  if (ng > 0 && m->family != FS_FAMILY_EAM && m->family != FS_FAMILY_PAIR)
    return set_error(h, FS_ERR_ARG, "set_model: global parameters belong to the pair and EAM families");
  std::vector<std::vector<int>> link_of(m->n_tables);
  for (int l = 0; l < nl; ++l) {
    const int g = m->link_global[l], t = m->link_table[l], k = m->link_param[l];
    if (g < 0 || g >= ng || t < 0 || t >= m->n_tables)
      return set_error(h, FS_ERR_ARG, "set_model: global link " + std::to_string(l) + " out of range");
    const fs_table &ft = m->tables[t];
    if (ft.kind != FS_TABLE_ANALYTIC || k < 0 || k >= ft.n)
      return set_error(h, FS_ERR_ARG,
                       "set_model: global link " + std::to_string(l) + " is not a parameter of an analytic table");
    if (link_of[t].empty()) link_of[t].assign(ft.n, -1);
    if (link_of[t][k] >= 0) return set_error(h, FS_ERR_ARG, "set_model: a parameter linked to two globals");
    link_of[t][k] = g;
  }
  for (int g = 0; g < ng; ++g)
    if (!std::isfinite(m->global_values[g]))
      return set_error(h, FS_ERR_ARG, "set_model: global " + std::to_string(g) + " is not finite");
  std::vector<HostTable> tabs(m->n_tables);
  int col = 0;
  for (int t = 0; t < m->n_tables; ++t) {
    const fs_table &ft = m->tables[t];
    HostTable &ht = tabs[t];
    if (ft.n < 1 || !ft.values) return set_error(h, FS_ERR_ARG, "set_model: empty table");
    ht.kind = ft.kind;
    ht.form = ft.form;
    ht.n = ft.n;
    ht.rmin = ft.rmin;
    ht.rmax = ft.rmax;
    const bool sw_fam = m->family == FS_FAMILY_SW;
    if (m->family == FS_FAMILY_ACSF) {
      // the descriptor table {rcut, nG1..nG5, parameters}, then one linear head
      // {w[S], b} per species, then optionally one standardization
      // {mean[S], inv_std[S]} per species, all fixed
      const fs_table &spec = m->tables[0];
      bool ok = spec.kind == FS_TABLE_ACSF && spec.n >= 6 && spec.values[0] > 0.0;
      int need = 6;
      for (int k = 1; ok && k < 6; ++k) ok = spec.values[k] >= 0 && spec.values[k] == std::floor(spec.values[k]);
      if (ok) {
        need += 2 * static_cast<int>(spec.values[2]) + static_cast<int>(spec.values[3]) +
                3 * static_cast<int>(spec.values[4]) + 3 * static_cast<int>(spec.values[5]);
        ok = spec.n == need;
      }
      if (!ok) return set_error(h, FS_ERR_ARG, "set_model: ACSF table {rcut, nG1..nG5, parameters} is malformed");
      if (t > 0) {
        const int nt = m->ntypes, P = nt * (nt + 1) / 2;
        const int S = nt * static_cast<int>(spec.values[1] + spec.values[2] + spec.values[3]) +
                      P * static_cast<int>(spec.values[4] + spec.values[5]);
        if (t <= nt && (ft.kind != FS_TABLE_LINEAR_HEAD || ft.n != S + 1))
          return set_error(h, FS_ERR_ARG, "set_model: ACSF heads are linear_head[nt] with S + 1 values");
        if (t > nt) {
          bool fixed = ft.fixed != nullptr;
          for (int k = 0; fixed && k < ft.n; ++k) fixed = ft.fixed[k] != 0;
          if (ft.kind != FS_TABLE_STANDARDIZATION || ft.n != 2 * S || !fixed)
            return set_error(h, FS_ERR_ARG,
                             "set_model: ACSF standardization tables hold {mean[S], inv_std[S]}, all fixed");
        }
      }
    } else if (m->family == FS_FAMILY_LMBTR) {
      // the descriptor table {rcut, weight_scale, normalize, n2, min2, max2,
      // sigma2, n3, min3, max3, sigma3}, then the heads and optional
      // standardization tables as for ACSF
      const fs_table &spec = m->tables[0];
      const double *v = spec.values;
      bool ok = spec.kind == FS_TABLE_LMBTR && spec.n == 11 && v[0] > 0.0 && v[1] > 0.0 && v[3] + v[7] > 0;
      for (int k : {3, 7})
        ok = ok && v[k] >= 0 && v[k] == std::floor(v[k]) && v[k] < 1e6 && (v[k] == 0 || v[k + 3] > 0.0) &&
             std::isfinite(v[k + 1]) && std::isfinite(v[k + 2]) && (v[k] <= 1 || v[k + 2] > v[k + 1]);
      if (!ok)
        return set_error(h, FS_ERR_ARG,
                         "set_model: LMBTR table {rcut, weight_scale, normalize, n2, min2, max2, sigma2, n3, min3, "
                         "max3, sigma3} is malformed");
      if (t > 0) {
        const int nt = m->ntypes, P = nt * (nt + 1) / 2;
        const int S = nt * static_cast<int>(v[3]) + P * static_cast<int>(v[7]);
        if (t <= nt && (ft.kind != FS_TABLE_LINEAR_HEAD || ft.n != S + 1))
          return set_error(h, FS_ERR_ARG, "set_model: LMBTR heads are linear_head[nt] with S + 1 values");
        if (t > nt) {
          bool fixed = ft.fixed != nullptr;
          for (int k = 0; fixed && k < ft.n; ++k) fixed = ft.fixed[k] != 0;
          if (ft.kind != FS_TABLE_STANDARDIZATION || ft.n != 2 * S || !fixed)
            return set_error(h, FS_ERR_ARG,
                             "set_model: LMBTR standardization tables hold {mean[S], inv_std[S]}, all fixed");
        }
      }
    } else if (ft.kind == FS_TABLE_ACSF || ft.kind == FS_TABLE_LINEAR_HEAD || ft.kind == FS_TABLE_STANDARDIZATION ||
               ft.kind == FS_TABLE_LMBTR) {
      return set_error(h, FS_ERR_ARG, "set_model: descriptor tables belong to the ACSF and LMBTR families");
    } else if (m->family == FS_FAMILY_TERSOFF) {
      if (ft.kind != FS_TABLE_TERSOFF || ft.n != 12)
        return set_error(h, FS_ERR_ARG, "set_model: Tersoff tables are tersoff[npair] with 12 params");
    } else if (ft.kind == FS_TABLE_TERSOFF) {
      return set_error(h, FS_ERR_ARG, "set_model: Tersoff tables belong to the Tersoff family");
    } else if (sw_fam) {
      const int want = t < np ? FS_TABLE_SW : FS_TABLE_LAMBDA;
      if (ft.kind != want) return set_error(h, FS_ERR_ARG, "set_model: SW tables are sw[npair], lambda");
      if (t < np && ft.n != 8) return set_error(h, FS_ERR_ARG, "set_model: SW table needs 8 params");
      if (t == np && ft.n != m->ntypes * np)
        return set_error(h, FS_ERR_ARG, "set_model: lambda needs ntypes*npair values");
    } else if (ft.kind == FS_TABLE_SPLINE) {
      if (ft.n < 2 || !(ft.rmax > ft.rmin)) return set_error(h, FS_ERR_ARG, "set_model: bad spline");
    } else if (ft.kind == FS_TABLE_ANALYTIC) {
      if (m->family != FS_FAMILY_EAM && m->family != FS_FAMILY_PAIR && m->family != FS_FAMILY_ANGULAR &&
          m->family != FS_FAMILY_ADP)
        return set_error(h, FS_ERR_UNSUPPORTED,
                         "set_model: analytic tables in EAM, pair, ADP and angular models only");
      if (ft.form < 0 || ft.form >= FS_FORM_COUNT || ft.n != fsg::form_param_count(ft.form))
        return set_error(h, FS_ERR_ARG, "set_model: analytic form and parameter count do not match");
      if (!(ft.rmax >= ft.rmin)) return set_error(h, FS_ERR_ARG, "set_model: bad analytic gate span");
    } else {
      return set_error(h, FS_ERR_ARG, "set_model: bad table kind");
    }
    ht.v.assign(ft.values, ft.values + ft.n);
    ht.fixed.assign(ft.n, 0);
    ht.lo.assign(ft.n, -std::numeric_limits<double>::infinity());
    ht.hi.assign(ft.n, std::numeric_limits<double>::infinity());
    ht.cols.assign(ft.n, -1);
    for (int k = 0; k < ft.n; ++k) {
      if (ft.fixed) ht.fixed[k] = ft.fixed[k] ? 1 : 0;
      if (ht.kind != FS_TABLE_SPLINE) {
        if (ft.lower) ht.lo[k] = ft.lower[k];
        if (ft.upper) ht.hi[k] = ft.upper[k];
      }
      if (!link_of[t].empty() && link_of[t][k] >= 0) {
        // finalize_globals: the linked slot is fixed at the global's value
        ht.fixed[k] = 1;
        ht.v[k] = m->global_values[link_of[t][k]];
        ht.lo[k] = -std::numeric_limits<double>::infinity();
        ht.hi[k] = std::numeric_limits<double>::infinity();
      }
      if (!ht.fixed[k]) ht.cols[k] = col++;
    }
  }
  // free globals take the columns after the tables'; their links share them
  std::vector<double> gval(m->global_values, m->global_values + ng);
  std::vector<int> gcol(ng, -1);
  for (int g = 0; g < ng; ++g)
    if (!(m->global_fixed && m->global_fixed[g])) gcol[g] = col++;
  for (int t = 0; t < m->n_tables; ++t)
    for (int k = 0; k < static_cast<int>(link_of[t].size()); ++k)
      if (link_of[t][k] >= 0) tabs[t].cols[k] = gcol[link_of[t][k]];
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  h->family = m->family;
  h->ntypes = m->ntypes;
  h->tables = std::move(tabs);
  h->global_val = std::move(gval);
  h->global_col = std::move(gcol);
  h->shared_cols = nl > 0 && std::any_of(h->global_col.begin(), h->global_col.end(), [](int c) { return c >= 0; });
  h->D = col;
  h->have_model = true;
  h->rcut_built = -1.0;
  h->jac_valid = false;
  h->runs_valid = false; // the pair runs depend on the model's knot grid
  free_jacobian(h);
  fsg::de_free(h->de);
  h->de = nullptr;
  fsg::surrogate_free(h->sur);
  h->sur = nullptr;
  fsg::mlp_free(h->mlp);
  h->mlp = nullptr;
  dfree(h->d_pop_spl);
  h->pop_spl_count = 0;
  FS_TRY(upload_tables(h));
  h->params_dirty = true;
  return FS_OK;
}

int fs_gpu_prepare(fs_gpu *h) {
  if (!h) return FS_ERR_ARG;
  if (h->n_cfg == 0) return set_error(h, FS_ERR_STATE, "prepare: no configurations");
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "prepare: no model");
  if (h->max_type >= h->ntypes)
    return set_error(h, FS_ERR_ARG, "prepare: an atom's species slot is >= the model's ntypes");
  cudaSetDevice(h->device);
  FS_TRY(build_neighbors(h, model_max_cutoff(h)));
  FS_TRY(ensure_eval_buffers(h, 1.0));
  return FS_OK;
}

int fs_gpu_num_pairs(fs_gpu *h, int64_t *n) {
  if (!h || !n) return FS_ERR_ARG;
  if (h->rcut_built < 0) return set_error(h, FS_ERR_STATE, "no neighbour lists");
  *n = h->n_pairs;
  return FS_OK;
}

int fs_gpu_get_neighbor_counts(fs_gpu *h, int32_t *counts) {
  if (!h || !counts) return FS_ERR_ARG;
  if (h->rcut_built < 0) return set_error(h, FS_ERR_STATE, "no neighbour lists");
  cudaSetDevice(h->device);
  FS_CUDA(cudaMemcpyAsync(counts, h->d_nb_count, h->n_atoms * sizeof(int32_t),
                          cudaMemcpyDeviceToHost, h->stream));
  return sync(h);
}

int fs_gpu_get_neighbors(fs_gpu *h, int32_t *j, int8_t *img3) {
  if (!h) return FS_ERR_ARG;
  if (h->rcut_built < 0) return set_error(h, FS_ERR_STATE, "no neighbour lists");
  cudaSetDevice(h->device);
  std::vector<uint32_t> pack(h->n_pairs);
  FS_CUDA(cudaMemcpyAsync(pack.data(), h->d_nb_pack, h->n_pairs * sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, h->stream));
  FS_TRY(sync(h));
  for (int c = 0; c < h->n_cfg; ++c) {
    const CfgDev &cd = h->cfg_host[c];
    const int wy = 2 * cd.sy + 1, wz = 2 * cd.sz + 1;
    const int64_t p0 = cd.pair0;
    const int64_t p1 = (c + 1 < h->n_cfg) ? h->cfg_host[c + 1].pair0 : h->n_pairs;
    for (int64_t p = p0; p < p1; ++p) {
      const uint32_t v = pack[p];
      if (j) j[p] = static_cast<int32_t>(v & 0xFFFFFu);
      const int img = static_cast<int>(v >> 20);
      if (img3) {
        img3[3 * p + 0] = static_cast<int8_t>(img / (wy * wz) - cd.sx);
        img3[3 * p + 1] = static_cast<int8_t>((img / wz) % wy - cd.sy);
        img3[3 * p + 2] = static_cast<int8_t>(img % wz - cd.sz);
      }
    }
  }
  return FS_OK;
}

int fs_gpu_param_count(fs_gpu *h, int32_t *D) {
  if (!h || !D) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "no model");
  *D = h->D;
  return FS_OK;
}

int fs_gpu_gather_params(fs_gpu *h, double *x) {
  if (!h || !x) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "no model");
  for (const HostTable &t : h->tables)
    for (int k = 0; k < t.n; ++k)
      if (t.cols[k] >= 0) x[t.cols[k]] = t.v[k];
  for (size_t g = 0; g < h->global_col.size(); ++g)
    if (h->global_col[g] >= 0) x[h->global_col[g]] = h->global_val[g];
  return FS_OK;
}

int fs_gpu_gather_bounds(fs_gpu *h, double *lo, double *hi) {
  if (!h || !lo || !hi) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "no model");
  for (const HostTable &t : h->tables)
    for (int k = 0; k < t.n; ++k)
      if (t.cols[k] >= 0) {
        lo[t.cols[k]] = t.lo[k];
        hi[t.cols[k]] = t.hi[k];
      }
  for (size_t g = 0; g < h->global_col.size(); ++g)
    if (h->global_col[g] >= 0) {
      lo[h->global_col[g]] = -std::numeric_limits<double>::infinity();
      hi[h->global_col[g]] = std::numeric_limits<double>::infinity();
    }
  return FS_OK;
}

int fs_gpu_set_params(fs_gpu *h, const double *x, int32_t D) {
  if (!h || !x) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "no model");
  if (D != h->D) return set_error(h, FS_ERR_ARG, "set_params: D mismatch");
  for (int k = 0; k < D; ++k)
    if (!std::isfinite(x[k]))
      return set_error(h, FS_ERR_NUMERIC, "set_params: parameter " + std::to_string(k) +
                                              " is not finite (the model is unchanged)");
  cudaSetDevice(h->device);
  for (HostTable &t : h->tables)
    for (int k = 0; k < t.n; ++k)
      if (t.cols[k] >= 0) t.v[k] = x[t.cols[k]];
  for (size_t g = 0; g < h->global_col.size(); ++g)
    if (h->global_col[g] >= 0) h->global_val[g] = x[h->global_col[g]];
  FS_TRY(upload_values(h));
  h->params_dirty = true;
  h->jac_valid = false;
  // A larger cutoff (SW a1/a2) needs longer lists; a smaller one does not:
  // pairs beyond the cutoff contribute exactly zero.
  if (h->rcut_built >= 0 && model_max_cutoff(h) > h->rcut_built)
    FS_TRY(build_neighbors(h, model_max_cutoff(h)));
  return FS_OK;
}

int fs_gpu_max_cutoff(fs_gpu *h, double *rc) {
  if (!h || !rc) return FS_ERR_ARG;
  if (!h->have_model) return set_error(h, FS_ERR_STATE, "max_cutoff: no model");
  *rc = model_max_cutoff(h);
  return FS_OK;
}

int fs_gpu_residual_count(fs_gpu *h, double w_s, int64_t *m) {
  if (!h || !m) return FS_ERR_ARG;
  if (h->n_cfg == 0) return set_error(h, FS_ERR_STATE, "no configurations");
  *m = rows_of(h, w_s);
  return FS_OK;
}

int fs_gpu_eval(fs_gpu *h, double w_e, double w_s, double *F, double *forces, double *energy,
                double *stress9, double *limit, double *obj) {
  FS_TRY(check_ready(h));
  cudaSetDevice(h->device);
  FS_TRY(ensure_eval_buffers(h, w_s));
  FS_TRY(ensure_params(h));
  FS_TRY(eval_residual(h, w_e, w_s));
  const int64_t m = rows_of(h, w_s);
  if (F) FS_CUDA(cudaMemcpyAsync(F, h->d_F, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (forces)
    FS_CUDA(cudaMemcpyAsync(forces, h->d_forces, 3 * h->n_atoms * sizeof(double),
                            cudaMemcpyDeviceToHost, h->stream));
  if (energy)
    FS_CUDA(cudaMemcpyAsync(energy, h->d_energy, h->n_cfg * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream));
  if (stress9)
    FS_CUDA(cudaMemcpyAsync(stress9, h->d_stress9, 9 * h->n_cfg * sizeof(double),
                            cudaMemcpyDeviceToHost, h->stream));
  if (limit)
    FS_CUDA(cudaMemcpyAsync(limit, h->d_limit, h->n_cfg * sizeof(double), cudaMemcpyDeviceToHost,
                            h->stream));
  if (obj) FS_CUDA(cudaMemcpyAsync(obj, h->d_obj, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return sync(h);
}

int fs_gpu_eval_jacobian_async(fs_gpu *h, double w_e, double w_s) {
  FS_TRY(check_ready(h));
  cudaSetDevice(h->device);
  FS_TRY(ensure_eval_buffers(h, w_s));
  FS_TRY(ensure_params(h));
  mark(h, 0);
  // spline EAM / pair: the residual and the per-atom Jacobian pass read the
  // same inputs and write disjoint buffers, so the residual runs on a side
  // stream beside it; the force-row pass waits for it (it reads F)
  bool side = h->family == FS_FAMILY_EAM || h->family == FS_FAMILY_PAIR;
  for (const HostTable &t : h->tables) side = side && t.kind == FS_TABLE_SPLINE;
  if (side) {
    FS_CUDA(cudaEventRecord(h->ev_fork, h->stream));
    FS_CUDA(cudaStreamWaitEvent(h->side, h->ev_fork, 0));
    std::swap(h->stream, h->side); // the residual's launches go to the side stream
    const int rc = eval_residual(h, w_e, w_s);
    std::swap(h->stream, h->side);
    FS_TRY(rc);
    FS_CUDA(cudaEventRecord(h->ev_join, h->side));
    h->join_pending = true;
  } else {
    FS_TRY(eval_residual(h, w_e, w_s));
  }
  mark(h, 1);
  const int rcj = eval_jacobian(h, w_e, w_s);
  if (h->join_pending) { // not consumed (an error path): keep the stream order
    cudaStreamWaitEvent(h->stream, h->ev_join, 0);
    h->join_pending = false;
  }
  FS_TRY(rcj);
  FS_TRY(gram(h, rows_of(h, w_s), h->d_JtJ, h->d_Jtr));
  mark(h, 4);
  if (h->prof_slots > 0 && h->prof_used < h->prof_slots) ++h->prof_used;
  h->last_we = w_e;
  h->last_ws = w_s;
  h->jac_valid = true;
  return FS_OK;
}

int fs_gpu_fetch_normal_equations(fs_gpu *h, double *JtJ, double *Jtr, double *obj) {
  if (!h) return FS_ERR_ARG;
  if (!h->jac_valid) return set_error(h, FS_ERR_STATE, "no Jacobian evaluated");
  cudaSetDevice(h->device);
  const size_t D = h->D, n = D * D + D + 1;
  // one DMA per part into a pinned buffer, one wait, then host copies
  FS_TRY(ensure_pinned(h, &h->h_ne_pin, &h->h_ne_pin_n, n));
  double *pin = h->h_ne_pin;
  if (JtJ) FS_CUDA(cudaMemcpyAsync(pin, h->d_JtJ, D * D * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (Jtr) FS_CUDA(cudaMemcpyAsync(pin + D * D, h->d_Jtr, D * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (obj) FS_CUDA(cudaMemcpyAsync(pin + D * D + D, h->d_obj, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  FS_TRY(sync(h));
  if (JtJ) std::memcpy(JtJ, pin, D * D * sizeof(double));
  if (Jtr) std::memcpy(Jtr, pin + D * D, D * sizeof(double));
  if (obj) *obj = pin[D * D + D];
  return FS_OK;
}

int fs_gpu_eval_jacobian(fs_gpu *h, double w_e, double w_s, double *F, double *J, double *JtJ,
                         double *Jtr, double *obj) {
  FS_TRY(fs_gpu_eval_jacobian_async(h, w_e, w_s));
  const int64_t m = rows_of(h, w_s);
  if (F) FS_CUDA(cudaMemcpyAsync(F, h->d_F, m * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  // column-major m × D (Eigen's fjac), widened and transposed on the device
  if (J) FS_TRY(fs_gpu_copy_jacobian_rows(h, 0, m, J, m));
  return fs_gpu_fetch_normal_equations(h, JtJ, Jtr, obj);
}

int fs_gpu_acsf_standardization(fs_gpu *h, double *mean, double *inv_std, int64_t *count) {
  if (!h || !mean || !inv_std || !count) return FS_ERR_ARG;
  FS_TRY(check_ready(h));
  if (h->family != FS_FAMILY_ACSF && h->family != FS_FAMILY_LMBTR)
    return set_error(h, FS_ERR_STATE, "acsf_standardization: not an ACSF or LMBTR model");
  cudaSetDevice(h->device);
  return acsf_standardization(h, mean, inv_std, count);
}

int fs_gpu_copy_normal_equations(fs_gpu *h, void *dst) {
  if (!h || !dst) return FS_ERR_ARG;
  if (!h->jac_valid) return set_error(h, FS_ERR_STATE, "no Jacobian evaluated");
  cudaSetDevice(h->device);
  const size_t D = h->D;
  double *d = static_cast<double *>(dst);
  FS_CUDA(cudaMemcpyAsync(d, h->d_JtJ, D * D * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(d + D * D, h->d_Jtr, D * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  FS_CUDA(cudaMemcpyAsync(d + D * D + D, h->d_obj, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  return FS_OK;
}

int fs_gpu_set_profiling(fs_gpu *h, int32_t max_steps) {
  if (!h || max_steps < 0) return FS_ERR_ARG;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  for (cudaEvent_t e : h->prof_ev) cudaEventDestroy(e);
  h->prof_ev.clear();
  h->prof_slots = h->prof_used = 0;
  if (max_steps == 0) return FS_OK;
  h->prof_ev.resize(static_cast<size_t>(max_steps) * (kPhases + 1));
  for (cudaEvent_t &e : h->prof_ev) FS_CUDA(cudaEventCreate(&e));
  h->prof_slots = max_steps;
  return FS_OK;
}

int fs_gpu_phase_times(fs_gpu *h, double *ms, int32_t n, int32_t *steps) {
  if (!h || !ms || n < kPhases) return FS_ERR_ARG;
  cudaSetDevice(h->device);
  FS_CUDA(cudaStreamSynchronize(h->stream));
  for (int p = 0; p < n; ++p) ms[p] = 0.0;
  for (int s = 0; s < h->prof_used; ++s)
    for (int p = 0; p < kPhases; ++p) {
      float t = 0.f;
      cudaEvent_t a = h->prof_ev[s * (kPhases + 1) + p], b = h->prof_ev[s * (kPhases + 1) + p + 1];
      FS_CUDA(cudaEventElapsedTime(&t, a, b));
      ms[p] += t;
    }
  if (steps) *steps = h->prof_used;
  h->prof_used = 0;
  return FS_OK;
}

int fs_gpu_launch_count(fs_gpu *h, int64_t *count) {
  if (!h || !count) return FS_ERR_ARG;
  *count = h->launches;
  return FS_OK;
}

int fs_gpu_lm_step(fs_gpu *h, double lambda, int32_t mode, double *dx) {
  if (!h || !dx) return FS_ERR_ARG;
  if (!h->jac_valid) return set_error(h, FS_ERR_STATE, "lm_step: no Jacobian evaluated");
  if (!(lambda >= 0.0) || (mode != 0 && mode != 1)) return set_error(h, FS_ERR_ARG, "lm_step: bad lambda/mode");
  cudaSetDevice(h->device);
  return lm_solve(h, lambda, mode, dx);
}

int fs_gpu_lsq_step(fs_gpu *h, double ridge, double *dx) {
  if (!h || !dx) return FS_ERR_ARG;
  if (!h->jac_valid) return set_error(h, FS_ERR_STATE, "lsq_step: no Jacobian evaluated");
  cudaSetDevice(h->device);
  double lambda = ridge;
  if (lambda <= 0.0) {
    // 1e-8 · max(mean diag(JᵀJ), 1)  (solver.cpp:252-255)
    std::vector<double> diag(h->D);
    FS_CUDA(cudaMemcpy2DAsync(diag.data(), sizeof(double), h->d_JtJ, (h->D + 1) * sizeof(double),
                              sizeof(double), h->D, cudaMemcpyDeviceToHost, h->stream));
    FS_TRY(sync(h));
    double mean = 0.0;
    for (double v : diag) mean += v;
    mean /= h->D;
    lambda = 1e-8 * std::max(mean, 1.0);
  }
  return lm_solve(h, lambda, 0, dx);
}

int fs_gpu_eval_population(fs_gpu *h, double w_e, double w_s, const double *xs, int32_t NP,
                           double *obj) {
  FS_TRY(check_ready(h));
  if (!xs || !obj || NP <= 0) return set_error(h, FS_ERR_ARG, "eval_population: bad arguments");
  cudaSetDevice(h->device);
  FS_TRY(ensure_eval_buffers(h, w_s));
  return eval_population(h, w_e, w_s, xs, NP, obj);
}

} // extern "C"

extern "C" int fs_gpu_abi_sizes(int64_t *sizes, int32_t n) {
  const int64_t s[6] = {static_cast<int64_t>(sizeof(fs_table)),       static_cast<int64_t>(sizeof(fs_model)),
                        static_cast<int64_t>(sizeof(fs_gpu_opts)),    static_cast<int64_t>(sizeof(fs_tune_report)),
                        static_cast<int64_t>(sizeof(fs_de_opts)),     static_cast<int64_t>(sizeof(fs_surrogate_opts))};
  if (!sizes || n < 0) return FS_ERR_ARG;
  for (int k = 0; k < n && k < 6; ++k) sizes[k] = s[k];
  return 6;
}
