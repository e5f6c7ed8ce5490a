// Families other than EAM / pair (Stillinger–Weber, ADP).
#include "internal.cuh"

namespace fsg {

int eval_residual_other(fs_gpu *h, double, double) {
  return set_error(h, FS_ERR_UNSUPPORTED, "residual: family not handled by this build");
}

int eval_jacobian_other(fs_gpu *h, double, double) {
  return set_error(h, FS_ERR_UNSUPPORTED, "Jacobian: family not handled by this build");
}

} // namespace fsg
