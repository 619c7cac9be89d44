// Split-BF16 tcgen05 tensor-core form of Signal (placeholder until the
// kernel lands; reports FM_ERR_UNSUPPORTED rather than computing elsewhere).
#include "signal_common.cuh"

namespace fm {

size_t tc_workspace(const fm_signal_args *) { return 0; }

int signal_tc(fm_ctx *, const fm_signal_args *, void *, size_t) {
  set_error(FM_ERR_UNSUPPORTED, "fm_signal(BF16X3): tensor-core form not built yet");
  return FM_ERR_UNSUPPORTED;
}

}  // namespace fm
