// hbg_mixed.cu -- the mixed-precision form (placeholder until its kernels land).
#include "hbg_mixed.h"

namespace hbg {

int mixed_solve_frequencies(const PanelsView&, const double*, const HbgProblem&, const HbgOptions&, bool, double,
                            cudaStream_t, double*, int64_t*, const char** msg, int64_t* freq) {
    *msg = "the mixed-precision form is not built yet";
    *freq = -1;
    return HB_ERR_UNSUPPORTED;
}

}  // namespace hbg
