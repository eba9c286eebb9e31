// Per-tile precision selection for the mixed-precision layouts.
#include <vector>

#include "tiles.h"

namespace mf {

// Builds the mixed-precision slab layouts of t. MF_MODE_FIXED stores every
// tile at opt.fixed_precision (one level).
int build_mixed_levels(mf_tiles *t, cudaStream_t s) {
    const int mode = t->opt.precision_mode;
    if (mode == MF_MODE_FIXED) {
        if (t->opt.fixed_precision < MF_PREC_FP64 || t->opt.fixed_precision > MF_PREC_FP8) return MF_ERR_ARG;
        std::vector<uint8_t> p(t->tilenum, (uint8_t)t->opt.fixed_precision);
        int rc = build_layout(t, t->Lmix[0], p, s);
        if (rc) return rc;
        t->mixed_ready = true;
        return MF_OK;
    }
    set_last_error("precision mode not available");
    return MF_ERR_UNSUPPORTED;
}

}  // namespace mf
