// bv_llh_mixed.cu -- mixed-precision evaluation path.
#include "../../include/bv.h"
#include "bv_common.cuh"
#include "bv_llh_mixed.cuh"

namespace bv {

int mixed_create(MixedWork &w, const MixedSetup &s)
{
    (void)w;
    (void)s;
    set_error("mixed precision path is not built in this version of the library");
    return BV_E_INVALID;
}

int mixed_enqueue(MixedWork &w, cudaStream_t st)
{
    (void)w;
    (void)st;
    set_error("mixed precision path is not built in this version of the library");
    return BV_E_INVALID;
}

void mixed_free(MixedWork &w) { (void)w; }

}  // namespace bv
