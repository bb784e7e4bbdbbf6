// Persistent work-queue kernel variants with 64 threads per cell chosen by
// the autotuner: LU panel widths 4 and 16, and compile-time matrix sizes.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_tuned_fn_g64(bool shared, int slim, int nb, int ms) {
    return persistent_tuned_variant<64>(shared, slim, nb, ms);
}
#ifdef GF_PHASE_TIMERS
int phase_cycles_g64t(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
