// Persistent work-queue kernel variants with 96 threads per cell (three warps) chosen by
// the autotuner: LU panel widths 4 and 16, and compile-time matrix sizes.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_tuned_fn_g96(bool shared, int slim, int nb, int ms) {
    return persistent_tuned_variant<96>(shared, slim, nb, ms);
}
#ifdef GF_PHASE_TIMERS
int phase_cycles_g96t(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
