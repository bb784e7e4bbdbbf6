// Persistent work-queue kernel variants with 32 threads per cell chosen by
// the autotuner: LU panel widths 4 and 16, and compile-time matrix sizes.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_tuned_fn_g32(bool shared, int slim, int nb, int ms) {
    return persistent_tuned_variant<32>(shared, slim, nb, ms);
}
#ifdef GF_PHASE_TIMERS
int phase_cycles_g32t(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
