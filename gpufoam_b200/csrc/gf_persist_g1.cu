// Persistent work-queue kernel variants with 1 thread(s) per cell.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_fn_g1(bool shared, int slim) { return persistent_variant<1>(shared, slim); }
#ifdef GF_PHASE_TIMERS
int phase_cycles_g1(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
