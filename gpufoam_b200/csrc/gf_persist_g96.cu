// Persistent work-queue kernel variants with 96 thread(s) per cell.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_fn_g96(bool shared, int slim) { return persistent_variant<96>(shared, slim); }
#ifdef GF_PHASE_TIMERS
int phase_cycles_g96(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
