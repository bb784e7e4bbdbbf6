// Persistent work-queue kernel variants with 4 thread(s) per cell.
#include "gf_persist.cuh"

namespace gf {
const void* persistent_fn_g4(bool shared, int slim) { return persistent_variant<4>(shared, slim); }
#ifdef GF_PHASE_TIMERS
int phase_cycles_g4(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif
}  // namespace gf
