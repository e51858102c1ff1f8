// The Monte Carlo kernels built for one formula set (KSET_MENGERBOX); see mc.cuh.
#include "kern_mc_impl.cuh"

namespace mb3dcu {
McTable mc_table_mengerbox() { return McTable{&LaunchMc<KSET_MENGERBOX>::run}; }
}  // namespace mb3dcu
