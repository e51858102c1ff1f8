// The Monte Carlo kernels built for one formula set (KSET_IP8); see mc.cuh.
#include "kern_mc_impl.cuh"

namespace mb3dcu {
McTable mc_table_ip8() { return McTable{&LaunchMc<KSET_IP8>::run}; }
}  // namespace mb3dcu
