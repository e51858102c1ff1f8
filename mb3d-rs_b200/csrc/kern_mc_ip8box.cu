// The Monte Carlo kernels built for one formula set (KSET_IP8BOX); see mc.cuh.
#include "kern_mc_impl.cuh"

namespace mb3dcu {
McTable mc_table_ip8box() { return McTable{&LaunchMc<KSET_IP8BOX>::run}; }
}  // namespace mb3dcu
