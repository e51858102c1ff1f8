// The Monte Carlo kernels built for one formula set (KSET_ALL); see mc.cuh.
#define MB3D_MC_COMMON
#include "kern_mc_impl.cuh"

namespace mb3dcu {
McTable mc_table_all() { return McTable{&LaunchMc<KSET_ALL>::run}; }

// the records of a render (every formula set)
void launch_mc_final(const McAcc &acc, uint32_t npix, int rays, float *radiance, uint8_t *hit, cudaStream_t s) {
    k_mc_final<<<148 * 4, 256, 0, s>>>(acc, npix, rays, radiance, hit);
}
}  // namespace mb3dcu
