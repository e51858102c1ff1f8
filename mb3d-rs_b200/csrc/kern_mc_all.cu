// The Monte Carlo kernels built for one formula set (KSET_ALL); see mc.cuh.
#define MB3D_MC_COMMON
#include "kern_mc_impl.cuh"

namespace mb3dcu {
McTable mc_table_all() { return McTable{&LaunchMc<KSET_ALL>::run}; }

// the records of a render (every formula set)
size_t mc_lane_bytes() { return sizeof(McLane); }
void launch_mc_logic(const DevParams &p, const McDev &m, const McAcc &acc, void *lanes, mb3d_cu_mc_req *reqs,
                     const mb3d_cu_mc_res *res, uint32_t n_slots, unsigned int *next, uint32_t n_items, uint32_t *list,
                     unsigned int *n_list, int sms, cudaStream_t s) {
    uint32_t blocks = (n_slots + 127) / 128;
    if (blocks > (uint32_t)sms * 16) blocks = (uint32_t)sms * 16;
    k_mc_logic<<<blocks, 128, 0, s>>>(p, m, acc, (McLane *)lanes, reqs, res, n_slots, next, n_items, list, n_list);
}
void launch_mc_final(const McAcc &acc, uint32_t npix, int rays, float *radiance, uint8_t *hit, cudaStream_t s) {
    k_mc_final<<<148 * 4, 256, 0, s>>>(acc, npix, rays, radiance, hit);
}
}  // namespace mb3dcu
