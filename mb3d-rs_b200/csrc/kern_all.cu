// The kernels built for one formula set (KSET_ALL); see kernels_impl.cuh.
#define MB3D_COMMON_KERNELS
#include "kernels_impl.cuh"

namespace mb3dcu {
LaunchTable table_all() {
    typedef Launch<KSET_ALL> L;
    return LaunchTable{&L::march, &L::finish, &L::post_start, &L::shadow_rays, &L::ao_rays, &L::de_probe,
                       &L::finish_fast, &L::finish_slow, &L::reflect, &L::reflect_first};
}

// the kernels every formula set shares
void launch_surface(const DevParams &p, int npix, int passes, mb3d_cu_silight *gbuf, uint32_t *list,
                    unsigned int *count, int blocks, cudaStream_t s) {
    k_surface<<<blocks, 256, 0, s>>>(p, npix, passes, gbuf, list, count);
}
void launch_ao_prep(const DevParams &p, PostStart *ps, const mb3d_cu_silight *gbuf, const unsigned int *count,
                    int blocks, cudaStream_t s) {
    k_ao_prep<<<blocks, 128, 0, s>>>(p, ps, gbuf, count);
}
void launch_ao_final(const DevParams &p, const PostStart *ps, const unsigned int *count, const float *min_ra,
                     mb3d_cu_silight *gbuf, int blocks, cudaStream_t s) {
    k_ao_final<<<blocks, 128, 0, s>>>(p, ps, count, min_ra, gbuf);
}
}  // namespace mb3dcu
