// The kernels built for one formula set (KSET_IP8); see kernels_impl.cuh.
#include "kernels_impl.cuh"

namespace mb3dcu {
LaunchTable table_ip8() {
    typedef Launch<KSET_IP8> L;
    return LaunchTable{&L::march, &L::finish, &L::post_start, &L::shadow_rays, &L::ao_rays, &L::de_probe,
                       &L::finish_fast, &L::finish_slow, &L::reflect, &L::reflect_first};
}
}  // namespace mb3dcu
