// The Monte Carlo kernels (mc.cuh) instantiated for one formula set.
#pragma once
#include "kernels_impl.cuh"
#include "mc.cuh"

namespace mb3dcu {

template <int FM>
struct LaunchMc {
    static void run(const DevParams &p, const McDev &m, bool mixed, bool batch, const McAcc &acc,
                    const mb3d_cu_mc_req *reqs, mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items, int blocks,
                    cudaStream_t s) {
        if (batch) {
            if (mixed) k_mc<float, FM, true><<<blocks, 128, 0, s>>>(p, m, acc, reqs, res, queue, n_items);
            else k_mc<double, FM, true><<<blocks, 128, 0, s>>>(p, m, acc, reqs, res, queue, n_items);
        } else {
            if (mixed) k_mc<float, FM, false><<<blocks, 128, 0, s>>>(p, m, acc, reqs, res, queue, n_items);
            else k_mc<double, FM, false><<<blocks, 128, 0, s>>>(p, m, acc, reqs, res, queue, n_items);
        }
    }
};

}  // namespace mb3dcu
