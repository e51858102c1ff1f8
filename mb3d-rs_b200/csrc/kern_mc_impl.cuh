// The Monte Carlo kernels (mc.cuh) instantiated for one formula set.
#pragma once
#include "kernels_impl.cuh"
#include "mc.cuh"

namespace mb3dcu {

template <int FM>
struct LaunchMc {
    // blocks: the SM count; the grid is as many blocks as stay resident
    template <typename R, bool B>
    static void go(const DevParams &p, const McDev &m, const McAcc &acc, const mb3d_cu_mc_req *reqs,
                   mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items, const uint32_t *list, int sms,
                   cudaStream_t s) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mc<R, FM, B>, 128, 0) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        k_mc<R, FM, B><<<sms * per_sm, 128, 0, s>>>(p, m, acc, reqs, res, queue, n_items, list);
    }
    static void run(const DevParams &p, const McDev &m, bool mixed, bool batch, const McAcc &acc,
                    const mb3d_cu_mc_req *reqs, mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items,
                    const uint32_t *list, int sms, cudaStream_t s) {
        if (batch) {
            if (mixed) go<float, true>(p, m, acc, reqs, res, queue, n_items, list, sms, s);
            else go<double, true>(p, m, acc, reqs, res, queue, n_items, list, sms, s);
        } else {
            if (mixed) go<float, false>(p, m, acc, reqs, res, queue, n_items, list, sms, s);
            else go<double, false>(p, m, acc, reqs, res, queue, n_items, list, sms, s);
        }
    }
};

}  // namespace mb3dcu
