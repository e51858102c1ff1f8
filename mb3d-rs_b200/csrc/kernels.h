// Launchers of the march kernels (kernels.cu) for the host code (capi.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mb3d_cu.h"
#include "devparams.h"

namespace mb3dcu {

// A ray the single precision march hands to the double precision finish.
struct Hand {
    double mzz;        // depth in step widths
    double last_step;
    double last_de;
    uint32_t pix;      // index in the band's G-buffer
    uint32_t flags;    // HAND_*
    float step_count;  // the dynamic fog's count so far
    float rsf;         // the step factor (rsf_mul)
    int32_t seed;
    uint32_t pad;
};
#define HAND_FULL 1u     // march the whole pixel in double precision
#define HAND_STEPPED 2u  // the hand-over came right after a step
#define HAND_FIRST 4u    // the random first step is still to come

int launch_march64(const DevParams &p, int row0, int rows, mb3d_cu_silight *out, cudaStream_t s);
int launch_march32(const DevParams &p, int row0, int rows, mb3d_cu_silight *out, Hand *list, unsigned int *counters,
                   int sms, cudaStream_t s);
int launch_finish64(const DevParams &p, int row0, const Hand *list, const unsigned int *counters, mb3d_cu_silight *out,
                    int sms, cudaStream_t s);
int launch_shadow(const DevParams &p, int row0, int rows, mb3d_cu_silight *gbuf, bool mixed, cudaStream_t s);
int launch_deao(const DevParams &p, int row0, int rows, mb3d_cu_silight *gbuf, bool mixed, cudaStream_t s);
int launch_de_probe(const DevParams &p, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s);

}  // namespace mb3dcu
