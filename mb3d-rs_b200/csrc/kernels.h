// Launchers of the march kernels (kernels.cu) for the host code (capi.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mb3d_cu.h"
#include "devparams.h"
#include "mc.h"

namespace mb3dcu {

// A ray the single precision march hands to the double precision finish.
struct Hand {
    double mzz;        // depth in step widths
    double last_step;
    double last_de;
    double dtmp;       // the DE at the surface (plain march)
    double c[3];       // the position (plain march: accumulated as the reference does)
    uint32_t pix;      // index in the band's G-buffer
    uint32_t flags;    // HAND_*
    float step_count;  // the dynamic fog's count so far
    float rsf;         // the step factor (rsf_mul)
    int32_t seed;
    int32_t it;        // the iteration count at the surface (plain march)
};
#define HAND_FULL 1u     // march the whole pixel in double precision
#define HAND_HALF 2u     // the state is right after the half step back (with its step factor rsf)
#define HAND_REMARCH 8u  // march on in double precision from this state

// Where a post pass starts on a surface pixel.
// a DE AO ray the single precision kernel hands over to double precision:
// its item, its length and openness so far, its step count (bit 31: the
// ray's last step); the list follows the rays' openness array min_ra
// (ao_slow_list), so that array holds AO_MINRA_BYTES per ray
struct AoSlow {
    uint32_t item;
    float dt1, s;
    uint32_t guard;
};
constexpr size_t AO_MINRA_BYTES = sizeof(float) + sizeof(AoSlow);
__host__ __device__ inline AoSlow *ao_slow_list(float *min_ra, uint32_t n_items) {
    return reinterpret_cast<AoSlow *>(min_ra + (((size_t)n_items + 3) & ~(size_t)3));
}
__host__ __device__ inline const AoSlow *ao_slow_list(const float *min_ra, uint32_t n_items) {
    return reinterpret_cast<const AoSlow *>(min_ra + (((size_t)n_items + 3) & ~(size_t)3));
}

struct PostStart {
    double sh_c[3];  // the shadow rays' start (0.1 step in front of the surface)
    double sh_mzz;
    double ao_c[3];  // the DE AO rays' start (on the surface)
    float ao_ms;     // the DE stop there
    uint32_t pix;
    uint32_t flags;  // bit l: the surface faces away from light l
    uint32_t pad;
    // the DE AO rays' per-pixel set-up (k_ao_prep): the turn of the ray
    // table to the surface normal, the first step, the rays' length, the
    // DE stop and the openness offset per unit of length
    float ao_rot[3][3];
    uint32_t pad2;
    double ao_step0, ao_max_dist, ao_msd, ao_md_d10;
};

// The formula sets the kernels are built for (FKIND_* bits, formulas.cuh):
// the smallest one that holds the scene's formulas is used.
#define KSET_IP8 1
#define KSET_IP8BOX 5
#define KSET_MENGERBOX 12
#define KSET_ALL 255
int kernel_set(int fmask);

// the launches of one formula set's kernels (kern_*.cu)
// the DE ambient occlusion of the reflection pass's hits (deao_1pos,
// src/reflect.rs:954-1090) per quality 0..3: its directions, its step
// multiplier and weight, and per pair of directions acos(dot) * abr as
// single precision, or REFL_AO_NO where the pair does not count (the host
// makes it with the C library's functions, as the reference's CPU does)
constexpr int REFL_AO_MAX = 13;  // directions of quality 3
constexpr float REFL_AO_NO = 1e30f;
struct ReflAO {
    int count[4], first[4];
    double d_step_mul[4];
    float corr_w[4];
    float dirs[3 + 3 + 7 + 13][3];
    float ang[4][REFL_AO_MAX][REFL_AO_MAX];
};
void reflect_ao_table(ReflAO &t);

struct LaunchTable {
    void (*march)(const DevParams &, bool mixed, int row0, int rows, mb3d_cu_silight *out, Hand *list,
                  unsigned int *counters, unsigned long long *gcount, int blocks, cudaStream_t s);
    void (*finish)(const DevParams &, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                   mb3d_cu_silight *out, int blocks, cudaStream_t s);
    void (*post_start)(const DevParams &, bool mixed, int row0, int passes, const mb3d_cu_silight *gbuf,
                       const uint32_t *list, const unsigned int *count, unsigned int *queue, PostStart *ps,
                       int blocks, cudaStream_t s);
    void (*shadow_rays)(const DevParams &, bool mixed, int row0, const PostStart *ps, const unsigned int *count,
                        mb3d_cu_silight *gbuf, unsigned int *queue, int blocks, cudaStream_t s);
    void (*ao_rays)(const DevParams &, bool mixed, const PostStart *ps, const mb3d_cu_silight *gbuf,
                    const unsigned int *count, float *min_ra, unsigned int *queue, int blocks, cudaStream_t s);
    void (*de_probe)(const DevParams &, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s);
    // the finish's two kernels one at a time (a budgeted call checks its
    // status between them): the wavefront, then the per-thread rare cases
    void (*finish_fast)(const DevParams &, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s);
    void (*finish_slow)(const DevParams &, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s);
    // the reflection pass's rays (reflect.cuh)
    void (*reflect)(const DevParams &, const mb3d_cu_reflect_ray *rays, uint32_t n, int far_fog, const ReflAO *tab,
                    mb3d_cu_reflect_hit *hits, int blocks, cudaStream_t s);
    void (*reflect_first)(const DevParams &, const mb3d_cu_silight *gbuf, mb3d_cu_reflect_ray *tmp,
                          unsigned char *valid, int blocks, cudaStream_t s);
};
LaunchTable table_ip8();
LaunchTable table_ip8box();
LaunchTable table_mengerbox();
LaunchTable table_all();

void launch_reflect_first(const DevParams &p, const mb3d_cu_silight *gbuf, mb3d_cu_reflect_ray *tmp,
                          unsigned char *valid, int blocks, cudaStream_t s);
// the flagged records of tmp in order into out: the count per block of 1024
// (flag_count), then the scatter from the blocks' offsets (flag_scatter)
void flag_count(const unsigned char *valid, size_t n, unsigned int *block_sum, cudaStream_t s);
void flag_scatter(const unsigned char *valid, const mb3d_cu_reflect_ray *tmp, size_t n, const unsigned int *offset,
                  mb3d_cu_reflect_ray *out, cudaStream_t s);
void launch_reflect(const DevParams &p, const mb3d_cu_reflect_ray *rays, uint32_t n, int far_fog, const ReflAO *tab,
                    mb3d_cu_reflect_hit *hits, int blocks, cudaStream_t s);
void launch_march(const DevParams &p, bool mixed, int row0, int rows, mb3d_cu_silight *out, Hand *list,
                  unsigned int *counters, unsigned long long *gcount, int blocks, cudaStream_t s);
void launch_finish(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                   mb3d_cu_silight *out, int blocks, cudaStream_t s);
void launch_finish_fast(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s);
void launch_finish_slow(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s);
void launch_surface(const DevParams &p, int npix, int passes, mb3d_cu_silight *gbuf, uint32_t *list,
                    unsigned int *count, int blocks, cudaStream_t s);
void launch_post_start(const DevParams &p, bool mixed, int row0, int passes, const mb3d_cu_silight *gbuf,
                       const uint32_t *list, const unsigned int *count, unsigned int *queue, PostStart *ps, int blocks,
                       cudaStream_t s);
void launch_shadow_rays(const DevParams &p, bool mixed, int row0, const PostStart *ps, const unsigned int *count,
                        mb3d_cu_silight *gbuf, unsigned int *queue, int blocks, cudaStream_t s);
void launch_ao_rays(const DevParams &p, bool mixed, const PostStart *ps, const mb3d_cu_silight *gbuf,
                    const unsigned int *count, float *min_ra, unsigned int *queue, int blocks, cudaStream_t s);
void launch_ao_prep(const DevParams &p, PostStart *ps, const mb3d_cu_silight *gbuf, const unsigned int *count,
                    int blocks, cudaStream_t s);
void launch_ao_final(const DevParams &p, const PostStart *ps, const unsigned int *count, const float *min_ra,
                     mb3d_cu_silight *gbuf, int blocks, cudaStream_t s);
void launch_de_probe(const DevParams &p, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s);
int launch_fma_peak(bool fp64, void *out, int blocks, int iters, cudaStream_t s);

// the Monte Carlo kernels of one formula set (kern_mc_*.cu)
struct McTable {
    void (*run)(const DevParams &, const McDev &, bool mixed, bool batch, const McAcc &, const mb3d_cu_mc_req *reqs,
                mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items, const uint32_t *list, int sms,
                cudaStream_t s);
};
McTable mc_table_ip8();
McTable mc_table_ip8box();
McTable mc_table_mengerbox();
McTable mc_table_all();
void launch_mc(const DevParams &p, const McDev &m, bool mixed, bool batch, const McAcc &acc, const mb3d_cu_mc_req *reqs,
               mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items, const uint32_t *list, int sms,
               cudaStream_t s);
// the split render's logic kernel (kern_mc_all.cu) and the bytes of a path's state
size_t mc_lane_bytes();
void launch_mc_logic(const DevParams &p, const McDev &m, const McAcc &acc, void *lanes, mb3d_cu_mc_req *reqs,
                     const mb3d_cu_mc_res *res, uint32_t n_slots, unsigned int *next, uint32_t n_items, uint32_t *list,
                     unsigned int *n_list, int sms, cudaStream_t s);
void launch_mc_final(const McAcc &acc, uint32_t npix, int rays, float *radiance, uint8_t *hit, cudaStream_t s);

// the adaptive pass's steps (mc_pass.cu)
void launch_mcp_start(const McPassArgs &a, int sms, cudaStream_t s);
void launch_mcp_count(const McPassArgs &a, unsigned int *block_sum, cudaStream_t s);
void launch_mcp_items(const McPassArgs &a, int b0, int b1, const unsigned int *offset, unsigned int *fill, uint2 *items,
                      const McAcc &acc, cudaStream_t s);
void launch_mcp_update(const McPassArgs &a, const McAcc &acc, unsigned int *more, int sms, cudaStream_t s);

// depth of field (dof.cu): one pass's constants (focus, src/dof.rs:49-78)
struct DofPass {
    int w, h, forward, rmax;
    float ap, dsf, z_sharp, r_sub, clip_r, max_r, bg, sm;
    double zc_mul_inv, zcorr_inv;
};
// a source pixel of a pass: its colour, disk and weights
struct DofSrc {
    float c[3];
    float s_ms, sw, rr;
    int ims, r;
    uint32_t flags;  // 1: descale (in front of the focus), 2: background
    uint32_t pad;
};
void dof_zrange(const mb3d_cu_silight *g, size_t n, unsigned int *zr, int sms, cudaStream_t s);
void dof_src(const DofPass &d, const mb3d_cu_silight *g, const uint8_t *rgb, DofSrc *src, unsigned long long *key,
             unsigned int *max_r_bits, int sms, cudaStream_t s);
int dof_tiles(const DofPass &d, const DofSrc *src, const unsigned long long *key, uint8_t *out, int cap,
              unsigned int *overflow, cudaStream_t s);

// paint_recs of the Monte Carlo records' colours (mc_paint.cu)
void mc_paint_launch(const float *col, const uint8_t *rays, uint32_t n, const mb3d_cu_mc_paint_opts &mc, uint8_t *out,
                     int blocks, cudaStream_t s);

// the 24-bit screen space ambient occlusion of a w x h G-buffer (ssao.cu);
// scratch holds ssao_scratch_bytes(w, h, random)
size_t ssao_scratch_bytes(int w, int h, int random);
// the 15-bit screen space ambient occlusion of a w x h G-buffer in device
// memory (ssao15.cu), scratch of ssao15_scratch_bytes(w, h); synchronises the
// stream; 0, -1 (a CUDA call failed) or -2 (a ring beyond its table)
size_t ssao15_scratch_bytes(int w, int h);
int ssao15_run(mb3d_cu_silight *g, int w, int h, double zc_mul, double zcorr, const mb3d_cu_ssao_opts &o,
               unsigned char *scratch, int sms, cudaStream_t s, uint32_t *launches);
void ssao24_launch(mb3d_cu_silight *gbuf, int w, int h, double zc_mul, double zcorr, const mb3d_cu_ssao_opts &o,
                   void *scratch, int sms, cudaStream_t s);

// render::paint of G-buffer records, default lighting (paint.cu)
void paint_launch(const mb3d_cu_scene &sc, const DevParams &p, uint32_t row0, const mb3d_cu_silight *gbuf, uint32_t n,
                  uint8_t *rgb, int blocks, cudaStream_t s);

}  // namespace mb3dcu
