/* mb3d_cu: the distance-estimated ray march ("Calculate 3D") and the Monte
 * Carlo path tracer of Mandelbulb3D on one NVIDIA B200 (sm_100a).
 *
 * This is the C ABI a host renderer calls in place of its graphics-card
 * backend.  Every entry point replaces one function of mb3d-rs's card
 * backend `src/gpu.rs`; the comment above each names it.  The host keeps its
 * scene model and its CPU renderer; this library has no CPU fallback inside:
 * it returns a negative status and the caller decides.
 *
 * Conventions (those of mb3d-rs's C API, capi/include/mb3d.h:12-15):
 *  - 0 is success, a negative errno-style status is a failure, and
 *    mb3d_cu_last_error() tells why, on the same thread;
 *  - a context is used by one thread at a time; contexts on different
 *    threads may run concurrently (each has its own CUDA stream);
 *  - buffers may be host or device memory (the library finds out which);
 *    host buffers are copied in and out inside the call; device buffers are
 *    read and written on the context's stream (mb3d_cu_set_stream), so a
 *    caller that fills them on another stream orders the two streams first.
 *
 * Precision modes: MB3D_CU_FP64 is the plain double precision march, the
 * drop-in for the reference's FP64 CPU march.  MB3D_CU_FP32_FP64 marches in
 * single precision with the camera origin and the ray parameter in double
 * precision and finishes every surface (hit re-check, binary search, depth)
 * in double precision; deep zooms where single precision cannot resolve the
 * DE offset switch to double precision per pixel.
 */
#ifndef MB3D_CU_H
#define MB3D_CU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (negative errno values) ---- */
#define MB3D_CU_OK 0
#define MB3D_CU_EINVAL (-22)     /* bad scene, size or pointer */
#define MB3D_CU_ENOMEM (-12)     /* device memory exhausted */
#define MB3D_CU_ENODEV (-19)     /* no CUDA device / not an sm_100 device */
#define MB3D_CU_EIO (-5)         /* a CUDA call failed (text in last_error) */
#define MB3D_CU_ECANCELED (-125) /* *cancel became non-zero */
#define MB3D_CU_ETIMEDOUT (-110) /* the device time budget ran out (resumable) */
#define MB3D_CU_EOVERFLOW (-75)  /* more than 1/500 of the pixels had a NaN DE */
#define MB3D_CU_ENOTSUP (-95)    /* a scene feature this backend does not do */

/* ---- formula numbers: MB3D's internal formula numbers as a .m3p slot
 * stores them (src/m3p.rs:797-823), plus the Menger IFS, which mb3d-rs runs
 * as a custom .m3f formula and this library has built in. ---- */
#define MB3D_CU_F_INTPOW 0        /* Integer Power: options power(2..8), z_mul */
#define MB3D_CU_F_REALPOWER 1     /* Real Power: power, z_mul */
#define MB3D_CU_F_QUATERNION 2    /* Quaternion (4D): yw_mul, w_add */
#define MB3D_CU_F_TRICORN 3       /* Tricorn: z_mul, cz_mul */
#define MB3D_CU_F_AMAZINGBOX 4    /* Amazing Box: scale, min_r, fold */
#define MB3D_CU_F_BULBOX 5        /* Bulbox: scale, min_r, fold, bulb_scale, r_thr, r_thr2 */
#define MB3D_CU_F_FOLDINGINTPOW 6 /* Folding Int Pow: power, z_mul, fold */
#define MB3D_CU_F_AEXIONC 9       /* Aexion C: power, z_mul, rot_c, cond_phi, power_c, cz_mul, powc_dist, mode */
#define MB3D_CU_F_MENGERIFS 100   /* Menger IFS: scale, cscale_x, cscale_y, cscale_z */

#define MB3D_CU_SLOTS 6

/* One hybrid slot (a .m3p THeaderCustomAddon slot, src/m3p.rs:771-777). */
typedef struct mb3d_cu_slot {
    int32_t iterations; /* consecutive iterations; negative: not counted; 0: empty */
    int32_t formula;    /* MB3D_CU_F_* */
    double options[16]; /* the formula's option values in .m3p order */
} mb3d_cu_slot;

/* One global light (TLight8, src/lighting.rs:95-122): its angles. */
typedef struct mb3d_cu_light {
    int32_t on;
    int32_t pad;
    double x_angle; /* radians (LXpos) */
    double y_angle; /* radians (LYpos) */
} mb3d_cu_light;

/* The scene fields the march, the post passes and the Monte Carlo tracer
 * read (Scene, src/scene.rs:398-530; defaults src/scene.rs:628-697). */
typedef struct mb3d_cu_scene {
    int32_t width, height;
    int32_t iterations;     /* maximum iterations */
    int32_t min_iterations; /* MB3D's minimum iterations (default 1) */
    double rstop;           /* bailout radius; <= 0: the formulas' default */
    double zoom;
    double mid[3];
    double z_start, z_end;
    double vgrads[3][3];    /* camera rows: screen x, screen y, view axis */
    double fov_y;           /* degrees */
    double de_stop;         /* in pixels */
    double z_step_div;      /* raystep */
    double raystep_limiter;
    int32_t smooth_normals; /* 0..8 */
    int32_t bin_search_steps;
    int32_t first_step_random;
    int32_t step_sub_de_stop;
    int32_t vary_de_stop_on_fov;
    int32_t normals_on_de;
    int32_t disable_analytic_de;
    int32_t julia;
    double julia_c[4];
    int32_t color_option;
    int32_t color_on_it;
    double color_mul;
    int32_t dfog_on_it;
    int32_t repeat_from;
    int32_t n_slots;        /* 1..6 */
    int32_t pad0;
    mb3d_cu_slot slots[MB3D_CU_SLOTS];
    /* lighting (for the shadow pass and the Monte Carlo tracer) */
    mb3d_cu_light lights[6];
    /* the hard shadow pass: bit i = light i casts shadows (0 = no pass) */
    int32_t shadow_lights;
    int32_t shadow_soft;    /* 1: one soft shadow (the last selected light) */
    float soft_radius;
    float hs_max_len_mul;   /* default 1 */
    /* the DE ambient occlusion pass: quality 0..3 = 3/7/17/33 rays, -1 off */
    int32_t deao_quality;
    int32_t deao_dither;    /* 0 (only 0 on the card path) */
    float deao_max_len;     /* default 1 */
    int32_t deao_first_step_random;
    /* the interpolation hybrid (Scene::interpolation, src/scene.rs:510;
     * doInterpolHybridPas, src/iteration.rs:347-475): with interpolation
     * non-zero the first two slots' formulas are applied to the same vector
     * in every iteration and their results blended with ipol_weights
     * (normalised to a sum of 1; the slots' iteration counts are not used) */
    int32_t interpolation;
    float ipol_weights[2];
    int32_t pad1;
    /* the 4D rotation of a 4D hybrid (Scene::rot_4d, src/scene.rs:459): the
     * XW, YW and ZW plane angles in radians (BuildSMatrix4) */
    double rot_4d[3];
    /* a DE combination of two hybrid parts (Scene::decomb, src/scene.rs:2178-2200;
     * CalcDEfull with FormulaType > 0, src/calc.rs:1365-1455): decomb 0 is
     * none, 1 min, 2 max, 3 max with the second part inverted, 4 smooth min
     * (linear), 5 smooth min, 6 mix (its second part must be dIFS, which is
     * not on the card: EINVAL as in the reference).  Slots are 0-based: part 1
     * is slots 0..decomb_end1, part 2 decomb_start2..decomb_end2 repeating
     * from decomb_repeat2, with decomb_iterations2 maximum iterations (0: the
     * scene's). decomb_smooth is the smooth combinations' distance (sDEcombS). Part 2
     * sits at part2_offset, turned by part2_rotation (degrees about x, y, z)
     * and scaled by part2_scale (Scene::part2_place; 0 reads as 1). Ignored in
     * an interpolation hybrid, as in the reference. */
    int32_t decomb;
    int32_t decomb_end1, decomb_start2, decomb_end2, decomb_repeat2, decomb_iterations2;
    float decomb_smooth, decomb_mix_pow;
    int32_t decomb_mix_color, pad2;
    double part2_offset[3], part2_rotation[3], part2_scale;
} mb3d_cu_scene;

/* The G-buffer record SiLight (src/gbuffer.rs:5-20), 20 bytes; mb3d-rs's
 * card backend packs the same fields into 5 u32 (src/gpu_march.wgsl:4765). */
typedef struct mb3d_cu_silight {
    int16_t normal[3];  /* view space, +-32767 */
    uint16_t pad;
    uint32_t zpos_fine; /* bits 8..31 depth, 0..7 roughness; zpos >= 32768: background */
    uint16_t shadow;    /* bits 0..9 step count, 10..15 shadow bits */
    uint16_t amb_shadow;
    uint16_t si_gradient;
    uint16_t otrap;
} mb3d_cu_silight;

/* ---- the Monte Carlo renderer (src/mc.rs) ---- */

/* A march request of the Monte Carlo tracer (McReq, src/mc.rs:402-437):
 * kind 0 a ray of CalcRay from pos along dir (one step width long) up to
 * len steps, zz the depth along the view, zz2 the ray's length so far,
 * zzplus the depth per step, probe: a primary ray that first checks
 * whether it starts inside the set; kind 1 a shadow ray of CalcHSMC
 * (len its length, zz the depth of its start, zz2/zzplus the depth along
 * it).  Kind 2 (through transparent objects) is not on the card. */
typedef struct mb3d_cu_mc_req {
    double pos[3], dir[3];
    double zz, zz2, zzplus, len;
    int32_t seed;
    uint8_t kind, probe, inside, pad;
} mb3d_cu_mc_req;

/* The result of a march (McRes, src/mc.rs:439-467): kind 0 open air (or a
 * shadow ray, with len the length left), 1 a surface, 2 a primary ray that
 * starts inside the set. */
typedef struct mb3d_cu_mc_res {
    double pos[3], normals[3];
    double zz, zz2, len;
    float dyn_fog, ms_de_stop;
    int32_t seed;
    uint16_t si_grad, otrap;
    uint8_t kind, de_limited, inside, pad;
    uint32_t pad2;
} mb3d_cu_mc_res;

/* The light values the Monte Carlo shading reads: the part of mb3d-rs's
 * LightVals (src/lighting.rs:605-690, LightVals::build src/lighting.rs:
 * 978-1190) for global (directional) lights that are not visible in the
 * picture, the surface palette, the ambient and depth colours and the fogs,
 * as the host renderer holds them (light and ambient colours 0..255,
 * palette colours 0..1, or squared with internal gamma 2). */
typedef struct mb3d_cu_mc_light {
    int32_t n_lights;     /* 0..6 (LightVals.lights, lights that are on) */
    int32_t sqr;          /* internal gamma 2 */
    float ln[6][3];       /* LightVal.ln: the light's direction, view space */
    float col[6][3];      /* LightVal.col */
    float lmax_l[6];      /* LightVal.lmax_l */
    int32_t pow_func[6];  /* LightVal.pow_func: the specular power, a power of two */
    float amb_col[3], amb_col2[3], depth_col[3], depth_col2[3], dyn_fog_col[3], dyn_fog_col2[3];
    float s_depth, s_shad, s_shad_gr, s_shad_zmul, s_dyn_fog_mul;
    float s_diff, s_spec, s_col_zmul, s_c_start, s_c_mul;
    int32_t col_cycling, col_on_otrap, far_fog, depth_func, no_col_ipol, dfog_options;
    int32_t col_pos[10];
    float col_dif[10][3], col_spe[10][3], col_spe_a[10], s_c_div[10];
} mb3d_cu_mc_light;

/* What one mb3d_cu_mc_render call traces: rays ray0 .. ray0+rays-1 of every
 * pixel of the rectangle (x0, y0, w, h) (w = 0: the whole picture).  A
 * ray's number fixes its random numbers (seed_of, src/mc.rs:1107-1116) and
 * its place in the Halton sequence; rays 0..3 go through the first pass's
 * fixed quarter-pixel positions (src/mc.rs:2493-2494), later rays through
 * a random point of the pixel.  depth is MCDepth (McSettings.depth, the
 * ambient bounces), secant McSettings.options bit 1 (the 4-step secant
 * search instead of the 10-step binary search). */
typedef struct mb3d_cu_mc_opts {
    int32_t rays, ray0;
    int32_t depth, secant;
    float soft_shadow_radius; /* McSettings.soft_shadow_radius */
    int32_t x0, y0, w, h;
    int32_t pad;
} mb3d_cu_mc_opts;

/* Per pixel outputs of mb3d_cu_mc_render (device or host buffers, w*h
 * pixels row-major; any but radiance may be NULL). */
typedef struct mb3d_cu_mc_out {
    float *radiance;  /* w*h*3: the mean light of the rays (McRecord.col, linear) */
    float *albedo;    /* w*h*3: the first surface's diffuse colour (ray ray0) */
    float *normal;    /* w*h*3: its unit normal, world space */
    float *depth;     /* w*h: its distance along the view in world units (0: none) */
    uint8_t *hit;     /* w*h: a ray of the pixel met the object (McRecord.hit) */
} mb3d_cu_mc_out;

/* One pixel of a Monte Carlo picture (McRecord, src/mc.rs:194-217; 24
 * bytes): the average colour of its rays (square roots with internal gamma
 * 2), their average luminance and squared luminance, how many rays it has
 * had, and whether one of them met the object. */
typedef struct mb3d_cu_mc_record {
    float col[3];
    float ysum, ysqr;
    uint16_t ray_count;
    uint8_t hit, pad;
} mb3d_cu_mc_record;

/* Per-render counters the last call measured on the device. */
typedef struct mb3d_cu_stats {
    float ms_march;       /* primary march (+ finish) kernels, CUDA events */
    float ms_finish;      /* the FP64 finish kernel alone */
    float ms_shadow;      /* the post passes' surface list, start points and shadow rays */
    float ms_deao;        /* the DE AO kernels (with both passes they run beside the shadow rays) */
    float ms_total;       /* first launch to last, device time */
    uint32_t launches;    /* this library's kernel launches in the call */
    uint32_t fp64_pixels; /* mixed mode: the pixels marched in double precision from the start plane or finished
                           * by the per-thread double precision marcher (all of them where the zoom needs double
                           * precision throughout); 0 in the FP64 mode */
    uint64_t de_evals;    /* DE evaluations of the march kernel (counting mode only, else 0) */
    uint64_t orbit_its[6];/* formula iterations per slot, all orbits (counting mode only) */
    uint32_t mc_inside_rays; /* Monte Carlo rays that started inside the set (left dark) */
    uint32_t mc_fp64_rays;   /* Monte Carlo rays whose single precision DE fell back to double */
    /* the march kernel's use of its warps' lanes (counting mode only): */
    uint64_t march_lane_its;   /* the DEs' iterations summed over the lanes */
    uint64_t march_warp_its;   /* per warp and loop trip the most iterations of its lanes, summed */
    uint64_t march_trips;      /* warp loop trips that evaluated DEs */
    uint64_t march_busy_lanes; /* the lanes with a ray in those trips, summed */
    uint32_t fp32_overflow_pixels; /* mixed mode: pixels whose single precision DE overflowed (marched on in
                                    * double precision) */
    uint32_t pad_stats;
} mb3d_cu_stats;

typedef struct mb3d_cu_ctx mb3d_cu_ctx;

#define MB3D_CU_FP64 0
#define MB3D_CU_FP32_FP64 1

#define MB3D_CU_POST_SHADOW 1
#define MB3D_CU_POST_DEAO 2

/* Library version text; not to be freed. */
const char *mb3d_cu_version(void);

/* Why the last failed call on this thread failed (capi/src/lib.rs:18-40). */
const char *mb3d_cu_last_error(void);

/* A context on CUDA device `device`, with its own stream.  Replaces the
 * card set-up of gpu.rs (device open, src/gpu.rs:1840-1900). */
int mb3d_cu_init(int device, mb3d_cu_ctx **out);
void mb3d_cu_free(mb3d_cu_ctx *ctx);

/* Launch the context's work on this CUDA stream (a cudaStream_t) instead
 * of its own; NULL goes back to its own. */
int mb3d_cu_set_stream(mb3d_cu_ctx *ctx, void *stream);

/* Replaces gpu::unsupported (src/gpu.rs:445): 0 when this backend can
 * render the scene, 1 when it cannot (the reason, user-visible, in
 * `reason`), negative on a bad scene. */
int mb3d_cu_unsupported(const mb3d_cu_scene *scene, char *reason, size_t cap);

/* Replaces gpu::march (src/gpu.rs:2296) and gpu::march_bands
 * (src/gpu.rs:1586): the rows row0 .. row0+rows of the picture marched into
 * `gbuf` (rows * width records, row-major).  `cancel` (may be NULL) is
 * polled between launches. */
int mb3d_cu_march(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, uint32_t row0, uint32_t rows,
                  mb3d_cu_silight *gbuf, const volatile int *cancel);

/* Called after each band of mb3d_cu_march_ex (gpu::march's `progress`,
 * src/gpu.rs:2296-2302): rows_done of the call's rows_total rows are in the
 * G-buffer (a host buffer has them copied back).  It runs on the calling
 * thread; a non-zero return cancels the call, which then returns
 * MB3D_CU_ECANCELED (the convention of mb3d_progress, capi/include/mb3d.h). */
typedef int (*mb3d_cu_progress_fn)(uint32_t rows_done, uint32_t rows_total, void *user);

/* What gpu::march (src/gpu.rs:2296) takes beyond mb3d_cu_march's arguments,
 * and the card's two limits.  All zero: mb3d_cu_march's behaviour. */
typedef struct mb3d_cu_march_opts {
    const volatile int *cancel;   /* polled between bands (NULL: never cancelled) */
    mb3d_cu_progress_fn progress; /* called after each band (NULL: none) */
    void *user;                   /* progress's last argument */
    uint32_t band_rows;           /* rows per band (0: the whole range is one band) */
    int32_t overflow_fail;        /* 1: return MB3D_CU_EOVERFLOW when the single precision DE overflowed in more
                                   * than 1/500 of the pixels, as the reference's card gives such a picture up
                                   * (src/gpu.rs:2361-2370); 0: those pixels are marched in double precision */
    double budget_ms;             /* device time budget of the call in ms (0: none): once it is spent the
                                   * kernels take no new rays, finish the ones they hold, and the call returns
                                   * MB3D_CU_ETIMEDOUT */
} mb3d_cu_march_opts;

/* Replaces gpu::march with its progress, cancel and sink (src/gpu.rs:2296,
 * march_card :2308-2400): the rows row0 .. row0+rows marched into `gbuf`
 * band by band (each band whole before the next; a host G-buffer gets each
 * band's rows as soon as it is done, as the reference's sink does).
 * MB3D_CU_ETIMEDOUT leaves the work done so far on the context: calling
 * again with the same arguments (scene bytes, precision, rows, gbuf,
 * band_rows) goes on where the budget stopped it, and the G-buffer it
 * finally returns equals one marched without a budget.  Any other call on
 * the context in between drops that state (the next call starts over).
 * `opts` may be NULL. */
int mb3d_cu_march_ex(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, uint32_t row0, uint32_t rows,
                     mb3d_cu_silight *gbuf, const mb3d_cu_march_opts *opts);

/* Replaces gpu::post_on_card (src/gpu.rs:1649) / post_bands (:1715): the
 * hard (or soft) shadows and/or the DE ambient occlusion computed in place
 * on the marched G-buffer rows.  `passes` is MB3D_CU_POST_* bits. */
int mb3d_cu_post(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, int passes, uint32_t row0,
                 uint32_t rows, mb3d_cu_silight *gbuf, const volatile int *cancel);

/* The march and the post passes of the whole picture in one call (what
 * render::calculate_with does on the card, src/render.rs:328-746). */
int mb3d_cu_render(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, mb3d_cu_silight *gbuf,
                   const volatile int *cancel);

/* Replaces gpu::de_probe (src/gpu.rs:3193) and calc::de_at
 * (src/calc.rs:2695): the distance estimate (world units) and iteration
 * count at n world positions (xyz triples). */
int mb3d_cu_de_probe(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, const double *pos, uint32_t n,
                     double *de, int32_t *its);

/* Launch settings of the wavefront kernels (picked by mb3d_cu_autotune). */
typedef struct mb3d_cu_tune {
    int32_t blocks_per_sm; /* resident blocks of 256 threads per SM the persistent kernels start with */
    int32_t refill_min;    /* idle lanes of a warp that make the march and finish kernels take new rays
                            * (32: only a wholly idle warp; the shadow and DE AO ray kernels keep 8) */
    int32_t streams;       /* frames in flight at once in a frame batch */
    int32_t pad;
} mb3d_cu_tune;

/* All frames of an animation (every frame the same size and formulas, its
 * own camera; `frames` is an array of n_frames scenes) marched with their
 * post passes into `out` (n_frames * width * height records, host or
 * device), the launches of all frames captured in one CUDA graph and the
 * frames spread over tune->streams streams so that one frame's tail
 * overlaps the next frame's work.  Replaces the per-frame loop of
 * frames::render_frames on the card (src/frames.rs:467).  tune may be NULL
 * (the defaults). */
int mb3d_cu_render_frames(mb3d_cu_ctx *ctx, const mb3d_cu_scene *frames, uint32_t n_frames, int precision,
                          const mb3d_cu_tune *tune, mb3d_cu_silight *out);

/* The launch settings that render a sample of the frames (every
 * n_frames / sample-th) fastest, from a small grid of candidates, each timed
 * with CUDA events after a warm-up. */
int mb3d_cu_autotune(mb3d_cu_ctx *ctx, const mb3d_cu_scene *frames, uint32_t n_frames, uint32_t sample,
                     int precision, mb3d_cu_tune *out);

/* The counters of the last call on this context. */
int mb3d_cu_stats_get(const mb3d_cu_ctx *ctx, mb3d_cu_stats *out);

/* Counting mode (on != 0): the march kernel also counts its DE evaluations
 * and formula iterations into the stats (a slower build of the kernel, for
 * the roofline's algorithmic work; the reference's ItStats counterpart,
 * src/calc.rs:140-180). */
int mb3d_cu_set_counting(mb3d_cu_ctx *ctx, int on);

/* Measurement helper: the FP32 (fp64 = 0) or FP64 (fp64 = 1) fused
 * multiply-add issue rate of this device, TFLOP/s (2 per FMA), from a
 * dependent-chain kernel timed with CUDA events. */
int mb3d_cu_fma_peak(mb3d_cu_ctx *ctx, int fp64, double *tflops);

/* The light values of MB3D's start-up light preset (Lighting::default,
 * src/lighting.rs:290-391) with the scene's lights (on flags and angles),
 * as LightVals::build makes them (src/lighting.rs:978-1190): for hosts
 * that do not have their own.  Host code only. */
int mb3d_cu_mc_light_default(const mb3d_cu_scene *scene, mb3d_cu_mc_light *out);

/* Replaces gpu::mc_batch (src/gpu.rs:3022): the n marches of the Monte
 * Carlo tracer in `reqs` (McMarch::run, src/mc.rs:488-501: kind 0 ray,
 * src/mc.rs:665-865; kind 1 shadow ray without transparency,
 * src/mc.rs:869-914) into `res`; `secant` as mb3d_cu_mc_opts.secant.
 * Buffers host or device.  The scene is taken as the Monte Carlo renderer
 * takes it (mc_scene, src/mc.rs:2842-2850; no smoothed normals). */
int mb3d_cu_mc_batch(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, int precision, int secant,
                     const mb3d_cu_mc_req *reqs, uint32_t n, mb3d_cu_mc_res *res);

/* Replaces mc::pass (src/mc.rs:2857, pass_inner :3110-3300 with
 * Tracer::pixel :2766-2834 and calc_n :2657-2762): one pass of the adaptive
 * Monte Carlo renderer over the whole picture.  recs (width * height
 * records, host or device) is the picture so far, all zero before the first
 * pass; every pixel takes its rays in rounds: 4 in a pixel without rays,
 * else as many as calc_n finds from its noise and its neighbours in the
 * records at the start of the pass, and more rounds while a round's mean
 * luminance leaves the record's by more than its noise.  A ray's number
 * (its seed and Halton place) follows the pixel's count, so a pass gives
 * the reference's rays.  `opts` gives depth, secant and the soft shadow
 * radius (its rays, ray0 and rectangle are not used); pass_nr is the
 * picture's count of passes so far (McImage::passes).  stats.orbit_its[0]
 * receives the number of rays traced. */
int mb3d_cu_mc_pass(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_mc_light *light,
                    const mb3d_cu_mc_opts *opts, int precision, uint32_t pass_nr, mb3d_cu_mc_record *recs,
                    const volatile int *cancel);

/* The Monte Carlo tracer's rays traced whole on the card: Tracer::ray
 * (src/mc.rs:2467-2627) with CalcRay (src/mc.rs:1904-2348), the direct
 * light of CalcPhongLight and CalcHSMC (src/mc.rs:1513-1768), the ambient
 * and depth colours (CalcBGLight, CalcVisLights) and the ambient bounces,
 * for scenes without reflections, transparency, cutting planes, depth of
 * field, volumetric light, water and clouds.  Each pixel's record is the
 * mean of its rays' light clamped to 0..400 (Tracer::pixel,
 * src/mc.rs:2766-2834, for a fixed number of rays).  Rays that start inside
 * the set are left dark and counted (stats.mc_inside_rays).
 * Work items are single rays; a pixel's rays are summed in 32.32 fixed
 * point, so the result does not depend on the order the card takes them. */
int mb3d_cu_mc_render(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_mc_light *light,
                      const mb3d_cu_mc_opts *opts, int precision, const mb3d_cu_mc_out *out,
                      const volatile int *cancel);

/* The display settings of the Monte Carlo picture (McSettings::contrast,
 * saturation, options; Lighting::gamma; src/scene.rs:591-598): */
typedef struct {
    uint8_t contrast;   /* MCcontrast, exposure 0..255 (128 = 1) */
    uint8_t saturation; /* 0..127 (32 = 1) */
    uint8_t options;    /* bit 0: soft clipping (HDR) */
    uint8_t pad;
    float gamma;        /* the lighting's gamma slider (32 = none) */
} mb3d_cu_mc_paint_opts;

/* mb3d_cu_mc_paint_opts of McSettings::default and Lighting::default. */
void mb3d_cu_mc_paint_default(mb3d_cu_mc_paint_opts *out);

/* paint_recs (src/mc.rs:3957-4005) on the card: the records' colours (3
 * floats per pixel, e.g. mb3d_cu_mc_render's radiance or the denoised
 * picture) to 8-bit RGB: exposure, squared, to Lab, the gamma curve and
 * the soft clip on L, saturation, back to RGB, square root, rounded.  `rays`
 * (npix bytes, or NULL: every pixel has rays) marks pixels without rays,
 * which stay black.  Host or device buffers. */
int mb3d_cu_mc_paint(mb3d_cu_ctx *ctx, const float *colour, const uint8_t *rays, uint32_t npix,
                     const mb3d_cu_mc_paint_opts *opts, uint8_t *rgb);

/* render::paint (src/render.rs:2499-2501, paint_core :2676-2720) on the
 * card: the 8-bit RGB picture (3 bytes per pixel) of rows row0 ..
 * row0+rows-1 of the scene from their G-buffer records (rows * width, e.g.
 * mb3d_cu_render's), with Lighting::default and the scene's lights
 * (src/lighting.rs:290-391): shade (src/lighting.rs:1802-2162) along its
 * default path -- directional lights not visible in the picture, the
 * palette's colours, ambient top/bottom light, the hard shadows the scene's
 * shadow pass marked, the DE ambient occlusion, the depth and dynamic fog --
 * and pixel_color_s (:1739-1760) clipped and rounded to 8 bits.  Single
 * precision, unfused, as the reference's CPU painter.  Host or device
 * buffers. */
int mb3d_cu_paint(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_silight *gbuf, uint32_t row0,
                  uint32_t rows, uint8_t *rgb);

/* The 24-bit screen space ambient occlusion (SsaoParams, src/ssao.rs:14-33): */
typedef struct {
    float threshold;     /* sAmbShadowThreshold (z/r); 2 by default */
    float border_mirror; /* bSSAO24BorderMirrorSize * 0.01, 0..0.9 */
    uint8_t t0;          /* the "threshold down to 0" variant (TAmbHiQCalcT0) */
    uint8_t wrap_x;      /* a panorama: the left and right edges are neighbours */
    uint8_t random;      /* random sampling with this many passes (TAmbHiQCalcR, SSAORcount); 0: regular */
    uint8_t pad;
} mb3d_cu_ssao_opts;

/* SsaoParams::default (threshold 2, no mirrored border, no wrap). */
void mb3d_cu_ssao_default(mb3d_cu_ssao_opts *out);

/* Replaces gpu::ssao24 (src/gpu.rs:3503; ssao::ssao24, src/ssao.rs:129-335):
 * the scene's whole G-buffer (width * height records, host or device) gets
 * the ambient shadow (amb_shadow, 0..16383) of its object pixels from the
 * depth buffer alone: per pixel the largest elevation angle in 32 directions
 * on ever smoother levels of the depth buffer, their arctangents summed.
 * Regular or random sampling (EINVAL for an opts outside the documented
 * ranges); the older 15-bit variant is mb3d_cu_ssao15. */
int mb3d_cu_ssao24(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_ssao_opts *opts,
                   mb3d_cu_silight *gbuf);

/* Replaces gpu::ssao15 (src/gpu.rs:3726; ssao15::ssao15,
 * src/ssao15.rs:282-411, SsaoParams::bits15): the older "15 bit" ambient
 * occlusion of the object pixels of the scene's whole G-buffer (host or
 * device): the depth buffer scaled to 0..128 and smoothed into "a trous"
 * levels, per pixel the steepest slope per 1/32 circle over rings of
 * samples that widen with the level, the slopes' arctangents summed into
 * amb_shadow.  Uses threshold, t0 and wrap_x of opts (border_mirror and
 * random belong to the 24-bit pass); pictures below 4 x 4 are left as they
 * are, as the reference does. */
int mb3d_cu_ssao15(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_ssao_opts *opts,
                   mb3d_cu_silight *gbuf);

/* ---- the reflection pass's rays ----
 * A ray of the reflection and transparency pass (RayReq, src/reflect.rs:
 * 313-327): from a surface point along the reflected (or refracted) view
 * vector, for the pixel whose view it continues. */
typedef struct {
    double origin[3]; /* where the ray starts */
    double dir[3];    /* its direction, one step long (the pixel's view vector turned) */
    double zz;        /* the view depth at the origin, in steps */
    double max_len;   /* the longest march in steps; <= 0: the march's far end */
    uint32_t pixel;   /* the pixel the ray belongs to: y * width + x of the scene's picture */
    uint32_t rit;     /* the bounce, 1 for the first reflection: the hit's DE ambient
                         occlusion has quality 2, 1, then 0 and the weight 8 / (8 + rit) */
} mb3d_cu_reflect_ray;

/* The march of a ray (RayHit, src/reflect.rs:329-337). */
typedef struct {
    mb3d_cu_silight si;  /* the hit's record: normal, depth, colour, shadow bits, ambient
                            occlusion; the step count in shadow's low 10 bits; open air:
                            zpos_fine 32768 << 16 */
    uint8_t hit;         /* a surface was met */
    uint8_t de_limited;  /* the march stopped on the DE (not on the iteration limit) */
    uint8_t pad[2];
    double pos[3];       /* where the march ended */
    double zz;           /* the view depth there, in steps */
    double zz2_paint;    /* the length marched before the surface search, in steps */
    double zz2;          /* and after it */
} mb3d_cu_reflect_hit;

/* Replaces gpu::reflect_batch (src/gpu.rs:2521; on the CPU
 * SrTracer::march_ray, src/reflect.rs:1464-1675): the n rays marched in
 * double precision to their hits, which get their normal, colour, depth
 * (through the fog formula with far_fog: LightVals far_fog or squared
 * depth), the scene's hard or soft shadows (calc_hs, src/reflect.rs:805-952)
 * and, with the scene's DE ambient occlusion on, its occlusion at the hit
 * (deao_1pos, src/reflect.rs:954-1090).  Every ray is independent.  Rays and
 * hits in host or device memory.  ENOTSUP for what the card's pass leaves
 * to the CPU: a random first AO step (deao_first_step_random), dithering.
 * EINVAL for a pixel outside the picture. */
int mb3d_cu_reflect_batch(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_reflect_ray *rays, uint32_t n,
                          int far_fog, mb3d_cu_reflect_hit *hits);

/* The first bounce of every object pixel of a G-buffer (the scene's whole
 * picture, width * height records, host or device): start_pixel
 * (src/reflect.rs:1686-1838: the surface found again from the stored depth,
 * outside rendering, no water or cutting plane) and the mirror ray of step
 * (:1286-1311), rit 1, in pixel order into rays (room for width * height,
 * host or device); *n_rays receives their count.  Pixels whose surface the
 * search cannot find again send none, as in the reference. */
int mb3d_cu_reflect_first_rays(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_silight *gbuf,
                               mb3d_cu_reflect_ray *rays, uint32_t *n_rays);

/* ---- the learned denoiser of the Monte Carlo pictures ----
 * A 5-level U-Net of 3x3 convolutions (32/48/64/80/96 channels) that
 * takes the noisy colour and the albedo, normal and depth guides of a
 * picture and returns the denoised colour: the card's counterpart of the
 * Open Image Denoise call of mb3d-rs (oidn::Input, src/oidn.rs:170-180;
 * denoise_mc, src/oidn.rs:262-277), which the reference does not train.
 * Its weights are BF16 (FP32 master copies), its convolutions run on the
 * tensor cores with FP32 accumulation, and it is trained on the card on
 * pictures the path tracer renders (mb3d_cu_dn_train_step).  Inputs are
 * float arrays of n pictures of h x w pixels (colour, albedo, normal: 3
 * floats per pixel; depth: 1), host or device; albedo, normal and depth may
 * be NULL (zero guides).  depth_scale scales the depth to about 0..1. */
typedef struct mb3d_cu_dn mb3d_cu_dn;

/* The number of parameters (FP32 master weights and biases). */
size_t mb3d_cu_dn_param_count(void);

/* A denoiser on the context's device, its weights He-initialised from seed. */
int mb3d_cu_dn_create(mb3d_cu_ctx *ctx, uint64_t seed, mb3d_cu_dn **out);
void mb3d_cu_dn_free(mb3d_cu_dn *dn);

/* The FP32 parameters (mb3d_cu_dn_param_count floats, host or device). */
int mb3d_cu_dn_get_params(mb3d_cu_dn *dn, float *params);
int mb3d_cu_dn_set_params(mb3d_cu_dn *dn, const float *params);

/* The denoised colour of the pictures into out (n * h * w * 3 floats). */
int mb3d_cu_dn_denoise(mb3d_cu_dn *dn, int n, int h, int w, const float *radiance, const float *albedo,
                       const float *normal, const float *depth, float depth_scale, float *out);

/* The training loss of the denoiser: the L1 loss of log(1 + x) (the
 * default); the mean squared error of the tone-mapped colour x / (1 + x)
 * (its optimum for noisy targets is their mean, where the L1 loss's is a
 * median); or that plus the mean squared error of the colour clamped to
 * 0..1, which is what paint_recs makes of a record with its default display
 * settings (src/mc.rs:3957-4005: contrast 1, gamma and saturation neutral,
 * so the Lab round trip is the identity). */
#define MB3D_CU_DN_LOSS_L1_LOG 0
#define MB3D_CU_DN_LOSS_TONE_MSE 1
#define MB3D_CU_DN_LOSS_TONE_DISPLAY 2
int mb3d_cu_dn_set_loss(mb3d_cu_dn *dn, int kind);

/* One Adam step (learning rate lr) on the loss (mb3d_cu_dn_set_loss)
 * against target (n * h * w * 3 floats); *loss (may be NULL) receives the
 * loss before the step. */
int mb3d_cu_dn_train_step(mb3d_cu_dn *dn, int n, int h, int w, const float *radiance, const float *albedo,
                          const float *normal, const float *depth, float depth_scale, const float *target, float lr,
                          float *loss);

/* The plain trace as the denoiser's fallback and the judge of its error:
 * half_a and half_b are two traces of the same h x w picture from disjoint
 * halves of the rays (h * w * 3 floats each), den the denoised picture of
 * the whole trace.  Per tile x tile piece (the last row and column ragged),
 * in the tone x / (1 + x) of max(x, 0): where the mean of the denoised
 * piece leaves the mean of (half_a + half_b) / 2 by more than k times that
 * mean's noise (the halves' mean squared difference / 4 / the piece's
 * samples, square root, +0.001), out keeps (half_a + half_b) / 2, elsewhere
 * den; *plain_share (may be NULL) receives the share of such pieces.  out
 * may be den; every buffer host or device memory.  No counterpart in the
 * reference (its denoiser, src/oidn.rs:262-277, has no fallback). */
int mb3d_cu_dn_fallback(mb3d_cu_dn *dn, int h, int w, const float *half_a, const float *half_b, const float *den,
                        int tile, float k, float *out, float *plain_share);

/* The loss and its gradient with respect to every parameter (grad:
 * mb3d_cu_dn_param_count floats, host or device), without a step. */
int mb3d_cu_dn_gradient(mb3d_cu_dn *dn, int n, int h, int w, const float *radiance, const float *albedo,
                        const float *normal, const float *depth, float depth_scale, const float *target, float *loss,
                        float *grad);

/* Test hook: one 3x3 convolution (NHWC, cin and cout multiples of 16,
 * cout <= 128, weights [cout][3][3][cin]) and its gradients for the output
 * gradient dy, through the same kernels, on float host arrays (BF16
 * inside). */
int mb3d_cu_dn_conv_check(mb3d_cu_ctx *ctx, int n, int h, int w, int cin, int cout, const float *x, const float *wt,
                          const float *b, const float *dy, float *y, float *dx, float *dw, float *db);

/* Test hook of the tensor-core pipeline's bounded waits: one 16 -> 16
 * channel convolution of a 16 x 16 picture whose waits give up after
 * wait_us microseconds (1 .. 2e6).  With no_issue the TMA and MMA lanes
 * issue nothing, so the epilogue's first accumulator wait runs out with no
 * copy or MMA in flight: the kernel frees its tensor memory and returns,
 * and the call answers MB3D_CU_EIO ("a pipeline wait ran out"); the context
 * stays usable.  No counterpart in the reference (it has no network). */
int mb3d_cu_dn_wait_check(mb3d_cu_ctx *ctx, double wait_us, int no_issue);

/* Depth of field (DofParams, src/dof.rs:13-31): every pixel of the painted
 * picture spread over a disk whose radius grows with its distance from the
 * focus. */
typedef struct mb3d_cu_dof_opts {
    float z_sharp, z_sharp2; /* the focus distances as a fraction of the picture's width; between them all is sharp */
    float aperture;          /* 0.0001 .. 2 */
    float clip_r;            /* the largest blur radius, pixels */
    uint8_t passes;          /* 1 .. 4, each with a larger radius */
    uint8_t forward;         /* 1: the forward variant (all pixels spread at once); 0: the default sorted one (the
                              * pixels back to front, near blurred objects covering the sharp ones behind them) */
    uint8_t pad[2];
} mb3d_cu_dof_opts;

/* DofParams::default (src/dof.rs:33-37).  Host code only. */
void mb3d_cu_dof_default(mb3d_cu_dof_opts *out);

/* Replaces dof::apply (src/dof.rs:81-122) with its card path
 * (src/dof.rs:425-723, gpu_dof.wgsl): all passes of the depth of field on
 * the 8-bit picture `rgb` (width * height * 3, in place) of the G-buffer
 * `gbuf` (width * height records) of `scene`; both host or device.  Each
 * output pixel takes its sources in the reference's order (the sorted
 * variant: back to front by fine depth, ties in pixel order; the forward
 * one: pixel order), so its sums are the reference's. */
int mb3d_cu_dof(mb3d_cu_ctx *ctx, const mb3d_cu_scene *scene, const mb3d_cu_dof_opts *opts,
                const mb3d_cu_silight *gbuf, uint8_t *rgb);

/* The march without any device allocation, for callers that cannot
 * allocate GPU memory: a renderer whose device memory belongs to another
 * allocator (an engine's fixed pool, PyTorch's caching allocator), which may
 * not call cudaMalloc/cudaFree behind that allocator's back, and render
 * loops that cannot take the device-wide synchronisation cudaMalloc and
 * cudaFree imply.  It has no counterpart in the reference (mb3d-rs's card
 * backend allocates its wgpu buffers per render).
 *
 * It marches rows row0 .. row0+rows of the picture into `gbuf`, which must
 * be device memory (rows * width records), on `stream` (a cudaStream_t of
 * gbuf's device, NULL for that device's default stream), and returns when the
 * work is queued; the calling thread's current device is the same after the
 * call as before it.  Its
 * scratch (the lists the march hands its surfaces over in) is a static
 * device array of this library, MB3D_CU_NOALLOC_MAX_PIXELS pixels' worth
 * (10.5 MB, held by every GPU that loads the library until the process
 * exits); a band larger than that is rejected (MB3D_CU_EINVAL).  The first
 * call on a device looks up the array's device address, so make that first
 * call before any stream capture.  Every call shares the one array: calls
 * that overlap on the GPU (two streams, or two host threads) race and must
 * be ordered by the caller.  Results are those of mb3d_cu_march. */
#define MB3D_CU_NOALLOC_MAX_PIXELS 65536
int mb3d_cu_march_noalloc(const mb3d_cu_scene *scene, int precision, uint32_t row0, uint32_t rows,
                          mb3d_cu_silight *gbuf, void *stream);

#ifdef __cplusplus
}
#endif

#endif
