// The C ABI (include/mb3d_cu.h): contexts, buffers, launches and the error
// convention of mb3d-rs's C API (a thread-local last error,
// capi/src/lib.rs:18-40).  There is no CPU fallback: a failure is a
// negative status and the caller decides what to do.
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/mb3d_cu.h"
#include "devparams.h"
#include "kernels.h"
#include "setup.h"
#include "mcsetup.h"

using namespace mb3dcu;

static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

struct mb3d_cu_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    mb3d_cu_silight *d_gbuf = nullptr;
    size_t gbuf_cap = 0;
    Hand *d_hand = nullptr;
    size_t hand_cap = 0;
    Hand *d_slow = nullptr;  // the finish's rare cases
    size_t slow_cap = 0;
    uint32_t *d_slist = nullptr;  // surface pixels of the post passes
    size_t slist_cap = 0;
    PostStart *d_ps = nullptr;
    size_t ps_cap = 0;
    float *d_minra = nullptr;     // the DE AO rays' openness
    size_t minra_cap = 0;
    unsigned int *d_counters = nullptr;
    unsigned int *h_counters = nullptr;  // (pinned) the march's list lengths, read back with each call
    bool read_slow = false;
    bool read_status = false;  // h_counters holds the march's status word
    double *d_probe = nullptr;
    size_t probe_cap = 0;
    cudaEvent_t ev[9] = {};
    // the post passes: the shadow rays run on `aux` beside the DE AO rays
    cudaStream_t aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // the frame batches: extra streams, their scratch sets, the output staging
    struct Scratch {
        Hand *hand = nullptr, *slow = nullptr;
        uint32_t *slist = nullptr;
        PostStart *ps = nullptr;
        float *minra = nullptr;
        unsigned int *counters = nullptr;
        size_t npix = 0, nray = 0;
    };
    std::vector<cudaStream_t> fstreams;
    std::vector<cudaEvent_t> fevents;
    std::vector<Scratch> fscratch;
    mb3d_cu_silight *d_frames = nullptr;
    size_t frames_cap = 0;
    mb3d_cu_stats stats = {};
    int counting = 0;
    unsigned long long *d_count = nullptr;
    // the Monte Carlo tracer: the Halton table, the pixel sums and the
    // staging of its requests, results and per pixel outputs
    uint2 *d_halton = nullptr;
    unsigned char *d_mc = nullptr;
    size_t mc_cap = 0;
    unsigned char *d_mcs = nullptr;  // the split render's paths, requests, results, list
    size_t mcs_cap = 0;
    unsigned char *d_mcitems = nullptr;  // the adaptive pass's items (pixel, ray number)
    size_t mcitems_cap = 0;
    unsigned char *d_dof = nullptr;    // the depth of field's pictures, sources and keys
    size_t dof_cap = 0;
    unsigned char *d_refl = nullptr;   // the reflection pass's rays, hits and AO table
    size_t refl_cap = 0;
    unsigned char *d_paint = nullptr;  // the painter's staging of host buffers
    size_t paint_cap = 0;
    unsigned char *d_ssao = nullptr;   // the SSAO's levels and angles (and a host G-buffer's staging)
    size_t ssao_cap = 0;
    // a budgeted march (mb3d_cu_march_ex) that ran out of time: where it
    // stopped; the device keeps its G-buffer rows, lists and queue counters
    // until the same call comes again (any other call drops it)
    struct Resume {
        bool active = false;
        mb3d_cu_scene scene;
        int precision = 0;
        uint32_t row0 = 0, rows = 0, band_rows = 0;
        mb3d_cu_silight *gbuf = nullptr;
        uint32_t band = 0;   // the band in progress
        int stage = 0;       // 0 its counters to clear, 1 the march, 2 the finish, 3 the slow finish
        uint64_t overflow = 0, fp64_pixels = 0;  // summed over the finished bands
    } resume;
    std::mutex mu;
};

#define CU_TRY(call)                                                                             \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? MB3D_CU_ENOMEM : MB3D_CU_EIO,          \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

static int grow(void **ptr, size_t *cap, size_t need) {
    if (*cap >= need) return 0;
    if (*ptr) cudaFree(*ptr);
    *ptr = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc(ptr, need);
    if (e != cudaSuccess) return fail(MB3D_CU_ENOMEM, std::string("device memory: ") + cudaGetErrorString(e));
    *cap = need;
    return 0;
}

static bool is_device_ptr(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

static int check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string(what) + ": " + cudaGetErrorString(e));
    return 0;
}

// the context's pieces the denoiser (dn.cu) uses
namespace mb3dcu {
int dn_fail(int code, const std::string &msg) { return fail(code, msg); }
bool dn_is_device_ptr(const void *p) { return is_device_ptr(p); }
cudaStream_t dn_stream(mb3d_cu_ctx *c) { return c->stream; }
int dn_device(mb3d_cu_ctx *c) { return c->device; }
}  // namespace mb3dcu

extern "C" {

const char *mb3d_cu_version(void) { return "mb3d_cu 0.1.0 (sm_100a)"; }

const char *mb3d_cu_last_error(void) { return g_last_error.c_str(); }

int mb3d_cu_init(int device, mb3d_cu_ctx **out) {
    if (!out) return fail(MB3D_CU_EINVAL, "out is NULL");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(MB3D_CU_ENODEV, "no CUDA device");
    if (device < 0 || device >= n) return fail(MB3D_CU_EINVAL, "no such device");
    cudaDeviceProp prop;
    CU_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(MB3D_CU_ENODEV, std::string("not an sm_100 device: ") + prop.name);
    CU_TRY(cudaSetDevice(device));
    mb3d_cu_ctx *c = new mb3d_cu_ctx();
    c->device = device;
    c->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return fail(MB3D_CU_EIO, "stream create failed");
    }
    c->stream = c->own;
    for (auto &ev : c->ev) cudaEventCreate(&ev);
    if (cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming) != cudaSuccess) {
        mb3d_cu_free(c);
        return fail(MB3D_CU_EIO, "stream create failed");
    }
    if (cudaMalloc(&c->d_counters, 64 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMallocHost(&c->h_counters, 64 * sizeof(unsigned int)) != cudaSuccess) {
        mb3d_cu_free(c);
        return fail(MB3D_CU_ENOMEM, "device memory");
    }
    *out = c;
    return 0;
}

void mb3d_cu_free(mb3d_cu_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->own) cudaStreamSynchronize(c->own);
    if (c->stream && c->stream != c->own) cudaStreamSynchronize(c->stream);
    if (c->aux) cudaStreamSynchronize(c->aux);
    cudaFree(c->d_gbuf);
    cudaFree(c->d_hand);
    cudaFree(c->d_slow);
    cudaFree(c->d_slist);
    cudaFree(c->d_ps);
    cudaFree(c->d_minra);
    cudaFree(c->d_counters);
    cudaFreeHost(c->h_counters);
    cudaFree(c->d_probe);
    cudaFree(c->d_count);
    cudaFree(c->d_halton);
    cudaFree(c->d_mc);
    cudaFree(c->d_mcs);
    cudaFree(c->d_mcitems);
    cudaFree(c->d_dof);
    cudaFree(c->d_refl);
    cudaFree(c->d_paint);
    cudaFree(c->d_ssao);
    for (auto &ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    for (auto &s : c->fscratch) {
        cudaFree(s.hand);
        cudaFree(s.slow);
        cudaFree(s.slist);
        cudaFree(s.ps);
        cudaFree(s.minra);
        cudaFree(s.counters);
    }
    for (auto s : c->fstreams) cudaStreamDestroy(s);
    for (auto e : c->fevents) cudaEventDestroy(e);
    cudaFree(c->d_frames);
    if (c->own) cudaStreamDestroy(c->own);
    if (c->aux) cudaStreamDestroy(c->aux);
    delete c;
}

int mb3d_cu_set_stream(mb3d_cu_ctx *c, void *stream) {
    if (!c) return fail(MB3D_CU_EINVAL, "ctx is NULL");
    c->stream = stream ? (cudaStream_t)stream : c->own;
    return 0;
}

int mb3d_cu_unsupported(const mb3d_cu_scene *sc, char *reason, size_t cap) {
    if (!sc) return fail(MB3D_CU_EINVAL, "scene is NULL");
    std::string why;
    int r = unsupported_reason(*sc, why);
    if (r == 0) {
        DevParams p;
        std::string err;
        int s = setup_params(*sc, p, err);
        if (s == MB3D_CU_ENOTSUP) {
            why = err;
            r = 1;
        } else if (s < 0) {
            why = err;
            r = s;
        }
    }
    if (reason && cap > 0) {
        std::strncpy(reason, why.c_str(), cap - 1);
        reason[cap - 1] = 0;
    }
    if (r < 0) return fail(r, why);
    return r;
}

// the march of rows row0.. into the device buffer dg (band-sized)
static int march_device(mb3d_cu_ctx *c, const DevParams &p, int precision, int row0, int rows, mb3d_cu_silight *dg) {
    cudaStream_t s = c->stream;
    size_t npix = (size_t)rows * p.width;
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    c->stats.fp64_pixels = (precision != MB3D_CU_FP64 && p.all_fp64) ? (uint32_t)npix : 0u;
    if (int r = grow((void **)&c->d_hand, &c->hand_cap, npix * sizeof(Hand))) return r;
    CU_TRY(cudaMemsetAsync(c->d_counters, 0, 64 * sizeof(unsigned int), s));
    if (c->counting) {
        if (!c->d_count) CU_TRY(cudaMalloc(&c->d_count, 16 * sizeof(unsigned long long)));
        CU_TRY(cudaMemsetAsync(c->d_count, 0, 16 * sizeof(unsigned long long), s));
    }
    int items = ((p.width + 7) / 8) * ((rows + 3) / 4);  // warps' worth of work
    int blocks = c->sms * (mixed ? p.blocks_march32 : p.blocks_per_sm);
    int need = (items + 7) / 8;
    if (blocks > need) blocks = need > 0 ? need : 1;
    CU_TRY(cudaEventRecord(c->ev[0], s));
    launch_march(p, mixed, row0, rows, dg, c->d_hand, c->d_counters, c->counting ? c->d_count : nullptr, blocks, s);
    if (int r = check_launch("k_march")) return r;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (int r = grow((void **)&c->d_slow, &c->slow_cap, npix * sizeof(Hand))) return r;
    launch_finish(p, mixed, row0, c->d_hand, c->d_counters, c->d_slow, dg, c->sms * p.blocks_per_sm, s);
    if (int r = check_launch("k_finish")) return r;
    CU_TRY(cudaEventRecord(c->ev[2], s));
    c->stats.launches += 3;
    // the slow list's length: the mixed mode's pixels finished by the
    // per-thread double precision marcher
    c->read_slow = mixed;
    c->read_status = true;
    CU_TRY(cudaMemcpyAsync(c->h_counters, c->d_counters, (CNT_OVERFLOW + 1) * sizeof(unsigned int),
                           cudaMemcpyDeviceToHost, s));
    return 0;
}

// the post passes: the surface pixels listed, their start points found,
// then one lane per shadow ray and per DE AO ray
static int post_device(mb3d_cu_ctx *c, const DevParams &p, int precision, int passes, int row0, int rows,
                       mb3d_cu_silight *dg) {
    cudaStream_t s = c->stream;
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    if (!(passes & MB3D_CU_POST_SHADOW) || p.n_lights == 0) passes &= ~MB3D_CU_POST_SHADOW;
    if (!(passes & MB3D_CU_POST_DEAO) || p.ao_quality < 0 || p.ao_rays == 0) passes &= ~MB3D_CU_POST_DEAO;
    size_t npix = (size_t)rows * p.width;
    if (int r = grow((void **)&c->d_slist, &c->slist_cap, npix * sizeof(uint32_t))) return r;
    if (int r = grow((void **)&c->d_ps, &c->ps_cap, npix * sizeof(PostStart))) return r;
    if (passes & MB3D_CU_POST_DEAO)
        if (int r = grow((void **)&c->d_minra, &c->minra_cap, (npix * (size_t)p.ao_rays + 4) * AO_MINRA_BYTES)) return r;
    // [0] surfaces, [1] shadow queue, [2] AO queue, [3] start queue, [4] AO rays handed to FP64, [5] their queue
    unsigned int *cnt = c->d_counters + 8;
    CU_TRY(cudaMemsetAsync(cnt, 0, 8 * sizeof(unsigned int), s));
    CU_TRY(cudaEventRecord(c->ev[3], s));
    launch_surface(p, (int)npix, passes, dg, c->d_slist, cnt, c->sms * 4, s);
    c->stats.launches += 1;
    if (passes) {
        launch_post_start(p, mixed, row0, passes, dg, c->d_slist, cnt, cnt + 3, c->d_ps, c->sms * p.blocks_per_sm, s);
        c->stats.launches += 1;
        if (int r = check_launch("k_post_start")) return r;
    }
    // with both passes the shadow rays run on the second stream beside the DE
    // AO rays (they share only the start points, read-only; the shadow bits
    // are atomic updates of a word the DE AO rays do not use), and the DE AO
    // pass's last kernel, which writes that word, waits for them
    const bool both = (passes & MB3D_CU_POST_SHADOW) && (passes & MB3D_CU_POST_DEAO);
    if (passes & MB3D_CU_POST_SHADOW) {
        cudaStream_t ss = s;
        if (both) {
            CU_TRY(cudaEventRecord(c->fork, s));
            CU_TRY(cudaStreamWaitEvent(c->aux, c->fork, 0));
            ss = c->aux;
        }
        launch_shadow_rays(p, mixed, row0, c->d_ps, cnt, dg, cnt + 1, c->sms * p.blocks_per_sm, ss);
        c->stats.launches += 1;
        if (int r = check_launch("k_shadow_rays")) return r;
        CU_TRY(cudaEventRecord(c->ev[8], ss));
        if (both) CU_TRY(cudaEventRecord(c->join, ss));
    } else {
        CU_TRY(cudaEventRecord(c->ev[8], s));
    }
    CU_TRY(cudaEventRecord(c->ev[4], s));
    if (passes & MB3D_CU_POST_DEAO) {
        launch_ao_prep(p, c->d_ps, dg, cnt, c->sms * 8, s);
        launch_ao_rays(p, mixed, c->d_ps, dg, cnt, c->d_minra, cnt + 2, c->sms * p.blocks_per_sm, s);
        if (both) CU_TRY(cudaStreamWaitEvent(s, c->join, 0));
        launch_ao_final(p, c->d_ps, cnt, c->d_minra, dg, c->sms * 8, s);
        c->stats.launches += 3;
        if (int r = check_launch("k_ao")) return r;
    }
    CU_TRY(cudaEventRecord(c->ev[5], s));
    return 0;
}

static int finish_call(mb3d_cu_ctx *c, bool marched, bool posted) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    if (marched && c->read_slow) {
        c->stats.fp64_pixels = c->h_counters[CNT_SLOW];
        c->stats.fp32_overflow_pixels = c->h_counters[CNT_OVERFLOW];
    }
    c->read_slow = false;
    if (marched && c->read_status && (c->h_counters[CNT_STATUS] & ST_TRIP_CAP)) {
        c->read_status = false;
        return fail(MB3D_CU_EIO, "a march kernel ran out of its loop trips: rays left unmarched");
    }
    c->read_status = false;
    if (marched && c->counting && c->d_count) {
        unsigned long long h[16];
        CU_TRY(cudaMemcpy(h, c->d_count, sizeof(h), cudaMemcpyDeviceToHost));
        for (int k = 0; k < 6; k++) c->stats.orbit_its[k] = h[k];
        c->stats.de_evals = h[6];
        c->stats.march_lane_its = h[7];
        c->stats.march_warp_its = h[8];
        c->stats.march_trips = h[9];
        c->stats.march_busy_lanes = h[10];
    }
    float ms = 0.f;
    if (marched) {
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]);
        c->stats.ms_march = ms;
        cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
        c->stats.ms_finish = ms;
    }
    if (posted) {
        cudaEventElapsedTime(&ms, c->ev[3], c->ev[8]);
        c->stats.ms_shadow = ms;
        cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
        c->stats.ms_deao = ms;
    }
    cudaEventElapsedTime(&ms, marched ? c->ev[0] : c->ev[3], posted ? c->ev[5] : c->ev[2]);
    c->stats.ms_total = ms;
    return 0;
}

// launch tuning: MB3D_CU_TUNE="refill=8,refill_sh=8,refill_ao=16,blocks=4,margin=4,back=2"
static void apply_tuning(DevParams &p) {
    const char *t = getenv("MB3D_CU_TUNE");
    if (!t) return;
    std::string s(t);
    size_t i = 0;
    while (i < s.size()) {
        size_t j = s.find(',', i);
        if (j == std::string::npos) j = s.size();
        std::string kv = s.substr(i, j - i);
        size_t e = kv.find('=');
        if (e != std::string::npos) {
            std::string k = kv.substr(0, e);
            double v = atof(kv.c_str() + e + 1);
            if (k == "refill" && v >= 1 && v <= 32) p.refill_min = (int)v;
            else if (k == "refill_sh" && v >= 1 && v <= 32) p.refill_shadow = (int)v;
            else if (k == "refill_ao" && v >= 1 && v <= 32) p.refill_ao = (int)v;
            else if (k == "blocks32" && v >= 1 && v <= 8) p.blocks_march32 = (int)v;
            else if (k == "blocks" && v >= 1 && v <= 16) p.blocks_per_sm = (int)v;
            else if (k == "margin" && v >= 1) p.hand_margin = (float)v;
            else if (k == "back" && v >= 0 && v <= 2) p.hand_back = (int)v;
            else if (k == "sched" && v == 0) p.sched = SCHED_GENERIC;
        }
        i = j + 1;
    }
}

static int run(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, int passes, bool do_march, uint32_t row0,
               uint32_t rows, mb3d_cu_silight *gbuf, const volatile int *cancel) {
    if (!c || !sc || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    apply_tuning(p);
    if ((uint64_t)row0 + rows > (uint64_t)p.height || rows == 0) return fail(MB3D_CU_EINVAL, "rows outside the picture");
    if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    std::memset(&c->stats, 0, sizeof(c->stats));
    size_t npix = (size_t)rows * p.width;
    bool dev = is_device_ptr(gbuf);
    mb3d_cu_silight *dg = gbuf;
    if (!dev) {
        if (int e = grow((void **)&c->d_gbuf, &c->gbuf_cap, npix * sizeof(mb3d_cu_silight))) return e;
        dg = c->d_gbuf;
        if (!do_march) CU_TRY(cudaMemcpyAsync(dg, gbuf, npix * sizeof(mb3d_cu_silight), cudaMemcpyHostToDevice, c->stream));
    }
    if (do_march) {
        if (int e = march_device(c, p, precision, (int)row0, (int)rows, dg)) return e;
    }
    if (passes) {
        if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
        if (int e = post_device(c, p, precision, passes, (int)row0, (int)rows, dg)) return e;
    }
    if (!dev) CU_TRY(cudaMemcpyAsync(gbuf, dg, npix * sizeof(mb3d_cu_silight), cudaMemcpyDeviceToHost, c->stream));
    if (int e = finish_call(c, do_march, passes != 0)) return e;
    if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    return 0;
}

int mb3d_cu_march(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, uint32_t row0, uint32_t rows,
                  mb3d_cu_silight *gbuf, const volatile int *cancel) {
    return run(c, sc, precision, 0, true, row0, rows, gbuf, cancel);
}

int mb3d_cu_post(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, int passes, uint32_t row0, uint32_t rows,
                 mb3d_cu_silight *gbuf, const volatile int *cancel) {
    if (passes & ~(MB3D_CU_POST_SHADOW | MB3D_CU_POST_DEAO)) return fail(MB3D_CU_EINVAL, "unknown post pass bits");
    if (passes == 0) return 0;
    return run(c, sc, precision, passes, false, row0, rows, gbuf, cancel);
}

int mb3d_cu_render(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, mb3d_cu_silight *gbuf,
                   const volatile int *cancel) {
    if (!sc) return fail(MB3D_CU_EINVAL, "scene is NULL");
    int passes = (sc->shadow_lights ? MB3D_CU_POST_SHADOW : 0) | (sc->deao_quality >= 0 ? MB3D_CU_POST_DEAO : 0);
    return run(c, sc, precision, passes, true, 0, (uint32_t)sc->height, gbuf, cancel);
}

// ---------------------------------------------------------------------------
// the march with gpu::march's progress and cancel per band, the device time
// budget (resumable) and the reference card's overflow rule

static bool same_scene(const mb3d_cu_scene &a, const mb3d_cu_scene &b) { return std::memcmp(&a, &b, sizeof a) == 0; }

// one stage of a band on the context's stream; with a budget it waits for
// the launch and tells whether the budget stopped it (*stopped)
static int band_stage(mb3d_cu_ctx *c, const DevParams &p, bool mixed, int stage, int r0, int nr, mb3d_cu_silight *dg,
                      bool *stopped) {
    cudaStream_t s = c->stream;
    *stopped = false;
    int blocks = c->sms * p.blocks_per_sm;
    if (stage == 1) {
        int items = ((p.width + 7) / 8) * ((nr + 3) / 4);
        int mb = c->sms * (mixed ? p.blocks_march32 : p.blocks_per_sm);
        int need = (items + 7) / 8;
        if (mb > need) mb = need > 0 ? need : 1;
        launch_march(p, mixed, r0, nr, dg, c->d_hand, c->d_counters, nullptr, mb, s);
    } else if (stage == 2) {
        launch_finish_fast(p, mixed, r0, c->d_hand, c->d_counters, c->d_slow, dg, blocks, s);
    } else {
        launch_finish_slow(p, mixed, r0, c->d_hand, c->d_counters, c->d_slow, dg, blocks, s);
    }
    if (int e = check_launch(stage == 1 ? "k_march" : stage == 2 ? "k_finish" : "k_finish_slow")) return e;
    c->stats.launches += 1;
    if (p.budget_ns != 0) {
        CU_TRY(cudaMemcpyAsync(c->h_counters, c->d_counters, (CNT_OVERFLOW + 1) * sizeof(unsigned int),
                               cudaMemcpyDeviceToHost, s));
        CU_TRY(cudaStreamSynchronize(s));
        const unsigned int bit = stage == 1 ? 1u : stage == 2 ? 2u : 4u;
        *stopped = (c->h_counters[CNT_STATUS] & bit) != 0;
    }
    return 0;
}

int mb3d_cu_march_ex(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, uint32_t row0, uint32_t rows,
                     mb3d_cu_silight *gbuf, const mb3d_cu_march_opts *opts) {
    if (!c || !sc || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    mb3d_cu_march_opts o = {};
    if (opts) o = *opts;
    if (!(o.budget_ms >= 0.0) || o.budget_ms > 3.6e6) return fail(MB3D_CU_EINVAL, "budget_ms outside 0 .. 3.6e6");
    std::lock_guard<std::mutex> lk(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) {
        c->resume.active = false;
        return fail(r, err);
    }
    apply_tuning(p);
    if ((uint64_t)row0 + rows > (uint64_t)p.height || rows == 0) {
        c->resume.active = false;
        return fail(MB3D_CU_EINVAL, "rows outside the picture");
    }
    const uint32_t band_rows = o.band_rows == 0 || o.band_rows > rows ? rows : o.band_rows;
    mb3d_cu_ctx::Resume &rs = c->resume;
    const bool resuming = rs.active && same_scene(rs.scene, *sc) && rs.precision == precision && rs.row0 == row0 &&
                          rs.rows == rows && rs.gbuf == gbuf && rs.band_rows == band_rows;
    if (!resuming) {
        rs = mb3d_cu_ctx::Resume();
        rs.scene = *sc;
        rs.precision = precision;
        rs.row0 = row0;
        rs.rows = rows;
        rs.band_rows = band_rows;
        rs.gbuf = gbuf;
    }
    rs.active = false;  // (set again only where the budget stops the call)
    std::memset(&c->stats, 0, sizeof(c->stats));
    p.budget_ns = (unsigned long long)(o.budget_ms * 1e6);
    if (o.budget_ms > 0.0 && p.budget_ns == 0) p.budget_ns = 1;
    const bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    const size_t npix = (size_t)rows * p.width, band_pix = (size_t)band_rows * p.width;
    const bool dev = is_device_ptr(gbuf);
    mb3d_cu_silight *dg = gbuf;
    if (!dev) {
        if (int e = grow((void **)&c->d_gbuf, &c->gbuf_cap, npix * sizeof(mb3d_cu_silight))) return e;
        dg = c->d_gbuf;
    }
    if (int e = grow((void **)&c->d_hand, &c->hand_cap, band_pix * sizeof(Hand))) return e;
    if (int e = grow((void **)&c->d_slow, &c->slow_cap, band_pix * sizeof(Hand))) return e;
    cudaStream_t s = c->stream;
    const uint32_t n_bands = (rows + band_rows - 1) / band_rows;
    for (; rs.band < n_bands; rs.band++, rs.stage = 0) {
        const uint32_t r0 = rs.band * band_rows, nr = std::min(band_rows, rows - r0);
        mb3d_cu_silight *bg = dg + (size_t)r0 * p.width;
        if (rs.stage == 0) {
            CU_TRY(cudaMemsetAsync(c->d_counters, 0, 64 * sizeof(unsigned int), s));
            rs.stage = 1;
        } else {
            // a new call: the budget's clock and status start again
            CU_TRY(cudaMemsetAsync(c->d_counters + CNT_T0, 0, 3 * sizeof(unsigned int), s));
        }
        for (; rs.stage <= 3; rs.stage++) {
            bool stopped = false;
            if (int e = band_stage(c, p, mixed, rs.stage, (int)(row0 + r0), (int)nr, bg, &stopped)) return e;
            if (stopped) {
                rs.active = true;
                c->stats.fp64_pixels = (uint32_t)rs.fp64_pixels;
                return fail(MB3D_CU_ETIMEDOUT, "the device time budget ran out in band " + std::to_string(rs.band) +
                                                   " (call again with the same arguments to go on)");
            }
        }
        // the band is done: its counts, its rows to the host, progress, cancel
        CU_TRY(cudaMemcpyAsync(c->h_counters, c->d_counters, (CNT_OVERFLOW + 1) * sizeof(unsigned int),
                               cudaMemcpyDeviceToHost, s));
        if (!dev)
            CU_TRY(cudaMemcpyAsync(gbuf + (size_t)r0 * p.width, bg, (size_t)nr * p.width * sizeof(mb3d_cu_silight),
                                   cudaMemcpyDeviceToHost, s));
        CU_TRY(cudaStreamSynchronize(s));
        rs.overflow += c->h_counters[CNT_OVERFLOW];
        if (mixed) rs.fp64_pixels += c->h_counters[CNT_SLOW];
        if (o.progress && o.progress(r0 + nr, rows, o.user) != 0) return fail(MB3D_CU_ECANCELED, "cancelled");
        if (o.cancel && *o.cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    }
    c->stats.fp64_pixels = (uint32_t)(mixed ? rs.fp64_pixels : (precision != MB3D_CU_FP64 ? npix : 0));
    c->stats.fp32_overflow_pixels = (uint32_t)rs.overflow;
    // src/gpu.rs:2361-2370: many pixels whose single precision DE overflowed
    // make the reference's card give the picture up (the host then renders
    // it on the CPU); here they were marched in double precision, and the
    // rule applies only where the caller asks for it
    if (o.overflow_fail && mixed && rs.overflow * 500 > npix)
        return fail(MB3D_CU_EOVERFLOW, "single precision overflows in " + std::to_string(rs.overflow) + " of " +
                                           std::to_string(npix) + " pixels");
    return 0;
}

int mb3d_cu_de_probe(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, const double *pos, uint32_t n, double *de,
                     int32_t *its) {
    if (!c || !sc || !pos || !de || !its) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (n == 0) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    size_t need = (size_t)n * 5 * sizeof(double);
    if (int e = grow((void **)&c->d_probe, &c->probe_cap, need)) return e;
    double *dpos = c->d_probe, *dde = c->d_probe + 3 * (size_t)n;
    int *dits = (int *)(c->d_probe + 4 * (size_t)n);
    CU_TRY(cudaMemcpyAsync(dpos, pos, (size_t)n * 3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    launch_de_probe(p, dpos, (int)n, dde, dits, precision != MB3D_CU_FP64 && !p.all_fp64, c->stream);
    if (int e = check_launch("k_de_probe")) return e;
    CU_TRY(cudaMemcpyAsync(de, dde, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU_TRY(cudaMemcpyAsync(its, dits, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CU_TRY(cudaStreamSynchronize(c->stream));
    return 0;
}

int mb3d_cu_stats_get(const mb3d_cu_ctx *c, mb3d_cu_stats *out) {
    if (!c || !out) return fail(MB3D_CU_EINVAL, "NULL argument");
    *out = c->stats;
    return 0;
}

// ---------------------------------------------------------------------------
// the allocation-free march: its scratch is this file's static device array
// (the march's hand-over list, the finish's slow list, the queue counters)

#define NOALLOC_COUNTER_BYTES 256
#define NOALLOC_BYTES (2 * (size_t)MB3D_CU_NOALLOC_MAX_PIXELS * sizeof(Hand) + NOALLOC_COUNTER_BYTES)
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

struct NoallocDevice {
    void *scratch = nullptr;  // the array's device address on this device
    int sms = 0;
};
static std::mutex g_noalloc_mu;
static NoallocDevice g_noalloc_dev[64];

// once per device, with the device current: the device address of the
// static array (its host-side name is only a stand-in) and the SM count
static int noalloc_setup(int dev, NoallocDevice &out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (dev < 0 || dev >= 64) return fail(MB3D_CU_ENODEV, "device index out of range");
    NoallocDevice &d = g_noalloc_dev[dev];
    if (!d.scratch) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(MB3D_CU_EIO, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || sms <= 0) return fail(MB3D_CU_EIO, std::string("SM count: ") + cudaGetErrorString(e));
        d.sms = sms;
        d.scratch = ptr;
    }
    out = d;
    return 0;
}

int mb3d_cu_march_noalloc(const mb3d_cu_scene *sc, int precision, uint32_t row0, uint32_t rows,
                          mb3d_cu_silight *gbuf, void *stream) {
    if (!sc || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    apply_tuning(p);  // (the launch settings mb3d_cu_march takes, so that the records are its records)
    if (rows == 0 || (uint64_t)row0 + rows > (uint64_t)p.height) return fail(MB3D_CU_EINVAL, "rows outside the picture");
    uint64_t npix = (uint64_t)rows * (uint64_t)p.width;
    if (npix > MB3D_CU_NOALLOC_MAX_PIXELS)
        return fail(MB3D_CU_EINVAL, "band of " + std::to_string(npix) + " pixels is over the allocation-free limit of " +
                                        std::to_string(MB3D_CU_NOALLOC_MAX_PIXELS) + " (march it in smaller bands)");
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, gbuf) != cudaSuccess ||
        !(a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged)) {
        cudaGetLastError();
        return fail(MB3D_CU_EINVAL, "gbuf must be device memory");
    }
    int dev = a.device;
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaGetDevice failed");
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    // the caller's current device is put back on every return
    struct Restore {
        int dev;
        ~Restore() { cudaSetDevice(dev); }
    } restore{cur};
    NoallocDevice d;
    if (int e = noalloc_setup(dev, d)) return e;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *base = (unsigned char *)d.scratch;
    Hand *list = (Hand *)base;
    Hand *slow = list + MB3D_CU_NOALLOC_MAX_PIXELS;
    unsigned int *counters = (unsigned int *)(slow + MB3D_CU_NOALLOC_MAX_PIXELS);
    // the queues and list lengths start at zero; the lists need no clearing
    CU_TRY(cudaMemsetAsync(counters, 0, NOALLOC_COUNTER_BYTES, s));
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    int items = ((p.width + 7) / 8) * (((int)rows + 3) / 4);
    int blocks = d.sms * (mixed ? p.blocks_march32 : p.blocks_per_sm);
    int need = (items + 7) / 8;
    if (blocks > need) blocks = need > 0 ? need : 1;
    launch_march(p, mixed, (int)row0, (int)rows, gbuf, list, counters, nullptr, blocks, s);
    if (int e = check_launch("k_march")) return e;
    launch_finish(p, mixed, (int)row0, list, counters, slow, gbuf, d.sms * p.blocks_per_sm, s);
    if (int e = check_launch("k_finish")) return e;
    return 0;
}

// ---------------------------------------------------------------------------
// frame batches (one CUDA graph over all frames, frames spread over streams)

// one frame's whole pipeline on stream s with scratch set sc (no events,
// no synchronisation: what the graph captures)
static int enqueue_frame(mb3d_cu_ctx *c, mb3d_cu_ctx::Scratch &sc, const DevParams &p, bool mixed, int passes,
                         mb3d_cu_silight *dg, cudaStream_t s) {
    int rows = p.height;
    size_t npix = (size_t)rows * p.width;
    CU_TRY(cudaMemsetAsync(sc.counters, 0, 64 * sizeof(unsigned int), s));
    int items = ((p.width + 7) / 8) * ((rows + 3) / 4);
    int blocks = c->sms * (mixed ? p.blocks_march32 : p.blocks_per_sm);
    int need = (items + 7) / 8;
    if (blocks > need) blocks = need > 0 ? need : 1;
    launch_march(p, mixed, 0, rows, dg, sc.hand, sc.counters, nullptr, blocks, s);
    launch_finish(p, mixed, 0, sc.hand, sc.counters, sc.slow, dg, c->sms * p.blocks_per_sm, s);
    if (passes) {
        unsigned int *cnt = sc.counters + 8;
        launch_surface(p, (int)npix, passes, dg, sc.slist, cnt, c->sms * 4, s);
        launch_post_start(p, mixed, 0, passes, dg, sc.slist, cnt, cnt + 3, sc.ps, c->sms * p.blocks_per_sm, s);
        if (passes & MB3D_CU_POST_SHADOW) launch_shadow_rays(p, mixed, 0, sc.ps, cnt, dg, cnt + 1, c->sms * p.blocks_per_sm, s);
        if (passes & MB3D_CU_POST_DEAO) {
            launch_ao_prep(p, sc.ps, dg, cnt, c->sms * 8, s);
            launch_ao_rays(p, mixed, sc.ps, dg, cnt, sc.minra, cnt + 2, c->sms * p.blocks_per_sm, s);
            launch_ao_final(p, sc.ps, cnt, sc.minra, dg, c->sms * 8, s);
        }
    }
    return check_launch("frame launches");
}

static int ensure_frame_resources(mb3d_cu_ctx *c, int streams, size_t npix, size_t nray) {
    while ((int)c->fstreams.size() < streams) {
        cudaStream_t s;
        cudaEvent_t e;
        CU_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->fstreams.push_back(s);
        c->fevents.push_back(e);
        c->fscratch.push_back(mb3d_cu_ctx::Scratch());
    }
    if (c->fevents.size() < (size_t)streams + 1) {
        cudaEvent_t e;
        CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->fevents.push_back(e);
    }
    for (int i = 0; i < streams; i++) {
        auto &sc = c->fscratch[i];
        if (sc.npix < npix || sc.nray < nray) {
            cudaFree(sc.hand); cudaFree(sc.slow); cudaFree(sc.slist); cudaFree(sc.ps); cudaFree(sc.minra); cudaFree(sc.counters);
            sc = mb3d_cu_ctx::Scratch();
            CU_TRY(cudaMalloc(&sc.hand, npix * sizeof(Hand)));
            CU_TRY(cudaMalloc(&sc.slow, npix * sizeof(Hand)));
            CU_TRY(cudaMalloc(&sc.slist, npix * sizeof(uint32_t)));
            CU_TRY(cudaMalloc(&sc.ps, npix * sizeof(PostStart)));
            CU_TRY(cudaMalloc(&sc.minra, (nray + 4) * AO_MINRA_BYTES));
            CU_TRY(cudaMalloc(&sc.counters, 64 * sizeof(unsigned int)));
            sc.npix = npix;
            sc.nray = nray;
        }
    }
    return 0;
}

static int render_frames_locked(mb3d_cu_ctx *c, const mb3d_cu_scene *frames, uint32_t n, int precision,
                                const mb3d_cu_tune *tune, mb3d_cu_silight *out, float *ms_out) {
    if (!frames || n == 0 || !out) return fail(MB3D_CU_EINVAL, "no frames");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    std::vector<DevParams> P(n);
    std::string err;
    for (uint32_t f = 0; f < n; f++) {
        if (frames[f].width != frames[0].width || frames[f].height != frames[0].height)
            return fail(MB3D_CU_EINVAL, "the frames of a batch must have one size");
        int r = setup_params(frames[f], P[f], err);
        if (r < 0) return fail(r, "frame " + std::to_string(f) + ": " + err);
        if (tune) {
            if (tune->blocks_per_sm >= 1 && tune->blocks_per_sm <= 16) P[f].blocks_per_sm = tune->blocks_per_sm;
            if (tune->refill_min >= 1 && tune->refill_min <= 32) P[f].refill_min = tune->refill_min;
        }
    }
    const DevParams &p0 = P[0];
    int streams = tune && tune->streams >= 1 ? (tune->streams > 8 ? 8 : tune->streams) : 2;
    size_t npix = (size_t)p0.width * p0.height;
    int passes = (frames[0].shadow_lights && p0.n_lights > 0 ? MB3D_CU_POST_SHADOW : 0) |
                 (p0.ao_quality >= 0 && p0.ao_rays > 0 ? MB3D_CU_POST_DEAO : 0);
    size_t nray = (passes & MB3D_CU_POST_DEAO) ? npix * (size_t)p0.ao_rays : 0;
    if (int e = ensure_frame_resources(c, streams, npix, nray)) return e;
    bool dev = is_device_ptr(out);
    mb3d_cu_silight *dg = out;
    if (!dev) {
        if (int e = grow((void **)&c->d_frames, &c->frames_cap, (size_t)n * npix * sizeof(mb3d_cu_silight))) return e;
        dg = c->d_frames;
    }
    cudaStream_t s0 = c->stream;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    CU_TRY(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal));
    int rc = 0;
    cudaEvent_t fork = c->fevents[streams];
    if (cudaEventRecord(fork, s0) != cudaSuccess) rc = fail(MB3D_CU_EIO, "capture: fork");
    for (int i = 0; i < streams && !rc; i++)
        if (cudaStreamWaitEvent(c->fstreams[i], fork, 0) != cudaSuccess) rc = fail(MB3D_CU_EIO, "capture: wait");
    for (uint32_t f = 0; f < n && !rc; f++) {
        bool mixed = precision != MB3D_CU_FP64 && !P[f].all_fp64;
        int i = (int)(f % (uint32_t)streams);
        rc = enqueue_frame(c, c->fscratch[i], P[f], mixed, passes, dg + (size_t)f * npix, c->fstreams[i]);
        c->stats.launches += 2 + (passes ? 2 : 0) + ((passes & MB3D_CU_POST_SHADOW) ? 1 : 0) + ((passes & MB3D_CU_POST_DEAO) ? 3 : 0);
    }
    for (int i = 0; i < streams && !rc; i++) {
        if (cudaEventRecord(c->fevents[i], c->fstreams[i]) != cudaSuccess || cudaStreamWaitEvent(s0, c->fevents[i], 0) != cudaSuccess)
            rc = fail(MB3D_CU_EIO, "capture: join");
    }
    cudaError_t ee = cudaStreamEndCapture(s0, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (ee != cudaSuccess) return fail(MB3D_CU_EIO, std::string("capture: ") + cudaGetErrorString(ee));
    ee = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ee != cudaSuccess) return fail(MB3D_CU_EIO, std::string("graph instantiate: ") + cudaGetErrorString(ee));
    cudaEventRecord(c->ev[6], s0);
    ee = cudaGraphLaunch(exec, s0);
    cudaEventRecord(c->ev[7], s0);
    if (ee == cudaSuccess) ee = cudaStreamSynchronize(s0);
    cudaGraphExecDestroy(exec);
    if (ee != cudaSuccess) return fail(MB3D_CU_EIO, std::string("frames: ") + cudaGetErrorString(ee));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
    c->stats.ms_total = ms;
    if (ms_out) *ms_out = ms;
    if (!dev) CU_TRY(cudaMemcpy(out, dg, (size_t)n * npix * sizeof(mb3d_cu_silight), cudaMemcpyDeviceToHost));
    return 0;
}

int mb3d_cu_render_frames(mb3d_cu_ctx *c, const mb3d_cu_scene *frames, uint32_t n, int precision,
                          const mb3d_cu_tune *tune, mb3d_cu_silight *out) {
    if (!c) return fail(MB3D_CU_EINVAL, "ctx is NULL");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    std::memset(&c->stats, 0, sizeof(c->stats));
    return render_frames_locked(c, frames, n, precision, tune, out, nullptr);
}

int mb3d_cu_autotune(mb3d_cu_ctx *c, const mb3d_cu_scene *frames, uint32_t n, uint32_t sample, int precision,
                     mb3d_cu_tune *out) {
    if (!c || !frames || n == 0 || !out) return fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    if (sample == 0 || sample > n) sample = n < 8 ? n : 8;
    std::vector<mb3d_cu_scene> pick;
    for (uint32_t k = 0; k < sample; k++) pick.push_back(frames[(size_t)k * n / sample]);
    size_t npix = (size_t)frames[0].width * frames[0].height;
    mb3d_cu_silight *buf = nullptr;
    if (int e = grow((void **)&c->d_frames, &c->frames_cap, pick.size() * npix * sizeof(mb3d_cu_silight))) return e;
    buf = c->d_frames;
    const int blocks[3] = {2, 3, 4}, refills[3] = {16, 24, 32}, streams[3] = {1, 2, 4};
    float best = 1e30f;
    mb3d_cu_tune bt = {3, 32, 2, 0};
    for (int b : blocks)
        for (int r : refills)
            for (int s : streams) {
                mb3d_cu_tune t = {b, r, s, 0};
                float ms = 0.f;
                if (int e = render_frames_locked(c, pick.data(), (uint32_t)pick.size(), precision, &t, buf, &ms)) return e;
                if (int e = render_frames_locked(c, pick.data(), (uint32_t)pick.size(), precision, &t, buf, &ms)) return e;
                if (ms < best) {
                    best = ms;
                    bt = t;
                }
            }
    *out = bt;
    c->stats.ms_total = best;
    return 0;
}

int mb3d_cu_set_counting(mb3d_cu_ctx *c, int on) {
    if (!c) return fail(MB3D_CU_EINVAL, "ctx is NULL");
    c->counting = on != 0;
    return 0;
}

int mb3d_cu_fma_peak(mb3d_cu_ctx *c, int fp64, double *tflops) {
    if (!c || !tflops) return fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    if (int e = grow((void **)&c->d_probe, &c->probe_cap, 64)) return e;
    int blocks = c->sms * 8, iters = fp64 ? 512 : 2048;
    launch_fma_peak(fp64 != 0, c->d_probe, blocks, iters, c->stream);  // warm-up
    if (int r = check_launch("k_fma_peak")) return r;
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        CU_TRY(cudaEventRecord(c->ev[6], c->stream));
        launch_fma_peak(fp64 != 0, c->d_probe, blocks, iters, c->stream);
        CU_TRY(cudaEventRecord(c->ev[7], c->stream));
        CU_TRY(cudaEventSynchronize(c->ev[7]));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev[6], c->ev[7]);
        if (ms < best) best = ms;
    }
    double flops = 2.0 * 8.0 * 16.0 * (double)iters * (double)blocks * 256.0;
    *tflops = flops / ((double)best * 1e-3) / 1e12;
    return 0;
}

// ---------------------------------------------------------------------------
// the Monte Carlo tracer

int mb3d_cu_mc_light_default(const mb3d_cu_scene *sc, mb3d_cu_mc_light *out) {
    if (!sc || !out) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (sc->width <= 0 || sc->height <= 0 || !(sc->zoom > 0.0)) return fail(MB3D_CU_EINVAL, "bad picture size or zoom");
    return mc_light_default(*sc, *out);
}

void mb3d_cu_mc_paint_default(mb3d_cu_mc_paint_opts *o) {
    if (!o) return;
    o->contrast = 128;
    o->saturation = 32;
    o->options = 2;
    o->pad = 0;
    o->gamma = 32.0f;
}

int mb3d_cu_mc_paint(mb3d_cu_ctx *c, const float *col, const uint8_t *rays, uint32_t npix, const mb3d_cu_mc_paint_opts *o,
                     uint8_t *rgb) {
    if (!c || !col || !o || !rgb) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (npix == 0) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = c->stream;
    const bool dc = is_device_ptr(col), dr = !rays || is_device_ptr(rays), dg = is_device_ptr(rgb);
    const size_t bc = (size_t)npix * 12, br = npix, bg = (size_t)npix * 3;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    size_t need = (dc ? 0 : up16(bc)) + (dr ? 0 : up16(br)) + (dg ? 0 : up16(bg));
    if (need)
        if (int r = grow((void **)&c->d_paint, &c->paint_cap, need)) return r;
    unsigned char *q = c->d_paint;
    const float *dcol = col;
    const uint8_t *drays = rays;
    uint8_t *drgb = rgb;
    if (!dc) {
        CU_TRY(cudaMemcpyAsync(q, col, bc, cudaMemcpyHostToDevice, s));
        dcol = (const float *)q;
        q += up16(bc);
    }
    if (!dr) {
        CU_TRY(cudaMemcpyAsync(q, rays, br, cudaMemcpyHostToDevice, s));
        drays = q;
        q += up16(br);
    }
    if (!dg) drgb = q;
    int blocks = (int)std::min<size_t>(((size_t)npix + 255) / 256, (size_t)c->sms * 8);
    mc_paint_launch(dcol, drays, npix, *o, drgb, blocks, s);
    if (int r = check_launch("k_mc_paint")) return r;
    if (!dg) CU_TRY(cudaMemcpyAsync(rgb, drgb, bg, cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    return 0;
}

int mb3d_cu_paint(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_silight *gbuf, uint32_t row0, uint32_t rows,
                  uint8_t *rgb) {
    if (!c || !sc || !gbuf || !rgb) return fail(MB3D_CU_EINVAL, "NULL argument");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    if ((uint64_t)row0 + rows > (uint64_t)p.height || rows == 0) return fail(MB3D_CU_EINVAL, "rows outside the picture");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = c->stream;
    const uint32_t npix = rows * (uint32_t)p.width;
    const bool dg = is_device_ptr(gbuf), dr = is_device_ptr(rgb);
    const size_t bg = (size_t)npix * sizeof(mb3d_cu_silight), br = (size_t)npix * 3;
    auto up16 = [](size_t b) { return (b + 15) & ~(size_t)15; };
    size_t need = (dg ? 0 : up16(bg)) + (dr ? 0 : up16(br));
    if (need)
        if (int e = grow((void **)&c->d_paint, &c->paint_cap, need)) return e;
    unsigned char *q = c->d_paint;
    const mb3d_cu_silight *dgb = gbuf;
    uint8_t *drgb = rgb;
    if (!dg) {
        CU_TRY(cudaMemcpyAsync(q, gbuf, bg, cudaMemcpyHostToDevice, s));
        dgb = (const mb3d_cu_silight *)q;
        q += up16(bg);
    }
    if (!dr) drgb = q;
    int blocks = (int)std::min<size_t>(((size_t)npix + 255) / 256, (size_t)c->sms * 8);
    paint_launch(*sc, p, row0, dgb, npix, drgb, blocks, s);
    if (int e = check_launch("k_paint")) return e;
    if (!dr) CU_TRY(cudaMemcpyAsync(rgb, drgb, br, cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    return 0;
}

void mb3d_cu_ssao_default(mb3d_cu_ssao_opts *o) {
    if (!o) return;
    o->threshold = 2.0f;
    o->border_mirror = 0.0f;
    o->t0 = 0;
    o->wrap_x = 0;
    o->random = 0;
    o->pad = 0;
}

int mb3d_cu_ssao24(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_ssao_opts *o, mb3d_cu_silight *gbuf) {
    if (!c || !sc || !o || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (!(o->border_mirror >= 0.0f && o->border_mirror <= 0.9f) || !(o->threshold == o->threshold))
        return fail(MB3D_CU_EINVAL, "border_mirror outside 0..0.9 or threshold not a number");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    const int w = p.width, h = p.height;
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = c->stream;
    const size_t npix = (size_t)w * h, gb = npix * sizeof(mb3d_cu_silight);
    const bool dev = is_device_ptr(gbuf);
    const size_t scratch = (ssao_scratch_bytes(w, h, o->random) + 255) & ~(size_t)255;
    if (int e = grow((void **)&c->d_ssao, &c->ssao_cap, scratch + (dev ? 0 : gb))) return e;
    mb3d_cu_silight *dg = dev ? gbuf : reinterpret_cast<mb3d_cu_silight *>(c->d_ssao + scratch);
    if (!dev) CU_TRY(cudaMemcpyAsync(dg, gbuf, gb, cudaMemcpyHostToDevice, s));
    std::memset(&c->stats, 0, sizeof(c->stats));
    CU_TRY(cudaEventRecord(c->ev[0], s));
    ssao24_launch(dg, w, h, p.zc_mul, p.zcorr, *o, c->d_ssao, c->sms, s);
    if (int e = check_launch("k_ssao")) return e;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dev) CU_TRY(cudaMemcpyAsync(gbuf, dg, gb, cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    return 0;
}

int mb3d_cu_ssao15(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_ssao_opts *o, mb3d_cu_silight *gbuf) {
    if (!c || !sc || !o || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (!(o->threshold == o->threshold)) return fail(MB3D_CU_EINVAL, "threshold not a number");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    const int w = p.width, h = p.height;
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = c->stream;
    const size_t npix = (size_t)w * h, gb = npix * sizeof(mb3d_cu_silight);
    const bool dev = is_device_ptr(gbuf);
    const size_t scratch = (ssao15_scratch_bytes(w, h) + 255) & ~(size_t)255;
    if (int e = grow((void **)&c->d_ssao, &c->ssao_cap, scratch + (dev ? 0 : gb))) return e;
    mb3d_cu_silight *dg = dev ? gbuf : reinterpret_cast<mb3d_cu_silight *>(c->d_ssao + scratch);
    if (!dev) CU_TRY(cudaMemcpyAsync(dg, gbuf, gb, cudaMemcpyHostToDevice, s));
    std::memset(&c->stats, 0, sizeof(c->stats));
    CU_TRY(cudaEventRecord(c->ev[0], s));
    uint32_t launches = 0;
    const int rr = ssao15_run(dg, w, h, p.zc_mul, p.zcorr, *o, c->d_ssao, c->sms, s, &launches);
    if (rr == -2) return fail(MB3D_CU_EIO, "ssao15: a ring's samples beyond the table");
    if (int e = check_launch("k15_sample")) return e;
    if (rr != 0) return fail(MB3D_CU_EIO, "ssao15: a CUDA call failed");
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dev) CU_TRY(cudaMemcpyAsync(gbuf, dg, gb, cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.launches = launches;
    return 0;
}

static int mc_halton(mb3d_cu_ctx *c) {
    if (c->d_halton) return 0;
    const std::vector<uint32_t> &t = mc_halton_table();
    CU_TRY(cudaMalloc(&c->d_halton, t.size() * sizeof(uint32_t)));
    CU_TRY(cudaMemcpy(c->d_halton, t.data(), t.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    return 0;
}

static size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

int mb3d_cu_mc_batch(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, int secant, const mb3d_cu_mc_req *reqs,
                     uint32_t n, mb3d_cu_mc_res *res) {
    if (!c || !sc || (n && (!reqs || !res))) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    if (n == 0) return 0;
    bool dreq = is_device_ptr(reqs), dres = is_device_ptr(res);
    if (!dreq)
        for (uint32_t i = 0; i < n; i++) {
            if (reqs[i].kind > 1) return fail(MB3D_CU_ENOTSUP, "march kind 2 (through transparent objects) is not on the card");
            if (reqs[i].inside) return fail(MB3D_CU_ENOTSUP, "inside rendering is not on the card");
        }
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    McDev m;
    mb3d_cu_mc_light lv;
    std::memset(&lv, 0, sizeof(lv));
    std::string err;
    int r = mc_setup(*sc, lv, 0, secant, 1.0f, p, m, err);
    if (r < 0) return fail(r, err);
    apply_tuning(p);
    std::memset(&c->stats, 0, sizeof(c->stats));
    size_t oreq = 256, ores = oreq + align256((size_t)n * sizeof(mb3d_cu_mc_req));
    size_t need = ores + align256((size_t)n * sizeof(mb3d_cu_mc_res));
    if (int e = grow((void **)&c->d_mc, &c->mc_cap, need)) return e;
    unsigned long long *cnt = (unsigned long long *)c->d_mc;
    const mb3d_cu_mc_req *dq = reqs;
    mb3d_cu_mc_res *dr = dres ? res : (mb3d_cu_mc_res *)(c->d_mc + ores);
    cudaStream_t s = c->stream;
    CU_TRY(cudaEventRecord(c->ev[0], s));
    if (!dreq) {
        CU_TRY(cudaMemcpyAsync(c->d_mc + oreq, reqs, (size_t)n * sizeof(mb3d_cu_mc_req), cudaMemcpyHostToDevice, s));
        dq = (const mb3d_cu_mc_req *)(c->d_mc + oreq);
    }
    CU_TRY(cudaMemsetAsync(c->d_mc, 0, 256, s));
    McAcc acc;
    std::memset(&acc, 0, sizeof(acc));
    acc.counters = cnt;
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    launch_mc(p, m, mixed, true, acc, dq, dr, (unsigned int *)(cnt + 8), n, nullptr, c->sms, s);
    c->stats.launches = 1;
    if (int e = check_launch("k_mc (batch)")) return e;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dres) CU_TRY(cudaMemcpyAsync(res, dr, (size_t)n * sizeof(mb3d_cu_mc_res), cudaMemcpyDeviceToHost, s));
    unsigned long long h[4];
    CU_TRY(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.ms_march = ms;
    c->stats.de_evals = h[0];
    c->stats.mc_fp64_rays = (uint32_t)h[3];
    return 0;
}

// the split render of n_items items: the paths' logic (k_mc_logic) and their
// marches (k_mc in batch mode on the list of waiting paths) in turns; ctrl:
// 3 words of device scratch (next item, list length, march queue)
static int mc_split(mb3d_cu_ctx *c, const DevParams &p, const McDev &mb, const McAcc &ab, uint32_t n_items, bool mixed,
                    unsigned int *ctrl, const volatile int *cancel, uint32_t &launches) {
    cudaStream_t s = c->stream;
    const uint32_t slots = std::min<uint32_t>(n_items, 1u << 21);
    const size_t lb = mc_lane_bytes();
    size_t s_req = align256((size_t)slots * lb), s_res = s_req + align256((size_t)slots * sizeof(mb3d_cu_mc_req));
    size_t s_list = s_res + align256((size_t)slots * sizeof(mb3d_cu_mc_res));
    size_t s_need = s_list + align256((size_t)slots * 4);
    if (int e = grow((void **)&c->d_mcs, &c->mcs_cap, s_need)) return e;
    unsigned char *S = c->d_mcs;
    mb3d_cu_mc_req *reqs = (mb3d_cu_mc_req *)(S + s_req);
    mb3d_cu_mc_res *res = (mb3d_cu_mc_res *)(S + s_res);
    uint32_t *list = (uint32_t *)(S + s_list);
    CU_TRY(cudaMemsetAsync(S, 0, (size_t)slots * lb, s));  // (every path idle)
    CU_TRY(cudaMemsetAsync(ctrl, 0, 12, s));
    for (int turn = 0;; turn++) {
        if (turn > 4000000) return fail(MB3D_CU_EIO, "Monte Carlo turns did not end");
        CU_TRY(cudaMemsetAsync(ctrl + 1, 0, 8, s));
        launch_mc_logic(p, mb, ab, S, reqs, res, slots, ctrl, n_items, list, ctrl + 1, c->sms, s);
        if (int e = check_launch("k_mc_logic")) return e;
        unsigned int h[2];
        CU_TRY(cudaMemcpyAsync(h, ctrl, 8, cudaMemcpyDeviceToHost, s));
        CU_TRY(cudaStreamSynchronize(s));
        launches++;
        if (h[1] == 0) {
            if (h[0] >= n_items) break;
            continue;  // (only padding items were taken this turn)
        }
        launch_mc(p, mb, mixed, true, ab, reqs, res, ctrl + 2, h[1], list, c->sms, s);
        launches++;
        if (int e = check_launch("k_mc (split)")) return e;
        if (cancel && (turn & 15) == 15 && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    }
    return 0;
}

// ---------------------------------------------------------------------------
// depth of field (dof.cu)

void mb3d_cu_dof_default(mb3d_cu_dof_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->z_sharp = 1.0f;
    o->z_sharp2 = 1.0f;
    o->aperture = 0.1f;
    o->clip_r = 30.0f;
    o->passes = 1;
    o->forward = 0;
}

static inline float clampf_(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

static float zsteps_h(double z, double zc_mul_inv, double zcorr_inv) {
    const double a = z * zc_mul_inv + 1.0;
    return (float)((a * a - 1.0) * zcorr_inv);
}

// focus (src/dof.rs:49-78) in the reference's single precision order
static void dof_focus(const mb3d_cu_dof_opts &p, uint32_t pass, bool sorted, int width, int height, double fov_y_deg,
                      DofPass &d) {
    const float ap0 = clampf_(p.aperture, 0.0001f, 2.0f);
    const int lp = (int)(p.passes < 1 ? 1 : p.passes > 4 ? 4 : p.passes) - 1;
    volatile float ap;
    if (lp == 0) {
        ap = ap0 * 0.5f;
    } else if (lp == 1) {
        ap = sorted ? ap0 * (0.25f + (float)pass * 0.58f) * 0.5f : ap0 * (0.3f + (float)pass * 0.55f) * 0.5f;
    } else {
        float p3 = 1.0f;
        for (uint32_t k = 0; k < pass; k++) p3 *= 3.0f;
        ap = sorted ? ap0 / 22.0f * p3 : ap0 / 12.0f * (float)(1u << pass);
    }
    const float dsf = (float)(std::fmax(fov_y_deg * (3.14159265358979323846 / 180.0), 0.0) / (double)height);
    const float dw = std::fmin(p.z_sharp, p.z_sharp2) * (float)width;
    const float st = std::fmax(p.z_sharp, p.z_sharp2) * (float)width;
    const float w = (1.0f + dw * dsf) / (1.0f + st * dsf);
    const float z_sharp = (w * st + dw) / (1.0f + w);
    d.ap = ap;
    d.dsf = dsf;
    d.z_sharp = z_sharp;
    d.r_sub = std::fabs((dw - z_sharp) / (1.0f + dw * dsf) * ap);
}

int mb3d_cu_dof(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_dof_opts *o, const mb3d_cu_silight *gbuf,
                uint8_t *rgb) {
    if (!c || !sc || !o || !gbuf || !rgb) return fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    const int w = p.width, h = p.height;
    const size_t n = (size_t)w * h;
    const bool dg = is_device_ptr(gbuf), dr = is_device_ptr(rgb);
    size_t o_misc = 0, o_g = 256, o_a = o_g + align256(n * sizeof(mb3d_cu_silight)), o_b = o_a + align256(n * 3);
    size_t o_src = o_b + align256(n * 3), o_key = o_src + align256(n * sizeof(DofSrc)), need = o_key + align256(n * 8);
    if (int e = grow((void **)&c->d_dof, &c->dof_cap, need)) return e;
    unsigned char *B = c->d_dof;
    unsigned int *misc = (unsigned int *)(B + o_misc);  // [0,1] z range, [2] largest radius bits, [3] overflow
    const mb3d_cu_silight *g = dg ? gbuf : (const mb3d_cu_silight *)(B + o_g);
    uint8_t *pa = (uint8_t *)(B + o_a), *pb = (uint8_t *)(B + o_b);
    DofSrc *src = (DofSrc *)(B + o_src);
    unsigned long long *key = (unsigned long long *)(B + o_key);
    cudaStream_t s = c->stream;
    std::memset(&c->stats, 0, sizeof(c->stats));
    CU_TRY(cudaEventRecord(c->ev[0], s));
    if (!dg) CU_TRY(cudaMemcpyAsync((void *)g, gbuf, n * sizeof(mb3d_cu_silight), cudaMemcpyHostToDevice, s));
    CU_TRY(cudaMemcpyAsync(pa, rgb, n * 3, dr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    const double zc_mul_inv = 1.0 / p.zc_mul, zcorr_inv = 1.0 / p.zcorr;
    const uint32_t passes = o->passes < 1 ? 1 : o->passes > 4 ? 4 : o->passes;
    const bool forward = o->forward != 0;
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device);
    // (the list's room in shared memory: a power of two, as the sort pads to one)
    int cap_max = 1024;
    while (cap_max * 2 * 8 + 1024 <= max_smem) cap_max *= 2;
    uint32_t launches = 0;
    for (uint32_t pass = 0; pass < passes; pass++) {
        DofPass d;
        std::memset(&d, 0, sizeof(d));
        d.w = w;
        d.h = h;
        d.forward = forward ? 1 : 0;
        d.zc_mul_inv = zc_mul_inv;
        d.zcorr_inv = zcorr_inv;
        dof_focus(*o, pass, !forward, w, h, sc->fov_y, d);
        d.clip_r = clampf_(o->clip_r, 0.1f, 1000.0f);
        CU_TRY(cudaMemsetAsync(misc, 0, 16, s));
        unsigned int hm[4] = {32768u, 0u, 0u, 0u};
        if (!forward) {
            // the nearest and farthest object depths (src/dof.rs:274-287)
            CU_TRY(cudaMemcpyAsync(misc, hm, 8, cudaMemcpyHostToDevice, s));
            dof_zrange(g, n, misc, c->sms, s);
            CU_TRY(cudaMemcpyAsync(hm, misc, 8, cudaMemcpyDeviceToHost, s));
            CU_TRY(cudaStreamSynchronize(s));
            const int64_t zmin = hm[0], zmax = hm[1];
            float zw = zsteps_h((double)((32768 - zmin) * 256), zc_mul_inv, zcorr_inv);
            const float r0 = std::fabs((zw - d.z_sharp) * d.ap / (1.0f + zw * d.dsf));
            zw = zsteps_h((double)((32768 - zmax) * 256), zc_mul_inv, zcorr_inv);
            d.max_r = std::fmin(d.clip_r, std::fmax(r0, std::fabs((zw - d.z_sharp) / (1.0f + zw * d.dsf) * d.ap)) * 1.5f);
            d.rmax = (int)std::nearbyint(std::fabs(d.max_r) + 0.5f);
        } else {
            d.bg = zsteps_h(8388353.0, zc_mul_inv, zcorr_inv);
        }
        dof_src(d, g, pa, src, key, misc + 2, c->sms, s);
        launches++;
        if (int e = check_launch("k_dof_src")) return e;
        if (forward) {
            unsigned int bits = 0;
            CU_TRY(cudaMemcpyAsync(&bits, misc + 2, 4, cudaMemcpyDeviceToHost, s));
            CU_TRY(cudaStreamSynchronize(s));
            float mr;
            std::memcpy(&mr, &bits, 4);
            // (every radius is clamped to clip_r <= 1000: a larger value is a fault of the reduction)
            if (!(mr >= 0.0f && mr <= d.clip_r)) return fail(MB3D_CU_EIO, "depth of field: largest radius out of range");
            d.max_r = mr;
            d.sm = 1.0f / (1.0f + mr);
            d.rmax = (int)std::nearbyint(mr + 0.5f);
        }
        const int64_t win = 16 + 2 * (int64_t)d.rmax;
        int cap = 1024;
        while (cap < cap_max && (int64_t)cap < win * win) cap *= 2;
        if (dof_tiles(d, src, key, pb, cap, misc + 3, s) != 0) return fail(MB3D_CU_EIO, "k_dof_tiles: shared memory");
        launches++;
        if (int e = check_launch("k_dof_tiles")) return e;
        std::swap(pa, pb);
    }
    unsigned int ovf = 0;
    CU_TRY(cudaMemcpyAsync(&ovf, misc + 3, 4, cudaMemcpyDeviceToHost, s));
    CU_TRY(cudaEventRecord(c->ev[1], s));
    CU_TRY(cudaStreamSynchronize(s));
    if (ovf)
        return fail(MB3D_CU_ENOTSUP, "depth of field: the blur radius is beyond the card's tile lists (the CPU does it)");
    CU_TRY(cudaMemcpyAsync(rgb, pa, n * 3, dr ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.launches = launches;
    return 0;
}


int mb3d_cu_reflect_batch(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_reflect_ray *rays, uint32_t n,
                          int far_fog, mb3d_cu_reflect_hit *hits) {
    if (!c || !sc || (n && (!rays || !hits))) return fail(MB3D_CU_EINVAL, "NULL argument");
    std::string why;
    int u = unsupported_reason(*sc, why);
    if (u < 0) return fail(u, why);
    if (u == 1) return fail(MB3D_CU_ENOTSUP, why);
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    if (n == 0) return 0;
    if (n > (1u << 26)) return fail(MB3D_CU_EINVAL, "more than 2^26 rays in one batch");
    const bool dr = is_device_ptr(rays), dh = is_device_ptr(hits);
    if (!dr) {
        const uint32_t np = (uint32_t)p.width * (uint32_t)p.height;
        for (uint32_t i = 0; i < n; i++)
            if (rays[i].pixel >= np) return fail(MB3D_CU_EINVAL, "a ray's pixel is outside the picture");
    }
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    const size_t br = (size_t)n * sizeof(mb3d_cu_reflect_ray), bh = (size_t)n * sizeof(mb3d_cu_reflect_hit);
    const size_t o_tab = 0, o_r = align256(sizeof(ReflAO)), o_h = o_r + (dr ? 0 : align256(br));
    const size_t need = o_h + (dh ? 0 : align256(bh));
    if (int e = grow((void **)&c->d_refl, &c->refl_cap, need)) return e;
    static ReflAO tab;  // (the same for every call; made once)
    static std::once_flag tab_once;
    std::call_once(tab_once, [] { reflect_ao_table(tab); });
    cudaStream_t s = c->stream;
    ReflAO *dtab = reinterpret_cast<ReflAO *>(c->d_refl + o_tab);
    const mb3d_cu_reflect_ray *drays = dr ? rays : reinterpret_cast<const mb3d_cu_reflect_ray *>(c->d_refl + o_r);
    mb3d_cu_reflect_hit *dhits = dh ? hits : reinterpret_cast<mb3d_cu_reflect_hit *>(c->d_refl + o_h);
    std::memset(&c->stats, 0, sizeof(c->stats));
    CU_TRY(cudaMemcpyAsync(dtab, &tab, sizeof(ReflAO), cudaMemcpyHostToDevice, s));
    if (!dr) CU_TRY(cudaMemcpyAsync((void *)drays, rays, br, cudaMemcpyHostToDevice, s));
    CU_TRY(cudaEventRecord(c->ev[0], s));
    const int blocks = (int)std::min<size_t>(((size_t)n + 127) / 128, (size_t)c->sms * 16);
    launch_reflect(p, drays, n, far_fog ? 1 : 0, dtab, dhits, blocks, s);
    if (int e = check_launch("k_reflect")) return e;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dh) CU_TRY(cudaMemcpyAsync(hits, dhits, bh, cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.launches = 1;
    return 0;
}

int mb3d_cu_reflect_first_rays(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_silight *gbuf,
                               mb3d_cu_reflect_ray *rays, uint32_t *n_rays) {
    if (!c || !sc || !gbuf || !rays || !n_rays) return fail(MB3D_CU_EINVAL, "NULL argument");
    *n_rays = 0;
    std::string why;
    int u = unsupported_reason(*sc, why);
    if (u < 0) return fail(u, why);
    if (u == 1) return fail(MB3D_CU_ENOTSUP, why);
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
    const size_t npix = (size_t)p.width * p.height;
    const size_t nblk = (npix + 1023) / 1024;
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    const bool dg = is_device_ptr(gbuf), dr = is_device_ptr(rays);
    const size_t bg = npix * sizeof(mb3d_cu_silight), br = npix * sizeof(mb3d_cu_reflect_ray);
    const size_t o_tmp = 0, o_valid = o_tmp + align256(br), o_sum = o_valid + align256(npix),
                 o_g = o_sum + align256(nblk * 4), o_out = o_g + (dg ? 0 : align256(bg));
    const size_t need = o_out + (dr ? 0 : align256(br));
    if (int e = grow((void **)&c->d_refl, &c->refl_cap, need)) return e;
    unsigned char *B = c->d_refl;
    mb3d_cu_reflect_ray *tmp = reinterpret_cast<mb3d_cu_reflect_ray *>(B + o_tmp);
    unsigned char *valid = B + o_valid;
    unsigned int *sums = reinterpret_cast<unsigned int *>(B + o_sum);
    const mb3d_cu_silight *g = dg ? gbuf : reinterpret_cast<const mb3d_cu_silight *>(B + o_g);
    mb3d_cu_reflect_ray *out = dr ? rays : reinterpret_cast<mb3d_cu_reflect_ray *>(B + o_out);
    cudaStream_t s = c->stream;
    std::memset(&c->stats, 0, sizeof(c->stats));
    if (!dg) CU_TRY(cudaMemcpyAsync((void *)g, gbuf, bg, cudaMemcpyHostToDevice, s));
    CU_TRY(cudaEventRecord(c->ev[0], s));
    const int blocks = (int)std::min<size_t>((npix + 127) / 128, (size_t)c->sms * 16);
    launch_reflect_first(p, g, tmp, valid, blocks, s);
    if (int e = check_launch("k_reflect_first")) return e;
    flag_count(valid, npix, sums, s);
    std::vector<unsigned int> h(nblk);
    CU_TRY(cudaMemcpyAsync(h.data(), sums, nblk * 4, cudaMemcpyDeviceToHost, s));
    CU_TRY(cudaStreamSynchronize(s));
    unsigned int total = 0;
    for (size_t b = 0; b < nblk; b++) {
        const unsigned int v = h[b];
        h[b] = total;
        total += v;
    }
    CU_TRY(cudaMemcpyAsync(sums, h.data(), nblk * 4, cudaMemcpyHostToDevice, s));
    flag_scatter(valid, tmp, npix, sums, out, s);
    if (int e = check_launch("k_flag_scatter")) return e;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dr && total) CU_TRY(cudaMemcpyAsync(rays, out, (size_t)total * sizeof(mb3d_cu_reflect_ray), cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.launches = 3;
    *n_rays = total;
    return 0;
}

int mb3d_cu_mc_pass(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_mc_light *lv, const mb3d_cu_mc_opts *o,
                    int precision, uint32_t pass_nr, mb3d_cu_mc_record *recs, const volatile int *cancel) {
    if (!c || !sc || !lv || !o || !recs) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    if (o->depth < 0 || o->depth > 64) return fail(MB3D_CU_EINVAL, "depth must be 0..64");
    if (sc->width < 1 || sc->height < 1) return fail(MB3D_CU_EINVAL, "empty picture");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    McDev m;
    std::string err;
    int r = mc_setup(*sc, *lv, o->depth, o->secant, o->soft_shadow_radius, p, m, err);
    if (r < 0) return fail(r, err);
    apply_tuning(p);
    if (int e = mc_halton(c)) return e;
    if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    std::memset(&c->stats, 0, sizeof(c->stats));
    const int w = sc->width, h = sc->height;
    const size_t npix = (size_t)w * (size_t)h;
    cudaStream_t s = c->stream;
    // StartCalc / CalcAvrgNoise (src/mc.rs:3226-3235; McImage::stats and
    // avg_sqr_noise :329-358) on the host's copy of the records
    const bool dev = is_device_ptr(recs);
    std::vector<mb3d_cu_mc_record> hrec;
    const mb3d_cu_mc_record *hr = recs;
    if (dev) {
        hrec.resize(npix);
        CU_TRY(cudaMemcpyAsync(hrec.data(), recs, npix * sizeof(mb3d_cu_mc_record), cudaMemcpyDeviceToHost, s));
        CU_TRY(cudaStreamSynchronize(s));
        hr = hrec.data();
    }
    bool fresh = true, zero_counts = false;
    double rsum = 0.0, noise_sum = 0.0;
    for (size_t i = 0; i < npix; i++) {
        const mb3d_cu_mc_record &q = hr[i];
        if (q.ray_count == 0) {
            zero_counts = true;
            continue;
        }
        fresh = false;
        rsum += (double)q.ray_count;
        const double y = (double)q.ysum;
        noise_sum += std::fmax(((double)q.ysqr - y * y) / (double)q.ray_count, 0.0);
    }
    const double l = (double)npix;
    const double avrg_sqr_noise = fresh ? 1.0 : std::fmax(noise_sum / l + 0.002, 0.002);
    McPassArgs a;
    a.w = w;
    a.h = h;
    a.avrg_rcount = fresh ? 0.0f : (float)(rsum / l);
    a.avrg_vari = std::fmax(avrg_sqr_noise, 0.001);
    {
        const volatile float ar = a.avrg_rcount;  // (single precision, as the reference forms it)
        const volatile float mv = (ar + ar * ar * 0.2f) * 10.0f;
        a.max_new = (int)std::round((float)mv);
    }
    a.skip_nonzero = fresh ? 1 : (zero_counts ? 1 : 0);
    a.sqr = lv->sqr != 0;
    a.pass_nr = pass_nr;
    // device memory: the records (a host array's copy), their snapshot, the
    // rays per pixel, the round's sums, the blocks' ray counts and the items
    const int nblk = (int)((npix + 1023) / 1024);
    size_t o_cnt = 0, o_rec = 256, o_snap = o_rec + align256(npix * sizeof(mb3d_cu_mc_record));
    size_t o_tot = o_snap + align256(npix * sizeof(mb3d_cu_mc_record)), o_sum = o_tot + align256(npix * 4);
    size_t o_ys = o_sum + align256(npix * 24), o_hit = o_ys + align256(npix * 16), o_bs = o_hit + align256(npix * 4);
    size_t o_off = o_bs + align256((size_t)nblk * 4), o_fill = o_off + align256((size_t)nblk * 4);
    size_t need = o_fill + align256((size_t)nblk * 4);
    if (int e = grow((void **)&c->d_mc, &c->mc_cap, need)) return e;
    unsigned char *B = c->d_mc;
    mb3d_cu_mc_record *drec = dev ? recs : (mb3d_cu_mc_record *)(B + o_rec);
    a.recs = drec;
    a.snap = (const mb3d_cu_mc_record *)(B + o_snap);
    a.total = (int *)(B + o_tot);
    McAcc acc;
    acc.counters = (unsigned long long *)(B + o_cnt);
    acc.sum = (unsigned long long *)(B + o_sum);
    acc.ysum = (unsigned long long *)(B + o_ys);
    acc.hit = (unsigned int *)(B + o_hit);
    acc.albedo = acc.normal = acc.depth = nullptr;
    unsigned int *bsum = (unsigned int *)(B + o_bs), *boff = (unsigned int *)(B + o_off), *bfill = (unsigned int *)(B + o_fill);
    unsigned int *more = (unsigned int *)(B + 64), *ctrl = (unsigned int *)(B + 128);
    CU_TRY(cudaEventRecord(c->ev[0], s));
    CU_TRY(cudaMemsetAsync(B, 0, 256, s));
    if (!dev) CU_TRY(cudaMemcpyAsync(drec, recs, npix * sizeof(mb3d_cu_mc_record), cudaMemcpyHostToDevice, s));
    CU_TRY(cudaMemcpyAsync((void *)a.snap, drec, npix * sizeof(mb3d_cu_mc_record), cudaMemcpyDeviceToDevice, s));
    launch_mcp_start(a, c->sms, s);
    if (int e = check_launch("k_mcp_start")) return e;
    const bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    m.x0 = 0;
    m.y0 = 0;
    m.w = w;
    m.h = h;
    m.rays = 1;
    m.ray0 = 0;
    m.tiles_x = (uint32_t)((w + 7) / 8);
    m.npad = m.tiles_x * (uint32_t)((h + 3) / 4) * 32u;
    m.halton = c->d_halton;
    uint32_t launches = 1;
    std::vector<unsigned int> hb(nblk), ho(nblk);
    uint64_t rays_total = 0;
    for (int round = 0;; round++) {
        if (round > 100000) return fail(MB3D_CU_EIO, "Monte Carlo rounds did not end");
        launch_mcp_count(a, bsum, s);
        CU_TRY(cudaMemcpyAsync(hb.data(), bsum, (size_t)nblk * 4, cudaMemcpyDeviceToHost, s));
        CU_TRY(cudaStreamSynchronize(s));
        uint64_t all = 0, most = 0;
        for (int b = 0; b < nblk; b++) {
            all += hb[b];
            most = std::max<uint64_t>(most, hb[b]);
        }
        if (all == 0) break;
        rays_total += all;
        // the blocks in chunks of at most `cap` items (a block's rays stay together)
        const uint64_t cap = std::max<uint64_t>((uint64_t)1 << 25, most);
        size_t items_need = (size_t)std::min<uint64_t>(all, cap) * sizeof(uint2);
        if (int e = grow((void **)&c->d_mcitems, &c->mcitems_cap, items_need)) return e;
        for (int b0 = 0; b0 < nblk;) {
            uint64_t n = 0;
            int b1 = b0;
            while (b1 < nblk && n + hb[b1] <= cap) {
                ho[b1 - b0] = (unsigned int)n;
                n += hb[b1];
                b1++;
            }
            if (n > 0) {
                CU_TRY(cudaMemcpyAsync(boff, ho.data(), (size_t)(b1 - b0) * 4, cudaMemcpyHostToDevice, s));
                CU_TRY(cudaMemsetAsync(bfill, 0, (size_t)(b1 - b0) * 4, s));
                launch_mcp_items(a, b0, b1, boff, bfill, (uint2 *)c->d_mcitems, acc, s);
                if (int e = check_launch("k_mcp_items")) return e;
                McDev mi = m;
                mi.items = (const uint2 *)c->d_mcitems;
                if (int e = mc_split(c, p, mi, acc, (uint32_t)n, mixed, ctrl, cancel, launches)) return e;
                launches += 1;
            }
            b0 = b1;
        }
        launch_mcp_update(a, acc, more, c->sms, s);
        if (int e = check_launch("k_mcp_update")) return e;
        launches += 2;
        if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    }
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!dev) CU_TRY(cudaMemcpyAsync(recs, drec, npix * sizeof(mb3d_cu_mc_record), cudaMemcpyDeviceToHost, s));
    unsigned long long hc[4];
    CU_TRY(cudaMemcpyAsync(hc, acc.counters, sizeof(hc), cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.ms_march = ms;
    c->stats.launches = launches;
    c->stats.de_evals = hc[0];
    c->stats.mc_inside_rays = (uint32_t)hc[2];
    c->stats.mc_fp64_rays = (uint32_t)hc[3];
    c->stats.orbit_its[0] = rays_total;  // (the pass's rays)
    return 0;
}

int mb3d_cu_mc_render(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, const mb3d_cu_mc_light *lv, const mb3d_cu_mc_opts *o,
                      int precision, const mb3d_cu_mc_out *out, const volatile int *cancel) {
    if (!c || !sc || !lv || !o || !out || !out->radiance) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    if (o->rays < 1 || o->ray0 < 0 || (int64_t)o->ray0 + o->rays > 0x7FFFFFFF) return fail(MB3D_CU_EINVAL, "bad ray numbers");
    if (o->depth < 0 || o->depth > 64) return fail(MB3D_CU_EINVAL, "depth must be 0..64");
    int x0 = o->x0, y0 = o->y0, w = o->w, h = o->h;
    if (w == 0) {
        x0 = 0;
        y0 = 0;
        w = sc->width;
        h = sc->height;
    }
    if (w <= 0 || h <= 0 || x0 < 0 || y0 < 0 || (int64_t)x0 + w > sc->width || (int64_t)y0 + h > sc->height)
        return fail(MB3D_CU_EINVAL, "rectangle outside the picture");
    std::lock_guard<std::mutex> lk(c->mu);
    c->resume.active = false;  // (this call reuses the scratch a stopped budgeted march keeps)
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    McDev m;
    std::string err;
    int r = mc_setup(*sc, *lv, o->depth, o->secant, o->soft_shadow_radius, p, m, err);
    if (r < 0) return fail(r, err);
    apply_tuning(p);
    if (int e = mc_halton(c)) return e;
    if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    std::memset(&c->stats, 0, sizeof(c->stats));
    size_t npix = (size_t)w * (size_t)h;
    uint32_t tiles_x = (uint32_t)((w + 7) / 8), tiles_y = (uint32_t)((h + 3) / 4);
    size_t npad = (size_t)tiles_x * tiles_y * 32;
    m.rays = o->rays;
    m.ray0 = o->ray0;
    m.x0 = x0;
    m.y0 = y0;
    m.w = w;
    m.h = h;
    m.npad = (uint32_t)npad;
    m.tiles_x = tiles_x;
    m.halton = c->d_halton;
    // the pixel sums, hits, counters, and staging for host outputs
    bool d_rad = is_device_ptr(out->radiance);
    bool d_alb = out->albedo && is_device_ptr(out->albedo);
    bool d_nrm = out->normal && is_device_ptr(out->normal);
    bool d_dep = out->depth && is_device_ptr(out->depth);
    bool d_hit = out->hit && is_device_ptr(out->hit);
    size_t o_cnt = 0, o_sum = 256, o_hit = o_sum + align256(npix * 24), o_rad = o_hit + align256(npix * 4);
    size_t o_alb = o_rad + align256(npix * 12), o_nrm = o_alb + align256(npix * 12), o_dep = o_nrm + align256(npix * 12);
    size_t o_hb = o_dep + align256(npix * 4), need = o_hb + align256(npix);
    if (int e = grow((void **)&c->d_mc, &c->mc_cap, need)) return e;
    unsigned char *B = c->d_mc;
    McAcc acc;
    acc.counters = (unsigned long long *)(B + o_cnt);
    acc.sum = (unsigned long long *)(B + o_sum);
    acc.hit = (unsigned int *)(B + o_hit);
    acc.albedo = out->albedo ? (d_alb ? out->albedo : (float *)(B + o_alb)) : nullptr;
    acc.normal = out->normal ? (d_nrm ? out->normal : (float *)(B + o_nrm)) : nullptr;
    acc.depth = out->depth ? (d_dep ? out->depth : (float *)(B + o_dep)) : nullptr;
    float *rad = d_rad ? out->radiance : (float *)(B + o_rad);
    uint8_t *hb = out->hit ? (d_hit ? out->hit : (uint8_t *)(B + o_hb)) : nullptr;
    cudaStream_t s = c->stream;
    CU_TRY(cudaEventRecord(c->ev[0], s));
    CU_TRY(cudaMemsetAsync(B, 0, o_rad, s));  // counters, sums, hits
    if (acc.albedo) CU_TRY(cudaMemsetAsync(acc.albedo, 0, npix * 12, s));
    if (acc.normal) CU_TRY(cudaMemsetAsync(acc.normal, 0, npix * 12, s));
    if (acc.depth) CU_TRY(cudaMemsetAsync(acc.depth, 0, npix * 4, s));
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    // the rays in groups of at most 2^30 items, the cancel flag polled between them
    uint32_t per = (uint32_t)std::max<size_t>(1, ((size_t)1 << 30) / npad);
    uint32_t launches = 0;
    const bool mega = getenv("MB3D_CU_MC_MEGA") != nullptr;  // (the one-kernel form, for comparison)
    for (int b0 = 0; b0 < o->rays; b0 += (int)per) {
        int nb = std::min<int>((int)per, o->rays - b0);
        McDev mb = m;
        mb.ray0 = o->ray0 + b0;
        // (the first surface of ray ray0 only)
        McAcc ab = acc;
        if (b0 > 0) ab.albedo = ab.normal = ab.depth = nullptr;
        const uint32_t n_items = (uint32_t)((size_t)nb * npad);
        if (mega) {
            unsigned int *queue = (unsigned int *)(B + 64);
            CU_TRY(cudaMemsetAsync(queue, 0, 4, s));
            launch_mc(p, mb, mixed, false, ab, nullptr, nullptr, queue, n_items, nullptr, c->sms, s);
            launches++;
            if (int e = check_launch("k_mc")) return e;
        } else {
            // the split render: the paths' logic (k_mc_logic) and their marches
            // (k_mc in batch mode on the list of waiting paths) in turns
            if (int e = mc_split(c, p, mb, ab, n_items, mixed, (unsigned int *)(B + 128), cancel, launches)) return e;
        }
        if (cancel && b0 + (int)per < o->rays) {
            CU_TRY(cudaStreamSynchronize(s));
            if (*cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
        }
    }
    launch_mc_final(acc, (uint32_t)npix, o->rays, rad, hb, s);
    if (int e = check_launch("k_mc_final")) return e;
    CU_TRY(cudaEventRecord(c->ev[1], s));
    if (!d_rad) CU_TRY(cudaMemcpyAsync(out->radiance, rad, npix * 12, cudaMemcpyDeviceToHost, s));
    if (out->albedo && !d_alb) CU_TRY(cudaMemcpyAsync(out->albedo, acc.albedo, npix * 12, cudaMemcpyDeviceToHost, s));
    if (out->normal && !d_nrm) CU_TRY(cudaMemcpyAsync(out->normal, acc.normal, npix * 12, cudaMemcpyDeviceToHost, s));
    if (out->depth && !d_dep) CU_TRY(cudaMemcpyAsync(out->depth, acc.depth, npix * 4, cudaMemcpyDeviceToHost, s));
    if (out->hit && !d_hit) CU_TRY(cudaMemcpyAsync(out->hit, hb, npix, cudaMemcpyDeviceToHost, s));
    unsigned long long hc[4];
    CU_TRY(cudaMemcpyAsync(hc, acc.counters, sizeof(hc), cudaMemcpyDeviceToHost, s));
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
    c->stats.ms_total = ms;
    c->stats.ms_march = ms;
    c->stats.launches = launches + 1;
    c->stats.de_evals = hc[0];
    c->stats.mc_inside_rays = (uint32_t)hc[2];
    c->stats.mc_fp64_rays = (uint32_t)hc[3];
    if (cancel && *cancel) return fail(MB3D_CU_ECANCELED, "cancelled");
    return 0;
}

}  // extern "C"
