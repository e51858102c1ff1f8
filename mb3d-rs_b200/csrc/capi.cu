// The C ABI (include/mb3d_cu.h): contexts, buffers, launches and the error
// convention of mb3d-rs's C API (a thread-local last error,
// capi/src/lib.rs:18-40).  There is no CPU fallback: a failure is a
// negative status and the caller decides what to do.
#include <cuda_runtime.h>
#include <cstring>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/mb3d_cu.h"
#include "devparams.h"
#include "kernels.h"
#include "setup.h"

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
    unsigned int *d_counters = nullptr;
    double *d_probe = nullptr;
    size_t probe_cap = 0;
    cudaEvent_t ev[8] = {};
    mb3d_cu_stats stats = {};
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
    if (cudaMalloc(&c->d_counters, 64 * sizeof(unsigned int)) != cudaSuccess) {
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
    cudaFree(c->d_gbuf);
    cudaFree(c->d_hand);
    cudaFree(c->d_counters);
    cudaFree(c->d_probe);
    for (auto &ev : c->ev)
        if (ev) cudaEventDestroy(ev);
    if (c->own) cudaStreamDestroy(c->own);
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
    c->stats.fp64_pixels = 0;
    CU_TRY(cudaEventRecord(c->ev[0], s));
    if (precision == MB3D_CU_FP64 || p.all_fp64) {
        launch_march64(p, row0, rows, dg, s);
        c->stats.launches += 1;
        if (int r = check_launch("k_march64")) return r;
        CU_TRY(cudaEventRecord(c->ev[1], s));
        CU_TRY(cudaEventRecord(c->ev[2], s));
        if (precision != MB3D_CU_FP64) c->stats.fp64_pixels = (uint32_t)npix;
    } else {
        if (int r = grow((void **)&c->d_hand, &c->hand_cap, npix * sizeof(Hand))) return r;
        CU_TRY(cudaMemsetAsync(c->d_counters, 0, 64 * sizeof(unsigned int), s));
        launch_march32(p, row0, rows, dg, c->d_hand, c->d_counters, c->sms, s);
        if (int r = check_launch("k_march32")) return r;
        CU_TRY(cudaEventRecord(c->ev[1], s));
        launch_finish64(p, row0, c->d_hand, c->d_counters, dg, c->sms, s);
        if (int r = check_launch("k_finish64")) return r;
        CU_TRY(cudaEventRecord(c->ev[2], s));
        c->stats.launches += 2;
    }
    return 0;
}

static int post_device(mb3d_cu_ctx *c, const DevParams &p, int precision, int passes, int row0, int rows,
                       mb3d_cu_silight *dg) {
    cudaStream_t s = c->stream;
    bool mixed = precision != MB3D_CU_FP64 && !p.all_fp64;
    CU_TRY(cudaEventRecord(c->ev[3], s));
    if ((passes & MB3D_CU_POST_SHADOW) && p.n_lights > 0) {
        launch_shadow(p, row0, rows, dg, mixed, s);
        c->stats.launches += 1;
        if (int r = check_launch("k_shadow")) return r;
    }
    CU_TRY(cudaEventRecord(c->ev[4], s));
    if ((passes & MB3D_CU_POST_DEAO) && p.ao_quality >= 0 && p.ao_rays > 0) {
        launch_deao(p, row0, rows, dg, mixed, s);
        c->stats.launches += 1;
        if (int r = check_launch("k_deao")) return r;
    }
    CU_TRY(cudaEventRecord(c->ev[5], s));
    return 0;
}

static int finish_call(mb3d_cu_ctx *c, bool marched, bool posted) {
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    float ms = 0.f;
    if (marched) {
        cudaEventElapsedTime(&ms, c->ev[0], c->ev[2]);
        c->stats.ms_march = ms;
        cudaEventElapsedTime(&ms, c->ev[1], c->ev[2]);
        c->stats.ms_finish = ms;
    }
    if (posted) {
        cudaEventElapsedTime(&ms, c->ev[3], c->ev[4]);
        c->stats.ms_shadow = ms;
        cudaEventElapsedTime(&ms, c->ev[4], c->ev[5]);
        c->stats.ms_deao = ms;
    }
    cudaEventElapsedTime(&ms, marched ? c->ev[0] : c->ev[3], posted ? c->ev[5] : c->ev[2]);
    c->stats.ms_total = ms;
    return 0;
}

static int run(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, int passes, bool do_march, uint32_t row0,
               uint32_t rows, mb3d_cu_silight *gbuf, const volatile int *cancel) {
    if (!c || !sc || !gbuf) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (precision != MB3D_CU_FP64 && precision != MB3D_CU_FP32_FP64) return fail(MB3D_CU_EINVAL, "unknown precision");
    std::lock_guard<std::mutex> lk(c->mu);
    if (cudaSetDevice(c->device) != cudaSuccess) return fail(MB3D_CU_EIO, "cudaSetDevice failed");
    DevParams p;
    std::string err;
    int r = setup_params(*sc, p, err);
    if (r < 0) return fail(r, err);
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

int mb3d_cu_de_probe(mb3d_cu_ctx *c, const mb3d_cu_scene *sc, int precision, const double *pos, uint32_t n, double *de,
                     int32_t *its) {
    if (!c || !sc || !pos || !de || !its) return fail(MB3D_CU_EINVAL, "NULL argument");
    if (n == 0) return 0;
    std::lock_guard<std::mutex> lk(c->mu);
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

}  // extern "C"
