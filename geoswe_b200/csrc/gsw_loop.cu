// gsw_loop.cu -- device-resident time-loop control and library plumbing.
//
// The reference computes dt on the host from a wave speed it reads back every step
// (geoswe/solver.py:2651, geoswe/compressed_solver.py:2238), which is a device sync
// per step. Here one single-thread kernel performs the same fp64 arithmetic on the
// device, so a window of steps can be captured in a CUDA graph and replayed with no
// host round trip; the host polls `done` once per window.
#include "gsw_common.cuh"
#include <atomic>
#include <cmath>
#include <mutex>
#include <string.h>
#include <unordered_map>

namespace gsw_rt {

static thread_local char g_err[512] = "";
static std::atomic<unsigned long long> g_launches{0};

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void count_launch(int n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }

int check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(GSW_ERR_CUDA, "%s: launch failed: %s", what, cudaGetErrorString(e));
    count_launch(1);
    return GSW_OK;
}

int sm_count() {
    static int cached = 0;
    if (cached == 0) {
        int dev = 0, n = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0)
            cached = n;
        else
            cached = 148;
    }
    return cached;
}

// RN(1/g) when the correction sequence of gsw::div_g reproduces the IEEE quotient h / g
// for every binary32 significand of h (checked exhaustively, once per g per process;
// the IEEE quotient by the double quotient rounded once more, exact since 53 >= 2*24+2
// bits), else 0 (the kernels then divide).
float div_const_recip(float g) {
    static std::mutex mu;
    static std::unordered_map<uint32_t, float> cache;
    uint32_t key;
    memcpy(&key, &g, sizeof(key));
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    float y = 0.0f;
    if (std::isnormal(g) && g > 0.0f) {
        const float yy = (float)(1.0 / (double)g);
        bool ok = std::isnormal(yy);
        for (uint32_t m = 0; ok && m < (1u << 23); ++m) {
            const uint32_t bits = 0x3f800000u | m;
            float h;
            memcpy(&h, &bits, sizeof(h));
            const float ref = (float)((double)h / (double)g);
            const float q0 = h * yy;
            const float r = std::fmaf(-g, q0, h);
            const float q = std::fmaf(r, yy, q0);
            ok = memcmp(&q, &ref, sizeof(q)) == 0;
        }
        if (ok) y = yy;
    }
    std::lock_guard<std::mutex> lock(mu);
    cache[key] = y;
    return y;
}

}  // namespace gsw_rt

namespace gsw {

__global__ void dt_finalize_kernel(GswDtParams p, GswLoopState* s) { dt_finalize_one(p, s, s->lam_bits); }
// The same with the parameters read from device memory: a captured launch then follows
// whatever t_end / dt_max / max_steps the last gsw_dt_params_upload wrote.
__global__ void dt_finalize_dev_kernel(const GswDtParams* p, GswLoopState* s) {
    dt_finalize_one(*p, s, s->lam_bits);
}

__global__ void loop_commit_kernel(GswLoopState* s) { loop_commit(s); }

}  // namespace gsw

using namespace gsw;

static int check_dt_params(const GswDtParams* p) {
    if (p->mode == 0 && !(p->cfl_dmin > 0.0)) return set_error(GSW_ERR_INVALID, "dt_finalize: cfl_dmin must be > 0");
    if (p->mode == 1 && !(p->fixed_dt > 0.0)) return set_error(GSW_ERR_INVALID, "dt_finalize: fixed_dt must be > 0");
    if (p->mode == 2 && !p->dt_table) return set_error(GSW_ERR_INVALID, "dt_finalize: dt_table is NULL");
    if (p->mode < 0 || p->mode > 2) return set_error(GSW_ERR_INVALID, "dt_finalize: mode %d", p->mode);
    if (p->n_rain > 0 && !p->rain_t) return set_error(GSW_ERR_INVALID, "dt_finalize: rain_t is NULL");
    return GSW_OK;
}

extern "C" int gsw_dt_finalize(const GswDtParams* p, GswLoopState* state, void* stream) {
    GSW_CHECK_ABI(p);
    if (!state) return set_error(GSW_ERR_INVALID, "dt_finalize: null state");
    if (int rc = check_dt_params(p)) return rc;
    dt_finalize_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(*p, state);
    return check_launch("dt_finalize");
}

extern "C" int gsw_dt_params_upload(const GswDtParams* p, GswDtParams* dev, void* stream) {
    GSW_CHECK_ABI(p);
    if (!dev) return set_error(GSW_ERR_INVALID, "dt_params_upload: null destination");
    if (int rc = check_dt_params(p)) return rc;
    // pageable source: the copy is staged before the call returns, so *p may be reused
    const cudaError_t e = cudaMemcpyAsync(dev, p, sizeof(GswDtParams), cudaMemcpyHostToDevice,
                                          (cudaStream_t)stream);
    if (e != cudaSuccess) return set_error(GSW_ERR_CUDA, "dt_params_upload: %s", cudaGetErrorString(e));
    return GSW_OK;
}

extern "C" int gsw_dt_finalize_dev(const GswDtParams* dev, GswLoopState* state, void* stream) {
    if (!dev || !state) return set_error(GSW_ERR_INVALID, "dt_finalize_dev: null pointer");
    dt_finalize_dev_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(dev, state);
    return check_launch("dt_finalize_dev");
}

extern "C" int gsw_loop_commit(GswLoopState* state, void* stream) {
    if (!state) return set_error(GSW_ERR_INVALID, "loop_commit: null state");
    loop_commit_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(state);
    return check_launch("loop_commit");
}

extern "C" float gsw_div_const_recip(float g) { return gsw_rt::div_const_recip(g); }
extern "C" const char* gsw_last_error(void) { return gsw_rt::g_err; }
extern "C" uint32_t gsw_abi_version(void) { return GSW_ABI_VERSION; }
extern "C" uint64_t gsw_launch_count(void) { return (uint64_t)gsw_rt::g_launches.load(); }
