// gsw_loop.cu -- device-resident time-loop control and library plumbing.
//
// The reference computes dt on the host from a wave speed it reads back every step
// (geoswe/solver.py:2651, geoswe/compressed_solver.py:2238), which is a device sync
// per step. Here one single-thread kernel performs the same fp64 arithmetic on the
// device, so a window of steps can be captured in a CUDA graph and replayed with no
// host round trip; the host polls `done` once per window.
#include "gsw_common.cuh"
#include <atomic>
#include <string.h>

namespace gsw {

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

// Commit the previous step (t = t_new, steps += 1).
__device__ __forceinline__ void commit(GswLoopState* s) {
    if (s->pending) {
        s->t = s->t_new;
        s->steps += 1;
        s->pending = 0;
    }
}

// One thread. Mirrors, in this order:
//   Solver2D.run   : while t < t_end - 1e-12 and steps < max_steps        (solver.py:2990)
//   cfl_dt         : non-finite -> error; lam = max(lam, sqrt(g h_cfl));
//                    dt = cfl*dmin / (lam + 1e-12)                        (solver.py:2652-2666)
//   _rain_step_limit: dt = min(dt, (cfl dmin)^(2/3) / (g Rmax)^(1/3))     (solver.py:3005-3027)
//   dt_max, then the clip onto t_end                                      (solver.py:2992-2995)
// The flat loop (compressed_solver.py:713-748, 2133-2197) is the same arithmetic with
// eps_end = 1e-9 and the rain limit folded into dt_max by the caller.
__global__ void dt_finalize_kernel(GswDtParams p, GswLoopState* s) {
    commit(s);
    if (s->done) return;
    if (!(s->t < p.t_end - p.eps_end) || (p.max_steps > 0 && s->steps >= p.max_steps)) {
        s->done = 1;
        return;
    }
    const double t = s->t;
    int idx = 0;
    if (p.rain_t != nullptr && p.n_rain > 0) {       // bisect_right(time_s, t) - 1, clamped
        int lo = 0, hi = p.n_rain;
        while (lo < hi) { const int mid = (lo + hi) >> 1; if (t < p.rain_t[mid]) hi = mid; else lo = mid + 1; }
        idx = lo - 1;
        if (idx < 0) idx = 0;
        if (idx > p.n_rain - 1) idx = p.n_rain - 1;
    }
    s->rain_idx = idx;
    double dt;
    if (p.mode == 1) {
        dt = p.fixed_dt;
        s->lam_used = 0.0;
    } else {
        const double lam_in = __longlong_as_double((long long)s->lam_bits);
        if (!(lam_in <= 1.0e308)) {                   // NaN or Inf: the host raises FloatingPointError
            s->error = GSW_ERR_NONFINITE;
            s->done = 1;
            s->lam_used = lam_in;
            return;
        }
        double lam = lam_in;
        if (lam < p.lam_floor) lam = p.lam_floor;
        s->lam_used = lam;
        dt = __ddiv_rn(p.cfl_dmin, __dadd_rn(lam, 1.0e-12));
        if (p.rain_lim != nullptr && p.rain_lim[idx] > 0.0 && p.rain_lim[idx] < dt) dt = p.rain_lim[idx];
        if (p.dt_max > 0.0 && dt > p.dt_max) dt = p.dt_max;
    }
    if (p.clip_flat) {
        const double rem = __dsub_rn(p.t_end, t);
        if (rem < dt) dt = rem;
    } else if (__dadd_rn(t, dt) > p.t_end) {
        dt = __dsub_rn(p.t_end, t);
    }
    s->dt = dt;
    s->dt_f32 = (float)dt;
    s->t_new = __dadd_rn(t, dt);
    s->pending = 1;
    s->lam_bits = 0ull;                               // this step's kernels reduce lambda(next)
}

__global__ void loop_commit_kernel(GswLoopState* s) { commit(s); }

}  // namespace gsw

using namespace gsw;

extern "C" int gsw_dt_finalize(const GswDtParams* p, GswLoopState* state, void* stream) {
    GSW_CHECK_ABI(p);
    if (!state) return set_error(GSW_ERR_INVALID, "dt_finalize: null state");
    if (p->mode == 0 && !(p->cfl_dmin > 0.0)) return set_error(GSW_ERR_INVALID, "dt_finalize: cfl_dmin must be > 0");
    if (p->mode == 1 && !(p->fixed_dt > 0.0)) return set_error(GSW_ERR_INVALID, "dt_finalize: fixed_dt must be > 0");
    if (p->n_rain > 0 && !p->rain_t) return set_error(GSW_ERR_INVALID, "dt_finalize: rain_t is NULL");
    dt_finalize_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(*p, state);
    return check_launch("dt_finalize");
}

extern "C" int gsw_loop_commit(GswLoopState* state, void* stream) {
    if (!state) return set_error(GSW_ERR_INVALID, "loop_commit: null state");
    loop_commit_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(state);
    return check_launch("loop_commit");
}

extern "C" const char* gsw_last_error(void) { return g_err; }
extern "C" uint32_t gsw_abi_version(void) { return GSW_ABI_VERSION; }
extern "C" uint64_t gsw_launch_count(void) { return (uint64_t)g_launches.load(); }
