// gsw_common.cuh -- shared plumbing of libgsw: error state, launch checks, reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <algorithm>
#include "../../include/gsw.h"
#include "gsw_core.cuh"

// Library runtime, defined once in gsw_loop.cu: the thread-local message behind
// gsw_last_error(), the launch counter, the SM count. Kept out of namespace gsw, which
// a second compilation of the step kernels renames (gsw_fast.cu).
namespace gsw_rt {
int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);
int sm_count();
void count_launch(int n = 1);
float div_const_recip(float g);
}  // namespace gsw_rt

namespace gsw {

// Whether this compilation's binary32 step kernels may evaluate Manning's power by powf
// (GSW_ARITH_EXACT): the exact compilation yes, the fast one never (it keeps pow_m43).
// The choice is a template parameter of the step kernels, so each kernel holds one path.
#ifdef GSW_FAST_ARITH
constexpr bool kRefPowBuild = false;
#else
constexpr bool kRefPowBuild = true;
#endif

using gsw_rt::set_error;
using gsw_rt::check_launch;
using gsw_rt::sm_count;
using gsw_rt::count_launch;
using gsw_rt::div_const_recip;

// Max of a non-negative IEEE-bits value over the block, then one atomicMax.
// Every thread of the block must call it (it holds a block barrier).
__device__ __forceinline__ void block_max_to(unsigned long long v, unsigned long long* target) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    __shared__ unsigned long long s_red[32];
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthreads + 31) >> 5;
    if (lane == 0) s_red[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = lane < nw ? s_red[lane] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
            v = w > v ? w : v;
        }
        if (lane == 0 && v != 0ull) atomicMax(target, v);
    }
}

// Commit the previous step (t = t_new, steps += 1).
__device__ __forceinline__ void loop_commit(GswLoopState* s) {
    if (s->pending) {
        s->t = s->t_new;
        s->steps += 1;
        s->pending = 0;
    }
}

// The time-step rule of one solver, evaluated by one thread (gsw.h, GswDtParams). Mirrors
// in this order:
//   Solver2D.run   : while t < t_end - 1e-12 and steps < max_steps        (solver.py:2990)
//   cfl_dt         : non-finite -> error; lam = max(lam, sqrt(g h_cfl));
//                    dt = cfl*dmin / (lam + 1e-12)                        (solver.py:2652-2666)
//   _rain_step_limit: dt = min(dt, (cfl dmin)^(2/3) / (g Rmax)^(1/3))     (solver.py:3005-3027)
//   dt_max, then the clip onto t_end                                      (solver.py:2992-2995)
// The flat loop (compressed_solver.py:713-748, 2133-2197) is the same arithmetic with
// eps_end = 1e-9, the rain limit folded into dt_max and dt = min(dt, t_end - t).
// Mode 2 replays a recorded dt schedule (the adjoint's frozen forward); dt_log records one.
__device__ __forceinline__ void dt_finalize_one(const GswDtParams& p, GswLoopState* s,
                                                unsigned long long lam_bits) {
    loop_commit(s);
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
    } else if (p.mode == 2) {                         // a recorded schedule, replayed as is
        dt = p.dt_table[s->steps];
        s->lam_used = 0.0;
        s->dt = dt;
        s->dt_f32 = (float)dt;
        s->t_new = __dadd_rn(t, dt);
        s->pending = 1;
        s->lam_bits = 0ull;
        return;
    } else {
        const double lam_in = __longlong_as_double((long long)lam_bits);
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
    if (p.dt_log != nullptr) p.dt_log[s->steps] = dt;
}

}  // namespace gsw

#define GSW_CHECK_ABI(a)                                                                     \
    do {                                                                                     \
        if ((a) == nullptr) return gsw::set_error(GSW_ERR_INVALID, "null argument struct");  \
        if ((a)->abi_version != GSW_ABI_VERSION)                                             \
            return gsw::set_error(GSW_ERR_ABI, "abi_version %u, library is %u",              \
                                  (unsigned)(a)->abi_version, (unsigned)GSW_ABI_VERSION);    \
    } while (0)
