// gsw_ensemble_march.cuh -- the persistent ensemble step kernel and its launcher.
//
// All members' bricks sit in one brick storage. A step is one launch of a persistent
// grid (a few blocks per SM): warps stride over the global brick list, look up the
// brick's member, and advance it with that member's dt, rain rate and Manning table
// (the per-brick march of gsw_flat_brick.cuh). Each member's new wave speed is reduced
// into its own GswLoopState. The block that finishes last (a ticket counter in scratch
// memory) then evaluates every member's time-step rule for the next launch, so members
// keep their own CFL dt with no grid-wide barrier and no host round trip; a member that
// reaches its end time drops out while the others continue. With a running-member list
// (GswEnsembleArgs.run) warps walk only the running members' bricks, and the last block
// rebuilds the list when a member finishes. Warps take their next brick from a counter
// in scratch memory, so the uneven bricks of uneven members balance over the grid.
//
// Included by gsw_ensemble.cu (exact arithmetic) and gsw_fast.cu (fast arithmetic,
// with namespace gsw renamed).
#pragma once
#include "gsw_flat_brick.cuh"

namespace gsw {

__device__ __forceinline__ FlatPhys<float> member_phys(const GswMember& mb, int ref_pow) {
    FlatPhys<float> ph;
    ph.inv_dx = mb.inv_dx; ph.inv_dy = mb.inv_dx;
    ph.half_dx = 0.5f * (1.0f / mb.inv_dx); ph.half_dy = ph.half_dx;
    ph.g = mb.g; ph.h_min = mb.h_min; ph.h_min_cfl = mb.h_min_cfl; ph.vcap = mb.vcap;
    ph.linf = mb.linf; ph.quad = mb.quadratic; ph.keep_h = mb.keep_h;
    ph.rain_kind = mb.rain_kind; ph.rain = mb.rain; ph.ntab = mb.n_tab;
    ph.ngh = 0; ph.nx = 0; ph.ny = 0; ph.lookup = nullptr; ph.ncol = 0;
    ph.g_recip = mb.g_recip; // 0: the member divides
    ph.ref_pow = ref_pow;
    return ph;
}

// Rebuild the running-member brick list (GswEnsembleArgs.run) from the members' done
// flags: each thread of the block takes a contiguous chunk of members, counts its
// running members and their bricks, one thread scans the per-thread totals, and each
// thread writes its chunk's entries. Every thread of the block calls it.
__device__ __forceinline__ void build_run_list(const GswEnsembleArgs& a, int tid, int nth) {
    __shared__ long long s_bricks[256];
    __shared__ int s_count[256];
    const int M = a.n_members;
    const int chunk = (M + nth - 1) / nth;
    const int k0 = min(M, tid * chunk), k1 = min(M, k0 + chunk);
    long long nb = 0;
    int nr = 0;
    for (int k = k0; k < k1; ++k)
        if (!a.states[k].done) { nb += a.member_brick_off[k + 1] - a.member_brick_off[k]; ++nr; }
    s_bricks[tid] = nb;
    s_count[tid] = nr;
    __syncthreads();
    if (tid == 0) {
        long long pb = 0;
        int pr = 0;
        for (int t = 0; t < nth; ++t) {
            const long long b = s_bricks[t];
            const int r = s_count[t];
            s_bricks[t] = pb; s_count[t] = pr;
            pb += b; pr += r;
        }
        a.run[0] = pr;
        a.run[1 + pr] = pb;
    }
    __syncthreads();
    long long pb = s_bricks[tid];
    int pr = s_count[tid];
    for (int k = k0; k < k1; ++k)
        if (!a.states[k].done) {
            a.run[1 + pr] = pb;
            a.run[M + 2 + pr] = k;
            pb += a.member_brick_off[k + 1] - a.member_brick_off[k];
            ++pr;
        }
}

// LEAN: every member in the production configuration (quadratic friction, keep-h, the L2
// norm; members take rain none or uniform), compiled in as in the stand-alone flat step.
template <int MINB, bool REFPOW, bool LEAN>
__global__ void __launch_bounds__(256, MINB) ensemble_step_kernel(GswEnsembleArgs a, FlatMesh<float> m) {
    if (*a.all_done) return;
    const int lane = threadIdx.x;
    const int W = blockDim.y;
    const bool listed = a.run != nullptr;
    const int n_run = listed ? (int)a.run[0] : 0;
    const int64_t bricks = listed ? a.run[1 + n_run] : a.n_bricks;
    const int S = a.segments > 0 ? a.segments                // row segments per brick, or by the work in flight
                                 : auto_segments(bricks, (int64_t)gridDim.x * W, m.bh);
    const int64_t total = bricks * S;
    // work items (brick, row segment) are taken from a counter (scratch[1]) as warps free
    // up, so bricks of uneven cost balance across the fixed persistent grid
    unsigned int* next_item = a.scratch + 1;
    for (;;) {
        long long got = 0;
        if (lane == 0) got = (long long)atomicAdd(next_item, 1u);
        const int64_t item = __shfl_sync(0xffffffffu, got, 0);
        if (item >= total) break;
        const int64_t v = item / S;
        const int seg = (int)(item - v * S);
        int64_t b;
        int mi;
        if (listed) {                  // the running member whose brick range holds v (warp-uniform)
            int lo = 0, hi = n_run - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (a.run[1 + mid] <= v) lo = mid; else hi = mid - 1;
            }
            mi = (int)a.run[a.n_members + 2 + lo];
            b = a.member_brick_off[mi] + (v - a.run[1 + lo]);
        } else {
            b = v;
            mi = a.brick_member[b];
        }
        const GswLoopState* st = a.states + mi;
        if (st->done) continue;                                   // warp-uniform
        const GswMember& mb = a.members[mi];
        if (LEAN && !(mb.quadratic != 0 && mb.keep_h != 0 && mb.linf == 0)) {   // warp-uniform
            if (lane == 0) {            // not what this step was compiled for: the member stops
                a.states[mi].error = GSW_ERR_INVALID;
                a.states[mi].done = 1;
            }
            continue;
        }
        const FlatPhys<float> ph = member_phys(mb, REFPOW ? 1 : 0);
        const float dt = st->dt_f32;
        const float rate = (mb.rain_kind == GSW_RAIN_UNIFORM) ? mb.rain[st->rain_idx] : 0.0f;
        unsigned long long lam = flat_brick<float, true, REFPOW, LEAN>(m, ph, b, seg * m.bh / S, (seg + 1) * m.bh / S,
                                                               dt, rate, nullptr);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(0xffffffffu, lam, o);
            lam = w > lam ? w : lam;
        }
        if (lane == 0 && lam != 0ull) atomicMax((unsigned long long*)&a.states[mi].lam_bits, lam);
    }
    // the last block to arrive evaluates every member's rule for the next step
    __shared__ int s_last;
    __syncthreads();
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    if (tid == 0) {
        __threadfence();
        const unsigned int ticket = atomicAdd(&a.scratch[0], 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const int nth = blockDim.x * blockDim.y;
    __shared__ int s_open, s_finished;
    if (tid == 0) { s_open = 0; s_finished = 0; }
    __syncthreads();
    for (int mi = tid; mi < a.n_members; mi += nth) {
        GswLoopState* st = a.states + mi;
        const unsigned long long lb = atomicAdd((unsigned long long*)&st->lam_bits, 0ull);  // coherent read
        const int was_done = st->done;
        dt_finalize_one(a.members[mi].dt, st, lb);
        if (!st->done) atomicAdd(&s_open, 1);
        else if (!was_done) s_finished = 1;
    }
    __syncthreads();
    if (listed && s_finished && s_open > 0) build_run_list(a, tid, nth);   // block-uniform condition
    if (tid == 0) {
        a.scratch[0] = 0u;           // every block has passed its loop: both counters back to zero
        a.scratch[1] = 0u;
        *a.all_done = (s_open == 0) ? 1 : 0;
    }
}

template <bool REFPOW, bool LEAN>
inline void launch_ensemble_caps(const GswEnsembleArgs* a, const FlatMesh<float>& m, int grid, int W, cudaStream_t st) {
    if (a->min_blocks == 3) ensemble_step_kernel<3, REFPOW, LEAN><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else if (a->min_blocks == 4) ensemble_step_kernel<4, REFPOW, LEAN><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else if (a->min_blocks == 5) ensemble_step_kernel<5, REFPOW, LEAN><<<grid, dim3(32, W), 0, st>>>(*a, m);
    else ensemble_step_kernel<1, REFPOW, LEAN><<<grid, dim3(32, W), 0, st>>>(*a, m);
}

template <bool REFPOW>
inline void launch_ensemble_shape(const GswEnsembleArgs* a, const FlatMesh<float>& m, int grid, int W, cudaStream_t st) {
    if (a->lean) launch_ensemble_caps<REFPOW, true>(a, m, grid, W, st);
    else launch_ensemble_caps<REFPOW, false>(a, m, grid, W, st);
}

// Launch of the step over checked arguments (outputs non-null).
inline int launch_ensemble_step(const GswEnsembleArgs* a, cudaStream_t st) {
    const int W = a->warps > 0 ? a->warps : 4;
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "ensemble: warps must be in [1, 8]");
    const int grid = a->grid > 0 ? a->grid : 2 * sm_count();
    const int S = a->segments > 0 ? a->segments : 1;
    if ((S != 1 && S != 2 && S != 4) || a->brick_h % S != 0 || a->segments < 0)
        return set_error(GSW_ERR_INVALID, "ensemble: segments must be 0, 1, 2 or 4 and divide brick_h");
    if (a->n_bricks * 4 >= (int64_t)UINT32_MAX) return set_error(GSW_ERR_INVALID, "ensemble: too many bricks");
    FlatMesh<float> m;
    m.q0 = a->q0; m.q1 = a->q1; m.q2 = a->q2;
    m.o0 = a->qn0; m.o1 = a->qn1; m.o2 = a->qn2;
    m.b = a->bed; m.flags = a->flags; m.ncls = a->n_cls; m.max_h = a->max_h;
    m.bij = a->brick_ij; m.bnbr = a->brick_nbr; m.nb = a->n_bricks; m.bh = a->brick_h;
    if (a->min_blocks != 0 && (a->min_blocks < 3 || a->min_blocks > 5))
        return set_error(GSW_ERR_INVALID, "ensemble: min_blocks must be 0, 3, 4 or 5");
    if (kRefPowBuild && a->arith == GSW_ARITH_EXACT) launch_ensemble_shape<kRefPowBuild>(a, m, grid, W, st);
    else launch_ensemble_shape<false>(a, m, grid, W, st);
    return check_launch("ensemble_step");
}

}  // namespace gsw
