// gsw_forcing.cu -- discharge inflow through ghost cells, on the device.
//
// The reference evaluates each inlet on the host every step: np.interp for Q(t), a
// NumPy sum of the inlet depths (a device sync on the GPU path) and fancy-index writes
// (geoswe/solver.py:1944-1971, geoswe/bc.py:175-235). This kernel performs the same
// arithmetic in one block per inlet, inside the captured step, including NumPy's
// pairwise float summation order so the depth weights are bit-identical.
#include "gsw_forcing.cuh"

namespace gsw {

template <typename T>
__global__ void inflow_kernel(GswInflowArgs a) {
    if (a.state->done) return;
    T* q0 = (T*)a.q0; T* q1 = (T*)a.q1; T* q2 = (T*)a.q2;
    const T* bed = (const T*)a.bed;
    __shared__ double s_Q, s_sum, s_add;
    __shared__ T s_zmin, s_zmax;
    __shared__ int s_wet, s_nlow, s_flat;
    if (threadIdx.x == 0) {
        s_Q = np_interp(a.state->t, a.t_knots, a.q_knots, a.n_knots);
        s_sum = a.hsum != nullptr ? *a.hsum : (double)pairwise_sum<T>(q0, a.inlet_off, 0, a.n);
        s_wet = s_sum > 0.0;
        if (!s_wet) {
            T zmin = bed[a.inlet_off[0]], zmax = zmin;
            for (int k = 1; k < a.n; ++k) {
                const T z = bed[a.inlet_off[k]];
                zmin = z < zmin ? z : zmin;        // np.min / np.max of finite values
                zmax = z > zmax ? z : zmax;
            }
            s_zmin = zmin; s_zmax = zmax;
            int nlow = 0;
            T hmax = (T)0;
            const T frac = (T)a.dry_frac;
            for (int k = 0; k < a.n; ++k) {
                const T z = bed[a.inlet_off[k]];
                nlow += (z <= zmin);
                T hf = zmin + frac * (zmax - zmin) - z;
                hf = hf > (T)0 ? hf : (T)0;
                hmax = (k == 0 || hf > hmax) ? hf : hmax;
            }
            s_nlow = nlow;
            s_flat = !((double)hmax > 0.0);
            s_add = 0.0;
            if (s_flat) {
                const double nl = nlow > 1 ? (double)nlow : 1.0;
                const double qc = __ddiv_rn(fabs(s_Q), __dmul_rn(nl, a.ds));
                s_add = pow(__ddiv_rn(__dmul_rn(qc, qc), 9.80665), 1.0 / 3.0);
            }
        }
    }
    __syncthreads();
    const double Q = s_Q;
    const int64_t total = (int64_t)a.n * a.ngh;
    for (int64_t t = threadIdx.x; t < total; t += blockDim.x) {
        const int k = (int)(t % a.n);
        const int gk = (int)(t / a.n) + 1;                       // ghost layer 1..ngh
        const int64_t src = a.inlet_off[k];
        const int64_t go = src + (int64_t)gk * a.step_off;
        const T h = q0[src];
        T hf, hu, hv;
        if (s_wet) {
            const T w = h / (T)s_sum;                            // h / s in the array dtype
            const T qn = (T)__ddiv_rn(Q, a.ds) * w;              // (Q/ds) * w
            hf = h;
            hu = qn * (T)a.nx_n;
            hv = qn * (T)a.ny_n;
        } else {
            const T z = bed[src];
            T f = s_zmin + (T)a.dry_frac * (s_zmax - s_zmin) - z;
            f = f > (T)0 ? f : (T)0;
            if (s_flat) f = f + (T)s_add;
            const double nl = s_nlow > 1 ? (double)s_nlow : 1.0;
            const double w = (z <= s_zmin) ? __ddiv_rn(1.0, nl) : 0.0;   // float64 weights
            const double qn = __dmul_rn(__ddiv_rn(Q, a.ds), w);
            hf = f;
            hu = (T)__dmul_rn(qn, a.nx_n);
            hv = (T)__dmul_rn(qn, a.ny_n);
        }
        q0[go] = hf; q1[go] = hu; q2[go] = hv;
    }
}

// This rank's share of an inlet's depth sum (a split run all-reduces these).
template <typename T>
__global__ void inflow_depth_sum_kernel(GswInflowArgs a, double* out) {
    if (threadIdx.x == 0)
        *out = a.n > 0 ? (double)pairwise_sum<T>((const T*)a.q0, a.inlet_off, 0, a.n) : 0.0;
}

template <typename T>
__global__ void flat_inflow_depth_sum_kernel(GswFlatInflowArgs a, double* out) {
    if (threadIdx.x == 0)
        *out = a.n > 0 ? (double)pairwise_sum<T>((const T*)a.q0, a.nbr_slot, 0, a.n) : 0.0;
}

// Flat-tier inlet (compressed_solver.py:2144-2167, dry seed :1559-1594). One block per
// inlet; thread 0 evaluates Q, the depth sum and the dry seed, all threads write ghosts.
template <typename T>
__global__ void flat_inflow_kernel(GswFlatInflowArgs a) {
    if (a.state->done) return;
    T* q0 = (T*)a.q0; T* q1 = (T*)a.q1; T* q2 = (T*)a.q2;
    const T* bed = (const T*)a.bed;
    __shared__ double s_Q, s_sum, s_zmin, s_add, s_nlow;
    __shared__ T s_seed;
    __shared__ int s_wet, s_flat;
    if (threadIdx.x == 0) {
        s_Q = np_interp(a.state->t, a.t_knots, a.q_knots, a.n_knots);
        s_sum = a.hsum != nullptr ? *a.hsum : (double)pairwise_sum<T>(q0, a.nbr_slot, 0, a.n);
        s_wet = s_sum > 0.0;
        if (!s_wet && a.dry != nullptr) {       // the seed's reductions over every rank's cells
            const double zlo = a.dry[0], zhi = a.dry[1];
            s_seed = (T)__dadd_rn(zlo, __dmul_rn(0.10, __dsub_rn(zhi, zlo)));
            s_zmin = zlo;
            s_nlow = a.dry[2] > 0.0 ? a.dry[2] : 1.0;
            s_flat = !(a.dry[3] > 0.0);
        } else if (!s_wet) {
            T zmin = bed[a.nbr_slot[0]], zmax = zmin;
            for (int k = 1; k < a.n; ++k) {
                const T z = bed[a.nbr_slot[k]];
                zmin = z < zmin ? z : zmin;
                zmax = z > zmax ? z : zmax;
            }
            const double zlo = (double)zmin, zhi = (double)zmax;
            const T seed = (T)__dadd_rn(zlo, __dmul_rn(0.10, __dsub_rn(zhi, zlo)));
            int nlow = 0;
            T hmax = (T)0;
            for (int k = 0; k < a.n; ++k) {
                const T z = bed[a.nbr_slot[k]];
                nlow += (z <= zmin);
                T hf = seed - z;
                hf = hf > (T)0 ? hf : (T)0;
                hmax = (k == 0 || hf > hmax) ? hf : hmax;
            }
            s_seed = seed;
            s_zmin = zlo;
            s_nlow = nlow > 0 ? (double)nlow : 1.0;
            s_flat = !((double)hmax > 0.0);
        }
        if (!s_wet) {
            s_add = 0.0;
            if (s_flat) {
                const double qc = __ddiv_rn(fabs(s_Q), __dmul_rn(s_nlow, a.ds));
                s_add = pow(__ddiv_rn(__dmul_rn(qc, qc), 9.80665), 1.0 / 3.0);
            }
        }
    }
    __syncthreads();
    const T qds = (T)__ddiv_rn(s_Q, a.ds);
    for (int k = threadIdx.x; k < a.n; k += blockDim.x) {
        const int64_t src = a.nbr_slot[k];
        T hf, w;
        if (s_wet) {
            hf = q0[src];
            w = hf / (T)s_sum;
        } else {
            const T z = bed[src];
            hf = s_seed - z;
            hf = hf > (T)0 ? hf : (T)0;
            if (s_flat) hf = hf + (T)s_add;
            w = ((double)z <= s_zmin) ? (T)__ddiv_rn(1.0, s_nlow) : (T)0;
        }
        const T qn = qds * w;
        const int64_t go = a.ghost_slot[k];
        q0[go] = hf;
        q1[go] = qn * (T)a.nx_n;
        q2[go] = qn * (T)a.ny_n;
    }
}

// Ring stage of the compressed mesh (ring_bc_flat, compressed_solver.py:287-307, with
// the on-device stage interpolation of :2338-2350). One thread per ring cell.
template <typename T>
__global__ void flat_ring_kernel(GswFlatRingArgs a) {
    if (a.state->done) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.n) return;
    const double t = a.state->t;
    int lo = 0, hi = a.n_t;                          // searchsorted(t_common, t, side="left")
    while (lo < hi) { const int mid = (lo + hi) >> 1; if (a.t_common[mid] < t) lo = mid + 1; else hi = mid; }
    int ti = lo - 1;
    if (ti > a.n_t - 2) ti = a.n_t - 2;
    if (ti < 0) ti = 0;
    double wt = __ddiv_rn(__dsub_rn(t, a.t_common[ti]),
                          __dadd_rn(__dsub_rn(a.t_common[ti + 1], a.t_common[ti]), 1.0e-12));
    wt = wt < 1.0 ? wt : 1.0;
    wt = wt > 0.0 ? wt : 0.0;
    const T w0 = (T)__dsub_rn(1.0, wt), w1 = (T)wt;
    const T* st = (const T*)a.stage_all;
    const T* w = (const T*)a.wg + (int64_t)k * a.NG;
    T eta = (T)0;
    for (int g = 0; g < a.NG; ++g) {
        T s = st[(int64_t)g * a.n_t + ti] * w0;
        s = s + st[(int64_t)g * a.n_t + ti + 1] * w1;
        eta = eta + w[g] * s;
    }
    const int64_t idx = a.slots[k];
    if (idx < 0) return;
    const T h = eta - ((const T*)a.bed)[k];
    ((T*)a.q0)[idx] = h > (T)0 ? h : (T)0;
    ((T*)a.q1)[idx] = (T)0;
    ((T*)a.q2)[idx] = (T)0;
}

// ---- per-step forcings of the flat loop (compressed_solver.py:2330-2366) ----
// Landcover infiltration, infiltrate_flat (:143-158).
__global__ void flat_infiltrate_kernel(GswFlatForcingArgs a) {
    if (a.state->done) return;
    const float dt = a.state->dt_f32;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a.nslots;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (!(a.flags[k] & GSW_SLOT_ACTIVE)) continue;
        const float h = a.q0[k];
        if (h < a.h_min) continue;
        const float dh = a.infil_tab[a.n_cls ? a.n_cls[k] : 0] * dt;
        float hn = h - dh;
        if (hn < 0.0f) hn = 0.0f;
        const float r = hn / h;
        a.q0[k] = hn; a.q1[k] = a.q1[k] * r; a.q2[k] = a.q2[k] * r;
    }
}

// Open-boundary sponge over its band, sponge_band (:1320-1328).
__global__ void flat_sponge_kernel(GswFlatForcingArgs a) {
    if (a.state->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.sp_n) return;
    const int64_t k = a.sp_slots[i];
    const float kp = a.sp_keep[i];
    a.q0[k] = __fadd_rn(__fmul_rn(a.q0[k], kp), a.sp_amb[i]);
    a.q1[k] = a.q1[k] * kp;
    a.q2[k] = a.q2[k] * kp;
}

// Green-Ampt infiltration and the linear-reservoir drain, ga_drain_flat / ga_flat /
// drain_tau_flat (:313-420): one momentum scale accumulated over both, as the reference.
__global__ void flat_ga_drain_kernel(GswFlatForcingArgs a) {
    if (a.state->done) return;
    const float dt = a.state->dt_f32;
    const bool ga = a.ga_mode == 1 || a.ga_mode == 2;
    const bool drain = a.ga_mode == 1 || a.ga_mode == 3;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < a.nslots;
         k += (int64_t)gridDim.x * blockDim.x) {
        if (!(a.flags[k] & GSW_SLOT_ACTIVE)) continue;
        float h = a.q0[k];
        if (h <= 0.0f) continue;
        float scale = 1.0f;
        if (ga) {
            const int c = a.ga_cls[k];
            const float K = a.Ks_t[c];
            if (K > 0.0f) {
                const float KsDt = K * dt;
                const float head = a.psi_t[c] + h;
                const float F0 = a.F[k];
                const float A = F0 + KsDt;
                const float disc = A * A + 4.0f * KsDt * head * a.dth_t[c];
                const float F1 = 0.5f * (A + sqrtf(fmaxf(disc, 0.0f)));
                const float dF_raw = F1 - F0;
                float dF = (dF_raw > 0.0f) ? dF_raw : 0.0f;
                if (dF > h) dF = h;
                const float room = (a.Fmax ? a.Fmax[k] : 3.0e38f) - F0;
                if (dF > room) dF = (room > 0.0f) ? room : 0.0f;
                const float hn = h - dF;
                if (drain) {
                    scale = scale * (hn / h);
                } else {
                    scale = hn / h;
                }
                h = hn;
                a.F[k] = F0 + dF;
            } else if (!drain) {
                continue;
            }
        }
        if (drain) {
            const float it = a.inv_tau[k];
            if (it > 0.0f && h > 0.0f) {
                const float decay = __expf(-dt * it);
                scale = scale * decay;
                h = h * decay;
            } else if (!ga) {
                continue;
            }
        }
        a.q0[k] = h;
        a.q1[k] = a.q1[k] * scale;
        a.q2[k] = a.q2[k] * scale;
    }
}

// Stage clamp, stage_clamp_flat (:422-437), then the karst drain cap, drain_cap (:268-283).
__global__ void flat_clamp_kernel(GswFlatForcingArgs a, bool cap) {
    if (a.state->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = cap ? a.dr_n : a.cl_n;
    if (i >= n) return;
    const int64_t k = cap ? a.dr_slots[i] : a.cl_slots[i];
    if (k < 0) return;
    const float h = a.q0[k];
    const float ht = cap ? a.dr_htgt[i] : a.cl_hmax[i];
    if (h > ht) {
        const float r = cap ? ((h > 1e-12f) ? ht / h : 0.0f) : ht / h;
        a.q0[k] = ht;
        a.q1[k] = a.q1[k] * r;
        a.q2[k] = a.q2[k] * r;
    }
}

}  // namespace gsw

using namespace gsw;

extern "C" int gsw_inflow_apply(const GswInflowArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n <= 0) return GSW_OK;
    if (!a->inlet_off || !a->q0 || !a->q1 || !a->q2 || !a->bed || !a->t_knots || !a->q_knots ||
        a->n_knots < 1 || !a->state || a->ngh < 1)
        return set_error(GSW_ERR_INVALID, "inflow: null pointer or empty hydrograph");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32) inflow_kernel<float><<<1, 256, 0, s>>>(*a);
    else if (a->dtype == GSW_F64) inflow_kernel<double><<<1, 256, 0, s>>>(*a);
    else return set_error(GSW_ERR_INVALID, "inflow: bad dtype");
    return check_launch("inflow");
}

extern "C" int gsw_inflow_depth_sum(const GswInflowArgs* a, double* out, void* stream) {
    GSW_CHECK_ABI(a);
    if (!out || !a->q0 || (a->n > 0 && !a->inlet_off) || a->n < 0)
        return set_error(GSW_ERR_INVALID, "inflow depth sum: null pointer or negative count");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32) inflow_depth_sum_kernel<float><<<1, 32, 0, s>>>(*a, out);
    else if (a->dtype == GSW_F64) inflow_depth_sum_kernel<double><<<1, 32, 0, s>>>(*a, out);
    else return set_error(GSW_ERR_INVALID, "inflow depth sum: bad dtype");
    return check_launch("inflow_depth_sum");
}

extern "C" int gsw_flat_inflow_depth_sum(const GswFlatInflowArgs* a, double* out, void* stream) {
    GSW_CHECK_ABI(a);
    if (!out || !a->q0 || (a->n > 0 && !a->nbr_slot) || a->n < 0)
        return set_error(GSW_ERR_INVALID, "flat inflow depth sum: null pointer or negative count");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32) flat_inflow_depth_sum_kernel<float><<<1, 32, 0, s>>>(*a, out);
    else if (a->dtype == GSW_F64) flat_inflow_depth_sum_kernel<double><<<1, 32, 0, s>>>(*a, out);
    else return set_error(GSW_ERR_INVALID, "flat inflow depth sum: bad dtype");
    return check_launch("flat_inflow_depth_sum");
}

extern "C" int gsw_flat_inflow_apply(const GswFlatInflowArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n <= 0) return GSW_OK;
    if (!a->ghost_slot || !a->nbr_slot || !a->q0 || !a->q1 || !a->q2 || !a->bed || !a->t_knots ||
        !a->q_knots || a->n_knots < 1 || !a->state || !(a->ds > 0.0))
        return set_error(GSW_ERR_INVALID, "flat inflow: null pointer, empty hydrograph or ds <= 0");
    cudaStream_t s = (cudaStream_t)stream;
    if (a->dtype == GSW_F32) flat_inflow_kernel<float><<<1, 256, 0, s>>>(*a);
    else if (a->dtype == GSW_F64) flat_inflow_kernel<double><<<1, 256, 0, s>>>(*a);
    else return set_error(GSW_ERR_INVALID, "flat inflow: bad dtype");
    return check_launch("flat_inflow");
}

extern "C" int gsw_flat_ring_stage(const GswFlatRingArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (a->n <= 0) return GSW_OK;
    if (!a->q0 || !a->q1 || !a->q2 || !a->slots || !a->bed || !a->wg || !a->t_common || !a->stage_all ||
        !a->state || a->NG < 1 || a->n_t < 2)
        return set_error(GSW_ERR_INVALID, "ring stage: null pointer, NG < 1 or fewer than 2 stage times");
    cudaStream_t s = (cudaStream_t)stream;
    const int grid = (a->n + 255) / 256;
    if (a->dtype == GSW_F32) flat_ring_kernel<float><<<grid, 256, 0, s>>>(*a);
    else if (a->dtype == GSW_F64) flat_ring_kernel<double><<<grid, 256, 0, s>>>(*a);
    else return set_error(GSW_ERR_INVALID, "ring stage: bad dtype");
    return check_launch("flat_ring");
}

extern "C" int gsw_flat_forcings(const GswFlatForcingArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (!a->q0 || !a->q1 || !a->q2 || !a->flags || !a->state || a->nslots < 0)
        return set_error(GSW_ERR_INVALID, "flat forcings: null state or flags");
    cudaStream_t s = (cudaStream_t)stream;
    const int grid_all = (int)std::max<int64_t>(1, std::min<int64_t>(sm_count() * 8, (a->nslots + 255) / 256));
    if (a->phase == 0) {
        if (a->infil_tab) {
            flat_infiltrate_kernel<<<grid_all, 256, 0, s>>>(*a);
            if (int rc = check_launch("flat_infiltrate")) return rc;
        }
        if (a->sp_n > 0) {
            if (!a->sp_slots || !a->sp_keep || !a->sp_amb) return set_error(GSW_ERR_INVALID, "sponge: null arrays");
            flat_sponge_kernel<<<(a->sp_n + 255) / 256, 256, 0, s>>>(*a);
            if (int rc = check_launch("flat_sponge")) return rc;
        }
        return GSW_OK;
    }
    if (a->phase != 1) return set_error(GSW_ERR_INVALID, "flat forcings: phase must be 0 or 1");
    if (a->ga_mode != 0) {
        if (a->ga_mode < 0 || a->ga_mode > 3) return set_error(GSW_ERR_INVALID, "Green-Ampt: bad mode");
        if ((a->ga_mode != 3 && (!a->ga_cls || !a->Ks_t || !a->psi_t || !a->dth_t || !a->F)) ||
            (a->ga_mode != 2 && !a->inv_tau))
            return set_error(GSW_ERR_INVALID, "Green-Ampt / drain: null arrays");
        flat_ga_drain_kernel<<<grid_all, 256, 0, s>>>(*a);
        if (int rc = check_launch("flat_ga_drain")) return rc;
    }
    if (a->cl_n > 0) {
        if (!a->cl_slots || !a->cl_hmax) return set_error(GSW_ERR_INVALID, "stage clamp: null arrays");
        flat_clamp_kernel<<<(a->cl_n + 63) / 64, 64, 0, s>>>(*a, false);
        if (int rc = check_launch("flat_clamp")) return rc;
    }
    if (a->dr_n > 0) {
        if (!a->dr_slots || !a->dr_htgt) return set_error(GSW_ERR_INVALID, "drain cap: null arrays");
        flat_clamp_kernel<<<(a->dr_n + 255) / 256, 256, 0, s>>>(*a, true);
        if (int rc = check_launch("flat_drain_cap")) return rc;
    }
    return GSW_OK;
}
