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
        const T sum = pairwise_sum<T>(q0, a.inlet_off, 0, a.n);
        s_sum = (double)sum;
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
        const T sum = pairwise_sum<T>(q0, a.nbr_slot, 0, a.n);
        s_sum = (double)sum;
        s_wet = s_sum > 0.0;
        if (!s_wet) {
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
