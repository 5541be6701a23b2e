// gsw_flat.cu -- the fused step on the compressed (flat) mesh (gsw_flat_march.cuh),
// its residual and its standalone wave speed, and their C ABI.
//
// Semantics of the reference's flat step (geoswe/compressed_rhs.py:673-865, 990-1118):
// stored cells that are not active (the two-cell ring) keep their state; active cells
// take rain, Euler, the wet/dry floor and Manning from the class table (always, as
// compressed_solver.py:2862-2879 gives a frictionless run the table [0]); the new
// state's wave speed uses the flat norm and floors.
#include "gsw_flat_march.cuh"
#include "gsw_fast.h"

namespace gsw {

template <typename T>
__global__ void __launch_bounds__(256) flat_lammax_kernel(FlatK<T> p, int64_t nslots, unsigned long long* out) {
    unsigned long long lam = 0ull;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (!(p.m.flags[s] & GSW_SLOT_ACTIVE)) continue;
        const unsigned long long lb = lam_flat_bits(p.m.q0[s], p.m.q1[s], p.m.q2[s], p.ph.g, p.ph.h_min,
                                                    p.ph.h_min_cfl, p.ph.linf != 0);
        lam = lb > lam ? lb : lam;
    }
    block_max_to(lam, out);
}

}  // namespace gsw

using namespace gsw;

static int check_dtype(const GswFlatArgs* a) {
    if (a->dtype != GSW_F32 && a->dtype != GSW_F64) return set_error(GSW_ERR_INVALID, "flat: dtype must be F32 or F64");
    if (a->arith != GSW_ARITH_EXACT && a->arith != GSW_ARITH_FAST && a->arith != GSW_ARITH_PORTABLE)
        return set_error(GSW_ERR_INVALID, "flat: bad arith %d", a->arith);
    if (a->arith == GSW_ARITH_FAST && a->dtype != GSW_F32)
        return set_error(GSW_ERR_INVALID, "flat: fast arithmetic is binary32 only");
    return GSW_OK;
}

extern "C" int gsw_flat_step(const GswFlatArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_dtype(a)) return rc;
    if (a->arith == GSW_ARITH_FAST) return gsw_fast_flat_launch(a, true, (cudaStream_t)stream);
    return a->dtype == GSW_F32 ? launch_flat<float, true>(a, (cudaStream_t)stream)
                               : launch_flat<double, true>(a, (cudaStream_t)stream);
}

extern "C" int gsw_flat_rhs(const GswFlatArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_dtype(a)) return rc;
    if (!a->qn0 || !a->qn1 || !a->qn2) return set_error(GSW_ERR_INVALID, "flat rhs: null output");
    const size_t es = a->dtype == GSW_F32 ? sizeof(float) : sizeof(double);
    const size_t n = (size_t)(a->n_bricks + 1) * a->brick_h * GSW_BRICK_PITCH * es;
    for (void* o : {a->qn0, a->qn1, a->qn2})
        if (cudaMemsetAsync(o, 0, n, (cudaStream_t)stream) != cudaSuccess)
            return set_error(GSW_ERR_CUDA, "flat rhs: memset failed");
    if (a->arith == GSW_ARITH_FAST) return gsw_fast_flat_launch(a, false, (cudaStream_t)stream);
    return a->dtype == GSW_F32 ? launch_flat<float, false>(a, (cudaStream_t)stream)
                               : launch_flat<double, false>(a, (cudaStream_t)stream);
}

template <typename T>
static int launch_flat_lammax(const GswFlatArgs* a, uint64_t* lam_bits, cudaStream_t s) {
    FlatK<T> k;
    int rc = fill_flat<T>(a, k, false);
    if (rc) return rc;
    const int64_t nslots = (k.m.nb + 1) * (int64_t)k.m.bh * GSW_BRICK_PITCH;
    const int grid = (int)std::min<int64_t>(sm_count() * 8, (nslots + 255) / 256);
    flat_lammax_kernel<T><<<std::max(grid, 1), 256, 0, s>>>(k, nslots, (unsigned long long*)lam_bits);
    return check_launch("flat_lammax");
}

extern "C" int gsw_flat_lammax(const GswFlatArgs* a, uint64_t* lam_bits, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_dtype(a)) return rc;
    if (!lam_bits) return set_error(GSW_ERR_INVALID, "flat lammax: null output");
    return a->dtype == GSW_F32 ? launch_flat_lammax<float>(a, lam_bits, (cudaStream_t)stream)
                               : launch_flat_lammax<double>(a, lam_bits, (cudaStream_t)stream);
}
