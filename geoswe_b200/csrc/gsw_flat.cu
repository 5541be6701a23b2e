// gsw_flat.cu -- the fused step on the compressed (flat) mesh, brick storage.
//
// One warp per brick of 30 x brick_h cells, the same column march as the dense kernel
// (gsw_dense.cu): lanes 1..30 are the brick's columns, lane 0 / lane 31 read the edge
// columns of the left / right brick, and the two rows above and below come from the
// bricks above and below. Every face is computed once from the shared core
// (gsw_core.cuh), so active-cell residuals are bit-identical to the dense kernel's.
//
// Semantics of the reference's flat step (geoswe/compressed_rhs.py:673-865, 990-1118):
// stored cells that are not active (the two-cell ring) keep their state; active cells
// take rain, Euler, the wet/dry floor and Manning from the class table (always, as
// compressed_solver.py:2862-2879 gives a frictionless run the table [0]); the new
// state's wave speed uses the flat norm and floors.
#include "gsw_flat_brick.cuh"

namespace gsw {

template <typename T, bool STEP, int MINB>
__global__ void __launch_bounds__(256, MINB) flat_march_kernel(FlatK<T> p) {
    if (STEP && p.st->done) return;
    const int64_t bidx = (int64_t)blockIdx.x * blockDim.y + threadIdx.y;
    unsigned long long lam_local = 0ull;
    T dt = (T)0, rate = (T)0;
    const T* frame = nullptr;
    if (STEP) {
        dt = sizeof(T) == 4 ? (T)p.st->dt_f32 : (T)p.st->dt;
        if (p.ph.rain_kind == GSW_RAIN_UNIFORM) rate = p.ph.rain[p.st->rain_idx];
        if (p.ph.rain_kind == GSW_RAIN_GRIDDED) frame = p.ph.rain + (int64_t)p.st->rain_idx * p.ph.nx * p.ph.ny;
        if (p.ph.rain_kind == GSW_RAIN_LOOKUP) frame = p.ph.rain + (int64_t)p.st->rain_idx * p.ph.ncol;
    }
    if (bidx < p.m.nb) lam_local = flat_brick<T, STEP>(p.m, p.ph, bidx, dt, rate, frame);
    if (STEP && p.lam != nullptr) block_max_to(lam_local, p.lam);
}

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

template <typename T>
static int fill_flat(const GswFlatArgs* a, FlatK<T>& k, bool step) {
    if (a->brick_h < 2 || a->n_bricks < 0 || !a->brick_ij || !a->brick_nbr || !a->flags)
        return set_error(GSW_ERR_INVALID, "flat: bad brick tables (brick_h >= 2)");
    if (!a->q0 || !a->q1 || !a->q2 || !a->bed) return set_error(GSW_ERR_INVALID, "flat: null state/bed");
    FlatMesh<T>& m = k.m;
    m.q0 = (const T*)a->q0; m.q1 = (const T*)a->q1; m.q2 = (const T*)a->q2;
    m.o0 = (T*)a->qn0; m.o1 = (T*)a->qn1; m.o2 = (T*)a->qn2;
    m.b = (const T*)a->bed; m.flags = a->flags; m.ncls = a->n_cls; m.max_h = (T*)a->max_h;
    m.bij = a->brick_ij; m.bnbr = a->brick_nbr; m.nb = a->n_bricks; m.bh = a->brick_h;
    FlatPhys<T>& ph = k.ph;
    ph.inv_dx = (T)a->inv_dx; ph.inv_dy = (T)a->inv_dy;
    ph.half_dx = (T)0.5 * ((T)1 / ph.inv_dx); ph.half_dy = (T)0.5 * ((T)1 / ph.inv_dy);
    ph.g = (T)a->g; ph.h_min = (T)a->h_min; ph.h_min_cfl = (T)a->h_min_cfl; ph.vcap = (T)a->vcap;
    ph.linf = a->linf; ph.quad = a->quadratic; ph.keep_h = a->keep_h;
    ph.rain_kind = a->rain_kind; ph.rain = (const T*)a->rain; ph.ngh = a->ngh; ph.nx = a->nx; ph.ny = a->ny;
    ph.ntab = (const T*)a->n_tab;
    ph.lookup = a->rain_lookup; ph.ncol = a->rain_ncol;
    k.st = a->state; k.lam = (unsigned long long*)a->lam_target;
    if (step) {
        if (!a->state) return set_error(GSW_ERR_INVALID, "flat step: state is required");
        if (!a->n_tab || a->n_tab_len < 1) return set_error(GSW_ERR_INVALID, "flat step: n_tab is required");
        if (a->rain_kind != GSW_RAIN_NONE && !a->rain) return set_error(GSW_ERR_INVALID, "flat step: rain is NULL");
        if (a->rain_kind == GSW_RAIN_GRIDDED && (a->nx <= 0 || a->ny <= 0 || a->ngh < 0))
            return set_error(GSW_ERR_INVALID, "flat step: gridded rain needs ngh, nx, ny");
        if (a->rain_kind == GSW_RAIN_LOOKUP && (!a->rain_lookup || a->rain_ncol < 1))
            return set_error(GSW_ERR_INVALID, "flat step: lookup rain needs rain_lookup and rain_ncol >= 1");
        if (!m.o0 || !m.o1 || !m.o2) return set_error(GSW_ERR_INVALID, "flat step: null output");
    }
    return GSW_OK;
}

static int check_dtype(const GswFlatArgs* a) {
    if (a->dtype != GSW_F32 && a->dtype != GSW_F64) return set_error(GSW_ERR_INVALID, "flat: dtype must be F32 or F64");
    return GSW_OK;
}

template <typename T, bool STEP>
static int launch_flat(const GswFlatArgs* a, cudaStream_t s) {
    FlatK<T> k;
    int rc = fill_flat<T>(a, k, STEP);
    if (rc) return rc;
    if (k.m.nb == 0) return GSW_OK;
    const int W = a->warps > 0 ? a->warps : 4;
    if (W < 1 || W > 8) return set_error(GSW_ERR_INVALID, "flat: warps must be in [1, 8]");
    const int64_t blocks = (k.m.nb + W - 1) / W;
    if (blocks > 0x7fffffffLL) return set_error(GSW_ERR_INVALID, "flat: too many bricks");
    const int mb = a->min_blocks;
    if (mb != 0 && mb != 4 && mb != 5) return set_error(GSW_ERR_INVALID, "flat: min_blocks must be 0, 4 or 5");
    if (STEP && sizeof(T) == 4 && mb == 4) flat_march_kernel<T, STEP, 4><<<(unsigned)blocks, dim3(32, W), 0, s>>>(k);
    else if (STEP && sizeof(T) == 4 && mb == 5) flat_march_kernel<T, STEP, 5><<<(unsigned)blocks, dim3(32, W), 0, s>>>(k);
    else flat_march_kernel<T, STEP, 1><<<(unsigned)blocks, dim3(32, W), 0, s>>>(k);
    return check_launch("flat_march");
}

extern "C" int gsw_flat_step(const GswFlatArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (int rc = check_dtype(a)) return rc;
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
