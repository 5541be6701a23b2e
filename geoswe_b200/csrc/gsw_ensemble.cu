// gsw_ensemble.cu -- a batch of compressed meshes advanced by one persistent kernel per
// step (gsw_ensemble_march.cuh): the step, the initial wave speed and dt rule, and
// their C ABI.
#include "gsw_ensemble_march.cuh"
#include "gsw_fast.h"
#include <mutex>

namespace gsw {

__global__ void ensemble_finalize_kernel(GswEnsembleArgs a) {
    __shared__ int s_open;
    if (threadIdx.x == 0) s_open = 0;
    __syncthreads();
    for (int mi = threadIdx.x; mi < a.n_members; mi += blockDim.x) {
        GswLoopState* st = a.states + mi;
        dt_finalize_one(a.members[mi].dt, st, st->lam_bits);
        if (!st->done) atomicAdd(&s_open, 1);
    }
    __syncthreads();
    if (a.run != nullptr) build_run_list(a, threadIdx.x, blockDim.x);
    if (threadIdx.x == 0) {
        if (a.scratch != nullptr) {   // NULL: the static-scratch step keeps its own words at zero
            a.scratch[0] = 0u;
            a.scratch[1] = 0u;
        }
        *a.all_done = (s_open == 0) ? 1 : 0;
    }
}

__global__ void __launch_bounds__(256) ensemble_lammax_kernel(GswEnsembleArgs a) {
    const int64_t BS = (int64_t)a.brick_h * GSW_BRICK_PITCH;
    const int64_t nslots = a.n_bricks * BS;
    for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nslots;
         s += (int64_t)gridDim.x * blockDim.x) {
        if (!(a.flags[s] & GSW_SLOT_ACTIVE)) continue;
        const int mi = a.brick_member[s / BS];
        const GswMember& mb = a.members[mi];
        const unsigned long long lb = lam_flat_bits(a.q0[s], a.q1[s], a.q2[s], mb.g, mb.h_min, mb.h_min_cfl,
                                                    mb.linf != 0);
        if (lb != 0ull) atomicMax((unsigned long long*)&a.states[mi].lam_bits, lb);
    }
}

}  // namespace gsw

using namespace gsw;

// need_scratch: the caller-scratch step needs a->scratch; the wave speed and the dt rule
// read none (finalize clears it when given), and the static-scratch step brings its own.
static int check_ens(const GswEnsembleArgs* a, bool need_scratch) {
    if (a->n_members <= 0 || a->n_members > 65536 || a->brick_h < 2 || a->n_bricks < 0)
        return set_error(GSW_ERR_INVALID, "ensemble: bad sizes");
    if (!a->brick_ij || !a->brick_nbr || !a->brick_member || !a->flags || !a->q0 || !a->q1 || !a->q2 ||
        !a->bed || !a->members || !a->states || !a->all_done)
        return set_error(GSW_ERR_INVALID, "ensemble: null pointer");
    if (need_scratch && !a->scratch) return set_error(GSW_ERR_INVALID, "ensemble step: scratch is NULL");
    if (a->run != nullptr && a->member_brick_off == nullptr)
        return set_error(GSW_ERR_INVALID, "ensemble: a running-member list needs member_brick_off");
    return GSW_OK;
}

extern "C" int gsw_ensemble_lammax(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a, false);
    if (rc) return rc;
    const int64_t nslots = a->n_bricks * (int64_t)a->brick_h * GSW_BRICK_PITCH;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(sm_count() * 8, (nslots + 255) / 256));
    ensemble_lammax_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("ensemble_lammax");
}

extern "C" int gsw_ensemble_finalize(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a, false);
    if (rc) return rc;
    ensemble_finalize_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(*a);
    return check_launch("ensemble_finalize");
}

extern "C" int gsw_ensemble_step(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    int rc = check_ens(a, true);
    if (rc) return rc;
    if (!a->qn0 || !a->qn1 || !a->qn2) return set_error(GSW_ERR_INVALID, "ensemble step: null output");
    if (a->arith == GSW_ARITH_FAST) return gsw_fast_ensemble_launch(a, (cudaStream_t)stream);
    if (a->arith != GSW_ARITH_EXACT && a->arith != GSW_ARITH_PORTABLE)
        return set_error(GSW_ERR_INVALID, "ensemble step: bad arith %d", a->arith);
    return launch_ensemble_step(a, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// gsw_ensemble_step_static: the same launch with the ticket counter in library memory.
static __device__ __align__(256) unsigned int g_ens_static_scratch[GSW_ENS_STATIC_SCRATCH_WORDS];
namespace {
constexpr int kMaxDevices = 64;
std::mutex g_static_mu;
unsigned int* g_static_ptr[kMaxDevices] = {};
}  // namespace

extern "C" int gsw_ensemble_step_static(const GswEnsembleArgs* a, void* stream) {
    GSW_CHECK_ABI(a);
    if (GSW_ENS_SCRATCH_WORDS > GSW_ENS_STATIC_SCRATCH_WORDS)
        return set_error(GSW_ERR_RANGE, "ensemble step (static scratch): needs %d words, the static array "
                         "holds %d", GSW_ENS_SCRATCH_WORDS, GSW_ENS_STATIC_SCRATCH_WORDS);
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): no device");
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(GSW_ERR_RANGE, "ensemble step (static scratch): device %d >= %d", dev, kMaxDevices);
    unsigned int* ptr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (g_static_ptr[dev] == nullptr) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_ens_static_scratch);
            if (e != cudaSuccess || p == nullptr)
                return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): cudaGetSymbolAddress: %s",
                                 cudaGetErrorString(e));
            e = cudaMemsetAsync(p, 0, sizeof(g_ens_static_scratch), (cudaStream_t)stream);
            if (e != cudaSuccess)
                return set_error(GSW_ERR_CUDA, "ensemble step (static scratch): clearing the ticket: %s",
                                 cudaGetErrorString(e));
            g_static_ptr[dev] = (unsigned int*)p;
        }
        ptr = g_static_ptr[dev];
    }
    GswEnsembleArgs b = *a;
    b.scratch = ptr;
    const int rc = gsw_ensemble_step(&b, stream);
    // a refused or failed launch must not leave a ticket behind for the next call
    if (rc != GSW_OK) (void)cudaMemsetAsync(ptr, 0, GSW_ENS_SCRATCH_WORDS * sizeof(unsigned int), (cudaStream_t)stream);
    return rc;
}
