// gsw_common.cuh -- shared plumbing of libgsw: error state, launch checks, reductions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <algorithm>
#include "../../include/gsw.h"
#include "gsw_core.cuh"

namespace gsw {

// Thread-local message behind gsw_last_error(); defined in gsw_loop.cu.
int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);
int sm_count();
void count_launch(int n = 1);

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

}  // namespace gsw

#define GSW_CHECK_ABI(a)                                                                     \
    do {                                                                                     \
        if ((a) == nullptr) return gsw::set_error(GSW_ERR_INVALID, "null argument struct");  \
        if ((a)->abi_version != GSW_ABI_VERSION)                                             \
            return gsw::set_error(GSW_ERR_ABI, "abi_version %u, library is %u",              \
                                  (unsigned)(a)->abi_version, (unsigned)GSW_ABI_VERSION);    \
    } while (0)
