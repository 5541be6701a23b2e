// gsw_fast.cu -- the binary32 step kernels (dense march, flat march, ensemble step)
// compiled a second time with fast arithmetic: GSW_FAST_ARITH selects the approximate
// square root and division of gsw_core.cuh, and this file alone is compiled with FMA
// contraction and flush-to-zero (geoswe_b200/build.py). Every name of namespace gsw is
// renamed gsw_fast here, so these kernels and their inline helpers never merge with
// the exact compilation's.
//
// Fast results are not bit-identical to the reference's; the tests hold them to a
// depth tolerance against the exact step and to the exact step's error against fp64.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdarg.h>
#include <stdio.h>
#include <algorithm>
#include "gsw_fast.h"

#define GSW_FAST_ARITH 1
#define gsw gsw_fast
#include "gsw_dense_march.cuh"
#include "gsw_flat_march.cuh"
#include "gsw_ensemble_march.cuh"
#undef gsw

int gsw_fast_dense_launch(const GswDenseArgs* a, bool step, cudaStream_t s) {
    return step ? gsw_fast::launch_march<float, true>(a, s) : gsw_fast::launch_march<float, false>(a, s);
}

int gsw_fast_flat_launch(const GswFlatArgs* a, bool step, cudaStream_t s) {
    return step ? gsw_fast::launch_flat<float, true>(a, s) : gsw_fast::launch_flat<float, false>(a, s);
}

int gsw_fast_ensemble_launch(const GswEnsembleArgs* a, cudaStream_t s) {
    return gsw_fast::launch_ensemble_step(a, s);
}
