// gsw_fast.h -- launchers of the fast-arithmetic compilation (gsw_fast.cu), for the C
// entry points of gsw_dense.cu, gsw_flat.cu and gsw_ensemble.cu. Library-internal.
#pragma once
#include <cuda_runtime.h>
#include "../../include/gsw.h"

int gsw_fast_dense_launch(const GswDenseArgs* a, bool step, cudaStream_t s);
int gsw_fast_flat_launch(const GswFlatArgs* a, bool step, cudaStream_t s);
int gsw_fast_ensemble_launch(const GswEnsembleArgs* a, cudaStream_t s);
