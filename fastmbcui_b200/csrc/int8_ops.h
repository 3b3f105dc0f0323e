// The FP64-accurate INT8 tensor-core matvec inside the solver (int8_ops.cu):
// dispatch from the FP64 matvec launchers; the digit planes are built by
// Solver::ensure_oz.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "solver.h"

namespace mbc {

// the INT8 path is selected and its planes are built
bool use_oz(const Solver &S);
// W = K V (rows direction); V n x R, W nf x R, FP64; returns the row tiles
int oz_launch_rows(const Solver &S, int R, const double *v, double *w, const int32_t *done, cudaStream_t st);
// T = K^T W (columns direction) with the optional curvature partials p.t per
// row tile; returns the row tiles (the rows of `part`)
int oz_launch_cols(const Solver &S, int R, const double *w, double *t, const double *pdot, double *part,
                   const int32_t *done, cudaStream_t st);

}  // namespace mbc
