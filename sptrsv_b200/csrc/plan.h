// plan.h — the solve plan: a level-ordered, solve-optimised copy of L.
//
// HBM layout (n rows, m = nnz - n off-diagonal entries), all in iorder
// sequence so that a warp's rows are contiguous:
//   ptr[n+1]    int32   off-diagonal offsets per position
//   rowid[n]    int32   original row of each position (b, x are indexed by it)
//   col[m]      int32   off-diagonal column (original index)
//   val64[m]    f64     off-diagonal values
//   val32[m]    f32     the same values rounded to FP32
//   dg64[n], dg32[n]    diagonal per position
//   inv[n]      int32   position of each original row (natural order walk)
//   ibase[n_warps+1], ivect[n_warps]  multirow warp map (analysis copy)
// Work buffers: w32a/w32b (n x nrhs f32) for the FP32 solves and residuals,
// hb/hx (n x nrhs f64) staging for the host-buffer entry point.
#pragma once

#include "sptrsv_b200.h"

struct sptrsv_plan_s {
    int device = -1;
    int n = 0, nnz_off = 0, nlevs = 0, n_warps = 0;
    int* ptr = nullptr;
    int* rowid = nullptr;
    int* col = nullptr;
    double* val64 = nullptr;
    float* val32 = nullptr;
    double* dg64 = nullptr;
    float* dg32 = nullptr;
    int* inv = nullptr;
    int* ibase = nullptr;
    int* ivect = nullptr;
    float* w32a = nullptr;
    float* w32b = nullptr;
    int cap_rhs = 0;
    double* hb = nullptr;
    double* hx = nullptr;
    int cap_host = 0;
    sptrsv_schedule_t sched{};
};
