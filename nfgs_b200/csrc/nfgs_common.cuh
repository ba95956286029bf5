// Shared definitions for the NFGS B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#define NFGS_HD __host__ __device__ __forceinline__

// Accumulation type: FP32 storage accumulates in FP32 inside stencils
// (the reference FP32 path does the same), FP64 storage in FP64.
template <typename T> struct AccT { using type = T; };

// Number of reduction values per block of the stencil pass.
#define NFGS_NRED 6
// 0 sigma numerator, 1 sigma denominator, 2 sum|divB|, 3 sum|B|,
// 4 sum|B|^2, 5 sum S_B^2

struct Geo {
    int nx, ny, nz;
    long long P;   // nx*ny
    long long V;   // nx*ny*nz
    double dx, dy, dz;
};

// Device-side iteration control.  Written by the single-thread control
// kernel, read by every per-iteration kernel (early exit once stopped).
struct DevCtl {
    int n;              // index of the accepted state (0 = initial)
    int stopped;        // stop decided (no further iteration work)
    int stop_reason;
    int cur, best, cand;  // state buffer indices (0..2)
    int rollback_now;     // the last candidate was rejected
    int not_rollback;     // 1 unless a rejected candidate needs re-sourcing
    int stall, flat, streak, rollbacks;
    int final_iter;
    int best_iter;
    int n_hist;           // rows written
    int policy_error;     // source zero-mode policy violation
    int have_last_imp;
    double best_sigma, prev_sigma, mu_cur, last_imp;
    double prev_energy;
    double cur_sigma;
    double sumsb2;        // sum S_B^2 of the sources awaiting the next solve
    double zero_ratio_last;
    // parameters
    int max_iter, patience, flat_required, use_imp, adaptive, growth_streak, max_rollbacks;
    int source_policy;
    double tol, eps, mu_min, mu_max, mu_backoff, mu_growth, div_factor, src_tol;
    double sigma0, divb0, e0;
};

// Iteration result for history (one row per iterate step).
#define NFGS_HCOLS 8

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block reduction of NV doubles; result valid in thread 0.  `sh` holds
// NV * 32 doubles.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* sh) {
    const int lane = threadIdx.x & 31;
    const int tid = threadIdx.x + threadIdx.y * blockDim.x;
    const int warp = tid >> 5;
    const int nwarp = (blockDim.x * blockDim.y + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) v[q] = warp_sum(v[q]);
    if ((tid & 31) == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q * 32 + warp] = v[q];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) {
            double t = (lane < nwarp) ? sh[q * 32 + lane] : 0.0;
            v[q] = warp_sum(t);
        }
    }
    (void)lane;
}
