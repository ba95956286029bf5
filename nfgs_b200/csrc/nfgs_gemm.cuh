// Strided, batched GEMM used for the per-axis DCT-I / DST-I contractions
// (SIMT path: FP64 storage and the boundary set-up).
//
//   C[b](r, c) = sum_m A[b](r, m) * B[b](m, c)
//
// Element (r, m) of A lives at A + b*a_bs + r*a_rs + m*a_cs, and likewise
// for B and C.  A transform along x multiplies data rows by a transposed
// transform matrix from the right; a transform along y multiplies each
// plane by the transform matrix from the left (nfgs_solver.py:1019-1081
// define the transforms as mirrored FFTs; here they are the same linear
// maps as dense matrices).
#pragma once
#include "nfgs_common.cuh"

struct GemmArgs {
    const void* A; long long a_rs, a_cs, a_bs;
    const void* B; long long b_rs, b_cs, b_bs;
    void* C;       long long c_rs, c_cs, c_bs;
    int M, N, K, batch;
    // Optional output indirection: C = c_table[*c_sel] + (long long)C
    // (C then holds a byte offset).  Used to write into the state buffer
    // chosen on the device.
    void* const* c_table;
    const int* c_sel;
    const DevCtl* ctl;  // when non-null, exit once ctl->stopped
};

#define GEMM_BM 64
#define GEMM_BN 64
#define GEMM_BK 16

template <typename T>
__global__ void __launch_bounds__(256) gemm_strided_kernel(GemmArgs g) {
    if (g.ctl != nullptr && g.ctl->stopped) return;
    __shared__ T As[GEMM_BK][GEMM_BM + 1];
    __shared__ T Bs[GEMM_BK][GEMM_BN + 1];
    const int b = blockIdx.z;
    const int r0 = blockIdx.y * GEMM_BM;
    const int c0 = blockIdx.x * GEMM_BN;
    const T* A = (const T*)g.A + (long long)b * g.a_bs;
    const T* Bm = (const T*)g.B + (long long)b * g.b_bs;
    const int tid = threadIdx.x;
    const int tr = tid / 16;  // 0..15 -> rows tr*4..
    const int tc = tid % 16;  // 0..15 -> cols tc*4..
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);

    const bool a_kfast = (g.a_cs == 1);
    const bool b_nfast = (g.b_cs == 1);
    for (int k0 = 0; k0 < g.K; k0 += GEMM_BK) {
        // A tile: BM x BK = 1024 elements, 4 per thread
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int e = tid + q * 256;
            int rr, kk;
            if (a_kfast) { rr = e / GEMM_BK; kk = e % GEMM_BK; }
            else         { kk = e / GEMM_BM; rr = e % GEMM_BM; }
            int r = r0 + rr, k = k0 + kk;
            T v = T(0);
            if (r < g.M && k < g.K) v = A[(long long)r * g.a_rs + (long long)k * g.a_cs];
            As[kk][rr] = v;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int e = tid + q * 256;
            int kk, cc;
            if (b_nfast) { kk = e / GEMM_BN; cc = e % GEMM_BN; }
            else         { cc = e / GEMM_BK; kk = e % GEMM_BK; }
            int k = k0 + kk, c = c0 + cc;
            T v = T(0);
            if (k < g.K && c < g.N) v = Bm[(long long)k * g.b_rs + (long long)c * g.b_cs];
            Bs[kk][cc] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GEMM_BK; ++kk) {
            T a[4], bb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tr * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][tc + j * 16];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], bb[j], acc[i][j]);
        }
        __syncthreads();
    }
    char* cbase;
    if (g.c_table != nullptr) cbase = (char*)g.c_table[*g.c_sel] + (long long)(intptr_t)g.C;
    else cbase = (char*)g.C;
    T* C = (T*)cbase + (long long)b * g.c_bs;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int r = r0 + tr * 4 + i;
        if (r >= g.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            int c = c0 + tc + j * 16;
            if (c < g.N) C[(long long)r * g.c_rs + (long long)c * g.c_cs] = acc[i][j];
        }
    }
}

// Small problems (a few planes: the boundary set-up's 2-D transforms) would
// occupy a few dozen 64 x 64 tiles; 16 x 16 tiles with one output per thread
// spread them over the SMs.
template <typename T>
__global__ void __launch_bounds__(256) gemm_small_kernel(GemmArgs g) {
    if (g.ctl != nullptr && g.ctl->stopped) return;
    __shared__ T As[16][17];
    __shared__ T Bs[16][17];
    const int b = blockIdx.z;
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    const int r = blockIdx.y * 16 + tr, c = blockIdx.x * 16 + tc;
    const T* A = (const T*)g.A + (long long)b * g.a_bs;
    const T* Bm = (const T*)g.B + (long long)b * g.b_bs;
    T acc = T(0);
    for (int k0 = 0; k0 < g.K; k0 += 16) {
        // A tile rows r0.., columns k0..: thread (tr, tc) loads A(r0 + tr, k0 + tc)
        const int ar = blockIdx.y * 16 + tr, ak = k0 + tc;
        As[tr][tc] = (ar < g.M && ak < g.K) ? A[(long long)ar * g.a_rs + (long long)ak * g.a_cs] : T(0);
        const int bk = k0 + tr, bc = blockIdx.x * 16 + tc;
        Bs[tr][tc] = (bk < g.K && bc < g.N) ? Bm[(long long)bk * g.b_rs + (long long)bc * g.b_cs] : T(0);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) acc = fma(As[tr][kk], Bs[kk][tc], acc);
        __syncthreads();
    }
    if (r >= g.M || c >= g.N) return;
    char* cbase;
    if (g.c_table != nullptr) cbase = (char*)g.c_table[*g.c_sel] + (long long)(intptr_t)g.C;
    else cbase = (char*)g.C;
    T* C = (T*)cbase + (long long)b * g.c_bs;
    C[(long long)r * g.c_rs + (long long)c * g.c_cs] = acc;
}

template <typename T>
static inline cudaError_t launch_gemm(const GemmArgs& g, cudaStream_t s) {
    if (g.M <= 0 || g.N <= 0 || g.batch <= 0) return cudaSuccess;
    const long long big_tiles =
        (long long)((g.N + GEMM_BN - 1) / GEMM_BN) * ((g.M + GEMM_BM - 1) / GEMM_BM) * g.batch;
    if (big_tiles < 148 && g.batch <= 65535) {
        dim3 grid((g.N + 15) / 16, (g.M + 15) / 16, g.batch);
        gemm_small_kernel<T><<<grid, 256, 0, s>>>(g);
        return cudaGetLastError();
    }
    dim3 grid((g.N + GEMM_BN - 1) / GEMM_BN, (g.M + GEMM_BM - 1) / GEMM_BM, g.batch);
    gemm_strided_kernel<T><<<grid, 256, 0, s>>>(g);
    return cudaGetLastError();
}
