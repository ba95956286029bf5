// Boundary set-up kernels (FP64, 2-D maps and the 3-D background).
// nfgs_solver.py:2000-2113 (boundary), 1498-1567 / 4489-4546 (bottom Jz),
// 3024-3057 (toroidal boundary), 4671-4919 (Gaussian separation).
#pragma once
#include "nfgs_common.cuh"

template <typename F>
__global__ void k_map(long long n, F f) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f(i);
}

template <typename F>
static inline cudaError_t launch_map(long long n, cudaStream_t s, F f) {
    if (n <= 0) return cudaSuccess;
    k_map<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, f);
    return cudaGetLastError();
}

// Embed (crop/pad) observed maps into the calculation grid
// (nfgs_solver.py:1593-1609), rounding to the solver storage type first.
__global__ void k_embed(const double* __restrict__ src, int src_nx, double* __restrict__ dst, int nx,
                        int fy0, int fx0, int sy0, int sx0, int cny, int cnx, int round_f32) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= cnx || j >= cny) return;
    double v = src[(long long)(sy0 + j) * src_nx + (sx0 + i)];
    if (round_f32) v = (double)(float)v;
    dst[(long long)(fy0 + j) * nx + (fx0 + i)] = v;
}

// Centred bottom Jz on a (helper) grid whose interior holds the calc maps
// at offset (by0, bx0) (nfgs_solver.py:1513-1526).
__global__ void k_jz_raw(const double* __restrict__ bx, const double* __restrict__ by, int nx, int ny, int hnx,
                         int hny, int bx0, int by0, double dx, double dy, double* __restrict__ jzh) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= hnx || j >= hny) return;
    double v = 0.0;
    if (i >= 1 && i <= hnx - 2 && j >= 1 && j <= hny - 2) {
        auto B = [&](const double* a, int jj, int ii) -> double {
            int cj = jj - by0, ci = ii - bx0;
            if (cj < 0 || cj >= ny || ci < 0 || ci >= nx) return 0.0;
            return a[(long long)cj * nx + ci];
        };
        v = (B(by, j, i + 1) - B(by, j, i - 1)) / (2.0 * dx) - (B(bx, j + 1, i) - B(bx, j - 1, i)) / (2.0 * dy);
    }
    jzh[(long long)j * hnx + i] = v;
}

// botbal cell sums (nfgs_solver.py:1531-1543): out[0] total, [1] positive,
// [2] negative parts.  Single block, deterministic order.
__global__ void k_cell_sums(const double* __restrict__ a, int nx, int ny, double* out) {
    __shared__ double sh[3 * 32];
    double v[3] = {0, 0, 0};
    for (long long q = threadIdx.x; q < (long long)nx * ny; q += blockDim.x) {
        int j = (int)(q / nx), i = (int)(q % nx);
        int cnt = 0;
        if (j >= 1 && j <= ny - 2 && i >= 2) cnt++;
        if (j >= 2 && i >= 1 && i <= nx - 2) cnt++;
        if (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2) cnt++;
        if (j >= 2 && i >= 2) cnt++;
        if (cnt == 0) continue;
        double x = a[q], w = 0.25 * cnt;
        v[0] += w * x;
        v[1] += w * (x >= 0.0 ? x : 0.0);
        v[2] += w * (x < 0.0 ? x : 0.0);
    }
    block_reduce<3>(v, sh);
    if (threadIdx.x == 0) { out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; }
}

// Scale positive/negative parts, zero the helper edges, crop the calc window.
__global__ void k_jz_finish(const double* __restrict__ jzh, int hnx, int hny, int bx0, int by0, double fp,
                            double fn, int zero_edges, double* __restrict__ jz, int nx, int ny) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= nx || j >= ny) return;
    int hi = i + bx0, hj = j + by0;
    double v = jzh[(long long)hj * hnx + hi];
    v = v >= 0.0 ? fp * v : fn * v;
    if (zero_edges && (hi == 0 || hi == hnx - 1 || hj == 0 || hj == hny - 1)) v = 0.0;
    jz[(long long)j * nx + i] = v;
}

// 3x3 binomial smoothing with reflect padding (nfgs_solver.py:1471-1483).
__global__ void k_smooth(const double* __restrict__ a, double* __restrict__ o, int nx, int ny) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (i >= nx || j >= ny) return;
    const double w[3] = {1.0, 2.0, 1.0};
    double s = 0.0;
    for (int dj = -1; dj <= 1; ++dj) {
        int jj = j + dj;
        jj = jj < 0 ? -jj : (jj >= ny ? 2 * ny - 2 - jj : jj);
        for (int di = -1; di <= 1; ++di) {
            int ii = i + di;
            ii = ii < 0 ? -ii : (ii >= nx ? 2 * nx - 2 - ii : ii);
            s += (w[dj + 1] * w[di + 1] / 16.0) * a[(long long)jj * nx + ii];
        }
    }
    o[(long long)j * nx + i] = s;
}

// FP64 reductions over n values: out[0] sum, [1] sum of squares,
// [2] sum |x|, [3] max |x|.  Single block.
__global__ void k_reduce4(const double* __restrict__ a, long long n, double* out) {
    __shared__ double sh[3 * 32];
    __shared__ double smax[32];
    double v[3] = {0, 0, 0};
    double mx = 0.0;
    for (long long q = threadIdx.x; q < n; q += blockDim.x) {
        double x = a[q];
        v[0] += x;
        v[1] += x * x;
        v[2] += fabs(x);
        mx = fmax(mx, fabs(x));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mx;
    block_reduce<3>(v, sh);
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmax(m, smax[w]);
        out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; out[3] = m;
    }
}

// Two-stage form for long arrays: block b reduces the chunk
// [b*chunk, (b+1)*chunk) in a fixed order into part[4b..4b+3]; then one block
// combines the partials in a fixed order.
__global__ void k_reduce4_part(const double* __restrict__ a, long long n, long long chunk, double* part) {
    __shared__ double sh[3 * 32];
    __shared__ double smax[32];
    const long long q0 = (long long)blockIdx.x * chunk, q1 = min(n, q0 + chunk);
    double v[3] = {0, 0, 0};
    double mx = 0.0;
    for (long long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        double x = a[q];
        v[0] += x;
        v[1] += x * x;
        v[2] += fabs(x);
        mx = fmax(mx, fabs(x));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mx;
    block_reduce<3>(v, sh);
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmax(m, smax[w]);
        part[4 * blockIdx.x] = v[0]; part[4 * blockIdx.x + 1] = v[1];
        part[4 * blockIdx.x + 2] = v[2]; part[4 * blockIdx.x + 3] = m;
    }
}

__global__ void k_reduce4_final(const double* __restrict__ part, int nb, double* out) {
    __shared__ double sh[3 * 32];
    __shared__ double smax[32];
    double v[3] = {0, 0, 0};
    double mx = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        v[0] += part[4 * b];
        v[1] += part[4 * b + 1];
        v[2] += part[4 * b + 2];
        mx = fmax(mx, part[4 * b + 3]);
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = mx;
    block_reduce<3>(v, sh);
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) m = fmax(m, smax[w]);
        out[0] = v[0]; out[1] = v[1]; out[2] = v[2]; out[3] = m;
    }
}

// 2-D derivative of a (ny, nx) map, one-sided ends
// (nfgs_solver.py:1429-1469): axis 0 -> d/dx, 1 -> d/dy.
__device__ __forceinline__ double d2d(const double* a, int nx, int ny, int j, int i, int axis, double h) {
    auto f = [&](int q) { return axis == 0 ? a[(long long)j * nx + q] : a[(long long)q * nx + i]; };
    int n = axis == 0 ? nx : ny;
    int p = axis == 0 ? i : j;
    if (p == 0) return (-3.0 * f(0) + 4.0 * f(1) - f(2)) / (2.0 * h);
    if (p == n - 1) return (3.0 * f(n - 1) - 4.0 * f(n - 2) + f(n - 3)) / (2.0 * h);
    return (f(p + 1) - f(p - 1)) / (2.0 * h);
}

__device__ __forceinline__ double lap2d(const double* a, int nx, int ny, int j, int i, double dx, double dy) {
    auto f = [&](int jj, int ii) { return a[(long long)jj * nx + ii]; };
    double l = 0.0;
    if (i >= 1 && i <= nx - 2) l += (f(j, i + 1) - 2.0 * f(j, i) + f(j, i - 1)) / (dx * dx);
    if (j >= 1 && j <= ny - 2) l += (f(j + 1, i) - 2.0 * f(j, i) + f(j - 1, i)) / (dy * dy);
    if (j == 0) l += (2.0 * f(1, i) - 2.0 * f(0, i)) / (dy * dy);
    if (j == ny - 1) l += (2.0 * f(ny - 2, i) - 2.0 * f(ny - 1, i)) / (dy * dy);
    if (i == 0) l += (2.0 * f(j, 1) - 2.0 * f(j, 0)) / (dx * dx);
    if (i == nx - 1) l += (2.0 * f(j, nx - 2) - 2.0 * f(j, nx - 1)) / (dx * dx);
    return l;
}
