// Evaluation metrics of a solution in one pass over a region of interest.
//
// For every cell of the region (z0..z1) x (y0..y1) x (x0..x1) of component-
// major (3, nz, ny, nx) volumes it accumulates, in FP64, the sums behind
//   * the reference-field metrics C_vec, C_CS, E'_n, E'_m, epsilon
//     (nfgs/_backend/util/metrics.py:123-178,
//      nfgs/_backend/scripts/recompute_td_referee_diagnostics.py:344-400);
//   * sigma_J on a given current, |J x B| / max(|B|, 1e-10) over |J|
//     (metrics.py:64-86, 89-120);
//   * sigma_J and |div B| on the second-order finite-difference curl and
//     divergence of the solution, taken on the full volume (central interior,
//     three-point one-sided ends; nfgs/diagnostics/common_fd2.py:21-78), so a
//     region that touches a wall uses the one-sided stencils there;
//   * counts of non-finite field and current values.
// Each block writes its partial sums; a second kernel adds them in a fixed
// order, so the result does not depend on scheduling.  Index arithmetic is
// 32-bit per axis (no division per cell); the 1/(2h) of the derivatives and
// 1/max(|b|, 1e-10) are products.  From HBM the pass reads 9 values per
// cell (6 or 3 without a reference or a current); the 18 neighbour samples
// of the derivatives come from L1/L2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace met {

constexpr int NS = 15;        // partial sums per block
constexpr int NT = 256;       // threads per block
enum {
    S_DOT = 0, S_REF2, S_SOL2, S_COS, S_ERR, S_REFN, S_ERRR, S_SJN, S_SJD, S_FDN, S_FDD, S_DIV, S_BN, S_NFB, S_NFJ
};

struct Args {
    const void* ref;   // may be null
    const void* sol;
    const void* cur;   // may be null
    int nz, ny, nx;
    int z0, y0, x0, cz, cy, cx;
    double dx, dy, dz;
};

// Second-order derivative stencil along one axis (common_fd2.py:21-37) as
// two samples at offsets s1, s2 (in elements) with integer weights:
//   d = (w0 f[c] + w1 f[c + s1] + w2 f[c + s2]) / (2 h)
//   interior      s1 = +1, s2 = -1, w = (0, 1, -1)
//   first point   s1 = +1, s2 = +2, w = (-3, 4, -1)
//   last point    s1 = -1, s2 = -2, w = (3, -4, 1)
//   n == 2        s1 = s2 = the other point, w = (-2 or 2, +-2, 0) (= (f1 - f0) / h)
//   n == 1        no samples, w = 0
// so every load of a cell is unconditional (no branch between a cell's
// loads) and the weights reproduce the reference's expressions exactly.
struct Stencil {
    int s1, s2;
    int w0, w1, w2;
};

__device__ __forceinline__ Stencil stencil_of(int idx, int n) {
    Stencil t;
    if (n == 1) { t.s1 = t.s2 = 0; t.w0 = t.w1 = t.w2 = 0; }
    else if (n == 2) {
        const int o = idx == 0 ? 1 : -1;
        t.s1 = t.s2 = o; t.w0 = -2 * o; t.w1 = 2 * o; t.w2 = 0;
    } else if (idx == 0) { t.s1 = 1; t.s2 = 2; t.w0 = -3; t.w1 = 4; t.w2 = -1; }
    else if (idx == n - 1) { t.s1 = -1; t.s2 = -2; t.w0 = 3; t.w1 = -4; t.w2 = 1; }
    else { t.s1 = 1; t.s2 = -1; t.w0 = 0; t.w1 = 1; t.w2 = -1; }
    return t;
}

__device__ __forceinline__ double apply(const Stencil& t, double f0, double f1, double f2, double i2h) {
    return ((double)t.w0 * f0 + (double)t.w1 * f1 + (double)t.w2 * f2) * i2h;
}

__device__ __forceinline__ double cross_norm(double ax, double ay, double az, double bx, double by, double bz) {
    const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    return sqrt(cx * cx + cy * cy + cz * cz);
}

__device__ __forceinline__ double warp_sum_d(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block (bx, by, bz) covers x in [x0 + 32 bx, +32) (one warp-wide row,
// coalesced) and y in [y0 + 8 by, +8) (one row per warp), and every
// gridDim.z-th plane of the region from z0 + bz.  REF / CUR: whether a
// reference field / a current is given.
template <typename T, bool REF, bool CUR>
__global__ void __launch_bounds__(NT, 2) k_metrics(Args a, double* __restrict__ part) {
    __shared__ double sh[NS][NT / 32];
    const T* __restrict__ sol = (const T*)a.sol;
    const T* __restrict__ ref = (const T*)a.ref;
    const T* __restrict__ cur = (const T*)a.cur;
    const long long P = (long long)a.ny * a.nx, V = (long long)a.nz * P;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int i = a.x0 + (int)blockIdx.x * 32 + lane;
    const int j = a.y0 + (int)blockIdx.y * (NT / 32) + warp;
    const double i2hx = 1.0 / (2.0 * a.dx), i2hy = 1.0 / (2.0 * a.dy), i2hz = 1.0 / (2.0 * a.dz);
    double s[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) s[q] = 0.0;
    if (i < a.x0 + a.cx && j < a.y0 + a.cy) {
        const Stencil sx = stencil_of(i, a.nx), sy = stencil_of(j, a.ny);
        const long long y1 = (long long)sy.s1 * a.nx, y2 = (long long)sy.s2 * a.nx;
        const T* __restrict__ bxp = sol;
        const T* __restrict__ byp = sol + V;
        const T* __restrict__ bzp = sol + 2 * V;
        for (int k = a.z0 + (int)blockIdx.z; k < a.z0 + a.cz; k += (int)gridDim.z) {
            const Stencil sz = stencil_of(k, a.nz);
            const long long z1 = (long long)sz.s1 * P, z2 = (long long)sz.s2 * P;
            const long long c = (long long)k * P + (long long)j * a.nx + i;
            // every sample of the cell, loaded together
            const double bx = (double)bxp[c], by = (double)byp[c], bz = (double)bzp[c];
            const double bx_x1 = (double)bxp[c + sx.s1], bx_x2 = (double)bxp[c + sx.s2];
            const double bx_y1 = (double)bxp[c + y1], bx_y2 = (double)bxp[c + y2];
            const double bx_z1 = (double)bxp[c + z1], bx_z2 = (double)bxp[c + z2];
            const double by_x1 = (double)byp[c + sx.s1], by_x2 = (double)byp[c + sx.s2];
            const double by_y1 = (double)byp[c + y1], by_y2 = (double)byp[c + y2];
            const double by_z1 = (double)byp[c + z1], by_z2 = (double)byp[c + z2];
            const double bz_x1 = (double)bzp[c + sx.s1], bz_x2 = (double)bzp[c + sx.s2];
            const double bz_y1 = (double)bzp[c + y1], bz_y2 = (double)bzp[c + y2];
            const double bz_z1 = (double)bzp[c + z1], bz_z2 = (double)bzp[c + z2];
            double Bx = 0, By = 0, Bz = 0, jx = 0, jy = 0, jz = 0;
            if (REF) { Bx = (double)ref[c]; By = (double)ref[V + c]; Bz = (double)ref[2 * V + c]; }
            if (CUR) { jx = (double)cur[c]; jy = (double)cur[V + c]; jz = (double)cur[2 * V + c]; }

            const double b2 = bx * bx + by * by + bz * bz;
            const double bn = sqrt(b2);
            bool finite = isfinite(bx) && isfinite(by) && isfinite(bz);
            if (REF) {
                finite = finite && isfinite(Bx) && isfinite(By) && isfinite(Bz);
                const double R2 = Bx * Bx + By * By + Bz * Bz;
                const double Bn = sqrt(R2);
                const double dot = Bx * bx + By * by + Bz * bz;
                const double ex = bx - Bx, ey = by - By, ez = bz - Bz;
                const double diff = sqrt(ex * ex + ey * ey + ez * ez);
                s[S_DOT] += dot;
                s[S_REF2] += R2;
                s[S_COS] += dot / (Bn * bn + 1.0e-12);
                s[S_ERR] += diff;
                s[S_REFN] += Bn;
                s[S_ERRR] += diff / (Bn + 1.0e-12);
            }
            s[S_SOL2] += b2;
            s[S_BN] += bn;
            if (!finite) s[S_NFB] += 1.0;
            const double ibfl = 1.0 / fmax(bn, 1.0e-10);
            if (CUR) {
                if (!(isfinite(jx) && isfinite(jy) && isfinite(jz))) s[S_NFJ] += 1.0;
                s[S_SJN] += cross_norm(jx, jy, jz, bx, by, bz) * ibfl;
                s[S_SJD] += sqrt(jx * jx + jy * jy + jz * jz);
            }
            // second-order curl and divergence of the solution (common_fd2.py:40-56)
            const double dBx_dx = apply(sx, bx, bx_x1, bx_x2, i2hx);
            const double dBx_dy = apply(sy, bx, bx_y1, bx_y2, i2hy);
            const double dBx_dz = apply(sz, bx, bx_z1, bx_z2, i2hz);
            const double dBy_dx = apply(sx, by, by_x1, by_x2, i2hx);
            const double dBy_dy = apply(sy, by, by_y1, by_y2, i2hy);
            const double dBy_dz = apply(sz, by, by_z1, by_z2, i2hz);
            const double dBz_dx = apply(sx, bz, bz_x1, bz_x2, i2hx);
            const double dBz_dy = apply(sy, bz, bz_y1, bz_y2, i2hy);
            const double dBz_dz = apply(sz, bz, bz_z1, bz_z2, i2hz);
            const double fx = dBz_dy - dBy_dz, fy = dBx_dz - dBz_dx, fz = dBy_dx - dBx_dy;
            s[S_FDN] += cross_norm(fx, fy, fz, bx, by, bz) * ibfl;
            s[S_FDD] += sqrt(fx * fx + fy * fy + fz * fz);
            s[S_DIV] += fabs(dBx_dx + dBy_dy + dBz_dz);
        }
    }
#pragma unroll
    for (int q = 0; q < NS; ++q) {
        const double v = warp_sum_d(s[q]);
        if (lane == 0) sh[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < NS) {
        double t = 0.0;
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) t += sh[threadIdx.x][w];
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        part[b * NS + threadIdx.x] = t;
    }
}

// out[q] = sum over blocks of part[b * NS + q], one warp per sum, fixed order.
__global__ void k_metrics_sum(const double* __restrict__ part, int nblocks, double* __restrict__ out) {
    const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
    if (q >= NS) return;
    double t = 0.0;
    for (int b = lane; b < nblocks; b += 32) t += part[(long long)b * NS + q];
    t = warp_sum_d(t);
    if (lane == 0) out[q] = t;
}

}  // namespace met
