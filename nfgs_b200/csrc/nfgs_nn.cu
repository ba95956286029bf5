// Kernels of the learned warm start: a 3-D neural operator on a truncated
// cosine basis (lifting, spectral layers, pointwise channel mixing, GELU,
// projection), its backward pass, the masked MSE loss and the Adam update.
// There is no reference counterpart: the reference starts every solve from
// the zero-source (gs_cfcf) state, nfgs_solver.py:6613-6645.
//
// Layout: activations are channel-major (C, Nz, Ny, Nx), FP32.  Spectral
// coefficients are (C, Kz, Ky, Kx).  A spectral layer applies
//   reduce3:  a[c,kz,ky,kx] = sum_{z,y,x} Mz[kz,z] My[ky,y] Mx[kx,x] v[c,z,y,x]
//   modemix:  b[o,k] = sum_i W[k,i,o] a[i,k]
//   expand3:  u[o,z,y,x] += sum_{k} Sz[kz,z] Sy[ky,y] Sx[kx,x] b[o,k]
// as separable per-axis contractions; the backward pass uses the same two
// contraction kernels with the roles of the bases swapped.  All reductions
// are in fixed order (block partials, then a fixed-order sum), so a training
// run is bitwise repeatable.
#include "../../include/nfgs_b200.h"
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string>

namespace {

thread_local std::string g_nn_err;

int nn_fail(int code, const std::string& msg) {
    g_nn_err = msg;
    return code;
}

#define NNCK(call)                                                                      \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess) return nn_fail(NFGS_ECUDA, std::string(#call) + ": " +   \
                                              cudaGetErrorString(e_));                  \
    } while (0)

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// pointwise channel mixing: y[o,v] (+)= sum_i W[o,i] x[i,v] + b[o]
// ---------------------------------------------------------------------------
template <int CI, int CO>
__global__ void k_pointwise(const float* __restrict__ x, const float* __restrict__ W, const float* __restrict__ b,
                            float* __restrict__ y, long long nvox, int accumulate) {
    __shared__ float sw[CI * CO];
    __shared__ float sb[CO];
    for (int q = threadIdx.x; q < CI * CO; q += blockDim.x) sw[q] = W[q];
    for (int q = threadIdx.x; q < CO; q += blockDim.x) sb[q] = b ? b[q] : 0.f;
    __syncthreads();
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    float xi[CI];
#pragma unroll
    for (int i = 0; i < CI; ++i) xi[i] = x[(long long)i * nvox + v];
#pragma unroll 4
    for (int o = 0; o < CO; ++o) {
        float acc = sb[o];
#pragma unroll
        for (int i = 0; i < CI; ++i) acc = fmaf(sw[o * CI + i], xi[i], acc);
        float* dst = y + (long long)o * nvox + v;
        *dst = accumulate ? *dst + acc : acc;
    }
}

// generic (any channel counts)
__global__ void k_pointwise_any(const float* __restrict__ x, const float* __restrict__ W, const float* __restrict__ b,
                                float* __restrict__ y, int ci, int co, long long nvox, int accumulate) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    for (int o = 0; o < co; ++o) {
        float acc = b ? b[o] : 0.f;
        for (int i = 0; i < ci; ++i) acc = fmaf(W[o * ci + i], x[(long long)i * nvox + v], acc);
        float* dst = y + (long long)o * nvox + v;
        *dst = accumulate ? *dst + acc : acc;
    }
}

// gx[i,v] (+)= sum_o W[o,i] gy[o,v]
__global__ void k_pointwise_bwd_x(const float* __restrict__ W, const float* __restrict__ gy, float* __restrict__ gx,
                                  int ci, int co, long long nvox, int accumulate) {
    const long long v = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nvox) return;
    for (int i = 0; i < ci; ++i) {
        float acc = 0.f;
        for (int o = 0; o < co; ++o) acc = fmaf(W[o * ci + i], gy[(long long)o * nvox + v], acc);
        float* dst = gx + (long long)i * nvox + v;
        *dst = accumulate ? *dst + acc : acc;
    }
}

// block partials of gW[o,i] = sum_v gy[o,v] x[i,v] and gb[o] = sum_v gy[o,v]
// over VB voxels per block: part[blk][co*ci + co]
constexpr int VB = 1024;
__global__ void k_pointwise_bwd_w(const float* __restrict__ x, const float* __restrict__ gy, float* __restrict__ part,
                                  int ci, int co, long long nvox) {
    extern __shared__ float sh[];  // 32-voxel staging of x (ci rows) and gy (co rows)
    const int tid = threadIdx.x;
    const int npair = co * ci + co;
    const long long v0 = (long long)blockIdx.x * VB;
    // each thread owns pairs p = tid, tid + blockDim ...; loop over the chunk in sub-tiles of 32 voxels
    float acc[8];
    const int per = (npair + blockDim.x - 1) / blockDim.x;  // <= 8 asserted by the host
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.f;
    float* sx = sh;            // [ci][32]
    float* sg = sh + ci * 32;  // [co][32]
    for (long long s0 = v0; s0 < v0 + VB && s0 < nvox; s0 += 32) {
        __syncthreads();
        for (int q = tid; q < (ci + co) * 32; q += blockDim.x) {
            const int ch = q / 32, l = q % 32;
            const long long v = s0 + l;
            float val = 0.f;
            if (v < nvox && v < v0 + VB) val = ch < ci ? x[(long long)ch * nvox + v] : gy[(long long)(ch - ci) * nvox + v];
            sh[q] = val;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int p = tid + q * blockDim.x;
            if (q >= per || p >= npair) break;
            float a = acc[q];
            if (p < co * ci) {
                const int o = p / ci, i = p % ci;
#pragma unroll 8
                for (int l = 0; l < 32; ++l) a = fmaf(sg[o * 32 + l], sx[i * 32 + l], a);
            } else {
                const int o = p - co * ci;
#pragma unroll 8
                for (int l = 0; l < 32; ++l) a += sg[o * 32 + l];
            }
            acc[q] = a;
        }
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int p = tid + q * blockDim.x;
        if (q < per && p < npair) part[(long long)blockIdx.x * npair + p] = acc[q];
    }
}

// fixed-order column sums of part[nb][n] added into out[n] (weights then bias)
__global__ void k_colsum_add(const float* __restrict__ part, int nb, int n, float* __restrict__ outW,
                             float* __restrict__ outb, int nw) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    double acc = 0.0;
    for (int b = 0; b < nb; ++b) acc += (double)part[(long long)b * n + p];
    if (p < nw) outW[p] += (float)acc;
    else if (outb) outb[p - nw] += (float)acc;
}

// ---------------------------------------------------------------------------
// GELU (erf form) and its derivative
// ---------------------------------------------------------------------------
__global__ void k_gelu(const float* __restrict__ x, float* __restrict__ y, long long n) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float v = x[q];
    y[q] = 0.5f * v * (1.f + erff(v * 0.70710678118654752f));
}

__global__ void k_gelu_bwd(const float* __restrict__ x, const float* __restrict__ gy, float* __restrict__ gx,
                           long long n, int accumulate) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float v = x[q];
    const float cdf = 0.5f * (1.f + erff(v * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * v * v);
    const float g = gy[q] * (cdf + v * pdf);
    gx[q] = accumulate ? gx[q] + g : g;
}

// ---------------------------------------------------------------------------
// Separable contractions.
//   contract_x: out[r, k] = sum_x M[k, x] in[r, x]        (rows r, reduce N -> K)
//   expand_x:   out[r, x] (+)= sum_k M[k, x] in[r, k]     (K -> N)
//   contract_mid: out[a, k, c] = sum_j M[k, j] in[a, j, c] (middle axis, any lengths)
// ---------------------------------------------------------------------------
constexpr int KMAX = 32;

// one warp per row; lanes stride the row; K partial sums per lane
__global__ void k_contract_x(const float* __restrict__ in, const float* __restrict__ M, float* __restrict__ out,
                             long long rows, int n, int K) {
    extern __shared__ float sm[];  // M [K][n]
    for (int q = threadIdx.x; q < K * n; q += blockDim.x) sm[q] = M[q];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= rows) return;
    float acc[KMAX];
#pragma unroll
    for (int k = 0; k < KMAX; ++k) acc[k] = 0.f;
    const float* row = in + r * n;
    for (int x = lane; x < n; x += 32) {
        const float v = row[x];
#pragma unroll
        for (int k = 0; k < KMAX; ++k)
            if (k < K) acc[k] = fmaf(sm[k * n + x], v, acc[k]);
    }
#pragma unroll
    for (int k = 0; k < KMAX; ++k) {
        if (k >= K) break;
        float a = acc[k];
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) out[r * K + k] = a;
    }
}

__global__ void k_expand_x(const float* __restrict__ in, const float* __restrict__ M, float* __restrict__ out,
                           long long rows, int n, int K, int accumulate) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= rows * n) return;
    const long long r = q / n;
    const int x = (int)(q - r * n);
    const float* src = in + r * K;
    float acc = 0.f;
    for (int k = 0; k < K; ++k) acc = fmaf(M[k * n + x], src[k], acc);
    out[q] = accumulate ? out[q] + acc : acc;
}

// middle axis: in (A, J, Cc) -> out (A, K, Cc) with out[a,k,c] = sum_j M[k,j] in[a,j,c]   (reduce)
// or (A, K, Cc) -> (A, J, Cc) with out[a,j,c] = sum_k M[k,j] in[a,k,c]                  (expand)
__global__ void k_mid(const float* __restrict__ in, const float* __restrict__ M, float* __restrict__ out, long long A,
                      int J, int K, int Cc, int expand, int accumulate) {
    const int L = expand ? J : K;      // output length along the axis
    const int Lin = expand ? K : J;    // input length along the axis
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= A * L * Cc) return;
    const long long a = q / ((long long)L * Cc);
    const int rem = (int)(q - a * L * Cc);
    const int l = rem / Cc, c = rem - l * Cc;
    const float* src = in + a * (long long)Lin * Cc + c;
    float acc = 0.f;
    if (expand) {
        for (int k = 0; k < K; ++k) acc = fmaf(M[k * J + l], src[(long long)k * Cc], acc);
    } else {
        for (int j = 0; j < J; ++j) acc = fmaf(M[l * J + j], src[(long long)j * Cc], acc);
    }
    out[q] = accumulate ? out[q] + acc : acc;
}

// ---------------------------------------------------------------------------
// mode-wise channel mixing with real weights W[k][i][o]
// ---------------------------------------------------------------------------
__global__ void k_modemix(const float* __restrict__ xh, const float* __restrict__ W, float* __restrict__ yh, int ci,
                          int co, int nm) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // (o, k)
    if (q >= (long long)co * nm) return;
    const int o = (int)(q / nm), k = (int)(q - (long long)o * nm);
    float acc = 0.f;
    const float* w = W + (long long)k * ci * co + o;
    for (int i = 0; i < ci; ++i) acc = fmaf(w[i * co], xh[(long long)i * nm + k], acc);
    yh[q] = acc;
}

__global__ void k_modemix_bwd(const float* __restrict__ xh, const float* __restrict__ W, const float* __restrict__ gyh,
                              float* __restrict__ gxh, float* __restrict__ gW, int ci, int co, int nm) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // (i, k)
    if (q >= (long long)ci * nm) return;
    const int i = (int)(q / nm), k = (int)(q - (long long)i * nm);
    const float* w = W + (long long)k * ci * co + (long long)i * co;
    float* gw = gW + (long long)k * ci * co + (long long)i * co;
    const float xv = xh[q];
    float acc = 0.f;
    for (int o = 0; o < co; ++o) {
        const float g = gyh[(long long)o * nm + k];
        acc = fmaf(w[o], g, acc);
        gw[o] += xv * g;
    }
    gxh[q] = acc;
}

// ---------------------------------------------------------------------------
// masked MSE: grad = 2 mask (p - t) / count, partial sums of mask (p - t)^2
// ---------------------------------------------------------------------------
__global__ void k_mse(const float* __restrict__ p, const float* __restrict__ t, const float* __restrict__ mask,
                      float* __restrict__ grad, long long n, float inv_count, double* __restrict__ part) {
    __shared__ double sh[32];
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (q < n) {
        const float m = mask ? mask[q] : 1.f;
        const float d = (p[q] - t[q]) * m;
        grad[q] = 2.f * d * inv_count;
        e = (double)d * (double)d;
    }
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = e;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) part[blockIdx.x] = v;
    }
}

__global__ void k_sum_double(const double* __restrict__ part, int n, double scale, double* __restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc = 0.0;
    for (int b = 0; b < n; ++b) acc += part[b];
    *out = acc * scale;
}

// ---------------------------------------------------------------------------
// Adam with decoupled weight decay
// ---------------------------------------------------------------------------
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float wd, float c1, float c2) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / c1, vh = vq / c2;
    p[q] = p[q] - lr * (mh / (sqrtf(vh) + eps) + wd * p[q]);
}

}  // namespace

extern "C" {

const char* nfgs_nn_last_error(void) { return g_nn_err.c_str(); }

int nfgs_nn_pointwise(const float* x, const float* W, const float* b, float* y, int32_t ci, int32_t co, int64_t nvox,
                      int32_t accumulate, void* stream) {
    if (!x || !W || !y || ci <= 0 || co <= 0 || nvox <= 0) return nn_fail(NFGS_EINVAL, "pointwise: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (ci == 32 && co == 32)
        k_pointwise<32, 32><<<nblk(nvox, 256), 256, 0, s>>>(x, W, b, y, nvox, accumulate);
    else
        k_pointwise_any<<<nblk(nvox, 256), 256, 0, s>>>(x, W, b, y, ci, co, nvox, accumulate);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_pointwise_bwd(const float* x, const float* W, const float* gy, float* gx, float* gW, float* gb, int32_t ci,
                          int32_t co, int64_t nvox, int32_t accumulate_gx, float* scratch, int64_t scratch_len,
                          void* stream) {
    if (!x || !W || !gy || !gW || ci <= 0 || co <= 0 || nvox <= 0) return nn_fail(NFGS_EINVAL, "pointwise_bwd: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    if (gx) {
        k_pointwise_bwd_x<<<nblk(nvox, 256), 256, 0, s>>>(W, gy, gx, ci, co, nvox, accumulate_gx);
        NNCK(cudaGetLastError());
    }
    const int npair = co * ci + co;
    const int threads = 256;
    if ((npair + threads - 1) / threads > 8) return nn_fail(NFGS_EINVAL, "pointwise_bwd: too many channel pairs");
    const long long nb = (nvox + VB - 1) / VB;
    if (!scratch || scratch_len < nb * npair) return nn_fail(NFGS_EINVAL, "pointwise_bwd: scratch too small");
    k_pointwise_bwd_w<<<(unsigned)nb, threads, (ci + co) * 32 * sizeof(float), s>>>(x, gy, scratch, ci, co, nvox);
    NNCK(cudaGetLastError());
    k_colsum_add<<<nblk(npair, 256), 256, 0, s>>>(scratch, (int)nb, npair, gW, gb, co * ci);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_gelu(const float* x, float* y, int64_t n, void* stream) {
    if (!x || !y || n <= 0) return nn_fail(NFGS_EINVAL, "gelu: bad arguments");
    k_gelu<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(x, y, n);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_gelu_bwd(const float* x, const float* gy, float* gx, int64_t n, int32_t accumulate, void* stream) {
    if (!x || !gy || !gx || n <= 0) return nn_fail(NFGS_EINVAL, "gelu_bwd: bad arguments");
    k_gelu_bwd<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(x, gy, gx, n, accumulate);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

// Trilinear resampling between node grids spanning the same box: target node
// (z', y', x') sits at source coordinates z' (nz-1)/(mz-1), ... (a single
// node maps to coordinate 0).
__global__ void k_resample_linear(const float* __restrict__ in, float* __restrict__ out, int C, int nz, int ny,
                                  int nx, int mz, int my, int mx) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long tot = (long long)C * mz * my * mx;
    if (t >= tot) return;
    const int xo = (int)(t % mx), yo = (int)((t / mx) % my), zo = (int)((t / ((long long)mx * my)) % mz);
    const int c = (int)(t / ((long long)mx * my * mz));
    auto axis = [](int o, int m, int n, int& i0, int& i1, float& w) {
        const float f = m > 1 ? (float)o * (float)(n - 1) / (float)(m - 1) : 0.f;
        i0 = min(max((int)floorf(f), 0), max(n - 2, 0));
        i1 = min(i0 + 1, n - 1);
        w = fminf(fmaxf(f - (float)i0, 0.f), 1.f);
    };
    int x0, x1, y0, y1, z0, z1;
    float wx, wy, wz;
    axis(xo, mx, nx, x0, x1, wx);
    axis(yo, my, ny, y0, y1, wy);
    axis(zo, mz, nz, z0, z1, wz);
    const float* b = in + (long long)c * nz * ny * nx;
    auto at = [&](int z, int y, int x) { return b[((long long)z * ny + y) * nx + x]; };
    const float c00 = at(z0, y0, x0) + wx * (at(z0, y0, x1) - at(z0, y0, x0));
    const float c01 = at(z0, y1, x0) + wx * (at(z0, y1, x1) - at(z0, y1, x0));
    const float c10 = at(z1, y0, x0) + wx * (at(z1, y0, x1) - at(z1, y0, x0));
    const float c11 = at(z1, y1, x0) + wx * (at(z1, y1, x1) - at(z1, y1, x0));
    const float d0 = c00 + wy * (c01 - c00), d1 = c10 + wy * (c11 - c10);
    out[t] = d0 + wz * (d1 - d0);
}

// in (C, nz, ny, nx) -> out (C, kz, ky, kx); t1 (C*nz*ny*kx), t2 (C*nz*ky*kx) scratch
int nfgs_nn_reduce3(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, const float* Mz,
                    const float* My, const float* Mx, int32_t kz, int32_t ky, int32_t kx, float* t1, float* t2,
                    void* stream) {
    if (!in || !out || !Mz || !My || !Mx || !t1 || !t2 || C <= 0 || kx > KMAX || kx <= 0 || ky <= 0 || kz <= 0)
        return nn_fail(NFGS_EINVAL, "reduce3: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const long long rows = (long long)C * nz * ny;
    const size_t shm = (size_t)kx * nx * sizeof(float);
    if (shm > 200 * 1024) return nn_fail(NFGS_EINVAL, "reduce3: x basis too large");
    if (shm > 48 * 1024) {
        static int raised = 0;  // the attribute is per device function; raise it once to the cap
        if (!raised) {
            NNCK(cudaFuncSetAttribute(k_contract_x, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            raised = 1;
        }
    }
    k_contract_x<<<nblk(rows, 8), 256, shm, s>>>(in, Mx, t1, rows, nx, kx);
    NNCK(cudaGetLastError());
    long long n2 = (long long)C * nz * ky * kx;
    k_mid<<<nblk(n2, 256), 256, 0, s>>>(t1, My, t2, (long long)C * nz, ny, ky, kx, 0, 0);
    NNCK(cudaGetLastError());
    long long n3 = (long long)C * kz * ky * kx;
    k_mid<<<nblk(n3, 256), 256, 0, s>>>(t2, Mz, out, (long long)C, nz, kz, ky * kx, 0, 0);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

// in (C, kz, ky, kx) -> out (C, nz, ny, nx) (accumulate optional); t1 (C*nz*ky*kx), t2 (C*nz*ny*kx)
int nfgs_nn_expand3(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, const float* Mz,
                    const float* My, const float* Mx, int32_t kz, int32_t ky, int32_t kx, int32_t accumulate,
                    float* t1, float* t2, void* stream) {
    if (!in || !out || !Mz || !My || !Mx || !t1 || !t2 || C <= 0 || kx <= 0 || ky <= 0 || kz <= 0)
        return nn_fail(NFGS_EINVAL, "expand3: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    long long n1 = (long long)C * nz * ky * kx;
    k_mid<<<nblk(n1, 256), 256, 0, s>>>(in, Mz, t1, (long long)C, nz, kz, ky * kx, 1, 0);
    NNCK(cudaGetLastError());
    long long n2 = (long long)C * nz * ny * kx;
    k_mid<<<nblk(n2, 256), 256, 0, s>>>(t1, My, t2, (long long)C * nz, ny, ky, kx, 1, 0);
    NNCK(cudaGetLastError());
    const long long rows = (long long)C * nz * ny;
    k_expand_x<<<nblk(rows * nx, 256), 256, 0, s>>>(t2, Mx, out, rows, nx, kx, accumulate);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_resample_linear(const float* in, float* out, int32_t C, int32_t nz, int32_t ny, int32_t nx, int32_t mz,
                            int32_t my, int32_t mx, void* stream) {
    if (!in || !out || C <= 0 || nz <= 0 || ny <= 0 || nx <= 0 || mz <= 0 || my <= 0 || mx <= 0)
        return nn_fail(NFGS_EINVAL, "resample_linear: bad arguments");
    const long long tot = (long long)C * mz * my * mx;
    k_resample_linear<<<nblk(tot, 256), 256, 0, (cudaStream_t)stream>>>(in, out, C, nz, ny, nx, mz, my, mx);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_modemix(const float* xh, const float* W, float* yh, int32_t ci, int32_t co, int32_t nm, void* stream) {
    if (!xh || !W || !yh || ci <= 0 || co <= 0 || nm <= 0) return nn_fail(NFGS_EINVAL, "modemix: bad arguments");
    k_modemix<<<nblk((long long)co * nm, 256), 256, 0, (cudaStream_t)stream>>>(xh, W, yh, ci, co, nm);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_modemix_bwd(const float* xh, const float* W, const float* gyh, float* gxh, float* gW, int32_t ci,
                        int32_t co, int32_t nm, void* stream) {
    if (!xh || !W || !gyh || !gxh || !gW || ci <= 0 || co <= 0 || nm <= 0)
        return nn_fail(NFGS_EINVAL, "modemix_bwd: bad arguments");
    k_modemix_bwd<<<nblk((long long)ci * nm, 256), 256, 0, (cudaStream_t)stream>>>(xh, W, gyh, gxh, gW, ci, co, nm);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

// loss_out: device double; part: device double scratch of >= ceil(n/256)
int nfgs_nn_mse(const float* pred, const float* target, const float* mask, float* grad, int64_t n, double count,
                double* part, double* loss_out, void* stream) {
    if (!pred || !target || !grad || !part || !loss_out || n <= 0 || !(count > 0))
        return nn_fail(NFGS_EINVAL, "mse: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const unsigned nb = nblk(n, 256);
    k_mse<<<nb, 256, 0, s>>>(pred, target, mask, grad, n, (float)(1.0 / count), part);
    NNCK(cudaGetLastError());
    k_sum_double<<<1, 32, 0, s>>>(part, (int)nb, 1.0 / count, loss_out);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

int nfgs_nn_adam(float* p, const float* g, float* m, float* v, int64_t n, float lr, float b1, float b2, float eps,
                 float wd, int32_t step, void* stream) {
    if (!p || !g || !m || !v || n <= 0 || step < 1) return nn_fail(NFGS_EINVAL, "adam: bad arguments");
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<nblk(n, 256), 256, 0, (cudaStream_t)stream>>>(p, g, m, v, n, lr, b1, b2, eps, wd, c1, c2);
    NNCK(cudaGetLastError());
    return NFGS_OK;
}

}  // extern "C"
