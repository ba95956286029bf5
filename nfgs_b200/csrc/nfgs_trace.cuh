// Field-line tracing and the squashing factor Q on a seed plane.
//
// Positions are in grid-index units (x in [0, nx-1], y in [0, ny-1],
// z in [0, nz-1]); B is sampled on the nodes of a (3, nz, ny, nx) volume and
// interpolated trilinearly.  A line follows the unit field direction with
// classical fourth-order Runge-Kutta steps of fixed length; the step that
// leaves the box is cut where its chord meets the first face, and the end
// point is snapped onto that face.  Q (Titov, Hornig & Demoulin 2002;
// Titov 2007) is ||D||^2 / |det D| for the footpoint map D; for seeds on a
// plane with in-plane unit axes u, v, the derivatives a = dr/du, b = dr/dv of
// the two end points give ||D||^2 |det D|^-1 =
//   [|a+|^2 |b-|^2 + |b+|^2 |a-|^2 - 2 (a+.b+)(a-.b-)] |Bn+ Bn-| / Bn0^2,
// using flux conservation |det(dr/d(u,v))| = |Bn0 / Bn|.
//
// One thread per (seed, direction): the threads of a warp trace neighbouring
// seeds, whose lines stay close, so the corner loads of the interpolation
// hit the same L1/L2 lines.  The field is repacked as 4 values per node
// (one 16-byte load in FP32, two in FP64).
#pragma once
#include "nfgs_common.cuh"

namespace trace {

template <typename T>
__device__ __forceinline__ void load3(const T* __restrict__ p, T& x, T& y, T& z);

template <>
__device__ __forceinline__ void load3<float>(const float* __restrict__ p, float& x, float& y, float& z) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    x = v.x; y = v.y; z = v.z;
}

template <>
__device__ __forceinline__ void load3<double>(const double* __restrict__ p, double& x, double& y, double& z) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    x = a.x; y = a.y; z = __ldg(p + 2);
}

// second-order derivative in grid units along a line of n samples (the
// centred difference inside, three-point one-sided ends; n >= 3)
template <typename T, typename F>
__device__ __forceinline__ T grad1(F f, int i, int n) {
    if (i == 0) return (T(-3) * f(0) + T(4) * f(1) - f(2)) * T(0.5);
    if (i == n - 1) return (T(3) * f(n - 1) - T(4) * f(n - 2) + f(n - 3)) * T(0.5);
    return (f(i + 1) - f(i - 1)) * T(0.5);
}

// (3, nz, ny, nx) component-major -> (Bx, By, Bz, 0) per node, followed with
// TW by (Jx, Jy, Jz, 0), J = curl B in grid units
template <typename T, bool TW>
__global__ void k_pack(const T* __restrict__ b, int nx, int ny, int nz, T* __restrict__ pk) {
    const long long V = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= V) return;
    constexpr int S = TW ? 8 : 4;
    pk[S * c] = b[c];
    pk[S * c + 1] = b[V + c];
    pk[S * c + 2] = b[2 * V + c];
    pk[S * c + 3] = T(0);
    if constexpr (TW) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
        const long long P = (long long)nx * ny;
        auto ax = [&](int comp) { return [=](int q) { return b[comp * V + c + (q - i)]; }; };
        auto ay = [&](int comp) { return [=](int q) { return b[comp * V + c + (long long)(q - j) * nx]; }; };
        auto az = [&](int comp) { return [=](int q) { return b[comp * V + c + (long long)(q - k) * P]; }; };
        const T dbz_dy = grad1<T>(ay(2), j, ny), dby_dz = grad1<T>(az(1), k, nz);
        const T dbx_dz = grad1<T>(az(0), k, nz), dbz_dx = grad1<T>(ax(2), i, nx);
        const T dby_dx = grad1<T>(ax(1), i, nx), dbx_dy = grad1<T>(ay(0), j, ny);
        pk[S * c + 4] = dbz_dy - dby_dz;
        pk[S * c + 5] = dbx_dz - dbz_dx;
        pk[S * c + 6] = dby_dx - dbx_dy;
        pk[S * c + 7] = T(0);
    }
}

struct Box {
    int nx, ny, nz;
    int st;  // values per node in the packed field: 4 (B) or 8 (B, J)
};

// trilinear interpolation at a position clamped into the box
template <typename T>
__device__ __forceinline__ void interp(const T* __restrict__ pk, Box bx, T x, T y, T z, T& ox, T& oy, T& oz,
                                       int off = 0) {
    x = fmin(fmax(x, T(0)), T(bx.nx - 1));
    y = fmin(fmax(y, T(0)), T(bx.ny - 1));
    z = fmin(fmax(z, T(0)), T(bx.nz - 1));
    const int i = min((int)floor(x), bx.nx - 2);
    const int j = min((int)floor(y), bx.ny - 2);
    const int k = min((int)floor(z), bx.nz - 2);
    const T fx = x - T(i), fy = y - T(j), fz = z - T(k);
    const long long sx = bx.st, sy = (long long)bx.st * bx.nx, sz = (long long)bx.st * bx.nx * bx.ny;
    const T* p = pk + k * sz + j * sy + i * sx + off;
    T c[8][3];
#pragma unroll
    for (int q = 0; q < 8; ++q)
        load3<T>(p + ((q >> 2) & 1) * sz + ((q >> 1) & 1) * sy + (q & 1) * sx, c[q][0], c[q][1], c[q][2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T x00 = c[0][d] + fx * (c[1][d] - c[0][d]);
        const T x10 = c[2][d] + fx * (c[3][d] - c[2][d]);
        const T x01 = c[4][d] + fx * (c[5][d] - c[4][d]);
        const T x11 = c[6][d] + fx * (c[7][d] - c[6][d]);
        const T y0 = x00 + fy * (x10 - x00);
        const T y1 = x01 + fy * (x11 - x01);
        const T v = y0 + fz * (y1 - y0);
        if (d == 0) ox = v; else if (d == 1) oy = v; else oz = v;
    }
}

// unit direction s B / |B|; false where |B| = 0
template <typename T>
__device__ __forceinline__ bool direction(const T* __restrict__ pk, Box bx, T s, const T (&p)[3], T (&d)[3]) {
    T b0, b1, b2;
    interp<T>(pk, bx, p[0], p[1], p[2], b0, b1, b2);
    const T m = sqrt(b0 * b0 + b1 * b1 + b2 * b2);
    if (!(m > T(0))) return false;
    const T f = s / m;
    d[0] = b0 * f; d[1] = b1 * f; d[2] = b2 * f;
    return true;
}

// unit direction and, with TW, the twist integrand J.B / (4 pi |B|^2)
template <typename T, bool TW>
__device__ __forceinline__ bool dir_tw(const T* __restrict__ pk, Box bx, T s, const T (&p)[3], T (&d)[3], T& f) {
    T b0, b1, b2;
    interp<T>(pk, bx, p[0], p[1], p[2], b0, b1, b2);
    const T m2 = b0 * b0 + b1 * b1 + b2 * b2;
    const T m = sqrt(m2);
    if (!(m > T(0))) return false;
    const T g = s / m;
    d[0] = b0 * g; d[1] = b1 * g; d[2] = b2 * g;
    if constexpr (TW) {
        T j0, j1, j2;
        interp<T>(pk, bx, p[0], p[1], p[2], j0, j1, j2, 4);
        f = (j0 * b0 + j1 * b1 + j2 * b2) / (T(4.0 * 3.14159265358979323846) * m2);
    }
    return true;
}

// Trace one line from p (inside the box) along s B: p becomes the end point;
// returns the face code (1..6), 0 after max_steps, -1 at a zero field.  With
// TW, twist integrates J.B / (4 pi |B|^2) ds with the same RK4 stages (the
// cut last step contributes its fraction t).
template <typename T, bool TW = false>
__device__ int trace_line(const T* __restrict__ pk, Box bx, const T (&hi)[3], T (&p)[3], T s, T h, int max_steps,
                          T& length, T& twist) {
    const T h2 = h * T(0.5), h6 = h / T(6);
    length = T(0);
    twist = T(0);
    for (int it = 0; it < max_steps; ++it) {
        T k1[3], k2[3], k3[3], k4[3], q[3];
        T f1 = T(0), f2 = T(0), f3 = T(0), f4 = T(0);
        if (!dir_tw<T, TW>(pk, bx, s, p, k1, f1)) return -1;
#pragma unroll
        for (int d = 0; d < 3; ++d) q[d] = p[d] + h2 * k1[d];
        if (!dir_tw<T, TW>(pk, bx, s, q, k2, f2)) return -1;
#pragma unroll
        for (int d = 0; d < 3; ++d) q[d] = p[d] + h2 * k2[d];
        if (!dir_tw<T, TW>(pk, bx, s, q, k3, f3)) return -1;
#pragma unroll
        for (int d = 0; d < 3; ++d) q[d] = p[d] + h * k3[d];
        if (!dir_tw<T, TW>(pk, bx, s, q, k4, f4)) return -1;
#pragma unroll
        for (int d = 0; d < 3; ++d) q[d] = p[d] + h6 * (k1[d] + T(2) * k2[d] + T(2) * k3[d] + k4[d]);
        const T dtw = TW ? h6 * (f1 + T(2) * f2 + T(2) * f3 + f4) : T(0);
        bool inside = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) inside = inside && q[d] >= T(0) && q[d] <= hi[d];
        if (inside) {
#pragma unroll
            for (int d = 0; d < 3; ++d) p[d] = q[d];
            length += h;
            if (TW) twist += dtw;
            continue;
        }
        // the chord p -> q meets the first face at fraction t
        T t = T(2);
        int face = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (q[d] < T(0)) {
                const T td = (T(0) - p[d]) / (q[d] - p[d]);
                if (td < t) { t = td; face = 2 * d + 1; }
            } else if (q[d] > hi[d]) {
                const T td = (hi[d] - p[d]) / (q[d] - p[d]);
                if (td < t) { t = td; face = 2 * d + 2; }
            }
        }
        if (face == 0) return 0;  // a non-finite step: no face (p stays inside)
#pragma unroll
        for (int d = 0; d < 3; ++d) p[d] = p[d] + t * (q[d] - p[d]);
        const int fd = (face - 1) >> 1;
        p[fd] = (face & 1) ? T(0) : hi[fd];
        length += t * h;
        if (TW) twist += t * dtw;
        return face;
    }
    return 0;
}

// |B.n| at an end on face `flag` (NaN without a face)
template <typename T>
__device__ __forceinline__ T end_bn(const T* __restrict__ pk, Box bx, const T (&p)[3], int flag) {
    if (flag <= 0) return T(NAN);
    T b[3];
    interp<T>(pk, bx, p[0], p[1], p[2], b[0], b[1], b[2]);
    return fabs(b[(flag - 1) >> 1]);
}

// Trace seed `si` along +B (dir 0) or -B (dir 1).  ends (2, n, 3), flags
// (2, n), bn (3, n): B.n0 at the seed, |B.n| at the forward and backward
// ends; len (2, n) per direction.
template <typename T, bool TW>
__global__ void __launch_bounds__(128) k_trace(const T* __restrict__ pk, Box bx, const T* __restrict__ seeds,
                                               long long n, T n0x, T n0y, T n0z, T h, int max_steps,
                                               T* __restrict__ ends, int* __restrict__ flags, T* __restrict__ bn,
                                               T* __restrict__ len, T* __restrict__ tw) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 2 * n) return;
    const int dir = tid >= n ? 1 : 0;
    const long long si = tid - (long long)dir * n;
    const T hi[3] = {T(bx.nx - 1), T(bx.ny - 1), T(bx.nz - 1)};
    // seeds are clamped into the box, so every chord that leaves it starts inside
    T p[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = fmin(fmax(seeds[3 * si + d], T(0)), hi[d]);
    if (dir == 0) {
        T b0, b1, b2;
        interp<T>(pk, bx, p[0], p[1], p[2], b0, b1, b2);
        bn[si] = b0 * n0x + b1 * n0y + b2 * n0z;
    }
    T length, twist;
    const int flag = trace_line<T, TW>(pk, bx, hi, p, dir == 0 ? T(1) : T(-1), h, max_steps, length, twist);
    ends[3 * tid] = p[0];
    ends[3 * tid + 1] = p[1];
    ends[3 * tid + 2] = p[2];
    flags[tid] = flag;
    len[tid] = length;
    if (TW) tw[tid] = twist;
    bn[n * (1 + dir) + si] = end_bn<T>(pk, bx, p, flag);
}

// Perpendicular frame at a seed: b = B0/|B0|, e1 = unit(b x a) with a the
// coordinate axis least aligned with b, e2 = b x e1.  False where |B0| = 0.
template <typename T>
__device__ __forceinline__ bool perp_frame(const T (&B)[3], T& bm, T (&e1)[3], T (&e2)[3]) {
    bm = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
    if (!(bm > T(0))) return false;
    const T b[3] = {B[0] / bm, B[1] / bm, B[2] / bm};
    int ax = 0;
    if (fabs(b[1]) < fabs(b[ax])) ax = 1;
    if (fabs(b[2]) < fabs(b[ax])) ax = 2;
    T c[3];  // b x a
    if (ax == 0) { c[0] = T(0); c[1] = b[2]; c[2] = -b[1]; }
    else if (ax == 1) { c[0] = -b[2]; c[1] = T(0); c[2] = b[0]; }
    else { c[0] = b[1]; c[1] = -b[0]; c[2] = T(0); }
    const T cm = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) e1[d] = c[d] / cm;
    e2[0] = b[1] * e1[2] - b[2] * e1[1];
    e2[1] = b[2] * e1[0] - b[0] * e1[2];
    e2[2] = b[0] * e1[1] - b[1] * e1[0];
    return true;
}

// Q_perp lines: per seed, the line through the seed and four through
// seed +- delta e1, seed +- delta e2 (clamped into the box), each traced both
// ways.  Thread tid = (dir * 5 + a) * n + si.  ends (2, 5, n, 3), flags
// (2, 5, n); bn (3, n): |B0|, |Bn+|, |Bn-| of the central line; len (2, n)
// of the central line.
template <typename T, bool TW>
__global__ void __launch_bounds__(128) k_trace_perp(const T* __restrict__ pk, Box bx, const T* __restrict__ seeds,
                                                    long long n, T delta, T h, int max_steps, T* __restrict__ ends,
                                                    int* __restrict__ flags, T* __restrict__ bn,
                                                    T* __restrict__ len, T* __restrict__ tw) {
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= 10 * n) return;
    const long long si = tid % n;
    const int da = (int)(tid / n);
    const int dir = da / 5, a = da % 5;
    const T hi[3] = {T(bx.nx - 1), T(bx.ny - 1), T(bx.nz - 1)};
    T p[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = fmin(fmax(seeds[3 * si + d], T(0)), hi[d]);
    T B0[3], bm, e1[3], e2[3];
    interp<T>(pk, bx, p[0], p[1], p[2], B0[0], B0[1], B0[2]);
    const bool ok = perp_frame<T>(B0, bm, e1, e2);
    if (a == 0 && dir == 0) bn[si] = ok ? bm : T(0);
    if (ok && a > 0) {
        const T sg = (a & 1) ? T(1) : T(-1);
        const T* e = a <= 2 ? e1 : e2;
#pragma unroll
        for (int d = 0; d < 3; ++d) p[d] = fmin(fmax(p[d] + sg * delta * e[d], T(0)), hi[d]);
    }
    T length = T(0), twist = T(0);
    const int flag =
        ok ? trace_line<T, TW>(pk, bx, hi, p, dir == 0 ? T(1) : T(-1), h, max_steps, length, twist) : -1;
    ends[3 * tid] = p[0];
    ends[3 * tid + 1] = p[1];
    ends[3 * tid + 2] = p[2];
    flags[tid] = flag;
    if (a == 0) {
        len[dir * n + si] = length;
        if (TW) tw[dir * n + si] = twist;
        bn[n * (1 + dir) + si] = end_bn<T>(pk, bx, p, flag);
    }
}

// Q_perp = [|a+|^2 |b-|^2 + |b+|^2 |a-|^2 - 2 (a+.b+)(a-.b-)] |Bn+ Bn-| / |B0|^2
// with a = dr/dp, b = dr/dq by central differences over +-delta along e1, e2
// (Titov 2007); NaN unless the five lines of each direction end on one face.
template <typename T>
__global__ void k_qperp(long long n, T delta, const T* __restrict__ ends, const int* __restrict__ flags,
                        const T* __restrict__ bn, T* __restrict__ q) {
    const long long si = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= n) return;
    T a[2][3], b[2][3];
    const T inv = T(1) / (T(2) * delta);
    for (int dir = 0; dir < 2; ++dir) {
        const int f0 = flags[(dir * 5) * n + si];
        bool ok = f0 > 0;
#pragma unroll
        for (int r = 1; r < 5; ++r) ok = ok && flags[(dir * 5 + r) * n + si] == f0;
        if (!ok) { q[si] = T(NAN); return; }
        const T* e = ends + 3 * (dir * 5) * n;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            a[dir][d] = (e[3 * (1 * n + si) + d] - e[3 * (2 * n + si) + d]) * inv;
            b[dir][d] = (e[3 * (3 * n + si) + d] - e[3 * (4 * n + si) + d]) * inv;
        }
    }
    auto dot = [](const T (&x)[3], const T (&y)[3]) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    const T br = dot(a[0], a[0]) * dot(b[1], b[1]) + dot(b[0], b[0]) * dot(a[1], a[1]) -
                 T(2) * dot(a[0], b[0]) * dot(a[1], b[1]);
    const T b0 = bn[si];
    q[si] = b0 > T(0) ? br * fabs(bn[n + si] * bn[2 * n + si]) / (b0 * b0) : T(NAN);
}

// Q on a regular nv x nu seed plane (seed iu + nu iv, unit spacing)
template <typename T>
__global__ void k_qmap(int nu, int nv, const T* __restrict__ ends, const int* __restrict__ flags,
                       const T* __restrict__ bn, T* __restrict__ q) {
    const int iu = blockIdx.x * blockDim.x + threadIdx.x;
    const int iv = blockIdx.y;
    if (iu >= nu || iv >= nv) return;
    const long long n = (long long)nu * nv;
    const long long c = (long long)iv * nu + iu;
    if (iu == 0 || iv == 0 || iu == nu - 1 || iv == nv - 1) { q[c] = T(NAN); return; }
    const long long nb[4] = {c + 1, c - 1, c + nu, c - nu};
    T a[2][3], b[2][3];
    for (int dir = 0; dir < 2; ++dir) {
        const int* f = flags + dir * n;
        const int fc = f[c];
        bool ok = fc > 0;
#pragma unroll
        for (int r = 0; r < 4; ++r) ok = ok && f[nb[r]] == fc;
        if (!ok) { q[c] = T(NAN); return; }
        const T* e = ends + 3 * dir * n;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            a[dir][d] = (e[3 * nb[0] + d] - e[3 * nb[1] + d]) * T(0.5);
            b[dir][d] = (e[3 * nb[2] + d] - e[3 * nb[3] + d]) * T(0.5);
        }
    }
    auto dot = [](const T (&x)[3], const T (&y)[3]) { return x[0] * y[0] + x[1] * y[1] + x[2] * y[2]; };
    const T br = dot(a[0], a[0]) * dot(b[1], b[1]) + dot(b[0], b[0]) * dot(a[1], a[1]) -
                 T(2) * dot(a[0], b[0]) * dot(a[1], b[1]);
    const T b0 = bn[c];
    q[c] = br * fabs(bn[n + c] * bn[2 * n + c]) / (b0 * b0);
}

}  // namespace trace
