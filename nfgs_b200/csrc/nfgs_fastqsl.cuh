// FastQSL-compatible field-line tracing and Q on a seed plane.
//
// The reference draws its topology maps (nfgs/_backend/util/fastqsl_plane.py:
// 203-506) with the vendored FastQSL adaptive tracer (TraceAllBline of
// third_party/FastQSL/fastqslpy/cu/TraceBlineAdaptive.cu) and its plane
// formula QCalcPlane (fastqslpy/FastQSL.py).  This file restates both for
// FP32 fields, in the reference's arithmetic, so that the maps match it:
//
//  * direction: trilinear B normalised to unit length, clamped to the
//    outermost cell at the faces (weights formed in double, as there);
//  * step: embedded Runge-Kutta-Fehlberg 4(5) (Fehlberg 1969) on grid-unit
//    positions; the fifth-order solution advances, the norm of the
//    difference of the two solutions is the error; the step factor is
//    (tol / err / 11.09)^(1/5), a step with factor < 0.618 is retried at
//    0.618 of its length, otherwise the next step is scaled and kept in
//    [0.1, 100] cells.  tol = 1e-3 |b.n|^1.5 (1e-3 / 8000 where |b.n| <= 0.05)
//    times the caller's tol, from the unit field at the seed;
//  * end: a step that leaves the box is undone; when it crosses one face
//    (|dx| > 1e-3 along that axis), the end is the chord's linear estimate
//    at that face where |b| along the face normal is below 0.2 at either end
//    of the step, else a fourth-order Runge-Kutta step in the face-normal
//    coordinate up to it (the max faces sit at N, one cell beyond the last
//    node, as in the reference); a step that leaves through an edge or
//    corner ends at its end point with code 42; the path length adds the
//    face-normal distance over (1e-4 + |b_n|);
//  * the twist number integrates J.B / (4 pi |B|^2) ds with the left-point
//    rule over the accepted steps (pi = 3.14159265 as in the reference);
//  * Q (QCalcPlane): the end points of each seed, projected on the face each
//    one reached ((x, y) on z faces, (z, x) on y faces, (y, z) on x faces),
//    are differenced over the four neighbours in the seed plane; with
//    a..d the 2 x 2 products of those differences,
//    Q = (a^2 + b^2 + c^2 + d^2) |Bz_start| |Bz_end| / (B.n)^2 / (2 stride)^4,
//    at least 1, NaN where any neighbour ended on another face and on the
//    plane's border.
//
// Face codes: 0 inside (length or step limit), 1/2 x min/max, 3/4 y min/max,
// 5/6 z min/max, 42 through an edge or corner (and at y exactly 0, which the
// reference's inside test excludes).
#pragma once
#include "nfgs_trace.cuh"

namespace fq {

constexpr double TOL0 = 1e-3;          // per-step tolerance before the seed factor
constexpr double STEP_RATIO = 3.0;     // path length limit: 3 (nx + ny + nz)
constexpr long long MAX_STEPS = 500000;
constexpr double PI_REF = 3.14159265;  // the reference's value of pi

struct F3 {
    float x, y, z;
};
__host__ __device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return f3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ F3 operator/(F3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float len3(F3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float comp(F3 a, int d) { return d == 0 ? a.x : (d == 1 ? a.y : a.z); }

// B (and, for the twist, J) as (3, nz, ny, nx) component-major FP32 volumes:
// three FP32 values per node, the footprint the reference reads (a 256^2 x 128
// field, 101 MB, stays in the 126 MB L2; padded to four values it would not)
struct Field {
    const float* b;  // (3, V)
    const float* j;  // (3, V) or null
    int nx, ny, nz;
    long long V;
};

// node value of B (cur == false) or J (cur == true)
__device__ __forceinline__ F3 node(const Field& f, int i, int j, int k, bool cur) {
    const float* a = cur ? f.j : f.b;
    const unsigned q = ((unsigned)k * (unsigned)f.ny + (unsigned)j) * (unsigned)f.nx + (unsigned)i;  // V < 2^31
    return f3(__ldg(a + q), __ldg(a + f.V + q), __ldg(a + 2 * f.V + q));
}

// trilinear vector at p with the faces' outermost cell (TraceBlineAdaptive
// Interp3dxyzn); unit length when norm
__device__ __forceinline__ F3 interp_dir(const Field& f, F3 p, bool norm, bool off = false) {
    float rx = p.x - floorf(p.x), ry = p.y - floorf(p.y), rz = p.z - floorf(p.z);
    int i = __float2int_rd(p.x), j = __float2int_rd(p.y), k = __float2int_rd(p.z);
    if (p.x <= 0.f) { rx = 0.f; i = 0; }
    if (p.x >= f.nx - 1) { rx = 1.f; i = f.nx - 2; }
    if (p.y <= 0.f) { ry = 0.f; j = 0; }
    if (p.y >= f.ny - 1) { ry = 1.f; j = f.ny - 2; }
    if (p.z <= 0.f) { rz = 0.f; k = 0; }
    if (p.z >= f.nz - 1) { rz = 1.f; k = f.nz - 2; }
    // a non-finite position indexes the first cell
    if (!(i >= 0 && i <= f.nx - 2)) i = 0;
    if (!(j >= 0 && j <= f.ny - 2)) j = 0;
    if (!(k >= 0 && k <= f.nz - 2)) k = 0;
    const double ux = 1.0 - (double)rx, uy = 1.0 - (double)ry, uz = 1.0 - (double)rz;
    const float w000 = (float)(ux * uy * uz), w001 = (float)(ux * uy * rz), w010 = (float)(ux * ry * uz);
    const float w011 = (float)(ux * ry * rz), w100 = (float)(rx * uy * uz), w101 = (float)(rx * uy * rz);
    const float w110 = (float)(rx * ry * uz), w111 = (float)(rx * ry * rz);
    const F3 a000 = node(f, i, j, k, off), a001 = node(f, i, j, k + 1, off);
    const F3 a010 = node(f, i, j + 1, k, off), a011 = node(f, i, j + 1, k + 1, off);
    const F3 a100 = node(f, i + 1, j, k, off), a101 = node(f, i + 1, j, k + 1, off);
    const F3 a110 = node(f, i + 1, j + 1, k, off), a111 = node(f, i + 1, j + 1, k + 1, off);
    F3 r;
    r.x = a000.x * w000 + a001.x * w001 + a010.x * w010 + a011.x * w011 + a100.x * w100 + a101.x * w101 +
          a110.x * w110 + a111.x * w111;
    r.y = a000.y * w000 + a001.y * w001 + a010.y * w010 + a011.y * w011 + a100.y * w100 + a101.y * w101 +
          a110.y * w110 + a111.y * w111;
    r.z = a000.z * w000 + a001.z * w001 + a010.z * w010 + a011.z * w011 + a100.z * w100 + a101.z * w101 +
          a110.z * w110 + a111.z * w111;
    if (norm) {
        const float m = sqrtf(r.x * r.x + r.y * r.y + r.z * r.z);
        r = f3(r.x / m, r.y / m, r.z / m);
    }
    return r;
}

// trilinear sample of one component (offset c of the packed field) inside
// [1e-4, N - 1 - 1e-4], the weights and the sum in double, for the field
// recorded at the seed and the ends (TraceBlineAdaptive.cu:46-99).  The sum
// keeps the reference's term order and operand types (FP32 corner value
// times double weights, left to right), and stays a separate function as
// there, so that its rounding is the reference's bit for bit.
__device__ __noinline__ float interp3d(const Field& f, int c, float px, float py, float pz) {
    px = (px > 0) ? px : 0.0001;
    py = (py > 0) ? py : 0.0001;
    pz = (pz > 0) ? pz : 0.0001;
    px = (px < f.nx - 1) ? px : ((float)f.nx - 1 - 0.0001);
    py = (py < f.ny - 1) ? py : ((float)f.ny - 1 - 0.0001);
    pz = (pz < f.nz - 1) ? pz : ((float)f.nz - 1 - 0.0001);
    const float tx = px - floorf(px), ty = py - floorf(py), tz = pz - floorf(pz);
    int i = __float2int_rd(px), j = __float2int_rd(py), k = __float2int_rd(pz);
    if (!(i >= 0 && i <= f.nx - 2)) i = 0;  // a non-finite position
    if (!(j >= 0 && j <= f.ny - 2)) j = 0;
    if (!(k >= 0 && k <= f.nz - 2)) k = 0;
    auto at = [&](int ii, int jj, int kk) -> float {
        return __ldg(f.b + c * f.V + (((unsigned)kk * (unsigned)f.ny + (unsigned)jj) * (unsigned)f.nx + (unsigned)ii));
    };
    const float c000 = at(i, j, k), c001 = at(i, j, k + 1), c010 = at(i, j + 1, k), c011 = at(i, j + 1, k + 1);
    const float c100 = at(i + 1, j, k), c101 = at(i + 1, j, k + 1), c110 = at(i + 1, j + 1, k);
    const float c111 = at(i + 1, j + 1, k + 1);
    const float v = c000 * (1. - tx) * (1. - ty) * (1. - tz) + c001 * (1. - tx) * (1. - ty) * (tz) +
                    c010 * (1. - tx) * (ty) * (1. - tz) + c011 * (1. - tx) * (ty) * (tz) +
                    c100 * (tx) * (1. - ty) * (1. - tz) + c101 * (tx) * (1. - ty) * (tz) +
                    c110 * (tx) * (ty) * (1. - tz) + c111 * (tx) * (ty) * (tz);
    return v;
}

__device__ __forceinline__ F3 interp_sample(const Field& f, F3 p) {
    return f3(interp3d(f, 0, p.x, p.y, p.z), interp3d(f, 1, p.x, p.y, p.z), interp3d(f, 2, p.x, p.y, p.z));
}

// J = curl B in grid units, centred with second-order one-sided edges (the
// current fastqsl_plane.py:287-305 passes to the tracer), (3, V) FP32
__global__ void k_curl(const float* __restrict__ b, int nx, int ny, int nz, float* __restrict__ jo) {
    const long long V = (long long)nx * ny * nz;
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= V) return;
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    const long long P = (long long)nx * ny;
    auto ax = [&](int comp) { return [=](int q) { return b[comp * V + c + (q - i)]; }; };
    auto ay = [&](int comp) { return [=](int q) { return b[comp * V + c + (long long)(q - j) * nx]; }; };
    auto az = [&](int comp) { return [=](int q) { return b[comp * V + c + (long long)(q - k) * P]; }; };
    jo[c] = trace::grad1<float>(ay(2), j, ny) - trace::grad1<float>(az(1), k, nz);
    jo[V + c] = trace::grad1<float>(az(0), k, nz) - trace::grad1<float>(ax(2), i, nx);
    jo[2 * V + c] = trace::grad1<float>(ax(1), i, nx) - trace::grad1<float>(ay(0), j, ny);
}

// Fehlberg 4(5) stage coefficients (Fehlberg 1969, as single-precision
// constants) and the fifth-order weights; E = fifth- minus fourth-order.
struct RKF {
    static constexpr float a21 = (float)(1. / 4.);
    static constexpr float a31 = (float)(3. / 32.), a32 = (float)(9. / 32.);
    static constexpr float a41 = (float)(1932. / 2197.), a42 = (float)(-7200. / 2197.), a43 = (float)(7296. / 2197.);
    static constexpr float a51 = (float)(439. / 216.), a52 = -8.f, a53 = (float)(3680. / 513.),
                           a54 = (float)(-845. / 4104.);
    static constexpr float a61 = (float)(-8. / 27.), a62 = 2.f, a63 = (float)(-3544. / 2565.),
                           a64 = (float)(1859. / 4104.), a65 = (float)(-11. / 40.);
    static constexpr float b1 = (float)(16. / 135.), b3 = (float)(6656. / 12825.), b4 = (float)(28561. / 56430.),
                           b5 = (float)(-9. / 50.), b6 = (float)(2. / 55.);
    static constexpr float e1 = (float)(1. / 360.), e3 = (float)(-128. / 4275.), e4 = (float)(-2197. / 75240.),
                           e5 = (float)(1. / 50.), e6 = (float)(2. / 55.);
};

// one Fehlberg step of length h from p: the fifth-order end point and the
// error norm
__device__ __forceinline__ F3 rkf45(const Field& f, F3 p, float h, float& err) {
    using R = RKF;
    const F3 k1 = h * interp_dir(f, p, true);
    const F3 k2 = h * interp_dir(f, p + (R::a21 * k1), true);
    const F3 k3 = h * interp_dir(f, p + (R::a31 * k1 + R::a32 * k2), true);
    const F3 k4 = h * interp_dir(f, p + (R::a41 * k1 + R::a42 * k2 + R::a43 * k3), true);
    const F3 k5 = h * interp_dir(f, p + (R::a51 * k1 + R::a52 * k2 + R::a53 * k3 + R::a54 * k4), true);
    const F3 k6 = h * interp_dir(f, p + (R::a61 * k1 + R::a62 * k2 + R::a63 * k3 + R::a64 * k4 + R::a65 * k5), true);
    err = len3(R::e1 * k1 + R::e3 * k3 + R::e4 * k4 + R::e5 * k5 + R::e6 * k6);
    return p + (R::b1 * k1 + R::b3 * k3 + R::b4 * k4 + R::b5 * k5 + R::b6 * k6);
}

// classical Runge-Kutta step of length s in coordinate d (dr/dx_d = b / b_d)
__device__ __forceinline__ F3 rk4_face(const Field& f, F3 p, float s, int d) {
    const F3 b1 = interp_dir(f, p, true);
    const F3 k1 = b1 / comp(b1, d);
    const F3 b2 = interp_dir(f, p + s * k1 / 2.f, true);
    const F3 k2 = b2 / comp(b2, d);
    const F3 b3 = interp_dir(f, p + s * k2 / 2.f, true);
    const F3 k3 = b3 / comp(b3, d);
    const F3 b4 = interp_dir(f, p + s * k3, true);
    const F3 k4 = b4 / comp(b4, d);
    return p + (float)((1. / 6.) * s) * (k1 + 2.0f * k2 + 2.0f * k3 + k4);
}

// 0 inside, 1..6 through one face, 42 otherwise (TraceBlineAdaptive checkFlag)
__device__ __forceinline__ int face_code(const Field& f, F3 p) {
    const float X = (float)(f.nx - 1), Y = (float)(f.ny - 1), Z = (float)(f.nz - 1);
    if (p.x >= 0.f && p.y > 0.f && p.z >= 0.f && p.x <= X && p.y <= Y && p.z <= Z) return 0;
    int c = 42;
    const bool lx = p.x < X, ly = p.y < Y, lz = p.z < Z;
    if (p.x < 0.f && p.y >= 0.f && p.z >= 0.f && lx && ly && lz) c = 1;
    if (p.x >= 0.f && p.y >= 0.f && p.z >= 0.f && !lx && ly && lz) c = 2;
    if (p.x >= 0.f && p.y < 0.f && p.z >= 0.f && lx && ly && lz) c = 3;
    if (p.x >= 0.f && p.y >= 0.f && p.z >= 0.f && lx && !ly && lz) c = 4;
    if (p.x >= 0.f && p.y >= 0.f && p.z < 0.f && lx && ly && lz) c = 5;
    if (p.x >= 0.f && p.y >= 0.f && p.z >= 0.f && lx && ly && !lz) c = 6;
    return c;
}

// One line from p0 along dir * B (dir = +1 or -1).  Returns the face code;
// pout the end, len the path length, tw the twist integral (with TW).
template <bool TW>
__device__ int trace_line(const Field& f, F3 p0, F3 n0, float h, float tol_coef, float dir, F3& pout, double& len,
                          double& tw) {
    const double len_lim = STEP_RATIO * (double)(f.nx + f.ny + f.nz);
    const float bn0 = fabsf(dot3(interp_dir(f, p0, true), n0));
    float tol = (double)bn0 <= 0.05 ? (float)(TOL0 / 8e3) : (float)(TOL0 * powf(bn0, 1.5f));
    tol = tol * tol_coef;
    F3 p1 = p0;
    pout = p0;
    len = 0.0;
    tw = 0.0;
    int code = 0;
    long long steps = 0;
    while (code == 0 && len < len_lim && steps < MAX_STEPS) {
        float err;
        F3 p2 = rkf45(f, p1, h * dir, err);
        const float scale = powf((float)((double)(tol / err) / 11.09), 0.2f);
        if ((double)scale < 0.618) {
            h = (float)(h * 0.618);
            continue;
        }
        h = h * scale;
        if ((double)h > 100.0) h = 100.f;
        if ((double)h < 0.1) h = (float)0.1;
        const float dl = len3(p1 - p2);
        len += dl;
        double dtw = 0.0;
        if (TW) {
            const F3 c1 = interp_dir(f, p1, false, true);
            const F3 b1 = interp_dir(f, p1, false, false);
            dtw = (double)(dot3(c1, b1) / dot3(b1, b1)) / 4.0 / PI_REF * (double)dl;
            tw += dtw;
        }
        code = face_code(f, p2);
        if (code > 0) {
            len -= dl;
            if (TW) tw -= dtw;
            if (code <= 6) {
                const int d = (code - 1) / 2;
                const float q1 = comp(p1, d), q2 = comp(p2, d);
                if ((double)fabsf(q1 - q2) > 1e-3) {
                    const float qm = (code % 2 == 1) ? 0.f : (float)(d == 0 ? f.nx : (d == 1 ? f.ny : f.nz));
                    const F3 u1 = interp_dir(f, p1, true), u2 = interp_dir(f, p2, true);
                    if ((double)fabsf(comp(u1, d)) < 0.2 || (double)fabsf(comp(u2, d)) < 0.2) {
                        pout = f3((p1.x * (q2 - qm) + p2.x * (qm - q1)) / (q2 - q1),
                                  (p1.y * (q2 - qm) + p2.y * (qm - q1)) / (q2 - q1),
                                  (p1.z * (q2 - qm) + p2.z * (qm - q1)) / (q2 - q1));
                    } else {
                        p2 = rk4_face(f, p1, qm - q1, d);
                        pout = p2;
                    }
                    len += (double)fabsf(qm - q1) / (1e-4 + (double)fabsf(comp(u1, d)));
                } else {
                    pout = p1;
                }
            } else {
                pout = p2;
            }
        }
        p1 = p2;
        ++steps;
    }
    // a line stopped by the length or step limit ends where it stands
    if (code == 0) pout = p1;
    return code;
}

// Lines are handed out dynamically: each warp takes the next 32 of the 2n
// half-lines (t = dir * n + seed) from a global counter, so that warps that
// drew short lines move on while others finish long ones, and the lanes of a
// warp follow neighbouring lines.  (TraceAllBline runs both halves of a seed
// in one thread; each half's result is the same.)  dir 0 traces along +B to
// the end, dir 1 along -B to the start.  ends (2, n, 3): [0] end, [1] start;
// flags (2, n); bs (3, 3, n): B at the seed, the end and the start (x, y, z
// rows); bflag (n): 1 where |B.n| < |B| / 100 at the seed; half (2, 2, n):
// each half's path length and twist, summed by k_fq_sum; counter zeroed.
template <bool TW>
__global__ void __launch_bounds__(128) k_trace_fq(Field f, const float* __restrict__ seeds, long long n, F3 n0,
                                                  float h, float tol_coef, float* __restrict__ ends,
                                                  int* __restrict__ flags, float* __restrict__ bs,
                                                  int* __restrict__ bflag, double* __restrict__ half,
                                                  unsigned long long* __restrict__ counter) {
    const int lane = threadIdx.x & 31;
    const unsigned long long total = 2ull * (unsigned long long)n;
    for (;;) {
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(counter, 32ull);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) return;
        const unsigned long long tt = base + lane;
        if (tt >= total) continue;
        const long long t = (long long)tt;
        const int dir = t >= n ? 1 : 0;
        const long long si = t - (long long)dir * n;
        const F3 p0 = f3(seeds[3 * si], seeds[3 * si + 1], seeds[3 * si + 2]);
        F3 pe;
        double le, te;
        const int code = trace_line<TW>(f, p0, n0, h, tol_coef, dir == 0 ? 1.0f : -1.0f, pe, le, te);
        ends[3 * t] = pe.x; ends[3 * t + 1] = pe.y; ends[3 * t + 2] = pe.z;
        flags[t] = code;
        const F3 be = interp_sample(f, pe);
        bs[(0 * 3 + 1 + dir) * n + si] = be.x;
        bs[(1 * 3 + 1 + dir) * n + si] = be.y;
        bs[(2 * 3 + 1 + dir) * n + si] = be.z;
        half[t] = le;
        if (TW) half[2 * n + t] = te;
        if (dir == 0) {
            const F3 b0 = interp_sample(f, p0);
            bs[0 * n + si] = b0.x;
            bs[3 * n + si] = b0.y;
            bs[6 * n + si] = b0.z;
            bflag[si] = (double)fabsf(b0.x * n0.x + b0.y * n0.y + b0.z * n0.z) * 100.0 < (double)len3(b0) ? 1 : 0;
        }
    }
}

// length (n) = forward + backward half, twist likewise (the reference's
// order of the two additions)
__global__ void k_fq_sum(long long n, const double* __restrict__ half, double* __restrict__ len,
                         double* __restrict__ tw) {
    const long long si = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= n) return;
    len[si] = half[si] + half[n + si];
    if (tw != nullptr) tw[si] = half[2 * n + si] + half[3 * n + si];
}

// QCalcPlane on an nv x nu seed plane (seed u + nu v), the end of each seed
// projected on its face ((x, y) on z faces, (z, x) on y faces, (y, z) on x
// faces, 0 otherwise).
__device__ __forceinline__ void face_xy(const float* e, int code, float& X, float& Y) {
    const int d = code >= 1 ? (code - 1) / 2 : -1;
    if (d == 2) { X = e[0]; Y = e[1]; }
    else if (d == 1) { X = e[2]; Y = e[0]; }
    else if (d == 0) { X = e[1]; Y = e[2]; }
    else { X = 0.f; Y = 0.f; }
}

__global__ void k_qcalc_plane(int nu, int nv, const float* __restrict__ ends, const int* __restrict__ flags,
                              const float* __restrict__ bs, F3 n0, float stride, float* __restrict__ q) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    if (u >= nu || v >= nv) return;
    const long long n = (long long)nu * nv;
    const long long c = (long long)v * nu + u;
    if (u == 0 || v == 0 || u == nu - 1 || v == nv - 1) { q[c] = NAN; return; }
    const long long nb[4] = {c + nu, c - nu, c + 1, c - 1};  // +v, -v, +u, -u
    const int* fe = flags;       // end (forward)
    const int* fs = flags + n;   // start (backward)
    int mism = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) mism += abs(fs[nb[r]] - fs[c]) + abs(fe[nb[r]] - fe[c]);
    // end (2) and start (1) coordinates at the four neighbours
    float X2[4], Y2[4], X1[4], Y1[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        face_xy(ends + 3 * nb[r], fe[nb[r]], X2[r], Y2[r]);
        face_xy(ends + 3 * (n + nb[r]), fs[nb[r]], X1[r], Y1[r]);
    }
    // "xc": along the plane's rows (v), "yc": along its columns (u)
    const float dx2xc = X2[0] - X2[1], dx2yc = X2[2] - X2[3];
    const float dy2xc = Y2[0] - Y2[1], dy2yc = Y2[2] - Y2[3];
    const float dx1xc = X1[0] - X1[1], dx1yc = X1[2] - X1[3];
    const float dy1xc = Y1[0] - Y1[1], dy1yc = Y1[2] - Y1[3];
    // element-wise FP32 array arithmetic, no fused multiply-adds
    auto mul = [](float x, float y) { return __fmul_rn(x, y); };
    auto add = [](float x, float y) { return __fadd_rn(x, y); };
    auto sub = [](float x, float y) { return __fsub_rn(x, y); };
    const float a = sub(mul(dx2xc, dy1yc), mul(dx2yc, dy1xc));
    const float b = sub(mul(dx2yc, dx1xc), mul(dx2xc, dx1yc));
    const float cc = sub(mul(dy2xc, dy1yc), mul(dy2yc, dy1xc));
    const float d = sub(mul(dy2yc, dx1xc), mul(dy2xc, dx1yc));
    const float bnorm = add(add(mul(bs[0 * n + c], n0.x), mul(bs[3 * n + c], n0.y)), mul(bs[6 * n + c], n0.z));
    const float bz_start = bs[(2 * 3 + 2) * n + c], bz_end = bs[(2 * 3 + 1) * n + c];
    const float sc = __fdiv_rn(1.f, mul(2.f, stride));
    const float s4 = mul(mul(mul(sc, sc), sc), sc);
    const float bnr = mul(mul(__fdiv_rn(fabsf(bz_start), mul(fabsf(bnorm), fabsf(bnorm))), fabsf(bz_end)), s4);
    float Q = mul(add(add(add(mul(a, a), mul(b, b)), mul(cc, cc)), mul(d, d)), bnr);
    if (Q < 1.0f) Q = 1.0f;
    if (mism > 0) Q = NAN;
    q[c] = Q;
}

}  // namespace fq
