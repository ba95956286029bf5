// soft_cfcf start: for every horizontal mode, the z profile that minimises the
// modal curl(J) functional with the bottom value and the transparent top
// exact (nfgs_solver.py:6150-6484).
//
// One thread per mode, FP64.  The profile is an affine function of the free
// unknowns (nfgs_solver.py:6234-6270); each row of the functional is an
// affine expression over a few neighbouring unknowns, so the normal matrix is
// banded (half-width 4 for Phi, 2 for A_z).  A thread assembles its band and
// right-hand side in global scratch (index-major, mode-minor: the threads of a
// warp touch consecutive words), factors it in place by banded Cholesky with
// the reference's pivot floor (nfgs_solver.py:6272-6319), solves, and writes
// the profile into the modal buffer that the inverse transforms read.  Every
// product and sum is rounded on its own (no fused multiply-add) and taken in
// the reference's order: rows by height, keys ascending within a row, affine
// sums term by term.
#pragma once
#include "nfgs_common.cuh"
#include <float.h>

namespace soft {

constexpr int W = 8;           // coefficient window of one affine expression
constexpr int BWMAX = 4;       // widest band the rows produce
constexpr int BS = BWMAX + 1;  // band words per unknown

// error codes written to the flag word
constexpr int ERR_WINDOW = 1;     // an expression spans more than W unknowns
constexpr int ERR_BAND = 2;       // a row spans more than BWMAX + 1 unknowns
constexpr int ERR_NONFINITE = 3;  // the normal solve produced a non-finite value

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }

// sum_q c[q] u[lo + q] + k over the keys set in `mask`
struct Aff {
    int lo;
    unsigned mask;
    double c[W];
    double k;
};

__device__ __forceinline__ void aff_zero(Aff& a) {
    a.lo = 0;
    a.mask = 0u;
#pragma unroll
    for (int q = 0; q < W; ++q) a.c[q] = 0.0;
    a.k = 0.0;
}

__device__ __forceinline__ Aff aff_unit(int idx) {
    Aff a;
    aff_zero(a);
    a.lo = idx;
    a.mask = 1u;
    a.c[0] = 1.0;
    return a;
}

// sum_t s[t] e[t] with keys merged (nfgs_solver.py:6151-6170): a key's first
// contribution is 0.0 + s c, later ones add in term order; the constant is
// ((0 + s_0 k_0) + s_1 k_1) + ...
template <int NT>
__device__ __forceinline__ Aff combine(const double (&s)[NT], const Aff* const (&e)[NT], int* err) {
    Aff r;
    aff_zero(r);
    int lo = 0x7fffffff, hi = -1;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        if (e[t]->mask == 0u) continue;
        lo = min(lo, e[t]->lo);
        hi = max(hi, e[t]->lo + 31 - __clz(e[t]->mask));
    }
    if (hi >= 0) {
        if (hi - lo >= W) { *err = ERR_WINDOW; hi = lo + W - 1; }
        r.lo = lo;
    }
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const Aff& a = *e[t];
        r.k = add(r.k, mul(s[t], a.k));
#pragma unroll
        for (int q = 0; q < W; ++q) {
            if (!((a.mask >> q) & 1u)) continue;
            const int d = a.lo + q - r.lo;
            if (d < 0 || d >= W) continue;
            const double v = mul(s[t], a.c[q]);
            r.c[d] = ((r.mask >> d) & 1u) ? add(r.c[d], v) : add(0.0, v);
            r.mask |= 1u << d;
        }
    }
    return r;
}

struct Mode {
    int kind;      // 0 Phi (DCT-I modes), 1 A_z (interior DST-I modes)
    int nz;
    double k, k2, b, dz, denom;
};

// plane value z below the top as an affine expression
// (nfgs_solver.py:6234-6262)
__device__ Aff field_below_top(const Mode& m, int z) {
    if (z == 0) {
        Aff a;
        aff_zero(a);
        a.k = m.b;
        return a;
    }
    if (m.kind == 0) {
        if (z == 1) {
            Aff a = aff_unit(0);
            a.c[0] = 0.25;
            a.k = mul(add(0.75, mul(0.5 * m.dz, m.k)), m.b);
            return a;
        }
        return aff_unit(z - 2);
    }
    return aff_unit(z - 1);
}

// any plane: the top one from the transparent Robin row
// (3u_N - 4u_{N-1} + u_{N-2})/(2dz) + k u_N = 0 (nfgs_solver.py:6264-6269)
__device__ Aff field(const Mode& m, int z, int* err) {
    if (z < m.nz - 1) return field_below_top(m, z);
    const Aff f2 = field_below_top(m, m.nz - 2), f3 = field_below_top(m, m.nz - 3);
    const double s[2] = {4.0 / m.denom, -1.0 / m.denom};
    const Aff* const e[2] = {&f2, &f3};
    return combine<2>(s, e, err);
}

// L_k = D_zz - k^2 at an interior height (nfgs_solver.py:6201-6232, 6329-6335)
__device__ Aff lap_at(const Mode& m, int z, int* err) {
    const double i2 = 1.0 / (m.dz * m.dz);
    const Aff fa = field(m, z - 1, err), fb = field(m, z, err), fc = field(m, z + 1, err);
    const double s3[3] = {i2, -2.0 * i2, i2};
    const Aff* const e3[3] = {&fa, &fb, &fc};
    const Aff d2 = combine<3>(s3, e3, err);
    const double s2[2] = {1.0, -m.k2};
    const Aff* const e2[2] = {&d2, &fb};
    return combine<2>(s2, e2, err);
}

// first derivative (nfgs_solver.py:6172-6199) of the interior L_k list of a
// Phi mode (entry j is height j + 1, count nz - 2)
__device__ Aff dlap_at(const Mode& m, int j, int* err) {
    const double h = 1.0 / (2.0 * m.dz);
    const int cnt = m.nz - 2;
    if (j == 0) {
        const Aff a = lap_at(m, 1, err), b = lap_at(m, 2, err), c = lap_at(m, 3, err);
        const double s[3] = {-3.0 * h, 4.0 * h, -h};
        const Aff* const e[3] = {&a, &b, &c};
        return combine<3>(s, e, err);
    }
    if (j == cnt - 1) {
        const Aff a = lap_at(m, cnt, err), b = lap_at(m, cnt - 1, err), c = lap_at(m, cnt - 2, err);
        const double s[3] = {3.0 * h, -4.0 * h, h};
        const Aff* const e[3] = {&a, &b, &c};
        return combine<3>(s, e, err);
    }
    const Aff a = lap_at(m, j, err), b = lap_at(m, j + 2, err);
    const double s[2] = {-h, h};
    const Aff* const e[2] = {&a, &b};
    return combine<2>(s, e, err);
}

// centred first derivative of the plane values at an interior height
__device__ Aff dfield_at(const Mode& m, int z, int* err) {
    const double h = 1.0 / (2.0 * m.dz);
    const Aff a = field(m, z - 1, err), b = field(m, z + 1, err);
    const double s[2] = {-h, h};
    const Aff* const e[2] = {&a, &b};
    return combine<2>(s, e, err);
}

// number of rows of the functional and row r with its weight
// (nfgs_solver.py:6337-6359)
__device__ __forceinline__ int row_count(const Mode& m, double eps) {
    return m.kind == 0 ? 2 * (m.nz - 2) : (eps > 0.0 ? 3 : 1) * (m.nz - 2);
}

__device__ Aff row_at(const Mode& m, double eps, int r, double* w, int* err) {
    if (m.kind == 0) {
        const int j = r >> 1;
        if ((r & 1) == 0) { *w = 1.0; return dlap_at(m, j, err); }
        *w = mul(1.0, add(m.k2, eps));
        return lap_at(m, j + 1, err);
    }
    const int per = eps > 0.0 ? 3 : 1;
    const int z = 1 + r / per, q = r % per;
    if (q == 0) { *w = 1.0; return lap_at(m, z, err); }
    if (q == 1) { *w = mul(1.0, eps); return dfield_at(m, z, err); }
    *w = mul(mul(1.0, eps), m.k2);
    return field(m, z, err);
}

// Profiles of modes m0 .. m0+cnt-1 of M.  kind 0: k = kk[m]; kind 1:
// k = sqrt(max(-lam[m], 0)).  Writes hat[z*M + m] for z = 1..nz-1 (storage
// type), and per-mode energies en[m] (curl-current) and en[M + m] (current),
// DCT endpoint weights applied for Phi (nfgs_solver.py:6486-6540).
// Scratch: band[(i*BS + d)*CH + t], vec[i*CH + t] for the chunk's thread t.
template <typename T>
__global__ void __launch_bounds__(128, 4) k_soft_profile(Geo g, int kind, long long m0, long long cnt, long long M,
                                                      const double* __restrict__ kk, const double* __restrict__ bot,
                                                      double eps, double ridge, long long CH,
                                                      double* __restrict__ band, double* __restrict__ vec,
                                                      T* __restrict__ hat, double* __restrict__ en, int* errflag) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= cnt) return;
    const long long mi = m0 + t;
    const int nz = g.nz;
    Mode md;
    md.kind = kind;
    md.nz = nz;
    md.k = kind == 0 ? kk[mi] : sqrt(fmax(-kk[mi], 0.0));
    md.k2 = mul(md.k, md.k);
    md.b = bot[mi];
    md.dz = g.dz;
    md.denom = add(3.0, mul(2.0 * g.dz, md.k));
    const int nx = g.nx, ny = g.ny;
    double wmode = 1.0;
    if (kind == 0) {
        const long long jy = mi / nx, ix = mi - jy * nx;
        wmode = ((ix == 0 || ix == nx - 1) ? 0.5 : 1.0) * ((jy == 0 || jy == ny - 1) ? 0.5 : 1.0);
    }
    if (!(md.k > 0.0)) {
        // inactive mode: zero profile (nfgs_solver.py:6407-6420)
        for (int z = 1; z < nz; ++z) hat[(long long)z * M + mi] = T(0);
        en[mi] = 0.0;
        en[M + mi] = 0.0;
        return;
    }
    int err = 0;
    const int n = kind == 0 ? nz - 3 : nz - 2;
    auto B = [&](int i, int d) -> double& { return band[((long long)i * BS + d) * CH + t]; };
    auto X = [&](int i) -> double& { return vec[(long long)i * CH + t]; };
    for (int i = 0; i < n; ++i) {
#pragma unroll
        for (int d = 0; d < BS; ++d) B(i, d) = 0.0;
        X(i) = 0.0;
    }
    // normal equations (nfgs_solver.py:6361-6383)
    int bw = 0;
    const int nr = row_count(md, eps);
    for (int r = 0; r < nr; ++r) {
        double w;
        const Aff e = row_at(md, eps, r, &w, &err);
        if (e.mask == 0u) continue;
        const int span = 31 - __clz(e.mask) - (__ffs(e.mask) - 1);
        if (span > BWMAX) { err = ERR_BAND; break; }
        bw = max(bw, span);
#pragma unroll
        for (int qi = 0; qi < W; ++qi) {
            if (!((e.mask >> qi) & 1u)) continue;
            const int ia = e.lo + qi;
            const double wci = mul(w, e.c[qi]);
            X(ia) = add(X(ia), mul(wci, e.k));
#pragma unroll
            for (int qj = 0; qj <= qi; ++qj) {
                if (!((e.mask >> qj) & 1u)) continue;
                const int d = qi - qj;
                B(ia, d) = add(B(ia, d), mul(wci, e.c[qj]));
            }
        }
    }
    // ridge on the diagonal, pivot floor (nfgs_solver.py:6384-6389, 6281-6283)
    double dmax = 0.0;
    for (int i = 0; i < n; ++i) dmax = fmax(dmax, fabs(B(i, 0)));
    const double dsc = fmax(dmax, 1.0);
    dmax = 0.0;
    for (int i = 0; i < n; ++i) {
        const double v = add(B(i, 0), mul(ridge, dsc));
        B(i, 0) = v;
        dmax = fmax(dmax, fabs(v));
    }
    const double floor_ = mul(DBL_EPSILON, fmax(dmax, 1.0));
    // banded Cholesky in place: B(r, d) becomes the factor entry (r, r - d)
    for (int i = 0; i < n && !err; ++i) {
        double dg = B(i, 0);
        for (int o = 1; o <= min(bw, i); ++o) {
            const double f = B(i, o);
            dg = sub(dg, mul(f, f));
        }
        const double piv = __dsqrt_rn(fmax(dg, floor_));
        B(i, 0) = piv;
        for (int r = i + 1; r < min(n, i + bw + 1); ++r) {
            double v = B(r, r - i);
            for (int c = max(max(0, i - bw), r - bw); c < i; ++c) v = sub(v, mul(B(r, r - c), B(i, i - c)));
            B(r, r - i) = __ddiv_rn(v, piv);
        }
    }
    // forward (rhs = -gradient) and back substitution, in place
    for (int i = 0; i < n; ++i) {
        double v = -X(i);
        for (int o = 1; o <= min(bw, i); ++o) v = sub(v, mul(B(i, o), X(i - o)));
        X(i) = __ddiv_rn(v, B(i, 0));
    }
    bool finite = true;
    for (int i = n - 1; i >= 0; --i) {
        double v = X(i);
        for (int r = i + 1; r < min(n, i + bw + 1); ++r) v = sub(v, mul(B(r, r - i), X(r)));
        v = __ddiv_rn(v, B(i, 0));
        X(i) = v;
        finite = finite && isfinite(v);
    }
    if (!finite && !err) err = ERR_NONFINITE;
    if (err) {
        atomicMax(errflag, err);
        for (int z = 1; z < nz; ++z) hat[(long long)z * M + mi] = T(0);
        en[mi] = 0.0;
        en[M + mi] = 0.0;
        return;
    }
    // plane values (nfgs_solver.py:6398-6405): constant, then the keys in
    // insertion order; the top plane's keys were inserted high index first
    for (int z = 1; z < nz; ++z) {
        double v;
        if (z == nz - 1) {
            const int hi = kind == 0 ? nz - 4 : nz - 3;
            v = add(0.0, mul(4.0 / md.denom, X(hi)));
            v = add(v, mul(-1.0 / md.denom, X(hi - 1)));
        } else if (kind == 0 && z == 1) {
            v = add(mul(add(0.75, mul(0.5 * md.dz, md.k)), md.b), mul(0.25, X(0)));
        } else {
            v = add(0.0, X(kind == 0 ? z - 2 : z - 1));
        }
        hat[(long long)z * M + mi] = (T)v;
    }
    // modal energies of the stored profile (nfgs_solver.py:6486-6540)
    const double dz = g.dz, i2 = 1.0 / (dz * dz), h = 1.0 / (2.0 * dz);
    auto P_ = [&](int z) -> double { return z == 0 ? (double)(T)md.b : (double)hat[(long long)z * M + mi]; };
    auto Q_ = [&](int j) -> double { return (P_(j + 2) - 2.0 * P_(j + 1) + P_(j)) * i2 - md.k2 * P_(j + 1); };
    const int nq = nz - 2;
    double s_cur = 0.0, s_curl = 0.0;
    for (int j = 0; j < nq; ++j) {
        const double q = Q_(j);
        if (kind == 0) {
            double dq;
            if (j == 0) dq = (-3.0 * q + 4.0 * Q_(1) - Q_(2)) * h;
            else if (j == nq - 1) dq = (3.0 * q - 4.0 * Q_(j - 1) + Q_(j - 2)) * h;
            else dq = (Q_(j + 1) - Q_(j - 1)) * h;
            s_cur += q * q;
            s_curl += dq * dq + md.k2 * q * q;
        } else {
            const double da = (P_(j + 2) - P_(j)) * h, a = P_(j + 1);
            s_cur += da * da + md.k2 * a * a;
            s_curl += q * q;
        }
    }
    en[mi] = wmode * (md.k2 * s_curl);
    en[M + mi] = wmode * (md.k2 * s_cur);
}

// Fixed-order sum of the per-mode energies: out[0] = sum en[0..M),
// out[1] = sum en[M..2M).  One block of 256 threads.
__global__ void k_soft_sum(const double* __restrict__ en, long long M, double* __restrict__ out) {
    __shared__ double sh[2 * 32];
    double v[2] = {0.0, 0.0};
    for (long long i = threadIdx.x; i < M; i += blockDim.x) {
        v[0] += en[i];
        v[1] += en[M + i];
    }
    block_reduce<2>(v, sh);
    if (threadIdx.x == 0) {
        out[0] = v[0];
        out[1] = v[1];
    }
}

}  // namespace soft
