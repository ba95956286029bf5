// Per-iteration kernels of the NFGS NFPT loop.
//
// State: (Phi_c, A_z) per state buffer; B and J are reconstructions of
// them (nfgs_solver.py:5901-5942 -> 3311-3341).  The pass structure:
//   k_recon  : Phi_c, A_z -> B (3 comps) and state J_z
//   k_face   : B, J_z -> vertical-face current, sigma_J / divB / energy
//              partial sums, face-aligned current alpha_f B_f
//   k_src    : face current -> J_parallel at centres -> S_B, S_J
//   transforms + k_zsolve (modal Robin and Dirichlet chains)
//   k_ctl    : reductions and the stop rule (one thread)
#pragma once
#include "nfgs_common.cuh"

struct Box { int z0, z1, y0, y1, x0, x1; };  // half-open cwsin box on faces

struct StateTab {
    void* phi[3];
    void* az[3];
};

template <typename T> __device__ __forceinline__ T ldg(const T* p, long long i) { return __ldg(p + i); }

// Second-order centred derivative with one-sided three-point ends
// (nfgs_solver.py:1361-1419).  f(q) returns the sample at index q.
template <typename T, typename F>
__device__ __forceinline__ T d1(F f, int i, int n, T inv2h) {
    if (i == 0) return (T(-3) * f(0) + T(4) * f(1) - f(2)) * inv2h;
    if (i == n - 1) return (T(3) * f(n - 1) - T(4) * f(n - 2) + f(n - 3)) * inv2h;
    return (f(i + 1) - f(i - 1)) * inv2h;
}

// One axis of the mirrored-Neumann horizontal Laplacian numerator
// (nfgs_solver.py:1741-1749), without the 1/h^2 factor.
template <typename T, typename F>
__device__ __forceinline__ T lap1(F f, int i, int n) {
    if (i == 0) return T(2) * f(1) - T(2) * f(0);
    if (i == n - 1) return T(2) * f(n - 2) - T(2) * f(n - 1);
    return f(i + 1) - T(2) * f(i) + f(i - 1);
}

// ---------------------------------------------------------------------------
// k_recon: carrier C = B - B_background = (Bc_x + H_x, Bc_y + H_y, Bc_z) with
// C_z(0) = Bz_obs - B_background,z(0) (B_z(0) = Bz_obs), and the state
// J_z = -lap_xy A_z with zero walls/top and J_z(0) = Jz_T.  The carrier is
// formed directly: the reference forms it as (B_bg + B_c + H) - B_bg
// (nfgs_solver.py:5759), which in FP32 cancels where B_c << B_bg.
//
// With a k_h=0 closure (hk3 != null) H is the selected buffer's profile by
// plane, which block (0, 0, k) also copies to hsel for the kernels that
// follow; with the constrained spline the state J_z is the face average
// mapped back to the planes (nfgs_solver.py:5915-5935: all three current
// components come from the face current there).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_recon(Geo g, StateTab st, const int* sel, const int* skip,
                                               const T* __restrict__ bbg, const T* __restrict__ bzobs,
                                               const T* __restrict__ jzt, T hx, T hy, int use_h,
                                               T* __restrict__ Bout, T* __restrict__ jzout,
                                               const double* __restrict__ hk3 = nullptr,
                                               double* __restrict__ hsel = nullptr, int spline = 0) {
    if (skip != nullptr && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const T* __restrict__ phi = (const T*)st.phi[*sel];
    const T* __restrict__ az = (const T*)st.az[*sel];
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P;
    const T i2dx = T(1.0 / (2.0 * g.dx)), i2dy = T(1.0 / (2.0 * g.dy)), i2dz = T(1.0 / (2.0 * g.dz));
    const T idx2 = T(1.0 / (g.dx * g.dx)), idy2 = T(1.0 / (g.dy * g.dy));
    auto PH = [&](int kk, int jj, int ii) -> T { return ldg(phi, kk * P + (long long)jj * nx + ii); };
    auto AZ = [&](int kk, int jj, int ii) -> T { return ldg(az, kk * P + (long long)jj * nx + ii); };
    auto dzphi = [&](int jj, int ii) -> T {
        return d1<T>([&](int q) { return PH(q, jj, ii); }, k, nz, i2dz);
    };
    const long long c = k * P + (long long)j * nx + i;
    // Bc_x = -Dx(Dz Phi) + Dy A ; Bc_y = -Dy(Dz Phi) - Dx A
    T dxdz = d1<T>([&](int q) { return dzphi(j, q); }, i, nx, i2dx);
    T dydz = d1<T>([&](int q) { return dzphi(q, i); }, j, ny, i2dy);
    T dya = d1<T>([&](int q) { return AZ(k, q, i); }, j, ny, i2dy);
    T dxa = d1<T>([&](int q) { return AZ(k, j, q); }, i, nx, i2dx);
    T bcx = -dxdz + dya;
    T bcy = -dydz - dxa;
    T bcz = lap1<T>([&](int q) { return PH(k, j, q); }, i, nx) * idx2 +
            lap1<T>([&](int q) { return PH(k, q, i); }, j, ny) * idy2;
    T cx = bcx, cy = bcy, cz = bcz;
    if (hk3 != nullptr) {
        const double* hp = hk3 + (long long)(*sel) * 2 * nz;
        cx = cx + (T)hp[k];
        cy = cy + (T)hp[nz + k];
        if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
            hsel[k] = hp[k];
            hsel[nz + k] = hp[nz + k];
        }
    } else if (use_h) {
        cx = cx + hx;
        cy = cy + hy;
    }
    if (k == 0) cz = ldg(bzobs, (long long)j * nx + i) - ldg(bbg, 2 * g.V + c);
    Bout[c] = cx;
    Bout[g.V + c] = cy;
    Bout[2 * g.V + c] = cz;
    const bool wall = i == 0 || i == nx - 1 || j == 0 || j == ny - 1;
    // state J_z of plane kk: J_z(0) = Jz_T, zero walls and top, -lap_xy A_z
    auto jzp = [&](int kk) -> T {
        if (kk == 0) return ldg(jzt, (long long)j * nx + i);
        if (kk == nz - 1 || wall) return T(0);
        return -(lap1<T>([&](int q) { return AZ(kk, j, q); }, i, nx) * idx2 +
                 lap1<T>([&](int q) { return AZ(kk, q, i); }, j, ny) * idy2);
    };
    T jz = jzp(k);
    if (spline && k >= 1 && k <= nz - 2 && !wall) {
        const T f0 = T(0.5) * (jz + jzp(k - 1));
        const T f1 = T(0.5) * (jzp(k + 1) + jz);
        jz = T(0.5) * (f0 + f1);
    }
    jzout[c] = jz;
}

// ---------------------------------------------------------------------------
// k_face: centre divB/|B|/|B|^2 sums and, on face f = k (k < nz-1), the
// staggered carrier curl (nfgs_solver.py:5738-5778), sigma_J terms on the
// cwsin box (nfgs_solver.py:5882-5895, 2656-2676) and the face-aligned
// current alpha_f B_f (nfgs_solver.py:5841-5853).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_face(Geo g, const int* skip, const T* __restrict__ B,
                                              const T* __restrict__ bbg, const T* __restrict__ jz, Box box,
                                              T alpha_max, T floor_b2, T* __restrict__ jpf,
                                              T* __restrict__ jb, double* __restrict__ partials, int raw_j,
                                              const double* __restrict__ jh_wall = nullptr) {
    __shared__ double sh[NFGS_NRED * 32];
    if (skip != nullptr && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    double red[5] = {0, 0, 0, 0, 0};
    if (i < nx && j < ny) {
        const long long c = k * P + (long long)j * nx + i;
        const T i2dx = T(1.0 / (2.0 * g.dx)), i2dy = T(1.0 / (2.0 * g.dy)), i2dz = T(1.0 / (2.0 * g.dz));
        const T idz = T(1.0 / g.dz);
        // B holds the carrier C; the field is B_background + C
        auto BX = [&](int kk, int jj, int ii) -> T {
            long long q = kk * P + (long long)jj * nx + ii;
            return ldg(bbg, q) + ldg(B, q);
        };
        auto BY = [&](int kk, int jj, int ii) -> T {
            long long q = V + kk * P + (long long)jj * nx + ii;
            return ldg(bbg, q) + ldg(B, q);
        };
        auto BZ = [&](int kk, int jj, int ii) -> T {
            long long q = 2 * V + kk * P + (long long)jj * nx + ii;
            return ldg(bbg, q) + ldg(B, q);
        };
        T bx = BX(k, j, i), by = BY(k, j, i), bz = BZ(k, j, i);
        T div = d1<T>([&](int q) { return BX(k, j, q); }, i, nx, i2dx) +
                d1<T>([&](int q) { return BY(k, q, i); }, j, ny, i2dy) +
                d1<T>([&](int q) { return BZ(q, j, i); }, k, nz, i2dz);
        T bm = sqrt(bx * bx + by * by + bz * bz);
        red[2] = fabs((double)div);
        red[3] = (double)bm;
        red[4] = (double)(bx * bx + by * by + bz * bz);
        if (k < nz - 1) {
            const long long c1 = c + P;
            T bx1 = BX(k + 1, j, i), by1 = BY(k + 1, j, i), bz1 = BZ(k + 1, j, i);
            T bfx = T(0.5) * (bx1 + bx), bfy = T(0.5) * (by1 + by), bfz = T(0.5) * (bz1 + bz);
            auto CZF = [&](int jj, int ii) -> T {
                long long q0 = 2 * V + k * P + (long long)jj * nx + ii;
                return T(0.5) * (ldg(B, q0 + P) + ldg(B, q0));
            };
            T cx0 = ldg(B, c), cx1 = ldg(B, c1);
            T cy0 = ldg(B, V + c), cy1 = ldg(B, V + c1);
            T dbx = (cx1 - cx0) * idz;
            T dby = (cy1 - cy0) * idz;
            T jxf = d1<T>([&](int q) { return CZF(q, i); }, j, ny, i2dy) - dby;
            T jyf = dbx - d1<T>([&](int q) { return CZF(j, q); }, i, nx, i2dx);
            T jzf = T(0.5) * (ldg(jz, c1) + ldg(jz, c));
            if (k >= box.z0 && k < box.z1 && j >= box.y0 && j < box.y1 && i >= box.x0 && i < box.x1) {
                T cxp = jyf * bfz - jzf * bfy;
                T cyp = jzf * bfx - jxf * bfz;
                T czp = jxf * bfy - jyf * bfx;
                T bn = sqrt(bfx * bfx + bfy * bfy + bfz * bfz);
                bn = bn > T(1e-10) ? bn : T(1e-10);
                red[0] = (double)(sqrt(cxp * cxp + cyp * cyp + czp * czp) / bn);
                red[1] = (double)sqrt(jxf * jxf + jyf * jyf + jzf * jzf);
            }
            T b2 = bfx * bfx + bfy * bfy + bfz * bfz;
            b2 = b2 > floor_b2 ? b2 : floor_b2;
            T alpha = (jxf * bfx + jyf * bfy + jzf * bfz) / b2;
            if (alpha_max > T(0)) alpha = fmin(fmax(alpha, -alpha_max), alpha_max);
            const long long f = k * P + (long long)j * nx + i;
            const long long FV = (long long)(nz - 1) * P;
            if (raw_j) {
                jpf[f] = jxf;
                jpf[FV + f] = jyf;
                jpf[2 * FV + f] = jzf;
            } else {
                jpf[f] = alpha * bfx;
                jpf[FV + f] = alpha * bfy;
                jpf[2 * FV + f] = alpha * bfz;
            }
            if (k == 0) {
                // the state current on the bottom plane: zero walls, or the
                // open harmonic current of the constrained spline there
                // (nfgs_solver.py:5920-5933)
                bool wall = (i == 0 || i == nx - 1 || j == 0 || j == ny - 1);
                T wx = T(0), wy = T(0);
                if (jh_wall != nullptr) {
                    const double dz = g.dz;
                    const int n = nz;
                    const double* hp = jh_wall;
                    const double dhx = (-3.0 * hp[0] + 4.0 * hp[1] - hp[2]) / (2.0 * dz);
                    const double dhy = (-3.0 * hp[n] + 4.0 * hp[n + 1] - hp[n + 2]) / (2.0 * dz);
                    wx = (T)(-dhy);
                    wy = (T)dhx;
                }
                jb[(long long)j * nx + i] = wall ? wx : jxf;
                jb[P + (long long)j * nx + i] = wall ? wy : jyf;
            }
        }
    }
    block_reduce<5>(red, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
#pragma unroll
        for (int q = 0; q < 5; ++q) partials[q * nb + b] = red[q];
    }
}

// ---------------------------------------------------------------------------
// k_src: J_parallel at centres (faces -> centres, bottom row rule,
// optional buffer window; nfgs_solver.py:6697-6716) and the sources
//   S_B = Dy Jp_x - Dx Jp_y                         (nfgs_solver.py:6726)
//   S_J = lap_xy Jp_z - D2xz Jp_x - D2yz Jp_y       (nfgs_solver.py:6730-6745)
// ---------------------------------------------------------------------------
struct SrcOpts {
    int polarity;     // 0 both, 1 positive, 2 negative
    int face_exact;   // bottom_parallel_current_mode == face_parallel_exact_jz
    int window;       // buffer window present
};

template <typename T>
__global__ void __launch_bounds__(128) k_src(Geo g, const int* skip, const T* __restrict__ jpf,
                                             const T* __restrict__ jb, const T* __restrict__ jzt,
                                             const T* __restrict__ bzobs, SrcOpts o, const T* __restrict__ wx,
                                             const T* __restrict__ wy, const T* __restrict__ wz,
                                             T* __restrict__ sb, T* __restrict__ sj, double* __restrict__ partials,
                                             double* __restrict__ kpart = nullptr) {
    __shared__ double sh[NFGS_NRED * 32];
    if (skip != nullptr && *skip) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P;
    const long long FV = (long long)(nz - 1) * P;
    double red[1] = {0};
    double kz[4] = {0, 0, 0, 0};
    if (i < nx && j < ny) {
        auto JP = [&](int comp, int kk, int jj, int ii) -> T {
            const long long q = (long long)jj * nx + ii;
            T v;
            if (kk == 0) {
                if (o.polarity == 0) {
                    if (comp == 2) v = ldg(jzt, q);
                    else if (o.face_exact) v = ldg(jpf, comp * FV + q);
                    else v = ldg(jb, comp * P + q);
                } else {
                    T bzv = ldg(bzobs, q);
                    bool m = (o.polarity == 1) ? (bzv > T(0)) : (bzv < T(0));
                    T base = (comp == 2) ? ldg(jzt, q) : ldg(jb, comp * P + q);
                    v = m ? base : T(0);
                }
            } else if (kk == nz - 1) {
                v = ldg(jpf, comp * FV + (long long)(nz - 2) * P + q);
            } else {
                v = T(0.5) * (ldg(jpf, comp * FV + (long long)(kk - 1) * P + q) +
                              ldg(jpf, comp * FV + (long long)kk * P + q));
            }
            if (o.window) v = v * (ldg(wz, kk) * ldg(wy, jj) * ldg(wx, ii));
            return v;
        };
        const T i2dx = T(1.0 / (2.0 * g.dx)), i2dy = T(1.0 / (2.0 * g.dy));
        T s_b = d1<T>([&](int q) { return JP(0, k, q, i); }, j, ny, i2dy) -
                d1<T>([&](int q) { return JP(1, k, j, q); }, i, nx, i2dx);
        const long long c = k * P + (long long)j * nx + i;
        sb[c] = s_b;
        red[0] = (double)s_b * (double)s_b;
        if (kpart != nullptr) {
            // plane sums for the k_h=0 closure: the parallel current with the
            // DCT-I zero-mode weights (nfgs_solver.py:4466-4468, 5944-5950)
            // and the face-aligned current of face k (nfgs_solver.py:5876-5879)
            const double w = (i == 0 || i == nx - 1 ? 1.0 : 2.0) * (j == 0 || j == ny - 1 ? 1.0 : 2.0);
            kz[0] = w * (double)JP(0, k, j, i);
            kz[1] = w * (double)JP(1, k, j, i);
            if (k < nz - 1) {
                kz[2] = (double)ldg(jpf, (long long)k * P + (long long)j * nx + i);
                kz[3] = (double)ldg(jpf, FV + (long long)k * P + (long long)j * nx + i);
            }
        }
        if (k >= 1 && k <= nz - 2 && i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
            const T idx2 = T(1.0 / (g.dx * g.dx)), idy2 = T(1.0 / (g.dy * g.dy));
            const T i4xz = T(1.0 / (4.0 * g.dx * g.dz)), i4yz = T(1.0 / (4.0 * g.dy * g.dz));
            T jz0 = JP(2, k, j, i);
            T lap = (JP(2, k, j, i + 1) - T(2) * jz0 + JP(2, k, j, i - 1)) * idx2 +
                    (JP(2, k, j + 1, i) - T(2) * jz0 + JP(2, k, j - 1, i)) * idy2;
            T dxz = (JP(0, k + 1, j, i + 1) - JP(0, k - 1, j, i + 1) - JP(0, k + 1, j, i - 1) +
                     JP(0, k - 1, j, i - 1)) * i4xz;
            T dyz = (JP(1, k + 1, j + 1, i) - JP(1, k - 1, j + 1, i) - JP(1, k + 1, j - 1, i) +
                     JP(1, k - 1, j - 1, i)) * i4yz;
            const long long ci = (long long)k * (nx - 2) * (ny - 2) + (long long)(j - 1) * (nx - 2) + (i - 1);
            sj[ci] = lap - dxz - dyz;
        }
    }
    block_reduce<1>(red, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        partials[b] = red[0];
    }
    if (kpart != nullptr) {
        __syncthreads();
        block_reduce<4>(kz, sh);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
            for (int q = 0; q < 4; ++q) kpart[4 * b + q] = kz[q];
        }
    }
}

// ---------------------------------------------------------------------------
// Modal z-solves.  Factor tables hold, per mode and row, the Thomas
// coefficient c'_r and 1/denominator_r in FP64.  They depend only on the
// grid and rho, so they are built once per boundary.  Beyond row rconv[m]
// both values equal their converged limits (checked bitwise when the
// tables are built), which are kept in registers instead of being re-read.
// ---------------------------------------------------------------------------
// Rows per batch of independent loads in the z-solves: rows whose factors
// still come from the tables load them with the values (ZB rows); rows past
// the warp's largest rconv use the converged factors held in registers and
// load only the values (ZBV rows: 32 in FP32, 16 in FP64), so a thread needs
// few round trips to memory with 64 registers, and both chains of the
// benchmark grid fit on the GPU in one wave.
#define ZB 8
template <typename T>
struct ZRows {
    static constexpr int V = 64 / (int)sizeof(T);
};

struct ZTab {
    const double* c;      // [rows][modes]
    const double* inv;    // [rows][modes]
    const double* inv_last;
    const double* c_inf;
    const double* i_inf;
    const int* rconv;
};

// Forward elimination over rows r_lo..r_hi (row r at plane r + 1):
// d = (hat * sc - low * d) * inv_r, inv_r from the table below row rc and
// iinf from it on; s_last is the scaled source of the last row.  Addresses
// advance by the plane stride, so a batch holds only its values.
template <typename T, int B, bool TAB>
__device__ __forceinline__ void zs_forward(T* __restrict__ hat, long long stride, long long m, int r_lo, int r_hi,
                                           double sc, double low, double& d, double& s_last,
                                           const double* __restrict__ inv, int rc, double iinf) {
    for (int r0 = r_lo; r0 <= r_hi; r0 += B) {
        T sv[B];
        double ivb[TAB ? B : 1];
        T* const row0 = hat + (long long)(r0 + 1) * stride + m;
        {
            const T* q = row0;
            const double* ti = inv + (long long)r0 * stride + m;
#pragma unroll
            for (int u = 0; u < B; ++u, q += stride, ti += stride) {
                const int r = r0 + u;
                sv[u] = (r <= r_hi) ? *q : T(0);
                if constexpr (TAB) ivb[u] = (r <= r_hi && r < rc) ? *ti : iinf;
            }
        }
        T* q = row0;
#pragma unroll
        for (int u = 0; u < B; ++u, q += stride) {
            const int r = r0 + u;
            if (r <= r_hi) {
                const double s = (double)sv[u] * sc;
                s_last = s;
                if constexpr (TAB) d = (s - low * d) * ivb[u];
                else d = (s - low * d) * iinf;
                *q = (T)d;
            }
        }
    }
}

// Back substitution over rows r_hi down to r_lo: u = hat - c_r u.
template <typename T, int B, bool TAB>
__device__ __forceinline__ void zs_back(T* __restrict__ hat, long long stride, long long m, int r_hi, int r_lo,
                                        double& u, const double* __restrict__ c, int rc, double cinf) {
    for (int r0 = r_hi; r0 >= r_lo; r0 -= B) {
        T dv[B];
        double crb[TAB ? B : 1];
        T* const row0 = hat + (long long)(r0 + 1) * stride + m;
        {
            const T* q = row0;
            const double* tc = c + (long long)r0 * stride + m;
#pragma unroll
            for (int k = 0; k < B; ++k, q -= stride, tc -= stride) {
                const int r = r0 - k;
                dv[k] = (r >= r_lo) ? *q : T(0);
                if constexpr (TAB) crb[k] = (r >= r_lo && r < rc) ? *tc : cinf;
            }
        }
        T* q = row0;
#pragma unroll
        for (int k = 0; k < B; ++k, q -= stride) {
            const int r = r0 - k;
            if (r >= r_lo) {
                if constexpr (TAB) u = (double)dv[k] - crb[k] * u;
                else u = (double)dv[k] - cinf * u;
                *q = (T)u;
            }
        }
    }
}

// Both sweeps of rows 0..last (hat rows at planes 1..last+1); row 0's
// forward value d0 and the row after last (the closing row, solved by the
// caller between the sweeps) are handled outside.  rcw >= rc: the warp's
// split between table rows and converged rows.
template <typename T>
struct ZSweep {
    T* hat;
    long long stride, m;
    int rc, rcw;
    const double* inv;
    const double* c;
    double iinf, cinf;
    __device__ __forceinline__ void forward(int last, double sc, double low, double& d, double& s_last) const {
        const int a_hi = min(rcw - 1, last);
        if (a_hi >= 1) zs_forward<T, ZB, true>(hat, stride, m, 1, a_hi, sc, low, d, s_last, inv, rc, iinf);
        zs_forward<T, ZRows<T>::V, false>(hat, stride, m, max(1, rcw), last, sc, low, d, s_last, inv, rc, iinf);
    }
    __device__ __forceinline__ void back(int last, double& u) const {
        zs_back<T, ZRows<T>::V, false>(hat, stride, m, last, max(0, rcw), u, c, rc, cinf);
        const int a_hi = min(rcw - 1, last);
        if (a_hi >= 0) zs_back<T, ZB, true>(hat, stride, m, a_hi, 0, u, c, rc, cinf);
    }
};

// Robin chain (nfgs_solver.py:5512-5625 with 5627-5672): unknown planes
// 1..nz-1, rhs_r = S_hat(plane r+1) / lambda (FP64), mode (0,0) forced 0.
template <typename T>
__device__ void zsolve_robin_mode(Geo g, long long m, T* __restrict__ hat, ZTab t, const double* __restrict__ lam,
                                  const double* __restrict__ bot_hat, const double* __restrict__ der_hat,
                                  double rho, double* __restrict__ s00, int rcw) {
    const long long P = g.P;
    const int nz = g.nz;
    const int n = nz - 1;
    if (m == 0) {
        // the (0,0) profile for the zero-mode diagnostic, loaded in batches
        for (int p0 = 0; p0 < nz; p0 += ZRows<T>::V) {
            T v[ZRows<T>::V];
#pragma unroll
            for (int q = 0; q < ZRows<T>::V; ++q) v[q] = (p0 + q < nz) ? hat[(long long)(p0 + q) * P] : T(0);
#pragma unroll
            for (int q = 0; q < ZRows<T>::V; ++q) {
                const int p = p0 + q;
                if (p < nz) {
                    if (s00 != nullptr) s00[p] = (double)v[q];
                    if (p >= 1) hat[(long long)p * P] = T(0);
                }
            }
        }
        return;
    }
    const double dz = g.dz, dz2 = dz * dz, low = 1.0 / dz2;
    const double ls = lam[m];
    const double ils = 1.0 / ls;
    const int rc = t.rconv[m];
    double rhs0;
    double s1 = (double)hat[P + m] * ils;
    if (rho > 0.0) {
        rhs0 = (1.0 - rho) * s1 - rho * der_hat[m] / dz - ((1.0 + 0.5 * rho) / dz2) * bot_hat[m];
    } else {
        rhs0 = s1 - low * bot_hat[m];
    }
    double d = rhs0 * t.inv[m];
    hat[P + m] = (T)d;
    double s_last = s1;  // source of plane nz-2 (used again by the Robin row)
    const ZSweep<T> sw{hat, P, m, rc, rcw, t.inv, t.c, t.i_inf[m], t.c_inf[m]};
    sw.forward(n - 2, ils, low, d, s_last);
    // Robin row after eliminating u_{N-2} (top_robin_hat = 0)
    const double rl = -ls * dz2 - 2.0;
    const double rr = -s_last * dz2;
    double u = (rr - rl * d) * t.inv_last[m];
    hat[(long long)nz * P - P + m] = (T)u;
    sw.back(n - 2, u);
}

// Dirichlet chain (nfgs_solver.py:3263-3306 with the Thomas solve at
// nfgs_solver.py:536-608): unknown planes 1..nz-2 of the interior DST
// modes, rhs = -S_hat / lambda_D, bottom T_hat, top 0.
template <typename T>
__device__ void zsolve_dir_mode(Geo g, long long m, long long PI, T* __restrict__ hat, ZTab t,
                                const double* __restrict__ lam, const double* __restrict__ bot_hat, int rcw) {
    const int nz = g.nz;
    const int n = nz - 2;
    const double dz2 = g.dz * g.dz, a = 1.0 / dz2;
    const double ilam = -1.0 / lam[m];
    const int rc = t.rconv[m];
    double r1 = (double)hat[PI + m] * ilam;
    double d;
    if (n == 1) {
        d = (r1 - a * bot_hat[m]) * t.inv_last[m];
        hat[PI + m] = (T)d;
        return;
    }
    d = (r1 - a * bot_hat[m]) * t.inv[m];
    hat[PI + m] = (T)d;
    double s_unused = 0.0;
    const ZSweep<T> sw{hat, PI, m, rc, rcw, t.inv, t.c, t.i_inf[m], t.c_inf[m]};
    sw.forward(n - 2, ilam, a, d, s_unused);
    {
        const long long q = (long long)n * PI + m;
        double s = (double)hat[q] * ilam;
        d = (s - a * d) * t.inv_last[m];
        hat[q] = (T)d;
    }
    double u = d;
    sw.back(n - 2, u);
}

// threads per z-solve block (one mode each); FP32 storage keeps 7 blocks
// (28 warps) resident per SM, so the 132k modes of the benchmark grid run in
// one wave
constexpr int ZS_THREADS = 128;
template <typename T>
__global__ void __launch_bounds__(ZS_THREADS, sizeof(T) == 4 ? 7 : 4) k_zsolve(Geo g, const int* skip, T* __restrict__ shat, ZTab tr,
                                                   const double* __restrict__ lamN,
                                                   const double* __restrict__ phi_bot_hat,
                                                   const double* __restrict__ der_hat, double rho, double* s00,
                                                   T* __restrict__ jhat, ZTab td, const double* __restrict__ lamD,
                                                   const double* __restrict__ az_bot_hat, int nb_robin) {
    if (skip != nullptr && *skip) return;
    // blocks are either all Robin or all Dirichlet modes, so every lane of a
    // warp takes part in the rconv maximum
    if ((int)blockIdx.x < nb_robin) {
        const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const bool ok = m < g.P;
        const int rcw = __reduce_max_sync(0xffffffffu, ok ? tr.rconv[m] : 0);
        if (ok) zsolve_robin_mode<T>(g, m, shat, tr, lamN, phi_bot_hat, der_hat, rho, s00, rcw);
    } else if (jhat != nullptr) {
        const long long PI = (long long)(g.nx - 2) * (g.ny - 2);
        const long long m = (long long)(blockIdx.x - nb_robin) * blockDim.x + threadIdx.x;
        const bool ok = m < PI;
        const int rcw = __reduce_max_sync(0xffffffffu, ok ? td.rconv[m] : 0);
        if (ok) zsolve_dir_mode<T>(g, m, PI, jhat, td, lamD, az_bot_hat, rcw);
    }
}

// Factor tables.  chain 0: Robin (modes P, rows nz-1); chain 1: Dirichlet
// (modes PI, rows nz-2).
__global__ void k_ztables(Geo g, int chain, double rho, const double* __restrict__ lam,
                          const double* __restrict__ kk, double* c, double* inv, double* inv_last,
                          double* c_inf, double* i_inf, int* rconv) {
    const long long M = chain == 0 ? g.P : (long long)(g.nx - 2) * (g.ny - 2);
    long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const double dz = g.dz, dz2 = dz * dz, low = 1.0 / dz2, up = 1.0 / dz2;
    const double l = lam[m];
    const int n = chain == 0 ? g.nz - 1 : g.nz - 2;
    double diag = l - 2.0 / dz2;
    double cprev;
    if (chain == 0) {
        double fdiag = rho > 0.0 ? (1.0 - rho) * l - 2.0 / dz2 : diag;
        double fup = rho > 0.0 ? (1.0 - 0.5 * rho) / dz2 : up;
        cprev = fup / fdiag;
        c[m] = cprev;
        inv[m] = 1.0 / fdiag;
        for (int r = 1; r <= n - 2; ++r) {
            double den = diag - low * cprev;
            cprev = up / den;
            c[(long long)r * M + m] = cprev;
            inv[(long long)r * M + m] = 1.0 / den;
        }
        double rl = -l * dz2 - 2.0;
        double rd = 2.0 + 2.0 * dz * kk[m];
        inv_last[m] = 1.0 / (rd - rl * cprev);
    } else {
        if (n == 1) {
            c[m] = 0.0;
            inv[m] = 1.0 / diag;
            inv_last[m] = 1.0 / diag;
            c_inf[m] = 0.0; i_inf[m] = 1.0 / diag; rconv[m] = 1;
            return;
        }
        cprev = up / diag;
        c[m] = cprev;
        inv[m] = 1.0 / diag;
        for (int r = 1; r <= n - 2; ++r) {
            double den = diag - low * cprev;
            cprev = up / den;
            c[(long long)r * M + m] = cprev;
            inv[(long long)r * M + m] = 1.0 / den;
        }
        inv_last[m] = 1.0 / (diag - low * cprev);
    }
    // converged tail: rows rc..n-2 equal row n-2 bitwise
    const int last = n - 2;
    if (last < 0) { c_inf[m] = 0.0; i_inf[m] = 0.0; rconv[m] = 0; return; }
    const double cl = c[(long long)last * M + m], il = inv[(long long)last * M + m];
    int rc = last;
    while (rc > 0 && c[(long long)(rc - 1) * M + m] == cl && inv[(long long)(rc - 1) * M + m] == il) --rc;
    c_inf[m] = cl;
    i_inf[m] = il;
    rconv[m] = rc;
}

// ---------------------------------------------------------------------------
// Source zero-mode ratio (nfgs_solver.py:5457-5476): rms over heights of
// the (0,0) DCT coefficient / (4 (Nx-1)(Ny-1)) divided by the source rms.
// ---------------------------------------------------------------------------
__global__ void k_zero_mode(Geo g, DevCtl* ctl, const double* s00) {
    if (ctl->stopped) return;
    // one warp: lane l sums planes l, l + 32, ...; then a fixed butterfly
    const double norm = 4.0 * (double)(g.nx - 1) * (double)(g.ny - 1);
    double acc = 0.0;
    for (int p = (int)threadIdx.x; p < g.nz; p += 32) {
        double v = s00[p] / norm;
        acc += v * v;
    }
    acc = warp_sum(acc);
    if (threadIdx.x != 0) return;
    double zr = sqrt(acc / g.nz);
    double srms = sqrt(ctl->sumsb2 / (double)g.V);
    double ratio = zr / fmax(srms, 1e-30);
    ctl->zero_ratio_last = ratio;
    if (ctl->source_policy == 0 && ratio > ctl->src_tol) {
        ctl->policy_error = 1;
        ctl->stopped = 1;
        ctl->stop_reason = 6;
    }
}

// ---------------------------------------------------------------------------
// Phi_c finalisation after the inverse transform: Phi_c(0) = Phi^> bottom,
// optional bottom-divergence projection (nfgs_solver.py:4948-4988) and the
// scalar under-relaxation mu (nfgs_solver.py:6789-6794).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_finalize(Geo g, StateTab st, const DevCtl* ctl, int use_ctl_mu, double mu_fixed,
                           const int* cand_sel, const int* cur_sel, const T* __restrict__ phi_above,
                           const T* __restrict__ dphi_target, double proj_w, int do_relax, int zero_az_top,
                           const T* __restrict__ az_bottom) {
    if (ctl != nullptr && ctl->stopped) return;
    const long long P = g.P;
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P) return;
    T* phi = (T*)st.phi[*cand_sel];
    T* az = (T*)st.az[*cand_sel];
    const T* phio = (const T*)st.phi[*cur_sel];
    const T* azo = (const T*)st.az[*cur_sel];
    const double mu = use_ctl_mu ? ctl->mu_cur : mu_fixed;
    // One thread per column: the projection reads and writes planes 1 and 2
    // of the un-relaxed candidate before the relaxation touches them.
    const T p0 = phi_above[idx];
    if (proj_w > 0.0) {
        const double dz = g.dz;
        double v1 = (double)phi[P + idx], v2 = (double)phi[2 * P + idx];
        double cur = (-3.0 * (double)p0 + 4.0 * v1 - v2) / (2.0 * dz);
        double res = (double)dphi_target[idx] - cur;
        v1 += (8.0 * dz / 17.0) * proj_w * res;
        v2 -= (2.0 * dz / 17.0) * proj_w * res;
        phi[P + idx] = (T)v1;
        phi[2 * P + idx] = (T)v2;
    }
    phi[idx] = p0;
    // Az_new[0] = Az_bottom (nfgs_solver.py:6790): a buffer that held a start
    // state with another bottom plane (the cfcf start's) is reset when reused
    if (az_bottom != nullptr) az[idx] = az_bottom[idx];
    if (do_relax && mu < 1.0) {
        const T m1 = (T)mu, m0 = (T)(1.0 - mu);
        for (int k = 1; k < g.nz; ++k) {
            const long long q = (long long)k * P + idx;
            phi[q] = m1 * phi[q] + m0 * phio[q];
            if (k < g.nz - 1) az[q] = m1 * az[q] + m0 * azo[q];
        }
    }
    // Az_new[-1] = 0 (nfgs_solver.py:6792): a buffer that held a start state
    // with a non-zero top plane (soft_cfcf) is cleared when it is reused
    if (zero_az_top && g.nz > 1) az[(long long)(g.nz - 1) * P + idx] = T(0);
}
