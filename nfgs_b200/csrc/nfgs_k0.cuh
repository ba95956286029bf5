// k_h=0 closures: the horizontally uniform field H(z) = (H_x(z), H_y(z))
// as a per-height unknown (horizontal_zero_mode_policy "coupled_k0" and
// "constrained_spline_harmonic", nfgs_solver.py:5058-5431, 5952-6067).
//
// Every state buffer carries its own H profile (2 x nz FP64) next to its
// Phi_c and A_z, so the iteration's buffer swaps, rollbacks and the
// best-state selection move H with the scalars.  Per iteration:
//   k_src        : per-block plane sums of the parallel current (DCT-I
//                  zero-mode weights) and of the face-aligned current
//   k_k0_pt      : plane sums of the horizontal PT current of the candidate
//                  scalars, evaluated on the lateral boundary strips only
//                  (the interior sum of a centred difference telescopes)
//   k_k0_update  : one block: target mean current by height, the closure's
//                  linear fit H* = G q + m H(0) (G, m precomputed on the
//                  host in FP64), the k0_update_mu blend into the candidate
//                  buffer's profile, and the fit's residual.
#pragma once
#include <cmath>
#include <vector>

#include "nfgs_common.cuh"
#include "nfgs_iter.cuh"

namespace k0 {

// Device views of the closure state.
struct Dev {
    double* hk;       // [3][2][nz] profile of each state buffer
    double* hlast;    // [2][nz] profile of the reference's running H_k0 (last update or the selected state)
    double* hbefore;  // [2][nz] hlast before the last update
    double* hstar;    // [2][nz] last fitted profile
    double* target;   // [2][nz] last target mean current (x, y)
    double* stats;    // [0] max relative fit residual, [1] updates, [2] KKT condition number
    double* ptm;      // [2][nz] plane sums of the candidate's PT current
    double* cell;     // [4][nz] plane sums of the parallel current (scratch of the update)
    double* kpart;    // [blocks of k_src][4] per-block plane sums
    double* G;        // [nz][nz] profile from the target by plane
    double* m;        // [nz] profile from H(0)
    double* wfac;     // [nz] zero mode of the buffer window on each plane (1 without a window)
};

// Plane sums of the PT current's horizontal components (ccu_pure_current,
// nfgs_solver.py:3311-3341 with 1760-1768):
//   J_x = Dx(Dz A_z) + Dy(L),  J_y = Dy(Dz A_z) - Dx(L),
//   L = lap_xy Phi_c + d2/dz2 Phi_c (the one-sided rows of nfgs_solver.py:1717-1727),
// summed over the interior columns (the walls and the top plane of J are
// zero, nfgs_solver.py:6069-6078).  A centred difference summed over the
// interior telescopes to its four edge samples, so only the two outermost
// rows and columns are read.
template <typename T>
__global__ void __launch_bounds__(256) k_k0_pt(Geo g, StateTab st, const int* sel, const int* skip,
                                               double* __restrict__ ptm) {
    __shared__ double sh[NFGS_NRED * 32];
    if (skip != nullptr && *skip) return;
    const int k = blockIdx.x;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (k == nz - 1) {
        if (threadIdx.x == 0) { ptm[k] = 0.0; ptm[nz + k] = 0.0; }
        return;
    }
    const T* __restrict__ phi = (const T*)st.phi[*sel];
    const T* __restrict__ az = (const T*)st.az[*sel];
    const long long P = g.P;
    const double dz = g.dz, i2dz = 1.0 / (2.0 * dz), idz2 = 1.0 / (dz * dz);
    const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    const double i2dx = 1.0 / (2.0 * g.dx), i2dy = 1.0 / (2.0 * g.dy);
    auto PH = [&](int kk, int jj, int ii) -> double { return (double)phi[kk * P + (long long)jj * nx + ii]; };
    auto AZ = [&](int kk, int jj, int ii) -> double { return (double)az[kk * P + (long long)jj * nx + ii]; };
    auto dzA = [&](int jj, int ii) -> double {
        if (k == 0) return (-3.0 * AZ(0, jj, ii) + 4.0 * AZ(1, jj, ii) - AZ(2, jj, ii)) * i2dz;
        return (AZ(k + 1, jj, ii) - AZ(k - 1, jj, ii)) * i2dz;
    };
    auto L = [&](int jj, int ii) -> double {
        const double c = PH(k, jj, ii);
        double lx, ly;
        if (ii == 0) lx = 2.0 * PH(k, jj, 1) - 2.0 * c;
        else if (ii == nx - 1) lx = 2.0 * PH(k, jj, nx - 2) - 2.0 * c;
        else lx = PH(k, jj, ii + 1) - 2.0 * c + PH(k, jj, ii - 1);
        if (jj == 0) ly = 2.0 * PH(k, 1, ii) - 2.0 * c;
        else if (jj == ny - 1) ly = 2.0 * PH(k, ny - 2, ii) - 2.0 * c;
        else ly = PH(k, jj + 1, ii) - 2.0 * c + PH(k, jj - 1, ii);
        double d2;
        if (k == 0)
            d2 = nz >= 4 ? (2.0 * c - 5.0 * PH(1, jj, ii) + 4.0 * PH(2, jj, ii) - PH(3, jj, ii)) * idz2
                         : (PH(1, jj, ii) - c) * idz2;
        else d2 = (PH(k + 1, jj, ii) - 2.0 * c + PH(k - 1, jj, ii)) * idz2;
        return lx * idx2 + ly * idy2 + d2;
    };
    double v[2] = {0.0, 0.0};
    const int nrow = ny - 2, ncol = nx - 2;
    for (int t = threadIdx.x; t < nrow + ncol; t += blockDim.x) {
        if (t < nrow) {
            const int j = t + 1;  // sum over i of Dx(.) at row j
            const double gx = dzA(j, nx - 1) + dzA(j, nx - 2) - dzA(j, 1) - dzA(j, 0);
            const double lx = L(j, nx - 1) + L(j, nx - 2) - L(j, 1) - L(j, 0);
            v[0] += gx * i2dx;
            v[1] -= lx * i2dx;
        } else {
            const int i = t - nrow + 1;  // sum over j of Dy(.) at column i
            const double gy = dzA(ny - 1, i) + dzA(ny - 2, i) - dzA(1, i) - dzA(0, i);
            const double ly = L(ny - 1, i) + L(ny - 2, i) - L(1, i) - L(0, i);
            v[0] += ly * i2dy;
            v[1] += gy * i2dy;
        }
    }
    block_reduce<2>(v, sh);
    if (threadIdx.x == 0) {
        ptm[k] = v[0];
        ptm[nz + k] = v[1];
    }
}

// One block.  q(k) = target mean current - mean PT current of the
// candidate; H_x* = G q_y + m H_x(0), H_y* = -G q_x + m H_y(0)
// (nfgs_solver.py:5952-5966, 6011-6023); the candidate buffer's profile is
// mu_k0 H* + (1 - mu_k0) H_cur with H_cur(0) the bottom target
// (nfgs_solver.py:6686-6693, 6782-6787).
__global__ void __launch_bounds__(256) k_k0_update(Geo g, Dev d, const int* cand_sel, const int* cur_sel,
                                                   const DevCtl* ctl, int use_ctl_mu, double mu_fixed,
                                                   double k0_mu, int face_target, int nbp, double t0, double t1) {
    if (ctl != nullptr && ctl->stopped) return;
    const int nz = g.nz, nx = g.nx, ny = g.ny;
    const double icell = 1.0 / (4.0 * (double)(nx - 1) * (double)(ny - 1));
    const double iface = 1.0 / ((double)nx * (double)ny);
    const double ipt = 1.0 / ((double)(nx - 1) * (double)(ny - 1));
    double* cell = d.cell;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        double s[4] = {0.0, 0.0, 0.0, 0.0};
        const double* kp = d.kpart + (long long)k * nbp * 4;
        for (int b = 0; b < nbp; ++b) {
#pragma unroll
            for (int q = 0; q < 4; ++q) s[q] += kp[4 * b + q];
        }
        cell[k] = s[0] * icell;
        cell[nz + k] = s[1] * icell;
        cell[2 * nz + k] = s[2] * iface;  // face k (k < nz-1)
        cell[3 * nz + k] = s[3] * iface;
    }
    __syncthreads();
    double* tg = d.target;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        double tx, ty;
        if (face_target) {
            // face profile to the planes (nfgs_solver.py:5796-5812), times the window's zero mode
            const double* fx = cell + 2 * nz;
            const double* fy = cell + 3 * nz;
            if (k == 0) { tx = fx[0]; ty = fy[0]; }
            else if (k == nz - 1) { tx = fx[nz - 2]; ty = fy[nz - 2]; }
            else { tx = 0.5 * (fx[k - 1] + fx[k]); ty = 0.5 * (fy[k - 1] + fy[k]); }
            tx *= d.wfac[k];
            ty *= d.wfac[k];
        } else {
            tx = cell[k];
            ty = cell[nz + k];
        }
        tg[k] = tx - d.ptm[k] * ipt;
        tg[nz + k] = ty - d.ptm[nz + k] * ipt;
    }
    __syncthreads();
    const double mu = k0_mu > 0.0 ? k0_mu : (use_ctl_mu ? ctl->mu_cur : mu_fixed);
    const double* hc = d.hk + (long long)(*cur_sel) * 2 * nz;
    double* hn = d.hk + (long long)(*cand_sel) * 2 * nz;
    for (int r = threadIdx.x; r < nz; r += blockDim.x) {
        const double* gr = d.G + (long long)r * nz;
        double ax = 0.0, ay = 0.0;
        for (int k = 0; k < nz; ++k) {
            ax += gr[k] * tg[nz + k];
            ay += gr[k] * tg[k];
        }
        const double hx = ax + d.m[r] * t0;
        const double hy = -ay + d.m[r] * t1;
        const double cx = r == 0 ? t0 : hc[r];
        const double cy = r == 0 ? t1 : hc[nz + r];
        const double nxv = mu < 1.0 ? mu * hx + (1.0 - mu) * cx : hx;
        const double nyv = mu < 1.0 ? mu * hy + (1.0 - mu) * cy : hy;
        d.hstar[r] = hx;
        d.hstar[nz + r] = hy;
        d.hbefore[r] = d.hlast[r];
        d.hbefore[nz + r] = d.hlast[nz + r];
        d.hlast[r] = nxv;
        d.hlast[nz + r] = nyv;
        hn[r] = nxv;
        hn[nz + r] = nyv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // relative residual of the fitted current against the target
        // (nfgs_solver.py:5967-5973): current of H* = (-dH_y/dz, dH_x/dz)
        const double dz = g.dz;
        const double* h = d.hstar;
        double rr = 0.0, tt = 0.0;
        for (int k = 0; k < nz; ++k) {
            double der[2];
            for (int c = 0; c < 2; ++c) {
                const double* p = h + c * nz;
                if (k == 0) der[c] = (-3.0 * p[0] + 4.0 * p[1] - p[2]) / (2.0 * dz);
                else if (k == nz - 1) der[c] = (3.0 * p[nz - 1] - 4.0 * p[nz - 2] + p[nz - 3]) / (2.0 * dz);
                else der[c] = 0.5 * ((p[k] - p[k - 1]) / dz + (p[k + 1] - p[k]) / dz);
            }
            const double ex = -der[1] - tg[k], ey = der[0] - tg[nz + k];
            rr += ex * ex + ey * ey;
            tt += tg[k] * tg[k] + tg[nz + k] * tg[nz + k];
        }
        const double rel = sqrt(rr / (2.0 * nz)) / fmax(sqrt(tt / (2.0 * nz)), 1e-30);
        d.stats[0] = d.stats[1] > 0.0 ? fmax(d.stats[0], rel) : rel;
        d.stats[1] += 1.0;
    }
}

// ---------------------------------------------------------------------------
// Host: the closure's linear map profile = G q + m h0 in FP64
// ---------------------------------------------------------------------------

// Cholesky factor (lower, row-major n x n) in place; false if not positive.
inline bool cholesky(std::vector<double>& a, int n) {
    for (int j = 0; j < n; ++j) {
        double s = a[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= a[(size_t)j * n + k] * a[(size_t)j * n + k];
        if (!(s > 0.0)) return false;
        const double d = std::sqrt(s);
        a[(size_t)j * n + j] = d;
        for (int i = j + 1; i < n; ++i) {
            double t = a[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= a[(size_t)i * n + k] * a[(size_t)j * n + k];
            a[(size_t)i * n + j] = t / d;
        }
    }
    return true;
}

inline void cholesky_solve(const std::vector<double>& l, int n, double* b) {
    for (int i = 0; i < n; ++i) {
        double t = b[i];
        for (int k = 0; k < i; ++k) t -= l[(size_t)i * n + k] * b[k];
        b[i] = t / l[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; --i) {
        double t = b[i];
        for (int k = i + 1; k < n; ++k) t -= l[(size_t)k * n + i] * b[k];
        b[i] = t / l[(size_t)i * n + i];
    }
}

// Solve A X = B (A n x n, B n x m, row-major) by Gaussian elimination with
// partial pivoting; false if singular.
inline bool lu_solve(std::vector<double> a, int n, std::vector<double>& b, int m) {
    for (int c = 0; c < n; ++c) {
        int p = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)p * n + c])) p = r;
        if (a[(size_t)p * n + c] == 0.0) return false;
        if (p != c) {
            for (int k = 0; k < n; ++k) std::swap(a[(size_t)p * n + k], a[(size_t)c * n + k]);
            for (int k = 0; k < m; ++k) std::swap(b[(size_t)p * m + k], b[(size_t)c * m + k]);
        }
        for (int r = c + 1; r < n; ++r) {
            const double f = a[(size_t)r * n + c] / a[(size_t)c * n + c];
            if (f == 0.0) continue;
            for (int k = c; k < n; ++k) a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
            for (int k = 0; k < m; ++k) b[(size_t)r * m + k] -= f * b[(size_t)c * m + k];
        }
    }
    for (int c = n - 1; c >= 0; --c) {
        for (int k = 0; k < m; ++k) {
            double t = b[(size_t)c * m + k];
            for (int j = c + 1; j < n; ++j) t -= a[(size_t)c * n + j] * b[(size_t)j * m + k];
            b[(size_t)c * m + k] = t / a[(size_t)c * n + c];
        }
    }
    return true;
}

// 2-norm condition number of a symmetric matrix: the ratio of the extreme
// eigenvalue magnitudes, by cyclic Jacobi rotations.
inline double symmetric_condition(std::vector<double> a, int n) {
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0, tot = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) {
                const double v = a[(size_t)i * n + j] * a[(size_t)i * n + j];
                tot += v;
                if (i != j) off += v;
            }
        if (off <= 1e-30 * tot) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = a[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double app = a[(size_t)p * n + p], aqq = a[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * akp - s * akq;
                    a[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * apk - s * aqk;
                    a[(size_t)q * n + k] = s * apk + c * aqk;
                }
            }
    }
    double lo = INFINITY, hi = 0.0;
    for (int i = 0; i < n; ++i) {
        const double v = std::fabs(a[(size_t)i * n + i]);
        lo = std::min(lo, v);
        hi = std::max(hi, v);
    }
    return lo > 0.0 ? hi / lo : INFINITY;
}

// Clamped open-uniform cubic B-spline collocation matrix on nz equally
// spaced points of [0, 1] (row-major nz x nb), Cox-de Boor recursion
// (nfgs_solver.py:5099-5147).
inline std::vector<double> bspline_basis(int nz, int nb) {
    const int deg = 3, inner = nb - deg - 1;
    std::vector<double> kn;
    for (int i = 0; i <= deg; ++i) kn.push_back(0.0);
    for (int i = 1; i <= inner; ++i) kn.push_back((double)i / (double)(inner + 1));
    for (int i = 0; i <= deg; ++i) kn.push_back(1.0);
    int width = (int)kn.size() - 1;
    std::vector<double> t(nz);
    for (int p = 0; p < nz; ++p) t[p] = nz > 1 ? (double)p / (double)(nz - 1) : 0.0;
    std::vector<double> cur((size_t)nz * width, 0.0);
    for (int i = 0; i < width; ++i)
        for (int p = 0; p < nz; ++p) cur[(size_t)p * width + i] = (t[p] >= kn[i] && t[p] < kn[i + 1]) ? 1.0 : 0.0;
    cur[(size_t)(nz - 1) * width + width - 1] = 1.0;
    for (int order = 1; order <= deg; ++order) {
        std::vector<double> nxt((size_t)nz * (width - 1), 0.0);
        for (int i = 0; i < width - 1; ++i) {
            const double left = kn[i + order] - kn[i], right = kn[i + order + 1] - kn[i + 1];
            for (int p = 0; p < nz; ++p) {
                double v = 0.0;
                if (left > 0.0) v += (t[p] - kn[i]) / left * cur[(size_t)p * width + i];
                if (right > 0.0) v += (kn[i + order + 1] - t[p]) / right * cur[(size_t)p * width + i + 1];
                nxt[(size_t)p * (width - 1) + i] = v;
            }
        }
        width -= 1;
        cur.swap(nxt);
        for (int i = 0; i < width; ++i) cur[(size_t)(nz - 1) * width + i] = 0.0;
        cur[(size_t)(nz - 1) * width + width - 1] = 1.0;
    }
    return cur;  // width == nb
}

// The closure as profile = G q + m h0 (G row-major nz x nz, q the target by
// plane).  coupled_k0: minimise |D_face H - avg(q)|^2 + s |C H|^2 over
// H(1..nz-1) with H(0) = h0 (staggered faces), or the plane-centred legacy
// rows (nfgs_solver.py:5262-5404).  constrained_spline_harmonic: the
// B-spline coefficients of the same face fit with a 1e-12 relative ridge
// and the exact rows H(0) = h0 and one-sided FD2 H'(top) = 0 as a KKT
// system (nfgs_solver.py:5149-5260).  cond_out: the KKT matrix's 2-norm
// condition number (spline) or NaN.  Returns false if a factorisation fails.
inline bool build_operator(int nz, double dz, bool spline, bool legacy, int nb, double smooth, std::vector<double>& G,
                           std::vector<double>& m, double* cond_out) {
    const int n = nz;
    const double root = std::sqrt(smooth);
    G.assign((size_t)n * n, 0.0);
    m.assign(n, 0.0);
    *cond_out = std::nan("");
    // face difference D ((n-1) x n), three-point curvature C ((n-2) x n)
    auto Dface = [&](int r, int c) -> double {
        return c == r ? -1.0 / dz : (c == r + 1 ? 1.0 / dz : 0.0);
    };
    auto Ccurv = [&](int r, int c) -> double {
        return c == r ? 1.0 / dz : (c == r + 1 ? -2.0 / dz : (c == r + 2 ? 1.0 / dz : 0.0));
    };
    if (!spline) {
        // rows of A over the unknowns H(1..n-1), the q map of the rhs and its h0 column
        std::vector<double> A, Rq, Rh;
        int rows = 0;
        const int u = n - 1;
        auto push_row = [&](const std::vector<double>& arow, const std::vector<double>& qrow, double hcoef) {
            A.insert(A.end(), arow.begin(), arow.end());
            Rq.insert(Rq.end(), qrow.begin(), qrow.end());
            Rh.push_back(hcoef);
            ++rows;
        };
        if (legacy) {
            std::vector<double> Dc((size_t)n * n, 0.0);
            if (n >= 3) {
                for (int r = 1; r < n - 1; ++r) {
                    Dc[(size_t)r * n + r - 1] = -0.5 / dz;
                    Dc[(size_t)r * n + r + 1] = 0.5 / dz;
                }
                Dc[0] = -1.5 / dz; Dc[1] = 2.0 / dz; Dc[2] = -0.5 / dz;
                Dc[(size_t)(n - 1) * n + n - 1] = 1.5 / dz;
                Dc[(size_t)(n - 1) * n + n - 2] = -2.0 / dz;
                Dc[(size_t)(n - 1) * n + n - 3] = 0.5 / dz;
            }
            std::vector<double> Cv((size_t)n * n, 0.0);  // Dc Dc
            for (int i = 0; i < n; ++i)
                for (int k = 0; k < n; ++k) {
                    const double a = Dc[(size_t)i * n + k];
                    if (a == 0.0) continue;
                    for (int j = 0; j < n; ++j) Cv[(size_t)i * n + j] += a * Dc[(size_t)k * n + j];
                }
            for (int r = 1; r < n; ++r) {
                std::vector<double> ar(u), qr(n, 0.0);
                for (int c = 1; c < n; ++c) ar[c - 1] = Dc[(size_t)r * n + c];
                qr[r] = 1.0;
                push_row(ar, qr, -Dc[(size_t)r * n]);
            }
            if (root > 0.0)
                for (int r = 1; r < n; ++r) {
                    std::vector<double> ar(u), qr(n, 0.0);
                    for (int c = 1; c < n; ++c) ar[c - 1] = root * Cv[(size_t)r * n + c];
                    push_row(ar, qr, -root * Cv[(size_t)r * n]);
                }
        } else {
            for (int r = 0; r < n - 1; ++r) {
                std::vector<double> ar(u), qr(n, 0.0);
                for (int c = 1; c < n; ++c) ar[c - 1] = Dface(r, c);
                qr[r] = 0.5;
                qr[r + 1] = 0.5;
                push_row(ar, qr, -Dface(r, 0));
            }
            if (root > 0.0)
                for (int r = 0; r < n - 2; ++r) {
                    std::vector<double> ar(u), qr(n, 0.0);
                    for (int c = 1; c < n; ++c) ar[c - 1] = root * Ccurv(r, c);
                    push_row(ar, qr, -root * Ccurv(r, 0));
                }
        }
        std::vector<double> N((size_t)u * u, 0.0);
        for (int r = 0; r < rows; ++r)
            for (int i = 0; i < u; ++i) {
                const double a = A[(size_t)r * u + i];
                if (a == 0.0) continue;
                for (int j = 0; j < u; ++j) N[(size_t)i * u + j] += a * A[(size_t)r * u + j];
            }
        if (!cholesky(N, u)) return false;
        std::vector<double> b(u);
        for (int col = 0; col <= n; ++col) {  // q columns, then h0
            std::fill(b.begin(), b.end(), 0.0);
            for (int r = 0; r < rows; ++r) {
                const double w = col < n ? Rq[(size_t)r * n + col] : Rh[r];
                if (w == 0.0) continue;
                for (int i = 0; i < u; ++i) b[i] += A[(size_t)r * u + i] * w;
            }
            cholesky_solve(N, u, b.data());
            for (int i = 0; i < u; ++i) {
                if (col < n) G[(size_t)(i + 1) * n + col] = b[i];
                else m[i + 1] = b[i];
            }
        }
        m[0] = 1.0;
        return true;
    }
    // constrained spline
    const std::vector<double> basis = bspline_basis(n, nb);
    std::vector<double> design;  // rows x nb
    std::vector<double> dq;      // rows x n: the q map of the rhs rows
    int rows = 0;
    for (int r = 0; r < n - 1; ++r) {
        for (int c = 0; c < nb; ++c)
            design.push_back((basis[(size_t)(r + 1) * nb + c] - basis[(size_t)r * nb + c]) / dz);
        std::vector<double> qr(n, 0.0);
        qr[r] = 0.5;
        qr[r + 1] = 0.5;
        dq.insert(dq.end(), qr.begin(), qr.end());
        ++rows;
    }
    if (smooth > 0.0)
        for (int r = 0; r < n - 2; ++r) {
            for (int c = 0; c < nb; ++c)
                design.push_back(root * (basis[(size_t)r * nb + c] - 2.0 * basis[(size_t)(r + 1) * nb + c] +
                                         basis[(size_t)(r + 2) * nb + c]) / dz);
            dq.insert(dq.end(), (size_t)n, 0.0);
            ++rows;
        }
    const int K = nb + 2;
    std::vector<double> kkt((size_t)K * K, 0.0);
    for (int i = 0; i < nb; ++i)
        for (int j = 0; j < nb; ++j) {
            double s = 0.0;
            for (int r = 0; r < rows; ++r) s += design[(size_t)r * nb + i] * design[(size_t)r * nb + j];
            kkt[(size_t)i * K + j] = s;
        }
    double dmax = 0.0;
    for (int i = 0; i < nb; ++i) dmax = std::max(dmax, std::fabs(kkt[(size_t)i * K + i]));
    const double ridge = std::max(dmax, 1.0) * 1.0e-12;
    for (int i = 0; i < nb; ++i) kkt[(size_t)i * K + i] += ridge;
    for (int c = 0; c < nb; ++c) {
        const double top = 3.0 / (2.0 * dz) * basis[(size_t)(n - 1) * nb + c] -
                           4.0 / (2.0 * dz) * basis[(size_t)(n - 2) * nb + c] +
                           1.0 / (2.0 * dz) * basis[(size_t)(n - 3) * nb + c];
        kkt[(size_t)nb * K + c] = kkt[(size_t)c * K + nb] = basis[c];
        kkt[(size_t)(nb + 1) * K + c] = kkt[(size_t)c * K + nb + 1] = top;
    }
    *cond_out = symmetric_condition(kkt, K);
    // right-hand sides: design^T dq for the q columns, e_nb for h0
    const int M = n + 1;
    std::vector<double> rhs((size_t)K * M, 0.0);
    for (int i = 0; i < nb; ++i)
        for (int col = 0; col < n; ++col) {
            double s = 0.0;
            for (int r = 0; r < rows; ++r) s += design[(size_t)r * nb + i] * dq[(size_t)r * n + col];
            rhs[(size_t)i * M + col] = s;
        }
    rhs[(size_t)nb * M + n] = 1.0;
    if (!lu_solve(kkt, K, rhs, M)) return false;
    for (int p = 0; p < n; ++p)
        for (int col = 0; col <= n; ++col) {
            double s = 0.0;
            for (int c = 0; c < nb; ++c) s += basis[(size_t)p * nb + c] * rhs[(size_t)c * M + col];
            if (col < n) G[(size_t)p * n + col] = s;
            else m[p] = s;
        }
    return true;
}

}  // namespace k0
