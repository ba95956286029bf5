// Per-iteration diagnostics of record_iteration_diagnostics
// (nfgs_solver.py:6660-6681, 6806-6933) for one attempted candidate: the
// map and update residuals, the poloidal / toroidal / mixed-row PDE
// residuals against the sources of the state the candidate came from, the
// bottom imprints and the alpha-clip / weak-field fractions of that state's
// vertical faces.  Off the production path: the iteration graph never
// launches these kernels; the host calls them after a single step.  Sums
// are FP64 block partials, added on the host in a fixed order.
#pragma once
#include "nfgs_iter.cuh"

namespace diag {

// second z-derivative with the reference's one-sided ends (nfgs_solver.py:1717-1727)
__device__ __forceinline__ double d2z(const double* f, long long P, int nz, int k, long long q, double idz2) {
    if (nz < 2) return 0.0;
    if (k > 0 && k < nz - 1) return (f[(k + 1) * P + q] - 2.0 * f[k * P + q] + f[(k - 1) * P + q]) * idz2;
    if (k == 0) {
        if (nz >= 4) return (2.0 * f[q] - 5.0 * f[P + q] + 4.0 * f[2 * P + q] - f[3 * P + q]) * idz2;
        if (nz >= 2) return (f[P + q] - f[q]) * idz2;
        return 0.0;
    }
    return (-2.0 * f[(long long)(nz - 1) * P + q] + 2.0 * f[(long long)(nz - 2) * P + q]) * idz2;
}

// mirrored-Neumann horizontal Laplacian of one plane (nfgs_solver.py:1741-1749)
__device__ __forceinline__ double lapd(const double* a, int nx, int ny, int j, int i, double idx2, double idy2) {
    const long long c = (long long)j * nx + i;
    double lx = 0.0, ly = 0.0;
    if (nx > 1) {
        if (i == 0) lx = 2.0 * a[c + 1] - 2.0 * a[c];
        else if (i == nx - 1) lx = 2.0 * a[c - 1] - 2.0 * a[c];
        else lx = a[c + 1] - 2.0 * a[c] + a[c - 1];
    }
    if (ny > 1) {
        if (j == 0) ly = 2.0 * a[c + nx] - 2.0 * a[c];
        else if (j == ny - 1) ly = 2.0 * a[c - nx] - 2.0 * a[c];
        else ly = a[c + nx] - 2.0 * a[c] + a[c - nx];
    }
    return lx * idx2 + ly * idy2;
}

// The unrelaxed candidate x* = (x_new - (1 - mu) x_prev) / mu (the relaxation
// of nfgs_solver.py:6778-6783 undone) of Phi_c and A_z as FP64 volumes,
// with B_c,z* = lap_xy Phi* and J_z* = -lap_xy A* (nfgs_solver.py:6754, 6811).
template <typename T>
__global__ void k_unrelaxed(Geo g, const T* __restrict__ phn, const T* __restrict__ php, const T* __restrict__ azn,
                            const T* __restrict__ azp, double mu, double* __restrict__ phs, double* __restrict__ azs) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.V) return;
    if (mu < 1.0) {
        phs[q] = ((double)phn[q] - (1.0 - mu) * (double)php[q]) / mu;
        azs[q] = ((double)azn[q] - (1.0 - mu) * (double)azp[q]) / mu;
    } else {
        phs[q] = (double)phn[q];
        azs[q] = (double)azn[q];
    }
}

__global__ void k_laps(Geo g, const double* __restrict__ phs, const double* __restrict__ azs, double* __restrict__ bcz,
                       double* __restrict__ jzs) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= g.V) return;
    const long long P = g.P, k = q / P, r = q % P;
    const int j = (int)(r / g.nx), i = (int)(r % g.nx);
    const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    bcz[q] = lapd(phs + k * P, g.nx, g.ny, j, i, idx2, idy2);
    jzs[q] = -lapd(azs + k * P, g.nx, g.ny, j, i, idx2, idy2);
}

// S_B and S_J on every cell from the face current of k_face (the J_par rows
// of k_src): S_J = lap_xy Jp_z - D2xz Jp_x - D2yz Jp_y with the mixed
// derivatives zero outside the x (y) interior and on the end planes
// (nfgs_solver.py:1729-1749, 6726-6745), walls included.
template <typename T>
__global__ void k_src_full(Geo g, const T* __restrict__ jpf, const T* __restrict__ jb, const T* __restrict__ jzt,
                           const T* __restrict__ bzobs, SrcOpts o, const T* __restrict__ wx, const T* __restrict__ wy,
                           const T* __restrict__ wz, double* __restrict__ sb, double* __restrict__ sj) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (i >= nx || j >= ny) return;
    const long long P = g.P;
    const long long FV = (long long)(nz - 1) * P;
    auto JP = [&](int comp, int kk, int jj, int ii) -> double {
        const long long q = (long long)jj * nx + ii;
        double v;
        if (kk == 0) {
            if (o.polarity == 0) {
                if (comp == 2) v = (double)jzt[q];
                else if (o.face_exact) v = (double)jpf[comp * FV + q];
                else v = (double)jb[comp * P + q];
            } else {
                const double bzv = (double)bzobs[q];
                const bool m = (o.polarity == 1) ? (bzv > 0.0) : (bzv < 0.0);
                const double base = (comp == 2) ? (double)jzt[q] : (double)jb[comp * P + q];
                v = m ? base : 0.0;
            }
        } else if (kk == nz - 1) {
            v = (double)jpf[comp * FV + (long long)(nz - 2) * P + q];
        } else {
            v = 0.5 * ((double)jpf[comp * FV + (long long)(kk - 1) * P + q] + (double)jpf[comp * FV + (long long)kk * P + q]);
        }
        if (o.window) v = v * ((double)wz[kk] * (double)wy[jj] * (double)wx[ii]);
        return v;
    };
    const double i2dx = 1.0 / (2.0 * g.dx), i2dy = 1.0 / (2.0 * g.dy);
    const double s_b = d1<double>([&](int t) { return JP(0, k, t, i); }, j, ny, i2dy) -
                       d1<double>([&](int t) { return JP(1, k, j, t); }, i, nx, i2dx);
    const long long c = (long long)k * P + (long long)j * nx + i;
    sb[c] = s_b;
    const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy);
    double lap = 0.0;
    if (nx > 1) lap += lap1<double>([&](int t) { return JP(2, k, j, t); }, i, nx) * idx2;
    if (ny > 1) lap += lap1<double>([&](int t) { return JP(2, k, t, i); }, j, ny) * idy2;
    double dxz = 0.0, dyz = 0.0;
    if (k >= 1 && k <= nz - 2) {
        if (i >= 1 && i <= nx - 2)
            dxz = (JP(0, k + 1, j, i + 1) - JP(0, k - 1, j, i + 1) - JP(0, k + 1, j, i - 1) + JP(0, k - 1, j, i - 1)) /
                  (4.0 * g.dx * g.dz);
        if (j >= 1 && j <= ny - 2)
            dyz = (JP(1, k + 1, j + 1, i) - JP(1, k - 1, j + 1, i) - JP(1, k + 1, j - 1, i) + JP(1, k - 1, j - 1, i)) /
                  (4.0 * g.dy * g.dz);
    }
    sj[c] = lap - dxz - dyz;
}

// Weak-field and alpha-clip counts of the vertical faces of a state
// (nfgs_solver.py:6660-6681): B from the carrier C (k_recon) and B_bg, the
// staggered face current of k_face's expressions.  partials[2][nblocks].
template <typename T>
__global__ void __launch_bounds__(128) k_face_counts(Geo g, const T* __restrict__ B, const T* __restrict__ bbg,
                                                     const T* __restrict__ jz, double alpha_max, double floor_b2,
                                                     double* __restrict__ partials) {
    __shared__ double sh[2 * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    double red[2] = {0.0, 0.0};
    if (i < nx && j < ny && k < nz - 1) {
        const long long c = k * P + (long long)j * nx + i, c1 = c + P;
        auto F = [&](long long q) -> double { return (double)bbg[q] + (double)B[q]; };
        const double bfx = 0.5 * (F(c1) + F(c)), bfy = 0.5 * (F(V + c1) + F(V + c)),
                     bfz = 0.5 * (F(2 * V + c1) + F(2 * V + c));
        auto CZF = [&](int jj, int ii) -> double {
            const long long q0 = 2 * V + k * P + (long long)jj * nx + ii;
            return 0.5 * ((double)B[q0 + P] + (double)B[q0]);
        };
        const double idz = 1.0 / g.dz, i2dx = 1.0 / (2.0 * g.dx), i2dy = 1.0 / (2.0 * g.dy);
        const double dbx = ((double)B[c1] - (double)B[c]) * idz;
        const double dby = ((double)B[V + c1] - (double)B[V + c]) * idz;
        const double jxf = d1<double>([&](int t) { return CZF(t, i); }, j, ny, i2dy) - dby;
        const double jyf = dbx - d1<double>([&](int t) { return CZF(j, t); }, i, nx, i2dx);
        const double jzf = 0.5 * ((double)jz[c1] + (double)jz[c]);
        const double b2 = bfx * bfx + bfy * bfy + bfz * bfz;
        red[0] = b2 <= floor_b2 ? 1.0 : 0.0;
        const double alpha = (jxf * bfx + jyf * bfy + jzf * bfz) / (b2 > floor_b2 ? b2 : floor_b2);
        red[1] = (alpha_max > 0.0 && fabs(alpha) > alpha_max) ? 1.0 : 0.0;
    }
    block_reduce<2>(red, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
        partials[b] = red[0];
        partials[nb + b] = red[1];
    }
}

// The residual sums.  Index of each sum in partials[NS][nblocks]:
enum {
    S_DPHI_U, S_PHI, S_DAZ_U, S_AZ, S_DPHI_M, S_DAZ_M,         // update / map residuals and scales
    S_BCZ_R, S_SB_BI,                                         // B_c,z PDE on bcz_interior
    S_JZ_R, S_SJ_I,                                           // J_z PDE on planes 1..nz-2
    S_POL_R, S_POL_D2, S_POL_LX, S_POL_SRC,                   // poloidal scalar PDE on bcz_interior
    S_TOR_R, S_TOR_D2, S_TOR_LX, S_TOR_SRC,                   // toroidal scalar PDE on the interior
    S_MIX_R, S_MIX_PDE, S_MIX_DER, S_MIX_SRC,                 // mixed first-interior row (plane 1)
    S_BOT_E, S_BOT_O, S_JZB_E, S_JZB_O,                       // bottom imprints
    NS
};

template <typename T>
__global__ void __launch_bounds__(128) k_diag_sums(
    Geo g, const T* __restrict__ php, const T* __restrict__ azp, const T* __restrict__ phn, const T* __restrict__ azn,
    const double* __restrict__ phs, const double* __restrict__ azs, const double* __restrict__ bczs,
    const double* __restrict__ jzs, const double* __restrict__ sb, const double* __restrict__ sj,
    const double* __restrict__ sphi, const double* __restrict__ saz, const double* __restrict__ dphi_tgt, double rho,
    const T* __restrict__ Bc, const T* __restrict__ bbg, const T* __restrict__ jzn, const double* __restrict__ bxo,
    const double* __restrict__ byo, const double* __restrict__ bzo, const double* __restrict__ jzt,
    double* __restrict__ partials) {
    __shared__ double sh[NS * 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    double red[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) red[q] = 0.0;
    if (i < nx && j < ny) {
        const long long r = (long long)j * nx + i, c = (long long)k * P + r;
        const double idx2 = 1.0 / (g.dx * g.dx), idy2 = 1.0 / (g.dy * g.dy), idz2 = 1.0 / (g.dz * g.dz);
        const double pp = (double)php[c], ap = (double)azp[c];
        const double du = (double)phn[c] - pp, da = (double)azn[c] - ap;
        const double dm = phs[c] - pp, dam = azs[c] - ap;
        red[S_DPHI_U] = du * du; red[S_PHI] = pp * pp; red[S_DAZ_U] = da * da; red[S_AZ] = ap * ap;
        red[S_DPHI_M] = dm * dm; red[S_DAZ_M] = dam * dam;
        const bool bi = (nz > 4) ? (k >= 2 && k <= nz - 2) : (k >= 1 && k <= nz - 2);
        const double d2p = d2z(phs, P, nz, k, r, idz2);
        const double lxp = lapd(phs + k * P, nx, ny, j, i, idx2, idy2);
        const double pres = d2p + lxp - sphi[c];
        if (bi) {
            const double rb = d2z(bczs, P, nz, k, r, idz2) + lapd(bczs + k * P, nx, ny, j, i, idx2, idy2) - sb[c];
            red[S_BCZ_R] = rb * rb; red[S_SB_BI] = sb[c] * sb[c];
            red[S_POL_R] = pres * pres; red[S_POL_D2] = d2p * d2p; red[S_POL_LX] = lxp * lxp;
            red[S_POL_SRC] = sphi[c] * sphi[c];
        }
        if (k >= 1 && k <= nz - 2) {
            const double rj = d2z(jzs, P, nz, k, r, idz2) + lapd(jzs + k * P, nx, ny, j, i, idx2, idy2) - sj[c];
            red[S_JZ_R] = rj * rj; red[S_SJ_I] = sj[c] * sj[c];
            if (i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2) {
                const double d2a = d2z(azs, P, nz, k, r, idz2);
                const double lxa = lapd(azs + k * P, nx, ny, j, i, idx2, idy2);
                const double ta = d2a + lxa - saz[c];
                red[S_TOR_R] = ta * ta; red[S_TOR_D2] = d2a * d2a; red[S_TOR_LX] = lxa * lxa;
                red[S_TOR_SRC] = saz[c] * saz[c];
            }
        }
        if (k == 1 && nz > 2) {
            const double dphi_b = (-3.0 * phs[r] + 4.0 * phs[P + r] - phs[2 * P + r]) / (2.0 * g.dz);
            const double tgt = dphi_tgt ? dphi_tgt[r] : 0.0;
            const double mp = (1.0 - rho) * pres, md = -rho * (dphi_b - tgt) / g.dz;
            red[S_MIX_R] = (mp + md) * (mp + md); red[S_MIX_PDE] = mp * mp; red[S_MIX_DER] = md * md;
            red[S_MIX_SRC] = sphi[c] * sphi[c];
        }
        if (k == 0) {
            const double bx = (double)bbg[r] + (double)Bc[r], by = (double)bbg[V + r] + (double)Bc[V + r];
            const double bz = (double)bbg[2 * V + r] + (double)Bc[2 * V + r];
            const double ex = bx - bxo[r], ey = by - byo[r], ez = bz - bzo[r];
            red[S_BOT_E] = ex * ex + ey * ey + ez * ez;
            red[S_BOT_O] = bxo[r] * bxo[r] + byo[r] * byo[r] + bzo[r] * bzo[r];
            const double ej = (double)jzn[r] - jzt[r];
            red[S_JZB_E] = ej * ej; red[S_JZB_O] = jzt[r] * jzt[r];
        }
    }
    block_reduce<NS>(red, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
#pragma unroll
        for (int q = 0; q < NS; ++q) partials[q * nb + b] = red[q];
    }
}

}  // namespace diag
