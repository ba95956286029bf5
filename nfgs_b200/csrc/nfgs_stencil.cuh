// Fused stencil pass of one NFPT iteration: a z-march over one 32 x 8
// column tile (and one z segment) per CTA.  From the state (Phi_c, A_z) and
// the fixed background it produces, plane by plane:
//   carrier C = B - B_bg and state J_z      (nfgs_solver.py:3311-3341, 5901-5942)
//   vertical-face current, alpha_f B_f     (nfgs_solver.py:5738-5778, 5841-5853)
//   sigma_J / divB / energy partial sums   (nfgs_solver.py:5882-5895, 2689-2697)
//   J_parallel at centres                  (nfgs_solver.py:5780-5794, 6697-6716)
//   sources S_B, S_J                       (nfgs_solver.py:6726, 6730-6745)
// The arithmetic is expression-for-expression that of k_recon / k_face /
// k_src; only the data movement differs.  Phi_c, A_z and B_bg plane halos
// are staged in shared memory with cp.async one plane ahead of use; the
// carrier and the centre current live in rolling shared-memory rings, and
// the face current and J_z of the previous plane stay in registers, so HBM
// sees 5 volume reads and 2 volume writes.
//
// Geometry.  Tiles: x0 = bx*TX, y0 = by*TY; the last tile of an axis
// absorbs a remainder of 1 or 2 cells (width up to TX+2 / TY+2), so every
// tile is at least 3 cells wide and the one-sided end stencils find their
// samples in the halo.  A shared array of halo level h is a fixed
// PW(h) x ROWS(h) box (PW(h) = TX+2+2h, ROWS(h) = TY+2+2h) whose element
// (row, col) holds tile cell (row-h, col-h).  Pitches and slot sizes are
// compile-time constants, so a neighbour access is one register plus an
// immediate offset.  Thread tid owns box entries q = tid + k*NT of every
// level (contiguous across a warp: no bank conflicts); entries outside the
// tile's halo or the domain are idle.
//
// Per plane p (two barriers):
//   B1: plane p staged, C_z(p) formed; stage plane p+1
//   loop F (level 1): C_x, C_y, J_z at p; face p-1 (current, sigma terms,
//           alpha B); centre p-1 from faces p-2, p-1
//   B2
//   loop E (level 0): divB/|B|/|B|^2 at p-1, S_B(p-1), S_J(p-2)
//   loop A (level 2): C_z(p+1)
#pragma once
#include "nfgs_iter.cuh"

namespace fs {

constexpr int TX = 32, TY = 8, NT = 512;
__host__ __device__ constexpr int PW(int h) { return TX + 2 + 2 * h; }
__host__ __device__ constexpr int ROWS(int h) { return TY + 2 + 2 * h; }
__host__ __device__ constexpr int CAP(int h) { return PW(h) * ROWS(h); }
constexpr int O_PHI = 0;                     // 4 planes x CAP(3), slot plane&3
constexpr int O_AZ = O_PHI + 4 * CAP(3);     // 2 planes x CAP(2), slot plane&1
constexpr int O_CZ = O_AZ + 2 * CAP(2);      // carrier z, 4 planes x CAP(2), slot plane&3
constexpr int O_CXY = O_CZ + 4 * CAP(2);     // carrier x,y, 3 planes x 2 x CAP(1), slot (plane%3)*2+comp
constexpr int O_BG = O_CXY + 6 * CAP(1);     // background, 4 planes x 3 x CAP(1), slot (plane&3)*3+comp
constexpr int O_JC = O_BG + 12 * CAP(1);     // centre J_par, 3 x 3 x CAP(1), slot (centre%3)*3+comp
constexpr int N_TOTAL = O_JC + 9 * CAP(1);
// entries per thread of each level
constexpr int NL3 = (CAP(3) + NT - 1) / NT, NL2 = (CAP(2) + NT - 1) / NT, NL1 = (CAP(1) + NT - 1) / NT,
              NL0 = (CAP(0) + NT - 1) / NT;

// offset in a level-h2 box of the cell at entry q (box row `row`) of level h
template <int h, int h2>
__device__ __forceinline__ int lift(int q, int row) {
    return q + row * (PW(h2) - PW(h)) + (h2 - h) * (PW(h2) + 1);
}

// Box geometry of a tile instance: edge tiles (E) may be up to 2 cells wider
// and taller (the remainder of an axis), interior tiles are exactly TX x TY,
// so their level-h boxes are (TX + 2h) x (TY + 2h) inside the same slots.
template <bool E> __host__ __device__ constexpr int pw(int h) { return TX + (E ? 2 : 0) + 2 * h; }
template <bool E> __host__ __device__ constexpr int rows(int h) { return TY + (E ? 2 : 0) + 2 * h; }
template <bool E, int h, int h2>
__device__ __forceinline__ int liftE(int q, int row) {
    return q + row * (pw<E>(h2) - pw<E>(h)) + (h2 - h) * (pw<E>(h2) + 1);
}
static_assert(pw<true>(3) == PW(3) && rows<true>(3) == ROWS(3), "edge boxes fill the slots");

template <typename T> constexpr size_t smem_bytes() { return (size_t)N_TOTAL * sizeof(T); }
template <typename T> constexpr int min_blocks() { return sizeof(T) == 4 ? 2 : 1; }

// tiles along an axis of n cells with tile size t (a remainder <= 2 is merged)
__host__ __device__ inline int ntiles(int n, int t) {
    int g = (n + t - 1) / t;
    if (g > 1 && n - (g - 1) * t <= 2) --g;
    return g;
}

struct Args {
    Geo g;
    StateTab st;
    const int* sel;
    const int* skip;
    const void* bbg;
    const void* bzobs;
    const void* jzt;
    double hx, hy;
    int use_h;
    Box box;
    double alpha_max;    // <= 0: no clip
    double floor_b2;
    SrcOpts o;
    const void *wx, *wy, *wz;
    void* sb;
    void* sj;
    double* partials;    // column-major [NFGS_NRED][nblocks]
    int nseg;            // z segments (gridDim.z)
    int gx, gy;          // tiles per axis
};

template <int B>
__device__ __forceinline__ void cp_async(unsigned dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Body of the z-march.  EDGE = false is the version of tiles none of whose
// cells (levels 0-2) lies on a lateral wall: every x/y stencil takes the
// interior form, so the one-sided wall code is dead and warps never diverge
// on it; the bottom and top planes keep their one-sided z forms (a branch
// uniform over the CTA).
template <typename T, bool EDGE>
__device__ __forceinline__ void stencil_body(const Args& a, unsigned char* sm_raw, double* shred) {
    T* const sm = (T*)sm_raw;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(sm_raw);

    const Geo g = a.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    const int tid = threadIdx.x;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tw = ((int)blockIdx.x == a.gx - 1) ? nx - x0 : TX;
    const int th = ((int)blockIdx.y == a.gy - 1) ? ny - y0 : TY;
    // z segment: output centres [c0, c1)
    const int per = (nz + a.nseg - 1) / a.nseg;
    const int c0 = blockIdx.z * per, c1 = min(nz, c0 + per);
    const int s = *a.sel;
    const T* __restrict__ phi = (const T*)a.st.phi[s];
    const T* __restrict__ az = (const T*)a.st.az[s];
    const T* __restrict__ bbg = (const T*)a.bbg;
    const T* __restrict__ bzobs = (const T*)a.bzobs;
    const T* __restrict__ jzt = (const T*)a.jzt;
    const T* __restrict__ wx = (const T*)a.wx;
    const T* __restrict__ wy = (const T*)a.wy;
    const T* __restrict__ wz = (const T*)a.wz;
    T* __restrict__ sb_out = (T*)a.sb;
    T* __restrict__ sj_out = (T*)a.sj;
    const T i2dx = T(1.0 / (2.0 * g.dx)), i2dy = T(1.0 / (2.0 * g.dy)), i2dz = T(1.0 / (2.0 * g.dz));
    const T idx2 = T(1.0 / (g.dx * g.dx)), idy2 = T(1.0 / (g.dy * g.dy)), idz = T(1.0 / g.dz);
    const T i4xz = T(1.0 / (4.0 * g.dx * g.dz)), i4yz = T(1.0 / (4.0 * g.dy * g.dz));
    const T hx = (T)a.hx, hy = (T)a.hy;
    const T amax = (T)(a.alpha_max > 0 ? a.alpha_max : -1.0), fl = (T)a.floor_b2;
    const long long FPI = (long long)(nx - 2) * (ny - 2);

    // ---- entry lists: in-plane global offset of the cell, or -1 when idle
    int G3[NL3], G2[NL2], G1[NL1], G0[NL0];
    auto build = [&](int h, int* G, int nmax) {
        for (int k = 0; k < nmax; ++k) {
            const int q = tid + k * NT;
            int v = -1;
            if (q < pw<EDGE>(h) * rows<EDGE>(h)) {
                const int r = q / pw<EDGE>(h) - h, c = q % pw<EDGE>(h) - h;
                const int jj = y0 + r, ii = x0 + c;
                if (r < th + h && c < tw + h && jj >= 0 && jj < ny && ii >= 0 && ii < nx) v = jj * nx + ii;
            }
            G[k] = v;
        }
    };
    build(3, G3, NL3);
    build(2, G2, NL2);
    build(1, G1, NL1);
    build(0, G0, NL0);

    // generic accessors by global coordinates (edge cells and edge planes,
    // one-sided stencils of nfgs_solver.py:1361-1419 / 1741-1749)
    auto OF = [&](int h, int jj, int ii) { return (jj - y0 + h) * pw<EDGE>(h) + (ii - x0 + h); };
    auto PHI = [&](int pl, int jj, int ii) -> T { return sm[O_PHI + (pl & 3) * CAP(3) + OF(3, jj, ii)]; };
    auto AZ = [&](int pl, int jj, int ii) -> T { return sm[O_AZ + (pl & 1) * CAP(2) + OF(2, jj, ii)]; };
    auto CC = [&](int pl, int comp, int jj, int ii) -> T {
        return comp == 2 ? sm[O_CZ + (pl & 3) * CAP(2) + OF(2, jj, ii)]
                         : sm[O_CXY + ((pl % 3) * 2 + comp) * CAP(1) + OF(1, jj, ii)];
    };
    auto BG = [&](int pl, int comp, int jj, int ii) -> T {
        return sm[O_BG + ((pl & 3) * 3 + comp) * CAP(1) + OF(1, jj, ii)];
    };
    auto BB = [&](int pl, int comp, int jj, int ii) -> T { return BG(pl, comp, jj, ii) + CC(pl, comp, jj, ii); };
    auto JC = [&](int c, int comp, int jj, int ii) -> T {
        return sm[O_JC + ((c % 3) * 3 + comp) * CAP(1) + OF(1, jj, ii)];
    };
    auto win = [&](int c, int jj, int ii) -> T { return (wz[c] * wy[jj]) * wx[ii]; };
    auto xy_in = [&](int jj, int ii) { return !EDGE || (ii > 0 && ii < nx - 1 && jj > 0 && jj < ny - 1); };

    double red[NFGS_NRED] = {0, 0, 0, 0, 0, 0};

    // ---- asynchronous plane staging
    auto hi_of = [&](int p) { return min(nz - 1, max(p + 1, 2)); };
    auto lo_of = [&](int p) { return max(0, min(p - 1, nz - 3)); };
    const int pstart = max(0, c0 - 2), pend = min(nz - 1, c1 + 1);
    auto stage_plane = [&](int p) {
        const int from = (p == pstart) ? lo_of(p) : hi_of(p - 1) + 1;
        for (int pl = from; pl <= hi_of(p); ++pl) {
            const T* src = phi + (long long)pl * P;
            const unsigned dst = sbase + (unsigned)((O_PHI + (pl & 3) * CAP(3) + tid) * sizeof(T));
#pragma unroll
            for (int k = 0; k < NL3; ++k)
                if (G3[k] >= 0) cp_async<sizeof(T)>(dst + k * NT * sizeof(T), src + G3[k]);
        }
        {
            const T* src = az + (long long)p * P;
            const unsigned dst = sbase + (unsigned)((O_AZ + (p & 1) * CAP(2) + tid) * sizeof(T));
#pragma unroll
            for (int k = 0; k < NL2; ++k)
                if (G2[k] >= 0) cp_async<sizeof(T)>(dst + k * NT * sizeof(T), src + G2[k]);
        }
        {
            const T* src = bbg + (long long)p * P;
            const unsigned dst = sbase + (unsigned)((O_BG + (p & 3) * 3 * CAP(1) + tid) * sizeof(T));
#pragma unroll
            for (int k = 0; k < NL1; ++k) {
                if (G1[k] < 0) continue;
#pragma unroll
                for (int comp = 0; comp < 3; ++comp)
                    cp_async<sizeof(T)>(dst + (comp * CAP(1) + k * NT) * sizeof(T), src + comp * V + G1[k]);
            }
        }
        cp_commit();
    };

    // ---- loop A: carrier z of plane p on level 2
    auto loop_a = [&](int p) {
        const T* const ph0 = sm + O_PHI + (p & 3) * CAP(3);
        T* const cz = sm + O_CZ + (p & 3) * CAP(2);
#pragma unroll
        for (int k = 0; k < NL2; ++k) {
            if (G2[k] < 0) continue;
            const int q = tid + k * NT, row = q / pw<EDGE>(2);
            const int jj = y0 + row - 2, ii = x0 + (q - row * pw<EDGE>(2)) - 2;
            T val;
            if (p == 0) {
                val = bzobs[G2[k]] - bbg[2 * V + G2[k]];
            } else if (xy_in(jj, ii)) {
                const T* const f = ph0 + liftE<EDGE, 2, 3>(q, row);
                const T f0 = f[0];
                val = ((f[1] - T(2) * f0) + f[-1]) * idx2 + ((f[pw<EDGE>(3)] - T(2) * f0) + f[-pw<EDGE>(3)]) * idy2;
            } else {
                val = lap1<T>([&](int t) { return PHI(p, jj, t); }, ii, nx) * idx2 +
                      lap1<T>([&](int t) { return PHI(p, t, ii); }, jj, ny) * idy2;
            }
            cz[q] = val;
        }
    };

    // ---- loop F state carried across planes (per level-1 entry)
    T jfx[NL1], jfy[NL1], jfz[NL1], jzp[NL1];
#pragma unroll
    for (int k = 0; k < NL1; ++k) jfx[k] = jfy[k] = jfz[k] = jzp[k] = T(0);

    auto loop_f = [&](int p) {
        const bool zin = p > 0 && p < nz - 1;
        const int f = p - 1;
        const bool do_face = f >= pstart;
        const bool do_centre = do_face && f >= 1 && f - 1 >= pstart;
        const bool sig = do_face && f >= c0 && f < c1 && f >= a.box.z0 && f < a.box.z1;
        const T* const phm = sm + O_PHI + ((p + 3) & 3) * CAP(3);
        const T* const php = sm + O_PHI + ((p + 1) & 3) * CAP(3);
        const T* const azs = sm + O_AZ + (p & 1) * CAP(2);
        const T* const czp = sm + O_CZ + (p & 3) * CAP(2);
        const T* const czf0 = sm + O_CZ + ((p + 3) & 3) * CAP(2);  // plane p-1
        T* const cxy = sm + O_CXY + (p % 3) * 2 * CAP(1);
        const T* const cxy0 = sm + O_CXY + ((p + 2) % 3) * 2 * CAP(1);
        const T* const bgp = sm + O_BG + ((p & 3) * 3) * CAP(1);
        const T* const bg0 = sm + O_BG + (((p + 3) & 3) * 3) * CAP(1);
        T* const jc = sm + O_JC + ((f + 3) % 3) * 3 * CAP(1);
#pragma unroll
        for (int k = 0; k < NL1; ++k) {
            if (G1[k] < 0) continue;
            const int o1 = tid + k * NT, row = o1 / pw<EDGE>(1);
            const int r = row - 1, c = o1 - row * pw<EDGE>(1) - 1;
            const int jj = y0 + r, ii = x0 + c;
            const int o2 = liftE<EDGE, 1, 2>(o1, row);
            const bool xin = xy_in(jj, ii);
            // carrier x, y and state J_z at plane p
            T cx, cy, jz;
            if (zin && xin) {
                const int o3 = liftE<EDGE, 1, 3>(o1, row);
                const T* const fp = php + o3;
                const T* const fm = phm + o3;
                const T* const A = azs + o2;
                auto dzp = [&](int d) -> T { return (fp[d] - fm[d]) * i2dz; };
                T dxdz = (dzp(1) - dzp(-1)) * i2dx;
                T dydz = (dzp(pw<EDGE>(3)) - dzp(-pw<EDGE>(3))) * i2dy;
                T dya = (A[pw<EDGE>(2)] - A[-pw<EDGE>(2)]) * i2dy;
                T dxa = (A[1] - A[-1]) * i2dx;
                cx = -dxdz + dya;
                cy = -dydz - dxa;
                const T a0 = A[0];
                jz = -(((A[1] - T(2) * a0) + A[-1]) * idx2 + ((A[pw<EDGE>(2)] - T(2) * a0) + A[-pw<EDGE>(2)]) * idy2);
            } else {
                auto dzphi = [&](int j2, int i2) -> T {
                    return d1<T>([&](int kk) { return PHI(kk, j2, i2); }, p, nz, i2dz);
                };
                T dxdz = d1<T>([&](int t) { return dzphi(jj, t); }, ii, nx, i2dx);
                T dydz = d1<T>([&](int t) { return dzphi(t, ii); }, jj, ny, i2dy);
                T dya = d1<T>([&](int t) { return AZ(p, t, ii); }, jj, ny, i2dy);
                T dxa = d1<T>([&](int t) { return AZ(p, jj, t); }, ii, nx, i2dx);
                cx = -dxdz + dya;
                cy = -dydz - dxa;
                if (p == 0) jz = jzt[G1[k]];
                else if (p == nz - 1 || !xin) jz = T(0);
                else jz = -(lap1<T>([&](int t) { return AZ(p, jj, t); }, ii, nx) * idx2 +
                            lap1<T>([&](int t) { return AZ(p, t, ii); }, jj, ny) * idy2);
            }
            if (a.use_h) { cx = cx + hx; cy = cy + hy; }
            cxy[o1] = cx;
            cxy[o1 + CAP(1)] = cy;
            if (do_face) {
                const T cx0 = cxy0[o1], cy0 = cxy0[o1 + CAP(1)];
                T bx0 = bg0[o1] + cx0, bx1 = bgp[o1] + cx;
                T by0 = bg0[o1 + CAP(1)] + cy0, by1 = bgp[o1 + CAP(1)] + cy;
                T bz0 = bg0[o1 + 2 * CAP(1)] + czf0[o2], bz1 = bgp[o1 + 2 * CAP(1)] + czp[o2];
                const T bfx = T(0.5) * (bx1 + bx0), bfy = T(0.5) * (by1 + by0), bfz = T(0.5) * (bz1 + bz0);
                const T dbx = (cx - cx0) * idz;
                const T dby = (cy - cy0) * idz;
                T jxf, jyf;
                if (xin) {
                    const T* const zp = czp + o2;
                    const T* const z0 = czf0 + o2;
                    auto czf = [&](int d) -> T { return T(0.5) * (zp[d] + z0[d]); };
                    jxf = (czf(pw<EDGE>(2)) - czf(-pw<EDGE>(2))) * i2dy - dby;
                    jyf = dbx - (czf(1) - czf(-1)) * i2dx;
                } else {
                    auto CZF = [&](int j2, int i2) -> T { return T(0.5) * (CC(p, 2, j2, i2) + CC(f, 2, j2, i2)); };
                    jxf = d1<T>([&](int t) { return CZF(t, ii); }, jj, ny, i2dy) - dby;
                    jyf = dbx - d1<T>([&](int t) { return CZF(jj, t); }, ii, nx, i2dx);
                }
                const T jzf = T(0.5) * (jz + jzp[k]);
                if (sig && r >= 0 && r < th && c >= 0 && c < tw && jj >= a.box.y0 && jj < a.box.y1 &&
                    ii >= a.box.x0 && ii < a.box.x1) {
                    T cxp = jyf * bfz - jzf * bfy;
                    T cyp = jzf * bfx - jxf * bfz;
                    T czp2 = jxf * bfy - jyf * bfx;
                    T bn = sqrt(bfx * bfx + bfy * bfy + bfz * bfz);
                    bn = bn > T(1e-10) ? bn : T(1e-10);
                    red[0] += (double)(sqrt(cxp * cxp + cyp * cyp + czp2 * czp2) / bn);
                    red[1] += (double)sqrt(jxf * jxf + jyf * jyf + jzf * jzf);
                }
                T b2 = bfx * bfx + bfy * bfy + bfz * bfz;
                b2 = b2 > fl ? b2 : fl;
                T alpha = (jxf * bfx + jyf * bfy + jzf * bfz) / b2;
                if (amax > T(0)) alpha = fmin(fmax(alpha, -amax), amax);
                const T ax = alpha * bfx, ay = alpha * bfy, azv = alpha * bfz;
                if (f == 0) {
                    // bottom row of J_par (nfgs_solver.py:6697-6713)
                    const bool wall = !xin;
                    const int pq = G1[k];
                    T vx, vy, vz;
                    if (a.o.polarity == 0) {
                        vz = jzt[pq];
                        if (a.o.face_exact) { vx = ax; vy = ay; }
                        else { vx = wall ? T(0) : jxf; vy = wall ? T(0) : jyf; }
                    } else {
                        const T bzv = bzobs[pq];
                        const bool m = (a.o.polarity == 1) ? (bzv > T(0)) : (bzv < T(0));
                        vx = m ? (wall ? T(0) : jxf) : T(0);
                        vy = m ? (wall ? T(0) : jyf) : T(0);
                        vz = m ? jzt[pq] : T(0);
                    }
                    if (a.o.window) {
                        const T w = win(0, jj, ii);
                        vx = vx * w; vy = vy * w; vz = vz * w;
                    }
                    jc[o1] = vx;
                    jc[o1 + CAP(1)] = vy;
                    jc[o1 + 2 * CAP(1)] = vz;
                } else if (do_centre) {
                    T vx = T(0.5) * (jfx[k] + ax), vy = T(0.5) * (jfy[k] + ay), vz = T(0.5) * (jfz[k] + azv);
                    if (a.o.window) {
                        const T w = win(f, jj, ii);
                        vx = vx * w; vy = vy * w; vz = vz * w;
                    }
                    jc[o1] = vx;
                    jc[o1 + CAP(1)] = vy;
                    jc[o1 + 2 * CAP(1)] = vz;
                }
                jfx[k] = ax;
                jfy[k] = ay;
                jfz[k] = azv;
            }
            jzp[k] = jz;
        }
    };

    // top centre nz-1 = face nz-2 (registers), written by the loop-F owners
    auto top_centre = [&]() {
        T* const jc = sm + O_JC + ((nz - 1) % 3) * 3 * CAP(1);
#pragma unroll
        for (int k = 0; k < NL1; ++k) {
            if (G1[k] < 0) continue;
            const int o1 = tid + k * NT;
            T vx = jfx[k], vy = jfy[k], vz = jfz[k];
            if (a.o.window) {
                const int row = o1 / pw<EDGE>(1);
                const T w = win(nz - 1, y0 + row - 1, x0 + (o1 - row * pw<EDGE>(1)) - 1);
                vx = vx * w; vy = vy * w; vz = vz * w;
            }
            jc[o1] = vx;
            jc[o1 + CAP(1)] = vy;
            jc[o1 + 2 * CAP(1)] = vz;
        }
    };

    // ---- loop E pieces (level-0 entry: box offsets o1, o2, global cell jj, ii)
    auto diag_cell = [&](int qd, int o1, int o2, int jj, int ii) {
        if (qd < c0 || qd >= c1) return;
        T bx, by, bz, div;
        if (qd > 0 && qd < nz - 1 && xy_in(jj, ii)) {
            const T* const bq = sm + O_BG + ((qd & 3) * 3) * CAP(1) + o1;
            const T* const cq = sm + O_CXY + ((qd % 3) * 2) * CAP(1) + o1;
            const T* const czq = sm + O_CZ + (qd & 3) * CAP(2) + o2;
            const T* const bzm = sm + O_BG + (((qd + 3) & 3) * 3 + 2) * CAP(1) + o1;
            const T* const bzp = sm + O_BG + (((qd + 1) & 3) * 3 + 2) * CAP(1) + o1;
            const T* const czm = sm + O_CZ + ((qd + 3) & 3) * CAP(2) + o2;
            const T* const czpp = sm + O_CZ + ((qd + 1) & 3) * CAP(2) + o2;
            bx = bq[0] + cq[0];
            by = bq[CAP(1)] + cq[CAP(1)];
            bz = bq[2 * CAP(1)] + czq[0];
            div = ((bq[1] + cq[1]) - (bq[-1] + cq[-1])) * i2dx +
                  ((bq[CAP(1) + pw<EDGE>(1)] + cq[CAP(1) + pw<EDGE>(1)]) - (bq[CAP(1) - pw<EDGE>(1)] + cq[CAP(1) - pw<EDGE>(1)])) * i2dy +
                  ((bzp[0] + czpp[0]) - (bzm[0] + czm[0])) * i2dz;
        } else {
            bx = BB(qd, 0, jj, ii);
            by = BB(qd, 1, jj, ii);
            bz = BB(qd, 2, jj, ii);
            div = d1<T>([&](int t) { return BB(qd, 0, jj, t); }, ii, nx, i2dx) +
                  d1<T>([&](int t) { return BB(qd, 1, t, ii); }, jj, ny, i2dy) +
                  d1<T>([&](int t) { return BB(t, 2, jj, ii); }, qd, nz, i2dz);
        }
        T bm = sqrt(bx * bx + by * by + bz * bz);
        red[2] += fabs((double)div);
        red[3] += (double)bm;
        red[4] += (double)(bx * bx + by * by + bz * bz);
    };
    auto sb_cell = [&](int cc, int o1, int gq, int jj, int ii) {
        if (cc < c0 || cc >= c1) return;
        T s_b;
        if (xy_in(jj, ii)) {
            const T* const jx = sm + O_JC + (cc % 3) * 3 * CAP(1) + o1;
            const T* const jy = jx + CAP(1);
            s_b = (jx[pw<EDGE>(1)] - jx[-pw<EDGE>(1)]) * i2dy - (jy[1] - jy[-1]) * i2dx;
        } else {
            s_b = d1<T>([&](int t) { return JC(cc, 0, t, ii); }, jj, ny, i2dy) -
                  d1<T>([&](int t) { return JC(cc, 1, jj, t); }, ii, nx, i2dx);
        }
        sb_out[(long long)cc * P + gq] = s_b;
        red[5] += (double)s_b * (double)s_b;
    };
    auto sj_cell = [&](int cc, int o1, int jj, int ii) {
        if (cc < c0 || cc >= c1 || cc < 1 || cc > nz - 2) return;
        if (!xy_in(jj, ii)) return;
        const T* const jm = sm + O_JC + ((cc + 2) % 3) * 3 * CAP(1) + o1;
        const T* const jp = sm + O_JC + ((cc + 1) % 3) * 3 * CAP(1) + o1;
        const T* const z = sm + O_JC + (cc % 3) * 3 * CAP(1) + 2 * CAP(1) + o1;
        T jz0 = z[0];
        T lap = ((z[1] - T(2) * jz0) + z[-1]) * idx2 + ((z[pw<EDGE>(1)] - T(2) * jz0) + z[-pw<EDGE>(1)]) * idy2;
        T dxz = (((jp[1] - jm[1]) - jp[-1]) + jm[-1]) * i4xz;
        T dyz = (((jp[CAP(1) + pw<EDGE>(1)] - jm[CAP(1) + pw<EDGE>(1)]) - jp[CAP(1) - pw<EDGE>(1)]) + jm[CAP(1) - pw<EDGE>(1)]) * i4yz;
        sj_out[(long long)cc * FPI + (long long)(jj - 1) * (nx - 2) + (ii - 1)] = lap - dxz - dyz;
    };
    auto loop_e = [&](int p, bool post) {
#pragma unroll
        for (int k = 0; k < NL0; ++k) {
            if (G0[k] < 0) continue;
            const int q = tid + k * NT, row = q / pw<EDGE>(0);
            const int jj = y0 + row, ii = x0 + (q - row * pw<EDGE>(0));
            const int o1 = liftE<EDGE, 0, 1>(q, row), o2 = liftE<EDGE, 0, 2>(q, row);
            if (post) {
                sb_cell(nz - 1, o1, G0[k], jj, ii);
                sj_cell(nz - 2, o1, jj, ii);
                continue;
            }
            if (p == 2) diag_cell(0, o1, o2, jj, ii);
            if (p >= 2) diag_cell(p - 1, o1, o2, jj, ii);
            if (p == nz - 1) diag_cell(nz - 1, o1, o2, jj, ii);
            if (p == 1 && pstart == 0) sb_cell(0, o1, G0[k], jj, ii);
            if (p >= 2 && p - 2 >= pstart) {
                sb_cell(p - 1, o1, G0[k], jj, ii);
                sj_cell(p - 2, o1, jj, ii);
            }
        }
    };

    // ---------------- the z march over planes [pstart, pend]
    // C_z of plane p + 1 is formed in the same phase as loop E of plane p:
    // its input Phi(p + 1) is staged with plane p, and the four-slot C_z ring
    // keeps planes p - 2 .. p (read by loop E) apart from p + 1.
    stage_plane(pstart);
    cp_wait_all();
    __syncthreads();
    loop_a(pstart);
    for (int p = pstart; p <= pend; ++p) {
        cp_wait_all();
        __syncthreads();  // B1: plane p staged, C_z(p) complete; iteration p-1 finished everywhere
        if (p < pend) stage_plane(p + 1);
        loop_f(p);
        __syncthreads();  // B2
        loop_e(p, false);
        if (p < pend) loop_a(p + 1);
    }
    if (pend == nz - 1) {
        __syncthreads();
        top_centre();
        __syncthreads();
        loop_e(nz - 1, true);
    }

    block_reduce<NFGS_NRED>(red, shred);
    if (tid == 0) {
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
        for (int q = 0; q < NFGS_NRED; ++q) a.partials[q * nb + b] = red[q];
    }
}

template <typename T>
__global__ void __launch_bounds__(NT, min_blocks<T>()) k_stencil(Args a) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    __shared__ double shred[NFGS_NRED * 32];
    if (a.skip != nullptr && *a.skip) return;
    const int nx = a.g.nx, ny = a.g.ny;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tw = ((int)blockIdx.x == a.gx - 1) ? nx - x0 : TX;
    const int th = ((int)blockIdx.y == a.gy - 1) ? ny - y0 : TY;
    // the level-2 box [x0-2, x0+tw+2) x [y0-2, y0+th+2) stays off the walls
    const bool interior = x0 - 2 >= 1 && x0 + tw + 1 <= nx - 2 && y0 - 2 >= 1 && y0 + th + 1 <= ny - 2;
    if (interior) stencil_body<T, false>(a, sm_raw, shred);
    else stencil_body<T, true>(a, sm_raw, shred);
}

}  // namespace fs
