// Fused stencil pass of one NFPT iteration, warp-row form.  Same arithmetic
// and outputs as fs::k_stencil (carrier and state J_z, vertical-face current,
// sigma_J / divB / energy / sum S_B^2 partials, J_parallel at centres,
// sources S_B and S_J; nfgs_solver.py:3311-3341, 5738-5895, 2689-2697,
// 6697-6745), with a thread layout that removes the per-entry index work:
//
// * A CTA owns a W x H = 30 x 14 output tile and one z segment.  Its 16
//   warps are the 16 rows of the tile's level-1 box (tile rows -1 .. H) and
//   the 32 lanes its 32 columns (tile columns -1 .. W), so every thread owns
//   one column of cells, fixed for the whole z-march: the face current,
//   alpha_f B_f, the carrier and the centre current of its own cell are
//   formed once per plane with no index arithmetic, and the values a cell
//   needs again one plane later (B, C_x, C_y, J_z, alpha_f B_f of the face
//   below) stay in its registers.
// * Shared memory holds only what neighbours read: Phi_c (halo 3) and A_z
//   (halo 2) plane boxes staged with cp.async one plane ahead, C_z (halo 2),
//   B_x / B_y of the last three planes (divB) and J_parallel of the last
//   three centres (S_B, S_J).  All boxes share one pitch, so a neighbour is
//   the thread's own offset plus a compile-time constant.  The level-2 ring
//   of C_z (the 100 cells outside the level-1 box) is formed by the warps
//   that have no level-0 work.
// * B_background is read straight into registers for the thread's own cell,
//   one plane ahead.
// * Tiles do not merge axis remainders: the last tile of an axis is shifted
//   back to end on the wall (it recomputes cells of its neighbour but only
//   writes and sums the cells it owns), so every tile is W x H and the
//   one-sided wall stencils always find their samples.
// * Tiles with a cell of level <= 2 on a lateral wall (EDGE) select the
//   one-sided forms per cell (x walls per lane, y walls per warp); interior
//   tiles compile them out.
//
// Per plane p, two CTA barriers:
//   S1: plane p staged, C_z(p) complete -> stage plane p+1
//   F : C_x, C_y, J_z, B at p; face p-1/2 (current, sigma terms, alpha B_f);
//       centre p-1 (J_parallel)
//   S2
//   E : divB/|B|/|B|^2 at centre p-1, S_B(p-1), S_J(p-2)   (level-0 threads)
//   A : C_z(p+1) on level 2
#pragma once
#include <type_traits>

#include "nfgs_stencil.cuh"

namespace fs2 {

using fs::Args;

constexpr int W = 30, H = 14;                 // output tile (x, y)
constexpr int NW = H + 2;                     // warps: level-1 rows -1 .. H
constexpr int NT = 32 * NW;                   // 512 threads
constexpr int SP = W + 8;                     // common pitch: tile columns -3 .. W+2, one column of alignment
                                              // slack, even (8-byte rows)
constexpr int CAP3 = (H + 6) * SP, CAP2 = (H + 4) * SP, CAP1 = (H + 2) * SP;
constexpr int O_PHI = 0;                      // 4 planes x CAP3, slot plane & 3
constexpr int O_AZ = O_PHI + 4 * CAP3;        // 2 planes x CAP2, slot plane & 1
constexpr int O_CZ = O_AZ + 2 * CAP2;         // 3 planes x CAP2, slot plane % 3
constexpr int O_BXY = O_CZ + 3 * CAP2;        // 3 planes x 2 comps x CAP1
constexpr int O_JP = O_BXY + 6 * CAP1;        // 3 centres x 3 comps x CAP1
constexpr int N_TOTAL = O_JP + 9 * CAP1;
// two rows of slack past the last box: a one-sided y stencil the compiler
// evaluates unconditionally stays inside the allocation
constexpr int N_ALLOC = N_TOTAL + 2 * SP + 4;
constexpr int NRING = 2 * (W + 4) + 2 * (H + 2);  // level-2 cells outside the level-1 box
static_assert(NRING <= NT, "ring fits one entry per thread");
// staging items: chunks of CW elements of the Phi (H+6 rows) and A_z (H+4 rows) boxes
template <int CW> __host__ __device__ constexpr int n_items() { return (2 * H + 10) * (SP / CW); }
template <int CW> __host__ __device__ constexpr int n_entries() { return (n_items<CW>() + NT - 1) / NT; }
static_assert(SP % 2 == 0 && CAP3 % 2 == 0 && CAP2 % 2 == 0 && CAP1 % 2 == 0, "8-byte chunks stay aligned");

template <typename T> constexpr size_t smem_bytes() { return (size_t)N_ALLOC * sizeof(T); }
template <typename T> constexpr int min_blocks() { return sizeof(T) == 4 ? 2 : 1; }

__host__ __device__ inline int tiles(int n, int t) { return (n + t - 1) / t; }
// tile origin: the last tile of an axis ends on the wall
__host__ __device__ inline int origin(int b, int n, int t) { return n >= t ? min(b * t, n - t) : 0; }

template <int B>
__device__ __forceinline__ void cp_async_z(unsigned dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(dst), "l"(src), "n"(B),
                 "r"(valid ? B : 0)
                 : "memory");
}

// d/dx at a cell of a box (pitch-1 neighbours) with the wall form `w`
// (-1 first cell, +1 last cell, 0 central); nfgs_solver.py:1361-1419
template <typename T>
__device__ __forceinline__ T d1w(const T* f, int step, int w, T inv2h) {
    if (w == 0) return (f[step] - f[-step]) * inv2h;
    if (w < 0) return (T(-3) * f[0] + T(4) * f[step] - f[2 * step]) * inv2h;
    return (T(3) * f[0] - T(4) * f[-step] + f[-2 * step]) * inv2h;
}
// one axis of the mirrored-Neumann Laplacian numerator; nfgs_solver.py:1741-1749
template <typename T>
__device__ __forceinline__ T lapw(const T* f, int step, int w) {
    if (w == 0) return (f[step] - T(2) * f[0]) + f[-step];
    if (w < 0) return T(2) * f[step] - T(2) * f[0];
    return T(2) * f[-step] - T(2) * f[0];
}

// square root and quotient of the pass: FP32 takes the hardware
// approximations (sqrt.approx: 2^-23 relative; the fast divide: 2 ulp),
// FP64 the correctly rounded operations
template <typename T> __device__ __forceinline__ T root(T x) { return sqrt(x); }
template <> __device__ __forceinline__ float root<float>(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <typename T> __device__ __forceinline__ T quot(T a, T b) { return a / b; }
template <> __device__ __forceinline__ float quot<float>(float a, float b) { return __fdividef(a, b); }

template <typename T, bool EDGE, int CW>
__device__ __forceinline__ void body(const Args& a, unsigned char* sm_raw, double* shred) {
    T* const sm = (T*)sm_raw;
    const unsigned sbase = (unsigned)__cvta_generic_to_shared(sm_raw);
    const Geo g = a.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int bx = blockIdx.x, by = blockIdx.y;
    const int x0 = origin(bx, nx, W), y0 = origin(by, ny, H);
    // own column: tile cell (r, c) = (w - 1, lane - 1)
    const int jj = y0 + w - 1, ii = x0 + lane - 1;
    const bool inD = jj >= 0 && jj < ny && ii >= 0 && ii < nx;
    const bool own = inD && w >= 1 && w <= H && lane >= 1 && lane <= W && ii >= bx * W && jj >= by * H;
    const int xw = EDGE ? (ii == 0 ? -1 : (ii == nx - 1 ? 1 : 0)) : 0;
    const int yw = EDGE ? (jj == 0 ? -1 : (jj == ny - 1 ? 1 : 0)) : 0;
    const bool xin = !EDGE || (ii > 0 && ii < nx - 1 && jj > 0 && jj < ny - 1);
    const int gq = inD ? jj * nx + ii : 0;
    // box column 0 is global column xs: x0 - 3, rounded down to even for
    // 8-byte staging chunks; tile column c sits at box column c + 3 + dx8
    const int dx8 = (CW == 2) ? ((x0 - 3) & 1) : 0;
    const int xs = x0 - 3 - dx8;
    const int o1 = w * SP + lane + 2 + dx8;  // own cell in a level-1 box
    const int o2 = o1 + SP;            // ... in a level-2 box
    const int o3 = o1 + 2 * SP;        // ... in a level-3 box
    // z segment: output centres [c0, c1), planes [pstart, pend]
    const int per = (nz + a.nseg - 1) / a.nseg;
    const int c0 = blockIdx.z * per, c1 = min(nz, c0 + per);
    const int pstart = max(0, c0 - 2), pend = min(nz - 1, c1 + 1);

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

    // ---- staging entries: item e = tid + k NT is chunk e % (SP / CW) of box
    // row e / (SP / CW), Phi rows first, then A_z rows.  ent_g: in-plane
    // offset of the chunk (-1 outside the domain: zero fill, -2 no item);
    // ent_s: box offset, | AZ_ITEM for A_z items
    constexpr int NCH = SP / CW, NE = n_entries<CW>(), AZ_ITEM = 1 << 20;
    int ent_g[NE], ent_s[NE];
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        const int e = tid + k * NT;
        int gv = -2, sv = 0;
        if (e < n_items<CW>()) {
            const bool isa = e >= (H + 6) * NCH;
            const int ee = isa ? e - (H + 6) * NCH : e;
            const int br = ee / NCH, bc = (ee % NCH) * CW;
            const int r = y0 - (isa ? 2 : 3) + br, c = xs + bc;
            gv = (r >= 0 && r < ny && c >= 0 && c + CW - 1 < nx) ? r * nx + c : -1;
            sv = (br * SP + bc) | (isa ? AZ_ITEM : 0);
        }
        ent_g[k] = gv;
        ent_s[k] = sv;
    }
    auto hi_of = [&](int p) __attribute__((always_inline)) { return min(nz - 1, max(p + 1, 2)); };
    auto lo_of = [&](int p) __attribute__((always_inline)) { return max(0, min(p - 1, nz - 3)); };
    auto stage_plane = [&](int p) __attribute__((always_inline)) {
        const int from = (p == pstart) ? lo_of(p) : hi_of(p - 1) + 1;
        for (int pl = from; pl <= hi_of(p); ++pl) {
            const T* src = phi + (long long)pl * P;
            const unsigned dst = sbase + (unsigned)((O_PHI + (pl & 3) * CAP3) * sizeof(T));
#pragma unroll
            for (int k = 0; k < NE; ++k)
                if (ent_g[k] >= -1 && !(ent_s[k] & AZ_ITEM))
                    cp_async_z<CW * sizeof(T)>(dst + ent_s[k] * sizeof(T), src + max(ent_g[k], 0), ent_g[k] >= 0);
        }
        const T* src = az + (long long)p * P;
        const unsigned dst = sbase + (unsigned)((O_AZ + (p & 1) * CAP2) * sizeof(T));
#pragma unroll
        for (int k = 0; k < NE; ++k)
            if (ent_g[k] >= -1 && (ent_s[k] & AZ_ITEM))
                cp_async_z<CW * sizeof(T)>(dst + (ent_s[k] - AZ_ITEM) * sizeof(T), src + max(ent_g[k], 0),
                                           ent_g[k] >= 0);
        fs::cp_commit();
    };

    // ---- level-2 ring cell of this thread (warps without level-0 work first)
    int ro2 = -1;  // level-2 box offset of the ring cell, -1 when none
    {
        const int q = (w == 0) ? 0 : NW - w;
        const int t = q * 32 + lane;
        if (t < NRING) {
            int r, c;
            if (t < W + 4) { r = -2; c = t - 2; }
            else if (t < 2 * (W + 4)) { r = H + 1; c = t - (W + 4) - 2; }
            else { const int u = t - 2 * (W + 4); r = -1 + (u >> 1); c = (u & 1) ? W + 1 : -2; }
            ro2 = (r + 2) * SP + c + 3 + dx8;
        }
    }

    // C_z at a level-2 cell (box offset q2 = level-2 offset; global jj2, ii2)
    auto cz_cell = [&](int p, int q2, int jj2, int ii2, bool in2) __attribute__((always_inline)) -> T {
        if (p == 0) {
            if (!in2) return T(0);
            const long long q = (long long)jj2 * nx + ii2;
            return bzobs[q] - bbg[2 * V + q];
        }
        const T* f = sm + O_PHI + (p & 3) * CAP3 + q2 + SP;  // level-3 offset
        if (!EDGE) return ((f[1] - T(2) * f[0]) + f[-1]) * idx2 + ((f[SP] - T(2) * f[0]) + f[-SP]) * idy2;
        const int cw = in2 ? (ii2 == 0 ? -1 : (ii2 == nx - 1 ? 1 : 0)) : 0;
        const int rw = in2 ? (jj2 == 0 ? -1 : (jj2 == ny - 1 ? 1 : 0)) : 0;
        return lapw<T>(f, 1, cw) * idx2 + lapw<T>(f, SP, rw) * idy2;
    };
    auto loop_a = [&](int p) __attribute__((always_inline)) {
        T* const cz = sm + O_CZ + (p % 3) * CAP2;
        cz[o2] = cz_cell(p, o2, jj, ii, inD);
        if (ro2 >= 0) {
            // global cell of the ring entry, recomputed here to keep registers free
            const int rjj = y0 + ro2 / SP - 2, rii = xs + ro2 % SP;
            const bool rin = rjj >= 0 && rjj < ny && rii >= 0 && rii < nx;
            cz[ro2] = cz_cell(p, ro2, rjj, rii, rin);
        }
    };

    // ---- per-thread state across planes
    T cxp = T(0), cyp = T(0), jzp = T(0);        // C_x, C_y, J_z at plane p-1
    T afx = T(0), afy = T(0), afz = T(0);        // alpha_f B_f at face p-3/2
    T bxp = T(0), byp = T(0), bzp = T(0);        // B at plane p-1
    T bzpp = T(0);                               // B_z at plane p-2
    T bgn0 = T(0), bgn1 = T(0), bgn2 = T(0);     // B_background at the next plane
    // per-thread partial sums: FP32 storage sums its (at most a few dozen)
    // terms per thread in FP32, FP64 storage in FP64; blocks add them in FP64
    using Acc = typename std::conditional<sizeof(T) == 4, float, double>::type;
    Acc red[NFGS_NRED] = {0, 0, 0, 0, 0, 0};

    auto load_bg = [&](int p) __attribute__((always_inline)) {
        if (inD) {
            const long long q = (long long)p * P + gq;
            bgn0 = __ldg(bbg + q);
            bgn1 = __ldg(bbg + V + q);
            bgn2 = __ldg(bbg + 2 * V + q);
        }
    };
    auto win = [&](int c) __attribute__((always_inline)) -> T { return (wz[c] * wy[jj]) * wx[ii]; };

    // per-thread constant: the own cell lies in the sigma_J box's x-y range
    const bool sbox = own && jj >= a.box.y0 && jj < a.box.y1 && ii >= a.box.x0 && ii < a.box.x1;

    // divB / |B| / |B|^2 at centre qd of the own cell: B own, B_x / B_y of
    // plane qd in ring slot `slot`, dBz/dz given
    auto diag = [&](int slot, T bx, T by, T bz, T dbz) __attribute__((always_inline)) {
        const T* const Bx = sm + O_BXY + (slot * 2) * CAP1 + o1;
        const T* const By = Bx + CAP1;
        const T div = d1w<T>(Bx, 1, xw, i2dx) + d1w<T>(By, SP, yw, i2dy) + dbz;
        const T b2 = bx * bx + by * by + bz * bz;
        red[2] += fabs((Acc)div);
        red[3] += (Acc)root<T>(b2);
        red[4] += (Acc)b2;
    };
    auto sb_cell = [&](int cc, int slot) __attribute__((always_inline)) {
        const T* const jx = sm + O_JP + slot * 3 * CAP1 + o1;
        const T* const jy = jx + CAP1;
        const T s_b = d1w<T>(jx, SP, yw, i2dy) - d1w<T>(jy, 1, xw, i2dx);
        sb_out[(long long)cc * P + gq] = s_b;
        red[5] += (Acc)s_b * (Acc)s_b;
    };
    // S_J at centre cc: J_par x/y of centres cc -/+ 1 in slots sm1 / sp1, J_par z of cc in slot s0
    auto sj_cell = [&](int cc, int sm1, int s0, int sp1) __attribute__((always_inline)) {
        if (!xin) return;
        const T* const jm = sm + O_JP + sm1 * 3 * CAP1 + o1;
        const T* const jp = sm + O_JP + sp1 * 3 * CAP1 + o1;
        const T* const z = sm + O_JP + s0 * 3 * CAP1 + 2 * CAP1 + o1;
        const T jz0 = z[0];
        const T lap = ((z[1] - T(2) * jz0) + z[-1]) * idx2 + ((z[SP] - T(2) * jz0) + z[-SP]) * idy2;
        const T dxz = (((jp[1] - jm[1]) - jp[-1]) + jm[-1]) * i4xz;
        const T dyz = (((jp[CAP1 + SP] - jm[CAP1 + SP]) - jp[CAP1 - SP]) + jm[CAP1 - SP]) * i4yz;
        sj_out[(long long)cc * FPI + (long long)(jj - 1) * (nx - 2) + (ii - 1)] = lap - dxz - dyz;
    };
    auto put_centre = [&](int slot, T vx, T vy, T vz) __attribute__((always_inline)) {
        T* const jc = sm + O_JP + slot * 3 * CAP1 + o1;
        jc[0] = vx;
        jc[CAP1] = vy;
        jc[2 * CAP1] = vz;
    };
    auto r3 = [](int q) __attribute__((always_inline)) { return q % 3; };

    // ---- one plane of the z-march.  STEADY: a plane whose face, centre and
    // every level-0 product lie inside the segment and away from the bottom
    // and top planes, so the plane-position branches compile out.
    auto plane = [&](int p, auto steady) __attribute__((always_inline)) {
        constexpr bool STEADY = decltype(steady)::value;
        const int s0 = r3(p), sm1 = s0 == 0 ? 2 : s0 - 1, sm2 = sm1 == 0 ? 2 : sm1 - 1;
        fs::cp_wait_all();
        __syncthreads();  // S1: plane p staged, C_z(p) complete, plane p-1 finished everywhere
        if (STEADY || p < pend) stage_plane(p + 1);
        const T bg0 = bgn0, bg1 = bgn1, bg2 = bgn2;
        if (STEADY || p < pend) load_bg(p + 1);

        // ---- F: carrier and J_z at p
        const T* const A = sm + O_AZ + (p & 1) * CAP2 + o2;
        T cx, cy, jz;
        {
            const bool zin = STEADY || (p > 0 && p < nz - 1);
            const T* Z0;
            const T* Z1;
            const T* Z2;
            if (zin) {
                Z0 = sm + O_PHI + ((p + 1) & 3) * CAP3 + o3;
                Z1 = sm + O_PHI + ((p + 3) & 3) * CAP3 + o3;
                Z2 = Z1;
            } else if (p == 0) {
                Z0 = sm + O_PHI + 0 * CAP3 + o3;
                Z1 = sm + O_PHI + 1 * CAP3 + o3;
                Z2 = sm + O_PHI + 2 * CAP3 + o3;
            } else {
                Z0 = sm + O_PHI + ((nz - 1) & 3) * CAP3 + o3;
                Z1 = sm + O_PHI + ((nz - 2) & 3) * CAP3 + o3;
                Z2 = sm + O_PHI + ((nz - 3) & 3) * CAP3 + o3;
            }
            auto dzp = [&](int d) __attribute__((always_inline)) -> T {
                if (zin) return (Z0[d] - Z1[d]) * i2dz;
                if (p == 0) return (T(-3) * Z0[d] + T(4) * Z1[d] - Z2[d]) * i2dz;
                return (T(3) * Z0[d] - T(4) * Z1[d] + Z2[d]) * i2dz;
            };
            T dxdz, dydz;
            if (xw == 0) dxdz = (dzp(1) - dzp(-1)) * i2dx;
            else if (xw < 0) dxdz = (T(-3) * dzp(0) + T(4) * dzp(1) - dzp(2)) * i2dx;
            else dxdz = (T(3) * dzp(0) - T(4) * dzp(-1) + dzp(-2)) * i2dx;
            if (yw == 0) dydz = (dzp(SP) - dzp(-SP)) * i2dy;
            else if (yw < 0) dydz = (T(-3) * dzp(0) + T(4) * dzp(SP) - dzp(2 * SP)) * i2dy;
            else dydz = (T(3) * dzp(0) - T(4) * dzp(-SP) + dzp(-2 * SP)) * i2dy;
            const T dya = d1w<T>(A, SP, yw, i2dy);
            const T dxa = d1w<T>(A, 1, xw, i2dx);
            cx = -dxdz + dya;
            cy = -dydz - dxa;
            if (!STEADY && p == 0) {
                jz = inD ? jzt[gq] : T(0);
            } else if ((!STEADY && p == nz - 1) || !xin) {
                jz = T(0);
            } else {
                const T a0 = A[0];
                jz = -(((A[1] - T(2) * a0) + A[-1]) * idx2 + ((A[SP] - T(2) * a0) + A[-SP]) * idy2);
            }
            if (a.use_h) { cx = cx + hx; cy = cy + hy; }
        }
        const T* const czp = sm + O_CZ + s0 * CAP2 + o2;
        const T bx1 = bg0 + cx, by1 = bg1 + cy, bz1 = bg2 + czp[0];
        {
            T* const bxy = sm + O_BXY + (s0 * 2) * CAP1 + o1;
            bxy[0] = bx1;
            bxy[CAP1] = by1;
        }
        // ---- face f = p - 1 (between planes p-1 and p) and centre f
        const int f = p - 1;
        if (STEADY || f >= pstart) {
            const bool sig = (STEADY || (f >= c0 && f < c1)) && f >= a.box.z0 && f < a.box.z1;
            const T bfx = T(0.5) * (bx1 + bxp), bfy = T(0.5) * (by1 + byp), bfz = T(0.5) * (bz1 + bzp);
            const T dbx = (cx - cxp) * idz;
            const T dby = (cy - cyp) * idz;
            const T* const z0 = sm + O_CZ + sm1 * CAP2 + o2;  // plane p-1
            auto czf = [&](int d) __attribute__((always_inline)) -> T { return T(0.5) * (czp[d] + z0[d]); };
            T gyz, gxz;
            if (yw == 0) gyz = (czf(SP) - czf(-SP)) * i2dy;
            else if (yw < 0) gyz = (T(-3) * czf(0) + T(4) * czf(SP) - czf(2 * SP)) * i2dy;
            else gyz = (T(3) * czf(0) - T(4) * czf(-SP) + czf(-2 * SP)) * i2dy;
            if (xw == 0) gxz = (czf(1) - czf(-1)) * i2dx;
            else if (xw < 0) gxz = (T(-3) * czf(0) + T(4) * czf(1) - czf(2)) * i2dx;
            else gxz = (T(3) * czf(0) - T(4) * czf(-1) + czf(-2)) * i2dx;
            const T jxf = gyz - dby;
            const T jyf = dbx - gxz;
            const T jzf = T(0.5) * (jz + jzp);
            const T bf2 = bfx * bfx + bfy * bfy + bfz * bfz;
            if (sig && sbox) {
                const T cxq = jyf * bfz - jzf * bfy;
                const T cyq = jzf * bfx - jxf * bfz;
                const T czq = jxf * bfy - jyf * bfx;
                T bn = root<T>(bf2);
                bn = bn > T(1e-10) ? bn : T(1e-10);
                red[0] += (Acc)quot<T>(root<T>(cxq * cxq + cyq * cyq + czq * czq), bn);
                red[1] += (Acc)root<T>(jxf * jxf + jyf * jyf + jzf * jzf);
            }
            const T b2 = bf2 > fl ? bf2 : fl;
            T alpha = quot<T>(jxf * bfx + jyf * bfy + jzf * bfz, b2);
            if (amax > T(0)) alpha = fmin(fmax(alpha, -amax), amax);
            const T ax = alpha * bfx, ay = alpha * bfy, azv = alpha * bfz;
            if (!STEADY && f == 0) {
                // bottom row of J_par (nfgs_solver.py:6697-6713)
                const bool wall = !xin;
                T vx, vy, vz;
                if (a.o.polarity == 0) {
                    vz = inD ? jzt[gq] : T(0);
                    if (a.o.face_exact) { vx = ax; vy = ay; }
                    else { vx = wall ? T(0) : jxf; vy = wall ? T(0) : jyf; }
                } else {
                    const T bzv = inD ? bzobs[gq] : T(0);
                    const bool m = (a.o.polarity == 1) ? (bzv > T(0)) : (bzv < T(0));
                    vx = m ? (wall ? T(0) : jxf) : T(0);
                    vy = m ? (wall ? T(0) : jyf) : T(0);
                    vz = m ? (inD ? jzt[gq] : T(0)) : T(0);
                }
                if (a.o.window && inD) {
                    const T wv = win(0);
                    vx = vx * wv; vy = vy * wv; vz = vz * wv;
                }
                put_centre(0, vx, vy, vz);
            } else if (STEADY || (f >= 1 && f - 1 >= pstart)) {
                T vx = T(0.5) * (afx + ax), vy = T(0.5) * (afy + ay), vz = T(0.5) * (afz + azv);
                if (a.o.window && inD) {
                    const T wv = win(f);
                    vx = vx * wv; vy = vy * wv; vz = vz * wv;
                }
                put_centre(sm1, vx, vy, vz);
            }
            afx = ax;
            afy = ay;
            afz = azv;
        }
        cxp = cx;
        cyp = cy;
        jzp = jz;
        __syncthreads();  // S2
        // ---- E: level-0 work of the own cell
        if (own) {
            if (STEADY) {
                diag(sm1, bxp, byp, bzp, (bz1 - bzpp) * i2dz);
                sb_cell(p - 1, sm1);
                sj_cell(p - 2, s0, sm2, sm1);  // J_par x/y of p-3 share slot p % 3
            } else {
                auto in_seg = [&](int q) __attribute__((always_inline)) { return q >= c0 && q < c1; };
                if (p == 2 && in_seg(0)) {
                    // centre 0 (one-sided in z): B(0) from the slot-0 boxes and the B_z history
                    const T* const b0 = sm + O_BXY + o1;
                    diag(0, b0[0], b0[CAP1], bzpp, (T(-3) * bzpp + T(4) * bzp - bz1) * i2dz);
                }
                if (p >= 2 && in_seg(p - 1)) diag(sm1, bxp, byp, bzp, (bz1 - bzpp) * i2dz);
                if (p == nz - 1 && in_seg(nz - 1)) diag(s0, bx1, by1, bz1, (T(3) * bz1 - T(4) * bzp + bzpp) * i2dz);
                if (p == 1 && pstart == 0 && in_seg(0)) sb_cell(0, 0);
                if (p >= 2 && p - 2 >= pstart) {
                    if (in_seg(p - 1)) sb_cell(p - 1, sm1);
                    if (in_seg(p - 2) && p - 2 >= 1 && p - 2 <= nz - 2) sj_cell(p - 2, s0, sm2, sm1);
                }
            }
        }
        bzpp = bzp;
        bxp = bx1;
        byp = by1;
        bzp = bz1;
        // ---- A: C_z(p+1) on level 2
        if (STEADY || p < pend) loop_a(p + 1);
    };

    // ---------------- the z-march
    // steady planes: face, centre and all level-0 products inside [c0, c1),
    // no bottom or top plane
    const int ps = max(pstart + 3, max(c0 + 2, 3));
    const int pe = min(pend - 1, nz - 2);
    load_bg(pstart);
    stage_plane(pstart);
    fs::cp_wait_all();
    __syncthreads();
    loop_a(pstart);
    int p = pstart;
    for (; p <= pend && p < ps; ++p) plane(p, std::false_type{});
    for (; p <= pe; ++p) plane(p, std::true_type{});
    for (; p <= pend; ++p) plane(p, std::false_type{});
    if (pend == nz - 1) {
        __syncthreads();
        // top centre nz-1 = face nz-2 (nfgs_solver.py:5780-5794)
        {
            T vx = afx, vy = afy, vz = afz;
            if (a.o.window && inD) {
                const T wv = win(nz - 1);
                vx = vx * wv; vy = vy * wv; vz = vz * wv;
            }
            put_centre(r3(nz - 1), vx, vy, vz);
        }
        __syncthreads();
        if (own) {
            if (nz - 1 >= c0 && nz - 1 < c1) sb_cell(nz - 1, r3(nz - 1));
            if (nz - 2 >= c0 && nz - 2 < c1 && nz - 2 >= 1) sj_cell(nz - 2, r3(nz - 3), r3(nz - 2), r3(nz - 1));
        }
    }

    double rd[NFGS_NRED];
#pragma unroll
    for (int q = 0; q < NFGS_NRED; ++q) rd[q] = (double)red[q];
    block_reduce<NFGS_NRED>(rd, shred);
    if (tid == 0) {
        const long long nb = (long long)gridDim.x * gridDim.y * gridDim.z;
        const long long b = ((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
#pragma unroll
        for (int q = 0; q < NFGS_NRED; ++q) a.partials[q * nb + b] = rd[q];
    }
}

template <typename T, int CW>
__global__ void __launch_bounds__(NT, min_blocks<T>()) k_stencil2(Args a) {
    extern __shared__ __align__(16) unsigned char sm_raw[];
    __shared__ double shred[NFGS_NRED * 32];
    if (a.skip != nullptr && *a.skip) return;
    const int nx = a.g.nx, ny = a.g.ny;
    const int x0 = origin(blockIdx.x, nx, W), y0 = origin(blockIdx.y, ny, H);
    // the level-2 box [x0-2, x0+W+2) x [y0-2, y0+H+2) stays off the walls
    const bool interior = nx >= W && ny >= H && x0 - 2 >= 1 && x0 + W + 1 <= nx - 2 && y0 - 2 >= 1 &&
                          y0 + H + 1 <= ny - 2;
    if (interior) body<T, false, CW>(a, sm_raw, shred);
    else body<T, true, CW>(a, sm_raw, shred);
}

}  // namespace fs2
