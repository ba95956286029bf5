// Tensor-core (tcgen05) DCT-I / DST-I contractions along one axis.
//
// The reference builds the transforms by mirroring and rfft
// (nfgs_solver.py:1019-1081).  Here a transform of length N (DCT-I) or
// n = N - 2 (DST-I), N - 1 odd, is split by the symmetry m <-> N-1-m into
// two dense P x P contractions (P = (N-2)/2 pairs): with s_m, d_m the pair
// sums / differences of a vector x,
//   DCT-I   X_{2j+2} = (x_0 + x_{N-1}) + sum_m s_m 2cos(pi (2j+2) m/(N-1))
//           X_{2j+1} = (x_0 - x_{N-1}) + sum_m d_m 2cos(pi (2j+1) m/(N-1))
//           X_0 = x_0 + x_{N-1} + 2 sum s_m,  X_{N-1} = x_0 - x_{N-1} + 2 sum (-1)^m d_m
//   DST-I   X_{2j+1} = sum_m s_m 2 sin(pi (2j+1) m/(n+1)),
//           X_{2j+2} = sum_m d_m 2 sin(pi (2j+2) m/(n+1))
// Each contraction runs on the tensor cores as D[mode][vec] = M[mode][pair]
// x data[pair][vec] with FP32 accumulation in TMEM.  Precision: each data
// vector is scaled by its own power of two (undone exactly per output
// column) and split into FP16 hi + lo; the matrix (|entries| <= 2) is split
// likewise; three products hi*hi + hi*lo + lo*hi per K step give ~2^-21
// relative error per product against the vector's maximum.  The tensor
// core's internal accumulation truncates, which biases long running sums
// toward zero: the hi*hi products accumulate in chunks of 32 pairs and the
// correction products apart, each in its own TMEM accumulator, and the
// epilogue adds them in FP32 (round to nearest).
//
// One persistent CTA per SM, warp-specialised and pipelined (NB = 3 tiles
// between operand build and epilogue):
//   * the four matrix operands (two halves, hi and lo; 128 KB) stay resident
//     in shared memory;
//   * the producer warps prefetch raw input tiles (16 vectors, FP32) two
//     tiles ahead with cp.async into a double-buffered staging area
//     (coalesced: vector rows on axis 0, 16-column rows on axis 1), then
//     form the FP16 hi/lo pair sums and differences of tile i in K-major
//     operand layout (NB buffers, 16 KB each);
//   * the last warp issues the MMAs of tile i into one of NB TMEM accumulators;
//   * the epilogue warps drain earlier tiles: TMEM -> registers -> the consumed
//     operand buffer (transposed for axis 1) -> row-contiguous global stores.
// Hand-offs are mbarriers (operands full, MMA done, accumulator free) with
// bounded waits; the producer and epilogue roles decide failures with a
// barrier-reduction so that their named barriers stay uniform.
#pragma once
#include <cuda_fp16.h>
#include "nfgs_common.cuh"

namespace tc {

constexpr int PP = 128;          // padded pair count (K) and modes per half (M)
constexpr int TV = 16;           // vectors per tile (N of the MMA)
constexpr int NPW = 8, NEW = 8;  // producer and epilogue warps
constexpr int NPROD = 32 * NPW, NEPI = 32 * NEW;
constexpr int NTHREADS = NPROD + NEPI + 32;  // + 1 MMA warp
constexpr int MAT_BYTES = PP * PP * 2;        // one fp16 matrix operand: 32 KB
constexpr int DAT_BYTES = PP * TV * 2;        // one fp16 data operand: 4 KB
constexpr int SMEM_MAT = 4 * MAT_BYTES;       // 128 KB
constexpr int NB = 3;                         // operand buffers / accumulators in flight
constexpr int SMEM_DAT = NB * 4 * DAT_BYTES;  // NB buffers of four operands: 48 KB
constexpr int STG_PITCH = 2 * PP + 10;        // axis-0 staging row pitch (floats; 8-byte rows, 16 rows on distinct banks)
constexpr int STG_FLOATS = TV * STG_PITCH;    // one raw tile: 16 rows (axis 0) or 2PP+2 rows of 16 (axis 1)
constexpr int SMEM_STG = 2 * STG_FLOATS * 4;  // double-buffered raw tiles: 33.9 KB
constexpr int SMEM_AUX = 8 * 1024;            // per-vector scalars, partial sums, barriers
constexpr int SMEM_TOTAL = SMEM_MAT + SMEM_DAT + SMEM_STG + SMEM_AUX;
constexpr long long WAIT_LIMIT = 1LL << 22;   // mbarrier polls before giving up
// Wide transforms (128 < P <= 256 pairs): four CTA roles (half, 128-mode
// block), each holding its 128 x 256 slice of one half's matrix (hi, lo:
// 128 KB) and contracting all 256 pairs of that half; one raw staging buffer
// of 16 rows of up to 514 elements.
constexpr int PW_K = 256;                     // K extent of the wide layout
// TMEM accumulators per operand buffer (columns of TV = 16): the hi x hi
// products accumulate in chunks of KC_STEPS K-steps (32 pairs), one
// accumulator each, and the correction products in their own; the
// epilogue adds them in FP32.  Normal: 2 halves x (4 chunks + 1); wide:
// 8 chunks + 1.
constexpr int KC_STEPS = 2;
constexpr int NCH_N = PP / 16 / KC_STEPS;     // hi x hi chunks per half, normal (4)
constexpr int NCH_W = 256 / 16 / KC_STEPS;    // hi x hi chunks, wide (8)
constexpr int ACC_COLS = 2 * (NCH_N + 1) * TV;  // columns per buffer (160)
static_assert(NCH_W + 1 <= 2 * (NCH_N + 1), "wide accumulators fit a buffer's columns");
constexpr int TMEM_COLS = 512;                // allocation (NB * ACC_COLS = 480 used)
static_assert(NB * ACC_COLS <= TMEM_COLS, "accumulators fit the TMEM allocation");
constexpr int STG_PITCH_W = 2 * PW_K + 10;    // wide axis-0 staging pitch (fits the staging area once)
static_assert(TV * STG_PITCH_W <= 2 * TV * STG_PITCH, "wide staging fits");

// Vector / element addressing: addr(v, m) = (v / vpb) * bstride + (v % vpb) * vstride + m * estride
struct Addr {
    long long off;      // element offset of vector 0 (or byte offset when indirected)
    long long vpb, bstride, vstride, estride;
};

struct Args {
    const float* in;
    float* out;           // direct output (or null when out_table is used)
    void* const* out_table;
    const int* out_sel;
    Addr ia, oa;
    int nvec;
    int P;                // real pairs (<= PP)
    int N;                // transform length (DCT: N, DST: n)
    int kind;             // 0 DCT-I, 1 DST-I
    int axis;             // 0: elements contiguous (K-major data), 1: strided (MN-major data)
    float norm;           // 1 or the inverse normalisation
    const uint4* mat;     // 128 KB operand image: [half A hi | half A lo | half B hi | half B lo]
    const int* skip;      // exit when *skip != 0
    int* err;             // set to 1 when a bounded wait runs out
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// UMMA shared-memory descriptor, no swizzle (version 1, base offset 0).
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

__device__ __forceinline__ void mma_f16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false if the limit ran out.
// After a few immediate polls the waiting warp sleeps between polls (up to
// 256 ns) so that it leaves the issue slots to the warps doing the work.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    unsigned ns = 0;
    for (long long it = 0; it < WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (it >= 4) {
            ns = ns == 0 ? 16 : (ns < 256 ? 2 * ns : 256);
            __nanosleep(ns);
        }
    }
    return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// sum over NCH chunk accumulators (8 columns each at col, col + TV, ...)
// and the correction accumulator after them, in FP32 round-to-nearest
template <int NCH>
__device__ __forceinline__ void acc_sum(uint32_t col, float (&v)[8]) {
    float t[8], u[8];
    tmem_ld8(col, v);
    tmem_ld8(col + TV, t);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] += t[q];
#pragma unroll
    for (int c = 2; c < NCH; c += 2) {
        tmem_ld8(col + c * TV, t);
        tmem_ld8(col + (c + 1) * TV, u);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] += t[q] + u[q];
    }
    tmem_ld8(col + NCH * TV, t);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] += t[q];
}

template <int B>
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(src), "n"(B) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// v < 2^31 and vpb < 2^31: the quotient and remainder in 32-bit arithmetic
__device__ __forceinline__ long long vaddr(const Addr& a, long long v) {
    const unsigned uv = (unsigned)v, up = (unsigned)a.vpb;
    const unsigned q = uv / up, r = uv - q * up;
    return a.off + (long long)q * a.bstride + (long long)r * a.vstride;
}

// byte offset of (vec, pair) in a data operand
//   axis 0 (K-major):  (v/8)*2048 + (k/8)*128 + (v%8)*16 + (k%8)*2
//   axis 1 (MN-major): (k/8)*(TV*16) + (v/8)*128 + (k%8)*16 + (v%8)*2
__device__ __forceinline__ uint32_t dat_off(int axis, int v, int k) {
    return axis == 0 ? (uint32_t)((v >> 3) * 2048 + (k >> 3) * 128 + (v & 7) * 16 + (k & 7) * 2)
                     : (uint32_t)((k >> 3) * (TV * 16) + (v >> 3) * 128 + (k & 7) * 16 + (v & 7) * 2);
}

// byte offset of (vec, pair) in a wide K-major data operand (256 pairs)
__device__ __forceinline__ uint32_t dat_off_w(int v, int k) {
    return (uint32_t)((v >> 3) * 4096 + (k >> 3) * 128 + (v & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
// barrier among the producer threads only
__device__ __forceinline__ void producer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(NPROD) : "memory"); }
// barrier among the epilogue threads only
__device__ __forceinline__ void epilogue_sync() { asm volatile("bar.sync 2, %0;" ::"n"(NEPI) : "memory"); }
// barrier of one role (id 1 producers, 2 epilogue; NPROD == NEPI threads) that also ORs a flag
template <int ID>
__device__ __forceinline__ bool role_any(bool x) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)x), "n"(ID), "n"(NPROD)
        : "memory");
    return r != 0;
}

// FP16 hi / lo split of two values at once: hi = rn(x), lo = rn(x - hi), by
// packed conversions (round to nearest even, element by element); hi in `h`,
// lo in `l`, the first value in the low 16 bits of each
__device__ __forceinline__ void split_h2(float x0, float x1, uint32_t& h, uint32_t& l) {
    const __half2 hh = __floats2half2_rn(x0, x1);
    const float2 hf = __half22float2(hh);
    const __half2 ll = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    h = *reinterpret_cast<const uint32_t*>(&hh);
    l = *reinterpret_cast<const uint32_t*>(&ll);
}

// AX: the axis (0 rows, 1 columns), KIND: 0 DCT-I, 1 DST-I -- compile-time, so
// the per-element index and layout choices are not branches (g.axis and
// g.kind must agree)
template <bool WIDE, int AX, int KIND>
__global__ void __launch_bounds__(NTHREADS, 1) k_tc_transform(Args g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* smat = smem;
    unsigned char* sdat = smem + SMEM_MAT;
    float* stg = (float*)(smem + SMEM_MAT + SMEM_DAT);   // [2][STG_FLOATS]
    unsigned char* saux = smem + SMEM_MAT + SMEM_DAT + SMEM_STG;
    // per-buffer tile scalars (written by producers, read by the epilogue)
    long long* obase = (long long*)saux;          // [NB][TV]
    int* vexp = (int*)(obase + NB * TV);          // [NB][TV]
    float* e0 = (float*)(vexp + NB * TV);         // [NB][TV]
    float* e1 = e0 + NB * TV;
    float* sp0 = e1 + NB * TV;
    float* sp1 = sp0 + NB * TV;
    float* vdown = sp1 + NB * TV;                 // [NB][TV] output scale norm * 2^-vexp
    // producer scratch
    float* part = vdown + NB * TV;                // [NPW][TV][2] (sized [16][TV][2])
    float* vmax = part + 32 * TV;                 // [NPW][TV] (sized [16][TV])
    long long* ibase = (long long*)(vmax + 16 * TV);  // [2][TV] input base of each vector (staging buffer)
    uint64_t* bars = (uint64_t*)(ibase + 2 * TV);  // full[NB] mmad[NB] afree[NB]
    uint32_t* tslot = (uint32_t*)(bars + 3 * NB);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // tile group of this CTA (wide: four consecutive CTAs, one per role, take
    // the same tiles, so the input they share is read from L2 after the first)
    const int grp = WIDE ? (int)(blockIdx.x >> 2) : (int)blockIdx.x;
    const int ngrp = WIDE ? (int)(gridDim.x >> 2) : (int)gridDim.x;
    const int role = WIDE ? (int)(blockIdx.x & 3) : 0;
    const int hh = role >> 1, mb = role & 1;    // wide: matrix half and 128-mode block
    const int ntiles = (g.nvec + TV - 1) / TV;
    const uint32_t full0 = smem_u32(bars), mmad0 = smem_u32(bars + NB), afree0 = smem_u32(bars + 2 * NB);
    if (tid == 0) {
        for (int b = 0; b < NB; ++b) {
            mbar_init(full0 + 8 * b, NPROD);
            mbar_init(mmad0 + 8 * b, 1);
            mbar_init(afree0 + 8 * b, NEPI);
        }
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == NPW + NEW) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "n"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = *tslot;
    const int P = g.P, N = g.N;
    constexpr bool dct = KIND == 0;
    bool failed = false;

    // The matrix operands (128 KB, constant) are copied in by the MMA and
    // epilogue warps, which need them first at the first MMA; the copy starts
    // before the wait for the previous kernel (programmatic launch: this
    // prologue may overlap its end), and the producers start on the first
    // tiles meanwhile.
    if (warp >= NPW) {
        const uint32_t d0 = smem_u32(smat);
        const uint4* src = g.mat + (size_t)role * (SMEM_MAT / 16);
        for (int q = tid - NPROD; q < SMEM_MAT / 16; q += NEPI + 32) cp_async4<16>(d0 + 16u * q, src + q);
        cp_commit();
    }
    auto load_matrices = [&]() {
        cp_wait0();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("bar.sync 3, %0;" ::"n"(NEPI + 32) : "memory");
    };
    // let the next kernel start its prologue; then wait for the previous
    // kernel, whose outputs (input vectors, skip flag, output selection) all
    // reads below depend on
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    asm volatile("griddepcontrol.wait;" ::: "memory");
    const bool skipped = g.skip != nullptr && *g.skip;
    const int nlocal = (!skipped && grp < ntiles) ? (ntiles - 1 - grp) / ngrp + 1 : 0;

    float* outp = g.out;
    if (g.out_table != nullptr && !skipped) outp = (float*)((char*)g.out_table[*g.out_sel]);

    if (warp < NPW) {
        // ================= producers
        const int t = tid;
        const uint32_t stg0 = smem_u32(stg);
        // raw tile of local index i into staging buffer i&1; one commit group
        // per call (possibly empty) keeps the group accounting uniform
        // input bases of the vectors of local tile i (into ibase[i & 1]);
        // written by threads 0..TV-1 ahead of a producer barrier
        auto bases = [&](int i) {
            if (t < TV) {
                const long long v = (long long)(grp + (long long)i * ngrp) * TV + t;
                ibase[(i & 1) * TV + t] = (i < nlocal && v < g.nvec) ? vaddr(g.ia, v) : -1;
            }
        };
        // 8-byte copies when every axis-0 row starts on an 8-byte boundary
        const bool pairs8 = AX == 0 && g.ia.estride == 1 && ((uintptr_t)g.in & 7) == 0 &&
                            (g.ia.off & 1) == 0 && (g.ia.bstride & 1) == 0 && (g.ia.vstride & 1) == 0;
        constexpr int SP = WIDE ? STG_PITCH_W : STG_PITCH;   // axis-0 staging pitch
        auto stg_buf = [&](int i) { return WIDE ? 0 : (i & 1); };
        auto prefetch = [&](int i) {
            if (i < nlocal) {
                const uint32_t dst = stg0 + (uint32_t)(stg_buf(i) * STG_FLOATS * 4);
                const long long* ib = ibase + (i & 1) * TV;
                if constexpr (AX == 0) {
                    // warp w: rows (TV/NPW) w ..., lanes along the row
#pragma unroll
                    for (int rr = 0; rr < TV / NPW; ++rr) {
                        const int r = (TV / NPW) * warp + rr;
                        const long long base = ib[r];
                        if (base < 0) continue;
                        const float* src = g.in + base;
                        const uint32_t drow = dst + (uint32_t)(r * SP * 4);
                        if (pairs8) {
                            for (int m2 = lane; 2 * m2 < N; m2 += 32) cp_async4<8>(drow + 8u * m2, src + 2 * m2);
                        } else {
                            for (int m = lane; m < N; m += 32)
                                cp_async4<4>(drow + 4u * m, src + (long long)m * g.ia.estride);
                        }
                    }
                } else {
                    // lanes 0-15: vectors, lanes 16-31: the next element row
                    const int vl = lane & 15;
                    const long long base = ib[vl];
                    if (base >= 0) {
                        const int m0 = 2 * warp + (lane >> 4);
                        const float* src = g.in + base + (long long)m0 * g.ia.estride;
                        const long long step = 2 * NPW * g.ia.estride;
                        uint32_t d = dst + (uint32_t)((m0 * TV + vl) * 4);
                        for (int m = m0; m < N; m += 2 * NPW, src += step, d += 2 * NPW * TV * 4)
                            cp_async4<4>(d, src);
                    }
                }
            }
            cp_commit();
        };
        bases(0);
        if (!WIDE) bases(1);
        producer_sync();
        prefetch(0);
        if (!WIDE) prefetch(1);
        const int vl = t & 15, kq = t >> 4;
        for (int i = 0; i < nlocal && !failed; ++i) {
            const int b = i % NB, u = i / NB;
            const long long v0 = (long long)(grp + (long long)i * ngrp) * TV;
            const bool ok_free = u < 1 || mbar_wait(afree0 + 8 * b, (u - 1) & 1);
            if (role_any<1>(!ok_free)) { failed = true; break; }
            if (WIDE) cp_wait0();   // the group of tile i has landed (one staging buffer)
            else cp_wait1();        // the group of tile i has landed (tile i+1 may be in flight)
            producer_sync();
            const float* raw = stg + stg_buf(i) * STG_FLOATS;
            const bool okv = v0 + vl < g.nvec;
            auto X = [&](int m) -> float {
                if constexpr (AX == 0) return raw[vl * SP + m];
                else return raw[m * TV + vl];
            };
            // normal: pair sums sv / differences dv of vector vl, pairs 8 kq .. 8 kq + 7;
            // wide: the values of half hh (sums or differences), pairs 16 kq .. 16 kq + 15
            // in sv (first 8) and dv (last 8)
            float sv[8], dv[8];
            float psum_s = 0.f, psum_d = 0.f, lmax = 0.f;
            if constexpr (!WIDE) {
#pragma unroll
                for (int tt = 0; tt < 8; ++tt) {
                    const int k = 8 * kq + tt;  // pair index, m = k + 1 (DCT)
                    float a = 0.f, c = 0.f;
                    if (okv && k < P) {
                        a = X(dct ? k + 1 : k);
                        c = X(dct ? N - 2 - k : N - 1 - k);
                    }
                    const float s = a + c, d = a - c;
                    sv[tt] = s;
                    dv[tt] = d;
                    psum_s += s;
                    psum_d += ((k + 1) & 1) ? -d : d;   // (-1)^m d_m, m = k + 1
                    lmax = fmaxf(lmax, fmaxf(fabsf(s), fabsf(d)));
                }
            } else {
#pragma unroll
                for (int tt = 0; tt < 16; ++tt) {
                    const int k = 16 * kq + tt;
                    float a = 0.f, c = 0.f;
                    if (okv && k < P) {
                        a = X(dct ? k + 1 : k);
                        c = X(dct ? N - 2 - k : N - 1 - k);
                    }
                    const float w = hh == 0 ? a + c : a - c;
                    if (tt < 8) sv[tt] = w;
                    else dv[tt - 8] = w;
                    psum_s += (hh == 0 || !((k + 1) & 1)) ? w : -w;   // sum s_m, or sum (-1)^m d_m
                    lmax = fmaxf(lmax, fabsf(w));
                }
            }
            // lanes l and l ^ 16 hold the same vector (pair groups kq, kq ^ 1)
            psum_s += __shfl_xor_sync(0xffffffffu, psum_s, 16);
            psum_d += __shfl_xor_sync(0xffffffffu, psum_d, 16);
            lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, 16));
            if (lane < 16) {
                part[(warp * TV + vl) * 2 + 0] = psum_s;
                part[(warp * TV + vl) * 2 + 1] = psum_d;
                vmax[warp * TV + vl] = lmax;
            }
            if (dct && kq == 0) {
                const float x0 = okv ? X(0) : 0.f, xn = okv ? X(N - 1) : 0.f;
                // wide: e0 holds the end term of this role's half
                e0[b * TV + vl] = (WIDE && hh == 1) ? x0 - xn : x0 + xn;
                e1[b * TV + vl] = x0 - xn;
            }
            // warp 0: lanes 0..TV-1 the input bases of the tile prefetched next,
            // lanes TV..2TV-1 the output bases of this tile, one address each
            if (t < 2 * TV) {
                const bool in = t < TV;
                const int c = t & (TV - 1);
                const int inext = i + (WIDE ? 1 : 2);
                const Addr& ad = in ? g.ia : g.oa;
                const long long v = in ? (long long)(grp + (long long)inext * ngrp) * TV + c : v0 + c;
                const bool valid = v < g.nvec && (!in || inext < nlocal);
                const long long base = valid ? vaddr(ad, v) : -1;
                if (in) ibase[(inext & 1) * TV + c] = base;
                else obase[b * TV + c] = base;
            }
            producer_sync();     // raw buffer consumed, partials and bases of the next prefetch ready
            // every thread forms the scale of its own vector from the 8 warp
            // partials (threads 0..TV-1 also publish it for the epilogue)
            int ex = 0;
            {
                float m = 0.f, ss = 0.f, sd = 0.f;
#pragma unroll
                for (int q = 0; q < NPW; ++q) {
                    m = fmaxf(m, vmax[q * TV + vl]);
                    ss += part[(q * TV + vl) * 2 + 0];
                    sd += part[(q * TV + vl) * 2 + 1];
                }
                if (m > 0.f) {
                    int e2;
                    frexpf(m, &e2);
                    ex = 14 - e2;   // scaled maximum in [2^13, 2^14)
                    // decayed modes hold subnormal maxima: keep 2^ex finite
                    ex = ex > 100 ? 100 : (ex < -100 ? -100 : ex);
                }
                if (t < TV) {
                    const int vv = b * TV + t;   // t == vl here
                    vexp[vv] = ex;
                    vdown[vv] = ldexpf(g.norm, -ex);
                    if (dct) {
                        // wide: sp0 is X_0 (half 0) or X_{N-1} (half 1) of this role
                        sp0[vv] = (e0[vv] + 2.f * ss) * g.norm;
                        sp1[vv] = (e1[vv] + 2.f * sd) * g.norm;
                        e0[vv] *= g.norm;
                        e1[vv] *= g.norm;
                    }
                }
            }
            const float up = ldexpf(1.f, ex);
            unsigned char* db = sdat + b * 4 * DAT_BYTES;
            if constexpr (!WIDE) {
                uint32_t hs[4], ls[4], hd[4], ld[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    split_h2(sv[2 * q] * up, sv[2 * q + 1] * up, hs[q], ls[q]);
                    split_h2(dv[2 * q] * up, dv[2 * q + 1] * up, hd[q], ld[q]);
                }
                const uint32_t o = dat_off(0, vl, 8 * kq);
                *(uint4*)(db + 0 * DAT_BYTES + o) = make_uint4(hs[0], hs[1], hs[2], hs[3]);
                *(uint4*)(db + 1 * DAT_BYTES + o) = make_uint4(ls[0], ls[1], ls[2], ls[3]);
                *(uint4*)(db + 2 * DAT_BYTES + o) = make_uint4(hd[0], hd[1], hd[2], hd[3]);
                *(uint4*)(db + 3 * DAT_BYTES + o) = make_uint4(ld[0], ld[1], ld[2], ld[3]);
            } else {
                // K-major, 256 pairs: [hi 8 KB | lo 8 KB]; pairs 16 kq .. +7 from sv, +8 .. +15 from dv
                uint32_t h0[4], l0[4], h1[4], l1[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    split_h2(sv[2 * q] * up, sv[2 * q + 1] * up, h0[q], l0[q]);
                    split_h2(dv[2 * q] * up, dv[2 * q + 1] * up, h1[q], l1[q]);
                }
                const uint32_t o0 = dat_off_w(vl, 16 * kq), o1 = dat_off_w(vl, 16 * kq + 8);
                *(uint4*)(db + o0) = make_uint4(h0[0], h0[1], h0[2], h0[3]);
                *(uint4*)(db + 2 * DAT_BYTES + o0) = make_uint4(l0[0], l0[1], l0[2], l0[3]);
                *(uint4*)(db + o1) = make_uint4(h1[0], h1[1], h1[2], h1[3]);
                *(uint4*)(db + 2 * DAT_BYTES + o1) = make_uint4(l1[0], l1[1], l1[2], l1[3]);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_arrive(full0 + 8 * b);
            // the next raw tile into the buffer this one left (off the path to
            // the MMA: it lands two tiles ahead of its use)
            prefetch(i + (WIDE ? 1 : 2));
        }
        cp_wait0();
    } else if (warp == NPW + NEW) {
        // ================= MMA issuer (both axes: K-major data operands)
        load_matrices();
        const uint32_t mat0 = smem_u32(smat), dat0 = smem_u32(sdat);
        const uint32_t idesc = (1u << 4) | ((uint32_t)(TV >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
        int issued[NB] = {0, 0, 0};
        for (int i = 0; i < nlocal && !failed; ++i) {
            const int b = i % NB, u = i / NB;
            bool ok = mbar_wait(full0 + 8 * b, u & 1);
            ok = ok && (u < 1 || mbar_wait(afree0 + 8 * b, (u - 1) & 1));
            if (!__all_sync(0xffffffffu, ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if (lane == 0) {
                if constexpr (!WIDE) {
                    // descriptors of K-step ks are those of step 0 plus 256 ks bytes in the
                    // address field (address >> 4: + 16 ks; shared memory stays below 256 KB,
                    // so the 14-bit field never carries), so the issuing thread only adds
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        // hi x hi in chunks of KC_STEPS K-steps (columns (h (NCH_N + 1) + chunk) TV),
                        // the correction products after them
                        const uint32_t accb = tbase + (uint32_t)(b * ACC_COLS + h * (NCH_N + 1) * TV);
                        const uint32_t acc2 = accb + NCH_N * TV;
                        const uint32_t mh = mat0 + (uint32_t)(2 * h) * MAT_BYTES, ml = mh + MAT_BYTES;
                        const uint32_t dh = dat0 + (uint32_t)(b * 4 + 2 * h) * DAT_BYTES, dl = dh + DAT_BYTES;
                        const uint64_t a_hi0 = sdesc(mh, 128u, 2048u), a_lo0 = sdesc(ml, 128u, 2048u);
                        const uint64_t b_hi0 = sdesc(dh, 128u, 2048u), b_lo0 = sdesc(dl, 128u, 2048u);
#pragma unroll
                        for (int ks = 0; ks < PP / 16; ++ks) {
                            const uint64_t o = (uint64_t)(16 * ks);
                            mma_f16(accb + (uint32_t)((ks / KC_STEPS) * TV), a_hi0 + o, b_hi0 + o, idesc,
                                    (ks % KC_STEPS) > 0 ? 1u : 0u);
                            mma_f16(acc2, a_hi0 + o, b_lo0 + o, idesc, ks > 0 ? 1u : 0u);
                            mma_f16(acc2, a_lo0 + o, b_hi0 + o, idesc, 1u);
                        }
                    }
                } else {
                    // this role's 128 x 256 slice [hi 64 KB | lo 64 KB] against 256 pairs;
                    // hi x hi in one accumulator, the two correction products in a second
                    const uint32_t accb = tbase + (uint32_t)(b * ACC_COLS), acc2 = accb + NCH_W * TV;
                    const uint32_t mh = mat0, ml = mat0 + 2 * MAT_BYTES;
                    const uint32_t dh = dat0 + (uint32_t)(b * 4) * DAT_BYTES, dl = dh + 2 * DAT_BYTES;
                    const uint64_t a_hi0 = sdesc(mh, 128u, 4096u), a_lo0 = sdesc(ml, 128u, 4096u);
                    const uint64_t b_hi0 = sdesc(dh, 128u, 4096u), b_lo0 = sdesc(dl, 128u, 4096u);
#pragma unroll
                    for (int ks = 0; ks < PW_K / 16; ++ks) {
                        const uint64_t o = (uint64_t)(16 * ks);
                        mma_f16(accb + (uint32_t)((ks / KC_STEPS) * TV), a_hi0 + o, b_hi0 + o, idesc,
                                (ks % KC_STEPS) > 0 ? 1u : 0u);
                        mma_f16(acc2, a_hi0 + o, b_lo0 + o, idesc, ks > 0 ? 1u : 0u);
                        mma_f16(acc2, a_lo0 + o, b_hi0 + o, idesc, 1u);
                    }
                }
                mma_commit(mmad0 + 8 * b);
            }
            __syncwarp();
            issued[b]++;
        }
        // outstanding MMAs must finish before the accumulator columns are released
        for (int b = 0; b < NB; ++b)
            if (issued[b] > 0) mbar_wait(mmad0 + 8 * b, (issued[b] - 1) & 1);
    } else {
        // ================= epilogue (warps NPW .. NPW+7): warp e reads TMEM
        // lanes 32*(e%4) (modes) and columns 8*(e/4) .. +8 (vectors) of each half.
        // Outputs go through the just-consumed operand buffer of the tile so
        // that global stores are row-contiguous: axis 0 stages S[c][k - koff]
        // (vector rows), axis 1 stages S[k - koff][c ^ ((k - koff)/2 % 16)]
        // (output rows across the tile's 16 vector columns).
        load_matrices();
        const int e = warp - NPW, q = e & 3, ch = e >> 2;
        const int j = 32 * q + lane;  // mode index within a half
        const uint32_t lanebits = (uint32_t)(32 * q) << 16;
        const int koff = dct ? 1 : 0, nk = 2 * P;
        for (int i = 0; i < nlocal && !failed; ++i) {
            const int b = i % NB, u = i / NB;
            const bool ok = mbar_wait(full0 + 8 * b, u & 1) && mbar_wait(mmad0 + 8 * b, u & 1);
            if (role_any<2>(!ok)) { failed = true; break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            if constexpr (!WIDE) {
                // each half: the sum of its chunk accumulators, then its corrections
                float va[8], vb[8];
                const uint32_t tb0 = tbase + lanebits + (uint32_t)(b * ACC_COLS + 8 * ch);
                acc_sum<NCH_N>(tb0, va);
                acc_sum<NCH_N>(tb0 + (NCH_N + 1) * TV, vb);
                float* S = (float*)(sdat + b * 4 * DAT_BYTES);
                if (j < P) {
                    const int ia = (dct ? 2 * j + 2 : 2 * j) - koff, ib = 2 * j + 1 - koff;
    #pragma unroll
                    for (int cc = 0; cc < 8; ++cc) {
                        const int c = 8 * ch + cc;
                        const float down = vdown[b * TV + c];
                        float av = va[cc] * down, bv = vb[cc] * down;
                        if (dct) { av += e0[b * TV + c]; bv += e1[b * TV + c]; }
                        if constexpr (AX == 0) {
                            S[c * (2 * PP) + ia] = av;
                            S[c * (2 * PP) + ib] = bv;
                        } else {
                            S[ia * TV + (c ^ ((ia >> 1) & 15))] = av;
                            S[ib * TV + (c ^ ((ib >> 1) & 15))] = bv;
                        }
                    }
                }
                epilogue_sync();
                if constexpr (AX == 0) {
                    for (int c = e; c < TV; c += NEW) {
                        const long long ob = obase[b * TV + c];
                        if (ob < 0) continue;
                        const float* sr = S + c * (2 * PP);
                        float* op = outp + ob + (long long)(lane + koff) * g.oa.estride;
                        const long long ostep = 32 * g.oa.estride;
                        for (int k = lane; k < nk; k += 32, op += ostep) *op = sr[k];
                    }
                } else {
                    const int c = lane & 15;
                    const long long ob = obase[b * TV + c];
                    if (ob >= 0) {
                        const int k0 = 2 * e + (lane >> 4);
                        float* op = outp + ob + (long long)(k0 + koff) * g.oa.estride;
                        const long long ostep = 2 * NEW * g.oa.estride;
                        for (int k = k0; k < nk; k += 2 * NEW, op += ostep) *op = S[k * TV + (c ^ ((k >> 1) & 15))];
                    }
                }
                if (dct && e == 0 && lane < TV) {
                    const long long ob = obase[b * TV + lane];
                    if (ob >= 0) {
                        outp[ob] = sp0[b * TV + lane];
                        outp[ob + (long long)(N - 1) * g.oa.estride] = sp1[b * TV + lane];
                    }
                }
            } else {
                // one accumulator: modes 128 mb + j of half hh, output element 2 (128 mb + j) + par
                float va[8];
                acc_sum<NCH_W>(tbase + lanebits + (uint32_t)(b * ACC_COLS + 8 * ch), va);
                float* S = (float*)(sdat + b * 4 * DAT_BYTES);
                const int par = dct ? (hh == 0 ? 1 : 0) : (hh == 0 ? 0 : 1);
                const int jg = 128 * mb + j;
#pragma unroll
                for (int cc = 0; cc < 8; ++cc) {
                    const int c = 8 * ch + cc;
                    float av = va[cc] * vdown[b * TV + c];
                    if (dct) av += e0[b * TV + c];
                    if constexpr (AX == 0) S[c * 128 + j] = av;
                    else S[j * TV + (c ^ ((j >> 1) & 15))] = av;
                }
                epilogue_sync();
                if constexpr (AX == 0) {
                    for (int c = e; c < TV; c += NEW) {
                        const long long ob = obase[b * TV + c];
                        if (ob < 0) continue;
                        const float* sr = S + c * 128;
                        for (int jl = lane; jl < 128; jl += 32) {
                            const int jj2 = 128 * mb + jl;
                            if (jj2 < P) outp[ob + (long long)(2 * jj2 + par + koff) * g.oa.estride] = sr[jl];
                        }
                    }
                } else {
                    const int c = lane & 15;
                    const long long ob = obase[b * TV + c];
                    if (ob >= 0) {
                        for (int jl = 2 * e + (lane >> 4); jl < 128; jl += 2 * NEW) {
                            const int jj2 = 128 * mb + jl;
                            if (jj2 < P)
                                outp[ob + (long long)(2 * jj2 + par + koff) * g.oa.estride] =
                                    S[jl * TV + (c ^ ((jl >> 1) & 15))];
                        }
                    }
                }
                // X_0 (half 0) or X_{N-1} (half 1), written by the first mode block
                if (dct && mb == 0 && e == 0 && lane < TV) {
                    const long long ob = obase[b * TV + lane];
                    if (ob >= 0) outp[ob + (hh == 0 ? 0LL : (long long)(N - 1) * g.oa.estride)] = sp0[b * TV + lane];
                }
                (void)jg;
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            mbar_arrive(afree0 + 8 * b);
        }
    }
    if (failed && g.err != nullptr) atomicExch(g.err, 1);
    __syncthreads();
    if (warp == NPW + NEW) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "n"(TMEM_COLS));
    }
}

}  // namespace tc
