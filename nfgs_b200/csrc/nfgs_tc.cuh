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
// relative error per product against the vector's maximum.
//
// One persistent CTA per SM: the four matrix operands (two halves, hi and
// lo; 128 KB) stay resident in shared memory; the 64-vector data tile
// (64 KB) is rebuilt per tile by all threads; one thread issues the MMAs;
// completion is signalled through an mbarrier with bounded waits.
#pragma once
#include <cuda_fp16.h>
#include "nfgs_common.cuh"

namespace tc {

constexpr int PP = 128;          // padded pair count (K) and modes per half (M)
constexpr int TV = 64;           // vectors per tile (N of the MMA)
constexpr int NTHREADS = 256;
constexpr int MAT_BYTES = PP * PP * 2;        // one fp16 matrix operand: 32 KB
constexpr int DAT_BYTES = PP * TV * 2;        // one fp16 data operand: 16 KB
constexpr int SMEM_MAT = 4 * MAT_BYTES;       // 128 KB
constexpr int SMEM_DAT = 4 * DAT_BYTES;       // 64 KB
constexpr int SMEM_AUX = 8 * 1024;            // per-vector scalars, partial sums, barrier
constexpr int SMEM_TOTAL = SMEM_MAT + SMEM_DAT + SMEM_AUX;
constexpr long long WAIT_LIMIT = 1LL << 26;   // mbarrier polls before giving up

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
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
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

__device__ __forceinline__ long long vaddr(const Addr& a, long long v) {
    return a.off + (v / a.vpb) * a.bstride + (v % a.vpb) * a.vstride;
}

// byte offset of (vec, pair) in a data operand
//   axis 0 (K-major):  (v/8)*2048 + (k/8)*128 + (v%8)*16 + (k%8)*2
//   axis 1 (MN-major): (k/8)*1024 + (v/8)*128 + (k%8)*16 + (v%8)*2
__device__ __forceinline__ uint32_t dat_off(int axis, int v, int k) {
    return axis == 0 ? (uint32_t)((v >> 3) * 2048 + (k >> 3) * 128 + (v & 7) * 16 + (k & 7) * 2)
                     : (uint32_t)((k >> 3) * 1024 + (v >> 3) * 128 + (k & 7) * 16 + (v & 7) * 2);
}

__device__ __forceinline__ void split_h(float x, __half& hi, __half& lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
}

__global__ void __launch_bounds__(NTHREADS, 1) k_tc_transform(Args g) {
    extern __shared__ __align__(1024) unsigned char smem[];
    if (g.skip != nullptr && *g.skip) return;
    unsigned char* smat = smem;
    unsigned char* sdat = smem + SMEM_MAT;
    float* aux = (float*)(smem + SMEM_MAT + SMEM_DAT);
    // aux layout (floats): e0[64] e1[64] sp0[64] sp1[64] part[4][64][2] red[16]
    float* e0 = aux;
    float* e1 = aux + 64;
    float* sp0 = aux + 128;
    float* sp1 = aux + 192;
    float* part = aux + 256;          // [4][64][2]
    float* red = aux + 256 + 512;     // [16]
    uint64_t* mbar = (uint64_t*)(aux + 256 + 512 + 16);
    uint32_t* tslot = (uint32_t*)(aux + 256 + 512 + 16 + 4);
    long long* ibase = (long long*)(aux + 256 + 512 + 16 + 8);   // [64] input base of each tile vector
    long long* obase = ibase + TV;                               // [64] output base
    int* vexp = (int*)(obase + TV);                              // [64] per-vector scale exponent
    float* vmax = (float*)(vexp + TV);                           // [4][64] partial maxima (axis 0)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int ntiles = (g.nvec + TV - 1) / TV;
    // resident matrices
    {
        uint4* d = (uint4*)smat;
        for (int q = tid; q < SMEM_MAT / 16; q += NTHREADS) d[q] = g.mat[q];
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 128;" ::"r"(smem_u32(tslot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tbase = *tslot;
    const uint32_t mb = smem_u32(mbar);
    const uint32_t mat0 = smem_u32(smat), dat0 = smem_u32(sdat);
    const uint32_t idesc = (1u << 4) | ((uint32_t)g.axis << 16) | ((uint32_t)(TV >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
    const int P = g.P, N = g.N;
    const bool dct = g.kind == 0;
    bool failed = false;
    uint32_t phase = 0;

    float* outp = g.out;
    if (g.out_table != nullptr) outp = (float*)((char*)g.out_table[*g.out_sel]);

    for (int tile = blockIdx.x; tile < ntiles && !failed; tile += gridDim.x) {
        const long long v0 = (long long)tile * TV;
        if (tid < TV) {
            const long long v = v0 + tid;
            ibase[tid] = v < g.nvec ? vaddr(g.ia, v) : 0;
            obase[tid] = v < g.nvec ? vaddr(g.oa, v) : -1;
        }
        __syncthreads();
        // ---------------- build the data operands
        float sv[32], dv[32];
        int myv;            // the tile vector this thread works on
        float psum_s = 0.f, psum_d = 0.f;
        float lmax = 0.f;
        if (g.axis == 0) {
            // units (row r, k-group kg): r fixed per thread, kg = tid/64 + 4 i
            myv = (tid & 7) + 8 * ((tid >> 3) & 7);
            const long long v = v0 + myv;
            const bool ok = v < g.nvec;
            const long long base = ibase[myv];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int kg = (tid >> 6) + 4 * i;
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int k = 8 * kg + t;  // pair index, m = k + 1
                    float a = 0.f, b = 0.f;
                    if (ok && k < P) {
                        const int ia = dct ? k + 1 : k;             // element index of x_m
                        const int ib = dct ? N - 2 - k : N - 1 - k; // element index of the partner
                        a = g.in[base + (long long)ia * g.ia.estride];
                        b = g.in[base + (long long)ib * g.ia.estride];
                    }
                    const float s = a + b, d = a - b;
                    sv[8 * i + t] = s;
                    dv[8 * i + t] = d;
                    psum_s += s;
                    psum_d += ((k + 1) & 1) ? -d : d;   // (-1)^m d_m, m = k + 1
                    lmax = fmaxf(lmax, fmaxf(fabsf(s), fabsf(d)));
                }
            }
            part[((tid >> 6) * 64 + myv) * 2 + 0] = psum_s;
            part[((tid >> 6) * 64 + myv) * 2 + 1] = psum_d;
            if (dct && (tid >> 6) == 0) {
                float x0 = 0.f, xn = 0.f;
                if (ok) {
                    x0 = g.in[base];
                    xn = g.in[base + (long long)(N - 1) * g.ia.estride];
                }
                e0[myv] = x0 + xn;
                e1[myv] = x0 - xn;
            }
        } else {
            // elements (vec, pair): vec = 8*warp + lane%8, pair = 4 i + lane/8
            myv = 8 * warp + (lane & 7);
            const long long v = v0 + myv;
            const bool ok = v < g.nvec;
            const long long base = ibase[myv];
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int k = 4 * i + (lane >> 3);
                float a = 0.f, b = 0.f;
                if (ok && k < P) {
                    const int ia = dct ? k + 1 : k;
                    const int ib = dct ? N - 2 - k : N - 1 - k;
                    a = g.in[base + (long long)ia * g.ia.estride];
                    b = g.in[base + (long long)ib * g.ia.estride];
                }
                const float s = a + b, d = a - b;
                sv[i] = s;
                dv[i] = d;
                psum_s += s;
                psum_d += ((k + 1) & 1) ? -d : d;
                lmax = fmaxf(lmax, fmaxf(fabsf(s), fabsf(d)));
            }
            // combine the four lanes that share a vector (lane%8 equal)
            psum_s += __shfl_xor_sync(0xffffffffu, psum_s, 8);
            psum_s += __shfl_xor_sync(0xffffffffu, psum_s, 16);
            psum_d += __shfl_xor_sync(0xffffffffu, psum_d, 8);
            psum_d += __shfl_xor_sync(0xffffffffu, psum_d, 16);
            if (lane < 8) {
                part[myv * 2 + 0] = psum_s;
                part[myv * 2 + 1] = psum_d;
                if (dct) {
                    float x0 = 0.f, xn = 0.f;
                    if (ok) {
                        x0 = g.in[base];
                        xn = g.in[base + (long long)(N - 1) * g.ia.estride];
                    }
                    e0[myv] = x0 + xn;
                    e1[myv] = x0 - xn;
                }
            }
        }
        // per-vector maximum -> power-of-two scale of each vector
        int myex = 0;
        if (g.axis == 0) {
            vmax[(tid >> 6) * 64 + myv] = lmax;
            __syncthreads();
            if (tid < TV) {
                float m = fmaxf(fmaxf(vmax[tid], vmax[64 + tid]), fmaxf(vmax[128 + tid], vmax[192 + tid]));
                int ex = 0;
                if (m > 0.f) {
                    int e2;
                    frexpf(m, &e2);
                    ex = 14 - e2;   // scaled maximum in [2^13, 2^14)
                    // decayed modes hold subnormal maxima: keep 2^ex finite
                    ex = ex > 100 ? 100 : (ex < -100 ? -100 : ex);
                }
                vexp[tid] = ex;
            }
            __syncthreads();
            myex = vexp[myv];
        } else {
            lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, 8));
            lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, 16));
            if (lmax > 0.f) {
                int e2;
                frexpf(lmax, &e2);
                myex = 14 - e2;
                myex = myex > 100 ? 100 : (myex < -100 ? -100 : myex);
            }
            if (lane < 8) vexp[myv] = myex;
        }
        const float up = ldexpf(1.f, myex);
        // convert and store
        if (g.axis == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int kg = (tid >> 6) + 4 * i;
                uint32_t hs[4], ls[4], hd[4], ld[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    __half a0, a1, b0, b1;
                    split_h(sv[8 * i + 2 * t] * up, a0, b0);
                    split_h(sv[8 * i + 2 * t + 1] * up, a1, b1);
                    hs[t] = (uint32_t)__half_as_ushort(a0) | ((uint32_t)__half_as_ushort(a1) << 16);
                    ls[t] = (uint32_t)__half_as_ushort(b0) | ((uint32_t)__half_as_ushort(b1) << 16);
                    split_h(dv[8 * i + 2 * t] * up, a0, b0);
                    split_h(dv[8 * i + 2 * t + 1] * up, a1, b1);
                    hd[t] = (uint32_t)__half_as_ushort(a0) | ((uint32_t)__half_as_ushort(a1) << 16);
                    ld[t] = (uint32_t)__half_as_ushort(b0) | ((uint32_t)__half_as_ushort(b1) << 16);
                }
                const uint32_t o = dat_off(0, myv, 8 * kg);
                *(uint4*)(sdat + 0 * DAT_BYTES + o) = make_uint4(hs[0], hs[1], hs[2], hs[3]);
                *(uint4*)(sdat + 1 * DAT_BYTES + o) = make_uint4(ls[0], ls[1], ls[2], ls[3]);
                *(uint4*)(sdat + 2 * DAT_BYTES + o) = make_uint4(hd[0], hd[1], hd[2], hd[3]);
                *(uint4*)(sdat + 3 * DAT_BYTES + o) = make_uint4(ld[0], ld[1], ld[2], ld[3]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 32; ++i) {
                const int k = 4 * i + (lane >> 3);
                __half hs, ls, hd, ld;
                split_h(sv[i] * up, hs, ls);
                split_h(dv[i] * up, hd, ld);
                const uint32_t o = dat_off(1, myv, k);
                *(__half*)(sdat + 0 * DAT_BYTES + o) = hs;
                *(__half*)(sdat + 1 * DAT_BYTES + o) = ls;
                *(__half*)(sdat + 2 * DAT_BYTES + o) = hd;
                *(__half*)(sdat + 3 * DAT_BYTES + o) = ld;
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        // ---------------- MMAs: half A (pair sums), half B (pair differences)
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t dsbo = g.axis == 0 ? 2048u : 128u;
            const uint32_t dlbo = g.axis == 0 ? 128u : 1024u;
            const uint32_t dstep = g.axis == 0 ? 256u : 2048u;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const uint32_t acc = tbase + (uint32_t)(h * TV);
                const uint32_t mh = mat0 + (uint32_t)(2 * h) * MAT_BYTES, ml = mh + MAT_BYTES;
                const uint32_t dh = dat0 + (uint32_t)(2 * h) * DAT_BYTES, dl = dh + DAT_BYTES;
#pragma unroll 1
                for (int ks = 0; ks < PP / 16; ++ks) {
                    const uint64_t a_hi = sdesc(mh + 256u * ks, 128u, 2048u);
                    const uint64_t a_lo = sdesc(ml + 256u * ks, 128u, 2048u);
                    const uint64_t b_hi = sdesc(dh + dstep * ks, dlbo, dsbo);
                    const uint64_t b_lo = sdesc(dl + dstep * ks, dlbo, dsbo);
                    mma_f16(acc, a_hi, b_hi, idesc, ks > 0 ? 1u : 0u);
                    mma_f16(acc, a_hi, b_lo, idesc, 1u);
                    mma_f16(acc, a_lo, b_hi, idesc, 1u);
                }
            }
            mma_commit(mb);
        }
        // specials and endpoint terms (DCT), per vector, while the MMAs run
        if (dct && tid < TV) {
            float ss = 0.f, sd = 0.f;
            if (g.axis == 0) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    ss += part[(q * 64 + tid) * 2 + 0];
                    sd += part[(q * 64 + tid) * 2 + 1];
                }
            } else {
                ss = part[tid * 2 + 0];
                sd = part[tid * 2 + 1];
            }
            sp0[tid] = (e0[tid] + 2.f * ss) * g.norm;
            sp1[tid] = (e1[tid] + 2.f * sd) * g.norm;
            e0[tid] *= g.norm;
            e1[tid] *= g.norm;
        }
        __syncthreads();
        const bool ok = mbar_wait(mb, phase);
        failed = __syncthreads_or(!ok) != 0;
        if (failed && tid == 0 && g.err != nullptr) atomicExch(g.err, 1);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        // ---------------- epilogue: TMEM -> global
        if (!failed) {
            const int q = warp & 3, ch = warp >> 2;
            const int j = 32 * q + lane;  // mode index within the half
            float va[32], vb[32];
            const uint32_t lanebits = (uint32_t)(32 * q) << 16;
            tmem_ld32(tbase + lanebits + (uint32_t)(32 * ch), va);
            tmem_ld32(tbase + lanebits + (uint32_t)(TV + 32 * ch), vb);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");

            if (j < P) {
                // output element indices of the two halves
                const int ka = dct ? 2 * j + 2 : 2 * j;
                const int kb = dct ? 2 * j + 1 : 2 * j + 1;
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int tv = 32 * ch + c;
                    const long long ob = obase[tv];
                    if (ob < 0) continue;
                    const float down = ldexpf(g.norm, -vexp[tv]);
                    float a = va[c] * down, b = vb[c] * down;
                    if (dct) { a += e0[tv]; b += e1[tv]; }
                    outp[ob + (long long)ka * g.oa.estride] = a;
                    outp[ob + (long long)kb * g.oa.estride] = b;
                }
            }
            if (dct && tid < TV) {
                const long long ob = obase[tid];
                if (ob >= 0) {
                    outp[ob] = sp0[tid];
                    outp[ob + (long long)(N - 1) * g.oa.estride] = sp1[tid];
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    if (failed) {
        // a completion never arrived: give the outstanding MMAs one more
        // bounded wait before the accumulator columns are released
        mbar_wait(mb, phase ^ 1u);
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 128;" ::"r"(tbase));
}

}  // namespace tc
