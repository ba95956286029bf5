// NFGS B200 solver: handle, boundary set-up, iteration driver, C ABI.
//
// Reference: nfgs_solver.py (spaceprod/NFGS), class NFGSSolverGPU
// (nfgs_solver.py:3905-7196) and its bases.  Each exported entry point
// names the reference method it replaces in include/nfgs_b200.h.
#include "../../include/nfgs_b200.h"
#include "nfgs_common.cuh"
#include "nfgs_gemm.cuh"
#include "nfgs_iter.cuh"
#include "nfgs_setup.cuh"
#include "nfgs_tc.cuh"
#include "nfgs_stencil.cuh"
#include "nfgs_stencil2.cuh"
#include "nfgs_diag.cuh"
#include "nfgs_k0.cuh"
#include "nfgs_metrics.cuh"
#include "nfgs_soft.cuh"
#include "nfgs_trace.cuh"
#include "nfgs_fastqsl.cuh"
#include <cuda_fp16.h>

#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <sys/mman.h>
#include <string>
#include <condition_variable>
#include <thread>
#include <vector>

static thread_local std::string g_err;

static int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return fail(NFGS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));     \
    } while (0)

#define TRY(call)                     \
    do {                              \
        int r_ = (call);              \
        if (r_ != NFGS_OK) return r_; \
    } while (0)

namespace {

// ---------------------------------------------------------------------------
// Device buffer helper
// ---------------------------------------------------------------------------
struct Buf {
    void* p = nullptr;
    size_t bytes = 0;
};

struct Handle {
    NfgsGeom geom{};
    NfgsParams prm{};
    Geo g{};
    int f32 = 1;
    size_t esz = 4;
    cudaStream_t s = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // ordering of nfgs_gaussian_above_noalloc (caller's stream) against the
    // handle's stream: ev_na_in marks the handle's work it must follow,
    // ev_na_out the end of its last call (set_boundary and destroy wait on it)
    cudaEvent_t ev_na_in = nullptr, ev_na_out = nullptr;
    std::vector<Buf> owned;
    int launches = 0;

    long long PI = 0;  // interior modes (nx-2)(ny-2)

    // transform matrices, row-major [out][in]
    double *dctx = nullptr, *idctx = nullptr, *dcty = nullptr, *idcty = nullptr;
    double *dstx = nullptr, *idstx = nullptr, *dsty = nullptr, *idsty = nullptr;
    void *dctx_t = nullptr, *idctx_t = nullptr, *dcty_t = nullptr, *idcty_t = nullptr;
    void *dstx_t = nullptr, *idstx_t = nullptr, *dsty_t = nullptr, *idsty_t = nullptr;

    // spectral tables
    double *lamN = nullptr, *kN = nullptr, *lamNs = nullptr, *lamD = nullptr, *alx = nullptr, *aly = nullptr;
    // z factor tables
    double *zr_c = nullptr, *zr_i = nullptr, *zr_il = nullptr, *zr_ci = nullptr, *zr_ii = nullptr;
    int* zr_rc = nullptr;
    double *zd_c = nullptr, *zd_i = nullptr, *zd_il = nullptr, *zd_ci = nullptr, *zd_ii = nullptr;
    int* zd_rc = nullptr;

    // boundary products (FP64 planes)
    double *bz_obs = nullptr, *bx_obs = nullptr, *by_obs = nullptr, *jz_obs = nullptr, *az_bot = nullptr,
           *jz_t = nullptr, *phi_above = nullptr, *bz_above = nullptr, *d0 = nullptr, *dphi_tgt = nullptr;
    double *phi_above_hat = nullptr, *phi_below_hat = nullptr;  // modal (P)
    double *phi_bot_hat = nullptr, *der_hat = nullptr, *az_bot_hat = nullptr;
    // bottom current of the Stable-NFPT solver behind the cfcf start: always
    // the legacy helper-grid derivation; aliases jz_obs when that is the
    // current in use (jz_stable_alias)
    double* jz_stable = nullptr;
    int jz_stable_alias = 1;
    // the last single step's state indices and relaxation factor, for the
    // per-step diagnostics (record_iteration_diagnostics)
    int diag_prev = 0, diag_cand = 1, diag_valid = 0;
    int select_final = 0;      // stop_mode="fixed_point": the solution is the final state
    double diag_mu = 1.0;
    double *bbg_d = nullptr;  // 3V FP64 background (kept for diagnostics)
    // storage-type constants
    void *bbg = nullptr, *bzobs_t = nullptr, *jzt_t = nullptr, *phiab_t = nullptr, *dphi_t = nullptr;
    void* azb_t = nullptr;     // Az_bottom in the storage type (every candidate's A_z bottom plane)
    void *wx = nullptr, *wy = nullptr, *wz = nullptr;
    double hx = 0.0, hy = 0.0;
    int use_h = 0;
    // k_h=0 closure (coupled_k0 / constrained_spline_harmonic): per-buffer H(z)
    bool k0_on = false;
    int k0_spline = 0;
    k0::Dev k0d{};
    double* k0_hsel = nullptr;  // [2][nz] profile of the last reconstructed state
    double k0_t[2] = {0.0, 0.0};  // bottom target H(0)
    double k0_cond = 0.0;
    double open_bz = 0.0;
    int boundary_set = 0;
    int fov_y0 = 0, fov_x0 = 0, nyo = 0, nxo = 0, nzo = 0;
    Box box{};

    // state and work (storage type)
    StateTab st{};
    StateTab* st_dev = nullptr;
    void *B = nullptr, *jz = nullptr, *jpf = nullptr, *jb = nullptr, *sb = nullptr, *sj = nullptr,
         *tmpA = nullptr, *tmpB = nullptr;
    double *pface = nullptr, *psrc = nullptr, *s00 = nullptr, *scal = nullptr;
    int nb_face = 0, nb_src = 0;
    dim3 sgrid, sblock;
    // fused stencil plan (source-producing passes)
    bool fs_on = false;
    bool fs_v2 = false;        // warp-row stencil (fs2::k_stencil2) instead of fs::k_stencil
    int fs_cw = 1;             // its staging chunk: 2 FP32 elements (8 bytes) on even-width grids
    dim3 fs_grid;
    int fs_nb = 0;
    // partial-sum layout of the last stencil pass
    const double *sum_pf = nullptr, *sum_ps = nullptr;
    int sum_nbf = 0, sum_nbs = 0;

    // iteration control
    DevCtl* ctl = nullptr;
    DevCtl* ctl_h = nullptr;  // pinned mirror
    int* consts = nullptr;    // device ints: [0]=0 [1]=1 [2]=2
    double* hist = nullptr;
    int hist_rows = 0;
    int iter_active = 0;
    int solution = -1;  // state index holding the stored solution
    NfgsStop stop{};
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    double init_zr = 0.0;
    float total_ms = 0.0f;
    int graph_kernels = 0;
    int cur_host = 0;       // current state index outside iterate
    void* bscratch = nullptr;  // 3V storage-type scratch (final-vs-best)
    double* fvb_part = nullptr;  // block partials of the final-vs-best sums
    double* dscratch = nullptr; // V FP64 scratch for host transfers
    int nzo_crop = 0;
    // tensor-core transform plan (FP32 storage, even N with (N-2)/2 <= 128)
    bool tc_on = false;
    void* tc_img[4] = {nullptr, nullptr, nullptr, nullptr};  // dct_x, dct_y, dst_x, dst_y
    int tc_px = 0, tc_py = 0, tc_nsm = 0;
    bool tc_wide[4] = {false, false, false, false};  // 128 < P <= 256: four-role kernel
    int* tc_err = nullptr;
    std::vector<void*> setup_scratch;  // freed at the end of a boundary set-up
    // field export: persistent device gather buffer and two pinned chunks
    void* fbuf = nullptr;
    size_t fbuf_bytes = 0;
    double* dsmall = nullptr;  // small device scratch for host decisions
    int fs_tuned = 0;          // the fused-stencil segment count has been tuned
    long long pface_len = 0;   // doubles in pface
    int advanced = 0;          // the current iteration has taken a step
    int stale_start = 0;       // restart mode 3 left the candidate's sources in place of the start's
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};
};

// Device memory of every handle comes from one stream-ordered pool per
// device whose release threshold keeps freed memory reserved (as torch's
// caching allocator does), so creating and destroying solvers and the
// set-up's scratch buffers cost no cudaMalloc / cudaFree device
// synchronisation after first use; nfgs_release_cached_memory returns it.
static std::mutex g_pool_mu;
static std::map<int, cudaMemPool_t> g_pools;

static int device_pool(int dev, cudaMemPool_t* out) {
    std::lock_guard<std::mutex> lk(g_pool_mu);
    auto it = g_pools.find(dev);
    if (it != g_pools.end()) { *out = it->second; return NFGS_OK; }
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    CK(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_pools[dev] = pool;
    *out = pool;
    return NFGS_OK;
}

// Allocation on the handle's stream, complete on return (usable from any
// stream, including the synchronous copies of the set-up).
template <typename T>
static int alloc(Handle* h, T** p, size_t bytes) {
    void* q = nullptr;
    if (bytes == 0) bytes = 16;
    cudaMemPool_t pool;
    TRY(device_pool(h->geom.device, &pool));
    cudaError_t e = cudaMallocFromPoolAsync(&q, bytes, pool, h->s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->s);
    if (e != cudaSuccess) return fail(NFGS_ENOMEM, std::string("device allocation failed: ") + cudaGetErrorString(e));
    h->owned.push_back({q, bytes});
    *p = (T*)q;
    return NFGS_OK;
}

// Return one owned allocation to the pool (stream-ordered).
static void release(Handle* h, void* p) {
    for (auto it = h->owned.begin(); it != h->owned.end(); ++it)
        if (it->p == p) { cudaFreeAsync(it->p, h->s); h->owned.erase(it); return; }
}

// 32 MB pinned host chunks for device-to-host staging, shared by every
// handle of the process (pinning costs milliseconds per chunk).
constexpr size_t PIN_CHUNK = (size_t)32 << 20;
static std::mutex g_pin_mu;
static std::vector<void*> g_pin_free;

static int pin_acquire(void** p) {
    {
        std::lock_guard<std::mutex> lk(g_pin_mu);
        if (!g_pin_free.empty()) { *p = g_pin_free.back(); g_pin_free.pop_back(); return NFGS_OK; }
    }
    CK(cudaHostAlloc(p, PIN_CHUNK, cudaHostAllocDefault));
    return NFGS_OK;
}
static void pin_release(void* p) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(g_pin_mu);
    g_pin_free.push_back(p);
}

// Page-locked host mirrors of the control block, kept for the next solver
// (pinning and unpinning cost far more than the block's copy).
static std::mutex g_ctl_mu;
static std::vector<DevCtl*> g_ctl_free;
static int ctl_mirror_acquire(DevCtl** p) {
    {
        std::lock_guard<std::mutex> lk(g_ctl_mu);
        if (!g_ctl_free.empty()) { *p = g_ctl_free.back(); g_ctl_free.pop_back(); return NFGS_OK; }
    }
    CK(cudaMallocHost(p, sizeof(DevCtl)));
    return NFGS_OK;
}
static void ctl_mirror_release(DevCtl* p) {
    std::lock_guard<std::mutex> lk(g_ctl_mu);
    g_ctl_free.push_back(p);
}

static void free_all(Handle* h) {
    if (h->gexec) cudaGraphExecDestroy(h->gexec);
    if (h->graph) cudaGraphDestroy(h->graph);
    for (auto& b : h->owned) cudaFreeAsync(b.p, h->s);
    h->owned.clear();
    if (h->s) cudaStreamSynchronize(h->s);
    if (h->ctl_h) ctl_mirror_release(h->ctl_h);
    for (int q = 0; q < 2; ++q)
        if (h->pin_ev[q]) cudaEventDestroy(h->pin_ev[q]);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->ev_na_in) cudaEventDestroy(h->ev_na_in);
    if (h->ev_na_out) cudaEventDestroy(h->ev_na_out);
    if (h->s) cudaStreamDestroy(h->s);
}

// ---------------------------------------------------------------------------
// Transform helpers.  Matrices are row-major [out][in].
//   apply_x: out(r, c) = sum_m M[c][m] in(r, m)      (rows contiguous)
//   apply_y: out(b, r, c) = sum_m M[r][m] in(b, m, c) (per plane)
// ---------------------------------------------------------------------------
template <typename T>
static int apply_x(Handle* h, const void* M, const void* in, long long in_rs, long long in_bs, void* out,
                   long long out_rs, long long out_bs, int rows, int K, int N, int batch, void* const* ctab = nullptr,
                   const int* csel = nullptr, const DevCtl* ctl = nullptr) {
    GemmArgs a{};
    a.A = in; a.a_rs = in_rs; a.a_cs = 1; a.a_bs = in_bs;
    a.B = M; a.b_rs = 1; a.b_cs = K; a.b_bs = 0;
    a.C = out; a.c_rs = out_rs; a.c_cs = 1; a.c_bs = out_bs;
    a.M = rows; a.N = N; a.K = K; a.batch = batch;
    a.c_table = ctab; a.c_sel = csel; a.ctl = ctl;
    h->launches++;
    CK(launch_gemm<T>(a, h->s));
    return NFGS_OK;
}

template <typename T>
static int apply_y(Handle* h, const void* M, const void* in, long long in_rs, long long in_bs, void* out,
                   long long out_rs, long long out_bs, int K, int N, int cols, int batch,
                   const DevCtl* ctl = nullptr) {
    GemmArgs a{};
    a.A = M; a.a_rs = K; a.a_cs = 1; a.a_bs = 0;
    a.B = in; a.b_rs = in_rs; a.b_cs = 1; a.b_bs = in_bs;
    a.C = out; a.c_rs = out_rs; a.c_cs = 1; a.c_bs = out_bs;
    a.M = N; a.N = cols; a.K = K; a.batch = batch;
    a.ctl = ctl;
    h->launches++;
    CK(launch_gemm<T>(a, h->s));
    return NFGS_OK;
}

// 2-D FP64 transforms of one (ny, nx) map (batch planes of pitch P).
static int dct2_d(Handle* h, const double* in, double* out, double* tmp, int batch = 1) {
    const int nx = h->g.nx, ny = h->g.ny;
    const long long P = h->g.P;
    TRY(apply_x<double>(h, h->dctx, in, nx, P, tmp, nx, P, ny, nx, nx, batch));
    TRY(apply_y<double>(h, h->dcty, tmp, nx, P, out, nx, P, ny, ny, nx, batch));
    return NFGS_OK;
}

static int idct2_d(Handle* h, const double* in, double* out, double* tmp, int batch = 1) {
    const int nx = h->g.nx, ny = h->g.ny;
    const long long P = h->g.P;
    TRY(apply_x<double>(h, h->idctx, in, nx, P, tmp, nx, P, ny, nx, nx, batch));
    TRY(apply_y<double>(h, h->idcty, tmp, nx, P, out, nx, P, ny, ny, nx, batch));
    return NFGS_OK;
}

static std::vector<double> d2h(Handle* h, const double* p, size_t n) {
    std::vector<double> v(n);
    cudaMemcpyAsync(v.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost, h->s);
    cudaStreamSynchronize(h->s);
    return v;
}

// reductions of n FP64 values: sum, sum of squares, sum |x|, max |x|
static int reduce4(Handle* h, const double* a, long long n, double out[4]) {
    if (n > (1LL << 18)) {
        // volumes: 512 fixed chunks, then their fixed-order combination
        constexpr int NBP = 512;
        const long long chunk = (n + NBP - 1) / NBP;
        double* part = nullptr;
        CK(cudaMallocAsync((void**)&part, NBP * 4 * sizeof(double), h->s));
        k_reduce4_part<<<NBP, 256, 0, h->s>>>(a, n, chunk, part);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) {
            k_reduce4_final<<<1, 512, 0, h->s>>>(part, NBP, h->scal);
            e = cudaGetLastError();
        }
        cudaFreeAsync(part, h->s);
        CK(e);
        h->launches += 2;
    } else {
        k_reduce4<<<1, 1024, 0, h->s>>>(a, n, h->scal);
        h->launches++;
    }
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, h->scal, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    return NFGS_OK;
}

static double rms_of(Handle* h, const double* a, long long n, int* rc) {
    double r[4];
    *rc = reduce4(h, a, n, r);
    return std::sqrt(r[1] / (double)n);
}

// Copy FP64 -> storage type
static int to_storage(Handle* h, const double* src, void* dst, long long n) {
    if (h->f32) {
        float* d = (float*)dst;
        CK(launch_map(n, h->s, [=] __device__(long long i) { d[i] = (float)src[i]; }));
    } else {
        CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, h->s));
    }
    h->launches++;
    return NFGS_OK;
}

static int from_storage(Handle* h, const void* src, double* dst, long long n) {
    if (h->f32) {
        const float* s = (const float*)src;
        CK(launch_map(n, h->s, [=] __device__(long long i) { dst[i] = (double)s[i]; }));
    } else {
        CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToDevice, h->s));
    }
    h->launches++;
    return NFGS_OK;
}

// ---------------------------------------------------------------------------
// Host-built tables
// ---------------------------------------------------------------------------
static std::vector<double> dct_matrix_build(int n, bool inverse) {
    std::vector<double> m((size_t)n * n);
    const double s = inverse ? 1.0 / (2.0 * (n - 1)) : 1.0;
    for (int k = 0; k < n; ++k)
        for (int q = 0; q < n; ++q) {
            double w = (q == 0 || q == n - 1) ? 1.0 : 2.0;
            // exact reduction of k*q modulo 2(n-1) keeps the argument small
            long long a = ((long long)k * q) % (2LL * (n - 1));
            m[(size_t)k * n + q] = s * w * std::cos(M_PI * (double)a / (double)(n - 1));
        }
    return m;
}

static std::vector<double> dst_matrix_build(int n, bool inverse) {
    std::vector<double> m((size_t)n * n);
    const double s = inverse ? 1.0 / (2.0 * (n + 1)) : 1.0;
    for (int k = 0; k < n; ++k)
        for (int q = 0; q < n; ++q) {
            long long a = ((long long)(k + 1) * (q + 1)) % (2LL * (n + 1));
            m[(size_t)k * n + q] = s * 2.0 * std::sin(M_PI * (double)a / (double)(n + 1));
        }
    return m;
}

static int upload(Handle* h, double** dp, const std::vector<double>& v) {
    TRY(alloc(h, dp, v.size() * sizeof(double)));
    CK(cudaMemcpy(*dp, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    return NFGS_OK;
}

static int upload_t(Handle* h, void** dp, const std::vector<double>& v) {
    TRY(alloc(h, dp, v.size() * h->esz));
    if (h->f32) {
        std::vector<float> f(v.begin(), v.end());
        CK(cudaMemcpy(*dp, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
    } else {
        CK(cudaMemcpy(*dp, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
    }
    return NFGS_OK;
}


// ---------------------------------------------------------------------------
// Tensor-core transform plan
// ---------------------------------------------------------------------------
// Operand image of one transform: four fp16 matrices [half A hi | half A lo |
// half B hi | half B lo], each 128 modes x 128 pairs in the no-swizzle
// K-major UMMA layout (j/8)*2048 + (k/8)*128 + (j%8)*16 + (k%8)*2 bytes.
static std::vector<uint16_t> tc_image_build(int kind, int n, int P) {
    std::vector<uint16_t> img(4 * 128 * 128, 0);
    const int period = kind == 0 ? n - 1 : n + 1;  // DCT: N-1, DST: n+1
    for (int h = 0; h < 2; ++h)
        for (int j = 0; j < 128; ++j)
            for (int k = 0; k < 128; ++k) {
                double val = 0.0;
                if (j < P && k < P) {
                    const long long m = k + 1;
                    long long kk;
                    if (kind == 0) kk = (h == 0) ? 2 * j + 2 : 2 * j + 1;
                    else kk = (h == 0) ? 2 * j + 1 : 2 * j + 2;
                    const long long a = (kk * m) % (2LL * period);
                    val = kind == 0 ? 2.0 * std::cos(M_PI * (double)a / period)
                                    : 2.0 * std::sin(M_PI * (double)a / period);
                }
                __half hi = __float2half_rn((float)val);
                __half lo = __float2half_rn((float)(val - (double)__half2float(hi)));
                const size_t off = ((size_t)(j / 8) * 2048 + (size_t)(k / 8) * 128 + (j % 8) * 16 + (k % 8) * 2) / 2;
                img[(size_t)(2 * h) * 16384 + off] = *(uint16_t*)&hi;
                img[(size_t)(2 * h + 1) * 16384 + off] = *(uint16_t*)&lo;
            }
    return img;
}

// Wide image (128 < P <= 256): four roles r = 2 h + mb, each the 128 x 256
// slice (modes 128 mb .. +127 of half h, all pairs) in K-major core-matrix
// layout (8-row groups 4096 B apart), [hi 64 KB | lo 64 KB] per role.
static std::vector<uint16_t> tc_image_wide_build(int kind, int n, int P) {
    const size_t per = (size_t)128 * tc::PW_K;   // halves per hi (or lo) slice
    std::vector<uint16_t> img(4 * 2 * per, 0);
    const int period = kind == 0 ? n - 1 : n + 1;
    for (int r = 0; r < 4; ++r) {
        const int h = r >> 1, mb = r & 1;
        for (int jl = 0; jl < 128; ++jl)
            for (int k = 0; k < tc::PW_K; ++k) {
                const int j = 128 * mb + jl;
                double val = 0.0;
                if (j < P && k < P) {
                    const long long m = k + 1;
                    long long kk;
                    if (kind == 0) kk = (h == 0) ? 2 * j + 2 : 2 * j + 1;
                    else kk = (h == 0) ? 2 * j + 1 : 2 * j + 2;
                    const long long a = (kk * m) % (2LL * period);
                    val = kind == 0 ? 2.0 * std::cos(M_PI * (double)a / period)
                                    : 2.0 * std::sin(M_PI * (double)a / period);
                }
                __half hi = __float2half_rn((float)val);
                __half lo = __float2half_rn((float)(val - (double)__half2float(hi)));
                const size_t off = ((size_t)(jl / 8) * 4096 + (size_t)(k / 8) * 128 + (jl % 8) * 16 + (k % 8) * 2) / 2;
                img[(size_t)r * 2 * per + off] = *(uint16_t*)&hi;
                img[(size_t)r * 2 * per + per + off] = *(uint16_t*)&lo;
            }
    }
    return img;
}

// The transform matrices depend only on their length and kind: they are
// built once per process (a solver created after the first of its size
// skips the cosine tables) and copied out of this cache.
static std::mutex g_mat_mu;
static std::map<std::tuple<int, int, int>, std::vector<double>> g_mat_cache;
static std::map<std::tuple<int, int, int, int>, std::vector<uint16_t>> g_img_cache;

static std::vector<double> dct_matrix(int n, bool inverse) {
    std::lock_guard<std::mutex> lk(g_mat_mu);
    auto& v = g_mat_cache[std::make_tuple(0, n, (int)inverse)];
    if (v.empty()) v = dct_matrix_build(n, inverse);
    return v;
}
static std::vector<double> dst_matrix(int n, bool inverse) {
    std::lock_guard<std::mutex> lk(g_mat_mu);
    auto& v = g_mat_cache[std::make_tuple(1, n, (int)inverse)];
    if (v.empty()) v = dst_matrix_build(n, inverse);
    return v;
}
// Device copies of the transform matrices, shared by every solver of the
// same size on a device (they are constant): keyed by (device, DCT/DST,
// length, inverse, element size).  They stay (a few MB per grid size), so
// creating a solver uploads nothing for a size seen before, until
// nfgs_release_cached_memory is called with no solver alive on the device.
static std::mutex g_dmat_mu;
static std::map<std::tuple<int, int, int, int, int>, void*> g_dmat_cache;
static std::map<int, int> g_live_handles;  // per device
static int shared_matrix(int device, int kind, int n, bool inverse, size_t esz, void** out) {
    std::lock_guard<std::mutex> lk(g_dmat_mu);
    void*& d = g_dmat_cache[std::make_tuple(device, kind, n, (int)inverse, (int)esz)];
    if (d == nullptr) {
        const std::vector<double> v = kind == 0 ? dct_matrix(n, inverse) : dst_matrix(n, inverse);
        void* q = nullptr;
        CK(cudaMalloc(&q, v.size() * esz));
        if (esz == 4) {
            std::vector<float> f(v.begin(), v.end());
            CK(cudaMemcpy(q, f.data(), f.size() * 4, cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy(q, v.data(), v.size() * 8, cudaMemcpyHostToDevice));
        }
        d = q;
    }
    *out = d;
    return NFGS_OK;
}

static std::vector<uint16_t> tc_image(int kind, int n, int P) {
    std::lock_guard<std::mutex> lk(g_mat_mu);
    auto& v = g_img_cache[std::make_tuple(0, kind, n, P)];
    if (v.empty()) v = tc_image_build(kind, n, P);
    return v;
}
static std::vector<uint16_t> tc_image_wide(int kind, int n, int P) {
    std::lock_guard<std::mutex> lk(g_mat_mu);
    auto& v = g_img_cache[std::make_tuple(1, kind, n, P)];
    if (v.empty()) v = tc_image_wide_build(kind, n, P);
    return v;
}

// Fused stencil plan: 32 x 8 column tiles and z segments of about 16
// planes.  A CTA is latency-bound on its plane-to-plane chain, so more
// resident and queued CTAs raise throughput until the three halo planes each
// segment re-marches (3/16 here) cost more than they hide.
static int fs_setup(Handle* h) {
    const int nx = h->g.nx, ny = h->g.ny, nz = h->g.nz;
    if (nz < 3 || nx < 3 || ny < 3 || getenv("NFGS_DISABLE_FUSED_STENCIL") != nullptr) return NFGS_OK;
    // NFGS_STENCIL_V1=1 keeps the entry-list stencil (fs::k_stencil)
    const bool v2 = getenv("NFGS_STENCIL_V1") == nullptr;
    int per_sm = 0;
    if (v2) {
        const size_t smem = h->f32 ? fs2::smem_bytes<float>() : fs2::smem_bytes<double>();
        h->fs_cw = (h->f32 && nx % 2 == 0) ? 2 : 1;
        if (h->f32 && h->fs_cw == 2) {
            CK(cudaFuncSetAttribute(fs2::k_stencil2<float, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs2::k_stencil2<float, 2>, fs2::NT, smem));
        } else if (h->f32) {
            CK(cudaFuncSetAttribute(fs2::k_stencil2<float, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs2::k_stencil2<float, 1>, fs2::NT, smem));
        } else {
            CK(cudaFuncSetAttribute(fs2::k_stencil2<double, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs2::k_stencil2<double, 1>, fs2::NT, smem));
        }
    } else {
        const size_t smem = h->f32 ? fs::smem_bytes<float>() : fs::smem_bytes<double>();
        if (h->f32) {
            CK(cudaFuncSetAttribute(fs::k_stencil<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs::k_stencil<float>, fs::NT, smem));
        } else {
            CK(cudaFuncSetAttribute(fs::k_stencil<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs::k_stencil<double>, fs::NT, smem));
        }
    }
    if (per_sm < 1) return NFGS_OK;
    const int gx = v2 ? fs2::tiles(nx, fs2::W) : fs::ntiles(nx, fs::TX);
    const int gy = v2 ? fs2::tiles(ny, fs2::H) : fs::ntiles(ny, fs::TY);
    const long long tiles = (long long)gx * gy;
    int best = std::max(1, std::min(16, nz / 16));
    if (const char* e = getenv("NFGS_STENCIL_NSEG")) {
        const int v = atoi(e);
        if (v >= 1 && v <= nz) best = v;
    }
    {
        const int per = (nz + best - 1) / best;
        best = (nz + per - 1) / per;  // no empty segments
    }
    h->fs_grid = dim3((unsigned)gx, (unsigned)gy, (unsigned)best);
    h->fs_nb = (int)(tiles * best);
    h->fs_on = true;
    h->fs_v2 = v2;
    return NFGS_OK;
}

// k_h=0 closure set-up (nfgs_solver.py:5058-5097, 5149-5225, 5262-5360):
// the FP64 linear map of the fit, the window's zero mode per plane and the
// per-buffer profile storage.
static int k0_setup(Handle* h, const std::vector<double>& wfac) {
    const NfgsParams& p = h->prm;
    const int nz = h->g.nz;
    const bool spline = p.horizontal_zero_mode == NFGS_HZM_CONSTRAINED_SPLINE;
    if (!(p.k0_smoothness >= 0.0) || !std::isfinite(p.k0_smoothness))
        return fail(NFGS_EINVAL, "k0_ode_smoothness must be non-negative");
    if (p.k0_update_mu > 1.0 || !std::isfinite(p.k0_update_mu))
        return fail(NFGS_EINVAL, "k0_update_mu must be in (0, 1]");
    if (spline) {
        if (p.k0_spline_basis < 4) return fail(NFGS_EINVAL, "k0_spline_basis_size must be >= 4");
        if (p.k0_spline_basis > nz) return fail(NFGS_EINVAL, "k0_spline_basis_size must not exceed Nz");
        if (p.k0_legacy) return fail(NFGS_EINVAL, "legacy coupled_k0 operator is not initialized");
    }
    std::vector<double> G, m;
    double cond = 0.0;
    if (!k0::build_operator(nz, h->g.dz, spline, p.k0_legacy != 0, p.k0_spline_basis, p.k0_smoothness, G, m, &cond))
        return fail(NFGS_EINVAL, "the k_h=0 closure's normal matrix is not positive definite");
    h->k0_on = true;
    h->k0_spline = spline ? 1 : 0;
    h->k0_cond = cond;
    k0::Dev& d = h->k0d;
    const size_t n2 = 2 * (size_t)nz;
    TRY(alloc(h, &d.hk, 3 * n2 * 8));
    TRY(alloc(h, &d.hlast, n2 * 8));
    TRY(alloc(h, &d.hbefore, n2 * 8));
    TRY(alloc(h, &d.hstar, n2 * 8));
    TRY(alloc(h, &d.target, n2 * 8));
    TRY(alloc(h, &d.stats, 4 * 8));
    TRY(alloc(h, &d.ptm, n2 * 8));
    TRY(alloc(h, &d.cell, 2 * n2 * 8));
    TRY(alloc(h, &d.kpart, 4 * (size_t)h->nb_src * 8));
    TRY(alloc(h, &h->k0_hsel, n2 * 8));
    TRY(upload(h, &d.G, G));
    TRY(upload(h, &d.m, m));
    TRY(upload(h, &d.wfac, wfac));
    for (double* q : {d.hk, d.hlast, d.hbefore, d.hstar, d.target, d.stats, d.ptm, d.cell, h->k0_hsel})
        CK(cudaMemsetAsync(q, 0, (q == d.hk ? 3 * n2 : (q == d.cell ? 2 * n2 : (q == d.stats ? 4 : n2))) * 8, h->s));
    CK(cudaStreamSynchronize(h->s));
    return NFGS_OK;
}

// Profile of the selected state as the closure's running H (its bottom
// value the target, nfgs_solver.py:6999-7004).
__global__ void k_k0_select(const double* hk, int idx, int nz, double t0, double t1, double* hlast) {
    for (int r = threadIdx.x; r < nz; r += blockDim.x) {
        hlast[r] = r == 0 ? t0 : hk[(long long)idx * 2 * nz + r];
        hlast[nz + r] = r == 0 ? t1 : hk[(long long)idx * 2 * nz + nz + r];
    }
}

// The transform kernel instantiated for (wide, axis, kind).
using TcKernel = void (*)(tc::Args);
static TcKernel tc_kernel(bool wide, int axis, int kind) {
    static const TcKernel k[2][2][2] = {
        {{tc::k_tc_transform<false, 0, 0>, tc::k_tc_transform<false, 0, 1>},
         {tc::k_tc_transform<false, 1, 0>, tc::k_tc_transform<false, 1, 1>}},
        {{tc::k_tc_transform<true, 0, 0>, tc::k_tc_transform<true, 0, 1>},
         {tc::k_tc_transform<true, 1, 0>, tc::k_tc_transform<true, 1, 1>}}};
    return k[wide ? 1 : 0][axis ? 1 : 0][kind ? 1 : 0];
}

static int tc_setup(Handle* h) {
    const int nx = h->g.nx, ny = h->g.ny;
    if (!h->f32 || (nx % 2) || (ny % 2)) return NFGS_OK;
    const int px = (nx - 2) / 2, py = (ny - 2) / 2;
    if (px < 1 || py < 1 || px > tc::PW_K || py > tc::PW_K) return NFGS_OK;
    if (getenv("NFGS_DISABLE_TC") != nullptr) return NFGS_OK;
    // Above 128 pairs per axis the four-role kernel is 3x faster than the
    // SIMT contractions, but FP32 solves through it end twice as far from the
    // FP64 solve (514^2 x 257 quadrupole: relative L2 of B 0.057 against
    // 0.029, energy ratio 0.979 against 1.001), so it runs only on request.
    if ((px > tc::PP || py > tc::PP) && getenv("NFGS_TC_WIDE") == nullptr) return NFGS_OK;
    int dev = 0, nsm = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    for (int w = 0; w < 2; ++w)
        for (int ax = 0; ax < 2; ++ax)
            for (int kd = 0; kd < 2; ++kd)
                CK(cudaFuncSetAttribute(tc_kernel(w != 0, ax, kd), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        tc::SMEM_TOTAL));
    if (nsm < 4) return NFGS_OK;
    const int kinds[4] = {0, 0, 1, 1};
    const int lens[4] = {nx, ny, nx - 2, ny - 2};
    const int ps[4] = {px, py, px, py};
    for (int q = 0; q < 4; ++q) {
        h->tc_wide[q] = ps[q] > tc::PP;
        auto img = h->tc_wide[q] ? tc_image_wide(kinds[q], lens[q], ps[q]) : tc_image(kinds[q], lens[q], ps[q]);
        TRY(alloc(h, &h->tc_img[q], img.size() * 2));
        CK(cudaMemcpy(h->tc_img[q], img.data(), img.size() * 2, cudaMemcpyHostToDevice));
    }
    TRY(alloc(h, &h->tc_err, sizeof(int)));
    CK(cudaMemset(h->tc_err, 0, sizeof(int)));
    h->tc_px = px;
    h->tc_py = py;
    h->tc_nsm = nsm;
    h->tc_on = true;
    return NFGS_OK;
}

static int tc_launch(Handle* h, int which, int inverse, const float* in, tc::Addr ia, float* out,
                     void* const* otab, const int* osel, tc::Addr oa, int nvec, const int* skip) {
    if (nvec <= 0) return NFGS_OK;
    tc::Args a{};
    a.in = in;
    a.out = out;
    a.out_table = otab;
    a.out_sel = osel;
    a.ia = ia;
    a.oa = oa;
    a.nvec = nvec;
    const int kinds[4] = {0, 0, 1, 1};
    const int lens[4] = {h->g.nx, h->g.ny, h->g.nx - 2, h->g.ny - 2};
    a.kind = kinds[which];
    a.axis = which & 1;
    a.N = lens[which];
    a.P = (which & 1) ? h->tc_py : h->tc_px;
    a.norm = inverse ? (float)(1.0 / (2.0 * (a.kind == 0 ? a.N - 1 : a.N + 1))) : 1.0f;
    a.mat = (const uint4*)h->tc_img[which];
    a.skip = skip;
    a.err = h->tc_err;
    const int ntiles = (nvec + tc::TV - 1) / tc::TV;
    // programmatic stream serialisation: the kernel waits (griddepcontrol)
    // for its predecessor before reading its outputs, so its prologue (TMEM,
    // barriers, the constant matrix copy) may overlap the predecessor's end
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.blockDim = dim3(tc::NTHREADS);
    cfg.dynamicSmemBytes = tc::SMEM_TOTAL;
    cfg.stream = h->s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (h->tc_wide[which]) {
        // four roles per tile group: one CTA per SM in groups of four
        cfg.gridDim = dim3((unsigned)(4 * std::min(ntiles, h->tc_nsm / 4)));
        CK(cudaLaunchKernelEx(&cfg, tc_kernel(true, a.axis, a.kind), a));
    } else {
        cfg.gridDim = dim3((unsigned)std::min(ntiles, h->tc_nsm));
        CK(cudaLaunchKernelEx(&cfg, tc_kernel(false, a.axis, a.kind), a));
    }
    CK(cudaGetLastError());
    h->launches++;
    return NFGS_OK;
}

static tc::Addr rows(long long off, long long nvec, long long pitch) { return tc::Addr{off, nvec, 0, pitch, 1}; }
static tc::Addr cols(long long off, long long ncols, long long plane, long long pitch) {
    return tc::Addr{off, ncols, plane, 1, pitch};
}

// Forward 2-D transforms of S_B (DCT-I, all planes) and S_J (DST-I,
// interior, planes 1..nz-2), in place through tmpA / tmpB.
template <typename T>
static int forward_transforms(Handle* h, const DevCtl* ctl) {
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, PI = h->PI;
    const int nxi = nx - 2, nyi = ny - 2;
    const int* skip = ctl ? &ctl->stopped : nullptr;
    if (h->tc_on) {
        float *sb = (float*)h->sb, *ta = (float*)h->tmpA, *sj = (float*)h->sj, *tb = (float*)h->tmpB;
        const long long nr = (long long)nz * ny, nc = (long long)nz * nx;
        TRY(tc_launch(h, 0, 0, sb, rows(0, nr, nx), ta, nullptr, nullptr, rows(0, nr, nx), (int)nr, skip));
        TRY(tc_launch(h, 1, 0, ta, cols(0, nx, P, nx), sb, nullptr, nullptr, cols(0, nx, P, nx), (int)nc, skip));
        if (nz > 2) {
            const long long nri = (long long)(nz - 2) * nyi, nci = (long long)(nz - 2) * nxi;
            TRY(tc_launch(h, 2, 0, sj, rows(PI, nri, nxi), tb, nullptr, nullptr, rows(PI, nri, nxi), (int)nri, skip));
            TRY(tc_launch(h, 3, 0, tb, cols(PI, nxi, PI, nxi), sj, nullptr, nullptr, cols(PI, nxi, PI, nxi), (int)nci,
                          skip));
        }
        return NFGS_OK;
    }
    TRY(apply_x<T>(h, h->dctx_t, h->sb, nx, P, h->tmpA, nx, P, ny * nz, nx, nx, 1, nullptr, nullptr, ctl));
    TRY(apply_y<T>(h, h->dcty_t, h->tmpA, nx, P, h->sb, nx, P, ny, ny, nx, nz, ctl));
    if (nz > 2) {
        const char* sjp = (const char*)h->sj + (size_t)PI * h->esz;
        char* tbp = (char*)h->tmpB + (size_t)PI * h->esz;
        TRY(apply_x<T>(h, h->dstx_t, sjp, nxi, PI, tbp, nxi, PI, nyi * (nz - 2), nxi, nxi, 1, nullptr, nullptr, ctl));
        TRY(apply_y<T>(h, h->dsty_t, tbp, nxi, PI, (void*)sjp, nxi, PI, nyi, nyi, nxi, nz - 2, ctl));
    }
    return NFGS_OK;
}

// Inverse 2-D transforms: Robin-chain planes 1..nz-1 into phi[*cand_sel]
// planes 1..nz-1; Dirichlet-chain planes 1..nz-2 into the interior of
// az[*cand_sel].
template <typename T>
static int inverse_transforms(Handle* h, const DevCtl* ctl, const int* cand_sel, int az_top = 0) {
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, PI = h->PI;
    const int nxi = nx - 2, nyi = ny - 2;
    // A_z planes 1..nz-2 (the iteration's top plane is zero); the soft_cfcf
    // start also transforms its Robin top plane
    const int naz = az_top ? nz - 1 : nz - 2;
    const int* skip = ctl ? &ctl->stopped : nullptr;
    void* const* ptab = (void* const*)h->st_dev->phi;
    void* const* atab = (void* const*)h->st_dev->az;
    if (h->tc_on) {
        float *sb = (float*)h->sb, *ta = (float*)h->tmpA, *sj = (float*)h->sj, *tb = (float*)h->tmpB;
        const long long nc = (long long)(nz - 1) * nx, nr = (long long)(nz - 1) * ny;
        TRY(tc_launch(h, 1, 1, sb, cols(P, nx, P, nx), ta, nullptr, nullptr, cols(P, nx, P, nx), (int)nc, skip));
        TRY(tc_launch(h, 0, 1, ta, rows(P, nr, nx), nullptr, ptab, cand_sel, rows(P, nr, nx), (int)nr, skip));
        if (nz > 2) {
            const long long nci = (long long)naz * nxi, nri = (long long)naz * nyi;
            TRY(tc_launch(h, 3, 1, sj, cols(PI, nxi, PI, nxi), tb, nullptr, nullptr, cols(PI, nxi, PI, nxi), (int)nci,
                          skip));
            TRY(tc_launch(h, 2, 1, tb, rows(PI, nri, nxi), nullptr, atab, cand_sel,
                          tc::Addr{P + nx + 1, nyi, P, nx, 1}, (int)nri, skip));
        }
        return NFGS_OK;
    }
    {
        const char* shp = (const char*)h->sb + (size_t)P * h->esz;
        char* tap = (char*)h->tmpA + (size_t)P * h->esz;
        TRY(apply_y<T>(h, h->idcty_t, shp, nx, P, tap, nx, P, ny, ny, nx, nz - 1, ctl));
        TRY(apply_x<T>(h, h->idctx_t, tap, nx, P, (void*)(intptr_t)(P * h->esz), nx, P, ny * (nz - 1), nx, nx, 1,
                       ptab, cand_sel, ctl));
    }
    if (nz > 2) {
        const char* sjp = (const char*)h->sj + (size_t)PI * h->esz;
        char* tbp = (char*)h->tmpB + (size_t)PI * h->esz;
        TRY(apply_y<T>(h, h->idsty_t, sjp, nxi, PI, tbp, nxi, PI, nyi, nyi, nxi, naz, ctl));
        TRY(apply_x<T>(h, h->idstx_t, tbp, nxi, PI, (void*)(intptr_t)((P + nx + 1) * h->esz), nx, P, nyi, nxi, nxi,
                       naz, atab, cand_sel, ctl));
    }
    return NFGS_OK;
}

template <typename T>
static int zsolve_launch(Handle* h, const int* skip);

// ---------------------------------------------------------------------------
// Stencil pass launchers
// ---------------------------------------------------------------------------
template <typename T>
static int run_fused(Handle* h, const int* sel, const int* skip, int polarity) {
    fs::Args a{};
    a.g = h->g;
    a.st = h->st;
    a.sel = sel;
    a.skip = skip;
    a.bbg = h->bbg;
    a.bzobs = h->bzobs_t;
    a.jzt = h->jzt_t;
    a.hx = h->hx;
    a.hy = h->hy;
    a.use_h = h->use_h;
    a.box = h->box;
    const double am = h->prm.alpha_max;
    a.alpha_max = (am > 0 && std::isfinite(am)) ? am : -1.0;
    a.floor_b2 = h->prm.weak_field_floor_b2;
    a.o = SrcOpts{polarity, h->prm.face_parallel_exact_jz, h->wx != nullptr};
    a.wx = h->wx;
    a.wy = h->wy;
    a.wz = h->wz;
    a.sb = h->sb;
    a.sj = h->sj;
    a.partials = h->pface;
    a.nseg = (int)h->fs_grid.z;
    a.gx = (int)h->fs_grid.x;
    a.gy = (int)h->fs_grid.y;
    if (sizeof(T) == 4 && h->fs_v2 && h->fs_cw == 2)
        fs2::k_stencil2<T, sizeof(T) == 4 ? 2 : 1><<<h->fs_grid, fs2::NT, fs2::smem_bytes<T>(), h->s>>>(a);
    else if (h->fs_v2)
        fs2::k_stencil2<T, 1><<<h->fs_grid, fs2::NT, fs2::smem_bytes<T>(), h->s>>>(a);
    else fs::k_stencil<T><<<h->fs_grid, fs::NT, fs::smem_bytes<T>(), h->s>>>(a);
    CK(cudaGetLastError());
    h->launches++;
    h->sum_pf = h->pface;
    h->sum_nbf = h->fs_nb;
    h->sum_ps = h->pface + 5 * (size_t)h->fs_nb;
    h->sum_nbs = h->fs_nb;
    return NFGS_OK;
}

// Stencil pass.  Source-producing passes run the fused z-march; passes that
// only reconstruct (fields, diagnostics) run the three-pass kernels, which
// leave B, J_z and the face currents in HBM for their callers.
template <typename T>
static int run_stencil(Handle* h, const int* sel, const int* skip, int with_src, int polarity, int raw_j = 0) {
    const Geo& g = h->g;
    // the k_h=0 closures need per-plane sums of the parallel current, which
    // the three-pass kernels provide
    if (with_src && !raw_j && h->fs_on && !h->k0_on) return run_fused<T>(h, sel, skip, polarity);
    k_recon<T><<<h->sgrid, h->sblock, 0, h->s>>>(g, h->st, sel, skip, (const T*)h->bbg, (const T*)h->bzobs_t,
                                                 (const T*)h->jzt_t, (T)h->hx, (T)h->hy, h->use_h, (T*)h->B,
                                                 (T*)h->jz, h->k0_on ? h->k0d.hk : nullptr, h->k0_hsel,
                                                 h->k0_spline);
    CK(cudaGetLastError());
    double am = h->prm.alpha_max;
    k_face<T><<<h->sgrid, h->sblock, 0, h->s>>>(g, skip, (const T*)h->B, (const T*)h->bbg, (const T*)h->jz, h->box,
                                                (T)(am > 0 && std::isfinite(am) ? am : -1.0),
                                                (T)h->prm.weak_field_floor_b2, (T*)h->jpf, (T*)h->jb, h->pface,
                                                raw_j, h->k0_spline ? h->k0_hsel : nullptr);
    CK(cudaGetLastError());
    h->launches += 2;
    h->sum_pf = h->pface;
    h->sum_nbf = h->nb_face;
    h->sum_ps = h->psrc;
    h->sum_nbs = h->nb_src;
    if (with_src) {
        SrcOpts o{polarity, h->prm.face_parallel_exact_jz, h->wx != nullptr};
        k_src<T><<<h->sgrid, h->sblock, 0, h->s>>>(g, skip, (const T*)h->jpf, (const T*)h->jb, (const T*)h->jzt_t,
                                                   (const T*)h->bzobs_t, o, (const T*)h->wx, (const T*)h->wy,
                                                   (const T*)h->wz, (T*)h->sb, (T*)h->sj, h->psrc,
                                                   h->k0_on ? h->k0d.kpart : nullptr);
        CK(cudaGetLastError());
        h->launches++;
    }
    return NFGS_OK;
}

// Candidate finalisation.  With a k_h=0 closure the candidate's profile is
// fitted between the bottom projection of the un-relaxed scalars and their
// relaxation (nfgs_solver.py:6760-6799): finalise without relaxing, sum the
// PT current of the candidate, fit and blend H, then relax the scalars.
template <typename T>
static int finalize_candidate(Handle* h, const DevCtl* ctl, int use_ctl_mu, double mu, const int* cand_sel,
                              const int* cur_sel) {
    const long long P = h->g.P;
    const unsigned nb = (unsigned)((P + 255) / 256);
    if (!h->k0_on) {
        k_finalize<T><<<nb, 256, 0, h->s>>>(h->g, h->st, ctl, use_ctl_mu, mu, cand_sel, cur_sel, (const T*)h->phiab_t,
                                            (const T*)h->dphi_t, h->prm.projection_weight, 1, 1,
                                            (const T*)h->azb_t);
        CK(cudaGetLastError());
        h->launches++;
        return NFGS_OK;
    }
    k_finalize<T><<<nb, 256, 0, h->s>>>(h->g, h->st, ctl, use_ctl_mu, mu, cand_sel, cur_sel, (const T*)h->phiab_t,
                                        (const T*)h->dphi_t, h->prm.projection_weight, 0, 1, (const T*)h->azb_t);
    k0::k_k0_pt<T><<<h->g.nz, 256, 0, h->s>>>(h->g, h->st, cand_sel, ctl ? &ctl->stopped : nullptr, h->k0d.ptm);
    k0::k_k0_update<<<1, 256, 0, h->s>>>(h->g, h->k0d, cand_sel, cur_sel, ctl, use_ctl_mu, mu, h->prm.k0_update_mu,
                                         h->prm.k0_face_target, (int)(h->sgrid.x * h->sgrid.y), h->k0_t[0],
                                         h->k0_t[1]);
    k_finalize<T><<<nb, 256, 0, h->s>>>(h->g, h->st, ctl, use_ctl_mu, mu, cand_sel, cur_sel, (const T*)h->phiab_t,
                                        (const T*)h->dphi_t, 0.0, 1, 1, (const T*)h->azb_t);
    CK(cudaGetLastError());
    h->launches += 4;
    return NFGS_OK;
}

// Sources -> modal solves -> candidate state (transforms, z-solves, inverse).
template <typename T>
static int run_solve(Handle* h, const DevCtl* ctl, const int* cand_sel, int zero_sources) {
    const Geo& g = h->g;
    if (!zero_sources) {
        TRY(forward_transforms<T>(h, ctl));
    } else {
        CK(cudaMemsetAsync(h->sb, 0, g.V * h->esz, h->s));
        CK(cudaMemsetAsync(h->sj, 0, (size_t)g.nz * h->PI * h->esz, h->s));
    }
    TRY(zsolve_launch<T>(h, ctl ? &ctl->stopped : nullptr));
    if (ctl != nullptr) {
        k_zero_mode<<<1, 32, 0, h->s>>>(g, (DevCtl*)ctl, h->s00);
        CK(cudaGetLastError());
        h->launches++;
    }
    TRY(inverse_transforms<T>(h, ctl, cand_sel));
    return NFGS_OK;
}

template <typename T>
static int zsolve_launch(Handle* h, const int* skip) {
    const Geo& g = h->g;
    const long long P = g.P, PI = h->PI;
    const int nz = g.nz;
    ZTab tr{h->zr_c, h->zr_i, h->zr_il, h->zr_ci, h->zr_ii, h->zr_rc};
    ZTab td{h->zd_c, h->zd_i, h->zd_il, h->zd_ci, h->zd_ii, h->zd_rc};
    int nbr = (int)((P + ZS_THREADS - 1) / ZS_THREADS);
    int nbd = nz > 2 ? (int)((PI + ZS_THREADS - 1) / ZS_THREADS) : 0;
    k_zsolve<T><<<nbr + nbd, ZS_THREADS, 0, h->s>>>(g, skip, (T*)h->sb, tr, h->lamNs, h->phi_bot_hat, h->der_hat,
                                             h->prm.robin_weight, h->s00, nz > 2 ? (T*)h->sj : nullptr, td, h->lamD,
                                             h->az_bot_hat, nbr);
    CK(cudaGetLastError());
    h->launches++;
    return NFGS_OK;
}

// ---------------------------------------------------------------------------
// Control kernels
// ---------------------------------------------------------------------------
// Deterministic column sums of the block partials (column-major: face
// columns 0..4 of length nbf, the source column of length nbs): stage 1
// reduces contiguous chunks into 6 x NCHUNK values, stage 2 sums those in a
// fixed order.
#define NCHUNK 64
__global__ void k_sum_stage1(const double* pf, int nbf, const double* ps, int nbs, double* mid) {
    const int col = blockIdx.y;
    const double* base = col < 5 ? pf + (long long)col * nbf : ps;
    const int nb = col < 5 ? nbf : nbs;
    const int per = (nb + NCHUNK - 1) / NCHUNK;
    const int b0 = blockIdx.x * per, b1 = min(nb, b0 + per);
    double acc = 0.0;
    for (int b = b0 + threadIdx.x; b < b1; b += blockDim.x) acc += base[b];
    __shared__ double sh[32];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
        t = warp_sum(t);
        if (threadIdx.x == 0) mid[col * NCHUNK + blockIdx.x] = t;
    }
}

__global__ void k_sum_stage2(const double* mid, double* out6) {
    const int col = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double t = mid[col * NCHUNK + lane] + mid[col * NCHUNK + 32 + lane];
    t = warp_sum(t);
    if (lane == 0) out6[col] = t;
}

__device__ __forceinline__ void scal_from_sums(Geo g, const double* s, double& sigma, double& divb, double& energy) {
    sigma = s[0] / fmax(s[1], 1e-30);
    double delta = fmin(g.dx, fmin(g.dy, g.dz));
    divb = (s[2] / (double)g.V) / (6.0 * (s[3] / (double)g.V) / delta + 1e-12);
    energy = s[4] * g.dx * g.dy * g.dz / 2.0;
}

__device__ __forceinline__ void pick_cand(DevCtl* c) {
    for (int q = 0; q < 3; ++q)
        if (q != c->cur && q != c->best) { c->cand = q; return; }
}

// Initial state statistics (nfgs_solver.py:3612-3614).
__global__ void k_ctl_init(Geo g, DevCtl* c, const double* sums, double* hist) {
    double sigma, divb, energy;
    scal_from_sums(g, sums, sigma, divb, energy);
    c->sigma0 = sigma; c->divb0 = divb; c->e0 = energy;
    c->best_sigma = sigma; c->prev_sigma = sigma; c->prev_energy = energy; c->cur_sigma = sigma;
    c->sumsb2 = sums[5];
    c->n = 0; c->cur = 0; c->best = 0;
    pick_cand(c);
    if (c->max_iter <= 0) { c->stopped = 1; c->stop_reason = 1; }
    (void)hist;
}

// One step of the stop rule (nfgs_solver.py:3658-3814).
__device__ __forceinline__ void ctl_step_body(Geo g, DevCtl* c, const double* sums, double* hist) {
    if (c->stopped) { c->not_rollback = 1; return; }
    double sigma, divb, energy;
    scal_from_sums(g, sums, sigma, divb, energy);
    const int n = c->n + 1;
    double* row = hist + (long long)c->n_hist * NFGS_HCOLS;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    bool diverged = !isfinite(sigma) || sigma > c->div_factor * fmax(c->best_sigma, 1e-30);
    c->rollback_now = 0;
    if (c->adaptive && diverged) {
        c->rollbacks += 1;
        c->mu_cur = fmax(c->mu_cur * c->mu_backoff, c->mu_min);
        c->cur = c->best;
        c->cur_sigma = c->best_sigma;
        c->streak = 0;
        row[0] = sigma; row[1] = nan; row[2] = nan; row[3] = c->mu_cur; row[4] = 1.0;
        row[5] = nan; row[6] = nan; row[7] = c->zero_ratio_last;
        c->n_hist += 1;
        c->prev_energy = nan;
        c->rollback_now = 1;
        c->n = n;
        if (c->rollbacks >= c->max_rollbacks) { c->stopped = 1; c->stop_reason = 5; }
    } else {
        c->cur = c->cand;
        double src = fabs(sigma - c->prev_sigma) / fmax(fabs(c->prev_sigma), 1e-30);
        double pe = c->prev_energy;
        double erc = fabs(energy - pe) / fmax(fabs(pe), 1e-30);
        row[0] = sigma; row[1] = divb; row[2] = energy; row[3] = c->mu_cur; row[4] = 0.0;
        row[5] = src; row[6] = erc; row[7] = c->zero_ratio_last;
        c->n_hist += 1;
        c->prev_energy = energy;
        c->final_iter = n;
        c->cur_sigma = sigma;
        double imp = c->prev_sigma - sigma;
        c->last_imp = imp; c->have_last_imp = 1;
        c->prev_sigma = sigma;
        c->flat = (imp < c->eps) ? c->flat + 1 : 0;
        if (sigma < c->best_sigma) {
            c->best_sigma = sigma; c->best_iter = n; c->best = c->cur; c->stall = 0; c->streak += 1;
            if (c->adaptive && c->streak >= c->growth_streak) {
                c->mu_cur = fmin(c->mu_cur * c->mu_growth, c->mu_max);
                c->streak = 0;
            }
        } else {
            c->stall += 1;
            c->streak = 0;
        }
        c->n = n;
        c->sumsb2 = sums[5];
        if (sigma < c->tol) { c->stopped = 1; c->stop_reason = 2; }
        else if (c->use_imp && c->flat >= c->flat_required) { c->stopped = 1; c->stop_reason = 3; }
        else if (c->patience > 0 && c->stall >= c->patience) { c->stopped = 1; c->stop_reason = 4; }
    }
    if (!c->stopped && n >= c->max_iter) { c->stopped = 1; c->stop_reason = 1; }
    pick_cand(c);
    c->not_rollback = (c->rollback_now && !c->stopped) ? 0 : 1;
}

__global__ void k_ctl_step(Geo g, DevCtl* c, const double* sums, double* hist) { ctl_step_body(g, c, sums, hist); }

// The second sum stage and the control step in one launch (iteration graph):
// the six fixed-order sums, then thread 0 steps the controller on them.
__global__ void k_sum_stage2_ctl(Geo g, const double* mid, double* out6, DevCtl* c, double* hist) {
    const int col = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double t = mid[col * NCHUNK + lane] + mid[col * NCHUNK + 32 + lane];
    t = warp_sum(t);
    if (lane == 0) out6[col] = t;
    __syncthreads();
    if (threadIdx.x == 0) ctl_step_body(g, c, out6, hist);
}

// After a rollback the restored state's sources were recomputed.
__global__ void k_ctl_rollback_sources(DevCtl* c, const double* sums) {
    if (c->not_rollback) return;
    c->sumsb2 = sums[5];
}

static void sum_partials(Handle* h) {
    k_sum_stage1<<<dim3(NCHUNK, 6), 256, 0, h->s>>>(h->sum_pf, h->sum_nbf, h->sum_ps, h->sum_nbs, h->scal + 8);
    k_sum_stage2<<<1, 192, 0, h->s>>>(h->scal + 8, h->scal);
    h->launches += 2;
}

// ---------------------------------------------------------------------------
// Boundary set-up
// ---------------------------------------------------------------------------
struct Fortran {
    int nx, ny, nz, bfx, bfy;
};

static int mudpack_axis(int n) {
    if (n < 2) return n < 1 ? 1 : n;
    double r = (double)n;
    int e2 = (int)std::ceil(std::log((r - 1.0) / 2.0) / std::log(2.0)) + 1;
    int e3 = (int)std::ceil(std::log((r - 1.0) / 3.0) / std::log(2.0)) + 1;
    int n2 = 2 * (1 << (e2 - 1)) + 1;
    int n3 = 3 * (1 << (e3 - 1)) + 1;
    return n2 < n3 ? n2 : n3;
}

template <typename T>
static int build_constants(Handle* h);

static int setup_boundary(Handle* h, const double* bx_h, const double* by_h, const double* bz_h, const double* jz_h,
                          const NfgsBoundaryOpts* o, double* diag) {
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, PI = h->PI;
    cudaStream_t s = h->s;
    double dg[NFGS_NDIAG];
    for (int q = 0; q < NFGS_NDIAG; ++q) dg[q] = 0.0;
    const size_t nobs = (size_t)o->ny_obs * o->nx_obs;
    double *up = nullptr;
    TRY(alloc(h, &up, 4 * nobs * sizeof(double)));
    CK(cudaMemcpyAsync(up, bx_h, nobs * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(up + nobs, by_h, nobs * 8, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(up + 2 * nobs, bz_h, nobs * 8, cudaMemcpyHostToDevice, s));
    if (o->jz_mode == NFGS_JZ_PROVIDED) CK(cudaMemcpyAsync(up + 3 * nobs, jz_h, nobs * 8, cudaMemcpyHostToDevice, s));
    double *w;  // scratch planes
    TRY(alloc(h, &w, 16 * (size_t)P * sizeof(double)));
    CK(cudaMemsetAsync(w, 0, 16 * (size_t)P * sizeof(double), s));
    double *bxo = h->bx_obs, *byo = h->by_obs, *bzo = h->bz_obs, *jzo = h->jz_obs;
    CK(cudaMemsetAsync(bxo, 0, P * 8, s));
    CK(cudaMemsetAsync(byo, 0, P * 8, s));
    CK(cudaMemsetAsync(bzo, 0, P * 8, s));
    CK(cudaMemsetAsync(jzo, 0, P * 8, s));
    {
        dim3 gr((o->copy_nx + 127) / 128, o->copy_ny);
        int rf = h->f32;
        k_embed<<<gr, 128, 0, s>>>(up, o->nx_obs, bxo, nx, o->fov_y0, o->fov_x0, o->src_y0, o->src_x0, o->copy_ny,
                                   o->copy_nx, rf);
        k_embed<<<gr, 128, 0, s>>>(up + nobs, o->nx_obs, byo, nx, o->fov_y0, o->fov_x0, o->src_y0, o->src_x0,
                                   o->copy_ny, o->copy_nx, rf);
        k_embed<<<gr, 128, 0, s>>>(up + 2 * nobs, o->nx_obs, bzo, nx, o->fov_y0, o->fov_x0, o->src_y0, o->src_x0,
                                   o->copy_ny, o->copy_nx, rf);
        if (o->jz_mode == NFGS_JZ_PROVIDED)
            k_embed<<<gr, 128, 0, s>>>(up + 3 * nobs, o->nx_obs, jzo, nx, o->fov_y0, o->fov_x0, o->src_y0, o->src_x0,
                                       o->copy_ny, o->copy_nx, rf);
        CK(cudaGetLastError());
        h->launches += 4;
    }
    // --- bottom Jz (nfgs_solver.py:1498-1567, 4489-4546)
    auto derive_jz = [&](int legacy, double* out) -> int {
        int hnx = nx, hny = ny, bx0 = 0, by0 = 0;
        if (legacy) {
            hnx = mudpack_axis(nx);
            hny = mudpack_axis(ny);
            bx0 = (hnx - nx) / 2;
            by0 = (hny - ny) / 2;
        }
        double* jzh = nullptr;
        TRY(alloc(h, &jzh, (size_t)hnx * hny * 8));
        h->setup_scratch.push_back(jzh);
        dim3 gr((hnx + 127) / 128, hny);
        k_jz_raw<<<gr, 128, 0, s>>>(bxo, byo, nx, ny, hnx, hny, bx0, by0, g.dx, g.dy, jzh);
        CK(cudaGetLastError());
        double fp = 1.0, fn = 1.0;
        int mode = o->ijzbcor;
        if (mode >= 2 && hnx >= 3 && hny >= 3) {
            k_cell_sums<<<1, 1024, 0, s>>>(jzh, hnx, hny, h->scal);
            CK(cudaGetLastError());
            double cs[3];
            CK(cudaMemcpyAsync(cs, h->scal, 24, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            double tot = cs[0], pos = cs[1], neg = cs[2];
            double tgt = 0.0;
            bool have = true;
            if (mode == 2) tgt = pos - 0.5 * tot;
            else if (mode == 3) tgt = std::max(pos, std::fabs(neg));
            else if (mode == 4) tgt = std::min(pos, std::fabs(neg));
            else have = false;
            if (have) {
                if (std::fabs(pos) > 0.0) fp = tgt / pos;
                if (std::fabs(neg) > 0.0) fn = tgt / std::fabs(neg);
            }
        }
        dim3 gc((nx + 127) / 128, ny);
        k_jz_finish<<<gc, 128, 0, s>>>(jzh, hnx, hny, bx0, by0, fp, fn, legacy, out, nx, ny);
        CK(cudaGetLastError());
        h->launches += 3;
        return NFGS_OK;
    };
    if (o->jz_mode != NFGS_JZ_PROVIDED) TRY(derive_jz(o->jz_mode == NFGS_JZ_DERIVE_LEGACY_HELPER, jzo));
    // the Stable-NFPT solver of the cfcf start derives its own current on the
    // legacy helper grid from the same maps (nfgs_solver.py:2071-2072)
    h->jz_stable_alias = o->jz_mode == NFGS_JZ_DERIVE_LEGACY_HELPER;
    if (!h->jz_stable_alias) TRY(derive_jz(1, h->jz_stable));
    // --- smoothing (nfgs_solver.py:2085-2090)
    if (o->smooth_passes > 0) {
        double* arr[5] = {bzo, jzo, bxo, byo, h->jz_stable};
        for (int a = 0; a < (h->jz_stable_alias ? 4 : 5); ++a)
            for (int pass = 0; pass < o->smooth_passes; ++pass) {
                dim3 gc((nx + 127) / 128, ny);
                k_smooth<<<gc, 128, 0, s>>>(arr[a], w, nx, ny);
                CK(cudaMemcpyAsync(arr[a], w, P * 8, cudaMemcpyDeviceToDevice, s));
                h->launches++;
            }
        CK(cudaGetLastError());
    }
    int rc = 0;
    if (o->zero_net_current) {
        double r[4];
        TRY(reduce4(h, jzo, P, r));
        double mean = r[0] / (double)P;
        CK(launch_map(P, s, [=] __device__(long long i) { jzo[i] -= mean; }));
        if (!h->jz_stable_alias) {
            double* jst = h->jz_stable;
            TRY(reduce4(h, jst, P, r));
            const double ms = r[0] / (double)P;
            CK(launch_map(P, s, [=] __device__(long long i) { jst[i] -= ms; }));
        }
    }
    // --- Az_bottom: endpoint-Dirichlet 2-D Poisson of -Jz (nfgs_solver.py:1132-1144)
    const int nxi = nx - 2, nyi = ny - 2;
    double *t1 = w + P, *t2 = w + 2 * P, *t3 = w + 3 * P, *t4 = w + 4 * P, *t5 = w + 5 * P, *t6 = w + 6 * P,
           *t7 = w + 7 * P, *t8 = w + 8 * P;
    {
        double* lamD = h->lamD;
        CK(launch_map(PI, s, [=] __device__(long long q) {
            long long j = q / nxi, i = q % nxi;
            t1[q] = -jzo[(j + 1) * nx + (i + 1)];
        }));
        TRY(apply_x<double>(h, h->dstx, t1, nxi, PI, t2, nxi, PI, nyi, nxi, nxi, 1));
        TRY(apply_y<double>(h, h->dsty, t2, nxi, PI, t3, nxi, PI, nyi, nyi, nxi, 1));
        CK(launch_map(PI, s, [=] __device__(long long q) { t3[q] /= lamD[q]; }));
        TRY(apply_y<double>(h, h->idsty, t3, nxi, PI, t2, nxi, PI, nyi, nyi, nxi, 1));
        TRY(apply_x<double>(h, h->idstx, t2, nxi, PI, t1, nxi, PI, nyi, nxi, nxi, 1));
        double* azb = h->az_bot;
        CK(launch_map(P, s, [=] __device__(long long q) {
            long long j = q / nx, i = q % nx;
            azb[q] = (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2) ? t1[(j - 1) * nxi + (i - 1)] : 0.0;
        }));
        if (h->f32) CK(launch_map(P, s, [=] __device__(long long q) { azb[q] = (double)(float)azb[q]; }));
        // Jz_T = -lap_xy Az_bottom, edges zeroed (nfgs_solver.py:3039-3046)
        double* jzt = h->jz_t;
        double dx = g.dx, dy = g.dy;
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            double v = -lap2d(azb, nx, ny, j, i, dx, dy);
            if (i == 0 || i == nx - 1 || j == 0 || j == ny - 1) v = 0.0;
            jzt[q] = v;
        }));
        dg[21] = rms_of(h, jzo, P, &rc); TRY(rc);
        dg[22] = rms_of(h, jzt, P, &rc); TRY(rc);
        CK(launch_map(P, s, [=] __device__(long long q) { t2[q] = jzo[q] - jzt[q]; }));
        dg[23] = rms_of(h, t2, P, &rc); TRY(rc);
    }
    // --- Gaussian separation (nfgs_solver.py:4671-4919)
    const double norm = 4.0 * (double)std::max(nx - 1, 1) * (double)std::max(ny - 1, 1);
    double *bxh = t4, *byh = t5, *bzh = t6;
    TRY(dct2_d(h, bxo, bxh, t1));
    TRY(dct2_d(h, byo, byh, t1));
    TRY(dct2_d(h, bzo, bzh, t1));
    {
        double m0[1], m1[1], m2[1];
        CK(cudaMemcpyAsync(m0, bxh, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(m1, byh, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(m2, bzh, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        dg[0] = m0[0] / norm; dg[1] = m1[0] / norm; dg[2] = m2[0] / norm;
        double r[4];
        TRY(reduce4(h, bxo, P, r)); dg[3] = r[0] / P;
        TRY(reduce4(h, byo, P, r)); dg[4] = r[0] / P;
        TRY(reduce4(h, bzo, P, r)); dg[5] = r[0] / P;
        double flux = std::fabs(r[0]) / std::max(r[2], 1e-30);
        dg[7] = flux;
        double res_mean = dg[2];
        double res_scale = std::max(std::sqrt(r[1] / P), 1e-30);
        if (h->prm.mean_bz_policy == NFGS_MEANBZ_UNIFORM_OPEN || h->prm.mean_bz_policy == NFGS_MEANBZ_REQUIRE_BALANCED) {
            if (h->prm.mean_bz_policy == NFGS_MEANBZ_REQUIRE_BALANCED && flux > h->prm.mean_mode_tolerance) {
                char b[256];
                snprintf(b, sizeof b, "The residual bottom Bz is not flux balanced: fraction=%.6e, tolerance=%.6e.", flux,
                         h->prm.mean_mode_tolerance);
                return fail(NFGS_EPOLICY, b);
            }
            h->open_bz = res_mean;
        } else {
            h->open_bz = h->prm.user_open_bz;
            double ratio = std::fabs(res_mean - h->open_bz) / res_scale;
            if (ratio > h->prm.mean_mode_tolerance) {
                char b[256];
                snprintf(b, sizeof b,
                         "user_supplied_open_bz does not match the residual Bz zero mode: ratio=%.6e, tolerance=%.6e.",
                         ratio, h->prm.mean_mode_tolerance);
                return fail(NFGS_EPOLICY, b);
            }
        }
        dg[6] = h->open_bz;
    }
    // divergence modes d_hat (spectral) or FD divergence
    double* dh = t7;
    double *alx = h->alx, *aly = h->aly;
    double dx = g.dx, dy = g.dy, dz = g.dz;
    auto spectral_div_hat = [&](const double* ax, const double* ay, double* out) -> int {
        // dstx_dcty_hat(ax): DCT along y, then DST along x of columns 1..nx-2
        TRY(apply_y<double>(h, h->dcty, ax, nx, P, t1, nx, P, ny, ny, nx, 1));
        CK(cudaMemsetAsync(t2, 0, P * 8, s));
        TRY(apply_x<double>(h, h->dstx, t1 + 1, nx, P, t2 + 1, nx, P, ny, nxi, nxi, 1));
        // dctx_dsty_hat(ay): DCT along x, then DST along y of rows 1..ny-2
        TRY(apply_x<double>(h, h->dctx, ay, nx, P, t1, nx, P, ny, nx, nx, 1));
        CK(cudaMemsetAsync(t3, 0, P * 8, s));
        TRY(apply_y<double>(h, h->dsty, t1 + nx, nx, P, t3 + nx, nx, P, nyi, nyi, nx, 1));
        CK(launch_map(P, s, [=] __device__(long long q) {
            long long j = q / nx, i = q % nx;
            out[q] = alx[i] * t2[q] + aly[j] * t3[q];
        }));
        return NFGS_OK;
    };
    double* D0 = h->d0;
    if (h->prm.gaussian_spectral) {
        TRY(spectral_div_hat(bxo, byo, dh));
        TRY(idct2_d(h, dh, D0, t1));
    } else {
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            D0[q] = d2d(bxo, nx, ny, j, i, 0, dx) + d2d(byo, nx, ny, j, i, 1, dy);
        }));
        TRY(dct2_d(h, D0, dh, t1));
    }
    {
        double m[1];
        CK(cudaMemcpyAsync(m, dh, 8, cudaMemcpyDeviceToHost, s));
        double r[4];
        TRY(reduce4(h, D0, P, r));
        double d0m = m[0] / norm;
        double ratio = std::fabs(d0m) / std::max(std::sqrt(r[1] / P), 1e-30);
        dg[8] = d0m;
        dg[9] = ratio;
        if (ratio > h->prm.mean_mode_tolerance) {
            if (h->prm.d0_policy == NFGS_POLICY_ERROR) {
                char b[256];
                snprintf(b, sizeof b,
                         "The bottom vector field is incompatible with the zero-mean endpoint-Neumann GS model "
                         "ratio=%.6e exceeds tolerance=%.6e.",
                         ratio, h->prm.mean_mode_tolerance);
                return fail(NFGS_EPOLICY, b);
            }
            if (h->prm.d0_policy == NFGS_POLICY_WARN_PROJECT) dg[30] = 1.0;
        }
    }
    // modal split (nfgs_solver.py:4798-4856)
    double *bzbh = t8, *pbh = h->phi_below_hat, *pah = h->phi_above_hat, *dpth = t1;
    double *lamN = h->lamN, *kN = h->kN;
    double* bzah = t2;
    CK(launch_map(P, s, [=] __device__(long long q) {
        double dq = q == 0 ? 0.0 : dh[q];
        double bzn = q == 0 ? 0.0 : bzh[q];
        double ks = q == 0 ? 1.0 : kN[q];
        double ls = q == 0 ? 1.0 : lamN[q];
        double below = q == 0 ? 0.0 : 0.5 * (bzn + dq / ks);
        double above = q == 0 ? 0.0 : 0.5 * (bzn - dq / ks);
        bzbh[q] = below;
        bzah[q] = above;
        pbh[q] = q == 0 ? 0.0 : below / ls;
        pah[q] = q == 0 ? 0.0 : above / ls;
        dpth[q] = q == 0 ? 0.0 : -dq / ls;
    }));
    // 2-D products
    double* t9 = w + 9 * P;
    double* t10 = w + 10 * P;
    TRY(idct2_d(h, bzah, h->bz_above, t9));
    TRY(idct2_d(h, pah, h->phi_above, t9));
    TRY(idct2_d(h, dpth, t10, t9));  // idct2(dphi_total_hat)
    // 3-D background, batches of planes through FP64 transforms
    const long long V = g.V;
    double* bbg = h->bbg_d;
    double* zmod;
    double* zout;
    const int chunk = 16;
    TRY(alloc(h, &zmod, (size_t)chunk * P * 8));
    TRY(alloc(h, &zout, (size_t)chunk * P * 8));
    double* ztmp;
    TRY(alloc(h, &ztmp, (size_t)chunk * P * 8));
    double open = h->open_bz;
    const int spectral = h->prm.gaussian_spectral;
    double* phib3 = nullptr;  // phi_below planes (needed for FD horizontals and diagnostics)
    TRY(alloc(h, &phib3, (size_t)V * 8));
    for (int z0 = 0; z0 < nz; z0 += chunk) {
        const int nb = std::min(chunk, nz - z0);
        // phi_below(z) = idct2(exp(-k z) phi_below_hat)
        CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
            long long p = q / P, m = q % P;
            double z = (double)(z0 + p) * dz;
            zmod[q] = exp(-z * kN[m]) * pbh[m];
        }));
        TRY(idct2_d(h, zmod, phib3 + (size_t)z0 * P, ztmp, nb));
        // bz_below(z)
        CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
            long long p = q / P, m = q % P;
            double z = (double)(z0 + p) * dz;
            zmod[q] = exp(-z * kN[m]) * bzbh[m];
        }));
        TRY(idct2_d(h, zmod, zout, ztmp, nb));
        CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
            bbg[2 * V + (long long)z0 * P + q] = zout[q] + open;
        }));
        if (spectral) {
            // bx_below = -gx, gx = IDST_x(IDCT_y(-alpha_x * dphi_dz_hat)),
            // dphi_dz_hat = -k exp(-kz) phi_below_hat (nfgs_solver.py:4847-4852)
            CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
                long long p = q / P, m = q % P;
                double z = (double)(z0 + p) * dz;
                double dpz = -kN[m] * exp(-z * kN[m]) * pbh[m];
                zmod[q] = -alx[m % nx] * dpz;
            }));
            TRY(apply_y<double>(h, h->idcty, zmod, nx, P, ztmp, nx, P, ny, ny, nx, nb));
            CK(cudaMemsetAsync(zout, 0, (size_t)nb * P * 8, s));
            TRY(apply_x<double>(h, h->idstx, ztmp + 1, nx, P, zout + 1, nx, P, ny, nxi, nxi, nb));
            CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
                bbg[(long long)z0 * P + q] = -zout[q];
            }));
            CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
                long long p = q / P, m = q % P;
                double z = (double)(z0 + p) * dz;
                double dpz = -kN[m] * exp(-z * kN[m]) * pbh[m];
                zmod[q] = -aly[m / nx] * dpz;
            }));
            TRY(apply_x<double>(h, h->idctx, zmod, nx, P, ztmp, nx, P, ny * nb, nx, nx, 1));
            CK(cudaMemsetAsync(zout, 0, (size_t)nb * P * 8, s));
            TRY(apply_y<double>(h, h->idsty, ztmp + nx, nx, P, zout + nx, nx, P, nyi, nyi, nx, nb));
            CK(launch_map((long long)nb * P, s, [=] __device__(long long q) {
                bbg[V + (long long)z0 * P + q] = -zout[q];
            }));
        }
    }
    if (!spectral) {
        // bx_below = -Dx(Dz phi_below), by_below = -Dy(Dz phi_below)
        CK(launch_map(V, s, [=] __device__(long long q) {
            int k = (int)(q / P);
            long long r = q % P;
            int j = (int)(r / nx), i = (int)(r % nx);
            auto dzp = [&](int jj, int ii) {
                auto f = [&](int kk) { return phib3[(long long)kk * P + (long long)jj * nx + ii]; };
                if (k == 0) return (-3.0 * f(0) + 4.0 * f(1) - f(2)) / (2.0 * dz);
                if (k == nz - 1) return (3.0 * f(nz - 1) - 4.0 * f(nz - 2) + f(nz - 3)) / (2.0 * dz);
                return (f(k + 1) - f(k - 1)) / (2.0 * dz);
            };
            auto dxf = [&](int ii) { return dzp(j, ii); };
            auto dyf = [&](int jj) { return dzp(jj, i); };
            double gx, gy;
            if (i == 0) gx = (-3.0 * dxf(0) + 4.0 * dxf(1) - dxf(2)) / (2.0 * dx);
            else if (i == nx - 1) gx = (3.0 * dxf(nx - 1) - 4.0 * dxf(nx - 2) + dxf(nx - 3)) / (2.0 * dx);
            else gx = (dxf(i + 1) - dxf(i - 1)) / (2.0 * dx);
            if (j == 0) gy = (-3.0 * dyf(0) + 4.0 * dyf(1) - dyf(2)) / (2.0 * dy);
            else if (j == ny - 1) gy = (3.0 * dyf(ny - 1) - 4.0 * dyf(ny - 2) + dyf(ny - 3)) / (2.0 * dy);
            else gy = (dyf(j + 1) - dyf(j - 1)) / (2.0 * dy);
            bbg[q] = -gx;
            bbg[V + q] = -gy;
        }));
    }
    // bottom_dphi_c_target = idct2(dphi_total_hat) - Dz(phi_below)(0)
    {
        double* tg = h->dphi_tgt;
        CK(launch_map(P, s, [=] __device__(long long q) {
            double dzp0 = (-3.0 * phib3[q] + 4.0 * phib3[P + q] - phib3[2 * P + q]) / (2.0 * dz);
            tg[q] = t10[q] - dzp0;
        }));
    }
    // diagnostics: bottom reconstruction and the scalar-background invariant
    {
        double* bza = h->bz_above;
        CK(launch_map(P, s, [=] __device__(long long q) { t9[q] = bbg[2 * V + q] + bza[q] - bzo[q]; }));
        double r[4];
        TRY(reduce4(h, t9, P, r));
        dg[10] = std::sqrt(r[1] / P);
        dg[11] = r[3];
        double* inv;
        TRY(alloc(h, &inv, (size_t)V * 8));
        h->setup_scratch.push_back(inv);
        CK(launch_map(V, s, [=] __device__(long long q) {
            int k = (int)(q / P);
            long long rr = q % P;
            int j = (int)(rr / nx), i = (int)(rr % nx);
            double lz = lap2d(phib3 + (long long)k * P, nx, ny, j, i, dx, dy);
            inv[q] = (lz + open) - bbg[2 * V + q];
        }));
        TRY(reduce4(h, inv, V, r));
        dg[12] = std::sqrt(r[1] / (3.0 * V));
    }
    // harmonic residual (nfgs_solver.py:4962-5029)
    {
        double *rx = w + 11 * P, *ry = w + 12 * P;  // residual maps
        double* azb = h->az_bot;
        // dphi_hat = k (phi_above_hat - phi_below_hat)
        double* dph = t10;
        CK(launch_map(P, s, [=] __device__(long long q) { dph[q] = kN[q] * (pah[q] - pbh[q]); }));
        double* gxm = t7;
        double* gym = t8;
        if (spectral) {
            // gx = IDST_x(IDCT_y(-alpha_x dphi_hat)) on interior columns
            CK(launch_map(P, s, [=] __device__(long long q) { t1[q] = -alx[q % nx] * dph[q]; }));
            TRY(apply_y<double>(h, h->idcty, t1, nx, P, t2, nx, P, ny, ny, nx, 1));
            CK(cudaMemsetAsync(gxm, 0, P * 8, s));
            TRY(apply_x<double>(h, h->idstx, t2 + 1, nx, P, gxm + 1, nx, P, ny, nxi, nxi, 1));
            CK(launch_map(P, s, [=] __device__(long long q) { t1[q] = -aly[q / nx] * dph[q]; }));
            TRY(apply_x<double>(h, h->idctx, t1, nx, P, t2, nx, P, ny, nx, nx, 1));
            CK(cudaMemsetAsync(gym, 0, P * 8, s));
            TRY(apply_y<double>(h, h->idsty, t2 + nx, nx, P, gym + nx, nx, P, nyi, nyi, nx, 1));
        } else {
            double* dphi = t1;
            TRY(idct2_d(h, dph, dphi, t2));
            CK(launch_map(P, s, [=] __device__(long long q) {
                int j = (int)(q / nx), i = (int)(q % nx);
                gxm[q] = d2d(dphi, nx, ny, j, i, 0, dx);
                gym[q] = d2d(dphi, nx, ny, j, i, 1, dy);
            }));
        }
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            double btx = d2d(azb, nx, ny, j, i, 1, dy);
            double bty = -d2d(azb, nx, ny, j, i, 0, dx);
            rx[q] = bxo[q] - (-gxm[q] + btx);
            ry[q] = byo[q] - (-gym[q] + bty);
        }));
        // constant modes via the DCT-I (0,0) weights
        double* cs = t5;
        TRY(dct2_d(h, rx, cs, t1));
        double cx[1], cy[1];
        CK(cudaMemcpyAsync(cx, cs, 8, cudaMemcpyDeviceToHost, s));
        TRY(dct2_d(h, ry, cs, t1));
        CK(cudaMemcpyAsync(cy, cs, 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double hxc = cx[0] / norm, hyc = cy[0] / norm;
        dg[15] = hxc; dg[16] = hyc;
        dg[17] = std::sqrt(0.5 * (hxc * hxc + hyc * hyc));
        double r[4], r2[4];
        TRY(reduce4(h, rx, P, r));
        TRY(reduce4(h, ry, P, r2));
        double res_rms = std::sqrt((r[1] + r2[1]) / (2.0 * P));
        // nonconstant rms: sum (x - c)^2 = sum x^2 - 2 c sum x + n c^2
        double ncs = (r[1] - 2 * hxc * r[0] + P * hxc * hxc) + (r2[1] - 2 * hyc * r2[0] + P * hyc * hyc);
        dg[18] = std::sqrt(std::max(ncs, 0.0) / (2.0 * P));
        double ro1[4], ro2[4];
        TRY(reduce4(h, bxo, P, ro1));
        TRY(reduce4(h, byo, P, ro2));
        double obs_rms = std::sqrt((ro1[1] + ro2[1]) / (2.0 * P));
        double ratio = res_rms / std::max(obs_rms, 1e-30);
        dg[13] = res_rms;
        dg[14] = ratio;
        // divergence and curl of the residual
        double* dv = t6;
        if (spectral) {
            TRY(spectral_div_hat(rx, ry, t4));
            TRY(idct2_d(h, t4, dv, t1));
        } else {
            CK(launch_map(P, s, [=] __device__(long long q) {
                int j = (int)(q / nx), i = (int)(q % nx);
                dv[q] = d2d(rx, nx, ny, j, i, 0, dx) + d2d(ry, nx, ny, j, i, 1, dy);
            }));
        }
        dg[19] = rms_of(h, dv, P, &rc); TRY(rc);
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            t4[q] = d2d(ry, nx, ny, j, i, 0, dx) - d2d(rx, nx, ny, j, i, 1, dy);
        }));
        dg[20] = rms_of(h, t4, P, &rc); TRY(rc);
        if (ratio > h->prm.mean_mode_tolerance) {
            if (h->prm.harmonic_policy == NFGS_HARM_ERROR) {
                char b[256];
                snprintf(b, sizeof b,
                         "Bottom horizontal reconstruction leaves a finite-domain harmonic residual ratio=%.6e, "
                         "tolerance=%.6e.",
                         ratio, h->prm.mean_mode_tolerance);
                return fail(NFGS_EPOLICY, b);
            }
            if (h->prm.harmonic_policy == NFGS_HARM_WARN) dg[31] = 1.0;
        }
        if (h->prm.horizontal_zero_mode == NFGS_HZM_FROZEN_LINEAR_HARMONIC) {
            h->hx = hxc; h->hy = hyc; h->use_h = 1;
        } else {
            h->hx = h->hy = 0.0; h->use_h = 0;
        }
        if (h->k0_on) {
            // H starts as the bottom target on every plane and the fit's
            // residual history restarts (nfgs_solver.py:5058-5067, 5200-5203)
            h->k0_t[0] = hxc;
            h->k0_t[1] = hyc;
            std::vector<double> hl(2 * (size_t)nz);
            for (int k = 0; k < nz; ++k) { hl[k] = hxc; hl[nz + k] = hyc; }
            double st[4] = {0.0, 0.0, h->k0_cond, 0.0};
            CK(cudaMemcpyAsync(h->k0d.hlast, hl.data(), hl.size() * 8, cudaMemcpyHostToDevice, s));
            CK(cudaMemcpyAsync(h->k0d.stats, st, sizeof st, cudaMemcpyHostToDevice, s));
            CK(cudaStreamSynchronize(s));
        }
    }
    dg[24] = (double)o->jz_mode;
    CK(cudaStreamSynchronize(s));
    // release the set-up scratch (kept allocations are the handle's)
    {
        std::vector<void*> drop = {up, w, zmod, zout, ztmp, phib3};
        for (void* p : h->setup_scratch) drop.push_back(p);
        h->setup_scratch.clear();
        for (auto it = h->owned.begin(); it != h->owned.end();) {
            bool d = false;
            for (void* p : drop) d = d || (it->p == p);
            if (d) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
        }
    }
    if (diag) std::memcpy(diag, dg, sizeof dg);
    if (h->f32) TRY(build_constants<float>(h));
    else TRY(build_constants<double>(h));
    h->boundary_set = 1;
    h->solution = -1;
    h->iter_active = 0;
    return NFGS_OK;
}

// Storage-type constants, modal boundary data, factor tables and state
// buffer boundary planes.
template <typename T>
static int build_constants(Handle* h) {
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V, PI = h->PI;
    cudaStream_t s = h->s;
    TRY(to_storage(h, h->bbg_d, h->bbg, 3 * V));
    TRY(to_storage(h, h->bz_obs, h->bzobs_t, P));
    TRY(to_storage(h, h->jz_t, h->jzt_t, P));
    TRY(to_storage(h, h->phi_above, h->phiab_t, P));
    TRY(to_storage(h, h->dphi_tgt, h->dphi_t, P));
    // modal boundary data from the storage-rounded planes
    double *tmp, *tmp2;
    TRY(alloc(h, &tmp, (size_t)P * 8));
    TRY(alloc(h, &tmp2, (size_t)P * 8));
    TRY(from_storage(h, h->phiab_t, tmp2, P));
    TRY(dct2_d(h, tmp2, h->phi_bot_hat, tmp));
    TRY(from_storage(h, h->dphi_t, tmp2, P));
    TRY(dct2_d(h, tmp2, h->der_hat, tmp));
    {
        double *a = h->phi_bot_hat, *b = h->der_hat;
        CK(launch_map(1, s, [=] __device__(long long) { a[0] = 0.0; b[0] = 0.0; }));
    }
    const int nxi = nx - 2, nyi = ny - 2;
    {
        // DST-I of the (storage-rounded) Az_bottom interior
        double* azb = h->az_bot;
        int f32 = h->f32;
        CK(launch_map(PI, s, [=] __device__(long long q) {
            long long j = q / nxi, i = q % nxi;
            double v = azb[(j + 1) * nx + (i + 1)];
            tmp2[q] = f32 ? (double)(float)v : v;
        }));
        TRY(apply_x<double>(h, h->dstx, tmp2, nxi, PI, tmp, nxi, PI, nyi, nxi, nxi, 1));
        TRY(apply_y<double>(h, h->dsty, tmp, nxi, PI, h->az_bot_hat, nxi, PI, nyi, nyi, nxi, 1));
    }
    // factor tables
    k_ztables<<<(unsigned)((P + 255) / 256), 256, 0, s>>>(g, 0, h->prm.robin_weight, h->lamN, h->kN, h->zr_c, h->zr_i,
                                                          h->zr_il, h->zr_ci, h->zr_ii, h->zr_rc);
    CK(cudaGetLastError());
    if (nz > 2) {
        k_ztables<<<(unsigned)((PI + 255) / 256), 256, 0, s>>>(g, 1, 0.0, h->lamD, nullptr, h->zd_c, h->zd_i, h->zd_il,
                                                               h->zd_ci, h->zd_ii, h->zd_rc);
        CK(cudaGetLastError());
    }
    // state buffers: zero, then the fixed bottom planes
    void* azb_t = h->azb_t;
    TRY(to_storage(h, h->az_bot, azb_t, P));
    for (int b = 0; b < 3; ++b) {
        CK(cudaMemsetAsync(h->st.phi[b], 0, V * h->esz, s));
        CK(cudaMemsetAsync(h->st.az[b], 0, V * h->esz, s));
        CK(cudaMemcpyAsync(h->st.phi[b], h->phiab_t, P * h->esz, cudaMemcpyDeviceToDevice, s));
        CK(cudaMemcpyAsync(h->st.az[b], azb_t, P * h->esz, cudaMemcpyDeviceToDevice, s));
    }
    CK(cudaStreamSynchronize(s));
    for (auto it = h->owned.begin(); it != h->owned.end();) {
        if (it->p == tmp || it->p == tmp2) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); }
        else ++it;
    }
    return NFGS_OK;
}

// ---------------------------------------------------------------------------
// Iteration driver
// ---------------------------------------------------------------------------
template <typename T>
static int enqueue_iteration(Handle* h) {
    DevCtl* c = h->ctl;
    // solve from the sources of the current state into the candidate buffer
    TRY(run_solve<T>(h, c, &c->cand, 0));
    TRY(finalize_candidate<T>(h, c, 1, 1.0, &c->cand, &c->cur));
    TRY(run_stencil<T>(h, &c->cand, &c->stopped, 1, h->stop.polarity_mask));
    k_sum_stage1<<<dim3(NCHUNK, 6), 256, 0, h->s>>>(h->sum_pf, h->sum_nbf, h->sum_ps, h->sum_nbs, h->scal + 8);
    k_sum_stage2_ctl<<<1, 192, 0, h->s>>>(h->g, h->scal + 8, h->scal, c, h->hist);
    CK(cudaGetLastError());
    h->launches += 2;
    if (h->stop.adaptive_mu) {
        TRY(run_stencil<T>(h, &c->cur, &c->not_rollback, 1, h->stop.polarity_mask));
        sum_partials(h);
        k_ctl_rollback_sources<<<1, 1, 0, h->s>>>(c, h->scal);
        CK(cudaGetLastError());
        h->launches += 2;
    }
    return NFGS_OK;
}

// ---------------------------------------------------------------------------
// Tile autotuner: the z-segment count of the fused stencil is chosen per grid
// shape by timing candidates on live data (the gs_cfcf start state) the
// first time a shape is iterated; the choice is cached for the process.
// NFGS_STENCIL_NSEG fixes it; NFGS_AUTOTUNE=0 keeps the built-in heuristic.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int>, int> g_tune_nseg;

template <typename T>
static int autotune_stencil(Handle* h, int polarity) {
    if (!h->fs_on || h->fs_tuned || h->k0_on) return NFGS_OK;
    h->fs_tuned = 1;
    if (getenv("NFGS_STENCIL_NSEG") != nullptr) return NFGS_OK;
    if (const char* e = getenv("NFGS_AUTOTUNE"))
        if (e[0] == '0') return NFGS_OK;
    const int nz = h->g.nz;
    const auto key = std::make_tuple(h->g.nx, h->g.ny, nz, (int)h->f32);
    // the lock is held through the tuning: handles of one shape begun on
    // several threads wait for the first one's choice and all use it
    std::lock_guard<std::mutex> lk(g_tune_mu);
    {
        auto it = g_tune_nseg.find(key);
        if (it != g_tune_nseg.end()) {
            const int per = (nz + it->second - 1) / it->second;
            h->fs_grid.z = (unsigned)((nz + per - 1) / per);
            h->fs_nb = (int)(h->fs_grid.x * h->fs_grid.y * h->fs_grid.z);
            return NFGS_OK;
        }
    }
    const int cands[] = {1, 2, 4, 8, 12, 16};
    const unsigned gz0 = h->fs_grid.z;
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    float best_ms = -1.0f;
    unsigned best = gz0;
    for (int c : cands) {
        if (c > nz / 4 && c != 1) continue;
        const int per = (nz + c - 1) / c;
        const unsigned gz = (unsigned)((nz + per - 1) / per);
        if ((long long)h->fs_grid.x * h->fs_grid.y * gz * NFGS_NRED > h->pface_len) continue;
        h->fs_grid.z = gz;
        h->fs_nb = (int)(h->fs_grid.x * h->fs_grid.y * gz);
        TRY(run_fused<T>(h, &h->consts[0], nullptr, polarity));
        CK(cudaEventRecord(a, h->s));
        for (int r = 0; r < 3; ++r) TRY(run_fused<T>(h, &h->consts[0], nullptr, polarity));
        CK(cudaEventRecord(b, h->s));
        CK(cudaEventSynchronize(b));
        float ms = 0.0f;
        CK(cudaEventElapsedTime(&ms, a, b));
        if (best_ms < 0 || ms < best_ms) { best_ms = ms; best = gz; }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    h->fs_grid.z = best;
    h->fs_nb = (int)(h->fs_grid.x * h->fs_grid.y * best);
    g_tune_nseg[key] = (int)best;
    return NFGS_OK;
}

template <typename T>
static int iterate_begin_t(Handle* h, const NfgsStop* stop) {
    if (!h->boundary_set)
        return fail(NFGS_ESTATE, "NFGS boundary is not set. Call set_bottom_vector_boundary() first.");
    h->stop = *stop;
    if (h->stop.check_every < 1) h->stop.check_every = 1;
    int rows = std::max(stop->max_iter, 0) + 2;
    if (rows > h->hist_rows) {
        if (h->hist) {
            for (auto it = h->owned.begin(); it != h->owned.end();) {
                if (it->p == h->hist) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
            }
        }
        TRY(alloc(h, &h->hist, (size_t)rows * NFGS_HCOLS * 8));
        h->hist_rows = rows;
    }
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    DevCtl c{};
    c.cur = 0; c.best = 0; c.cand = 1;
    c.max_iter = stop->max_iter;
    c.patience = stop->patience;
    c.flat_required = std::max(stop->patience, 1);
    c.use_imp = stop->sigma_improvement_tol > 0.0;
    c.eps = c.use_imp ? stop->sigma_improvement_tol : 0.0;
    c.adaptive = stop->adaptive_mu;
    c.growth_streak = stop->growth_streak;
    c.max_rollbacks = stop->max_rollbacks;
    c.source_policy = h->prm.source_policy;
    c.tol = stop->tol;
    c.mu_min = stop->mu_min; c.mu_max = stop->mu_max; c.mu_backoff = stop->mu_backoff; c.mu_growth = stop->mu_growth;
    c.div_factor = stop->divergence_factor;
    c.src_tol = h->prm.source_zero_mode_tolerance;
    c.mu_cur = stop->mu;
    c.not_rollback = 1;
    CK(cudaMemcpyAsync(h->ctl, &c, sizeof c, cudaMemcpyHostToDevice, h->s));
    h->launches = 0;
    CK(cudaEventRecord(h->ev0, h->s));
    if (h->k0_on) {
        // every start state carries the closure's running H
        // (nfgs_solver.py:6613-6645 reconstructs with the current _H_k0)
        const size_t n2 = 2 * (size_t)h->g.nz;
        for (int b = 0; b < 3; ++b)
            CK(cudaMemcpyAsync(h->k0d.hk + b * n2, h->k0d.hlast, n2 * 8, cudaMemcpyDeviceToDevice, h->s));
    }
    // gs_cfcf: zero-source modal solves into state 0 (nfgs_solver.py:6630-6645)
    TRY(run_solve<T>(h, nullptr, &h->consts[0], 1));
    {
        const long long P = h->g.P;
        k_finalize<T><<<(unsigned)((P + 255) / 256), 256, 0, h->s>>>(
            h->g, h->st, nullptr, 0, 1.0, &h->consts[0], &h->consts[0], (const T*)h->phiab_t, (const T*)h->dphi_t,
            h->prm.projection_weight, 0, 1, (const T*)h->azb_t);
        CK(cudaGetLastError());
        h->launches++;
    }
    TRY(autotune_stencil<T>(h, stop->polarity_mask));
    TRY(run_stencil<T>(h, &h->consts[0], nullptr, 1, stop->polarity_mask));
    sum_partials(h);
    k_ctl_init<<<1, 1, 0, h->s>>>(h->g, h->ctl, h->scal, h->hist);
    CK(cudaGetLastError());
    h->launches += 2;
    h->init_zr = 0.0;
    h->iter_active = 1;
    h->select_final = 0;
    h->diag_valid = 0;
    h->advanced = 0;
    h->solution = -1;
    h->total_ms = 0.0f;
    return NFGS_OK;
}

// sigma, divB and energy of a set of partial sums (for host decisions)
__global__ void k_scal_out(Geo g, const double* sums, double* out3) {
    double sigma, divb, energy;
    scal_from_sums(g, sums, sigma, divb, energy);
    out3[0] = sigma;
    out3[1] = divb;
    out3[2] = energy;
}

// Start state prepared by iterate_begin (buffer 0).
static int start_state(Handle* h, void** phi, void** az) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    if (h->advanced) return fail(NFGS_ESTATE, "the iteration has already advanced");
    CK(cudaStreamSynchronize(h->s));  // the views are complete for any stream
    *phi = h->st.phi[0];
    *az = h->st.az[0];
    return NFGS_OK;
}

// sigma_J of a supplied state (device, storage type), and optionally make it
// the start: mode 0 evaluates only, 1 replaces the gs_cfcf start when the
// supplied sigma_J is lower, 2 replaces it unconditionally.  Buffer 2 is free
// right after iterate_begin (current = best = 0, candidate = 1).
template <typename T>
static int adopt_buffer2(Handle* h, int mode, double* out);

// Sources and sums of the start state (buffer 0) again, and buffer 2 a copy
// of it: the modal solves never write some boundary entries of a candidate
// buffer, so nothing of a rejected state may outlive the restart calls.
template <typename T>
static int restore_start(Handle* h) {
    const size_t vb = (size_t)h->g.V * h->esz;
    TRY(run_stencil<T>(h, &h->consts[0], nullptr, 1, h->stop.polarity_mask));
    sum_partials(h);
    CK(cudaMemcpyAsync(h->st.phi[2], h->st.phi[0], vb, cudaMemcpyDeviceToDevice, h->s));
    CK(cudaMemcpyAsync(h->st.az[2], h->st.az[0], vb, cudaMemcpyDeviceToDevice, h->s));
    h->stale_start = 0;
    return NFGS_OK;
}

template <typename T>
static int restart_from_t(Handle* h, const void* phi, const void* az, int mode, double* out) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    if (h->advanced) return fail(NFGS_ESTATE, "the iteration has already advanced");
    const size_t vb = (size_t)h->g.V * h->esz;
    if (mode == 4) {
        if (h->stale_start) TRY(restore_start<T>(h));
        CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
        CK(cudaStreamSynchronize(h->s));
        out[0] = std::nan("");
        out[1] = h->ctl_h->sigma0;
        out[2] = 0.0;
        return NFGS_OK;
    }
    CK(cudaMemcpyAsync(h->st.phi[2], phi, vb, cudaMemcpyDeviceToDevice, h->s));
    CK(cudaMemcpyAsync(h->st.az[2], az, vb, cudaMemcpyDeviceToDevice, h->s));
    return adopt_buffer2<T>(h, mode, out);
}

// Evaluate the state in buffer 2 and, per `mode`, make it the start (the
// tail of restart_from_t, shared with the soft_cfcf start).
template <typename T>
static int adopt_buffer2(Handle* h, int mode, double* out) {
    const size_t vb = (size_t)h->g.V * h->esz;
    if (!h->dsmall) TRY(alloc(h, &h->dsmall, 8 * sizeof(double)));
    TRY(run_stencil<T>(h, &h->consts[2], nullptr, 1, h->stop.polarity_mask));
    sum_partials(h);
    k_scal_out<<<1, 1, 0, h->s>>>(h->g, h->scal, h->dsmall);
    CK(cudaGetLastError());
    double sc[3];
    CK(cudaMemcpyAsync(sc, h->dsmall, sizeof sc, cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    const double s_gs = h->ctl_h->sigma0;
    const bool accept = mode == 2 || (mode == 1 && std::isfinite(sc[0]) && sc[0] < s_gs);
    if (accept) {
        // the sources and sums of the supplied state are current: make it state 0
        CK(cudaMemcpyAsync(h->st.phi[0], h->st.phi[2], vb, cudaMemcpyDeviceToDevice, h->s));
        CK(cudaMemcpyAsync(h->st.az[0], h->st.az[2], vb, cudaMemcpyDeviceToDevice, h->s));
        k_ctl_init<<<1, 1, 0, h->s>>>(h->g, h->ctl, h->scal, h->hist);
        CK(cudaGetLastError());
        h->stale_start = 0;
    } else if (mode == 3) {
        // evaluation only: the start's sources are restored by the next
        // restart call of another mode or before the first advance
        h->stale_start = 1;
    } else {
        TRY(restore_start<T>(h));
    }
    CK(cudaStreamSynchronize(h->s));
    out[0] = sc[0];
    out[1] = s_gs;
    out[2] = accept ? 1.0 : 0.0;
    return NFGS_OK;
}

// soft_cfcf start (nfgs_solver.py:6427-6484): after iterate_begin, the
// modal profiles of the Phi (DCT-I) and A_z (interior DST-I) modes go into
// the modal buffers, the inverse transforms (A_z with its Robin top plane)
// build the state in buffer 2, the bottom Phi plane is restored, and the
// state replaces the gs_cfcf start.  out[0..2]: curl-current energy, current
// energy and objective of the modal quadrature (nfgs_solver.py:6486-6540),
// out[3]: sigma_J of the start.
template <typename T>
static int soft_cfcf_start_t(Handle* h, double eps, double ridge, double* out) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    if (h->advanced) return fail(NFGS_ESTATE, "the iteration has already advanced");
    const Geo& g = h->g;
    if (g.nz < 5) return fail(NFGS_EINVAL, "soft_cfcf requires Nz >= 5");
    if (g.nx < 3 || g.ny < 3) return fail(NFGS_EINVAL, "soft_cfcf requires Nx, Ny >= 3");
    if (!(eps >= 0.0) || !std::isfinite(eps)) return fail(NFGS_EINVAL, "soft_cfcf_epsilon must be non-negative");
    if (!(ridge >= 0.0) || !std::isfinite(ridge))
        return fail(NFGS_EINVAL, "soft_cfcf_normal_ridge must be non-negative");
    const long long P = g.P, PI = h->PI;
    const long long n = g.nz - 2;
    // modes per launch: band + vector scratch of at most 1 GB (about 90k
    // modes at 257 heights, more than the ~76k threads the SMs hold at once)
    const long long per_mode = n * (soft::BS + 1) * 8;
    const long long CH = std::max(1LL, std::min(P, (1LL << 30) / per_mode));
    double *band = nullptr, *vec = nullptr, *en = nullptr, *sums = nullptr;
    int* err = nullptr;
    auto cleanup = [&]() {
        if (band) release(h, band);
        if (vec) release(h, vec);
        if (en) release(h, en);
        if (sums) release(h, sums);
        if (err) release(h, err);
    };
    int rc = NFGS_OK;
    do {
        if ((rc = alloc(h, &band, (size_t)(n * soft::BS * CH) * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &vec, (size_t)(n * CH) * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &en, (size_t)(2 * (P + PI)) * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &sums, 4 * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &err, sizeof(int))) != NFGS_OK) break;
    } while (0);
    if (rc != NFGS_OK) { cleanup(); return rc; }
    cudaError_t ce = cudaMemsetAsync(err, 0, sizeof(int), h->s);
    for (int kind = 0; kind < 2 && ce == cudaSuccess; ++kind) {
        const long long M = kind == 0 ? P : PI;
        const double* kk = kind == 0 ? h->kN : h->lamD;
        const double* bot = kind == 0 ? h->phi_bot_hat : h->az_bot_hat;
        T* hat = (T*)(kind == 0 ? h->sb : h->sj);
        double* enk = kind == 0 ? en : en + 2 * P;
        for (long long m0 = 0; m0 < M && ce == cudaSuccess; m0 += CH) {
            const long long cnt = std::min(CH, M - m0);
            soft::k_soft_profile<T><<<(unsigned)((cnt + 127) / 128), 128, 0, h->s>>>(
                g, kind, m0, cnt, M, kk, bot, eps, ridge, CH, band, vec, hat, enk, err);
            ce = cudaGetLastError();
            h->launches++;
        }
        if (ce == cudaSuccess) {
            soft::k_soft_sum<<<1, 256, 0, h->s>>>(enk, M, sums + 2 * kind);
            ce = cudaGetLastError();
            h->launches++;
        }
    }
    int herr = 0;
    double hs[4] = {0, 0, 0, 0};
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, h->s);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(hs, sums, sizeof hs, cudaMemcpyDeviceToHost, h->s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->s);
    cleanup();
    CK(ce);
    if (herr == soft::ERR_NONFINITE) return fail(NFGS_ESTATE, "soft_cfcf modal normal solve produced non-finite values");
    if (herr != 0) return fail(NFGS_EUNSUPPORTED, "soft_cfcf modal rows wider than the kernel's band");
    // state in buffer 2: Phi planes 1..nz-1, A_z interior planes 1..nz-1
    // (walls and the bottom plane as every state holds them), Phi bottom
    TRY(inverse_transforms<T>(h, nullptr, &h->consts[2], 1));
    k_finalize<T><<<(unsigned)((P + 255) / 256), 256, 0, h->s>>>(g, h->st, nullptr, 0, 1.0, &h->consts[2],
                                                                &h->consts[2], (const T*)h->phiab_t,
                                                                (const T*)h->dphi_t, 0.0, 0, 0, (const T*)h->azb_t);
    CK(cudaGetLastError());
    h->launches++;
    const double fac = g.dx * g.dy * g.dz / (4.0 * (double)(g.nx - 1) * (double)(g.ny - 1));
    out[0] = fac * (hs[0] + hs[2]);
    out[1] = fac * (hs[1] + hs[3]);
    out[2] = out[0] + eps * out[1];
    double ad[3];
    TRY(adopt_buffer2<T>(h, 2, ad));
    out[3] = ad[0];
    return NFGS_OK;
}

// Zero-source modal solve along z with a Dirichlet bottom u0 and a
// Dirichlet (zero) or mirrored-ghost Neumann top, one thread per mode, FP64
// in the reference's operation order (_thomas_solve_batched_lowmem,
// nfgs_solver.py:536-608).  out is [nz][M]; cs is [nz][M] scratch.
__global__ void k_modal_harmonic(long long M, int nz, double dz, const double* __restrict__ lam,
                                 const double* __restrict__ u0, int top_dirichlet, double* __restrict__ out,
                                 double* __restrict__ cs) {
    const long long m = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const double dz2 = dz * dz, a = 1.0 / dz2, c = 1.0 / dz2;
    const double b = lam[m] - 2.0 / dz2;
    const int n = top_dirichlet ? nz - 2 : nz - 1;
    const double ub = u0[m];
    out[m] = ub;
    for (int k = 1; k < nz; ++k) out[(long long)k * M + m] = 0.0;
    if (n <= 0) return;
    // forward sweep: c*_i in cs, d*_i in out row i + 1
    const double bottom_a = (n == 1 && !top_dirichlet) ? 2.0 * a : a;
    const double d0 = 0.0 - bottom_a * ub;
    double cp, dp;
    if (n == 1) {
        cp = 0.0;
        dp = d0 / b;
    } else {
        cp = c / b;
        dp = d0 / b;
    }
    cs[m] = cp;
    out[M + m] = dp;
    for (int i = 1; i < n; ++i) {
        double ae = a, ce = c;
        if (i == n - 1) {
            ce = 0.0;
            if (!top_dirichlet) ae = 2.0 * a;
        }
        const double den = b - ae * cp;
        cp = ce / den;
        dp = (0.0 - ae * dp) / den;
        cs[(long long)i * M + m] = cp;
        out[(long long)(i + 1) * M + m] = dp;
    }
    // back substitution: u_{i} = d*_i - c*_i u_{i+1}
    double up = dp;
    for (int i = n - 2; i >= 0; --i) {
        const long long q = (long long)(i + 1) * M + m;
        up = out[q] - cs[(long long)i * M + m] * up;
        out[q] = up;
    }
}

// cfcf start (nfgs_solver.py:6080-6147): the Stable-NFPT curl-free-current
// state projected into the NFGS scalars, after iterate_begin.
//  * A_z: the zero-source Dirichlet extension of the stable solver's
//    T = Poisson2D(-Jz) (nfgs_solver.py:2331-2351, 1305-1333, 3394-3398): the
//    gs_cfcf start's A_z when the stable current is the one in use, else
//    built from the legacy helper-grid current;
//  * B_z of the stable state: the potential field's, the harmonic extension
//    of Bz_obs with a Neumann top (nfgs_solver.py:1611-1627), with the BC1
//    wall and top copies when lateral_bc1 (nfgs_solver.py:2138-2164) and
//    Bz_obs on the bottom plane (nfgs_solver.py:2180);
//  * Phi_c: lap_xy Phi_c = B_z - B_background,z on planes 1..nz-1 (mean
//    mode dropped, nfgs_solver.py:1120-1130, 1146-1181), Phi_c(0) = Phi^>.
// The state replaces the gs_cfcf start (buffer 2 -> 0).  mean_out (nz
// doubles, optional): the mean B_c,z per height the reference reports;
// out[0]: sigma_J of the start, out[1]: 1 when A_z differs from gs_cfcf's.
template <typename T>
static int cfcf_start_t(Handle* h, int lateral_bc1, double* mean_out, double* out) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    if (h->advanced) return fail(NFGS_ESTATE, "the iteration has already advanced");
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, nxi = nx - 2, nyi = ny - 2;
    const long long P = g.P, V = g.V, PI = h->PI;
    cudaStream_t s = h->s;
    double *vol = nullptr, *cs = nullptr, *tmp = nullptr, *pl = nullptr;
    auto cleanup = [&]() {
        if (vol) release(h, vol);
        if (cs) release(h, cs);
        if (tmp) release(h, tmp);
        if (pl) release(h, pl);
    };
    int rc = NFGS_OK;
    do {
        if ((rc = alloc(h, &vol, (size_t)V * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &cs, (size_t)V * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &tmp, (size_t)V * 8)) != NFGS_OK) break;
        if ((rc = alloc(h, &pl, (size_t)4 * P * 8)) != NFGS_OK) break;
    } while (0);
    if (rc != NFGS_OK) { cleanup(); return rc; }
    rc = [&]() -> int {
        // B_z of the potential field: modal harmonic extension of Bz_obs
        double* bzh = pl;
        TRY(dct2_d(h, h->bz_obs, bzh, pl + P));
        k_modal_harmonic<<<(unsigned)((P + 127) / 128), 128, 0, s>>>(P, nz, g.dz, h->lamN, bzh, 0, tmp, cs);
        CK(cudaGetLastError());
        h->launches++;
        TRY(idct2_d(h, tmp, vol, cs, nz));
        // BC1: x walls on rows 1..ny-2, then y walls, then the top plane
        if (lateral_bc1) {
            if (nx > 1)
                CK(launch_map((long long)nz * ny, s, [=] __device__(long long q) {
                    const long long k = q / ny, j = q % ny;
                    if (j < 1 || j > ny - 2) return;
                    double* r = vol + k * P + j * nx;
                    r[0] = r[1];
                    r[nx - 1] = r[nx - 2];
                }));
            if (ny > 1)
                CK(launch_map((long long)nz * nx, s, [=] __device__(long long q) {
                    const long long k = q / nx, i = q % nx;
                    double* c0 = vol + k * P + i;
                    c0[0] = c0[nx];
                    c0[(long long)(ny - 1) * nx] = c0[(long long)(ny - 2) * nx];
                }));
            if (nz > 1)
                CK(launch_map(P, s, [=] __device__(long long q) {
                    vol[(long long)(nz - 1) * P + q] = vol[(long long)(nz - 2) * P + q];
                }));
        }
        // B_c,z = B_z - B_background,z (bottom plane: Bz_obs - B_background,z)
        {
            const double* bzo = h->bz_obs;
            const double* bgz = h->bbg_d + 2 * V;
            CK(launch_map(V, s, [=] __device__(long long q) {
                const double bz = q < P ? bzo[q] : vol[q];
                vol[q] = bz - bgz[q];
            }));
        }
        TRY(dct2_d(h, vol, tmp, cs, nz));
        if (mean_out) {
            const double norm = 4.0 * (double)std::max(nx - 1, 1) * (double)std::max(ny - 1, 1);
            std::vector<double> mh(nz);
            CK(cudaMemcpy2DAsync(mh.data(), 8, tmp, (size_t)P * 8, 8, nz, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            for (int k = 0; k < nz; ++k) mean_out[k] = mh[k] / norm;
        }
        // Phi_c modes of planes 1..nz-1 into the Robin chain's modal buffer
        {
            T* hat = (T*)h->sb;
            const double* lam = h->lamN;
            CK(launch_map(V - P, s, [=] __device__(long long q) {
                const long long m = q % P;
                const double v = m == 0 ? 0.0 : tmp[P + q] / lam[m];
                hat[P + q] = (T)v;
            }));
        }
        // A_z modes of the stable solver's current (planes 1..nz-2) when it
        // differs from the one in use
        const bool own_az = !h->jz_stable_alias && nx >= 3 && ny >= 3;
        double* tst = pl + P;  // T of the stable solver, calculation grid
        if (own_az) {
            double *t1 = pl + 2 * P, *t2 = pl + 3 * P;
            const double* jst = h->jz_stable;
            const double* lamD = h->lamD;
            CK(launch_map(PI, s, [=] __device__(long long q) {
                const long long j = q / nxi, i = q % nxi;
                t1[q] = -jst[(j + 1) * nx + (i + 1)];
            }));
            TRY(apply_x<double>(h, h->dstx, t1, nxi, PI, t2, nxi, PI, nyi, nxi, nxi, 1));
            TRY(apply_y<double>(h, h->dsty, t2, nxi, PI, t1, nxi, PI, nyi, nyi, nxi, 1));
            CK(launch_map(PI, s, [=] __device__(long long q) { t1[q] /= lamD[q]; }));  // modes of T
            TRY(apply_y<double>(h, h->idsty, t1, nxi, PI, t2, nxi, PI, nyi, nyi, nxi, 1));
            TRY(apply_x<double>(h, h->idstx, t2, nxi, PI, cs, nxi, PI, nyi, nxi, nxi, 1));
            CK(launch_map(P, s, [=] __device__(long long q) {
                const long long j = q / nx, i = q % nx;
                tst[q] = (j >= 1 && j <= ny - 2 && i >= 1 && i <= nx - 2) ? cs[(j - 1) * nxi + (i - 1)] : 0.0;
            }));
            k_modal_harmonic<<<(unsigned)((PI + 127) / 128), 128, 0, s>>>(PI, nz, g.dz, lamD, t1, 1, tmp, cs);
            CK(cudaGetLastError());
            h->launches++;
            T* hat = (T*)h->sj;
            CK(launch_map((long long)(nz - 2) * PI, s, [=] __device__(long long q) { hat[PI + q] = (T)tmp[PI + q]; }));
        }
        // inverse transforms into buffer 2; Phi_c bottom plane Phi^>
        TRY(inverse_transforms<T>(h, nullptr, &h->consts[2], 0));
        k_finalize<T><<<(unsigned)((P + 255) / 256), 256, 0, s>>>(g, h->st, nullptr, 0, 1.0, &h->consts[2],
                                                                   &h->consts[2], (const T*)h->phiab_t,
                                                                   (const T*)h->dphi_t, 0.0, 0, 0, (const T*)h->azb_t);
        CK(cudaGetLastError());
        h->launches++;
        if (own_az) {
            T* az2 = (T*)h->st.az[2];
            CK(launch_map(V, s, [=] __device__(long long q) {
                const long long k = q / P, r = q % P, j = r / nx, i = r % nx;
                if (k == 0) az2[q] = (T)tst[r];
                else if (k == nz - 1 || i == 0 || i == nx - 1 || j == 0 || j == ny - 1) az2[q] = T(0);
            }));
        } else {
            CK(cudaMemcpyAsync(h->st.az[2], h->st.az[0], (size_t)V * h->esz, cudaMemcpyDeviceToDevice, s));
        }
        double ad[3];
        TRY(adopt_buffer2<T>(h, 2, ad));
        out[0] = ad[0];
        out[1] = own_az ? 1.0 : 0.0;
        return NFGS_OK;
    }();
    CK(cudaStreamSynchronize(s));
    cleanup();
    return rc;
}

// Per-step diagnostics of record_iteration_diagnostics (nfgs_solver.py:
// 6660-6681, 6806-6933) for the candidate of the last single step: built from
// the state it came from (diag_prev) and the candidate (diag_cand), both
// still in their buffers right after the step.  out[15] in the order of the
// reference's dictionary: phi_update, az_update, phi_map_residual,
// az_map_residual, h_k0_update, h_k0_map_residual, bcz_pde_residual,
// jz_pde_residual, poloidal_pde_residual, toroidal_pde_residual,
// mixed_row_residual, bottom_field_imprint, bottom_jz_imprint (relative),
// alpha_clip_fraction, weak_field_floor_fraction.  Uses the export buffers
// (B, J_z, face current) and FP64 scratch; the iteration state and the
// sources awaiting the next step are untouched.
template <typename T>
static int step_diagnostics_t(Handle* h, double* out) {
    if (!h->iter_active || !h->advanced || !h->diag_valid)
        return fail(NFGS_ESTATE, "no single iteration step to diagnose (advance one step at a time)");
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz, nxi = nx - 2, nyi = ny - 2;
    const long long P = g.P, V = g.V, PI = h->PI;
    cudaStream_t s = h->s;
    const int prev = h->diag_prev, cand = h->diag_cand;
    const double mu = h->diag_mu;
    const long long nbf = h->nb_face;
    std::vector<double*> sc;
    auto cleanup = [&]() { for (double* p : sc) release(h, p); };
    auto get = [&](double** p, size_t n) -> int {
        int r = alloc(h, p, n * 8);
        if (r == NFGS_OK) sc.push_back(*p);
        return r;
    };
    double *phs, *azs, *bcz, *jzs, *sb, *sj, *sphi, *saz, *t1, *t2, *pf, *pc, *pd;
    int rc = NFGS_OK;
    do {
        if ((rc = get(&phs, V)) || (rc = get(&azs, V)) || (rc = get(&bcz, V)) || (rc = get(&jzs, V))) break;
        if ((rc = get(&sb, V)) || (rc = get(&sj, V)) || (rc = get(&sphi, V)) || (rc = get(&saz, V))) break;
        if ((rc = get(&t1, V)) || (rc = get(&t2, V))) break;
        if ((rc = get(&pf, 5 * nbf)) || (rc = get(&pc, 2 * nbf)) || (rc = get(&pd, diag::NS * nbf))) break;
    } while (0);
    if (rc != NFGS_OK) { cleanup(); return rc; }
    rc = [&]() -> int {
        const unsigned nb = (unsigned)((V + 255) / 256);
        // unrelaxed candidate and its Laplacians
        diag::k_unrelaxed<T><<<nb, 256, 0, s>>>(g, (const T*)h->st.phi[cand], (const T*)h->st.phi[prev],
                                                (const T*)h->st.az[cand], (const T*)h->st.az[prev], mu, phs, azs);
        diag::k_laps<<<nb, 256, 0, s>>>(g, phs, azs, bcz, jzs);
        CK(cudaGetLastError());
        // sources and face fractions of the state the candidate came from
        const double am = h->prm.alpha_max;
        const double amax = (am > 0 && std::isfinite(am)) ? am : -1.0;
        k_recon<T><<<h->sgrid, h->sblock, 0, s>>>(g, h->st, &h->consts[prev], nullptr, (const T*)h->bbg,
                                                  (const T*)h->bzobs_t, (const T*)h->jzt_t, (T)h->hx, (T)h->hy,
                                                  h->use_h, (T*)h->B, (T*)h->jz, h->k0_on ? h->k0d.hk : nullptr,
                                                  h->k0_hsel, h->k0_spline);
        k_face<T><<<h->sgrid, h->sblock, 0, s>>>(g, nullptr, (const T*)h->B, (const T*)h->bbg, (const T*)h->jz,
                                                 h->box, (T)amax, (T)h->prm.weak_field_floor_b2, (T*)h->jpf,
                                                 (T*)h->jb, pf, 0, h->k0_spline ? h->k0_hsel : nullptr);
        diag::k_face_counts<T><<<h->sgrid, h->sblock, 0, s>>>(g, (const T*)h->B, (const T*)h->bbg, (const T*)h->jz,
                                                              amax, h->prm.weak_field_floor_b2, pc);
        SrcOpts o{h->stop.polarity_mask, h->prm.face_parallel_exact_jz, h->wx != nullptr};
        diag::k_src_full<T><<<h->sgrid, h->sblock, 0, s>>>(g, (const T*)h->jpf, (const T*)h->jb, (const T*)h->jzt_t,
                                                           (const T*)h->bzobs_t, o, (const T*)h->wx,
                                                           (const T*)h->wy, (const T*)h->wz, sb, sj);
        CK(cudaGetLastError());
        // source_phi = idct2(dct2(S_B) / lambda), mean mode zero
        TRY(dct2_d(h, sb, t1, t2, nz));
        {
            const double* lam = h->lamN;
            CK(launch_map(V, s, [=] __device__(long long q) {
                const long long m = q % P;
                t1[q] = m == 0 ? 0.0 : t1[q] / lam[m];
            }));
        }
        TRY(idct2_d(h, t1, sphi, t2, nz));
        // source_az_rhs = -idst2(dst2(S_J interior) / lambda_D) on the interior
        CK(cudaMemsetAsync(saz, 0, (size_t)V * 8, s));
        if (nx >= 3 && ny >= 3) {
            CK(launch_map((long long)nz * PI, s, [=] __device__(long long q) {
                const long long k = q / PI, r = q % PI, j = r / nxi, i = r % nxi;
                t1[q] = sj[k * P + (j + 1) * nx + (i + 1)];
            }));
            TRY(apply_x<double>(h, h->dstx, t1, nxi, PI, t2, nxi, PI, nyi, nxi, nxi, nz));
            TRY(apply_y<double>(h, h->dsty, t2, nxi, PI, t1, nxi, PI, nyi, nyi, nxi, nz));
            const double* lamD = h->lamD;
            CK(launch_map((long long)nz * PI, s, [=] __device__(long long q) { t1[q] = -t1[q] / lamD[q % PI]; }));
            TRY(apply_x<double>(h, h->idstx, t1, nxi, PI, t2, nxi, PI, nyi, nxi, nxi, nz));
            TRY(apply_y<double>(h, h->idsty, t2, nxi, PI, t1, nxi, PI, nyi, nyi, nxi, nz));
            CK(launch_map((long long)nz * PI, s, [=] __device__(long long q) {
                const long long k = q / PI, r = q % PI, j = r / nxi, i = r % nxi;
                saz[k * P + (j + 1) * nx + (i + 1)] = t1[q];
            }));
        }
        // the candidate's field for the bottom imprints
        k_recon<T><<<h->sgrid, h->sblock, 0, s>>>(g, h->st, &h->consts[cand], nullptr, (const T*)h->bbg,
                                                  (const T*)h->bzobs_t, (const T*)h->jzt_t, (T)h->hx, (T)h->hy,
                                                  h->use_h, (T*)h->B, (T*)h->jz, h->k0_on ? h->k0d.hk : nullptr,
                                                  h->k0_hsel, h->k0_spline);
        diag::k_diag_sums<T><<<h->sgrid, h->sblock, 0, s>>>(
            g, (const T*)h->st.phi[prev], (const T*)h->st.az[prev], (const T*)h->st.phi[cand],
            (const T*)h->st.az[cand], phs, azs, bcz, jzs, sb, sj, sphi, saz,
            h->prm.robin_weight > 0.0 ? h->dphi_tgt : nullptr, h->prm.robin_weight, (const T*)h->B,
            (const T*)h->bbg, (const T*)h->jz, h->bx_obs, h->by_obs, h->bz_obs, h->jz_t, pd);
        CK(cudaGetLastError());
        h->launches += 9;
        std::vector<double> hd((size_t)diag::NS * nbf), hc((size_t)2 * nbf);
        CK(cudaMemcpyAsync(hd.data(), pd, hd.size() * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hc.data(), pc, hc.size() * 8, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double S[diag::NS], C[2] = {0.0, 0.0};
        for (int q = 0; q < diag::NS; ++q) {
            double a = 0.0;
            for (long long b = 0; b < nbf; ++b) a += hd[(size_t)q * nbf + b];
            S[q] = a;
        }
        for (int q = 0; q < 2; ++q)
            for (long long b = 0; b < nbf; ++b) C[q] += hc[(size_t)q * nbf + b];
        // counts of each slice (rms = sqrt(sum / count), clamped at 1e-30)
        const double nV = (double)V;
        const double nbi = (double)((nz > 4) ? std::max(0, nz - 3) : std::max(0, nz - 2)) * (double)P;
        const double njz = (double)std::max(0, nz - 2) * (double)P;
        const double ntor = (double)std::max(0, nz - 2) * (double)std::max(0, nxi) * (double)std::max(0, nyi);
        const double nmix = (double)P, nbot = 3.0 * (double)P, njb = (double)P;
        auto rms = [](double sum, double n) { return n > 0 ? std::sqrt(sum / n) : 0.0; };
        auto rel = [&](double num, double den, double n) { return rms(num, n) / std::max(rms(den, n), 1e-30); };
        auto relop = [&](double num, std::initializer_list<double> terms, double n) {
            double m = 0.0;
            for (double t : terms) m = std::max(m, rms(t, n));
            return rms(num, n) / std::max(m, 1e-30);
        };
        using namespace diag;
        out[0] = rel(S[S_DPHI_U], S[S_PHI], nV);
        out[1] = rel(S[S_DAZ_U], S[S_AZ], nV);
        out[2] = rel(S[S_DPHI_M], S[S_PHI], nV);
        out[3] = rel(S[S_DAZ_M], S[S_AZ], nV);
        out[4] = 0.0;
        out[5] = 0.0;
        if (h->k0_on) {
            // h_k0_update / h_k0_map_residual (nfgs_solver.py:6884-6893)
            std::vector<double> hb(2 * nz), hl(2 * nz), hs(2 * nz);
            CK(cudaMemcpyAsync(hb.data(), h->k0d.hbefore, 16 * (size_t)nz, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(hl.data(), h->k0d.hlast, 16 * (size_t)nz, cudaMemcpyDeviceToHost, s));
            CK(cudaMemcpyAsync(hs.data(), h->k0d.hstar, 16 * (size_t)nz, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            double db = 0.0, du = 0.0, dm = 0.0;
            for (int q = 0; q < 2 * nz; ++q) {
                db += hb[q] * hb[q];
                du += (hl[q] - hb[q]) * (hl[q] - hb[q]);
                dm += (hs[q] - hb[q]) * (hs[q] - hb[q]);
            }
            out[4] = rel(du, db, 2.0 * nz);
            out[5] = rel(dm, db, 2.0 * nz);
        }
        out[6] = rel(S[S_BCZ_R], S[S_SB_BI], nbi);
        out[7] = rel(S[S_JZ_R], S[S_SJ_I], njz);
        out[8] = relop(S[S_POL_R], {S[S_POL_D2], S[S_POL_LX], S[S_POL_SRC]}, nbi);
        out[9] = relop(S[S_TOR_R], {S[S_TOR_D2], S[S_TOR_LX], S[S_TOR_SRC]}, ntor);
        out[10] = relop(S[S_MIX_R], {S[S_MIX_PDE], S[S_MIX_DER], S[S_MIX_SRC]}, nmix);
        out[11] = rel(S[S_BOT_E], S[S_BOT_O], nbot);
        out[12] = rel(S[S_JZB_E], S[S_JZB_O], njb);
        const double nfaces = (double)std::max(0, nz - 1) * (double)P;
        out[13] = (am > 0 && std::isfinite(am) && nfaces > 0) ? C[1] / nfaces : 0.0;
        out[14] = nfaces > 0 ? C[0] / nfaces : 0.0;
        return NFGS_OK;
    }();
    cudaStreamSynchronize(s);
    cleanup();
    return rc;
}

// Capture the per-iteration launch sequence of a handle into its CUDA graph
// (once per iterate call; the graph holds device-side indices only).
template <typename T>
static int ensure_graph_t(Handle* h) {
    if (h->gexec) return NFGS_OK;
    CK(cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    int before = h->launches;
    int r = enqueue_iteration<T>(h);
    cudaGraph_t gr = nullptr;
    cudaError_t e = cudaStreamEndCapture(h->s, &gr);
    if (r != NFGS_OK) { if (gr) cudaGraphDestroy(gr); return r; }
    CK(e);
    h->graph = gr;
    CK(cudaGraphInstantiate(&h->gexec, h->graph, 0));
    h->launches = before;  // counted per graph launch
    size_t nn = 0;
    CK(cudaGraphGetNodes(h->graph, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(h->graph, nodes.data(), &nn));
    int kn = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        CK(cudaGraphNodeGetType(nd, &t));
        kn += (t == cudaGraphNodeTypeKernel);
    }
    h->graph_kernels = kn;
    return NFGS_OK;
}

template <typename T>
static int iterate_advance_t(Handle* h, int max_steps, int32_t* stop_reason, int32_t* n_done) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    if (h->stale_start) TRY(restore_start<T>(h));
    h->advanced = 1;
    CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    int done = 0;
    while (!h->ctl_h->stopped && done < max_steps) {
        int k = std::min(h->stop.check_every, max_steps - done);
        h->diag_prev = h->ctl_h->cur;
        h->diag_cand = h->ctl_h->cand;
        h->diag_mu = h->ctl_h->mu_cur;
        h->diag_valid = (k == 1);
        if (h->stop.use_graph) {
            TRY(ensure_graph_t<T>(h));
            for (int q = 0; q < k; ++q) CK(cudaGraphLaunch(h->gexec, h->s));
            h->launches += k * h->graph_kernels;
        } else {
            for (int q = 0; q < k; ++q) TRY(enqueue_iteration<T>(h));
        }
        done += k;
        CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
        CK(cudaStreamSynchronize(h->s));
    }
    if (stop_reason) *stop_reason = h->ctl_h->stopped ? h->ctl_h->stop_reason : NFGS_STOP_RUNNING;
    if (n_done) *n_done = h->ctl_h->n;
    return NFGS_OK;
}

}  // namespace

namespace {

// Fields of a state (nfgs_solver.py:2881-2903): B from k_recon, J_z state,
// J_x,y = vertical faces mapped to centres with zero walls and top
// (nfgs_solver.py:5780-5794, 5935-5941).
template <typename T, typename O>
__global__ void k_gather_fields(Geo g, const T* __restrict__ B, const T* __restrict__ bbg, const T* __restrict__ jz,
                                const T* __restrict__ jf, int nzc, int y0, int ny_c, int x0, int nx_c,
                                O* __restrict__ out, const double* __restrict__ jh_wall = nullptr) {
    long long n = (long long)nzc * ny_c * nx_c;
    long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int k = (int)(q / ((long long)ny_c * nx_c));
    long long r = q % ((long long)ny_c * nx_c);
    int j = (int)(r / nx_c) + y0, i = (int)(r % nx_c) + x0;
    const long long P = g.P, V = g.V, FV = (long long)(g.nz - 1) * P;
    const long long c = (long long)k * P + (long long)j * g.nx + i;
    const long long pq = (long long)j * g.nx + i;
    // B holds the carrier; the field is B_background + carrier
    out[q] = (O)(bbg[c] + B[c]);
    out[n + q] = (O)(bbg[V + c] + B[V + c]);
    out[2 * n + q] = (O)(bbg[2 * V + c] + B[2 * V + c]);
    bool wall = (i == 0 || i == g.nx - 1 || j == 0 || j == g.ny - 1 || k == g.nz - 1);
    double jx = 0.0, jy = 0.0;
    if (wall && jh_wall != nullptr && k < g.nz - 1) {
        // constrained spline: the open harmonic current (-dH_y/dz, dH_x/dz)
        // on the side walls (nfgs_solver.py:5920-5933, 5406-5432)
        const int n = g.nz;
        const double dz = g.dz;
        double der[2];
        for (int c2 = 0; c2 < 2; ++c2) {
            const double* p = jh_wall + c2 * n;
            der[c2] = k == 0 ? (-3.0 * p[0] + 4.0 * p[1] - p[2]) / (2.0 * dz)
                             : 0.5 * ((p[k] - p[k - 1]) / dz + (p[k + 1] - p[k]) / dz);
        }
        jx = -der[1];
        jy = der[0];
    } else if (!wall) {
        if (k == 0) {
            jx = (double)jf[pq];
            jy = (double)jf[FV + pq];
        } else {
            // the storage-type average of the reference (0.5 * (a + b) in T)
            jx = (double)(T(0.5) * (jf[(long long)(k - 1) * P + pq] + jf[(long long)k * P + pq]));
            jy = (double)(T(0.5) * (jf[FV + (long long)(k - 1) * P + pq] + jf[FV + (long long)k * P + pq]));
        }
    }
    out[3 * n + q] = (O)jx;
    out[4 * n + q] = (O)jy;
    out[5 * n + q] = (O)jz[c];
}

// sum (B_a - B_b)^2 and sum B_b^2 with B = bg + carrier
template <typename T>
__global__ void k_diff_sums(const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ bg, long long n,
                            double* out) {
    __shared__ double sh[2 * 32];
    double v[2] = {0, 0};
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        double x = (double)(bg[q] + a[q]), y = (double)(bg[q] + b[q]);
        v[0] += (x - y) * (x - y);
        v[1] += y * y;
    }
    block_reduce<2>(v, sh);
    if (threadIdx.x == 0) { out[2 * blockIdx.x] = v[0]; out[2 * blockIdx.x + 1] = v[1]; }
}

static int resolve_state(Handle* h, int which, int* idx) {
    if (which == 0) {
        if (h->solution < 0) return fail(NFGS_ESTATE, "No solution stored; call iterate() first.");
        *idx = h->solution;
    } else {
        *idx = h->cur_host;
    }
    return NFGS_OK;
}

static void host_scalars(const Geo& g, const double* s, double out[3]) {
    out[0] = s[0] / std::max(s[1], 1e-30);
    double delta = std::min(g.dx, std::min(g.dy, g.dz));
    out[1] = (s[2] / (double)g.V) / (6.0 * (s[3] / (double)g.V) / delta + 1e-12);
    out[2] = s[4] * g.dx * g.dy * g.dz / 2.0;
}

template <typename T>
static int state_scalars(Handle* h, int idx, double out[3]) {
    TRY(run_stencil<T>(h, &h->consts[idx], nullptr, 0, 0));
    sum_partials(h);
    CK(cudaGetLastError());
    double sums[6];
    CK(cudaMemcpyAsync(sums, h->scal, 6 * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    host_scalars(h->g, sums, out);
    return NFGS_OK;
}

template <typename T>
static int iterate_end_t(Handle* h, NfgsIterResult* res, double* hist, int hist_rows) {
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    CK(cudaEventRecord(h->ev1, h->s));
    CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    const DevCtl& c = *h->ctl_h;
    NfgsIterResult r{};
    r.n_hist = c.n_hist;
    r.best_iter = c.best_iter;
    r.final_iter = c.final_iter;
    r.stop_reason = c.stop_reason;
    r.rollbacks = c.rollbacks;
    r.best_sigma = c.best_sigma;
    r.final_sigma = c.cur_sigma;
    r.sigma0 = c.sigma0;
    r.divB0 = c.divb0;
    r.energy0 = c.e0;
    r.last_sigma_improvement = c.have_last_imp ? c.last_imp : std::nan("");
    r.init_source_zero_mode_ratio = h->init_zr;
    r.device_ms = ms;
    if (hist && hist_rows > 0) {
        int n = std::min(hist_rows, c.n_hist);
        if (n > 0) CK(cudaMemcpy(hist, h->hist, (size_t)n * NFGS_HCOLS * 8, cudaMemcpyDeviceToHost));
    }
    h->iter_active = 0;
    h->solution = h->select_final ? c.cur : c.best;
    if (h->k0_on) {
        k_k0_select<<<1, 256, 0, h->s>>>(h->k0d.hk, h->solution, h->g.nz, h->k0_t[0], h->k0_t[1], h->k0d.hlast);
        CK(cudaGetLastError());
        h->launches++;
    }
    h->select_final = 0;
    h->cur_host = c.cur;
    // final-vs-best relative B difference (nfgs_solver.py:3820-3824)
    if (c.cur != c.best) {
        const long long V3 = 3 * h->g.V;
        if (!h->bscratch) TRY(alloc(h, &h->bscratch, V3 * h->esz));
        TRY(run_stencil<T>(h, &h->consts[c.best], nullptr, 0, 0));
        CK(cudaMemcpyAsync(h->bscratch, h->B, V3 * h->esz, cudaMemcpyDeviceToDevice, h->s));
        TRY(run_stencil<T>(h, &h->consts[c.cur], nullptr, 0, 0));
        // block partials over the whole device, summed on the host in block order
        constexpr int kFvbBlocks = 592;
        if (!h->fvb_part) TRY(alloc(h, &h->fvb_part, 2 * kFvbBlocks * sizeof(double)));
        k_diff_sums<T><<<kFvbBlocks, 256, 0, h->s>>>((const T*)h->B, (const T*)h->bscratch, (const T*)h->bbg, V3,
                                                     h->fvb_part);
        CK(cudaGetLastError());
        std::vector<double> part(2 * kFvbBlocks);
        CK(cudaMemcpyAsync(part.data(), h->fvb_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->s));
        CK(cudaStreamSynchronize(h->s));
        double sums[2] = {0.0, 0.0};
        for (int b = 0; b < kFvbBlocks; ++b) {
            sums[0] += part[2 * b];
            sums[1] += part[2 * b + 1];
        }
        r.final_vs_best_B_relative = std::sqrt(sums[0] / V3) / std::max(std::sqrt(sums[1] / V3), 1e-30);
        h->launches += 5;
    } else {
        r.final_vs_best_B_relative = 0.0;
    }
    r.kernel_launches = h->launches;
    if (res) *res = r;
    if (c.policy_error) {
        // the row that failed is the next step's source (nfgs_solver.py:5457-5476)
        char b[256];
        snprintf(b, sizeof b,
                 "The Phi_c nonlinear source has an incompatible zero mode ratio=%.6e exceeds tolerance=%.6e.",
                 c.zero_ratio_last, h->prm.source_zero_mode_tolerance);
        return fail(NFGS_EPOLICY, b);
    }
    return NFGS_OK;
}

// Host copy of one chunk on up to 8 threads (a fresh pageable destination
// costs a page fault per page; the threads take those in parallel).
// A persistent pool of host-copy workers (up to 16, one per hardware thread),
// created on first use: the copies of a chunk into a fresh destination take
// its page faults in parallel, and no thread is created per chunk.
class CopyPool {
public:
    // never destroyed: the workers wait on its condition variable until the
    // process ends
    static CopyPool& get() {
        static CopyPool* pool = new CopyPool();
        return *pool;
    }
    // copy len bytes in page-aligned slices, one per worker plus the caller
    void copy(char* dst, const char* src, size_t len) {
        const size_t parts = workers_.size() + 1;
        const size_t per = ((len + parts - 1) / parts + 4095) & ~(size_t)4095;
        if (workers_.empty() || len <= per) {
            std::memcpy(dst, src, len);
            return;
        }
        std::unique_lock<std::mutex> call(call_mu_);  // one copy at a time through the pool
        {
            std::lock_guard<std::mutex> lk(mu_);
            dst_ = dst; src_ = src; len_ = len; per_ = per;
            pending_ = (int)workers_.size();
            ++gen_;
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(per, len));
        std::unique_lock<std::mutex> lk(mu_);
        done_.wait(lk, [&] { return pending_ == 0; });
    }

private:
    CopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        const unsigned n = std::min(16u, hw > 1 ? hw : 1u) - 1;
        for (unsigned w = 0; w < n; ++w) workers_.emplace_back([this, w] { run(w + 1); });
        for (auto& t : workers_) t.detach();
    }
    void run(unsigned slot) {
        unsigned long long seen = 0;
        for (;;) {
            char* dst;
            const char* src;
            size_t len, per;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                dst = dst_; src = src_; len = len_; per = per_;
            }
            const size_t off = (size_t)slot * per;
            if (off < len) std::memcpy(dst + off, src + off, std::min(per, len - off));
            std::lock_guard<std::mutex> lk(mu_);
            if (--pending_ == 0) done_.notify_one();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex mu_, call_mu_;
    std::condition_variable cv_, done_;
    char* dst_ = nullptr;
    const char* src_ = nullptr;
    size_t len_ = 0, per_ = 0;
    int pending_ = 0;
    unsigned long long gen_ = 0;
};

static void host_copy(char* dst, const char* src, size_t len) { CopyPool::get().copy(dst, src, len); }

// Copy n bytes from device memory to pageable host memory through two pinned
// chunks: the DMA of chunk k overlaps the host copy of chunk k-1.
static int d2h_chunked(Handle* h, void* host, const void* dev, size_t n) {
    const size_t CH = PIN_CHUNK;
    // a page-locked destination takes the copy directly
    {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, host) == cudaSuccess && pa.type == cudaMemoryTypeHost) {
            CK(cudaMemcpyAsync(host, dev, n, cudaMemcpyDeviceToHost, h->s));
            CK(cudaStreamSynchronize(h->s));
            return NFGS_OK;
        }
        (void)cudaGetLastError();
    }
    // a fresh destination faults its pages in during the copy: ask for 2 MB
    // pages on the 2 MB-aligned part of it (advice only; ignored where the
    // memory is not anonymous or the kernel declines)
    {
        const uintptr_t lo = ((uintptr_t)host + (2u << 20) - 1) & ~(uintptr_t)((2u << 20) - 1);
        const uintptr_t hi = ((uintptr_t)host + n) & ~(uintptr_t)((2u << 20) - 1);
        if (hi > lo) (void)madvise((void*)lo, hi - lo, MADV_HUGEPAGE);
    }
    struct Pins {
        void* p[2] = {nullptr, nullptr};
        ~Pins() { pin_release(p[0]); pin_release(p[1]); }
    } pins;
    for (int q = 0; q < 2; ++q) {
        TRY(pin_acquire(&pins.p[q]));
        if (!h->pin_ev[q]) CK(cudaEventCreateWithFlags(&h->pin_ev[q], cudaEventDisableTiming));
    }
    void* const* pin = pins.p;
    const size_t nch = (n + CH - 1) / CH;
    for (size_t k = 0; k <= nch; ++k) {
        if (k < nch) {
            const size_t off = k * CH, len = std::min(CH, n - off);
            CK(cudaMemcpyAsync(pin[k & 1], (const char*)dev + off, len, cudaMemcpyDeviceToHost, h->s));
            CK(cudaEventRecord(h->pin_ev[k & 1], h->s));
        }
        if (k >= 1) {
            const size_t kp = k - 1, off = kp * CH, len = std::min(CH, n - off);
            CK(cudaEventSynchronize(h->pin_ev[kp & 1]));
            host_copy((char*)host + off, (const char*)pin[kp & 1], len);
        }
    }
    return NFGS_OK;
}

// Region of the exported fields: the observed field of view (crop) or the
// whole calculation grid.
static void export_region(const Handle* h, int crop, int* nzc, int* y0, int* nyc, int* x0, int* nxc) {
    *nzc = h->g.nz; *y0 = 0; *x0 = 0; *nyc = h->g.ny; *nxc = h->g.nx;
    if (crop) {
        *nzc = h->nzo_crop; *y0 = h->fov_y0; *x0 = h->fov_x0; *nyc = h->nyo; *nxc = h->nxo;
    }
}

// Reconstruct the state `which` and gather its six fields into dst (device).
template <typename T>
static int gather_t(Handle* h, int which, int crop, void* dst, int odtype) {
    int idx;
    TRY(resolve_state(h, which, &idx));
    TRY(run_stencil<T>(h, &h->consts[idx], nullptr, 0, 0, 1));
    int nzc, y0, nyc, x0, nxc;
    export_region(h, crop, &nzc, &y0, &nyc, &x0, &nxc);
    const long long n = (long long)nzc * nyc * nxc;
    const unsigned grid = (unsigned)((n + 255) / 256);
    if (odtype == NFGS_F32)
        k_gather_fields<T, float><<<grid, 256, 0, h->s>>>(h->g, (const T*)h->B, (const T*)h->bbg, (const T*)h->jz,
                                                          (const T*)h->jpf, nzc, y0, nyc, x0, nxc, (float*)dst,
                                                          h->k0_spline ? h->k0_hsel : nullptr);
    else
        k_gather_fields<T, double><<<grid, 256, 0, h->s>>>(h->g, (const T*)h->B, (const T*)h->bbg, (const T*)h->jz,
                                                           (const T*)h->jpf, nzc, y0, nyc, x0, nxc, (double*)dst,
                                                          h->k0_spline ? h->k0_hsel : nullptr);
    CK(cudaGetLastError());
    return NFGS_OK;
}

template <typename T>
static int fields_t(Handle* h, int which, int crop, void* out, int odtype, int32_t* dims) {
    int nzc, y0, nyc, x0, nxc;
    export_region(h, crop, &nzc, &y0, &nyc, &x0, &nxc);
    const long long n = (long long)nzc * nyc * nxc;
    const size_t osz = odtype == NFGS_F32 ? 4 : 8;
    const size_t bytes = 6 * (size_t)n * osz;
    if (bytes > h->fbuf_bytes) {
        if (h->fbuf) {
            for (auto it = h->owned.begin(); it != h->owned.end();) {
                if (it->p == h->fbuf) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
            }
            h->fbuf = nullptr;
            h->fbuf_bytes = 0;
        }
        TRY(alloc(h, &h->fbuf, bytes));
        h->fbuf_bytes = bytes;
    }
    TRY(gather_t<T>(h, which, crop, h->fbuf, odtype));
    TRY(d2h_chunked(h, out, h->fbuf, bytes));
    if (dims) { dims[0] = nzc; dims[1] = nyc; dims[2] = nxc; }
    return NFGS_OK;
}

template <typename T>
static int fields_device_t(Handle* h, int which, int crop, void* out_dev, int odtype, int32_t* dims) {
    int nzc, y0, nyc, x0, nxc;
    export_region(h, crop, &nzc, &y0, &nyc, &x0, &nxc);
    if (dims) { dims[0] = nzc; dims[1] = nyc; dims[2] = nxc; }
    if (!out_dev) return NFGS_OK;
    TRY(gather_t<T>(h, which, crop, out_dev, odtype));
    CK(cudaStreamSynchronize(h->s));
    return NFGS_OK;
}

// Metrics of one region (nfgs_metrics.cuh); out gets NFGS_MET_COUNT values.
template <typename T>
static int field_metrics_t(const met::Args& a, cudaStream_t s, double* out) {
    int dev = 0, nsm = 148;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const long long cells = (long long)a.cz * a.cy * a.cx;
    const int gx = (a.cx + 31) / 32, gy = (a.cy + met::NT / 32 - 1) / (met::NT / 32);
    const long long gxy = (long long)gx * gy;
    const int gz = (int)std::max<long long>(1, std::min<long long>(a.cz, ((long long)nsm * 8 + gxy - 1) / gxy));
    if (gy > 65535) return fail(NFGS_EINVAL, "field metrics: region too tall");
    const int nblocks = (int)(gxy * gz);
    double* part = nullptr;
    CK(cudaMallocAsync((void**)&part, ((size_t)nblocks + 1) * met::NS * sizeof(double), s));
    const dim3 grid((unsigned)gx, (unsigned)gy, (unsigned)gz);
    if (a.ref && a.cur) met::k_metrics<T, true, true><<<grid, met::NT, 0, s>>>(a, part);
    else if (a.ref) met::k_metrics<T, true, false><<<grid, met::NT, 0, s>>>(a, part);
    else if (a.cur) met::k_metrics<T, false, true><<<grid, met::NT, 0, s>>>(a, part);
    else met::k_metrics<T, false, false><<<grid, met::NT, 0, s>>>(a, part);
    cudaError_t e = cudaGetLastError();
    double sums[met::NS];
    if (e == cudaSuccess) {
        met::k_metrics_sum<<<1, 32 * met::NS, 0, s>>>(part, nblocks, part + (size_t)nblocks * met::NS);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(sums, part + (size_t)nblocks * met::NS, sizeof(sums), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(part, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("field metrics: ") + cudaGetErrorString(e));
    using namespace met;
    const double nan = std::nan("");
    const double cnt = (double)cells, cm = std::max(cnt, 1.0);
    for (int q = 0; q < NFGS_MET_COUNT; ++q) out[q] = nan;
    if (a.ref) {
        out[NFGS_MET_C_VEC] = sums[S_DOT] / (std::sqrt(sums[S_REF2] * sums[S_SOL2]) + 1.0e-12);
        out[NFGS_MET_C_CS] = sums[S_COS] / cm;
        out[NFGS_MET_EPRIME_N] = 1.0 - sums[S_ERR] / (sums[S_REFN] + 1.0e-12);
        out[NFGS_MET_EPRIME_M] = 1.0 - sums[S_ERRR] / cm;
        out[NFGS_MET_EPSILON] = sums[S_SOL2] / (sums[S_REF2] + 1.0e-12);
        out[NFGS_MET_SUM_REF2] = sums[S_REF2];
    }
    if (a.cur) {
        out[NFGS_MET_SIGMA_J] = sums[S_SJN] / std::max(sums[S_SJD], 1.0e-30);
        out[NFGS_MET_NONFINITE_J] = sums[S_NFJ];
    }
    out[NFGS_MET_SIGMA_J_FD2] = sums[S_FDN] / std::max(sums[S_FDD], 1.0e-30);
    const double h_eff = 3.0 / (1.0 / a.dx + 1.0 / a.dy + 1.0 / a.dz);
    out[NFGS_MET_DIVB_NORM] = (sums[S_DIV] / cm) / (6.0 * (sums[S_BN] / cm) / h_eff + 1.0e-12);
    out[NFGS_MET_CELLS] = cnt;
    out[NFGS_MET_SUM_B2] = sums[S_SOL2];
    out[NFGS_MET_NONFINITE_B] = sums[S_NFB];
    return NFGS_OK;
}

template <typename T>
static int get_state_t(Handle* h, int which, double* phi, double* az, double* sc) {
    int idx;
    TRY(resolve_state(h, which, &idx));
    const long long V = h->g.V;
    if (!h->dscratch) TRY(alloc(h, &h->dscratch, V * 8));
    if (phi) {
        TRY(from_storage(h, h->st.phi[idx], h->dscratch, V));
        CK(cudaMemcpyAsync(phi, h->dscratch, V * 8, cudaMemcpyDeviceToHost, h->s));
    }
    if (az) {
        CK(cudaStreamSynchronize(h->s));
        TRY(from_storage(h, h->st.az[idx], h->dscratch, V));
        CK(cudaMemcpyAsync(az, h->dscratch, V * 8, cudaMemcpyDeviceToHost, h->s));
    }
    CK(cudaStreamSynchronize(h->s));
    if (sc) TRY(state_scalars<T>(h, idx, sc));
    return NFGS_OK;
}

template <typename T>
static int step_t(Handle* h, double mu, int polarity) {
    if (!h->boundary_set) return fail(NFGS_ESTATE, "NFGS boundary is not configured");
    const int cur = h->cur_host;
    const int cand = (cur + 1) % 3 == h->solution ? (cur + 2) % 3 : (cur + 1) % 3;
    TRY(run_stencil<T>(h, &h->consts[cur], nullptr, 1, polarity));
    TRY(run_solve<T>(h, nullptr, &h->consts[cand], 0));
    TRY(finalize_candidate<T>(h, nullptr, 0, mu, &h->consts[cand], &h->consts[cur]));
    CK(cudaStreamSynchronize(h->s));
    h->cur_host = cand;
    return NFGS_OK;
}

// B^> on z = 0 (nfgs_solver.py:4921-4946) and the harmonic-style gradient.
static int gaussian_above_impl(Handle* h, double* out) {
    if (!h->boundary_set) return fail(NFGS_ESTATE, "NFGS Gaussian separation is not configured");
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nxi = nx - 2, nyi = ny - 2;
    const long long P = g.P;
    cudaStream_t s = h->s;
    double* w;
    TRY(alloc(h, &w, 6 * P * 8));
    CK(cudaMemsetAsync(w, 0, 6 * P * 8, s));
    double *t1 = w, *t2 = w + P, *gx = w + 2 * P, *gy = w + 3 * P, *dph = w + 4 * P;
    double *kN = h->kN, *pah = h->phi_above_hat, *alx = h->alx, *aly = h->aly;
    double dx = g.dx, dy = g.dy;
    CK(launch_map(P, s, [=] __device__(long long q) { dph[q] = kN[q] * pah[q]; }));
    if (h->prm.gaussian_spectral) {
        CK(launch_map(P, s, [=] __device__(long long q) { t1[q] = -alx[q % nx] * dph[q]; }));
        TRY(apply_y<double>(h, h->idcty, t1, nx, P, t2, nx, P, ny, ny, nx, 1));
        TRY(apply_x<double>(h, h->idstx, t2 + 1, nx, P, gx + 1, nx, P, ny, nxi, nxi, 1));
        CK(launch_map(P, s, [=] __device__(long long q) { t1[q] = -aly[q / nx] * dph[q]; }));
        TRY(apply_x<double>(h, h->idctx, t1, nx, P, t2, nx, P, ny, nx, nx, 1));
        TRY(apply_y<double>(h, h->idsty, t2 + nx, nx, P, gy + nx, nx, P, nyi, nyi, nx, 1));
    } else {
        TRY(idct2_d(h, dph, t1, t2));
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            gx[q] = d2d(t1, nx, ny, j, i, 0, dx);
            gy[q] = d2d(t1, nx, ny, j, i, 1, dy);
        }));
    }
    std::vector<double> a = d2h(h, gx, P), b = d2h(h, gy, P), c = d2h(h, h->bz_above, P);
    for (long long q = 0; q < P; ++q) {
        out[q] = -a[q];
        out[P + q] = -b[q];
        out[2 * P + q] = c[q];
    }
    for (auto it = h->owned.begin(); it != h->owned.end();) {
        if (it->p == w) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
    }
    return NFGS_OK;
}

// Post-solve source diagnostics (nfgs_solver.py:7014-7100, scalar keys).
template <typename T>
static int source_diag_t(Handle* h, double* out) {
    int idx;
    TRY(resolve_state(h, 0, &idx));
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V;
    cudaStream_t s = h->s;
    TRY(run_stencil<T>(h, &h->consts[idx], nullptr, 0, 0));
    double* w;
    const int NW = 29;
    TRY(alloc(h, &w, NW * P * 8));
    CK(cudaMemsetAsync(w, 0, NW * P * 8, s));
    // plane map: bc 0..5, bx0 6, by0 7, hat 8..13, dct scratch 14..19,
    // rob 20, prob 21, upw 22, ph1 23, ph2 24, sp 25, sp2 26, o 27, scratch 28
    double* bc = w;  // Bc_z = B_z - B_bg,z on planes 0,1,2 and nz-3, nz-2, nz-1
    const T* Bt = (const T*)h->B;
    const T* bgt = (const T*)h->bbg;
    CK(launch_map(6 * P, s, [=] __device__(long long q) {
        int p = (int)(q / P);
        long long m = q % P;
        int k = p < 3 ? p : nz - 6 + p;
        bc[q] = (double)Bt[2 * V + (long long)k * P + m];  // carrier = B_z - B_bg,z
    }));
    double *bx0 = w + 6 * P, *by0 = w + 7 * P;
    CK(launch_map(P, s, [=] __device__(long long q) {
        bx0[q] = (double)(bgt[q] + Bt[q]);
        by0[q] = (double)(bgt[V + q] + Bt[V + q]);
    }));
    double* hat = w + 8 * P;
    TRY(dct2_d(h, bc, hat, w + 14 * P, 6));
    double* lamN = h->lamN;
    double* kN = h->kN;
    const double dz = g.dz;
    double *rob = w + 20 * P, *prob = w + 21 * P, *upw = w + 22 * P, *ph1 = w + 23 * P, *ph2 = w + 24 * P;
    double *sp = w + 25 * P, *sp2 = w + 26 * P, *o = w + 27 * P, *scr = w + 28 * P;
    CK(launch_map(P, s, [=] __device__(long long q) {
        double h3 = hat[3 * P + q], h4 = hat[4 * P + q], h5 = hat[5 * P + q];
        double der = (3.0 * h5 - 4.0 * h4 + h3) / (2.0 * dz);
        double ls = q == 0 ? 1.0 : lamN[q];
        double p3 = q == 0 ? 0.0 : h3 / ls, p4 = q == 0 ? 0.0 : h4 / ls, p5 = q == 0 ? 0.0 : h5 / ls;
        double pder = (3.0 * p5 - 4.0 * p4 + p3) / (2.0 * dz);
        double ks = q == 0 ? 1.0 : kN[q];
        rob[q] = q == 0 ? 0.0 : der + kN[q] * h5;
        prob[q] = q == 0 ? 0.0 : pder + kN[q] * p5;
        upw[q] = q == 0 ? 0.0 : 0.5 * (h5 + der / ks);
        ph1[q] = q == 0 ? 0.0 : hat[P + q] / ls;   // Neumann solves of planes 1, 2
        ph2[q] = q == 0 ? 0.0 : hat[2 * P + q] / ls;
    }));
    double res[NFGS_NSRCDIAG];
    for (int q = 0; q < NFGS_NSRCDIAG; ++q) res[q] = 0.0;
    int rc = 0;
    double r[4];
    {
        double *bza = h->bz_above, *bzo = h->bz_obs, *bbgd = h->bbg_d;
        CK(launch_map(P, s, [=] __device__(long long q) { sp[q] = bbgd[2 * V + q] + bza[q] - bzo[q]; }));
        TRY(reduce4(h, sp, P, r));
        res[0] = std::sqrt(r[1] / P);
        res[1] = r[3];
        CK(launch_map(P, s, [=] __device__(long long q) { sp[q] = bc[q] - bza[q]; }));
        res[2] = rms_of(h, sp, P, &rc); TRY(rc);
    }
    TRY(idct2_d(h, rob, sp, scr)); res[3] = rms_of(h, sp, P, &rc); TRY(rc);
    TRY(idct2_d(h, prob, sp, scr)); res[4] = rms_of(h, sp, P, &rc); TRY(rc);
    TRY(idct2_d(h, upw, sp, scr));
    double up_rms = rms_of(h, sp, P, &rc); TRY(rc);
    double top_rms = rms_of(h, bc + 5 * P, P, &rc); TRY(rc);
    res[5] = up_rms;
    res[6] = up_rms / std::max(top_rms, 1e-30);
    {
        double* d0 = h->d0;
        double dx = g.dx, dy = g.dy;
        CK(launch_map(P, s, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            sp[q] = d2d(bx0, nx, ny, j, i, 0, dx) + d2d(by0, nx, ny, j, i, 1, dy) - d0[q];
        }));
        double er = rms_of(h, sp, P, &rc); TRY(rc);
        double ds = rms_of(h, d0, P, &rc); TRY(rc);
        res[9] = er;
        res[10] = er / std::max(ds, 1e-30);
    }
    {
        TRY(idct2_d(h, ph1, sp, scr));
        TRY(idct2_d(h, ph2, sp2, scr));
        double *pab = h->phi_above, *tg = h->dphi_tgt;
        CK(launch_map(P, s, [=] __device__(long long q) {
            double d = (-3.0 * pab[q] + 4.0 * sp[q] - sp2[q]) / (2.0 * dz);
            o[q] = d - tg[q];
        }));
        res[11] = rms_of(h, o, P, &rc); TRY(rc);
    }
    std::memcpy(out, res, sizeof res);
    for (auto it = h->owned.begin(); it != h->owned.end();) {
        if (it->p == w) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
    }
    return NFGS_OK;
}

template <typename T>
static int time_phases_t(Handle* h, int n_iters, double* ms_out) {
    if (!h->boundary_set) return fail(NFGS_ESTATE, "boundary is not set");
    if (h->k0_on) return fail(NFGS_EUNSUPPORTED, "phase timing covers the frozen and omitted k_h=0 policies only");
    cudaEvent_t ev[6];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    double acc[5] = {0, 0, 0, 0, 0};
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, PI = h->PI;
    const int nxi = nx - 2, nyi = ny - 2;
    for (int it = 0; it < n_iters; ++it) {
        const int cur = h->cur_host;
        const int cand = (cur + 1) % 3 == h->solution ? (cur + 2) % 3 : (cur + 1) % 3;
        CK(cudaEventRecord(ev[0], h->s));
        TRY(run_stencil<T>(h, &h->consts[cur], nullptr, 1, 0));
        sum_partials(h);
        CK(cudaEventRecord(ev[1], h->s));
        TRY(forward_transforms<T>(h, nullptr));
        CK(cudaEventRecord(ev[2], h->s));
        TRY(zsolve_launch<T>(h, nullptr));
        CK(cudaEventRecord(ev[3], h->s));
        TRY(inverse_transforms<T>(h, nullptr, &h->consts[cand]));
        CK(cudaEventRecord(ev[4], h->s));
        k_finalize<T><<<(unsigned)((P + 255) / 256), 256, 0, h->s>>>(h->g, h->st, nullptr, 0, 1.0, &h->consts[cand],
                                                                    &h->consts[cur], (const T*)h->phiab_t,
                                                                    (const T*)h->dphi_t, h->prm.projection_weight, 1, 1, (const T*)h->azb_t);
        CK(cudaGetLastError());
        CK(cudaEventRecord(ev[5], h->s));
        CK(cudaEventSynchronize(ev[5]));
        for (int q = 0; q < 5; ++q) {
            float ms = 0.0f;
            CK(cudaEventElapsedTime(&ms, ev[q], ev[q + 1]));
            acc[q] += ms;
        }
        h->cur_host = cand;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    for (int q = 0; q < 5; ++q) ms_out[q] = acc[q];
    return NFGS_OK;
}

template <typename T>
static int apply_transform_t(Handle* h, int chain, int inverse, const double* in, double* out) {
    const Geo& g = h->g;
    const long long P = g.P, PI = h->PI, V = g.V;
    const long long n = chain == 0 ? V : (long long)g.nz * PI;
    if (!h->dscratch) TRY(alloc(h, &h->dscratch, V * 8));
    CK(cudaMemcpyAsync(h->dscratch, in, n * 8, cudaMemcpyHostToDevice, h->s));
    CK(cudaMemsetAsync(h->sb, 0, V * h->esz, h->s));
    CK(cudaMemsetAsync(h->sj, 0, (size_t)g.nz * PI * h->esz, h->s));
    TRY(to_storage(h, h->dscratch, chain == 0 ? h->sb : h->sj, n));
    const int* sel = &h->consts[2];
    if (!inverse) {
        TRY(forward_transforms<T>(h, nullptr));
        TRY(from_storage(h, chain == 0 ? h->sb : h->sj, h->dscratch, n));
    } else {
        CK(cudaMemsetAsync(h->st.phi[2], 0, V * h->esz, h->s));
        CK(cudaMemsetAsync(h->st.az[2], 0, V * h->esz, h->s));
        TRY(inverse_transforms<T>(h, nullptr, sel));
        if (chain == 0) {
            TRY(from_storage(h, h->st.phi[2], h->dscratch, V));
        } else {
            // interior of az[2] back to the compact (nz, ny-2, nx-2) layout
            TRY(from_storage(h, h->st.az[2], h->dscratch, V));
            double* tmp;
            TRY(alloc(h, &tmp, n * 8));
            const int nx = g.nx, nxi = g.nx - 2, nyi = g.ny - 2;
            double* src = h->dscratch;
            CK(launch_map(n, h->s, [=] __device__(long long q) {
                long long k = q / PI, r = q % PI, j = r / nxi, i = r % nxi;
                tmp[q] = src[k * P + (j + 1) * nx + (i + 1)];
            }));
            CK(cudaMemcpyAsync(out, tmp, n * 8, cudaMemcpyDeviceToHost, h->s));
            CK(cudaStreamSynchronize(h->s));
            for (auto it = h->owned.begin(); it != h->owned.end();) {
                if (it->p == tmp) { cudaFreeAsync(it->p, h->s); it = h->owned.erase(it); } else ++it;
            }
            return NFGS_OK;
        }
    }
    CK(cudaMemcpyAsync(out, h->dscratch, n * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    int err = 0;
    if (h->tc_err) {
        CK(cudaMemcpy(&err, h->tc_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return fail(NFGS_ETIMEDOUT, "tensor-core transform wait ran out");
    }
    return NFGS_OK;
}

static int create_impl(const NfgsGeom* geom, const NfgsParams* prm, void** out) {
    if (!geom || !prm || !out) return fail(NFGS_EINVAL, "null argument");
    if (geom->nx < 3 || geom->ny < 3) return fail(NFGS_EINVAL, "NFGS requires a calculation grid with Nx, Ny >= 3");
    if (geom->nz < 3) return fail(NFGS_EINVAL, "NFGS requires Nz >= 3");
    if (geom->dtype != NFGS_F32 && geom->dtype != NFGS_F64) return fail(NFGS_EINVAL, "dtype must be F32 or F64");
    if (!(geom->dx > 0) || !(geom->dy > 0) || !(geom->dz > 0)) return fail(NFGS_EINVAL, "grid spacing must be positive");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(NFGS_ECUDA, "no CUDA device: the NFGS B200 library has no CPU path");
    if (geom->device < 0 || geom->device >= ndev) return fail(NFGS_EINVAL, "device ordinal out of range");
    if (cudaSetDevice(geom->device) != cudaSuccess) return fail(NFGS_ECUDA, "cudaSetDevice failed");
    Handle* h = new Handle();
    h->geom = *geom;
    h->prm = *prm;
    h->f32 = geom->dtype == NFGS_F32;
    h->esz = h->f32 ? 4 : 8;
    Geo& g = h->g;
    g.nx = geom->nx; g.ny = geom->ny; g.nz = geom->nz;
    g.P = (long long)g.nx * g.ny;
    g.V = g.P * g.nz;
    g.dx = geom->dx; g.dy = geom->dy; g.dz = geom->dz;
    h->PI = (long long)(g.nx - 2) * (g.ny - 2);
    // counted alive from here, so that a concurrent nfgs_release_cached_memory
    // keeps the shared matrices this solver is about to take
    {
        std::lock_guard<std::mutex> lk(g_dmat_mu);
        ++g_live_handles[geom->device];
    }
    auto bail = [&](int r) {
        free_all(h);
        {
            std::lock_guard<std::mutex> lk(g_dmat_mu);
            --g_live_handles[geom->device];
        }
        delete h;
        return r;
    };
#define TRYC(call) do { int r_ = (call); if (r_ != NFGS_OK) return bail(r_); } while (0)
#define CKC(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) { fail(NFGS_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); return bail(NFGS_ECUDA); } } while (0)
    CKC(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
    CKC(cudaEventCreate(&h->ev0));
    CKC(cudaEventCreate(&h->ev1));
    CKC(cudaEventCreateWithFlags(&h->ev_na_in, cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&h->ev_na_out, cudaEventDisableTiming));
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const long long P = g.P, V = g.V, PI = h->PI;
    // transforms
    {
        const int dv = h->geom.device;
        struct M { double** d64; void** dt; int kind, n; bool inv; };
        const M ms[8] = {{&h->dctx, &h->dctx_t, 0, nx, false}, {&h->idctx, &h->idctx_t, 0, nx, true},
                         {&h->dcty, &h->dcty_t, 0, ny, false}, {&h->idcty, &h->idcty_t, 0, ny, true},
                         {&h->dstx, &h->dstx_t, 1, nx - 2, false}, {&h->idstx, &h->idstx_t, 1, nx - 2, true},
                         {&h->dsty, &h->dsty_t, 1, ny - 2, false}, {&h->idsty, &h->idsty_t, 1, ny - 2, true}};
        for (const M& m : ms) {
            void* q = nullptr;
            TRYC(shared_matrix(dv, m.kind, m.n, m.inv, 8, &q));
            *m.d64 = (double*)q;
            TRYC(shared_matrix(dv, m.kind, m.n, m.inv, h->esz, m.dt));
        }
    }
    // eigenvalues (nfgs_solver.py:1083-1118, 4357-4383, 4811)
    {
        std::vector<double> lx(nx), ly(ny), ax(nx), ay(ny), ln(P), kn(P), lns(P), ld(PI);
        for (int i = 0; i < nx; ++i) {
            double sn = std::sin(M_PI * i / (2.0 * std::max(nx - 1, 1)));
            lx[i] = -4.0 * sn * sn / (g.dx * g.dx);
            ax[i] = 2.0 * sn / g.dx;
        }
        for (int j = 0; j < ny; ++j) {
            double sn = std::sin(M_PI * j / (2.0 * std::max(ny - 1, 1)));
            ly[j] = -4.0 * sn * sn / (g.dy * g.dy);
            ay[j] = 2.0 * sn / g.dy;
        }
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                double l = ly[j] + lx[i];
                ln[(size_t)j * nx + i] = l;
                kn[(size_t)j * nx + i] = std::sqrt(std::max(-l, 0.0));
                lns[(size_t)j * nx + i] = (i == 0 && j == 0) ? 1.0 : l;
            }
        for (int j = 0; j < ny - 2; ++j)
            for (int i = 0; i < nx - 2; ++i) {
                double sx = std::sin(M_PI * (i + 1) / (2.0 * (nx - 1)));
                double sy = std::sin(M_PI * (j + 1) / (2.0 * (ny - 1)));
                ld[(size_t)j * (nx - 2) + i] = -4.0 * sx * sx / (g.dx * g.dx) + -4.0 * sy * sy / (g.dy * g.dy);
            }
        TRYC(upload(h, &h->lamN, ln)); TRYC(upload(h, &h->kN, kn)); TRYC(upload(h, &h->lamNs, lns));
        TRYC(upload(h, &h->lamD, ld)); TRYC(upload(h, &h->alx, ax)); TRYC(upload(h, &h->aly, ay));
    }
    // factor tables
    TRYC(alloc(h, &h->zr_c, (size_t)nz * P * 8)); TRYC(alloc(h, &h->zr_i, (size_t)nz * P * 8));
    TRYC(alloc(h, &h->zr_il, P * 8)); TRYC(alloc(h, &h->zr_ci, P * 8)); TRYC(alloc(h, &h->zr_ii, P * 8));
    TRYC(alloc(h, &h->zr_rc, P * 4));
    TRYC(alloc(h, &h->zd_c, (size_t)nz * PI * 8)); TRYC(alloc(h, &h->zd_i, (size_t)nz * PI * 8));
    TRYC(alloc(h, &h->zd_il, PI * 8)); TRYC(alloc(h, &h->zd_ci, PI * 8)); TRYC(alloc(h, &h->zd_ii, PI * 8));
    TRYC(alloc(h, &h->zd_rc, PI * 4));
    // boundary planes
    double** planes[] = {&h->bz_obs, &h->bx_obs, &h->by_obs, &h->jz_obs, &h->az_bot, &h->jz_t,
                         &h->phi_above, &h->bz_above, &h->d0, &h->dphi_tgt, &h->phi_above_hat,
                         &h->phi_below_hat, &h->phi_bot_hat, &h->der_hat, &h->jz_stable};
    for (auto pp : planes) { TRYC(alloc(h, pp, P * 8)); CKC(cudaMemset(*pp, 0, P * 8)); }
    TRYC(alloc(h, &h->az_bot_hat, PI * 8));
    TRYC(alloc(h, &h->bbg_d, 3 * V * 8));
    TRYC(alloc(h, &h->bbg, 3 * V * h->esz));
    TRYC(alloc(h, &h->bzobs_t, P * h->esz)); TRYC(alloc(h, &h->jzt_t, P * h->esz));
    TRYC(alloc(h, &h->phiab_t, P * h->esz)); TRYC(alloc(h, &h->dphi_t, P * h->esz));
    TRYC(alloc(h, &h->azb_t, P * h->esz));
    // buffer window (nfgs_solver.py:1569-1591)
    std::vector<double> k0_wfac(nz, 1.0);
    if (prm->buffer_thickness > 0) {
        const int t = prm->buffer_thickness;
        auto bell = [&](int n) {
            std::vector<double> w(n);
            int tt = std::min(t, std::max(1, (n - 1) / 2));
            for (int q = 0; q < n; ++q) {
                int d = std::min(q, n - 1 - q);
                w[q] = d >= tt ? 1.0 : 0.5 * (1.0 - std::cos(M_PI * d / (double)tt));
            }
            return w;
        };
        std::vector<double> wz(nz, 1.0);
        const std::vector<double> bx_w = bell(nx), by_w = bell(ny);
        if (!prm->buffer_xy_only) {
            int tz = std::min(t, std::max(1, nz - 1));
            for (int k = 0; k < nz; ++k) {
                int d = nz - 1 - k;
                wz[k] = d >= tz ? 1.0 : 0.5 * (1.0 - std::cos(M_PI * d / (double)tz));
            }
            wz[0] = 1.0;
        }
        TRYC(upload_t(h, &h->wx, bx_w));
        TRYC(upload_t(h, &h->wy, by_w));
        TRYC(upload_t(h, &h->wz, wz));
        // DCT-I zero mode of the window on each plane (the face-placed k_h=0
        // target is a uniform plane times the window, nfgs_solver.py:6718-6724)
        double sx = 0.0, sy = 0.0;
        for (int i = 0; i < nx; ++i) sx += (i == 0 || i == nx - 1 ? 1.0 : 2.0) * bx_w[i];
        for (int j = 0; j < ny; ++j) sy += (j == 0 || j == ny - 1 ? 1.0 : 2.0) * by_w[j];
        for (int k = 0; k < nz; ++k) k0_wfac[k] = wz[k] * sx * sy / (4.0 * (nx - 1) * (double)(ny - 1));
    }
    // state and work buffers
    for (int b = 0; b < 3; ++b) {
        TRYC(alloc(h, &h->st.phi[b], V * h->esz));
        TRYC(alloc(h, &h->st.az[b], V * h->esz));
        CKC(cudaMemset(h->st.phi[b], 0, V * h->esz));
        CKC(cudaMemset(h->st.az[b], 0, V * h->esz));
    }
    TRYC(alloc(h, &h->st_dev, sizeof(StateTab)));
    CKC(cudaMemcpy(h->st_dev, &h->st, sizeof(StateTab), cudaMemcpyHostToDevice));
    TRYC(alloc(h, &h->B, 3 * V * h->esz));
    TRYC(alloc(h, &h->jz, V * h->esz));
    TRYC(alloc(h, &h->jpf, 3 * (size_t)(nz - 1) * P * h->esz));
    TRYC(alloc(h, &h->jb, 2 * P * h->esz));
    TRYC(alloc(h, &h->sb, V * h->esz));
    TRYC(alloc(h, &h->sj, (size_t)nz * PI * h->esz));
    TRYC(alloc(h, &h->tmpA, V * h->esz));
    TRYC(alloc(h, &h->tmpB, (size_t)nz * PI * h->esz));
    CKC(cudaMemset(h->sj, 0, (size_t)nz * PI * h->esz));
    CKC(cudaMemset(h->jpf, 0, 3 * (size_t)(nz - 1) * P * h->esz));
    h->sblock = dim3(32, 4, 1);
    h->sgrid = dim3((nx + 31) / 32, (ny + 3) / 4, nz);
    h->nb_face = h->nb_src = (int)(h->sgrid.x * h->sgrid.y * h->sgrid.z);
    TRYC(fs_setup(h));
    if (prm->horizontal_zero_mode == NFGS_HZM_COUPLED_K0 || prm->horizontal_zero_mode == NFGS_HZM_CONSTRAINED_SPLINE)
        TRYC(k0_setup(h, k0_wfac));
    {
        // room for the tuner's largest candidate (16 z segments)
        const long long fs_max = (long long)h->fs_grid.x * h->fs_grid.y * std::max(16u, h->fs_grid.z) * NFGS_NRED;
        h->pface_len = std::max((long long)h->nb_face * 5, fs_max);
        TRYC(alloc(h, &h->pface, (size_t)h->pface_len * 8));
    }
    TRYC(alloc(h, &h->psrc, (size_t)h->nb_src * 8));
    TRYC(alloc(h, &h->s00, (size_t)nz * 8));
    TRYC(alloc(h, &h->scal, (8 + 6 * NCHUNK) * 8));
    TRYC(alloc(h, &h->ctl, sizeof(DevCtl)));
    TRYC(ctl_mirror_acquire(&h->ctl_h));
    std::memset(h->ctl_h, 0, sizeof(DevCtl));
    TRYC(alloc(h, &h->consts, 4 * sizeof(int)));
    {
        int cs[4] = {0, 1, 2, 0};
        CKC(cudaMemcpy(h->consts, cs, sizeof cs, cudaMemcpyHostToDevice));
    }
    TRYC(tc_setup(h));
#undef TRYC
#undef CKC
    *out = h;
    return NFGS_OK;
}

}  // namespace

// ===========================================================================
// Allocation-free B^> (variant of gaussian_above_impl)
//
// Callers that cannot allocate device memory at run time use this path:
// host programs whose own pool allocator already holds the free HBM (a
// fresh cudaMalloc from inside this library would fail or fragment it),
// and programs sharing the GPU with latency-critical streams (cudaMalloc and
// cudaFree synchronise the whole device).  The scratch planes live in one
// file-scope device array, reserved on every GPU that loads this library
// until the process exits.
// ===========================================================================
namespace {

// 2^21 doubles = 16 MiB; five scratch planes -> at most 419,430 cells per
// calculation-grid plane (e.g. 646 x 646).
constexpr long long kNoAllocScratchDoubles = 1LL << 21;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of the scratch array on the current device.  The array's
// name is only a host-side stand-in; the address is looked up on every call
// (cheap once the module is loaded), so a device or primary-context reset
// between calls leaves no stale pointer behind.
static int noalloc_scratch(double** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
        return fail(NFGS_ECUDA, std::string("cudaGetSymbolAddress(scratch) failed: ") + cudaGetErrorString(e));
    *out = (double*)p;
    return NFGS_OK;
}

// out(r, c) = sum_m M[c][m] in(r, m), rows of pitch `pitch`, on `st`
static int noalloc_gemm_x(cudaStream_t st, const double* M, const double* in, double* out, long long pitch, int rows,
                          int K, int N) {
    GemmArgs a{};
    a.A = in; a.a_rs = pitch; a.a_cs = 1; a.a_bs = 0;
    a.B = M; a.b_rs = 1; a.b_cs = K; a.b_bs = 0;
    a.C = out; a.c_rs = pitch; a.c_cs = 1; a.c_bs = 0;
    a.M = rows; a.N = N; a.K = K; a.batch = 1;
    CK(launch_gemm<double>(a, st));
    return NFGS_OK;
}

// out(r, c) = sum_m M[r][m] in(m, c), on `st`
static int noalloc_gemm_y(cudaStream_t st, const double* M, const double* in, double* out, long long pitch, int K,
                          int N, int cols) {
    GemmArgs a{};
    a.A = M; a.a_rs = K; a.a_cs = 1; a.a_bs = 0;
    a.B = in; a.b_rs = pitch; a.b_cs = 1; a.b_bs = 0;
    a.C = out; a.c_rs = pitch; a.c_cs = 1; a.c_bs = 0;
    a.M = N; a.N = cols; a.K = K; a.batch = 1;
    CK(launch_gemm<double>(a, st));
    return NFGS_OK;
}

static int gaussian_above_noalloc_impl(Handle* h, double* out, cudaStream_t st) {
    const Geo& g = h->g;
    const int nx = g.nx, ny = g.ny, nxi = nx - 2, nyi = ny - 2;
    const long long P = g.P;
    if (5 * P > kNoAllocScratchDoubles) {
        char b[200];
        snprintf(b, sizeof b,
                 "calculation plane of %lld cells exceeds the static scratch limit of %lld cells per plane",
                 P, kNoAllocScratchDoubles / 5);
        return fail(NFGS_EINVAL, b);
    }
    if (!h->boundary_set) return fail(NFGS_ESTATE, "NFGS Gaussian separation is not configured");
    double* w = nullptr;
    TRY(noalloc_scratch(&w));
    // follow the handle's own queued work (boundary set-up writes the planes
    // read here)
    CK(cudaEventRecord(h->ev_na_in, h->s));
    CK(cudaStreamWaitEvent(st, h->ev_na_in, 0));
    double *t1 = w, *t2 = w + P, *gx = w + 2 * P, *gy = w + 3 * P, *dph = w + 4 * P;
    double *kN = h->kN, *pah = h->phi_above_hat, *alx = h->alx, *aly = h->aly, *bza = h->bz_above;
    const double dx = g.dx, dy = g.dy;
    // the scratch keeps the previous call's data; the gradient borders are
    // never written by the transforms and must start at zero
    CK(cudaMemsetAsync(gx, 0, 2 * P * sizeof(double), st));
    CK(launch_map(P, st, [=] __device__(long long q) { dph[q] = kN[q] * pah[q]; }));
    if (h->prm.gaussian_spectral) {
        CK(launch_map(P, st, [=] __device__(long long q) { t1[q] = -alx[q % nx] * dph[q]; }));
        TRY(noalloc_gemm_y(st, h->idcty, t1, t2, nx, ny, ny, nx));
        TRY(noalloc_gemm_x(st, h->idstx, t2 + 1, gx + 1, nx, ny, nxi, nxi));
        CK(launch_map(P, st, [=] __device__(long long q) { t1[q] = -aly[q / nx] * dph[q]; }));
        TRY(noalloc_gemm_x(st, h->idctx, t1, t2, nx, ny, nx, nx));
        TRY(noalloc_gemm_y(st, h->idsty, t2 + nx, gy + nx, nx, nyi, nyi, nx));
    } else {
        TRY(noalloc_gemm_x(st, h->idctx, dph, t2, nx, ny, nx, nx));
        TRY(noalloc_gemm_y(st, h->idcty, t2, t1, nx, ny, ny, nx));
        CK(launch_map(P, st, [=] __device__(long long q) {
            int j = (int)(q / nx), i = (int)(q % nx);
            gx[q] = d2d(t1, nx, ny, j, i, 0, dx);
            gy[q] = d2d(t1, nx, ny, j, i, 1, dy);
        }));
    }
    CK(launch_map(P, st, [=] __device__(long long q) {
        out[q] = -gx[q];
        out[P + q] = -gy[q];
        out[2 * P + q] = bza[q];
    }));
    // a later nfgs_set_boundary / nfgs_destroy waits for this call to finish
    CK(cudaEventRecord(h->ev_na_out, st));
    return NFGS_OK;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
namespace {

// B (and with a twist output J = curl B in grid units) packed per node
template <typename T>
static cudaError_t pack_field(const void* b, int nx, int ny, int nz, bool tw, T** pk, cudaStream_t s) {
    const long long V = (long long)nz * ny * nx;
    cudaError_t e = cudaMallocAsync((void**)pk, (size_t)V * (tw ? 8 : 4) * sizeof(T), s);
    if (e != cudaSuccess) return e;
    if (tw) trace::k_pack<T, true><<<(unsigned)((V + 255) / 256), 256, 0, s>>>((const T*)b, nx, ny, nz, *pk);
    else trace::k_pack<T, false><<<(unsigned)((V + 255) / 256), 256, 0, s>>>((const T*)b, nx, ny, nz, *pk);
    return cudaGetLastError();
}

template <typename T>
static int trace_lines_t(const void* b, int32_t nz, int32_t ny, int32_t nx, const void* seeds, int64_t n,
                         const double* nrm, double step, int32_t max_steps, void* ends, int32_t* flags, void* bn,
                         void* len, void* tw, cudaStream_t s) {
    T* pk = nullptr;
    cudaError_t e = pack_field<T>(b, nx, ny, nz, tw != nullptr, &pk, s);
    if (e == cudaSuccess && n > 0) {
        const trace::Box bx{nx, ny, nz, tw ? 8 : 4};
        const unsigned grid = (unsigned)((2 * n + 127) / 128);
        if (tw)
            trace::k_trace<T, true><<<grid, 128, 0, s>>>(pk, bx, (const T*)seeds, n, (T)nrm[0], (T)nrm[1],
                                                         (T)nrm[2], (T)step, max_steps, (T*)ends, flags, (T*)bn,
                                                         (T*)len, (T*)tw);
        else
            trace::k_trace<T, false><<<grid, 128, 0, s>>>(pk, bx, (const T*)seeds, n, (T)nrm[0], (T)nrm[1],
                                                          (T)nrm[2], (T)step, max_steps, (T*)ends, flags, (T*)bn,
                                                          (T*)len, nullptr);
        e = cudaGetLastError();
    }
    if (pk) cudaFreeAsync(pk, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("trace: ") + cudaGetErrorString(e));
    return NFGS_OK;
}

template <typename T>
static int trace_qperp_t(const void* b, int32_t nz, int32_t ny, int32_t nx, const void* seeds, int64_t n,
                         double delta, double step, int32_t max_steps, void* ends, int32_t* flags, void* bn,
                         void* len, void* q, void* tw, cudaStream_t s) {
    T *pk = nullptr, *e5 = nullptr;
    int* f5 = nullptr;
    cudaError_t e = pack_field<T>(b, nx, ny, nz, tw != nullptr, &pk, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&e5, (size_t)std::max<int64_t>(n, 1) * 30 * sizeof(T), s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&f5, (size_t)std::max<int64_t>(n, 1) * 10 * sizeof(int), s);
    if (e == cudaSuccess && n > 0) {
        const trace::Box bx{nx, ny, nz, tw ? 8 : 4};
        const unsigned grid = (unsigned)((10 * n + 127) / 128);
        if (tw)
            trace::k_trace_perp<T, true><<<grid, 128, 0, s>>>(pk, bx, (const T*)seeds, n, (T)delta, (T)step,
                                                              max_steps, e5, f5, (T*)bn, (T*)len, (T*)tw);
        else
            trace::k_trace_perp<T, false><<<grid, 128, 0, s>>>(pk, bx, (const T*)seeds, n, (T)delta, (T)step,
                                                               max_steps, e5, f5, (T*)bn, (T*)len, nullptr);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            trace::k_qperp<T><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(n, (T)delta, e5, f5, (const T*)bn, (T*)q);
            e = cudaGetLastError();
        }
        // the central line of each direction
        for (int d = 0; d < 2 && e == cudaSuccess; ++d) {
            e = cudaMemcpyAsync((T*)ends + (size_t)3 * d * n, e5 + (size_t)3 * (d * 5) * n, (size_t)3 * n * sizeof(T),
                                cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(flags + (size_t)d * n, f5 + (size_t)(d * 5) * n, (size_t)n * sizeof(int),
                                    cudaMemcpyDeviceToDevice, s);
        }
    }
    if (f5) cudaFreeAsync(f5, s);
    if (e5) cudaFreeAsync(e5, s);
    if (pk) cudaFreeAsync(pk, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("trace: ") + cudaGetErrorString(e));
    return NFGS_OK;
}

}  // namespace

extern "C" {

const char* nfgs_last_error(void) { return g_err.c_str(); }

const char* nfgs_version(void) { return "nfgs_b200 0.1 (sm_100a)"; }

int nfgs_release_cached_memory(int32_t device) {
    g_err.clear();
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        auto it = g_pools.find(device);
        if (it != g_pools.end()) {
            CK(cudaSetDevice(device));
            CK(cudaDeviceSynchronize());
            CK(cudaMemPoolTrimTo(it->second, 0));
        }
    }
    {
        // shared transform matrices of a device no solver uses any more
        std::lock_guard<std::mutex> lk(g_dmat_mu);
        if (g_live_handles[device] == 0) {
            for (auto it = g_dmat_cache.begin(); it != g_dmat_cache.end();) {
                if (std::get<0>(it->first) == device) {
                    if (it->second) cudaFree(it->second);
                    it = g_dmat_cache.erase(it);
                } else {
                    ++it;
                }
            }
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_ctl_mu);
        for (DevCtl* p : g_ctl_free) cudaFreeHost(p);
        g_ctl_free.clear();
    }
    std::lock_guard<std::mutex> lk(g_pin_mu);
    for (void* p : g_pin_free) cudaFreeHost(p);
    g_pin_free.clear();
    return NFGS_OK;
}

int nfgs_create(const NfgsGeom* geom, const NfgsParams* params, void** handle_out) {
    g_err.clear();
    return create_impl(geom, params, handle_out);
}

int nfgs_destroy(void* handle) {
    if (!handle) return NFGS_OK;
    Handle* h = (Handle*)handle;
    cudaSetDevice(h->geom.device);
    // a pending nfgs_gaussian_above_noalloc on another stream reads this
    // handle's buffers
    if (h->s && h->ev_na_out) cudaStreamWaitEvent(h->s, h->ev_na_out, 0);
    if (h->s) cudaStreamSynchronize(h->s);
    free_all(h);
    {
        std::lock_guard<std::mutex> lk(g_dmat_mu);
        --g_live_handles[h->geom.device];
    }
    delete h;
    return NFGS_OK;
}

int nfgs_set_boundary(void* handle, const double* bx, const double* by, const double* bz, const double* jz,
                      const NfgsBoundaryOpts* opts, double* diag_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !bx || !by || !bz || !opts) return fail(NFGS_EINVAL, "null argument");
    if (opts->jz_mode == NFGS_JZ_PROVIDED && !jz) return fail(NFGS_EINVAL, "jz is required when provided");
    if (opts->copy_ny <= 0 || opts->copy_nx <= 0 || opts->fov_y0 < 0 || opts->fov_x0 < 0 ||
        opts->fov_y0 + opts->copy_ny > h->g.ny || opts->fov_x0 + opts->copy_nx > h->g.nx ||
        opts->src_y0 < 0 || opts->src_x0 < 0 || opts->src_y0 + opts->copy_ny > opts->ny_obs ||
        opts->src_x0 + opts->copy_nx > opts->nx_obs)
        return fail(NFGS_EINVAL, "inconsistent boundary placement");
    if (opts->nzo < 1 || opts->nzo > h->g.nz) return fail(NFGS_EINVAL, "observed height out of range");
    // the boundary planes are rewritten on h->s: a pending
    // nfgs_gaussian_above_noalloc on another stream must finish reading first
    if (h->ev_na_out) CK(cudaStreamWaitEvent(h->s, h->ev_na_out, 0));
    h->fov_y0 = opts->fov_y0;
    h->fov_x0 = opts->fov_x0;
    h->nyo = opts->copy_ny;
    h->nxo = opts->copy_nx;
    h->nzo_crop = opts->nzo;
    // cwsin box on the face grid (nfgs_solver.py:2656-2676)
    {
        const int nzf = h->g.nz - 1, ny = h->g.ny, nx = h->g.nx;
        const int nzo = opts->nzo;
        const int bfz = std::max(0, nzf - nzo);
        const int ax = opts->nx_obs / 8 + opts->fov_x0;
        const int ay = opts->ny_obs / 8 + opts->fov_y0;
        const int az = nzo / 4 + bfz;
        Box b;
        b.z0 = 1; b.z1 = std::max(1, nzf - 1 - az + 1);
        b.y0 = ay; b.y1 = std::max(ay + 1, ny - 1 - ay + 1);
        b.x0 = ax; b.x1 = std::max(ax + 1, nx - 1 - ax + 1);
        b.z1 = std::min(b.z1, nzf); b.y1 = std::min(b.y1, ny); b.x1 = std::min(b.x1, nx);
        h->box = b;
    }
    h->launches = 0;
    int r = setup_boundary(h, bx, by, bz, jz, opts, diag_out);
    if (r != NFGS_OK) h->boundary_set = 0;
    return r;
}

int nfgs_iterate_begin(void* handle, const NfgsStop* stop) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !stop) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? iterate_begin_t<float>(h, stop) : iterate_begin_t<double>(h, stop);
}

int nfgs_iterate_start_state(void* handle, void** phi_out, void** az_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !phi_out || !az_out) return fail(NFGS_EINVAL, "null argument");
    return start_state(h, phi_out, az_out);
}

int nfgs_iterate_restart_from(void* handle, const void* phi, const void* az, int32_t mode, double* out3) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out3 || (mode != 4 && (!phi || !az))) return fail(NFGS_EINVAL, "null argument");
    if (mode < 0 || mode > 4) return fail(NFGS_EINVAL, "mode must be 0 to 4");
    return h->f32 ? restart_from_t<float>(h, phi, az, mode, out3) : restart_from_t<double>(h, phi, az, mode, out3);
}

__global__ void k_ctl_force_stop(DevCtl* c, int reason) {
    if (!c->stopped) {
        c->stopped = 1;
        c->stop_reason = reason;
    }
}

int nfgs_k0_state(void* handle, double* out, int32_t n) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    if (!h->k0_on) return fail(NFGS_EUNSUPPORTED, "the horizontal zero mode has no k_h=0 closure");
    const int nz = h->g.nz;
    if (n < 6 * nz + NFGS_K0_EXTRA) return fail(NFGS_EINVAL, "output too small: need 6 nz + 3 doubles");
    if (cudaSetDevice(h->geom.device) != cudaSuccess) return fail(NFGS_ECUDA, "cudaSetDevice failed");
    const size_t n2 = 2 * (size_t)nz;
    double st[4];
    CK(cudaMemcpyAsync(out, h->k0d.hlast, n2 * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemcpyAsync(out + n2, h->k0d.hstar, n2 * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemcpyAsync(out + 2 * n2, h->k0d.target, n2 * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaMemcpyAsync(st, h->k0d.stats, sizeof st, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    out[3 * n2] = st[0];
    out[3 * n2 + 1] = h->k0_spline ? h->k0_cond : std::nan("");
    out[3 * n2 + 2] = st[1];
    return NFGS_OK;
}

int nfgs_k0_operator(int32_t nz, double dz, int32_t spline, int32_t legacy, int32_t n_basis, double smoothness,
                     double* G, double* m, double* cond_out) {
    g_err.clear();
    if (!G || !m || !cond_out) return fail(NFGS_EINVAL, "null argument");
    if (nz < 3 || !(dz > 0.0)) return fail(NFGS_EINVAL, "the closure needs nz >= 3 and dz > 0");
    if (!(smoothness >= 0.0)) return fail(NFGS_EINVAL, "k0_ode_smoothness must be non-negative");
    if (spline && (n_basis < 4 || n_basis > nz)) return fail(NFGS_EINVAL, "k0_spline_basis_size must be in [4, Nz]");
    std::vector<double> g, mm;
    double cond = 0.0;
    if (!k0::build_operator(nz, dz, spline != 0, legacy != 0, n_basis, smoothness, g, mm, &cond))
        return fail(NFGS_EINVAL, "the k_h=0 closure's normal matrix is not positive definite");
    std::memcpy(G, g.data(), g.size() * sizeof(double));
    std::memcpy(m, mm.data(), mm.size() * sizeof(double));
    *cond_out = cond;
    return NFGS_OK;
}

int nfgs_iterate_fixed_point(void* handle, int32_t stop_now) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (!h) return fail(NFGS_EINVAL, "null argument");
    if (cudaSetDevice(h->geom.device) != cudaSuccess) return fail(NFGS_ECUDA, "cudaSetDevice failed");
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    h->select_final = 1;
    if (stop_now) {
        k_ctl_force_stop<<<1, 1, 0, h->s>>>(h->ctl, NFGS_STOP_FIXED_POINT);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->s));
    }
    return NFGS_OK;
}

int nfgs_step_diagnostics(void* handle, double* out15) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (!h || !out15) return fail(NFGS_EINVAL, "null argument");
    if (cudaSetDevice(h->geom.device) != cudaSuccess) return fail(NFGS_ECUDA, "cudaSetDevice failed");
    return h->f32 ? step_diagnostics_t<float>(h, out15) : step_diagnostics_t<double>(h, out15);
}

int nfgs_iterate_cfcf_start(void* handle, int32_t lateral_bc1, double* mean_bcz_out, double* out2) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (!h || !out2) return fail(NFGS_EINVAL, "null argument");
    if (cudaSetDevice(h->geom.device) != cudaSuccess) return fail(NFGS_ECUDA, "cudaSetDevice failed");
    return h->f32 ? cfcf_start_t<float>(h, lateral_bc1, mean_bcz_out, out2)
                  : cfcf_start_t<double>(h, lateral_bc1, mean_bcz_out, out2);
}

int nfgs_iterate_soft_cfcf_start(void* handle, double epsilon, double normal_ridge, double* out4) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out4) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? soft_cfcf_start_t<float>(h, epsilon, normal_ridge, out4)
                  : soft_cfcf_start_t<double>(h, epsilon, normal_ridge, out4);
}

// ---------------------------------------------------------------------------
// Batched scan: many begun iterations advanced together by one graph launch.
// ---------------------------------------------------------------------------
struct NfgsScanObj {
    std::vector<Handle*> hs;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t s = nullptr;
    int iters = 0;
    int device = 0;
};

// (Re)build the scan graph: `iters` chained copies of each handle's
// iteration graph, the handles' chains independent of one another.
static int scan_build(NfgsScanObj* sc) {
    if (sc->exec) { cudaGraphExecDestroy(sc->exec); sc->exec = nullptr; }
    if (sc->graph) { cudaGraphDestroy(sc->graph); sc->graph = nullptr; }
    if (cudaGraphCreate(&sc->graph, 0) != cudaSuccess) return fail(NFGS_ECUDA, "scan: graph create");
    for (Handle* h : sc->hs) {
        cudaGraphNode_t prev = nullptr;
        for (int k = 0; k < sc->iters; ++k) {
            cudaGraphNode_t nd;
            if (cudaGraphAddChildGraphNode(&nd, sc->graph, prev ? &prev : nullptr, prev ? 1 : 0, h->graph) !=
                cudaSuccess)
                return fail(NFGS_ECUDA, "scan: add child graph");
            prev = nd;
        }
    }
    if (cudaGraphInstantiate(&sc->exec, sc->graph, 0) != cudaSuccess) return fail(NFGS_ECUDA, "scan: instantiate");
    return NFGS_OK;
}

int nfgs_scan_create(void* const* handles, int32_t n, int32_t iters, void** scan_out) {
    g_err.clear();
    if (!handles || n <= 0 || iters <= 0 || !scan_out) return fail(NFGS_EINVAL, "scan: bad arguments");
    Handle* h0 = (Handle*)handles[0];
    if (!h0) return fail(NFGS_EINVAL, "scan: null handle");
    cudaSetDevice(h0->geom.device);
    auto* sc = new NfgsScanObj();
    sc->iters = iters;
    sc->device = h0->geom.device;
    auto bail = [&](int code) {
        if (sc->exec) cudaGraphExecDestroy(sc->exec);
        if (sc->graph) cudaGraphDestroy(sc->graph);
        if (sc->s) cudaStreamDestroy(sc->s);
        delete sc;
        return code;
    };
    for (int i = 0; i < n; ++i) {
        Handle* h = (Handle*)handles[i];
        if (!h || h->geom.device != sc->device) return bail(fail(NFGS_EINVAL, "scan: handles must share a device"));
        if (!h->iter_active) return bail(fail(NFGS_ESTATE, "scan: every handle needs nfgs_iterate_begin"));
        if (!h->stop.use_graph) return bail(fail(NFGS_EINVAL, "scan: handles must iterate with use_graph"));
        int r = h->f32 ? ensure_graph_t<float>(h) : ensure_graph_t<double>(h);
        if (r != NFGS_OK) return bail(r);
        // the begin work (gs_cfcf start) ran on the handle's stream
        if (cudaStreamSynchronize(h->s) != cudaSuccess) return bail(fail(NFGS_ECUDA, "scan: sync"));
        h->advanced = 1;
        sc->hs.push_back(h);
    }
    {
        const int r = scan_build(sc);
        if (r != NFGS_OK) return bail(r);
    }
    if (cudaStreamCreateWithFlags(&sc->s, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(NFGS_ECUDA, "scan: stream"));
    *scan_out = sc;
    return NFGS_OK;
}

int nfgs_scan_add(void* scan, void* const* handles, int32_t n) {
    g_err.clear();
    auto* sc = (NfgsScanObj*)scan;
    if (!sc || !handles || n <= 0) return fail(NFGS_EINVAL, "scan: bad arguments");
    cudaSetDevice(sc->device);
    for (int i = 0; i < n; ++i) {
        Handle* h = (Handle*)handles[i];
        if (!h || h->geom.device != sc->device) return fail(NFGS_EINVAL, "scan: handles must share a device");
        if (!h->iter_active) return fail(NFGS_ESTATE, "scan: every handle needs nfgs_iterate_begin");
        if (!h->stop.use_graph) return fail(NFGS_EINVAL, "scan: handles must iterate with use_graph");
        for (Handle* q : sc->hs)
            if (q == h) return fail(NFGS_EINVAL, "scan: handle already in the scan");
    }
    for (int i = 0; i < n; ++i) {
        Handle* h = (Handle*)handles[i];
        TRY(h->f32 ? ensure_graph_t<float>(h) : ensure_graph_t<double>(h));
        CK(cudaStreamSynchronize(h->s));
        h->advanced = 1;
        sc->hs.push_back(h);
    }
    // the running graph finished with the last launch (nfgs_scan_launch waits for it)
    return scan_build(sc);
}

int nfgs_scan_launch(void* scan, int32_t* n_active_out) {
    g_err.clear();
    auto* sc = (NfgsScanObj*)scan;
    if (!sc) return fail(NFGS_EINVAL, "null scan");
    cudaSetDevice(sc->device);
    CK(cudaGraphLaunch(sc->exec, sc->s));
    CK(cudaStreamSynchronize(sc->s));
    int active = 0;
    for (Handle* h : sc->hs) {
        CK(cudaMemcpy(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost));
        h->launches += sc->iters * h->graph_kernels;
        active += h->ctl_h->stopped ? 0 : 1;
    }
    // once half the solves of the graph have stopped, rebuild it from the
    // others: stopped solves' kernels would still be launched (and return)
    if (active > 0 && 2 * active <= (int)sc->hs.size()) {
        std::vector<Handle*> keep;
        for (Handle* h : sc->hs)
            if (!h->ctl_h->stopped) keep.push_back(h);
        sc->hs.swap(keep);
        TRY(scan_build(sc));
    }
    if (n_active_out) *n_active_out = active;
    return NFGS_OK;
}

int nfgs_scan_destroy(void* scan) {
    auto* sc = (NfgsScanObj*)scan;
    if (!sc) return NFGS_OK;
    cudaSetDevice(sc->device);
    if (sc->s) cudaStreamSynchronize(sc->s);
    if (sc->exec) cudaGraphExecDestroy(sc->exec);
    if (sc->graph) cudaGraphDestroy(sc->graph);
    if (sc->s) cudaStreamDestroy(sc->s);
    delete sc;
    return NFGS_OK;
}

int nfgs_iterate_initial(void* handle, double* scalars3) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !scalars3) return fail(NFGS_EINVAL, "null argument");
    if (!h->iter_active) return fail(NFGS_ESTATE, "iterate_begin() has not been called");
    CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    scalars3[0] = h->ctl_h->sigma0;
    scalars3[1] = h->ctl_h->divb0;
    scalars3[2] = h->ctl_h->e0;
    return NFGS_OK;
}

int nfgs_iterate_advance(void* handle, int32_t max_steps, int32_t* stop_reason, int32_t* n_done) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? iterate_advance_t<float>(h, max_steps, stop_reason, n_done)
                  : iterate_advance_t<double>(h, max_steps, stop_reason, n_done);
}

int nfgs_iterate_end(void* handle, NfgsIterResult* result, double* hist, int32_t hist_rows) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? iterate_end_t<float>(h, result, hist, hist_rows) : iterate_end_t<double>(h, result, hist, hist_rows);
}

int nfgs_get_history(void* handle, int32_t first, int32_t n, double* out, int32_t* n_total) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    if (!h->hist) { if (n_total) *n_total = 0; return NFGS_OK; }
    CK(cudaMemcpyAsync(h->ctl_h, h->ctl, sizeof(DevCtl), cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    int tot = h->ctl_h->n_hist;
    if (n_total) *n_total = tot;
    if (out && n > 0 && first >= 0 && first < tot) {
        int m = std::min(n, tot - first);
        CK(cudaMemcpy(out, h->hist + (size_t)first * NFGS_HCOLS, (size_t)m * NFGS_HCOLS * 8, cudaMemcpyDeviceToHost));
    }
    return NFGS_OK;
}

int nfgs_iterate(void* handle, const NfgsStop* stop, NfgsIterResult* result, double* hist, int32_t hist_rows) {
    TRY(nfgs_iterate_begin(handle, stop));
    int32_t reason = 0, n = 0;
    TRY(nfgs_iterate_advance(handle, stop->max_iter + 1, &reason, &n));
    return nfgs_iterate_end(handle, result, hist, hist_rows);
}

int nfgs_fields(void* handle, int32_t which, int32_t crop, double* out, int32_t* dims_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? fields_t<float>(h, which, crop, out, NFGS_F64, dims_out)
                  : fields_t<double>(h, which, crop, out, NFGS_F64, dims_out);
}

int nfgs_fields_into(void* handle, int32_t which, int32_t crop, void* out, int32_t out_dtype, int32_t* dims_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    if (out_dtype != NFGS_F32 && out_dtype != NFGS_F64) return fail(NFGS_EINVAL, "out_dtype must be NFGS_F32 or NFGS_F64");
    return h->f32 ? fields_t<float>(h, which, crop, out, out_dtype, dims_out)
                  : fields_t<double>(h, which, crop, out, out_dtype, dims_out);
}

int nfgs_fields_device(void* handle, int32_t which, int32_t crop, void* out_dev, int32_t out_dtype,
                       int32_t* dims_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    if (out_dtype != NFGS_F32 && out_dtype != NFGS_F64) return fail(NFGS_EINVAL, "out_dtype must be F32 or F64");
    if (out_dev && !h->boundary_set) return fail(NFGS_ESTATE, "boundary not set");
    return h->f32 ? fields_device_t<float>(h, which, crop, out_dev, out_dtype, dims_out)
                  : fields_device_t<double>(h, which, crop, out_dev, out_dtype, dims_out);
}

int nfgs_field_metrics(const void* ref, const void* sol, const void* cur, int32_t dtype, int32_t nz, int32_t ny,
                       int32_t nx, const double* spacing3, const int32_t* roi6, double* out, void* stream) {
    g_err.clear();
    if (!sol || !spacing3 || !roi6 || !out) return fail(NFGS_EINVAL, "null argument");
    if (dtype != NFGS_F32 && dtype != NFGS_F64) return fail(NFGS_EINVAL, "dtype must be F32 or F64");
    if (nz < 1 || ny < 1 || nx < 1) return fail(NFGS_EINVAL, "volume dimensions must be positive");
    const int lo[3] = {roi6[0], roi6[2], roi6[4]}, hi[3] = {roi6[1], roi6[3], roi6[5]}, n[3] = {nz, ny, nx};
    for (int d = 0; d < 3; ++d)
        if (!(0 <= lo[d] && lo[d] < hi[d] && hi[d] <= n[d]))
            return fail(NFGS_EINVAL, "Scoring box is outside the field or is empty");
    for (int d = 0; d < 3; ++d)
        if (!(spacing3[d] > 0.0) || !std::isfinite(spacing3[d]))
            return fail(NFGS_EINVAL, "spacing must be positive: a scalar or (dx, dy, dz)");
    met::Args a;
    a.ref = ref; a.sol = sol; a.cur = cur;
    a.nz = nz; a.ny = ny; a.nx = nx;
    a.z0 = lo[0]; a.y0 = lo[1]; a.x0 = lo[2];
    a.cz = hi[0] - lo[0]; a.cy = hi[1] - lo[1]; a.cx = hi[2] - lo[2];
    a.dx = spacing3[0]; a.dy = spacing3[1]; a.dz = spacing3[2];
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == NFGS_F32 ? field_metrics_t<float>(a, s, out) : field_metrics_t<double>(a, s, out);
}

int nfgs_trace_field_lines(const void* b, int32_t dtype, int32_t nz, int32_t ny, int32_t nx, const void* seeds,
                           int64_t n, const double* normal3, double step, int32_t max_steps, void* ends,
                           int32_t* flags, void* bn, void* length, void* twist, void* stream) {
    g_err.clear();
    if (!b || !normal3 || (n > 0 && (!seeds || !ends || !flags || !bn || !length)))
        return fail(NFGS_EINVAL, "null argument");
    if (dtype != NFGS_F32 && dtype != NFGS_F64) return fail(NFGS_EINVAL, "dtype must be F32 or F64");
    if (nz < 2 || ny < 2 || nx < 2) return fail(NFGS_EINVAL, "the field needs at least 2 nodes per axis");
    if (n < 0 || 2 * n > (int64_t)INT32_MAX * 128) return fail(NFGS_EINVAL, "bad seed count");
    if (!(step > 0.0) || !std::isfinite(step)) return fail(NFGS_EINVAL, "step must be positive");
    if (max_steps < 1) return fail(NFGS_EINVAL, "max_steps must be positive");
    if (twist && (nz < 3 || ny < 3 || nx < 3)) return fail(NFGS_EINVAL, "the twist needs at least 3 nodes per axis");
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == NFGS_F32 ? trace_lines_t<float>(b, nz, ny, nx, seeds, n, normal3, step, max_steps, ends, flags,
                                                    bn, length, twist, s)
                             : trace_lines_t<double>(b, nz, ny, nx, seeds, n, normal3, step, max_steps, ends, flags,
                                                     bn, length, twist, s);
}

int nfgs_trace_qperp(const void* b, int32_t dtype, int32_t nz, int32_t ny, int32_t nx, const void* seeds, int64_t n,
                     double delta, double step, int32_t max_steps, void* ends, int32_t* flags, void* bn, void* length,
                     void* q, void* twist, void* stream) {
    g_err.clear();
    if (!b || (n > 0 && (!seeds || !ends || !flags || !bn || !length || !q))) return fail(NFGS_EINVAL, "null argument");
    if (dtype != NFGS_F32 && dtype != NFGS_F64) return fail(NFGS_EINVAL, "dtype must be F32 or F64");
    if (nz < 2 || ny < 2 || nx < 2) return fail(NFGS_EINVAL, "the field needs at least 2 nodes per axis");
    if (n < 0 || 10 * n > (int64_t)INT32_MAX * 128) return fail(NFGS_EINVAL, "bad seed count");
    if (!(step > 0.0) || !std::isfinite(step)) return fail(NFGS_EINVAL, "step must be positive");
    if (!(delta > 0.0) || !std::isfinite(delta)) return fail(NFGS_EINVAL, "delta must be positive");
    if (max_steps < 1) return fail(NFGS_EINVAL, "max_steps must be positive");
    if (twist && (nz < 3 || ny < 3 || nx < 3)) return fail(NFGS_EINVAL, "the twist needs at least 3 nodes per axis");
    cudaStream_t s = (cudaStream_t)stream;
    return dtype == NFGS_F32 ? trace_qperp_t<float>(b, nz, ny, nx, seeds, n, delta, step, max_steps, ends, flags, bn,
                                                    length, q, twist, s)
                             : trace_qperp_t<double>(b, nz, ny, nx, seeds, n, delta, step, max_steps, ends, flags,
                                                     bn, length, q, twist, s);
}

int nfgs_trace_fastqsl(const float* b, int32_t nz, int32_t ny, int32_t nx, const float* seeds, int64_t n,
                       const double* normal3, double step, double tol_coef, int32_t with_twist, float* ends,
                       int32_t* flags, float* bsamp, int32_t* bflag, double* length, double* twist, void* stream) {
    g_err.clear();
    if (!b || !normal3 || (n > 0 && (!seeds || !ends || !flags || !bsamp || !bflag || !length)))
        return fail(NFGS_EINVAL, "null argument");
    if (with_twist && n > 0 && !twist) return fail(NFGS_EINVAL, "null twist output");
    if (nz < 3 || ny < 3 || nx < 3) return fail(NFGS_EINVAL, "the field needs at least 3 nodes per axis");
    if ((long long)nx * ny * nz >= (1LL << 31)) return fail(NFGS_EINVAL, "the field needs fewer than 2^31 nodes");
    if (n < 0 || 2 * n > (int64_t)INT32_MAX * 128) return fail(NFGS_EINVAL, "bad seed count");
    if (!(step > 0.0) || !std::isfinite(step)) return fail(NFGS_EINVAL, "step must be positive");
    if (!(tol_coef > 0.0) || !std::isfinite(tol_coef)) return fail(NFGS_EINVAL, "tol must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    const long long V = (long long)nx * ny * nz;
    float* pk = nullptr;   // J for the twist
    double* half = nullptr;  // per-half path lengths and twists
    cudaError_t e = cudaSuccess;
    if (n > 0) e = cudaMallocAsync((void**)&half, (size_t)(4 * n + 1) * sizeof(double), s);
    unsigned long long* counter = half ? (unsigned long long*)(half + 4 * n) : nullptr;
    if (e == cudaSuccess && n > 0) e = cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess && with_twist && n > 0) {
        e = cudaMallocAsync((void**)&pk, (size_t)3 * V * sizeof(float), s);
        if (e == cudaSuccess) {
            fq::k_curl<<<(unsigned)((V + 255) / 256), 256, 0, s>>>(b, nx, ny, nz, pk);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess && n > 0) {
        const fq::Field f{b, pk, nx, ny, nz, V};
        const fq::F3 n0 = fq::f3((float)normal3[0], (float)normal3[1], (float)normal3[2]);
        // enough resident warps to keep every SM busy; each pulls lines until none are left
        int dev = 0, nsm = 148, per_sm = 8;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        if (with_twist) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fq::k_trace_fq<true>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fq::k_trace_fq<false>, 128, 0);
        const long long need = (2 * n + 127) / 128;
        const unsigned grid = (unsigned)std::max(1LL, std::min(need, (long long)nsm * std::max(per_sm, 1)));
        if (with_twist)
            fq::k_trace_fq<true><<<grid, 128, 0, s>>>(f, seeds, n, n0, (float)step, (float)tol_coef, ends, flags,
                                                      bsamp, bflag, half, counter);
        else
            fq::k_trace_fq<false><<<grid, 128, 0, s>>>(f, seeds, n, n0, (float)step, (float)tol_coef, ends, flags,
                                                       bsamp, bflag, half, counter);
        fq::k_fq_sum<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, half, length, with_twist ? twist : nullptr);
        e = cudaGetLastError();
    }
    if (half) cudaFreeAsync(half, s);
    if (pk) cudaFreeAsync(pk, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("trace_fastqsl: ") + cudaGetErrorString(e));
    return NFGS_OK;
}

int nfgs_qcalc_plane(int32_t nu, int32_t nv, const float* ends, const int32_t* flags, const float* bsamp,
                     const double* normal3, double stride, float* q, void* stream) {
    g_err.clear();
    if (!ends || !flags || !bsamp || !normal3 || !q) return fail(NFGS_EINVAL, "null argument");
    if (nu < 1 || nv < 1 || nv > 65535) return fail(NFGS_EINVAL, "bad seed plane size");
    if (!(stride > 0.0) || !std::isfinite(stride)) return fail(NFGS_EINVAL, "stride must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)((nu + 127) / 128), (unsigned)nv);
    const fq::F3 n0 = fq::f3((float)normal3[0], (float)normal3[1], (float)normal3[2]);
    fq::k_qcalc_plane<<<grid, 128, 0, s>>>(nu, nv, ends, flags, bsamp, n0, (float)stride, q);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("qcalc_plane: ") + cudaGetErrorString(e));
    return NFGS_OK;
}

int nfgs_qmap_plane(int32_t dtype, int32_t nu, int32_t nv, const void* ends, const int32_t* flags, const void* bn,
                    void* q, void* stream) {
    g_err.clear();
    if (!ends || !flags || !bn || !q) return fail(NFGS_EINVAL, "null argument");
    if (dtype != NFGS_F32 && dtype != NFGS_F64) return fail(NFGS_EINVAL, "dtype must be F32 or F64");
    if (nu < 1 || nv < 1 || nv > 65535) return fail(NFGS_EINVAL, "bad seed plane size");
    cudaStream_t s = (cudaStream_t)stream;
    const dim3 grid((unsigned)((nu + 127) / 128), (unsigned)nv);
    if (dtype == NFGS_F32)
        trace::k_qmap<float><<<grid, 128, 0, s>>>(nu, nv, (const float*)ends, flags, (const float*)bn, (float*)q);
    else
        trace::k_qmap<double><<<grid, 128, 0, s>>>(nu, nv, (const double*)ends, flags, (const double*)bn, (double*)q);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NFGS_ECUDA, std::string("qmap: ") + cudaGetErrorString(e));
    return NFGS_OK;
}

int nfgs_get_scalars_state(void* handle, int32_t which, double* phi, double* az, double* scalars3) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? get_state_t<float>(h, which, phi, az, scalars3) : get_state_t<double>(h, which, phi, az, scalars3);
}

int nfgs_step(void* handle, double mu, int32_t polarity_mask) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? step_t<float>(h, mu, polarity_mask) : step_t<double>(h, mu, polarity_mask);
}

int nfgs_gaussian_above(void* handle, double* out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    return gaussian_above_impl(h, out);
}

int nfgs_gaussian_above_noalloc(void* handle, double* out_dev, void* stream) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (!h || !out_dev) return fail(NFGS_EINVAL, "null argument");
    // the caller's current device is restored on return
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(NFGS_ECUDA, "cudaGetDevice failed");
    if (prev != h->geom.device && cudaSetDevice(h->geom.device) != cudaSuccess)
        return fail(NFGS_ECUDA, "cudaSetDevice failed");
    const int rc = gaussian_above_noalloc_impl(h, out_dev, (cudaStream_t)stream);
    if (prev != h->geom.device) cudaSetDevice(prev);
    return rc;
}

int nfgs_get_plane(void* handle, int32_t which, double* out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    if (!h->boundary_set) return fail(NFGS_ESTATE, "boundary is not set");
    const double* src[] = {h->bz_obs, h->bx_obs, h->by_obs, h->jz_obs, h->az_bot,
                           h->jz_t, h->phi_above, h->bz_above, h->d0, h->dphi_tgt};
    if (which < 0 || which > 9) return fail(NFGS_EINVAL, "plane index out of range");
    CK(cudaMemcpyAsync(out, src[which], h->g.P * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    return NFGS_OK;
}

int nfgs_get_background(void* handle, double* out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    if (!h->boundary_set) return fail(NFGS_ESTATE, "boundary is not set");
    CK(cudaMemcpyAsync(out, h->bbg_d, 3 * h->g.V * 8, cudaMemcpyDeviceToHost, h->s));
    CK(cudaStreamSynchronize(h->s));
    return NFGS_OK;
}

int nfgs_time_phases(void* handle, int32_t n_iters, double* ms_out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !ms_out) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? time_phases_t<float>(h, n_iters, ms_out) : time_phases_t<double>(h, n_iters, ms_out);
}

int nfgs_apply_transform(void* handle, int32_t chain, int32_t inverse, const double* in, double* out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !in || !out) return fail(NFGS_EINVAL, "null argument");
    if (chain != 0 && chain != 1) return fail(NFGS_EINVAL, "chain must be 0 or 1");
    return h->f32 ? apply_transform_t<float>(h, chain, inverse, in, out)
                  : apply_transform_t<double>(h, chain, inverse, in, out);
}

int nfgs_source_diagnostics(void* handle, double* out) {
    g_err.clear();
    Handle* h = (Handle*)handle;
    if (h) cudaSetDevice(h->geom.device);
    if (!h || !out) return fail(NFGS_EINVAL, "null argument");
    return h->f32 ? source_diag_t<float>(h, out) : source_diag_t<double>(h, out);
}

}  // extern "C"
