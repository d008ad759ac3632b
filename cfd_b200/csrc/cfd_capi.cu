// cfd_capi.cu - C ABI (include/cfd_b200.h) of the B200 hot path: context set-up,
// device buffers, kernel orchestration of one RK3 substep, CUDA-graph replay of whole
// steps, layout conversion for the reference's f(j,column) arrays, and the reference's
// FFT entry points on device memory.
//
// Build: nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -shared -Xcompiler -fPIC

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cfd_b200.h"
#include "channel_kernels.cuh"
#include "bands_kernels.cuh"
#include "stats_kernels.cuh"
#include "xmarch.cuh"

using namespace cfd;

#define CFD_VERSION_STR "cfd_b200 0.1.0 (sm_100a)"

namespace {

const double kRKa[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
const double kRKb[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
const double kRKg[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
const double kRKc[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
const double kRKd[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};

bool fft_plan(int n, FFTDesc& d) {
    d.n = n;
    d.nrad = 0;
    int m = n;
    while (m % 4 == 0 && d.nrad < 10) { d.rad[d.nrad++] = 4; m /= 4; }
    while (m % 2 == 0 && d.nrad < 10) { d.rad[d.nrad++] = 2; m /= 2; }
    while (m % 3 == 0 && d.nrad < 10) { d.rad[d.nrad++] = 3; m /= 3; }
    return m == 1 && n >= 2;
}

struct IBDev {
    int n = 0;
    int npl = 0;
    int* idx = nullptr;
    double* w = nullptr;
    int* planes = nullptr;
    int* slot_of_j = nullptr;
    std::vector<int> h_planes;
    // z rows (0-based) that hold a forcing point or one of its two stencil points: only
    // these go through the x round trip; on the others it only zeroes Im of the kx = 0 entry
    int nact = 0;
    int* arow = nullptr;
    unsigned char* rowflag = nullptr;
};

}  // namespace

struct cfd_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    Dims d{};
    Geo g{};
    int ny = 0, dsty = 0;
    int precision = CFD_PREC_FP64;
    double re = 0, alp = 0, bet = 0, dt = 0, qxt = 0, mpgx0 = 0, mean_diag = 0;
    int ctpress = 1;
    double* geo = nullptr;
    // fields
    double2 *u1 = nullptr, *u2 = nullptr, *u3 = nullptr, *p = nullptr, *psi = nullptr, *div = nullptr;
    double2 *du1 = nullptr, *du2 = nullptr, *du3 = nullptr;
    void *Nu1 = nullptr, *Nu2 = nullptr, *Nu3 = nullptr;
    void* H[4] = {nullptr, nullptr, nullptr, nullptr};
    void* S[4] = {nullptr, nullptr, nullptr, nullptr};
    double* cs = nullptr;
    double* cs_v = nullptr;
    int JC = 16;
    int SNT = 64;           // threads per CTA of the column sweeps (k_solve_uvw, k_solve_p)
    int nch = 1;
    double* scal = nullptr;
    double* mf_work = nullptr;
    double2* stage0 = nullptr;
    double2* stage1 = nullptr;
    // reference-layout transfers of u, v, w, p: one staging buffer per field, moved in
    // kXC column chunks, host-to-device copies on xin, device-to-host copies on xout,
    // ordered per field and chunk by xev (allocated at the first such transfer)
    static constexpr int kXC = 8;
    double2* xstage[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaStream_t xin = nullptr, xout = nullptr;
    cudaEvent_t xev[4][kXC] = {};
    double* part = nullptr;
    int npart = 0;
    IBDev ibu, ibv;
    void* Hib = nullptr;    // IB round-trip planes of the u grid (u, w: 4 fields)
    void* Hib_v = nullptr;  // and of the v grid (2 fields), so the two round trips can overlap
    void* phys_v = nullptr;
    cudaStream_t side = nullptr;                     // the v-grid IB branch
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    bool hx_valid = false;  // Hx holds the z transforms of the current u, w, v (nonlinear pass)
    void* Hx = nullptr;     // z-transformed u, w, v on their own planes (two-step x-line path)
    void* phys = nullptr;
    // FFT
    FFTDesc fx{}, fz{};
    double2 *twx_d = nullptr, *twz_d = nullptr;
    float2 *twx_f = nullptr, *twz_f = nullptr;
    int CHz = 8, RWx = 4, RWib = 4, RWibf = 4;
    int RW2 = 0, NT2 = 0;
    bool XL3 = false;       // packed two-step x-line kernel (k_xline3) instead of k_xline2
    bool XALT = false, ZALT = false;  // transposed two-step splits (x-line; nonlinear z kernels)
    bool XR64 = false;      // FP32 x-line kernel held to 64 registers (k_xline2r, path 5)
    // x-line pass marching in y (k_xmarch, path 6, FP32): rows per CTA, threads, emission
    // steps per CTA (the y-chunk), shared memory
    int XMRW = 0, NTXM = 0, XMC = 0;
    size_t SMXM = 0;
    bool ZR = false;        // FP64 nonlinear z kernels held to 112 registers (k_zinv2sd, k_zfwd2d)
    // three bands: the launch dimensions of the nonlinear pass over the bottom wall band,
    // the middle band and the top wall band; the middle band's transforms
    bool mb = false;
    Dims dB{}, dM{}, dT{};
    FFTDesc fxm{};
    double2 *twxm_d = nullptr, *twzm_d = nullptr;
    float2 *twxm_f = nullptr, *twzm_f = nullptr;
    int NTZm = 0;
    size_t SMZm = 0;
    int NTZN = 0;           // threads and shared memory of the nonlinear pass's z kernels
    size_t SMZN = 0;
    int RW4 = 0, NT4 = 0;   // line-pair x-line kernel (k_xline4, FP32): rows per CTA (0 = not used), threads
    size_t SM4 = 0;
    size_t SM3 = 0;   // two-step x-line kernel: rows per CTA (0 = not used), threads
    int LZ2 = -1, NTZ2 = 0; // two-step z kernels: log2(columns per CTA) (-1 = not used), threads
    size_t SMZ2 = 0;
    int RWIX2 = 0, RWFX2 = 0;  // two-step IB x kernels: rows per CTA (0 = not used)
    int NTIX2 = 0, NTFX2 = 0;
    size_t SMIX2 = 0, SMFX2 = 0;
    size_t SM2 = 0;
    bool state_loaded = false;
    // graph of one RK3 step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int64_t graph_launches = 0;
    int64_t launches = 0;
    bool capturing = false;
    int64_t epoch = 0;      // bumped when dt or the stream changes (ensembles capture again)
    int lastplane = 0;      // single-slab x/z advective term (cfd_set_lastplane)
    bool profiling = false;
    cudaEvent_t prof_last = nullptr;
    std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> prof;
    std::string err;
    std::vector<void*> allocs;
    // statistics pass (stats.f90) and CFL maxima (dtc_calc)
    struct {
        bool on = false;          // accumulators configured
        int jband = 0, dnx = 0, dnz = 0, nbu = 0, nbv = 0, nbp = 0;
        int istat = 0;
        int cp = 48;              // planes per field in one chunk
        int ns = 8;               // CTAs per plane of the plane sums
        double* su = nullptr;     // [6][nyu]
        double* sv = nullptr;     // [5][nyv]
        double* sp = nullptr;     // [2][nyp]
        double* cu = nullptr;     // [2 bottom/top][6][nbu][dnz][dnx]
        double* cv = nullptr;     // [2][5][nbv][dnz][dnx]
        double* cp_ = nullptr;    // [2][2][nbp][dnz][dnx]
        double* planes = nullptr; // [3][cp] physical planes
        double* mx = nullptr;     // [3][nyu]: |u|, |w| per u plane, |v| dthdyv per v plane
        // the sources of every plane of a pass, [kind u, v, p][chunk][field][cp], built once
        // per context (the state pointers and the y weights do not change)
        cfd::PlaneSrc* src = nullptr;
        double* part = nullptr;   // [cp][ns][8] partial plane sums
        int nseg = 1;             // segments of tile rows of the conditional sums
        double* cpart = nullptr;  // [cp][2][nseg][6][dnx*dnz] their partial sums (nseg > 1)
        // spectra (spectra.f90): [plane][column] each; null when not configured
        double *spu = nullptr, *spv = nullptr, *spw = nullptr, *spuv = nullptr, *spp = nullptr;
    } st;
};

struct cfd_ensemble {
    std::vector<cfd_ctx*> m;
    std::vector<cudaStream_t> streams;  // one branch stream per member (owned)
    std::vector<cudaEvent_t> pre, join; // member stream -> master, branch -> master
    std::vector<int64_t> epochs;        // member epochs the graph was captured with
    cudaEvent_t fork = nullptr, done = nullptr;
    cudaStream_t master = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    int device = 0;
    std::string err;
};

namespace {

int fail(cfd_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

int cuda_check(cfd_ctx* c, cudaError_t e, const char* what) {
    if (e != cudaSuccess) return fail(c, CFD_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return CFD_OK;
}

#define CK(call)                                                   \
    do {                                                           \
        int _s = cuda_check(c, (call), #call);                     \
        if (_s != CFD_OK) return _s;                               \
    } while (0)

int launched(cfd_ctx* c, const char* name) {
    c->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(c, CFD_ERR_CUDA, "launch %s: %s", name, cudaGetErrorString(e));
    if (c->profiling && !c->capturing) {
        cudaEvent_t ev;
        if (cudaEventCreate(&ev) == cudaSuccess) {
            cudaEventRecord(ev, c->stream);
            c->prof.push_back({name, {c->prof_last, ev}});
            c->prof_last = ev;
        }
    }
    return CFD_OK;
}

// start event of the next profiled launch: recorded right before it is enqueued
void prof_mark(cfd_ctx* c) {
    if (c->profiling && !c->capturing) {
        cudaEvent_t ev;
        if (cudaEventCreate(&ev) == cudaSuccess) {
            cudaEventRecord(ev, c->stream);
            c->prof_last = ev;
            c->prof.push_back({"", {ev, ev}});
        }
    }
}

#define LK(name)                                    \
    do {                                            \
        int _s = launched(c, name);                 \
        if (_s != CFD_OK) return _s;                \
    } while (0)

template <typename T>
int dalloc(cfd_ctx* c, T** p, size_t n) {
    void* q = nullptr;
    if (n == 0) n = 1;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return fail(c, CFD_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    c->allocs.push_back(q);
    *p = (T*)q;
    return CFD_OK;
}

#define AL(ptr, type, n)                                     \
    do {                                                     \
        int _s = dalloc<type>(c, (type**)&(ptr), (n));       \
        if (_s != CFD_OK) return _s;                         \
    } while (0)

size_t zsmem(int n, int CH, size_t esz) { return (size_t)(2 * n * CH + n) * esz; }

int ilog2(int b) {
    int s = 0;
    while ((1 << s) < b) ++s;
    return s;
}

// Run BODY with NF = the fixed transform length of n (or 0 = runtime plan).
#define FFT_SWITCH(n, ...)                                \
    switch (n) {                                           \
        case 64: { constexpr int NF = 64; __VA_ARGS__; } break;   \
        case 96: { constexpr int NF = 96; __VA_ARGS__; } break;   \
        case 128: { constexpr int NF = 128; __VA_ARGS__; } break; \
        case 192: { constexpr int NF = 192; __VA_ARGS__; } break; \
        case 384: { constexpr int NF = 384; __VA_ARGS__; } break; \
        case 768: { constexpr int NF = 768; __VA_ARGS__; } break; \
        default: { constexpr int NF = 0; __VA_ARGS__; } break;    \
    }

// Run BODY with (TN1, TN2) = the two-step split of n; sets ok = false if n has none.
#define TWO_SWITCH(n, ok, ...)                                               \
    switch (n) {                                                             \
        case 64: { constexpr int TN1 = 8, TN2 = 8; __VA_ARGS__; } break;     \
        case 96: { constexpr int TN1 = 8, TN2 = 12; __VA_ARGS__; } break;    \
        case 128: { constexpr int TN1 = 8, TN2 = 16; __VA_ARGS__; } break;   \
        case 192: { constexpr int TN1 = 16, TN2 = 12; __VA_ARGS__; } break;  \
        case 384: { constexpr int TN1 = 16, TN2 = 24; __VA_ARGS__; } break;  \
        case 768: { constexpr int TN1 = 32, TN2 = 24; __VA_ARGS__; } break;  \
        default: ok = false; break;                                          \
    }

// Splits of the marching x-line kernel (x-line path 6): its second step holds N2 = 8 or 16
// points per lane, so that the unpack partners kb and N2 - kb share a warp
#define MARCH_SWITCH(n, ok, ...)                                             \
    switch (n) {                                                             \
        case 64: { constexpr int TN1 = 8, TN2 = 8; __VA_ARGS__; } break;     \
        case 96: { constexpr int TN1 = 12, TN2 = 8; __VA_ARGS__; } break;    \
        case 128: { constexpr int TN1 = 8, TN2 = 16; __VA_ARGS__; } break;   \
        case 192: { constexpr int TN1 = 12, TN2 = 16; __VA_ARGS__; } break;  \
        case 384: { constexpr int TN1 = 24, TN2 = 16; __VA_ARGS__; } break;  \
        default: ok = false; break;                                          \
    }

// The transposed splits (the other radix order), selected by cfd_tuning.xsplit/zsplit = 2
// for the x-line kernel and the nonlinear pass's z kernels.
#define TWO_SWITCH_ALT(n, ok, ...)                                           \
    switch (n) {                                                             \
        case 64: { constexpr int TN1 = 16, TN2 = 4; __VA_ARGS__; } break;    \
        case 96: { constexpr int TN1 = 12, TN2 = 8; __VA_ARGS__; } break;    \
        case 128: { constexpr int TN1 = 16, TN2 = 8; __VA_ARGS__; } break;   \
        case 192: { constexpr int TN1 = 12, TN2 = 16; __VA_ARGS__; } break;  \
        case 384: { constexpr int TN1 = 24, TN2 = 16; __VA_ARGS__; } break;  \
        case 768: { constexpr int TN1 = 24, TN2 = 32; __VA_ARGS__; } break;  \
        default: ok = false; break;                                          \
    }
#define TWO_SWITCH_SEL(alt, n, ok, ...)          \
    do {                                         \
        if (alt) {                               \
            TWO_SWITCH_ALT(n, ok, __VA_ARGS__);  \
        } else {                                 \
            TWO_SWITCH(n, ok, __VA_ARGS__);      \
        }                                        \
    } while (0)

// shared memory of k_xline2 (elements): B*LX + N
// Launch-shape overrides (unset: the built-in choice; a cfd_tuning field takes precedence).
//   CFD_XLINE_ROWS   rows per CTA of the two-step x-line kernel (power of two, 2..8)
//   CFD_ZLINES_LOG2  log2 of the lines per CTA of the two-step z kernels (2..4)
//   CFD_XLINE_STOCKHAM 1: nonlinear through the Stockham x-line kernel and per-slot z pass
//   CFD_XLINE_PATH   3: packed two-step x-line kernel (1.5 inverse lines per row)
//   CFD_SOLVE_WARP   1: Helmholtz solves one warp per column on precomputed LU factors
//   CFD_SOLVE_COLS   columns (warps) per CTA of the warp-per-column solve (1..8)
//   CFD_RHS_CHUNK    y-planes per thread of the right-hand-side kernel (2..64)
int env_int(const char* name, int dflt, int lo, int hi) {
    const char* v = std::getenv(name);
    if (!v || !*v) return dflt;
    const int x = std::atoi(v);
    return (x >= lo && x <= hi) ? x : dflt;
}

// explicit launch shapes of cfd_create_tuned (a zero field: environment, then default)
thread_local const cfd_tuning* g_tuning = nullptr;
int tune_int(int32_t cfd_tuning::*field, const char* env, int dflt, int lo, int hi) {
    if (g_tuning && g_tuning->*field >= lo && g_tuning->*field <= hi && g_tuning->*field != 0)
        return g_tuning->*field;
    return env_int(env, dflt, lo, hi);
}

size_t xline2_smem(int n1s, int n2s, int rw, size_t esz) {
    const int N = n1s * n2s;
    const int L1 = n1s * (n2s + 1) + 1, L2 = n2s * (n1s + 1) + 1, LU = N + 1;
    const int LX = std::max(L1, std::max(L2, LU));
    return ((size_t)2 * rw * LX + (size_t)n1s * (n2s + 1)) * esz;  // exchange rows + twiddle table
}

// ---------------------------------------------------------------------------------------
template <typename T2>
int set_smem_attrs(cfd_ctx* c) {
    const size_t esz = sizeof(T2);
    const int n2 = c->d.ngal2, n1 = c->d.ngal1;
    size_t sz = zsmem(n2, c->CHz, esz);
    size_t sx = (size_t)(2 * (2 * c->RWx) * n1 + n1) * esz;
    size_t si = (size_t)(2 * c->RWib * n1 + n1) * esz;
    size_t sf = (size_t)(2 * (c->RWibf / 2) * n1 + n1) * esz;
    cudaError_t e = cudaSuccess;
    FFT_SWITCH(n2, {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zinv<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zfwd<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ib_zinv<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ib_zfwd<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sz);
    });
    FFT_SWITCH(n1, {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xline<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ib_xinv<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)si);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ib_xfwd<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sf);
    });
    if (c->LZ2 >= 0) {
        bool ok = true;
        TWO_SWITCH(n2, ok, {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_zinv2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZ2);
        });
        TWO_SWITCH_SEL(c->ZALT, n2, ok, {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_zinv2s<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZN);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_zfwd2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZN);
            if constexpr (std::is_same<T2, double2>::value) {
                if (e == cudaSuccess && c->ZR)
                    e = cudaFuncSetAttribute(k_zinv2sd<TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZN);
                if (e == cudaSuccess && c->ZR)
                    e = cudaFuncSetAttribute(k_zfwd2d<TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZN);
            }
        });
    }
    if (c->LZ2 >= 0) {
        bool ok = true;
        TWO_SWITCH(n2, ok, {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_ib_zinv2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZ2);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_ib_zfwd2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMZ2);
        });
    }
    if (c->RWIX2) {
        bool ok = true;
        TWO_SWITCH(n1, ok, {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_ib_xinv2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMIX2);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_ib_xfwd2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SMFX2);
        });
    }
    if (c->RW2) {
        bool ok = true;
        TWO_SWITCH_SEL(c->XALT, n1, ok, {
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_xline2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SM2);
            if constexpr (std::is_same<T2, float2>::value)
                if (e == cudaSuccess && c->XR64)
                    e = cudaFuncSetAttribute(k_xline2r<TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SM2);
        });
        if constexpr (std::is_same<T2, float2>::value)
            if (c->XMRW) {
                MARCH_SWITCH(n1, ok, {
                    if (e == cudaSuccess)
                        e = cudaFuncSetAttribute(k_xmarch<float2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)c->SMXM);
                });
            }
        TWO_SWITCH(n1, ok, {
            if (e == cudaSuccess && c->XL3)
                e = cudaFuncSetAttribute(k_xline3<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SM3);
            if constexpr (std::is_same<T2, float2>::value)
                if (e == cudaSuccess && c->RW4)
                    e = cudaFuncSetAttribute(k_xline4<TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->SM4);
        });
    }
    if (c->mb && c->LZ2 >= 0) {
        bool ok = true;
        const int smz = (int)std::max(c->SMZ2, c->SMZm);
        TWO_SWITCH(c->dM.ngal2, ok, {
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zinv2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz);
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zfwd2<T2, TN1, TN2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smz);
        });
        FFT_SWITCH(c->dM.ngal1, {
            if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xline<T2, NF>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sx);
        });
    }
    CK(e);
    return CFD_OK;
}

template <typename T2> const T2* twx(cfd_ctx* c);
template <typename T2> const T2* twz(cfd_ctx* c);
template <> const double2* twx<double2>(cfd_ctx* c) { return c->twx_d; }
template <> const double2* twz<double2>(cfd_ctx* c) { return c->twz_d; }
template <> const float2* twx<float2>(cfd_ctx* c) { return c->twx_f; }
template <> const float2* twz<float2>(cfd_ctx* c) { return c->twz_f; }

RKCoef coef(cfd_ctx* c, int krk) {
    RKCoef k;
    const int r = krk - 1;
    k.C1 = kRKa[r] / c->re;
    k.C2 = -kRKc[r];
    k.dRK = kRKd[r];
    k.mg = -kRKg[r];
    k.dt = c->dt;
    k.krk = krk;
    k.lastplane = c->lastplane;
    return k;
}

// nonlinear passes 1-3 (FOU3D.f90:79-155)
// the nonlinear passes of a three-band channel: each kernel launched over the bottom wall
// band, the middle band and the top wall band with that band's sizes and transforms
template <typename T2>
int nl_transforms_mb(cfd_ctx* c) {
    const size_t e = sizeof(T2);
    const Dims* bands[3] = {&c->dB, &c->dM, &c->dT};
    const int CH2 = 1 << c->LZ2;
    auto twx_b = [&](bool mid) -> const T2* {
        if constexpr (std::is_same<T2, float2>::value) return mid ? c->twxm_f : c->twx_f;
        else return mid ? c->twxm_d : c->twx_d;
    };
    auto twz_b = [&](bool mid) -> const T2* {
        if constexpr (std::is_same<T2, float2>::value) return mid ? c->twzm_f : c->twz_f;
        else return mid ? c->twzm_d : c->twz_d;
    };
    prof_mark(c);
    for (const Dims* bp : bands) {
        const Dims& d = *bp;
        const bool mid = bp == &c->dM;
        dim3 gz2((std::max(d.nsu, d.nsv) * d.nkx + CH2 - 1) / CH2, 3, 2);
        bool ok = true;
        TWO_SWITCH(d.ngal2, ok, {
            k_zinv2<T2, TN1, TN2><<<gz2, mid ? c->NTZm : c->NTZ2, mid ? c->SMZm : c->SMZ2, c->stream>>>(
                d, c->g, c->u1, c->u2, c->u3, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], twz_b(mid), c->LZ2);
        });
        if (!ok) return fail(c, CFD_ERR_SIZE, "no two-step split for Ngal2=%d", d.ngal2);
    }
    LK("k_zinv2");
    prof_mark(c);
    for (const Dims* bp : bands) {
        const Dims& d = *bp;
        const bool mid = bp == &c->dM;
        dim3 gx(d.ngal2 / c->RWx, d.nsu + d.nsv);
        FFT_SWITCH(d.ngal1, {
            k_xline<T2, NF><<<gx, 256, (size_t)(2 * (2 * c->RWx) * d.ngal1 + d.ngal1) * e, c->stream>>>(
                d, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3], mid ? c->fxm : c->fx, twx_b(mid), c->RWx,
                ilog2(2 * c->RWx));
        });
    }
    LK("k_xline");
    prof_mark(c);
    for (const Dims* bp : bands) {
        const Dims& d = *bp;
        const bool mid = bp == &c->dM;
        dim3 gf2((std::max(d.nsu, d.nsv) * d.nkx + CH2 - 1) / CH2, 4, 2);
        bool ok = true;
        TWO_SWITCH(d.ngal2, ok, {
            k_zfwd2<T2, TN1, TN2><<<gf2, mid ? c->NTZm : c->NTZ2, mid ? c->SMZm : c->SMZ2, c->stream>>>(
                d, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3], (T2*)c->S[0], (T2*)c->S[1], (T2*)c->S[2],
                (T2*)c->S[3], twz_b(mid), c->LZ2);
        });
    }
    LK("k_zfwd2");
    return CFD_OK;
}

template <typename T2>
int nl_transforms(cfd_ctx* c) {
    if (c->mb) return nl_transforms_mb<T2>(c);
    const Dims& d = c->d;
    const int CH = c->CHz;
    const size_t e = sizeof(T2);
    prof_mark(c);
    if (c->RW2) {
        // each field transformed once on its own planes; the x-line kernel interpolates in y
        const int CH2 = 1 << c->LZ2;
        dim3 gz2((std::max(d.nyu, d.nyv) * d.nkx + CH2 - 1) / CH2, 3);
        bool ok = true;
        TWO_SWITCH_SEL(c->ZALT, d.ngal2, ok, {
            bool capped = false;
            if constexpr (std::is_same<T2, double2>::value) {
                if (c->ZR) {
                    k_zinv2sd<TN1, TN2><<<gz2, c->NTZN, c->SMZN, c->stream>>>(d, c->u1, c->u2, c->u3, (double2*)c->Hx,
                                                                            twz<double2>(c), c->LZ2);
                    capped = true;
                }
            }
            if (!capped)
                k_zinv2s<T2, TN1, TN2><<<gz2, c->NTZN, c->SMZN, c->stream>>>(d, c->u1, c->u2, c->u3, (T2*)c->Hx,
                                                                          twz<T2>(c), c->LZ2);
        });
        LK("k_zinv2s");
        c->hx_valid = true;
    } else if (c->LZ2 >= 0) {
        const int CH2 = 1 << c->LZ2;
        dim3 gz2((std::max(d.nyu, d.nyv) * d.nkx + CH2 - 1) / CH2, 3, 2);
        bool ok = true;
        TWO_SWITCH(d.ngal2, ok, {
            k_zinv2<T2, TN1, TN2><<<gz2, c->NTZ2, c->SMZ2, c->stream>>>(d, c->g, c->u1, c->u2, c->u3, (T2*)c->H[0],
                                                                     (T2*)c->H[1], (T2*)c->H[2], twz<T2>(c), c->LZ2);
        });
        LK("k_zinv2");
    } else {
        dim3 gz((d.nkx + CH - 1) / CH, d.nslot, 3);
        FFT_SWITCH(d.ngal2, {
            k_zinv<T2, NF><<<gz, 256, zsmem(d.ngal2, CH, e), c->stream>>>(d, c->g, c->u1, c->u2, c->u3, (T2*)c->H[0],
                                                                         (T2*)c->H[1], (T2*)c->H[2], c->fz, twz<T2>(c),
                                                                         CH, ilog2(CH));
        });
        LK("k_zinv");
    }
    prof_mark(c);
    bool xdone = false;
    if constexpr (std::is_same<T2, float2>::value) {
        if (c->RW4) {
            dim3 gx4(d.ngal2 / c->RW4, d.nslot);
            bool ok = true;
            TWO_SWITCH(d.ngal1, ok, {
                k_xline4<TN1, TN2><<<gx4, c->NT4, c->SM4, c->stream>>>(d, c->g, (const float2*)c->Hx, (float2*)c->H[0],
                                                                     (float2*)c->H[1], (float2*)c->H[2],
                                                                     (float2*)c->H[3], twx<float2>(c), c->RW4);
            });
            LK("k_xline4");
            xdone = true;
        }
    }
    if constexpr (std::is_same<T2, float2>::value) {
        if (!xdone && c->XMRW) {
            dim3 gxm(d.ngal2 / c->XMRW, (d.nyu - 1 + c->XMC - 1) / c->XMC);
            bool ok = true;
            MARCH_SWITCH(d.ngal1, ok, {
                k_xmarch<float2, TN1, TN2><<<gxm, c->NTXM, c->SMXM, c->stream>>>(
                    d, c->g, (const float2*)c->Hx, (float2*)c->H[0], (float2*)c->H[1], (float2*)c->H[2],
                    (float2*)c->H[3], twx<float2>(c), c->XMRW, c->XMC);
            });
            LK("k_xmarch");
            xdone = true;
        }
    }
    if (xdone) {
    } else if (c->RW2 && c->XL3) {
        dim3 gx3(d.ngal2 / c->RW2, d.nslot);
        bool ok = true;
        TWO_SWITCH(d.ngal1, ok, {
            k_xline3<T2, TN1, TN2><<<gx3, c->NT2, c->SM3, c->stream>>>(d, c->g, (const T2*)c->Hx, (T2*)c->H[0],
                                                                    (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3],
                                                                    twx<T2>(c), c->RW2);
        });
        LK("k_xline3");
    } else if (c->RW2) {
        dim3 gx2(d.ngal2 / c->RW2, d.nslot);
        bool ok = true;
        TWO_SWITCH_SEL(c->XALT, d.ngal1, ok, {
            bool capped = false;
            if constexpr (std::is_same<T2, float2>::value) {
                if (c->XR64) {
                    k_xline2r<TN1, TN2><<<gx2, c->NT2, c->SM2, c->stream>>>(
                        d, c->g, (const float2*)c->Hx, (float2*)c->H[0], (float2*)c->H[1], (float2*)c->H[2],
                        (float2*)c->H[3], twx<float2>(c), c->RW2, ilog2(c->RW2));
                    capped = true;
                }
            }
            if (!capped)
                k_xline2<T2, TN1, TN2><<<gx2, c->NT2, c->SM2, c->stream>>>(d, c->g, (const T2*)c->Hx, (T2*)c->H[0],
                                                                        (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3],
                                                                        twx<T2>(c), c->RW2, ilog2(c->RW2));
        });
        LK("k_xline2");
    } else {
        dim3 gx(d.ngal2 / c->RWx, d.nslot);
        FFT_SWITCH(d.ngal1, {
            k_xline<T2, NF><<<gx, 256, (size_t)(2 * (2 * c->RWx) * d.ngal1 + d.ngal1) * e, c->stream>>>(
                d, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3], c->fx, twx<T2>(c), c->RWx, ilog2(2 * c->RWx));
        });
        LK("k_xline");
    }
    prof_mark(c);
    if (c->LZ2 >= 0) {
        const int CH2 = 1 << c->LZ2;
        dim3 gf2((std::max(d.nyu, d.nyv) * d.nkx + CH2 - 1) / CH2, 4, 2);
        bool ok = true;
        TWO_SWITCH_SEL(c->ZALT, d.ngal2, ok, {
            bool capped = false;
            if constexpr (std::is_same<T2, double2>::value) {
                if (c->ZR) {
                    k_zfwd2d<TN1, TN2><<<gf2, c->NTZN, c->SMZN, c->stream>>>(
                        d, (double2*)c->H[0], (double2*)c->H[1], (double2*)c->H[2], (double2*)c->H[3],
                        (double2*)c->S[0], (double2*)c->S[1], (double2*)c->S[2], (double2*)c->S[3], twz<double2>(c),
                        c->LZ2);
                    capped = true;
                }
            }
            if (!capped)
                k_zfwd2<T2, TN1, TN2><<<gf2, c->NTZN, c->SMZN, c->stream>>>(
                    d, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3], (T2*)c->S[0], (T2*)c->S[1],
                    (T2*)c->S[2], (T2*)c->S[3], twz<T2>(c), c->LZ2);
        });
        LK("k_zfwd2");
    } else {
        dim3 gf((d.nkx + CH - 1) / CH, d.nslot, 4);
        FFT_SWITCH(d.ngal2, {
            k_zfwd<T2, NF><<<gf, 256, zsmem(d.ngal2, CH, e), c->stream>>>(
                d, (T2*)c->H[0], (T2*)c->H[1], (T2*)c->H[2], (T2*)c->H[3], (T2*)c->S[0], (T2*)c->S[1], (T2*)c->S[2],
                (T2*)c->S[3], c->fz, twz<T2>(c), CH, ilog2(CH));
        });
        LK("k_zfwd");
    }
    return CFD_OK;
}

template <typename T2, int MODE>
int rhs_kernel(cfd_ctx* c, int krk) {
    const Dims& d = c->d;
    dim3 gb((d.ncol + 255) / 256);
    prof_mark(c);
    if (c->mb) {
        k_mb_rhs<T2, MODE><<<gb, 256, 0, c->stream>>>(d, c->g, coef(c, krk), c->scal, c->u1, c->u2, c->u3, c->p,
                                                      (T2*)c->Nu1, (T2*)c->Nu2, (T2*)c->Nu3, c->du1, c->du2, c->du3,
                                                      (const T2*)c->S[0], (const T2*)c->S[1], (const T2*)c->S[2],
                                                      (const T2*)c->S[3]);
        LK("k_mb_rhs");
        return CFD_OK;
    }
    gb.y = c->nch;
    k_rhs<T2, MODE><<<gb, 256, 0, c->stream>>>(d, c->g, coef(c, krk), c->scal, c->u1, c->u2, c->u3, c->p, (T2*)c->Nu1,
                                               (T2*)c->Nu2, (T2*)c->Nu3, c->du1, c->du2, c->du3, (const T2*)c->S[0],
                                               (const T2*)c->S[1], (const T2*)c->S[2], (const T2*)c->S[3], c->JC);
    LK("k_rhs");
    return CFD_OK;
}

// immersed_boundaries_U (u1,u3) and immersed_boundaries_V (u2)
template <typename T2>
int ib_grid(cfd_ctx* c, const IBDev& ib, int j0, int nb, double2* rhs_a, double2* u_a, double2* rhs_b, double2* u_b,
            void* Hib, void* phys, int voff0, int voff1) {
    if (ib.npl == 0) return CFD_OK;
    // the velocities' inverse z transforms are those of the nonlinear pass when it left them
    IBVel vel{nullptr, {voff0, voff1}, ib.planes, j0};
    if (c->hx_valid && c->RW2 && c->LZ2 >= 0 && c->RWIX2) vel.H = c->Hx;
    using R = decltype(T2::x);
    const Dims& d = c->d;
    const int CH = c->CHz;
    const size_t e = sizeof(T2);
    IBSrc src;
    src.f[0] = rhs_a; src.f[1] = u_a; src.f[2] = rhs_b; src.f[3] = u_b;
    IBDst dst;
    dst.f[0] = rhs_a; dst.f[1] = rhs_b;
    prof_mark(c);
    if (c->LZ2 >= 0) {
        const int CH2 = 1 << c->LZ2;
        dim3 g1((ib.npl * d.nkx + CH2 - 1) / CH2, 1, vel.H ? nb : 2 * nb);
        bool ok = true;
        TWO_SWITCH(d.ngal2, ok, {
            k_ib_zinv2<T2, TN1, TN2><<<g1, c->NTZ2, c->SMZ2, c->stream>>>(d, src, j0, ib.planes, ib.npl, (T2*)Hib,
                                                                        twz<T2>(c), c->LZ2, vel.H ? 2 : 1);
        });
        LK("k_ib_zinv2");
    } else {
        dim3 g1((d.nkx + CH - 1) / CH, ib.npl, 2 * nb);
        FFT_SWITCH(d.ngal2, {
            k_ib_zinv<T2, NF><<<g1, 256, zsmem(d.ngal2, CH, e), c->stream>>>(d, src, j0, ib.planes, ib.npl, (T2*)Hib,
                                                                            c->fz, twz<T2>(c), CH, ilog2(CH));
        });
        LK("k_ib_zinv");
    }
    prof_mark(c);
    if (c->RWIX2) {
        dim3 g2((ib.nact + c->RWIX2 - 1) / c->RWIX2, ib.npl, nb);
        bool ok = true;
        if (ib.nact > 0) {
            TWO_SWITCH(d.ngal1, ok, {
                k_ib_xinv2<T2, TN1, TN2><<<g2, c->NTIX2, c->SMIX2, c->stream>>>(d, (T2*)Hib, ib.npl, (R*)phys,
                                                                              ib.arow, ib.nact, twx<T2>(c), c->RWIX2,
                                                                              vel);
            });
            LK("k_ib_xinv2");
        }
    } else {
        dim3 g2(d.ngal2 / c->RWib, ib.npl, nb);
        FFT_SWITCH(d.ngal1, {
            k_ib_xinv<T2, NF><<<g2, 256, (size_t)(2 * c->RWib * d.ngal1 + d.ngal1) * e, c->stream>>>(
                d, (T2*)Hib, ib.npl, (R*)phys, c->fx, twx<T2>(c), c->RWib, ilog2(c->RWib));
        });
        LK("k_ib_xinv");
    }
    if (ib.n > 0) {
        dim3 g3((ib.n + 255) / 256, nb);
        prof_mark(c);
        k_ib_force<R><<<g3, 256, 0, c->stream>>>(d, ib.idx, ib.w, ib.n, ib.slot_of_j, j0, ib.npl, (R*)phys);
        LK("k_ib_force");
    }
    prof_mark(c);
    if (c->RWIX2) {
        dim3 g4((ib.nact + c->RWFX2 - 1) / c->RWFX2, ib.npl, nb);
        bool ok = true;
        if (ib.nact > 0) {
            TWO_SWITCH(d.ngal1, ok, {
                k_ib_xfwd2<T2, TN1, TN2><<<g4, c->NTFX2, c->SMFX2, c->stream>>>(
                    d, (T2*)Hib, ib.npl, (const R*)phys, ib.arow, ib.nact, twx<T2>(c), c->RWFX2);
            });
            LK("k_ib_xfwd2");
        }
    } else {
        dim3 g4(d.ngal2 / c->RWibf, ib.npl, nb);
        FFT_SWITCH(d.ngal1, {
            k_ib_xfwd<T2, NF><<<g4, 256, (size_t)(2 * (c->RWibf / 2) * d.ngal1 + d.ngal1) * e, c->stream>>>(
                d, (T2*)Hib, ib.npl, (const R*)phys, c->fx, twx<T2>(c), c->RWibf, ilog2(c->RWibf / 2));
        });
        LK("k_ib_xfwd");
    }
    prof_mark(c);
    if (c->LZ2 >= 0) {
        const int CH2 = 1 << c->LZ2;
        dim3 g5((ib.npl * d.nkx + CH2 - 1) / CH2, 1, nb);
        bool ok = true;
        TWO_SWITCH(d.ngal2, ok, {
            k_ib_zfwd2<T2, TN1, TN2><<<g5, c->NTZ2, c->SMZ2, c->stream>>>(d, (const T2*)Hib, ib.npl, dst, j0,
                                                                        ib.planes, c->RWIX2 ? ib.rowflag : nullptr,
                                                                        twz<T2>(c), c->LZ2);
        });
        LK("k_ib_zfwd2");
    } else {
        dim3 g5((d.nkx + CH - 1) / CH, ib.npl, nb);
        FFT_SWITCH(d.ngal2, {
            k_ib_zfwd<T2, NF><<<g5, 256, zsmem(d.ngal2, CH, e), c->stream>>>(d, (const T2*)Hib, ib.npl, dst, j0,
                                                                            ib.planes, c->fz, twz<T2>(c), CH, ilog2(CH));
        });
        LK("k_ib_zfwd");
    }
    return CFD_OK;
}

// immersed_boundaries_U on u and w, immersed_boundaries_V on v.  The two round trips touch
// disjoint fields and buffers, so the v-grid one runs on a side stream forked from and joined
// back into the context stream (two parallel branches when captured in a graph).  With the
// per-kernel profiler on they run one after the other on the context stream.
template <typename T2>
int ib_all(cfd_ctx* c) {
    const bool par = c->side && c->ibu.npl > 0 && c->ibv.npl > 0 && !c->profiling;
    if (!par) {
        int s = ib_grid<T2>(c, c->ibu, c->d.ju0, 2, c->du1, c->u1, c->du3, c->u3, c->Hib, c->phys, 0, c->d.nyu);
        if (s != CFD_OK) return s;
        return ib_grid<T2>(c, c->ibv, c->d.jv0, 1, c->du2, c->u2, nullptr, nullptr, c->Hib_v, c->phys_v,
                           2 * c->d.nyu, 0);
    }
    CK(cudaEventRecord(c->ev_fork, c->stream));
    CK(cudaStreamWaitEvent(c->side, c->ev_fork, 0));
    cudaStream_t main = c->stream;
    c->stream = c->side;
    int s = ib_grid<T2>(c, c->ibv, c->d.jv0, 1, c->du2, c->u2, nullptr, nullptr, c->Hib_v, c->phys_v, 2 * c->d.nyu, 0);
    c->stream = main;
    const cudaError_t ej = cudaEventRecord(c->ev_join, c->side);  // join even after a failure
    if (ej == cudaSuccess) cudaStreamWaitEvent(c->stream, c->ev_join, 0);
    if (s != CFD_OK) return s;
    CK(ej);
    return ib_grid<T2>(c, c->ibu, c->d.ju0, 2, c->du1, c->u1, c->du3, c->u3, c->Hib, c->phys, 0, c->d.nyu);
}

// One launch of the Helmholtz solves on stream st: the systems part0 .. part0 + nsys - 1
// (0 = u/w, 1 = v).
int launch_solve(cfd_ctx* c, cudaStream_t st, double beta, int part0, int nsys) {
    const Dims& d = c->d;
    const dim3 gb((d.ncol + c->SNT - 1) / c->SNT, nsys);
    k_solve_uvw<<<gb, c->SNT, 0, st>>>(d, c->g, beta, c->u1, c->u2, c->u3, c->du1, c->du2, c->du3, c->cs, c->cs_v,
                                       part0);
    return launched(c, "k_solve_uvw");
}

int solve_kernel(cfd_ctx* c, int krk);

// The IB round trips (u/w and v grids on two streams inside ib_all), then one solve launch
// over both systems.  Measured at re550: running the v solve beside the u/w round trip as
// a second graph branch split the solve into two launches of half the CTAs and lost 4.5 %
// (FP32-mixed) and 3.8 % (FP64) of the step rate.
template <typename T2>
int ib_solve_all(cfd_ctx* c, int krk) {
    int s = ib_all<T2>(c);
    if (s != CFD_OK) return s;
    c->hx_valid = false;  // the solve changes u, v, w
    return solve_kernel(c, krk);
}

int solve_kernel(cfd_ctx* c, int krk) {
    const Dims& d = c->d;
    const double beta = kRKb[krk - 1] * c->dt / c->re;
    prof_mark(c);
    if (c->mb) {
        dim3 gb((d.ncol + 255) / 256);
        k_mb_solve_uvw<<<gb, 256, 0, c->stream>>>(d, c->g, beta, c->u1, c->u2, c->u3, c->du1, c->du2, c->du3, c->cs,
                                                 c->cs_v);
        LK("k_mb_solve_uvw");
        return CFD_OK;
    }
    return launch_solve(c, c->stream, beta, 0, 2);
}

int meanflow_kernel(cfd_ctx* c, int krk) {
    const double beta = kRKb[krk - 1] * c->dt / c->re;
    const double bdt = -kRKd[krk - 1] * c->dt;
    prof_mark(c);
    k_meanflow<<<1, 32, 0, c->stream>>>(c->d, c->g, beta, bdt, c->qxt, c->ctpress, c->u1, c->scal, c->mf_work);
    LK("k_meanflow");
    return CFD_OK;
}

int solvep_kernel(cfd_ctx* c, int krk, bool with_div) {
    const Dims& d = c->d;
    const double dtirk = (1.0 / c->dt) / (kRKa[krk - 1] + kRKb[krk - 1]);
    dim3 gb((d.ncol + 255) / 256);
    prof_mark(c);
    if (c->mb) {
        k_mb_solve_p<false><<<gb, 256, 0, c->stream>>>(d, c->g, dtirk, c->u1, c->u2, c->u3, c->p, c->psi,
                                                       with_div ? c->div : nullptr, c->cs, c->mean_diag, 0.0);
        LK("k_mb_solve_p");
        return CFD_OK;
    }
    const dim3 gp((d.ncol + c->SNT - 1) / c->SNT);
    k_solve_p<false><<<gp, c->SNT, 0, c->stream>>>(d, c->g, dtirk, c->u1, c->u2, c->u3, c->p, c->psi,
                                                   with_div ? c->div : nullptr, c->cs, c->mean_diag, 0.0);
    LK("k_solve_p");
    return CFD_OK;
}

int vcorr_kernel(cfd_ctx* c, int krk, bool with_div) {
    const Dims& d = c->d;
    const double dtrk = c->dt * (kRKa[krk - 1] + kRKb[krk - 1]);
    dim3 gb((d.ncol + 255) / 256);
    prof_mark(c);
    if (c->mb) {
        k_mb_vcorr<<<gb, 256, 0, c->stream>>>(d, c->g, dtrk, c->u1, c->u2, c->u3, c->psi, with_div ? c->div : nullptr);
        LK("k_mb_vcorr");
        return CFD_OK;
    }
    if (with_div) {
        k_vcorr<<<gb, 256, 0, c->stream>>>(d, c->g, dtrk, c->u1, c->u2, c->u3, c->psi, c->div);
        LK("k_vcorr");
    } else {
        gb.y = c->nch;
        k_vcorr_chunk<<<gb, 256, 0, c->stream>>>(d, c->g, dtrk, c->u1, c->u2, c->u3, c->psi, c->JC);
        LK("k_vcorr_chunk");
    }
    return CFD_OK;
}

template <typename T2>
int substep(cfd_ctx* c, int krk) {
    int s;
    if ((s = nl_transforms<T2>(c)) != CFD_OK) return s;
    if ((s = rhs_kernel<T2, 7>(c, krk)) != CFD_OK) return s;
    if ((s = ib_solve_all<T2>(c, krk)) != CFD_OK) return s;
    if (c->ctpress == 0 && (s = meanflow_kernel(c, krk)) != CFD_OK) return s;
    // solveP + v_corr in one column sweep (psi is not stored on this path)
    const Dims& d = c->d;
    const double dtirk = (1.0 / c->dt) / (kRKa[krk - 1] + kRKb[krk - 1]);
    const double dtrk = c->dt * (kRKa[krk - 1] + kRKb[krk - 1]);
    dim3 gb((d.ncol + 255) / 256);
    prof_mark(c);
    if (c->mb) {
        k_mb_solve_p<true><<<gb, 256, 0, c->stream>>>(d, c->g, dtirk, c->u1, c->u2, c->u3, c->p, c->psi, nullptr,
                                                      c->cs, c->mean_diag, dtrk);
        LK("k_mb_solve_p_vcorr");
        return CFD_OK;
    }
    const dim3 gp((d.ncol + c->SNT - 1) / c->SNT);
    k_solve_p<true><<<gp, c->SNT, 0, c->stream>>>(d, c->g, dtirk, c->u1, c->u2, c->u3, c->p, c->psi, nullptr,
                                                  c->cs, c->mean_diag, dtrk);
    LK("k_solve_p_vcorr");
    return CFD_OK;
}

int substep_any(cfd_ctx* c, int krk) {
    return c->precision == CFD_PREC_MIXED ? substep<float2>(c, krk) : substep<double2>(c, krk);
}

int check_krk(cfd_ctx* c, int krk) {
    if (!c) return CFD_ERR_ARG;
    if (krk < 1 || krk > 3) return fail(c, CFD_ERR_ARG, "krk must be 1..3 (got %d)", krk);
    if (!c->state_loaded) return fail(c, CFD_ERR_STATE, "state not uploaded");
    return CFD_OK;
}

struct FieldInfo {
    void* ptr;
    int j0;
    int nplanes;
    bool single;  // stored as float2
};

bool field_info(const cfd_ctx* c, int f, FieldInfo& fi) {
    const Dims& d = c->d;
    const bool mixed = c->precision == CFD_PREC_MIXED;
    switch (f) {
        case CFD_FIELD_U1: fi = {c->u1, d.ju0, d.nyu, false}; return true;
        case CFD_FIELD_U2: fi = {c->u2, d.jv0, d.nyv, false}; return true;
        case CFD_FIELD_U3: fi = {c->u3, d.ju0, d.nyu, false}; return true;
        case CFD_FIELD_P: fi = {c->p, d.jp0, d.nyp, false}; return true;
        case CFD_FIELD_NU1: fi = {c->Nu1, d.ju0, d.nyu, mixed}; return true;
        case CFD_FIELD_NU2: fi = {c->Nu2, d.jv0, d.nyv, mixed}; return true;
        case CFD_FIELD_NU3: fi = {c->Nu3, d.ju0, d.nyu, mixed}; return true;
        case CFD_FIELD_DIV: fi = {c->div, d.jp0, d.nyp, false}; return true;
        case CFD_FIELD_PSI: fi = {c->psi, d.jp0, d.nyp, false}; return true;
        case CFD_FIELD_DU1: fi = {c->du1, d.ju0, d.nyu, false}; return true;
        case CFD_FIELD_DU2: fi = {c->du2, d.jv0, d.nyv, false}; return true;
        case CFD_FIELD_DU3: fi = {c->du3, d.ju0, d.nyu, false}; return true;
    }
    return false;
}

__global__ void k_d2f(const double2* __restrict__ a, float2* __restrict__ b, size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        b[t] = make_float2((float)a[t].x, (float)a[t].y);
}
__global__ void k_f2d(const float2* __restrict__ a, double2* __restrict__ b, size_t n) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        b[t] = make_double2((double)a[t].x, (double)a[t].y);
}

void destroy_graph(cfd_ctx* c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
}

int fill_tw(cfd_ctx* c, int n, double2** dd, float2** df) {
    std::vector<double2> hd(n);
    std::vector<float2> hf(n);
    const long double PI_L = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < n; ++k) {
        long double a = -2.0L * PI_L * (long double)k / (long double)n;
        long double cr = cosl(a), ci = sinl(a);
        hd[k] = make_double2((double)cr, (double)ci);
        hf[k] = make_float2((float)cr, (float)ci);
    }
    AL(*dd, double2, n);
    AL(*df, float2, n);
    CK(cudaMemcpy(*dd, hd.data(), n * sizeof(double2), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(*df, hf.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
    return CFD_OK;
}

int setup_ib(cfd_ctx* c, const cfd_ib_list* l, int j0, int j1, IBDev& ib, const char* name) {
    if (!l) return CFD_OK;
    if (l->n < 0) return fail(c, CFD_ERR_ARG, "%s: negative point count", name);
    if (l->n > 0 && (!l->idx || !l->w)) return fail(c, CFD_ERR_ARG, "%s: null list arrays", name);
    // round-trip planes: interior planes inside either range (modes_to_planes_dU, FOU3D.f90:1318-1319)
    std::vector<int> slot(j1 - j0 + 1, -1);
    for (int s = 0; s < 2; ++s)
        for (int j = std::max(l->jlo[s], j0 + 1); j <= std::min(l->jhi[s], j1 - 1); ++j)
            if (slot[j - j0] < 0) {
                slot[j - j0] = (int)ib.h_planes.size();
                ib.h_planes.push_back(j);
            }
    ib.npl = (int)ib.h_planes.size();
    const int ng1 = c->d.ngal1, ng2 = c->d.ngal2;
    for (int p = 0; p < l->n; ++p) {
        const int32_t* id = l->idx + 9 * (size_t)p;
        for (int t = 0; t < 3; ++t) {
            const int i = id[3 * t], k = id[3 * t + 1], j = id[3 * t + 2];
            if (i < 1 || i > ng1 || k < 1 || k > ng2)
                return fail(c, CFD_ERR_ARG, "%s: point %d has (i,k)=(%d,%d) outside 1..%d x 1..%d", name, p, i, k, ng1, ng2);
            if (j < j0 || j > j1 || slot[j - j0] < 0)
                return fail(c, CFD_ERR_ARG, "%s: point %d references plane %d outside the round-trip ranges", name, p, j);
        }
        if (p > 0) {
            const int32_t* pv = id - 9;
            const long a = ((long)pv[2] * ng2 + pv[1]) * ng1 + pv[0], b = ((long)id[2] * ng2 + id[1]) * ng1 + id[0];
            if (b < a) return fail(c, CFD_ERR_ARG, "%s: points must be sorted by (j,k,i) (point %d)", name, p);
        }
    }
    ib.n = l->n;
    AL(ib.idx, int, 9 * (size_t)l->n);
    AL(ib.w, double, 3 * (size_t)l->n);
    AL(ib.planes, int, ib.npl);
    AL(ib.slot_of_j, int, slot.size());
    if (l->n > 0) {
        CK(cudaMemcpy(ib.idx, l->idx, 9 * sizeof(int) * (size_t)l->n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ib.w, l->w, 3 * sizeof(double) * (size_t)l->n, cudaMemcpyHostToDevice));
    }
    if (ib.npl > 0) CK(cudaMemcpy(ib.planes, ib.h_planes.data(), sizeof(int) * ib.npl, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ib.slot_of_j, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice));
    std::vector<unsigned char> flag(ng2, 0);
    for (int p = 0; p < l->n; ++p)
        for (int t = 0; t < 3; ++t) flag[l->idx[9 * (size_t)p + 3 * t + 1] - 1] = 1;
    std::vector<int> rows;
    for (int k = 0; k < ng2; ++k)
        if (flag[k]) rows.push_back(k);
    ib.nact = (int)rows.size();
    AL(ib.arow, int, std::max(ib.nact, 1));
    AL(ib.rowflag, unsigned char, ng2);
    if (ib.nact > 0) CK(cudaMemcpy(ib.arow, rows.data(), sizeof(int) * ib.nact, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ib.rowflag, flag.data(), ng2, cudaMemcpyHostToDevice));
    return CFD_OK;
}

int create_impl(const cfd_config* cfg, const cfd_ib_list* ibu, const cfd_ib_list* ibv, int device, cfd_ctx* c) {
    if (!cfg || !cfg->yu || !cfg->yv || !cfg->dthdyu || !cfg->dthdyv || !cfg->dyu2i || !cfg->dyv2i)
        return fail(c, CFD_ERR_ARG, "null config or grid array");
    if (cfg->precision != CFD_PREC_FP64 && cfg->precision != CFD_PREC_MIXED)
        return fail(c, CFD_ERR_ARG, "precision must be CFD_PREC_FP64 or CFD_PREC_MIXED");
    if (cfg->flag_ctpress != 0 && cfg->flag_ctpress != 1) return fail(c, CFD_ERR_ARG, "flag_ctpress must be 0 or 1");
    if (!(cfg->re > 0) || !(cfg->dt > 0)) return fail(c, CFD_ERR_ARG, "Re and dt must be positive");
    FFTDesc fx, fz;
    if (!fft_plan(cfg->ngal1, fx) || !fft_plan(cfg->ngal2, fz) || cfg->ngal1 < 6 || cfg->ngal2 < 6 || (cfg->ngal1 & 1) ||
        (cfg->ngal2 & 1))
        return fail(c, CFD_ERR_SIZE, "Ngal1=%d, Ngal2=%d must be even 2^a*3^b >= 6 (rft_buff.f:303-310)", cfg->ngal1, cfg->ngal2);
    if (cfg->ngal1 > 1536 || cfg->ngal2 > 1536) return fail(c, CFD_ERR_SIZE, "Ngal above 1536 not supported");
    if (cfg->ny < 4 || cfg->dsty < 0) return fail(c, CFD_ERR_SIZE, "ny must be >= 4 and dsty >= 0");
    c->device = device;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
    c->stream = c->own_stream;
    c->fx = fx;
    c->fz = fz;
    Dims& d = c->d;
    d.ngal1 = cfg->ngal1; d.ngal2 = cfg->ngal2;
    d.n1 = 2 * (cfg->ngal1 / 3); d.n2 = 2 * (cfg->ngal2 / 3);
    d.nkx = d.n1 / 2 + 1; d.ncol = d.nkx * d.n2;
    c->ny = cfg->ny; c->dsty = cfg->dsty;
    d.ny = cfg->ny;
    d.ju0 = -cfg->dsty; d.ju1 = cfg->ny + cfg->dsty;
    d.jv0 = -cfg->dsty; d.jv1 = cfg->ny + cfg->dsty - 1;
    d.jp0 = -cfg->dsty + 1; d.jp1 = cfg->ny + cfg->dsty - 1;
    d.nyu = d.ju1 - d.ju0 + 1; d.nyv = d.jv1 - d.jv0 + 1; d.nyp = d.jp1 - d.jp0 + 1;
    d.nslot = d.nyu + d.nyv;
    // stored layout and slot range of a launch over the whole channel (one band)
    d.pstride = d.ncol; d.kstride = d.nkx; d.qshift = 0; d.hstride = (long long)d.ngal2 * d.nkx;
    d.su0 = 0; d.nsu = d.nyu; d.sv0 = 0; d.nsv = d.nyv;
    d.mb = 0; d.jb = 0; d.n1m = d.n1; d.n2m = d.n2;
    c->precision = cfg->precision;
    if (cfg->band_vface > 0 && (cfg->ngal1_mid != cfg->ngal1 || cfg->ngal2_mid != cfg->ngal2)) {
        // three bands (start.f90:76-111): middle band ngal1_mid x ngal2_mid between the
        // v faces band_vface+1 .. ny-2-band_vface
        const int jb = cfg->band_vface, m = cfg->ny - 2 - jb;
        FFTDesc fxm, fzm;
        if (jb + 2 >= m || jb + 1 <= d.jv0 + 1)
            return fail(c, CFD_ERR_SIZE, "band_vface=%d leaves no middle band of two planes", jb);
        if (!fft_plan(cfg->ngal1_mid, fxm) || !fft_plan(cfg->ngal2_mid, fzm) || cfg->ngal1_mid < 6 ||
            cfg->ngal2_mid < 6 || (cfg->ngal1_mid & 1) || (cfg->ngal2_mid & 1) || cfg->ngal1_mid > cfg->ngal1 ||
            cfg->ngal2_mid > cfg->ngal2)
            return fail(c, CFD_ERR_SIZE, "middle band %d x %d: even 2^a*3^b >= 6, at most the wall bands' size",
                        cfg->ngal1_mid, cfg->ngal2_mid);
        c->mb = true;
        c->fxm = fxm;
        d.mb = 1; d.jb = jb;
        d.n1m = 2 * (cfg->ngal1_mid / 3); d.n2m = 2 * (cfg->ngal2_mid / 3);
        // launches of the nonlinear pass: the bottom wall band (u centres up to jb+1, v faces
        // up to jb), the middle band, the top wall band (planelim, start.f90:1778-1800)
        c->dB = d; c->dM = d; c->dT = d;
        c->dB.nsu = jb + 2 - d.ju0; c->dB.nsv = jb + 1 - d.jv0;
        c->dT.su0 = m + 1 - d.ju0; c->dT.nsu = d.ju1 - m; c->dT.sv0 = m + 1 - d.jv0; c->dT.nsv = d.jv1 - m;
        Dims& dm = c->dM;
        dm.su0 = jb + 2 - d.ju0; dm.nsu = m - jb - 1; dm.sv0 = jb + 1 - d.jv0; dm.nsv = m - jb;
        dm.ngal1 = cfg->ngal1_mid; dm.ngal2 = cfg->ngal2_mid; dm.n1 = d.n1m; dm.n2 = d.n2m;
        dm.nkx = dm.n1 / 2 + 1; dm.ncol = dm.nkx * dm.n2;
        dm.qshift = d.n2 - d.n2m;
    }
    c->re = cfg->re; c->alp = cfg->alp; c->bet = cfg->bet; c->dt = cfg->dt; c->qxt = cfg->qxt;
    c->mpgx0 = cfg->mpgx; c->ctpress = cfg->flag_ctpress;

    // grid + wavenumbers in one allocation
    const int nyu = d.nyu, nyv = d.nyv;
    std::vector<double> hg;
    auto push = [&](const double* a, size_t n) { hg.insert(hg.end(), a, a + n); };
    push(cfg->yu, nyu); push(cfg->yv, nyv); push(cfg->dthdyu, nyu); push(cfg->dthdyv, nyv);
    push(cfg->dyu2i, 3 * (size_t)nyu); push(cfg->dyv2i, 3 * (size_t)nyv);
    const size_t okx = hg.size();
    for (int i = 0; i < d.nkx; ++i) hg.push_back(cfg->alp * i);
    const size_t okz = hg.size();
    for (int q = 0; q < d.n2; ++q) hg.push_back(q < d.n2 / 2 ? cfg->bet * q : -cfg->bet * (d.n2 - q));
    // interpolation weights (interp_v: centres from faces; interp_u: faces from centres)
    auto YUh = [&](int j) { return cfg->yu[j - d.ju0]; };
    auto YVh = [&](int j) { return cfg->yv[j - d.jv0]; };
    const size_t ovc = hg.size();
    for (int j = d.ju0; j <= d.ju1; ++j) {
        const bool in = j > d.ju0 && j < d.ju1;
        hg.push_back(in ? (YUh(j) - YVh(j - 1)) / (YVh(j) - YVh(j - 1)) : 0.0);
    }
    for (int j = d.ju0; j <= d.ju1; ++j) {
        const bool in = j > d.ju0 && j < d.ju1;
        hg.push_back(in ? (YVh(j) - YUh(j)) / (YVh(j) - YVh(j - 1)) : 0.0);
    }
    const size_t ouf = hg.size();
    for (int j = d.jv0; j <= d.jv1; ++j) hg.push_back((YVh(j) - YUh(j)) / (YUh(j + 1) - YUh(j)));
    for (int j = d.jv0; j <= d.jv1; ++j) hg.push_back((YUh(j + 1) - YVh(j)) / (YUh(j + 1) - YUh(j)));
    for (double v : hg)
        if (!std::isfinite(v)) return fail(c, CFD_ERR_ARG, "non-finite grid value");
    AL(c->geo, double, hg.size());
    CK(cudaMemcpy(c->geo, hg.data(), hg.size() * sizeof(double), cudaMemcpyHostToDevice));
    Geo& g = c->g;
    g.yu = c->geo;
    g.yv = g.yu + nyu;
    g.dthdyu = g.yv + nyv;
    g.dthdyv = g.dthdyu + nyu;
    g.dyu2i = g.dthdyv + nyv;
    g.dyv2i = g.dyu2i + 3 * nyu;
    g.kx = c->geo + okx;
    g.kz = c->geo + okz;
    g.vca = c->geo + ovc;
    g.vcb = g.vca + nyu;
    g.ufa = c->geo + ouf;
    g.ufb = g.ufa + nyv;
    auto YU = [&](int j) { return cfg->yu[j - d.ju0]; };
    auto YV = [&](int j) { return cfg->yv[j - d.jv0]; };
    g.gwb = -(YV(d.jv0) - YU(d.ju0)) / (YV(d.jv0) - YU(d.ju0 + 1));
    g.gwt = (YU(d.ju1) - YV(d.jv1)) / (YV(d.jv1) - YU(d.ju1 - 1));
    g.gwib = (YU(d.ju0) - YU(d.ju0 + 1)) / (YV(d.jv0) - YU(d.ju0 + 1));
    g.gwit = (YU(d.ju1) - YU(d.ju1 - 1)) / (YV(d.jv1) - YU(d.ju1 - 1));
    if (c->mb) {  // gridweighting(1,2) and gridweighting(3,1) (start.f90:496, 499)
        const int jb = d.jb, m = d.ny - 2 - d.jb;
        g.gw1t = (YU(jb + 2) - YV(jb + 1)) / (YV(jb + 1) - YU(jb + 1));
        g.gw3b = -(YV(m) - YU(m)) / (YV(m) - YU(m + 1));
    }
    // mean-mode Poisson row (tridLU_3D_IB.f90:468-474): 1/(yu(2)-yu(1))^2
    if (d.ju0 > 1 || d.ju1 < 2) return fail(c, CFD_ERR_SIZE, "grid too small");
    c->mean_diag = 1.0 / ((YU(2) - YU(1)) * (YU(2) - YU(1)));

    // launch shapes
    const bool mixed = c->precision == CFD_PREC_MIXED;
    const size_t esz = mixed ? sizeof(float2) : sizeof(double2);
    const size_t budget = 110 * 1024;
    c->CHz = 8;
    while (c->CHz > 1 && zsmem(d.ngal2, c->CHz, esz) > budget) c->CHz /= 2;
    c->RWx = 8;
    while (c->RWx > 1 && ((d.ngal2 % c->RWx) || (size_t)(2 * (2 * c->RWx) * d.ngal1 + d.ngal1) * esz > budget)) c->RWx /= 2;
    c->RWib = 8;
    while (c->RWib > 1 && ((d.ngal2 % c->RWib) || (size_t)(2 * c->RWib * d.ngal1 + d.ngal1) * esz > budget)) c->RWib /= 2;
    c->RWibf = 8;
    while (c->RWibf > 2 && ((d.ngal2 % c->RWibf) || (size_t)(2 * (c->RWibf / 2) * d.ngal1 + d.ngal1) * esz > budget))
        c->RWibf /= 2;
    if (d.ngal2 % c->RWibf) return fail(c, CFD_ERR_SIZE, "Ngal2 must be even");
    // the transposed split of the x-line transform (tuning xsplit = 2) is for path 1 only
    const int xpath = g_tuning && g_tuning->xline_path ? g_tuning->xline_path : env_int("CFD_XLINE_PATH", (mixed && d.ngal1 == 384) ? 6 : 1, 1, 6);
    const bool xalt = (xpath == 1 || xpath == 5) && tune_int(&cfd_tuning::xsplit, "CFD_XSPLIT", 1, 1, 2) == 2;
    {
        bool ok = true;
        int n1s = 0, n2s = 0;
        TWO_SWITCH_SEL(xalt, d.ngal1, ok, { n1s = TN1; n2s = TN2; });
        if (ok) {
            int rw = tune_int(&cfd_tuning::xline_rows, "CFD_XLINE_ROWS", 4, 2, 8);
            rw = 1 << (31 - __builtin_clz(rw));  // a power of two
            while (rw >= 2 && ((d.ngal2 % rw) || xline2_smem(n1s, n2s, rw, esz) > budget)) rw /= 2;
            if (rw >= 2 && d.ngal2 % rw == 0 && (2 * rw * n1s) % 32 == 0) {
                c->RW2 = rw;
                c->NT2 = 2 * rw * std::max(n1s, n2s);
                c->SM2 = xline2_smem(n1s, n2s, rw, esz);
                // packed lines (k_xline3): twiddles, exchange of 2*rw lines, physical rows /
                // forward spectra
                const size_t N = (size_t)n1s * n2s, LX = (size_t)((n1s * (n2s + 1)) | 1);
                c->SM3 = (N + 2 * rw * LX + std::max((size_t)3 * (rw / 2) * N, (size_t)2 * rw * (N + 1))) * esz;
                const int xp = xpath;
                c->XL3 = xp == 3 && c->SM3 <= 220 * 1024;
                if (xp == 4 && mixed) {
                    // line pairs: rows per CTA from the same tuning field, up to 8 (the
                    // kernel's launch bound, 8*max(N1,N2) threads)
                    int r4 = tune_int(&cfd_tuning::xline_rows, "CFD_XLINE_ROWS", 8, 2, 8);
                    r4 = 1 << (31 - __builtin_clz(r4));
                    const size_t N4 = (size_t)n1s * n2s;
                    const size_t LX4 = (size_t)std::max(n1s * (n2s + 1) + 1, std::max(n2s * (n1s + 1) + 1, n1s * n2s + 1));
                    auto sm4 = [&](int r) { return ((size_t)r * LX4 + N4) * 2 * sizeof(float2); };
                    while (r4 >= 2 && ((d.ngal2 % r4) || sm4(r4) > 220 * 1024)) r4 /= 2;
                    if (r4 >= 2 && d.ngal2 % r4 == 0) {
                        c->RW4 = r4;
                        c->NT4 = r4 * std::max(n1s, n2s);
                        c->SM4 = sm4(r4);
                    }
                }
            }
        }
    }
    if ((g_tuning && g_tuning->xline_path == 2) ||
        (!(g_tuning && (g_tuning->xline_path == 1 || g_tuning->xline_path == 3 || g_tuning->xline_path == 4 ||
                         g_tuning->xline_path == 5 || g_tuning->xline_path == 6)) &&
         env_int("CFD_XLINE_STOCKHAM", 0, 0, 1)))
        c->RW2 = 0;
    {
        bool ok = true;
        int n1s = 0, n2s = 0;
        TWO_SWITCH(d.ngal2, ok, { n1s = TN1; n2s = TN2; });
        if (ok) {
            const int zl = g_tuning && (g_tuning->zlines == 4 || g_tuning->zlines == 8 || g_tuning->zlines == 16) ? g_tuning->zlines : 0;
            const int lb = zl ? ilog2(zl) : env_int("CFD_ZLINES_LOG2", mixed ? 4 : 3, 2, 4);
            c->LZ2 = lb;
            c->NTZ2 = (1 << lb) * std::max(n1s, n2s);
            c->SMZ2 = ((size_t)(1 << lb) * ((n1s * (n2s + 1)) | 1) + (size_t)n1s * n2s) * esz;
            c->NTZN = c->NTZ2;
            c->SMZN = c->SMZ2;
        }
    }
    if (c->LZ2 < 0) c->RW2 = 0;  // the two-step x-line kernels read the output of k_zinv2s
    if (!c->RW2) c->RW4 = 0;
    c->XALT = c->RW2 && xalt;  // (xalt implies path 1: neither k_xline3 nor k_xline4)
    c->XR64 = c->RW2 && !c->XL3 && !c->RW4 && mixed && xpath == 5;
    // the x-line pass marching in y (FP32-mixed, one band; the default for 384-point x lines,
    // where it measured 0.607 against 0.811 ms per launch; at 64 and 192 points the per-slot
    // kernels were faster; FP64 contexts and lengths without its split run path 1): rows per
    // CTA from xline_rows (2 or 4); emission steps per CTA from CFD_XMARCH_STEPS, by default
    // the longest chunk that keeps 20 CTAs per SM (re550: 16 steps, 0.621 ms per launch
    // against 0.625-0.636 at 8, 12, 20 and 0.65 at 32; re395: 8 steps)
    if (c->RW2 && mixed && xpath == 6 && !c->mb && d.nyu >= 4) {
        bool ok = true;
        int n1s = 0, n2s = 0;
        MARCH_SWITCH(d.ngal1, ok, { n1s = TN1; n2s = TN2; });
        if (ok) {
            int rw = tune_int(&cfd_tuning::xline_rows, "CFD_XLINE_ROWS", 2, 2, 8) >= 4 ? 4 : 2;
            auto smx = [&](int r) { return (size_t)xmarch_smem_elems(n1s, n2s, r) * sizeof(float2); };
            if (rw == 4 && (d.ngal2 % 4 || smx(4) > budget)) rw = 2;
            if (d.ngal2 % rw == 0 && smx(rw) <= budget) {
                c->XMRW = rw;
                c->NTXM = xmarch_threads(n1s, n2s, rw);
                c->SMXM = smx(rw);
                // y-chunk: the longest of 16, 12, 8, 6, 4 steps that still gives 20 CTAs per SM
                const int nrb = d.ngal2 / rw, ns = d.nyu - 1;
                int cs = 4;
                for (int cand : {16, 12, 8, 6})
                    if ((long long)nrb * ((ns + cand - 1) / cand) >= 20LL * 148) { cs = cand; break; }
                c->XMC = env_int("CFD_XMARCH_STEPS", cs, 2, 1 << 20);
            }
        }
    }
    // FP64 z kernels at 112 registers (3 CTAs of 8 lines per SM): measured 0.31 / 0.59 against
    // 0.34 / 0.61 ms per launch at re550; the 768-point split spills at that cap
    c->ZR = c->RW2 && c->precision == CFD_PREC_FP64 && d.ngal2 <= 384 && env_int("CFD_Z_R112", 1, 0, 1);
    if (c->RW2 && c->LZ2 >= 0 && tune_int(&cfd_tuning::zsplit, "CFD_ZSPLIT", 1, 1, 2) == 2) {
        bool ok = true;
        int n1s = 0, n2s = 0;
        TWO_SWITCH_ALT(d.ngal2, ok, { n1s = TN1; n2s = TN2; });
        if (ok) {
            c->ZALT = true;
            c->NTZN = (1 << c->LZ2) * std::max(n1s, n2s);
            c->SMZN = ((size_t)(1 << c->LZ2) * ((n1s * (n2s + 1)) | 1) + (size_t)n1s * n2s) * esz;
        }
    }
    {
        bool ok = true;
        int n1s = 0, n2s = 0;
        TWO_SWITCH(d.ngal1, ok, { n1s = TN1; n2s = TN2; });
        if (ok) {
            const int N = n1s * n2s, L1 = (n1s * (n2s + 1)) | 1, mx = std::max(n1s, n2s);
            for (int rw = 8; rw >= 1; rw /= 2) {
                const size_t sm = ((size_t)N + (size_t)rw * L1) * esz;
                if (d.ngal2 % rw == 0 && sm <= budget && rw * mx <= 1024) { c->RWIX2 = rw; c->SMIX2 = sm; c->NTIX2 = rw * mx; break; }
            }
            for (int rw = 16; rw >= 2; rw /= 2) {
                const size_t sm = ((size_t)N + (size_t)(rw / 2) * (N + 1) + (size_t)(rw / 2) * L1) * esz;
                if (d.ngal2 % rw == 0 && sm <= budget && (rw / 2) * mx <= 1024) { c->RWFX2 = rw; c->SMFX2 = sm; c->NTFX2 = (rw / 2) * mx; break; }
            }
            if (!c->RWIX2 || !c->RWFX2) c->RWIX2 = c->RWFX2 = 0;
        }
    }
    if (c->mb) {
        // three bands: the per-slot interpolating z pass, the Stockham x-line kernel and the
        // two-step forward z pass, launched once per band; thread-per-column solves
        c->RW2 = 0; c->XL3 = false; c->RW4 = 0; c->XALT = c->ZALT = false; c->XR64 = false; c->ZR = false;
        bool ok = true;
        int n1s = 0, n2s = 0;
        TWO_SWITCH(cfg->ngal2_mid, ok, { n1s = TN1; n2s = TN2; });
        if (c->LZ2 < 0 || !ok)
            return fail(c, CFD_ERR_SIZE, "three bands need two-step z lengths (64, 96, 128, 192, 384, 768) in both");
        c->NTZm = (1 << c->LZ2) * std::max(n1s, n2s);
        c->SMZm = ((size_t)(1 << c->LZ2) * ((n1s * (n2s + 1)) | 1) + (size_t)n1s * n2s) * esz;
        while (c->RWx > 1 && (cfg->ngal2_mid % c->RWx)) c->RWx /= 2;
    }
    int s = mixed ? set_smem_attrs<float2>(c) : set_smem_attrs<double2>(c);
    if (s != CFD_OK) return s;
    if ((s = fill_tw(c, d.ngal1, &c->twx_d, &c->twx_f)) != CFD_OK) return s;
    if ((s = fill_tw(c, d.ngal2, &c->twz_d, &c->twz_f)) != CFD_OK) return s;
    if (c->mb) {
        if ((s = fill_tw(c, cfg->ngal1_mid, &c->twxm_d, &c->twxm_f)) != CFD_OK) return s;
        if ((s = fill_tw(c, cfg->ngal2_mid, &c->twzm_d, &c->twzm_f)) != CFD_OK) return s;
    }

    // fields
    const size_t nc = d.ncol;
    AL(c->u1, double2, nc * nyu); AL(c->u3, double2, nc * nyu); AL(c->u2, double2, nc * nyv);
    AL(c->p, double2, nc * d.nyp); AL(c->psi, double2, nc * d.nyp); AL(c->div, double2, nc * d.nyp);
    AL(c->du1, double2, nc * nyu); AL(c->du3, double2, nc * nyu); AL(c->du2, double2, nc * nyv);
    if (mixed) {
        AL(c->Nu1, float2, nc * nyu); AL(c->Nu3, float2, nc * nyu); AL(c->Nu2, float2, nc * nyv);
    } else {
        AL(c->Nu1, double2, nc * nyu); AL(c->Nu3, double2, nc * nyu); AL(c->Nu2, double2, nc * nyv);
    }
    const size_t hsz = (size_t)d.nslot * d.ngal2 * d.nkx;
    for (int k = 0; k < 4; ++k) {
        if (mixed) { AL(c->H[k], float2, hsz); AL(c->S[k], float2, (size_t)d.nslot * nc); }
        else { AL(c->H[k], double2, hsz); AL(c->S[k], double2, (size_t)d.nslot * nc); }
        // three bands: the products of a short column on a middle-band plane are never
        // written and must read as zero
        if (c->mb) CK(cudaMemset(c->S[k], 0, (size_t)d.nslot * nc * esz));
    }
    if (c->RW2) {
        const size_t hxs = (size_t)(2 * nyu + nyv) * d.ngal2 * d.nkx;
        if (mixed) AL(c->Hx, float2, hxs); else AL(c->Hx, double2, hxs);
    }
    AL(c->cs, double, nc * nyu);
    AL(c->cs_v, double, nc * nyv);
    c->JC = tune_int(&cfd_tuning::rhs_chunk, "CFD_RHS_CHUNK", 4, 2, 64);
    c->SNT = 1 << ilog2(tune_int(&cfd_tuning::solve_cols, "CFD_SOLVE_THREADS", 64, 32, 256));
    c->nch = (d.nyu - 2 + c->JC - 1) / c->JC;
    AL(c->scal, double, 4);
    AL(c->mf_work, double, 4 * (size_t)(cfg->ny + 4));
    AL(c->stage0, double2, nc * nyu);
    AL(c->stage1, double2, nc * nyu);
    c->npart = 1024;
    AL(c->part, double, c->npart);
    CK(cudaMemset(c->Nu1, 0, nc * nyu * esz));
    CK(cudaMemset(c->Nu3, 0, nc * nyu * esz));
    CK(cudaMemset(c->Nu2, 0, nc * nyv * esz));
    for (double2* f : {c->u1, c->u3, c->du1, c->du3}) CK(cudaMemset(f, 0, nc * nyu * sizeof(double2)));
    for (double2* f : {c->u2, c->du2}) CK(cudaMemset(f, 0, nc * nyv * sizeof(double2)));
    for (double2* f : {c->p, c->psi, c->div}) CK(cudaMemset(f, 0, nc * d.nyp * sizeof(double2)));
    double sc[4] = {cfg->mpgx, 0.0, 0.0, 0.0};
    CK(cudaMemcpy(c->scal, sc, sizeof(sc), cudaMemcpyHostToDevice));

    // immersed boundaries
    if ((s = setup_ib(c, ibu, d.ju0, d.ju1, c->ibu, "ibu")) != CFD_OK) return s;
    if ((s = setup_ib(c, ibv, d.jv0, d.jv1, c->ibv, "ibv")) != CFD_OK) return s;
    const size_t nibu = (size_t)4 * c->ibu.npl, nibv = (size_t)2 * c->ibv.npl;
    const size_t hz = (size_t)d.ngal2 * d.nkx, hx = (size_t)d.ngal2 * d.ngal1;
    if (mixed) {
        if (nibu) { AL(c->Hib, float2, nibu * hz); AL(c->phys, float, nibu * hx); }
        if (nibv) { AL(c->Hib_v, float2, nibv * hz); AL(c->phys_v, float, nibv * hx); }
    } else {
        if (nibu) { AL(c->Hib, double2, nibu * hz); AL(c->phys, double, nibu * hx); }
        if (nibv) { AL(c->Hib_v, double2, nibv * hz); AL(c->phys_v, double, nibv * hx); }
    }
    if (nibu && nibv) {
        CK(cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
    }
    CK(cudaDeviceSynchronize());
    return CFD_OK;
}

int fft_generic_smem(int n, int CH) { return (2 * n * CH + n) * (int)sizeof(double2); }

int strided_cft(cfd_ctx* c, double* dptr, int n, int ise, int isa, int m, long long bstride, int nb, int iopt) {
    FFTDesc fd;
    if (!fft_plan(n, fd)) return fail(c, CFD_ERR_SIZE, "length %d not 2^a*3^b", n);
    const double2* tw = n == c->d.ngal2 ? c->twz_d : (n == c->d.ngal1 ? c->twx_d : nullptr);
    if (!tw) return fail(c, CFD_ERR_SIZE, "cft length must be Ngal2 or Ngal1");
    const int CH = 8;
    const int sm = fft_generic_smem(n, CH);
    CK(cudaFuncSetAttribute(k_cft_strided, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    dim3 grid((m + CH - 1) / CH, nb);
    prof_mark(c);
    k_cft_strided<<<grid, 256, sm, c->stream>>>(dptr, ise, isa, m, bstride, fd, tw, iopt, CH);
    LK("k_cft_strided");
    return CFD_OK;
}

int strided_rft(cfd_ctx* c, double* dptr, int n, int isa, int m, long long bstride, int nb, int iopt) {
    FFTDesc fd;
    if (!fft_plan(n, fd) || (n & 1)) return fail(c, CFD_ERR_SIZE, "length %d not even 2^a*3^b", n);
    const double2* tw = n == c->d.ngal1 ? c->twx_d : (n == c->d.ngal2 ? c->twz_d : nullptr);
    if (!tw) return fail(c, CFD_ERR_SIZE, "rft length must be Ngal1 or Ngal2");
    const int CH = 8;
    const int sm = fft_generic_smem(n, CH);
    CK(cudaFuncSetAttribute(k_rft_strided, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    // the inverse transforms two lines per complex transform
    const int lines = iopt > 0 ? (m + 1) / 2 : m;
    dim3 grid((lines + CH - 1) / CH, nb);
    prof_mark(c);
    k_rft_strided<<<grid, 256, sm, c->stream>>>(dptr, isa, m, bstride, fd, tw, iopt, CH);
    LK("k_rft_strided");
    return CFD_OK;
}

void dfree(cfd_ctx* c, void* p) {
    if (!p) return;
    for (auto it = c->allocs.begin(); it != c->allocs.end(); ++it)
        if (*it == p) { c->allocs.erase(it); break; }
    cudaFree(p);
}

// Plane scratch and maxima of the statistics pass (also used by the CFL query alone).
int stats_scratch(cfd_ctx* c) {
    if (c->st.planes) return CFD_OK;
    const Dims& d = c->d;
    AL(c->st.planes, double, (size_t)3 * c->st.cp * (d.ngal1 + 2) * d.ngal2);
    AL(c->st.mx, double, (size_t)3 * d.nyu);
    AL(c->st.part, double, (size_t)c->st.cp * c->st.ns * 8);
    // plane sources of the whole pass
    const Geo& g = c->g;
    const size_t nc = d.ncol;
    const int cp = c->st.cp;
    std::vector<double> hvca(d.nyu), hvcb(d.nyu), ufa(d.nyv), ufb(d.nyv), dthv(d.nyv);
    CK(cudaMemcpy(hvca.data(), g.vca, sizeof(double) * d.nyu, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(hvcb.data(), g.vcb, sizeof(double) * d.nyu, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ufa.data(), g.ufa, sizeof(double) * d.nyv, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(ufb.data(), g.ufb, sizeof(double) * d.nyv, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(dthv.data(), g.dthdyv, sizeof(double) * d.nyv, cudaMemcpyDeviceToHost));
    std::vector<PlaneSrc> hs;
    for (int kind = 0; kind < 3; ++kind) {
        const int nyg = kind == 0 ? d.nyu : (kind == 1 ? d.nyv : d.nyp);
        for (int j0 = 0; j0 < nyg; j0 += cp) {
            const int nch = std::min(cp, nyg - j0);
            const size_t base = hs.size();
            hs.resize(base + (size_t)3 * cp, PlaneSrc{nullptr, nullptr, nullptr, 1.0, 0.0, 0.0});
            for (int pl = 0; pl < nch; ++pl) {
                const int jr = j0 + pl;
                PlaneSrc* f = &hs[base + pl];
                PlaneSrc* f1 = &hs[base + nch + pl];
                PlaneSrc* f2 = &hs[base + 2 * nch + pl];
                if (kind == 0) {  // u, w, v interpolated to the centre (interp_v, FOU3D.f90:285-308)
                    f->a = c->u1 + (size_t)jr * nc;
                    f1->a = c->u3 + (size_t)jr * nc;
                    if (jr == 0) {
                        f2->a = c->u2 + nc; f2->b = c->u2;
                        f2->ca = (1.0 - g.gwib) * hvca[1]; f2->cb = g.gwib + (1.0 - g.gwib) * hvcb[1];
                    } else if (jr == d.nyu - 1) {
                        f2->a = c->u2 + (size_t)(jr - 1) * nc; f2->b = c->u2 + (size_t)(jr - 2) * nc;
                        f2->ca = g.gwit + (1.0 - g.gwit) * hvca[jr - 1]; f2->cb = (1.0 - g.gwit) * hvcb[jr - 1];
                    } else {
                        f2->a = c->u2 + (size_t)jr * nc; f2->b = c->u2 + (size_t)(jr - 1) * nc;
                        f2->ca = hvca[jr]; f2->cb = hvcb[jr];
                    }
                } else if (kind == 1) {  // v, w at the face (interp_u), omega_x = dw/dy - dv/dz
                    f->a = c->u2 + (size_t)jr * nc;
                    f1->a = c->u3 + (size_t)(jr + 1) * nc; f1->b = c->u3 + (size_t)jr * nc;
                    f1->ca = ufa[jr]; f1->cb = ufb[jr];
                    f2->a = c->u3 + (size_t)(jr + 1) * nc; f2->b = c->u3 + (size_t)jr * nc;
                    f2->ca = dthv[jr]; f2->cb = -dthv[jr];
                    f2->c = c->u2 + (size_t)jr * nc; f2->cc = -1.0;
                } else {
                    f->a = c->p + (size_t)jr * nc;
                }
            }
        }
    }
    AL(c->st.src, PlaneSrc, hs.size());
    CK(cudaMemcpy(c->st.src, hs.data(), sizeof(PlaneSrc) * hs.size(), cudaMemcpyHostToDevice));
    return CFD_OK;
}

// One pass over the u, v and p planes in chunks of cp planes per field: build the planes
// of the chunk from the spectral state, transform them to physical space (FP64), reduce.
// acc = false computes only the CFL maxima (u, w on u planes, v on v planes).
int stats_pass(cfd_ctx* c, bool acc) {
    const Dims& d = c->d;
    const Geo& g = c->g;
    auto& st = c->st;
    const long long ps = (long long)(d.ngal1 + 2) * d.ngal2;
    const int rowc = (d.ngal1 + 2) / 2;
    const PlaneSrc* src = st.src;  // advances by 3*cp entries per chunk, in pass order
    for (int kind = 0; kind < 3; ++kind) {
        const int nyg = kind == 0 ? d.nyu : (kind == 1 ? d.nyv : d.nyp);
        const int nf = kind == 2 ? 1 : 3;
        if (!acc && kind == 2) break;
        for (int j0 = 0; j0 < nyg; j0 += st.cp, src += 3 * st.cp) {
            const int nch = std::min(st.cp, nyg - j0);
            prof_mark(c);
            dim3 gb((rowc * d.ngal2 + 255) / 256, nf * nch);
            k_st_build<<<gb, 256, 0, c->stream>>>(d, g, src, st.planes);
            LK("k_st_build");
            // four_to_phys (the oddball row Ngal2/2 zeroed by four_to_phys_u lies inside the
            // dealiasing gap, which the build leaves zero)
            int s = strided_cft(c, st.planes, d.ngal2, d.ngal1 + 2, 2, d.nkx, ps, nf * nch, +1);
            if (s) return s;
            s = strided_rft(c, st.planes, d.ngal1, d.ngal1 + 2, d.ngal2, ps, nf * nch, +1);
            if (s) return s;
            prof_mark(c);
            dim3 gs(st.ns, nch);
            const int fb = (nch + 63) / 64;
            if (kind == 0) {
                k_st_sums<0><<<gs, 256, 0, c->stream>>>(d, st.planes, nch, st.part);
                k_st_fin<0><<<fb, 64, 0, c->stream>>>(d, g, st.part, nch, st.ns, j0, acc ? st.su : nullptr, d.nyu, st.mx);
            } else if (kind == 1) {
                k_st_sums<1><<<gs, 256, 0, c->stream>>>(d, st.planes, nch, st.part);
                k_st_fin<1><<<fb, 64, 0, c->stream>>>(d, g, st.part, nch, st.ns, j0, acc ? st.sv : nullptr, d.nyv,
                                                      st.mx + 2 * d.nyu);
            } else {
                k_st_sums<2><<<gs, 256, 0, c->stream>>>(d, st.planes, nch, st.part);
                k_st_fin<2><<<fb, 64, 0, c->stream>>>(d, g, st.part, nch, st.ns, j0, st.sp, d.nyp, nullptr);
            }
            LK("k_st_sums");
            if (acc && st.dnx > 0) {
                const int nb = kind == 0 ? st.nbu : (kind == 1 ? st.nbv : st.nbp);
                const size_t half = (size_t)(kind == 0 ? 6 : (kind == 1 ? 5 : 2)) * nb * st.dnx * st.dnz;
                double* cb = kind == 0 ? st.cu : (kind == 1 ? st.cv : st.cp_);
                const int tsz = st.dnx * st.dnz, nseg = st.nseg;
                dim3 gc((tsz * nseg + 255) / 256, nch), gf((tsz + 255) / 256, nch);
                prof_mark(c);
                if (kind == 0) {
                    k_st_cond<0><<<gc, 256, 0, c->stream>>>(d, st.planes, nch, j0, nyg, nb, st.dnx, st.dnz, nseg,
                                                            st.cpart, cb, cb + half);
                    if (nseg > 1)
                        k_st_cond_fin<0><<<gf, 256, 0, c->stream>>>(st.cpart, j0, nyg, nb, tsz, nseg, cb, cb + half);
                } else if (kind == 1) {
                    k_st_cond<1><<<gc, 256, 0, c->stream>>>(d, st.planes, nch, j0, nyg, nb, st.dnx, st.dnz, nseg,
                                                            st.cpart, cb, cb + half);
                    if (nseg > 1)
                        k_st_cond_fin<1><<<gf, 256, 0, c->stream>>>(st.cpart, j0, nyg, nb, tsz, nseg, cb, cb + half);
                } else {
                    k_st_cond<2><<<gc, 256, 0, c->stream>>>(d, st.planes, nch, j0, nyg, nb, st.dnx, st.dnz, nseg,
                                                            st.cpart, cb, cb + half);
                    if (nseg > 1)
                        k_st_cond_fin<2><<<gf, 256, 0, c->stream>>>(st.cpart, j0, nyg, nb, tsz, nseg, cb, cb + half);
                }
                LK("k_st_cond");
            }
        }
    }
    return CFD_OK;
}

}  // namespace

// =======================================================================================
extern "C" {

const char* cfd_version(void) { return CFD_VERSION_STR; }

const char* cfd_last_error(const cfd_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int cfd_create(const cfd_config* cfg, const cfd_ib_list* ibu, const cfd_ib_list* ibv, int32_t device, cfd_ctx** out) {
    if (!out) return CFD_ERR_ARG;
    *out = nullptr;
    cfd_ctx* c = new cfd_ctx();
    int s = create_impl(cfg, ibu, ibv, device, c);
    *out = c;  // returned even on failure so cfd_last_error can report; caller destroys
    return s;
}

int cfd_create_tuned(const cfd_config* cfg, const cfd_ib_list* ibu, const cfd_ib_list* ibv, int32_t device,
                     const cfd_tuning* tuning, cfd_ctx** out) {
    g_tuning = tuning;
    const int s = cfd_create(cfg, ibu, ibv, device, out);
    g_tuning = nullptr;
    return s;
}

int cfd_get_tuning(const cfd_ctx* c, cfd_tuning* t) {
    if (!c || !t) return CFD_ERR_ARG;
    t->xline_path = c->RW2 ? (c->XMRW ? 6 : (c->RW4 ? 4 : (c->XL3 ? 3 : (c->XR64 ? 5 : 1)))) : 2;
    t->xline_rows = c->XMRW ? c->XMRW : (c->RW4 ? c->RW4 : (c->RW2 ? c->RW2 : 0));
    t->zlines = c->LZ2 >= 0 ? (1 << c->LZ2) : 0;
    t->solve_kind = 1;
    t->solve_cols = c->SNT;
    t->rhs_chunk = c->JC;
    t->xsplit = c->XALT ? 2 : 1;
    t->zsplit = c->ZALT ? 2 : 1;
    return CFD_OK;
}

int cfd_destroy(cfd_ctx* c) {
    if (!c) return CFD_ERR_ARG;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    destroy_graph(c);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->xin) cudaStreamSynchronize(c->xin);
    if (c->xout) cudaStreamSynchronize(c->xout);
    for (void* p : c->allocs) cudaFree(p);
    for (int f = 0; f < 4; ++f)
        for (int k = 0; k < cfd_ctx::kXC; ++k)
            if (c->xev[f][k]) cudaEventDestroy(c->xev[f][k]);
    if (c->xin) cudaStreamDestroy(c->xin);
    if (c->xout) cudaStreamDestroy(c->xout);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return CFD_OK;
}

int cfd_set_stream(cfd_ctx* c, void* stream) {
    if (!c) return CFD_ERR_ARG;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->own_stream;
    if (s != c->stream) {
        destroy_graph(c);
        c->epoch++;
    }
    c->stream = s;
    return CFD_OK;
}

int cfd_synchronize(cfd_ctx* c) {
    if (!c) return CFD_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return CFD_OK;
}

int cfd_field_shape(const cfd_ctx* c, int32_t field, int64_t* ncomplex, int32_t* j0, int32_t* nplanes, int32_t* ncolumns) {
    if (!c) return CFD_ERR_ARG;
    FieldInfo fi;
    if (!field_info(c, field, fi)) return CFD_ERR_ARG;
    if (ncomplex) *ncomplex = (int64_t)fi.nplanes * c->d.ncol;
    if (j0) *j0 = fi.j0;
    if (nplanes) *nplanes = fi.nplanes;
    if (ncolumns) *ncolumns = c->d.ncol;
    return CFD_OK;
}

// Staging buffer, copy streams and ordering events of a reference-layout transfer of u, v,
// w or p.  A field moves in column chunks (contiguous in the f(j,column) layout), and the
// upload of a chunk only waits for the download that last used that chunk of the buffer,
// so the uploads of the next step run while this step's downloads are still in flight (the
// two directions of the host link at once).
int xfer_ready(cfd_ctx* c, int field) {
    if (!c->xin) {
        CK(cudaStreamCreateWithFlags(&c->xin, cudaStreamNonBlocking));
        CK(cudaStreamCreateWithFlags(&c->xout, cudaStreamNonBlocking));
    }
    if (!c->xstage[field]) {
        FieldInfo fi;
        field_info(c, field, fi);
        const size_t n = (size_t)fi.nplanes * c->d.ncol;
        double2* p = nullptr;
        CK(cudaMalloc(&p, n * sizeof(double2)));
        c->allocs.push_back(p);
        c->xstage[field] = p;
        for (int k = 0; k < cfd_ctx::kXC; ++k) {
            CK(cudaEventCreateWithFlags(&c->xev[field][k], cudaEventDisableTiming));
            CK(cudaEventRecord(c->xev[field][k], c->stream));
        }
    }
    return CFD_OK;
}

// columns [c0, c1) of transfer chunk k
void xchunk(const cfd_ctx* c, int k, int& c0, int& c1) {
    const int per = (c->d.ncol + cfd_ctx::kXC - 1) / cfd_ctx::kXC;
    c0 = std::min(c->d.ncol, k * per);
    c1 = std::min(c->d.ncol, c0 + per);
}

int cfd_upload_field(cfd_ctx* c, int32_t field, const double* host, int32_t layout) {
    if (!c || !host) return fail(c, CFD_ERR_ARG, "null argument");
    FieldInfo fi;
    if (!field_info(c, field, fi)) return fail(c, CFD_ERR_ARG, "bad field %d", field);
    if (layout != CFD_LAYOUT_REF && layout != CFD_LAYOUT_PLANE) return fail(c, CFD_ERR_ARG, "bad layout %d", layout);
    CK(cudaSetDevice(c->device));
    if (field <= CFD_FIELD_U3) c->hx_valid = false;  // the nonlinear pass's transforms are stale
    const size_t n = (size_t)fi.nplanes * c->d.ncol;
    if (layout == CFD_LAYOUT_REF && field <= CFD_FIELD_P && !fi.single) {
        int s = xfer_ready(c, field);
        if (s != CFD_OK) return s;
        for (int k = 0; k < cfd_ctx::kXC; ++k) {
            int c0, c1;
            xchunk(c, k, c0, c1);
            if (c0 >= c1) continue;
            cudaEvent_t ev = c->xev[field][k];
            const size_t off = (size_t)c0 * fi.nplanes, m = (size_t)(c1 - c0) * fi.nplanes;
            // the copy waits for the last download out of this chunk of the buffer, the
            // transpose on the context stream for the copy
            CK(cudaStreamWaitEvent(c->xin, ev, 0));
            CK(cudaMemcpyAsync(c->xstage[field] + off, host + 2 * off, m * sizeof(double2), cudaMemcpyHostToDevice,
                               c->xin));
            CK(cudaEventRecord(ev, c->xin));
            CK(cudaStreamWaitEvent(c->stream, ev, 0));
            dim3 grid((fi.nplanes + 31) / 32, (c1 - c0 + 31) / 32);
            prof_mark(c);
            k_transpose<<<grid, dim3(32, 8), 0, c->stream>>>(c->xstage[field] + off, (double2*)fi.ptr + c0, c1 - c0,
                                                             fi.nplanes, fi.nplanes, c->d.ncol);
            LK("k_transpose");
            CK(cudaEventRecord(ev, c->stream));
        }
        c->state_loaded = true;
        return CFD_OK;
    }
    double2* dst = fi.single ? c->stage1 : (double2*)fi.ptr;
    if (layout == CFD_LAYOUT_PLANE) {
        CK(cudaMemcpyAsync(dst, host, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
    } else {
        CK(cudaMemcpyAsync(c->stage0, host, n * sizeof(double2), cudaMemcpyHostToDevice, c->stream));
        dim3 grid((fi.nplanes + 31) / 32, (c->d.ncol + 31) / 32);
        prof_mark(c);
        k_transpose<<<grid, dim3(32, 8), 0, c->stream>>>(c->stage0, dst, c->d.ncol, fi.nplanes, fi.nplanes,
                                                         c->d.ncol);
        LK("k_transpose");
    }
    if (fi.single) {
        prof_mark(c);
        k_d2f<<<1024, 256, 0, c->stream>>>(dst, (float2*)fi.ptr, n);
        LK("k_d2f");
    }
    if (field <= CFD_FIELD_P) c->state_loaded = true;
    return CFD_OK;
}

int cfd_download_field(cfd_ctx* c, int32_t field, double* host, int32_t layout) {
    if (!c || !host) return fail(c, CFD_ERR_ARG, "null argument");
    FieldInfo fi;
    if (!field_info(c, field, fi)) return fail(c, CFD_ERR_ARG, "bad field %d", field);
    if (layout != CFD_LAYOUT_REF && layout != CFD_LAYOUT_PLANE) return fail(c, CFD_ERR_ARG, "bad layout %d", layout);
    CK(cudaSetDevice(c->device));
    const size_t n = (size_t)fi.nplanes * c->d.ncol;
    const double2* src = (const double2*)fi.ptr;
    if (layout == CFD_LAYOUT_REF && field <= CFD_FIELD_P && !fi.single) {
        int s = xfer_ready(c, field);
        if (s != CFD_OK) return s;
        for (int k = 0; k < cfd_ctx::kXC; ++k) {
            int c0, c1;
            xchunk(c, k, c0, c1);
            if (c0 >= c1) continue;
            cudaEvent_t ev = c->xev[field][k];
            const size_t off = (size_t)c0 * fi.nplanes, m = (size_t)(c1 - c0) * fi.nplanes;
            CK(cudaStreamWaitEvent(c->stream, ev, 0));  // the last copy out of this chunk
            dim3 grid((c1 - c0 + 31) / 32, (fi.nplanes + 31) / 32);
            prof_mark(c);
            k_transpose<<<grid, dim3(32, 8), 0, c->stream>>>(src + c0, c->xstage[field] + off, fi.nplanes, c1 - c0,
                                                             c->d.ncol, fi.nplanes);
            LK("k_transpose");
            CK(cudaEventRecord(ev, c->stream));
            CK(cudaStreamWaitEvent(c->xout, ev, 0));
            CK(cudaMemcpyAsync(host + 2 * off, c->xstage[field] + off, m * sizeof(double2), cudaMemcpyDeviceToHost,
                               c->xout));
            CK(cudaEventRecord(ev, c->xout));
            // work issued later on the context stream (and its synchronisation) follows the copy
            CK(cudaStreamWaitEvent(c->stream, ev, 0));
        }
        return CFD_OK;
    }
    if (fi.single) {
        prof_mark(c);
        k_f2d<<<1024, 256, 0, c->stream>>>((const float2*)fi.ptr, c->stage1, n);
        LK("k_f2d");
        src = c->stage1;
    }
    if (layout == CFD_LAYOUT_PLANE) {
        CK(cudaMemcpyAsync(host, src, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    } else {
        dim3 grid((c->d.ncol + 31) / 32, (fi.nplanes + 31) / 32);
        prof_mark(c);
        k_transpose<<<grid, dim3(32, 8), 0, c->stream>>>(src, c->stage0, fi.nplanes, c->d.ncol, c->d.ncol,
                                                         fi.nplanes);
        LK("k_transpose");
        CK(cudaMemcpyAsync(host, c->stage0, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    }
    return CFD_OK;
}

int cfd_field_device_ptr(cfd_ctx* c, int32_t field, void** dev_ptr) {
    if (!c || !dev_ptr) return CFD_ERR_ARG;
    FieldInfo fi;
    if (!field_info(c, field, fi)) return fail(c, CFD_ERR_ARG, "bad field %d", field);
    *dev_ptr = fi.ptr;
    if (field <= CFD_FIELD_P) c->state_loaded = true;
    if (field <= CFD_FIELD_U3) c->hx_valid = false;  // the caller may write the field
    return CFD_OK;
}

int cfd_rhs0(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    return c->precision == CFD_PREC_MIXED ? rhs_kernel<float2, 1>(c, krk) : rhs_kernel<double2, 1>(c, krk);
}

int cfd_nonlinear(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    if (c->precision == CFD_PREC_MIXED) {
        if ((s = nl_transforms<float2>(c))) return s;
        return rhs_kernel<float2, 2>(c, krk);
    }
    if ((s = nl_transforms<double2>(c))) return s;
    return rhs_kernel<double2, 2>(c, krk);
}

int cfd_solve_uvw(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    if (c->precision == CFD_PREC_MIXED) {
        if ((s = rhs_kernel<float2, 4>(c, krk))) return s;
        if ((s = ib_all<float2>(c))) return s;
    } else {
        if ((s = rhs_kernel<double2, 4>(c, krk))) return s;
        if ((s = ib_all<double2>(c))) return s;
    }
    c->hx_valid = false;  // the solve changes u, v, w
    return solve_kernel(c, krk);
}

int cfd_meanflow(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    return meanflow_kernel(c, krk);
}

int cfd_solve_p(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    return solvep_kernel(c, krk, true);
}

int cfd_vcorr(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    return vcorr_kernel(c, krk, true);
}

int cfd_rk_substep(cfd_ctx* c, int32_t krk) {
    int s = check_krk(c, krk);
    if (s) return s;
    return substep_any(c, krk);
}

int cfd_step(cfd_ctx* c, int32_t nsteps) {
    int s = check_krk(c, 1);
    if (s) return s;
    if (nsteps < 0) return fail(c, CFD_ERR_ARG, "nsteps < 0");
    CK(cudaSetDevice(c->device));
    if (!c->gexec) {
        const int64_t before = c->launches;
        CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        c->capturing = true;
        int st = CFD_OK;
        for (int k = 1; k <= 3 && st == CFD_OK; ++k) st = substep_any(c, k);
        if (st == CFD_OK && c->ctpress == 1) st = meanflow_kernel(c, 1);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
        c->capturing = false;
        if (st != CFD_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) return fail(c, CFD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        c->graph = graph;
        CK(cudaGraphInstantiate(&c->gexec, c->graph, 0));
        c->graph_launches = c->launches - before;
        c->launches = before;
    }
    for (int n = 0; n < nsteps; ++n) {
        CK(cudaGraphLaunch(c->gexec, c->stream));
        c->launches += c->graph_launches;
    }
    return CFD_OK;
}

int cfd_get_scalars(cfd_ctx* c, double* mpgx, double* qx, double* dgx) {
    if (!c) return CFD_ERR_ARG;
    double h[4];
    CK(cudaMemcpyAsync(h, c->scal, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (mpgx) *mpgx = h[0];
    if (qx) *qx = h[1];
    if (dgx) *dgx = h[2];
    if (!std::isfinite(h[0]) || !std::isfinite(h[1]) || !std::isfinite(h[2]))
        return fail(c, CFD_ERR_NONFINITE, "non-finite mean-flow scalars (mpgx %g, Qx %g)", h[0], h[1]);
    return CFD_OK;
}

int cfd_divergence_max(cfd_ctx* c, double* errmax) {
    if (!c || !errmax) return CFD_ERR_ARG;
    const Dims& d = c->d;
    // recompute div from the current state (divergence, littleharsh.f90:209-244)
    prof_mark(c);
    if (c->mb)
        k_mb_divergence<<<(d.ncol + 255) / 256, 256, 0, c->stream>>>(d, c->g, c->u1, c->u2, c->u3, c->div);
    else
        k_divergence<<<(d.ncol + 255) / 256, 256, 0, c->stream>>>(d, c->g, c->u1, c->u2, c->u3, c->div);
    LK("k_divergence");
    prof_mark(c);
    k_absmax<<<c->npart, 256, 0, c->stream>>>(c->div, (size_t)d.ncol * d.nyp, c->part);
    LK("k_absmax");
    std::vector<double> h(c->npart);
    CK(cudaMemcpyAsync(h.data(), c->part, sizeof(double) * c->npart, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double m = 0.0;
    bool bad = false;
    for (double v : h) {
        if (!std::isfinite(v)) bad = true;
        m = std::max(m, v);
    }
    *errmax = bad ? NAN : m;
    if (bad) return fail(c, CFD_ERR_NONFINITE, "non-finite divergence");
    return CFD_OK;
}

int cfd_stats_configure(cfd_ctx* c, const cfd_stats_config* sc) {
    if (c && c->mb) return fail(c, CFD_ERR_ARG, "statistics of a three-band channel are not supported");
    if (!c || !sc) return fail(c, CFD_ERR_ARG, "bad arguments");
    const Dims& d = c->d;
    auto& st = c->st;
    const bool cond = sc->jband >= d.jv0;
    if (cond) {
        if (sc->dnx <= 0 || sc->dnz <= 0 || d.ngal1 % sc->dnx || d.ngal2 % sc->dnz)
            return fail(c, CFD_ERR_ARG, "tile %d x %d must divide Ngal1 x Ngal2", sc->dnx, sc->dnz);
        if (sc->jband + 1 > d.ju1) return fail(c, CFD_ERR_ARG, "jband %d above the channel", sc->jband);
    }
    for (double* p : {st.su, st.sv, st.sp, st.cu, st.cv, st.cp_, st.spu, st.spv, st.spw, st.spuv, st.spp, st.cpart})
        dfree(c, p);
    st.su = st.sv = st.sp = st.cu = st.cv = st.cp_ = st.cpart = nullptr;
    st.spu = st.spv = st.spw = st.spuv = st.spp = nullptr;
    int s = stats_scratch(c);
    if (s) return s;
    st.jband = sc->jband;
    st.dnx = cond ? sc->dnx : 0;
    st.dnz = cond ? sc->dnz : 0;
    // bottom band: u planes -dsty..jband+1, v planes -dsty..jband, p planes -dsty+1..jband
    st.nbu = cond ? sc->jband + 1 - d.ju0 + 1 : 0;
    st.nbv = cond ? sc->jband - d.jv0 + 1 : 0;
    st.nbp = cond ? sc->jband - d.jp0 + 1 : 0;
    AL(st.su, double, (size_t)6 * d.nyu);
    AL(st.sv, double, (size_t)5 * d.nyv);
    AL(st.sp, double, (size_t)2 * d.nyp);
    const size_t tsz = (size_t)st.dnx * st.dnz;
    AL(st.cu, double, 2 * 6 * st.nbu * tsz);
    AL(st.cv, double, 2 * 5 * st.nbv * tsz);
    AL(st.cp_, double, 2 * 2 * st.nbp * tsz);
    // conditional sums: tile rows split into segments so that a plane has about 1024 threads
    st.nseg = tsz ? (int)std::max<size_t>(1, std::min<size_t>({16, (size_t)(d.ngal2 / st.dnz), 1024 / tsz})) : 1;
    if (st.nseg > 1) AL(st.cpart, double, (size_t)st.cp * 2 * st.nseg * 6 * tsz);
    if (sc->spectra) {
        AL(st.spu, double, (size_t)d.nyu * d.ncol);
        AL(st.spv, double, (size_t)d.nyv * d.ncol);
        AL(st.spw, double, (size_t)d.nyu * d.ncol);
        AL(st.spuv, double, (size_t)d.nyu * d.ncol);
        AL(st.spp, double, (size_t)d.nyp * d.ncol);
    }
    st.on = true;
    return cfd_stats_reset(c);
}

int cfd_stats_reset(cfd_ctx* c) {
    if (!c) return CFD_ERR_ARG;
    const Dims& d = c->d;
    auto& st = c->st;
    if (!st.on) return fail(c, CFD_ERR_STATE, "statistics not configured");
    const size_t tsz = (size_t)st.dnx * st.dnz;
    CK(cudaMemsetAsync(st.su, 0, sizeof(double) * 6 * d.nyu, c->stream));
    CK(cudaMemsetAsync(st.sv, 0, sizeof(double) * 5 * d.nyv, c->stream));
    CK(cudaMemsetAsync(st.sp, 0, sizeof(double) * 2 * d.nyp, c->stream));
    if (tsz) {
        CK(cudaMemsetAsync(st.cu, 0, sizeof(double) * 2 * 6 * st.nbu * tsz, c->stream));
        CK(cudaMemsetAsync(st.cv, 0, sizeof(double) * 2 * 5 * st.nbv * tsz, c->stream));
        CK(cudaMemsetAsync(st.cp_, 0, sizeof(double) * 2 * 2 * st.nbp * tsz, c->stream));
    }
    if (st.spu) {
        const size_t nc = d.ncol;
        CK(cudaMemsetAsync(st.spu, 0, sizeof(double) * d.nyu * nc, c->stream));
        CK(cudaMemsetAsync(st.spv, 0, sizeof(double) * d.nyv * nc, c->stream));
        CK(cudaMemsetAsync(st.spw, 0, sizeof(double) * d.nyu * nc, c->stream));
        CK(cudaMemsetAsync(st.spuv, 0, sizeof(double) * d.nyu * nc, c->stream));
        CK(cudaMemsetAsync(st.spp, 0, sizeof(double) * d.nyp * nc, c->stream));
    }
    st.istat = 0;
    return CFD_OK;
}

int cfd_stats_accumulate(cfd_ctx* c) {
    if (!c) return CFD_ERR_ARG;
    if (!c->st.on) return fail(c, CFD_ERR_STATE, "statistics not configured");
    int s = stats_pass(c, true);
    if (s) return s;
    auto& st = c->st;
    if (st.spu) {
        const Dims& d = c->d;
        dim3 grid((d.ncol + 255) / 256, d.nyu);
        prof_mark(c);
        k_spectra<<<grid, 256, 0, c->stream>>>(d, c->g, c->u1, c->u2, c->u3, c->p, st.spu, st.spv, st.spw, st.spuv,
                                               st.spp);
        LK("k_spectra");
    }
    st.istat += 1;
    return CFD_OK;
}

int cfd_spectra_read(cfd_ctx* c, double* spu, double* spv, double* spw, double* spuv, double* spp) {
    if (!c) return CFD_ERR_ARG;
    const Dims& d = c->d;
    auto& st = c->st;
    if (!st.on || !st.spu) return fail(c, CFD_ERR_STATE, "spectra not configured");
    CK(cudaStreamSynchronize(c->stream));
    // device [plane][column] -> the reference's sp(j,column), j fastest
    std::vector<double> h;
    auto get = [&](double* out, const double* dev, int ny) -> int {
        if (!out) return CFD_OK;
        const size_t nc = d.ncol;
        h.resize((size_t)ny * nc);
        CK(cudaMemcpy(h.data(), dev, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
        for (int j = 0; j < ny; ++j)
            for (size_t col = 0; col < nc; ++col) out[col * ny + j] = h[(size_t)j * nc + col];
        return CFD_OK;
    };
    int s = get(spu, st.spu, d.nyu);
    if (!s) s = get(spv, st.spv, d.nyv);
    if (!s) s = get(spw, st.spw, d.nyu);
    if (!s) s = get(spuv, st.spuv, d.nyu);
    if (!s) s = get(spp, st.spp, d.nyp);
    return s;
}

int cfd_stats_read(cfd_ctx* c, double* u_sums, double* v_sums, double* p_sums, double* cu, double* cv, double* cp,
                   int32_t* istat) {
    if (!c) return CFD_ERR_ARG;
    const Dims& d = c->d;
    auto& st = c->st;
    if (!st.on) return fail(c, CFD_ERR_STATE, "statistics not configured");
    CK(cudaStreamSynchronize(c->stream));
    if (u_sums) CK(cudaMemcpy(u_sums, st.su, sizeof(double) * 6 * d.nyu, cudaMemcpyDeviceToHost));
    if (v_sums) CK(cudaMemcpy(v_sums, st.sv, sizeof(double) * 5 * d.nyv, cudaMemcpyDeviceToHost));
    if (p_sums) CK(cudaMemcpy(p_sums, st.sp, sizeof(double) * 2 * d.nyp, cudaMemcpyDeviceToHost));
    const size_t tsz = (size_t)st.dnx * st.dnz;
    // bottom band plus mirrored top band (xC + buffC of recvXC, stats.f90:491-509)
    auto combine = [&](double* out, const double* dev, size_t n) -> int {
        if (!out || !n) return CFD_OK;
        std::vector<double> h(2 * n);
        CK(cudaMemcpy(h.data(), dev, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) out[i] = h[i] + h[n + i];
        return CFD_OK;
    };
    int s = combine(cu, st.cu, (size_t)6 * st.nbu * tsz);
    if (!s) s = combine(cv, st.cv, (size_t)5 * st.nbv * tsz);
    if (!s) s = combine(cp, st.cp_, (size_t)2 * st.nbp * tsz);
    if (s) return s;
    if (istat) *istat = st.istat;
    return CFD_OK;
}

namespace {
int efail(cfd_ensemble* e, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (e) e->err = buf;
    return code;
}
#define ECK(call)                                                                        \
    do {                                                                                 \
        cudaError_t _e = (call);                                                         \
        if (_e != cudaSuccess) return efail(e, CFD_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

void ens_release_graph(cfd_ensemble* e) {
    if (e->gexec) cudaGraphExecDestroy(e->gexec);
    if (e->graph) cudaGraphDestroy(e->graph);
    e->gexec = nullptr;
    e->graph = nullptr;
}

// One RK3 step of every member as parallel branches of one graph on the master stream.
int ens_capture(cfd_ensemble* e) {
    ens_release_graph(e);
    ECK(cudaStreamBeginCapture(e->master, cudaStreamCaptureModeThreadLocal));
    cudaError_t ce = cudaEventRecord(e->fork, e->master);
    int st = ce == cudaSuccess ? CFD_OK : efail(e, CFD_ERR_CUDA, "fork: %s", cudaGetErrorString(ce));
    for (size_t i = 0; i < e->m.size() && st == CFD_OK; ++i) {
        cfd_ctx* c = e->m[i];
        cudaStream_t saved = c->stream;
        c->stream = e->streams[i];
        if ((ce = cudaStreamWaitEvent(c->stream, e->fork, 0)) != cudaSuccess) {
            st = efail(e, CFD_ERR_CUDA, "branch %zu: %s", i, cudaGetErrorString(ce));
        } else {
            const int64_t before = c->launches;
            c->capturing = true;
            for (int k = 1; k <= 3 && st == CFD_OK; ++k) st = substep_any(c, k);
            if (st == CFD_OK && c->ctpress == 1) st = meanflow_kernel(c, 1);
            c->capturing = false;
            c->launches = before;
            if (st != CFD_OK) efail(e, st, "member %zu: %s", i, c->err.c_str());
            else if ((ce = cudaEventRecord(e->join[i], c->stream)) != cudaSuccess ||
                     (ce = cudaStreamWaitEvent(e->master, e->join[i], 0)) != cudaSuccess)
                st = efail(e, CFD_ERR_CUDA, "join %zu: %s", i, cudaGetErrorString(ce));
        }
        c->stream = saved;
        e->epochs[i] = c->epoch;
    }
    cudaGraph_t g = nullptr;
    ce = cudaStreamEndCapture(e->master, &g);
    if (st != CFD_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (ce != cudaSuccess) return efail(e, CFD_ERR_CUDA, "ensemble capture: %s", cudaGetErrorString(ce));
    e->graph = g;
    ECK(cudaGraphInstantiate(&e->gexec, e->graph, 0));
    return CFD_OK;
}
}  // namespace

int cfd_ensemble_create(cfd_ctx* const* members, int32_t n, cfd_ensemble** out) {
    if (!out) return CFD_ERR_ARG;
    *out = nullptr;
    cfd_ensemble* e = new cfd_ensemble();
    *out = e;  // returned even on failure so cfd_ensemble_last_error can report
    if (!members || n <= 0) return efail(e, CFD_ERR_ARG, "need at least one member");
    for (int i = 0; i < n; ++i) {
        if (!members[i]) return efail(e, CFD_ERR_ARG, "member %d is NULL", i);
        for (int k = 0; k < i; ++k)
            if (members[k] == members[i]) return efail(e, CFD_ERR_ARG, "member %d repeated", i);
        if (members[i]->device != members[0]->device)
            return efail(e, CFD_ERR_ARG, "member %d is on device %d, member 0 on %d", i, members[i]->device,
                         members[0]->device);
        e->m.push_back(members[i]);
    }
    e->device = members[0]->device;
    ECK(cudaSetDevice(e->device));
    ECK(cudaStreamCreateWithFlags(&e->master, cudaStreamNonBlocking));
    ECK(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    ECK(cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming));
    e->streams.assign(n, nullptr);
    e->pre.assign(n, nullptr);
    e->join.assign(n, nullptr);
    e->epochs.assign(n, -1);
    for (int i = 0; i < n; ++i) {
        ECK(cudaStreamCreateWithFlags(&e->streams[i], cudaStreamNonBlocking));
        ECK(cudaEventCreateWithFlags(&e->pre[i], cudaEventDisableTiming));
        ECK(cudaEventCreateWithFlags(&e->join[i], cudaEventDisableTiming));
    }
    return CFD_OK;
}

int cfd_ensemble_step(cfd_ensemble* e, int32_t nsteps) {
    if (!e) return CFD_ERR_ARG;
    if (nsteps < 0) return efail(e, CFD_ERR_ARG, "nsteps < 0");
    ECK(cudaSetDevice(e->device));
    bool stale = !e->gexec;
    for (size_t i = 0; i < e->m.size(); ++i) {
        if (!e->m[i]->state_loaded) return efail(e, CFD_ERR_STATE, "member %zu has no state", i);
        if (e->m[i]->epoch != e->epochs[i]) stale = true;
    }
    // the members' pending work comes first
    for (size_t i = 0; i < e->m.size(); ++i) {
        ECK(cudaEventRecord(e->pre[i], e->m[i]->stream));
        ECK(cudaStreamWaitEvent(e->master, e->pre[i], 0));
    }
    if (stale) {
        int st = ens_capture(e);
        if (st != CFD_OK) return st;
    }
    for (int k = 0; k < nsteps; ++k) ECK(cudaGraphLaunch(e->gexec, e->master));
    // later work on a member's stream waits for the ensemble
    ECK(cudaEventRecord(e->done, e->master));
    for (cfd_ctx* c : e->m) ECK(cudaStreamWaitEvent(c->stream, e->done, 0));
    return CFD_OK;
}

int cfd_ensemble_synchronize(cfd_ensemble* e) {
    if (!e) return CFD_ERR_ARG;
    ECK(cudaStreamSynchronize(e->master));
    return CFD_OK;
}

int cfd_ensemble_stream(cfd_ensemble* e, void** stream) {
    if (!e || !stream) return CFD_ERR_ARG;
    *stream = (void*)e->master;
    return CFD_OK;
}

const char* cfd_ensemble_last_error(const cfd_ensemble* e) { return e ? e->err.c_str() : "null ensemble"; }

int cfd_ensemble_destroy(cfd_ensemble* e) {
    if (!e) return CFD_OK;
    cudaSetDevice(e->device);
    if (e->master) cudaStreamSynchronize(e->master);
    ens_release_graph(e);
    for (cudaStream_t s : e->streams) if (s) cudaStreamDestroy(s);
    for (cudaEvent_t v : e->pre) if (v) cudaEventDestroy(v);
    for (cudaEvent_t v : e->join) if (v) cudaEventDestroy(v);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->done) cudaEventDestroy(e->done);
    if (e->master) cudaStreamDestroy(e->master);
    delete e;
    return CFD_OK;
}

int cfd_set_dt(cfd_ctx* c, double dt) {
    if (!c) return CFD_ERR_ARG;
    if (!(dt > 0) || !std::isfinite(dt)) return fail(c, CFD_ERR_ARG, "dt must be positive and finite");
    CK(cudaStreamSynchronize(c->stream));
    c->dt = dt;
    c->epoch++;
    destroy_graph(c);
    return CFD_OK;
}

int cfd_set_lastplane(cfd_ctx* c, int32_t on) {
    if (!c) return CFD_ERR_ARG;
    if (on != 0 && on != 1) return fail(c, CFD_ERR_ARG, "lastplane must be 0 or 1");
    if (on && c->mb) return fail(c, CFD_ERR_ARG, "the single-slab term needs one band");
    CK(cudaStreamSynchronize(c->stream));
    c->lastplane = on;
    c->epoch++;
    destroy_graph(c);
    return CFD_OK;
}

int cfd_cfl(cfd_ctx* c, double* dtc, double* terms) {
    if (c && c->mb) return fail(c, CFD_ERR_ARG, "cfd_cfl of a three-band channel is not supported");
    if (!c || !dtc) return fail(c, CFD_ERR_ARG, "bad arguments");
    const Dims& d = c->d;
    int s = stats_scratch(c);
    if (!s) s = stats_pass(c, false);
    if (s) return s;
    std::vector<double> h((size_t)3 * d.nyu);
    CK(cudaStreamSynchronize(c->stream));  // the pass runs on the (non-blocking) context stream
    CK(cudaMemcpy(h.data(), c->st.mx, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    double um = 0.0, wm = 0.0, vm = 1e-6;
    bool bad = false;
    for (int j = 0; j < d.nyu; ++j) {
        bad = bad || !std::isfinite(h[j]) || !std::isfinite(h[d.nyu + j]);
        um = std::max(um, h[j]);
        wm = std::max(wm, h[d.nyu + j]);
    }
    for (int j = 1; j < d.nyv - 1; ++j) {
        bad = bad || !std::isfinite(h[2 * d.nyu + j]);
        vm = std::max(vm, h[2 * d.nyu + j]);
    }
    const double t0 = 1.0 / (c->alp * (d.n1 / 2) * um), t1 = 1.0 / (c->bet * (d.n2 / 2) * wm), t2 = 1.0 / vm;
    if (terms) { terms[0] = bad ? NAN : t0; terms[1] = bad ? NAN : t1; terms[2] = bad ? NAN : t2; }
    *dtc = bad ? NAN : std::min(t0, t1);
    if (bad) return fail(c, CFD_ERR_NONFINITE, "non-finite velocity in the physical planes");
    return CFD_OK;
}

int cfd_four_to_phys(cfd_ctx* c, double* planes, int32_t nplanes, int32_t zero_oddball) {
    if (!c || !planes || nplanes < 0) return fail(c, CFD_ERR_ARG, "bad arguments");
    const Dims& d = c->d;
    const long long ps = (long long)(d.ngal1 + 2) * d.ngal2;
    if (nplanes == 0) return CFD_OK;
    if (zero_oddball)
        CK(cudaMemset2DAsync(planes + (size_t)(d.ngal2 / 2) * (d.ngal1 + 2), ps * sizeof(double), 0,
                             (d.ngal1 + 2) * sizeof(double), nplanes, c->stream));
    int s = strided_cft(c, planes, d.ngal2, d.ngal1 + 2, 2, d.nkx, ps, nplanes, +1);
    if (s) return s;
    return strided_rft(c, planes, d.ngal1, d.ngal1 + 2, d.ngal2, ps, nplanes, +1);
}

int cfd_phys_to_four(cfd_ctx* c, double* planes, int32_t nplanes) {
    if (!c || !planes || nplanes < 0) return fail(c, CFD_ERR_ARG, "bad arguments");
    const Dims& d = c->d;
    const long long ps = (long long)(d.ngal1 + 2) * d.ngal2;
    if (nplanes == 0) return CFD_OK;
    int s = strided_rft(c, planes, d.ngal1, d.ngal1 + 2, d.ngal2, ps, nplanes, -1);
    if (s) return s;
    return strided_cft(c, planes, d.ngal2, d.ngal1 + 2, 2, d.nkx, ps, nplanes, -1);
}

int cfd_rft(cfd_ctx* c, double* cdev, int32_t isa, int32_t m, int32_t iopt) {
    if (!c || !cdev || m < 0 || isa < c->d.ngal1 + 2) return fail(c, CFD_ERR_ARG, "bad arguments (isa >= Ngal1+2)");
    if (m == 0) return CFD_OK;
    return strided_rft(c, cdev, c->d.ngal1, isa, m, 0, 1, iopt);
}

int cfd_cft(cfd_ctx* c, double* cdev, int32_t ise, int32_t isa, int32_t m, int32_t iopt) {
    if (!c || !cdev || m < 0 || ise < 2) return fail(c, CFD_ERR_ARG, "bad arguments (ise >= 2)");
    if (m == 0) return CFD_OK;
    return strided_cft(c, cdev, c->d.ngal2, ise, isa, m, 0, 1, iopt);
}

int cfd_profile(cfd_ctx* c, int32_t enable) {
    if (!c) return CFD_ERR_ARG;
    c->profiling = enable != 0;
    return CFD_OK;
}

int cfd_profile_read(cfd_ctx* c, char* buf, int32_t buflen) {
    if (!c || !buf || buflen <= 0) return CFD_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    std::vector<std::string> names;
    std::vector<double> ms;
    std::vector<long> calls;
    std::vector<cudaEvent_t> all;
    for (auto& r : c->prof) {
        all.push_back(r.second.second);
        if (r.first.empty()) continue;
        float t = 0.f;
        if (r.second.first && cudaEventElapsedTime(&t, r.second.first, r.second.second) != cudaSuccess) t = 0.f;
        size_t k = 0;
        while (k < names.size() && names[k] != r.first) ++k;
        if (k == names.size()) { names.push_back(r.first); ms.push_back(0.0); calls.push_back(0); }
        ms[k] += t;
        calls[k] += 1;
    }
    std::sort(all.begin(), all.end());
    all.erase(std::unique(all.begin(), all.end()), all.end());
    for (cudaEvent_t e : all) cudaEventDestroy(e);
    c->prof.clear();
    c->prof_last = nullptr;
    std::string out;
    char line[256];
    for (size_t k = 0; k < names.size(); ++k) {
        snprintf(line, sizeof(line), "%s %ld %.6f\n", names[k].c_str(), calls[k], ms[k]);
        out += line;
    }
    strncpy(buf, out.c_str(), (size_t)buflen - 1);
    buf[buflen - 1] = 0;
    return CFD_OK;
}

int cfd_launch_count(const cfd_ctx* c, int64_t* count) {
    if (!c || !count) return CFD_ERR_ARG;
    *count = c->launches;
    return CFD_OK;
}

}  // extern "C"
