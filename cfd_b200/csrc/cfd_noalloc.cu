// cfd_noalloc.cu - the one entry point of the library that allocates no device memory.
//
// Who needs it: a caller that cannot call cudaMalloc/cudaFree.  Typical cases are a host
// driver whose device memory is entirely owned by another allocator (a pool handed out by
// its own framework, or a process running under a hard device-memory cap), and a caller
// in a latency-critical loop that must not trigger the implicit device synchronisation of
// cudaFree.  Such a caller already holds its inputs and outputs on the device; the only
// thing missing for the u/w Helmholtz solve is the scratch of the Thomas sweep, which lives
// here in a fixed file-scope device array instead of a per-context allocation.
//
// Cost of that choice: every GPU that loads the library keeps the array (128 MiB) until the
// process exits, the problem size is capped by it, and all calls share it.

#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cfd_b200.h"

namespace {

// 16 Mi doubles = 128 MiB: enough for (nplanes-1) * columns up to 16,777,216, e.g. the
// 384 x 257 x 384 channel with 45 canopy planes per wall (347 x 33,024 = 11.5 M).
constexpr size_t kScratchDoubles = CFD_NOALLOC_MAX_SCRATCH;

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

// Host-side address of this device's copy of g_noalloc_scratch.  The symbol name seen by
// host code is only a stand-in, never a device address, so it is looked up once per device
// (with that device current) and cached.
int scratch_for_current_device(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CFD_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CFD_ERR_CUDA;
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_ptr[dev];
    return CFD_OK;
}

// Same sweep as the u/w part of k_solve_uvw (LUsolU with LU_buildU + LU_dec computed on
// the fly, tridLU_3D_IB.f90:50-103, 349-380, 521-559) for one right-hand side; the scaled
// upper diagonal of the forward sweep goes to `cs` (the file-scope scratch).  r and u may
// be the same array: plane jj of r is read before plane jj of u is written, and the back
// sweep reads u only, so they carry no __restrict__.
__global__ void __launch_bounds__(256) k_lusol_u_noalloc(int nkx, int n2, int n, double beta, double gwb, double gwt,
                                                         const double* __restrict__ kx, const double* __restrict__ kz,
                                                         const double* __restrict__ dyu2i,
                                                         const double2* r, double2* u,
                                                         double* __restrict__ cs) {
    const int ncol = nkx * n2;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int i = col % nkx, q = col / nkx;
    const double k2x = -kx[i] * kx[i], k2z = -kz[q] * kz[q];
    const size_t nc = (size_t)ncol;
    double dprev = 1.0;
    double a3prev = gwb;
    double2 y = r[col];
    u[col] = y;
    for (int jj = 1; jj < n; ++jj) {
        double a1, a2, a3;
        if (jj < n - 1) {
            a1 = -beta * dyu2i[3 * jj + 0];
            a2 = 1.0 - beta * (dyu2i[3 * jj + 1] + k2x + k2z);
            a3 = -beta * dyu2i[3 * jj + 2];
        } else {
            a1 = gwt;
            a2 = 1.0;
            a3 = 0.0;
        }
        const double csm = a3prev * dprev;
        cs[(size_t)(jj - 1) * nc + col] = csm;
        const double dj = 1.0 / (a2 - a1 * csm);
        const double2 rj = r[(size_t)jj * nc + col];
        y = make_double2(dj * (rj.x - a1 * y.x), dj * (rj.y - a1 * y.y));
        u[(size_t)jj * nc + col] = y;
        dprev = dj;
        a3prev = a3;
    }
    double2 x = y;
    for (int jj = n - 2; jj >= 0; --jj) {
        const double c = cs[(size_t)jj * nc + col];
        const double2 yj = u[(size_t)jj * nc + col];
        x = make_double2(yj.x - c * x.x, yj.y - c * x.y);
        u[(size_t)jj * nc + col] = x;
    }
}

}  // namespace

extern "C" int cfd_lusol_u_noalloc(int32_t nkx, int32_t n2, int32_t nplanes, double beta, double gw_bot,
                                   double gw_top, const double* kx_dev, const double* kz_dev,
                                   const double* dyu2i_dev, const double* rhs_dev, double* u_dev, void* stream) {
    if (nkx <= 0 || n2 <= 0 || nplanes < 3 || !kx_dev || !kz_dev || !dyu2i_dev || !rhs_dev || !u_dev)
        return CFD_ERR_ARG;
    const size_t ncol = (size_t)nkx * (size_t)n2;
    if (ncol > (size_t)0x7fffffff || ncol * (size_t)(nplanes - 1) > kScratchDoubles) return CFD_ERR_SIZE;
    double* cs = nullptr;
    int st = scratch_for_current_device(&cs);
    if (st != CFD_OK) return st;
    const unsigned blocks = (unsigned)((ncol + 255) / 256);
    k_lusol_u_noalloc<<<blocks, 256, 0, (cudaStream_t)stream>>>(nkx, n2, nplanes, beta, gw_bot, gw_top, kx_dev, kz_dev,
                                                               dyu2i_dev, reinterpret_cast<const double2*>(rhs_dev),
                                                               reinterpret_cast<double2*>(u_dev), cs);
    return cudaGetLastError() == cudaSuccess ? CFD_OK : CFD_ERR_CUDA;
}
