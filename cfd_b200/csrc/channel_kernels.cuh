// channel_kernels.cuh - sm_100a kernels of one RK3 substep of the LittleHarsh channel DNS.
//
// Device layout (HBM): a spectral field is [plane][column] complex, column = q*nkx + i
// (kx-mode i fastest, then kz-mode q), i.e. every y-plane is a contiguous (N2 x N1/2+1)
// array.  Thread-per-column kernels that march in y therefore read/write coalesced rows,
// and per-plane FFT kernels read contiguous planes: the reference's MPI transposes
// (modes_to_planes_* / planes_to_modes_*, FOU3D.f90:808-906, 1662-2170) disappear into
// this layout.
//
// Nonlinear term (FOU3D.f90:41-259, 1529-1617) in three passes over "half-physical"
// buffers H[slot][z][kx] (z physical, x still spectral; slot = u-plane or v-plane):
//   k_zinv  : y-interpolation (interp_u/v) + zero-padded inverse z transform
//   k_xline : inverse x transform, velocity products, forward x transform (fused)
//   k_zfwd  : forward z transform + truncation to the N2 retained modes
// and the column kernel k_rhs forms x/z/y derivatives and the RK right-hand side.
#pragma once

#include <type_traits>

#include "fft_smem.cuh"
#include "fft_reg.cuh"
#include "fft_pair.cuh"

namespace cfd {

struct Dims {
    int ngal1, ngal2, n1, n2, nkx, ncol;
    int ju0, ju1, jv0, jv1, jp0, jp1, nyu, nyv, nyp;
    int nslot;  // nyu + nyv
    int ny;     // faces from y=-1 to y=1 (input.in ny)
    // Stored layout of the spectral fields (the wall bands' column list) as seen by a launch
    // over one band (the transform kernels of the nonlinear pass): columns per plane, per kz
    // row, and the stored kz index q + qshift of the negative modes q >= n2/2; the elements
    // per slot of the half-physical buffers; the u-slots su0..su0+nsu-1 and v-slots
    // sv0..sv0+nsv-1 (0-based within their grid) of the launch.  With one band: ncol, nkx,
    // 0, ngal2*nkx, and every slot.
    int pstride, kstride, qshift;
    long long hstride;
    int su0, nsu, sv0, nsv;
    // three bands: 1, the last v face of the bottom band (N(3,1)) and the middle band's N1, N2
    int mb, jb, n1m, n2m;
};

// stored column of spectral entry (kx i, kz q) in a launch over one band
__device__ __forceinline__ size_t scol(const Dims& d, int i, int q) {
    return (size_t)(q < d.n2 / 2 ? q : q + d.qshift) * d.kstride + i;
}

// Grid and wavenumber tables on the device (array index = j - j0 of the grid).
struct Geo {
    const double* yu;
    const double* yv;
    const double* dthdyu;
    const double* dthdyv;
    const double* dyu2i;  // [nyu][3]
    const double* dyv2i;  // [nyv][3]
    const double* kx;     // [nkx]
    const double* kz;     // [n2]
    // linear y-interpolation weights (interp_u/interp_v, FOU3D.f90:261-308):
    // v at centre j = vca[j]*v(j) + vcb[j]*v(j-1)   (index j - ju0, interior centres)
    // u at face j   = ufa[j]*u(j+1) + ufb[j]*u(j)   (index j - jv0)
    const double* vca;
    const double* vcb;
    const double* ufa;
    const double* ufb;
    double gwb, gwt, gwib, gwit;
    double gw1t, gw3b;  // three bands: gridweighting(1,2) and gridweighting(3,1)
};

__device__ __forceinline__ int row_of(const Dims& d, int q) { return q < d.n2 / 2 ? q : q + (d.ngal2 - d.n2); }

__device__ __forceinline__ double2 dc(double a, double b) { double2 r; r.x = a; r.y = b; return r; }
__device__ __forceinline__ double2 dadd(double2 a, double2 b) { return dc(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 dsub(double2 a, double2 b) { return dc(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 dscl(double s, double2 a) { return dc(s * a.x, s * a.y); }
// (i*k) * a
__device__ __forceinline__ double2 dik(double k, double2 a) { return dc(-k * a.y, k * a.x); }

template <typename T2> __device__ __forceinline__ T2 to_t2(double2 a);
template <> __device__ __forceinline__ float2 to_t2<float2>(double2 a) { return make_float2((float)a.x, (float)a.y); }
template <> __device__ __forceinline__ double2 to_t2<double2>(double2 a) { return a; }
// max that keeps a NaN (fmax drops it), so that the reductions of the diagnostics see a
// non-finite field
__device__ __forceinline__ double nan_max(double a, double b) { return (b > a || b != b) ? b : a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return dc((double)a.x, (double)a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }

// --------------------------------------------------------------------------------------
// Pass 1: y-interpolation + inverse z transform (interp_u/interp_v FOU3D.f90:261-308,
// modes_to_planes_UVP, cft inverse of four_to_phys_u FOU3D.f90:546-572).
// grid: x = kx chunk of CH modes, y = slot (u-planes then v-planes), z = field 0..2
//   u-plane j: U = u1(j), W = u3(j), V = v interpolated to the centre (with ghost rows)
//   v-plane j: U = u1 interpolated to the face, W = u3 interpolated, V = u2(j)
// --------------------------------------------------------------------------------------
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_zinv(Dims d, Geo g, const double2* __restrict__ u1,
                                              const double2* __restrict__ u2, const double2* __restrict__ u3,
                                              T2* __restrict__ H0, T2* __restrict__ H1, T2* __restrict__ H2,
                                              FFTDesc fz, const T2* __restrict__ twz, int CH, int bshift) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)d.ngal2 * CH;
    T2* tw = buf1 + (size_t)d.ngal2 * CH;
    const int kx0 = blockIdx.x * CH;
    const int slot = blockIdx.y;
    const int f = blockIdx.z;
    const int n = d.ngal2;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
    for (int t = threadIdx.x; t < n * CH; t += blockDim.x) buf0[t] = cx<T2>(0, 0);
    __syncthreads();
    const bool uplane = slot < d.nyu;
    const int j = uplane ? d.ju0 + slot : d.jv0 + (slot - d.nyu);
    for (int t = threadIdx.x; t < (d.n2 << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), q = t >> bshift;
        const int i = kx0 + b;
        if (i >= d.nkx) continue;
        const size_t col = (size_t)q * d.nkx + i;
        double2 val;
        if (uplane) {
            if (f == 0) val = u1[(size_t)(j - d.ju0) * d.ncol + col];
            else if (f == 1) val = u3[(size_t)(j - d.ju0) * d.ncol + col];
            else {
                // interp_v (FOU3D.f90:296-304): v at centre j from faces j-1, j; ghosts extrapolated
                auto itp = [&](int jj) {
                    const double2 va = u2[(size_t)(jj - d.jv0) * d.ncol + col];
                    const double2 vb = u2[(size_t)(jj - 1 - d.jv0) * d.ncol + col];
                    const double wa = g.vca[jj - d.ju0], wb = g.vcb[jj - d.ju0];
                    return dc(wa * va.x + wb * vb.x, wa * va.y + wb * vb.y);
                };
                if (j == d.ju0) {
                    const double2 vi = itp(d.ju0 + 1);
                    const double2 vw = u2[(size_t)0 * d.ncol + col];
                    val = dadd(dscl(g.gwib, dsub(vw, vi)), vi);
                } else if (j == d.ju1) {
                    const double2 vi = itp(d.ju1 - 1);
                    const double2 vw = u2[(size_t)(d.jv1 - d.jv0) * d.ncol + col];
                    val = dadd(dscl(g.gwit, dsub(vw, vi)), vi);
                } else {
                    val = itp(j);
                }
            }
        } else {
            if (f == 2) val = u2[(size_t)(j - d.jv0) * d.ncol + col];
            else {
                // interp_u (FOU3D.f90:272-279): u at face j from centres j, j+1
                const double2* s = f == 0 ? u1 : u3;
                const double2 ua = s[(size_t)(j + 1 - d.ju0) * d.ncol + col];
                const double2 ub = s[(size_t)(j - d.ju0) * d.ncol + col];
                const double wa = g.ufa[j - d.jv0], wb = g.ufb[j - d.jv0];
                val = dc(wa * ua.x + wb * ub.x, wa * ua.y + wb * ub.y);
            }
        }
        buf0[swz(row_of(d, q), b, bshift)] = to_t2<T2>(val);
    }
    __syncthreads();
    T2* res = fft_batch<T2, NF, +1>(buf0, buf1, CH, bshift, fz, tw);
    T2* H = f == 0 ? H0 : (f == 1 ? H1 : H2);
    const size_t base = (size_t)slot * n * d.nkx;
    for (int t = threadIdx.x; t < (n << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), z = t >> bshift;
        const int i = kx0 + b;
        if (i < d.nkx) H[base + (size_t)z * d.nkx + i] = res[swz(z, b, bshift)];
    }
}

// --------------------------------------------------------------------------------------
// Pass 2: per z-row of a plane, inverse real x transform (rft inverse), products, forward
// real x transform (rft forward, x 1/Ngal1), truncation to kx <= N1/2
// (ops_in_planes FOU3D.f90:1553-1569, 1588-1600).  Two real rows share one complex
// transform: line = A + i*B with A, B the Hermitian spectra of two real signals.
// u-plane: (u + i w), (v + i 0) -> (uu + i uw), (vv + i ww)
// v-plane: (u + i w), (v + i 0) -> (uv + i vw)
// grid: x = chunk of RW rows, y = slot
// --------------------------------------------------------------------------------------
template <typename T2>
__device__ __forceinline__ T2 herm_line(const Dims& d, const T2* A, const T2* B, int k) {
    // entry k (0..Ngal1-1) of the complex line A + iB from kx-spectra A, B (i = 0..N1/2);
    // the rft inverse ignores Im of the kx = 0 entry (rft_buff.f:78-80)
    using R = decltype(T2::x);
    const int h = d.n1 / 2;
    if (k <= h) {
        T2 a = A ? A[k] : cx<T2>(0, 0);
        T2 b = B ? B[k] : cx<T2>(0, 0);
        if (k == 0) { a.y = 0; b.y = 0; }
        return cx<T2>(a.x - b.y, a.y + b.x);
    }
    if (k >= d.ngal1 - h) {
        const int kk = d.ngal1 - k;
        T2 a = A ? A[kk] : cx<T2>(0, 0);
        T2 b = B ? B[kk] : cx<T2>(0, 0);
        return cx<T2>(a.x + b.y, -a.y + b.x);
    }
    return cx<T2>((R)0, (R)0);
}

template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_xline(Dims d, T2* __restrict__ H0, T2* __restrict__ H1, T2* __restrict__ H2,
                                               T2* __restrict__ H3, FFTDesc fx, const T2* __restrict__ twx, int RW,
                                               int bshift) {
    using R = decltype(T2::x);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal1;
    const int B = 2 * RW;  // line 2*rr = (u + i w) of row rr, line 2*rr+1 = (v + i 0)
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * B;
    T2* tw = buf1 + (size_t)n * B;
    // the launch's u-slots, then its v-slots
    const int by = blockIdx.y;
    const int slot = by < d.nsu ? d.su0 + by : d.nyu + d.sv0 + (by - d.nsu);
    const int z0 = blockIdx.x * RW;
    const bool uplane = slot < d.nyu;
    const int h = d.n1 / 2;  // retained kx modes 0..h
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twx[t];
    // zero the padding modes h < k < n-h of every line
    const int ngap = n - 2 * h - 1;
    for (int t = threadIdx.x; t < ngap * B; t += blockDim.x) {
        const int b = t & (B - 1), k = h + 1 + (t >> bshift);
        buf0[swz(k, b, bshift)] = cx<T2>((R)0, (R)0);
    }
    // Hermitian lines from the kx spectra, k fastest across threads (coalesced rows);
    // the rft inverse ignores Im of the kx = 0 entry (rft_buff.f:78-80)
    const size_t pbase = (size_t)slot * d.hstride;
    const int nk = d.nkx;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int b = warp; b < B; b += nwarp) {
        const int rr = b >> 1, which = b & 1;
        const T2* ra = (which == 0 ? H0 : H2) + pbase + (size_t)(z0 + rr) * nk;
        const T2* rc = H1 + pbase + (size_t)(z0 + rr) * nk;
        for (int k = lane; k < nk; k += 32) {
            T2 a = ra[k];
            T2 c = which == 0 ? rc[k] : cx<T2>((R)0, (R)0);
            if (k == 0) { a.y = 0; c.y = 0; }
            buf0[swz(k, b, bshift)] = cx<T2>(a.x - c.y, a.y + c.x);
            if (k > 0) buf0[swz(n - k, b, bshift)] = cx<T2>(a.x + c.y, -a.y + c.x);
        }
    }
    __syncthreads();
    T2* P = fft_batch<T2, NF, +1>(buf0, buf1, B, bshift, fx, tw);
    T2* Q = P == buf0 ? buf1 : buf0;
    for (int t = threadIdx.x; t < n * RW; t += blockDim.x) {
        const int rr = t & (RW - 1), k = t >> (bshift - 1);
        const int a0 = swz(k, 2 * rr, bshift), a1 = swz(k, 2 * rr + 1, bshift);
        const T2 l0 = P[a0], l1 = P[a1];
        const R u = l0.x, w = l0.y, v = l1.x;
        if (uplane) {
            P[a0] = cx<T2>(u * u, u * w);
            P[a1] = cx<T2>(v * v, w * w);
        } else {
            P[a0] = cx<T2>(u * v, w * v);
            P[a1] = cx<T2>((R)0, (R)0);
        }
    }
    __syncthreads();
    T2* F = fft_batch<T2, NF, -1>(P, Q, B, bshift, fx, tw);
    const R s = (R)1 / (R)n;
    const int nl = uplane ? B : RW;  // v-planes carry one output line per row
    const R hs = (R)0.5 * s;
    for (int bl = warp; bl < nl; bl += nwarp) {
        const int b = uplane ? bl : 2 * bl;
        const int rr = b >> 1, which = b & 1;
        T2* oa = (which == 0 ? H0 : H2) + pbase + (size_t)(z0 + rr) * nk;
        T2* ob = (which == 0 ? H1 : H3) + pbase + (size_t)(z0 + rr) * nk;
        for (int k = lane; k < nk; k += 32) {
            const T2 Pk = F[swz(k, b, bshift)];
            const T2 Qc = cconj(F[swz(k == 0 ? 0 : n - k, b, bshift)]);
            oa[k] = cx<T2>((Pk.x + Qc.x) * hs, (Pk.y + Qc.y) * hs);
            ob[k] = cx<T2>((Pk.y - Qc.y) * hs, -(Pk.x - Qc.x) * hs);
        }
    }
}

// Pass 2 with the register-resident two-step transform (N = N1*N2, fft_reg.cuh).  A CTA
// holds RW rows = B = 2*RW lines (line 2r = u + i v, line 2r+1 = w + i 0) and runs with
// B*max(N1,N2) threads:
//   step 1  thread (b, n2): reads its stride-N2 subsequence of the Hermitian-extended
//           spectrum straight from global memory, N1-point DFT, twiddle, exchange
//   step 2  thread (b, k1): N2-point DFT -> physical x = k1 + N1*k2 in registers; the two
//           lines of a row sit in adjacent lanes and pass one value with a shuffle, form
//           the products, and start the forward transform from registers (N2-point DFT):
//             u-plane: line 2r -> uu + i vv, line 2r+1 -> ww + i uw (u from lane 2r)
//             v-plane: line 2r -> uv + i vw (w from lane 2r+1), line 2r+1 unused
//   step 2' thread (b, kb): N1-point DFT -> X[kb + N2*ka]; unpack the two real spectra.
// The retained modes are kx = 0..N/3 (N1 = 2*(Ngal1/3)), a compile-time bound, so which
// elements of a subsequence are zero, direct or conjugated is resolved at compile time
// except in the two blocks that straddle a boundary.
template <typename T2, int N1, int N2, int TPAD = 1>
__device__ __forceinline__ void xline2_body(Dims d, Geo g, const T2* __restrict__ Hx, T2* __restrict__ H0, T2* __restrict__ H1, T2* __restrict__ H2,
                         T2* __restrict__ H3, const T2* __restrict__ twx, int RW, int lrw) {
    using R = decltype(T2::x);
    constexpr int N = N1 * N2;
    constexpr int HX = N / 3;               // highest retained kx
    constexpr int NK = HX + 1;              // kx columns per row (= d.nkx)
    constexpr int L1 = N1 * (N2 + 1) + 1;  // inverse exchange, per line: [k1][n2]
    constexpr int L2 = N2 * (N1 + 1) + 1;  // forward exchange, per line: [kb][na]
    constexpr int LU = N + 1;               // unpack buffer, per line
    constexpr int LX = (L1 > L2 ? (L1 > LU ? L1 : LU) : (L2 > LU ? L2 : LU));
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int B = 2 * RW;
    T2* ex = reinterpret_cast<T2*>(smem_raw);       // B * LX
    // twt[b*(N2+TPAD) + a] = w^(a*b), a < N2, b < N1; an odd row pitch (TPAD = 1) keeps the
    // lanes of a step-2 wavefront, which read two or more rows b at once, in distinct banks
    constexpr int TP = N2 + TPAD;
    T2* twt = ex + (size_t)B * LX;
    // u- and v-slots interleaved in y (nyu = nyv + 1), so that the y-neighbour planes read
    // by the interpolation are still in L2 from the adjacent slots
    const int slot = (blockIdx.y & 1) ? d.nyu + (blockIdx.y >> 1) : (blockIdx.y >> 1);
    const int z0 = blockIdx.x * RW;
    const bool uplane = slot < d.nyu;
    const int t = threadIdx.x;
    for (int i = t; i < N; i += blockDim.x) {
        const int b = i / N2, a = i - b * N2;
        twt[TPAD ? b * TP + a : i] = twx[(a * b) % N];
    }
    const size_t pbase = (size_t)slot * d.ngal2 * NK;
    // y-interpolated sources of this slot, each ca * plane a + cb * plane b of Hx:
    // u-plane j: u, w direct; v at the centre (ghost centres: the extrapolation of
    // FOU3D.f90:261-283 folded into the weights).  v-plane j: v direct; u, w at the face.
    const size_t pls = (size_t)d.ngal2 * NK;
    const T2* Hu = Hx;
    const T2* Hw = Hx + (size_t)d.nyu * pls;
    const T2* Hv = Hx + (size_t)(2 * d.nyu) * pls;
    const T2 *ua, *ub, *va, *vb, *wa, *wb;
    R uca = 1, ucb = 0, vca = 1, vcb = 0;
    if (uplane) {
        const int sl = slot;
        ua = ub = Hu + sl * pls;
        wa = wb = Hw + sl * pls;
        double ca, cb;
        int pa;
        if (sl == 0) {
            pa = 1; ca = (1.0 - g.gwib) * g.vca[1]; cb = g.gwib + (1.0 - g.gwib) * g.vcb[1];
        } else if (sl == d.nyu - 1) {
            pa = sl - 1; ca = g.gwit + (1.0 - g.gwit) * g.vca[sl - 1]; cb = (1.0 - g.gwit) * g.vcb[sl - 1];
        } else {
            pa = sl; ca = g.vca[sl]; cb = g.vcb[sl];
        }
        va = Hv + pa * pls; vb = va - pls; vca = (R)ca; vcb = (R)cb;
    } else {
        const int sl = slot - d.nyu;
        va = vb = Hv + sl * pls;
        ua = Hu + (sl + 1) * pls; ub = ua - pls;
        wa = Hw + (sl + 1) * pls; wb = wa - pls;
        uca = (R)g.ufa[sl]; ucb = (R)g.ufb[sl];
    }
    __syncthreads();

    // ---- step 1: inverse, thread (b, n2)
    if (t < B * N2) {
        const int b = (unsigned)t / N2, n2 = t - b * N2;
        const int rr = b >> 1, which = b & 1;
        const size_t ro = (size_t)(z0 + rr) * NK;
        // line 2r: A = u, C = v; line 2r+1: A = w.  u-plane: C interpolated; v-plane: A
        const T2* A0 = (which == 0 ? ua : wa) + ro;
        const T2* A1 = (which == 0 ? ub : wb) + ro;
        const T2* C0 = va + ro;
        const T2* C1 = vb + ro;
        const bool hasc = which == 0;
        T2 v[N1];
        // the uniform branch on the plane type sits outside the element loop, so that the
        // loads of all elements are straight-line (predicated) and issue back to back
        auto fill = [&](auto vplane) {
            constexpr bool VP = decltype(vplane)::value;
            auto fetch = [&](int k, T2& a, T2& c) {
                const T2 z = cx<T2>((R)0, (R)0);
                if (VP) {
                    const T2 a0 = A0[k], a1 = A1[k];
                    a = cx<T2>(uca * a0.x + ucb * a1.x, uca * a0.y + ucb * a1.y);
                    c = hasc ? C0[k] : z;
                } else {
                    a = A0[k];
                    const T2 c0 = hasc ? C0[k] : z, c1 = hasc ? C1[k] : z;
                    c = cx<T2>(vca * c0.x + vcb * c1.x, vca * c0.y + vcb * c1.y);
                }
            };
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                const int e0 = n1 * N2, e = e0 + n2;
                const bool lo = (e0 + N2 - 1 <= HX) || (e0 <= HX && e <= HX);
                const bool hi = (e0 >= N - HX) || (e0 + N2 - 1 >= N - HX && e >= N - HX);
                T2 val = cx<T2>((R)0, (R)0);
                T2 a, c;
                if (lo) {  // A_e + i C_e; the rft inverse ignores Im of the kx = 0 entries
                    fetch(e, a, c);
                    if (n1 == 0 && n2 == 0) { a.y = 0; c.y = 0; }
                    val = cx<T2>(a.x - c.y, a.y + c.x);
                } else if (hi) {  // conj(A_k) + i conj(C_k), k = N - e
                    fetch(N - e, a, c);
                    val = cx<T2>(a.x + c.y, -a.y + c.x);
                }
                v[n1] = val;
            }
        };
        if (uplane) fill(std::false_type{});
        else fill(std::true_type{});
        rdft_z<N1, +1, gap_blocks<N1, N2, HX>()>(v);
        T2* o = ex + (size_t)b * L1 + n2;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) o[k1 * (N2 + 1)] = k1 == 0 ? v[0] : cmulc(v[k1], twt[k1 * TP + n2]);
    }
    __syncthreads();

    // ---- step 2: inverse N2-point DFT, products, forward N2-point DFT; thread (b, k1)
    T2 y[N2];
    const bool act2 = t < B * N1;
    const int par = t & 1, rest = t >> 1;
    const int rr2 = rest & (RW - 1), k1 = rest >> lrw;
    const int b2 = 2 * rr2 + par;
    if (act2) {
        const T2* o = ex + (size_t)b2 * L1 + k1 * (N2 + 1);
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) y[n2] = o[n2];
        rdft<N2, +1>(y);
        // lane pair (u + i v, w + i 0); each lane passes its real part to the other:
        // u-plane (a*a, b*b) on the even lane, (a*a, a*o) on the odd lane; v-plane (a*b, b*o)
        const bool sa = uplane && par, sb = uplane && !par;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            const R a = y[k2].x, b = y[k2].y;
            const R o = __shfl_xor_sync(0xffffffffu, a, 1);
            y[k2] = cx<T2>(a * (uplane ? a : b), (sa ? a : b) * (sb ? b : o));
        }
        rdft<N2, -1>(y);
#pragma unroll
        for (int kb = 1; kb < N2; ++kb) y[kb] = cmul(y[kb], twt[k1 * TP + kb]);
    }
    __syncthreads();  // every lane has read the inverse exchange
    if (act2) {
        T2* o = ex + (size_t)b2 * L2 + k1;
#pragma unroll
        for (int kb = 0; kb < N2; ++kb) o[kb * (N1 + 1)] = y[kb];
    }
    __syncthreads();

    // ---- step 2': forward N1-point DFT, thread (b, kb) -> X[kb + N2*ka]; even lines take
    // the first RW*N2 threads, so on v-planes (odd lines are zero) whole warps drop out
    T2 z[N1];
    const int kb = t % N2, i3 = t / N2;
    const int b3 = i3 < RW ? 2 * i3 : 2 * (i3 - RW) + 1;
    const bool act3 = t < B * N2 && (uplane || i3 < RW);
    if (act3) {
        const T2* o = ex + (size_t)b3 * L2 + kb * (N1 + 1);
#pragma unroll
        for (int na = 0; na < N1; ++na) z[na] = o[na];
        rdft<N1, -1>(z);
    }
    __syncthreads();
    if (act3) {
        T2* o = ex + (size_t)b3 * LU + kb;
        // X[kb + N2*ka] is read by the unpack only for k <= HX or k >= N - HX; the blocks of
        // ka that lie wholly between are not stored, so their last butterflies are dead code
#pragma unroll
        for (int ka = 0; ka < N1; ++ka)
            if (!(N2 * ka > HX && N2 * ka + N2 - 1 < N - HX)) o[N2 * ka] = z[ka];
    }
    __syncthreads();

    // ---- unpack A_k = (P_k + conj P_{N-k})/2, B_k = (P_k - conj P_{N-k})/(2i), x 1/N;
    // work items (line, k) flattened so that no lane idles on a partial last chunk
    const R hs = (R)0.5 / (R)N;
    const int nl = uplane ? B : RW;
    for (int it = t; it < nl * NK; it += blockDim.x) {
        const int bl = (unsigned)it / NK, k = it - bl * NK;
        const int b = uplane ? bl : 2 * bl;
        const int rr = b >> 1, which = b & 1;
        const size_t o = pbase + (size_t)(z0 + rr) * NK + k;
        const T2* line = ex + (size_t)b * LU;
        const T2 Pk = line[k];
        const T2 Qc = cconj(line[k == 0 ? 0 : N - k]);
        // real parts: u-plane uu / ww, v-plane uv; imaginary parts: u-plane vv / uw, v-plane vw
        T2* da = which == 0 ? H0 : H3;
        T2* db = which == 0 ? (uplane ? H2 : H1) : H1;
        da[o] = cx<T2>((Pk.x + Qc.x) * hs, (Pk.y + Qc.y) * hs);
        db[o] = cx<T2>((Pk.y - Qc.y) * hs, -(Pk.x - Qc.x) * hs);
    }
}

template <typename T2, int N1, int N2>
__global__ void __launch_bounds__(16 * (N1 > N2 ? N1 : N2), (sizeof(T2) == 8 && (N1 > N2 ? N1 : N2) <= 24) ? 2 : 1) k_xline2(Dims d, Geo g, const T2* __restrict__ Hx, T2* __restrict__ H0, T2* __restrict__ H1, T2* __restrict__ H2,
                         T2* __restrict__ H3, const T2* __restrict__ twx, int RW, int lrw) {
    xline2_body<T2, N1, N2>(d, g, Hx, H0, H1, H2, H3, twx, RW, lrw);
}

// The FP32 x-line kernel held to 64 registers per thread: with 4 rows per CTA (192 threads
// at the 24 x 16 split of 384) five CTAs fit on an SM instead of four (x-line path 5).  The
// FP64 kernel capped at 112 registers (three CTAs instead of two) measured slower at re550
// (1.72 against 1.53 ms per launch) and is not built.
template <int N1, int N2>
__global__ void __maxnreg__(64) k_xline2r(Dims d, Geo g, const float2* __restrict__ Hx, float2* __restrict__ H0,
                                          float2* __restrict__ H1, float2* __restrict__ H2, float2* __restrict__ H3,
                                          const float2* __restrict__ twx, int RW, int lrw) {
    xline2_body<float2, N1, N2, 0>(d, g, Hx, H0, H1, H2, H3, twx, RW, lrw);  // unpadded: no spill at 64
}

// Pass 2 on packed line pairs (FP32 only).  The two lines of a row (u + i v, w + i 0) travel
// together, one cpair per element (fft_pair.cuh), so every DFT instruction of k_xline2
// serves both lines through the .f32x2 instructions.  A CTA holds RW rows and runs with
// RW*max(N1,N2) threads: the steps of k_xline2 with one thread per row where k_xline2 has
// one per line, and the products formed inside the thread instead of across a lane pair.
// On v-planes the second line of the forward transform is idle (one product line per row).
template <int N1, int N2>
__global__ void __launch_bounds__(8 * (N1 > N2 ? N1 : N2)) k_xline4(Dims d, Geo g, const float2* __restrict__ Hx,
                                                                     float2* __restrict__ H0, float2* __restrict__ H1,
                                                                     float2* __restrict__ H2, float2* __restrict__ H3,
                                                                     const float2* __restrict__ twx, int RW) {
    using T2 = float2;
    using R = float;
    constexpr int N = N1 * N2;
    constexpr int HX = N / 3;
    constexpr int NK = HX + 1;
    constexpr int L1 = N1 * (N2 + 1) + 1;  // inverse exchange, per row: [k1][n2]
    constexpr int L2 = N2 * (N1 + 1) + 1;  // forward exchange, per row: [kb][na]
    constexpr int LU = N + 1;               // unpack buffer, per row
    constexpr int LX = (L1 > L2 ? (L1 > LU ? L1 : LU) : (L2 > LU ? L2 : LU));
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpair* ex = reinterpret_cast<cpair*>(smem_raw);  // RW * LX
    cpair* twt = ex + (size_t)RW * LX;               // N: twt[b*N2 + a] = w^(a*b) in both lanes
    const int slot = (blockIdx.y & 1) ? d.nyu + (blockIdx.y >> 1) : (blockIdx.y >> 1);
    const int z0 = blockIdx.x * RW;
    const bool uplane = slot < d.nyu;
    const int t = threadIdx.x;
    for (int i = t; i < N; i += blockDim.x) {
        const int b = i / N2, a = i - b * N2;
        const T2 w = twx[(a * b) % N];
        twt[i] = cpair{f2b(w.x), f2b(w.y)};
    }
    const size_t pbase = (size_t)slot * d.ngal2 * NK;
    const size_t pls = (size_t)d.ngal2 * NK;
    const T2* Hu = Hx;
    const T2* Hw = Hx + (size_t)d.nyu * pls;
    const T2* Hv = Hx + (size_t)(2 * d.nyu) * pls;
    const T2 *ua, *ub, *va, *vb, *wa, *wb;
    R uca = 1, ucb = 0, vca = 1, vcb = 0;
    if (uplane) {
        const int sl = slot;
        ua = ub = Hu + sl * pls;
        wa = wb = Hw + sl * pls;
        double ca, cb;
        int pa;
        if (sl == 0) {
            pa = 1; ca = (1.0 - g.gwib) * g.vca[1]; cb = g.gwib + (1.0 - g.gwib) * g.vcb[1];
        } else if (sl == d.nyu - 1) {
            pa = sl - 1; ca = g.gwit + (1.0 - g.gwit) * g.vca[sl - 1]; cb = (1.0 - g.gwit) * g.vcb[sl - 1];
        } else {
            pa = sl; ca = g.vca[sl]; cb = g.vcb[sl];
        }
        va = Hv + pa * pls; vb = va - pls; vca = (R)ca; vcb = (R)cb;
    } else {
        const int sl = slot - d.nyu;
        va = vb = Hv + sl * pls;
        ua = Hu + (sl + 1) * pls; ub = ua - pls;
        wa = Hw + (sl + 1) * pls; wb = wa - pls;
        uca = (R)g.ufa[sl]; ucb = (R)g.ufb[sl];
    }
    __syncthreads();

    // ---- step 1: inverse, thread (row r, n2)
    if (t < RW * N2) {
        const int r = (unsigned)t / N2, n2 = t - r * N2;
        const size_t ro = (size_t)(z0 + r) * NK;
        const T2 *A0 = ua + ro, *A1 = ub + ro, *C0 = va + ro, *C1 = vb + ro, *W0 = wa + ro, *W1 = wb + ro;
        cpair v[N1];
        auto fill = [&](auto vplane) {
            constexpr bool VP = decltype(vplane)::value;
            auto fetch = [&](int k, T2& a, T2& c, T2& w) {
                if (VP) {
                    const T2 a0 = A0[k], a1 = A1[k], w0 = W0[k], w1 = W1[k];
                    a = cx<T2>(uca * a0.x + ucb * a1.x, uca * a0.y + ucb * a1.y);
                    w = cx<T2>(uca * w0.x + ucb * w1.x, uca * w0.y + ucb * w1.y);
                    c = C0[k];
                } else {
                    a = A0[k];
                    w = W0[k];
                    const T2 c0 = C0[k], c1 = C1[k];
                    c = cx<T2>(vca * c0.x + vcb * c1.x, vca * c0.y + vcb * c1.y);
                }
            };
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) {
                const int e0 = n1 * N2, e = e0 + n2;
                const bool lo = (e0 + N2 - 1 <= HX) || (e0 <= HX && e <= HX);
                const bool hi = (e0 >= N - HX) || (e0 + N2 - 1 >= N - HX && e >= N - HX);
                cpair val = cpair{f2b(0.0f), f2b(0.0f)};
                T2 a, c, w;
                if (lo) {  // (A_e + i C_e, W_e); the rft inverse ignores Im of the kx = 0 entries
                    fetch(e, a, c, w);
                    if (n1 == 0 && n2 == 0) { a.y = 0; c.y = 0; w.y = 0; }
                    val = cpair{f2p(a.x - c.y, w.x), f2p(a.y + c.x, w.y)};
                } else if (hi) {  // (conj A_k + i conj C_k, conj W_k), k = N - e
                    fetch(N - e, a, c, w);
                    val = cpair{f2p(a.x + c.y, w.x), f2p(c.x - a.y, -w.y)};
                }
                v[n1] = val;
            }
        };
        if (uplane) fill(std::false_type{});
        else fill(std::true_type{});
        rdft<N1, +1>(v);
        cpair* o = ex + (size_t)r * L1 + n2;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) o[k1 * (N2 + 1)] = k1 == 0 ? v[0] : cmulc(v[k1], twt[k1 * N2 + n2]);
    }
    __syncthreads();

    // ---- step 2: inverse N2-point DFT, products, forward N2-point DFT; thread (row, k1)
    cpair y[N2];
    const bool act2 = t < RW * N1;
    const int k1 = t % N1, r2 = t / N1;
    if (act2) {
        const cpair* o = ex + (size_t)r2 * L1 + k1 * (N2 + 1);
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) y[n2] = o[n2];
        rdft<N2, +1>(y);
        // lanes (u, w) in x and (v, -) in y.  u-plane: (uu + i vv, ww + i uw); v-plane:
        // (uv + i vw, idle)
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
            const R u = y[k2].x.v.x, w = y[k2].x.v.y, vv = y[k2].y.v.x;
            if (uplane) y[k2] = cpair{mul2(y[k2].x, y[k2].x), f2p(vv * vv, u * w)};
            else y[k2] = cpair{f2p(u * vv, 0.0f), f2p(vv * w, 0.0f)};
        }
        rdft<N2, -1>(y);
#pragma unroll
        for (int kb = 1; kb < N2; ++kb) y[kb] = cmul(y[kb], twt[k1 * N2 + kb]);
    }
    __syncthreads();  // every thread has read the inverse exchange
    if (act2) {
        cpair* o = ex + (size_t)r2 * L2 + k1;
#pragma unroll
        for (int kb = 0; kb < N2; ++kb) o[kb * (N1 + 1)] = y[kb];
    }
    __syncthreads();

    // ---- step 2': forward N1-point DFT, thread (row, kb) -> X[kb + N2*ka]
    cpair z[N1];
    const int kb = t % N2, r3 = t / N2;
    const bool act3 = t < RW * N2;
    if (act3) {
        const cpair* o = ex + (size_t)r3 * L2 + kb * (N1 + 1);
#pragma unroll
        for (int na = 0; na < N1; ++na) z[na] = o[na];
        rdft<N1, -1>(z);
    }
    __syncthreads();
    if (act3) {
        cpair* o = ex + (size_t)r3 * LU + kb;
#pragma unroll
        for (int ka = 0; ka < N1; ++ka) o[N2 * ka] = z[ka];
    }
    __syncthreads();

    // ---- unpack both lines: A_k = (P_k + conj P_{N-k})/2, B_k = (P_k - conj P_{N-k})/(2i), x 1/N
    const f2x hs = f2b((R)0.5 / (R)N);
    for (int it = t; it < RW * NK; it += blockDim.x) {
        const int r = (unsigned)it / NK, k = it - r * NK;
        const size_t o = pbase + (size_t)(z0 + r) * NK + k;
        const cpair* line = ex + (size_t)r * LU;
        const cpair P = line[k], Q = line[k == 0 ? 0 : N - k];
        const f2x ax = mul2(add2(P.x, Q.x), hs), ay = mul2(sub2(P.y, Q.y), hs);
        const f2x bx = mul2(add2(P.y, Q.y), hs), by = mul2(sub2(Q.x, P.x), hs);
        // lane 0: u-plane uu / vv, v-plane uv / vw; lane 1 (u-plane): ww / uw
        H0[o] = cx<T2>(ax.v.x, ay.v.x);
        if (uplane) {
            H2[o] = cx<T2>(bx.v.x, by.v.x);
            H3[o] = cx<T2>(ax.v.y, ay.v.y);
            H1[o] = cx<T2>(bx.v.y, by.v.y);
        } else {
            H1[o] = cx<T2>(bx.v.x, by.v.x);
        }
    }
}

// Pass 2, packed form.  Three real inputs per row take 1.5 complex lines instead of 2: a
// CTA holds RW rows as RW/2 row pairs (r0, r1) with three inverse lines each
//   u-plane: u_r0 + i v_r0,  u_r1 + i v_r1,  w_r0 + i w_r1
//   v-plane: u_r0 + i w_r0,  u_r1 + i w_r1,  v_r0 + i v_r1
// (v on u-planes and u, w on v-planes y-interpolated as in k_xline2).  The inverse
// transforms land in shared memory as physical rows; the forward lines are formed from them
//   u-plane: uu + i vv per row, ww + i uw per row;   v-plane: uv + i vw per row
// so v-planes run one forward line per row.  Both directions are two_step_lines
// (element-fastest thread mapping, coalesced x-rows); the unpack writes the products to
// H0..H3 as k_xline2 does.
template <typename T2, int N1, int N2>
__global__ void __launch_bounds__(16 * (N1 > N2 ? N1 : N2), (sizeof(T2) == 8 && (N1 > N2 ? N1 : N2) <= 24) ? 2 : 1)
    k_xline3(Dims d, Geo g, const T2* __restrict__ Hx, T2* __restrict__ H0, T2* __restrict__ H1,
             T2* __restrict__ H2, T2* __restrict__ H3, const T2* __restrict__ twx, int RW) {
    using R = decltype(T2::x);
    constexpr int N = N1 * N2;
    constexpr int HX = N / 3, NK = HX + 1;
    constexpr int LX = exch_row<N1, N2>();
    constexpr int LU = N + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int NP = RW >> 1, NLI = 3 * NP;
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;                   // exchange of two_step_lines, 2*RW lines
    T2* PU = ex + (size_t)2 * RW * LX;  // physical rows [NLI][N], then forward spectra [NLF][LU]
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int b = i / N2, a = i - b * N2;
        twt[i] = twx[(a * b) % N];
    }
    const int slot = (blockIdx.y & 1) ? d.nyu + (blockIdx.y >> 1) : (blockIdx.y >> 1);
    const bool uplane = slot < d.nyu;
    const int z0 = blockIdx.x * RW;
    const int NLF = uplane ? 4 * NP : 2 * NP;
    const size_t pls = (size_t)d.ngal2 * NK;
    // field sources of this slot: value = ca * A[row] + cb * B[row]  (fields U = 0, V = 1, W = 2)
    const T2* Hu = Hx;
    const T2* Hw = Hx + (size_t)d.nyu * pls;
    const T2* Hv = Hx + (size_t)(2 * d.nyu) * pls;
    const T2 *fa0, *fb0, *fa1, *fb1, *fa2, *fb2;
    R ca0 = 1, cb0 = 0, ca1 = 1, cb1 = 0, ca2 = 1, cb2 = 0;
    if (uplane) {
        const int sl = slot;
        fa0 = fb0 = Hu + sl * pls;
        fa2 = fb2 = Hw + sl * pls;
        double ca, cb;
        int pa;
        if (sl == 0) {
            pa = 1; ca = (1.0 - g.gwib) * g.vca[1]; cb = g.gwib + (1.0 - g.gwib) * g.vcb[1];
        } else if (sl == d.nyu - 1) {
            pa = sl - 1; ca = g.gwit + (1.0 - g.gwit) * g.vca[sl - 1]; cb = (1.0 - g.gwit) * g.vcb[sl - 1];
        } else {
            pa = sl; ca = g.vca[sl]; cb = g.vcb[sl];
        }
        fa1 = Hv + pa * pls; fb1 = fa1 - pls; ca1 = (R)ca; cb1 = (R)cb;
    } else {
        const int sl = slot - d.nyu;
        fa1 = fb1 = Hv + sl * pls;
        fa0 = Hu + (sl + 1) * pls; fb0 = fa0 - pls; ca0 = (R)g.ufa[sl]; cb0 = (R)g.ufb[sl];
        fa2 = Hw + (sl + 1) * pls; fb2 = fa2 - pls; ca2 = (R)g.ufa[sl]; cb2 = (R)g.ufb[sl];
    }
    __syncthreads();

    // ---- inverse: line b = 3p + t, thread (b, n2) of two_step_lines' step 1
    const int tt = threadIdx.x;
    const int bme = tt / N2, n2me = tt - bme * N2;
    {
        const int t = bme % 3, p = bme / 3;
        const int r0 = z0 + 2 * p;
        // A and C of this thread's line: (field, row)
        const int fA = t < 2 ? 0 : (uplane ? 2 : 1);
        const int fC = t < 2 ? (uplane ? 1 : 2) : fA;
        const int rA = t == 1 ? r0 + 1 : r0;
        const int rC = t == 0 ? r0 : r0 + 1;
        const bool live = bme < NLI;
        auto sel = [&](int f, const T2* x0, const T2* x1, const T2* x2) { return f == 0 ? x0 : (f == 1 ? x1 : x2); };
        auto selr = [&](int f, R x0, R x1, R x2) { return f == 0 ? x0 : (f == 1 ? x1 : x2); };
        const T2* A0 = sel(fA, fa0, fa1, fa2) + (size_t)(live ? rA : 0) * NK;
        const T2* A1 = sel(fA, fb0, fb1, fb2) + (size_t)(live ? rA : 0) * NK;
        const T2* C0 = sel(fC, fa0, fa1, fa2) + (size_t)(live ? rC : 0) * NK;
        const T2* C1 = sel(fC, fb0, fb1, fb2) + (size_t)(live ? rC : 0) * NK;
        const R cA = selr(fA, ca0, ca1, ca2), dA = selr(fA, cb0, cb1, cb2);
        const R cC = selr(fC, ca0, ca1, ca2), dC = selr(fC, cb0, cb1, cb2);
        const bool twoA = dA != (R)0, twoC = dC != (R)0;
        auto fetch = [&](int k, T2& a, T2& c) {
            const T2 z = cx<T2>((R)0, (R)0);
            const T2 a0 = A0[k], a1 = twoA ? A1[k] : z, c0 = C0[k], c1 = twoC ? C1[k] : z;
            a = cx<T2>(cA * a0.x + dA * a1.x, cA * a0.y + dA * a1.y);
            c = cx<T2>(cC * c0.x + dC * c1.x, cC * c0.y + dC * c1.y);
        };
        auto load = [&](int e, int) -> T2 {
            const int e0 = e - n2me;
            const bool lo = (e0 + N2 - 1 <= HX) || (e0 <= HX && e <= HX);
            const bool hi = (e0 >= N - HX) || (e0 + N2 - 1 >= N - HX && e >= N - HX);
            T2 a, c;
            if (lo) {  // A_e + i C_e; the rft inverse ignores Im of the kx = 0 entries
                fetch(e, a, c);
                if (e == 0) { a.y = 0; c.y = 0; }
                return cx<T2>(a.x - c.y, a.y + c.x);
            }
            if (hi) {  // conj(A_k) + i conj(C_k), k = N - e
                fetch(N - e, a, c);
                return cx<T2>(a.x + c.y, -a.y + c.x);
            }
            return cx<T2>((R)0, (R)0);
        };
        auto store = [&](int x, int b, T2 v) { PU[(size_t)b * N + x] = v; };
        two_step_lines<T2, N1, N2, +1, false>(0, ex, twt, load, store, NLI);
    }

    // ---- forward: line f, products from the physical rows
    {
        const int s = uplane ? (bme & 3) : (bme & 1), p = uplane ? (bme >> 2) : (bme >> 1);
        const bool live = bme < NLF;
        const int pp = live ? p : 0;
        const T2* La = PU + (size_t)(3 * pp + (s & 1)) * N;  // u, v (u-plane) / u, w (v-plane) of the row
        const T2* Lb = PU + (size_t)(3 * pp + 2) * N;        // w pair (u-plane) / v pair (v-plane)
        const bool odd = (s & 1) != 0, sq = uplane && s < 2;
        auto load = [&](int x, int) -> T2 {
            const T2 a = La[x];
            if (sq) return cx<T2>(a.x * a.x, a.y * a.y);  // uu + i vv
            const T2 bb = Lb[x];
            const R o = odd ? bb.y : bb.x;                // w (u-plane) or v (v-plane) of the row
            return uplane ? cx<T2>(o * o, a.x * o)        // ww + i uw
                          : cx<T2>(a.x * o, a.y * o);     // uv + i vw
        };
        auto store = [&](int k, int f, T2 v) { PU[(size_t)f * LU + k] = v; };
        // the forward step 1 reads every physical row before any spectrum is stored: the
        // stores of two_step_lines come after its internal barrier
        two_step_lines<T2, N1, N2, -1, false>(0, ex, twt, load, store, NLF);
    }

    // ---- unpack A_k = (P_k + conj P_{N-k})/2, B_k = (P_k - conj P_{N-k})/(2i), x 1/N
    const R hs = (R)0.5 / (R)N;
    const size_t pbase = (size_t)slot * d.ngal2 * NK;
    for (int it = threadIdx.x; it < NLF * NK; it += blockDim.x) {
        const int f = (unsigned)it / NK, k = it - f * NK;
        const int s = uplane ? (f & 3) : (f & 1), p = uplane ? (f >> 2) : (f >> 1);
        const int row = z0 + 2 * p + (s & 1);
        const T2* line = PU + (size_t)f * LU;
        const T2 Pk = line[k];
        const T2 Qc = cconj(line[k == 0 ? 0 : N - k]);
        T2* da = uplane ? (s < 2 ? H0 : H3) : H0;  // uu / ww / uv
        T2* db = uplane ? (s < 2 ? H2 : H1) : H1;  // vv / uw / vw
        const size_t o = pbase + (size_t)row * NK + k;
        da[o] = cx<T2>((Pk.x + Qc.x) * hs, (Pk.y + Qc.y) * hs);
        db[o] = cx<T2>((Pk.y - Qc.y) * hs, -(Pk.x - Qc.x) * hs);
    }
}

// --------------------------------------------------------------------------------------
// Pass 3: forward z transform (cft forward of phys_to_four_du, x 1/Ngal2) and truncation
// to the retained kz modes (planes_to_modes_UVP/NUVP picks rows k and k+Ngal2-N2).
// Output spectral products S_f[slot][column]:  u-plane: S0=uu S1=uw S2=vv S3=ww;
// v-plane: S0=uv S1=vw.   grid: x = kx chunk, y = slot, z = field 0..3
// --------------------------------------------------------------------------------------
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_zfwd(Dims d, const T2* __restrict__ H0, const T2* __restrict__ H1,
                                              const T2* __restrict__ H2, const T2* __restrict__ H3,
                                              T2* __restrict__ S0, T2* __restrict__ S1, T2* __restrict__ S2,
                                              T2* __restrict__ S3, FFTDesc fz, const T2* __restrict__ twz, int CH, int bshift) {
    using R = decltype(T2::x);
    const int slot = blockIdx.y;
    const int f = blockIdx.z;
    if (slot >= d.nyu && f >= 2) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal2;
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * CH;
    T2* tw = buf1 + (size_t)n * CH;
    const int kx0 = blockIdx.x * CH;
    const T2* H = f == 0 ? H0 : (f == 1 ? H1 : (f == 2 ? H2 : H3));
    T2* S = f == 0 ? S0 : (f == 1 ? S1 : (f == 2 ? S2 : S3));
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
    const size_t base = (size_t)slot * n * d.nkx;
    for (int t = threadIdx.x; t < (n << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), z = t >> bshift;
        const int i = kx0 + b;
        buf0[swz(z, b, bshift)] = i < d.nkx ? H[base + (size_t)z * d.nkx + i] : cx<T2>((R)0, (R)0);
    }
    __syncthreads();
    T2* res = fft_batch<T2, NF, -1>(buf0, buf1, CH, bshift, fz, tw);
    const R s = (R)1 / (R)n;
    for (int t = threadIdx.x; t < (d.n2 << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), q = t >> bshift;
        const int i = kx0 + b;
        if (i < d.nkx) S[(size_t)slot * d.ncol + (size_t)q * d.nkx + i] = cscale(res[swz(row_of(d, q), b, bshift)], s);
    }
}

// Retained-row index q of z element e = e0 + r of a two-step line, where r (0 <= r < W) is
// the thread's own offset and e0 a compile-time constant once the element loop is
// unrolled; -1 inside the truncated band.  Rows 0..N/3-1 hold kz >= 0, rows N-N/3..N-1 the
// negative kz (N2 = 2*(Ngal2/3) modes kept), so only blocks straddling a band edge test e.
template <int N, int W>
__device__ __forceinline__ int zrow_q(int e, int r) {
    constexpr int HQ = N / 3, GAP = N - 2 * (N / 3);
    const int e0 = e - r;
    if (e0 + W - 1 < HQ) return e;
    if (e0 >= N - HQ) return e - GAP;
    if (e0 >= HQ && e0 + W - 1 < N - HQ) return -1;
    return e < HQ ? e : (e >= N - HQ ? e - GAP : -1);
}

// Passes 1 and 3 with the two-step transform.  Lines are numbered across a slot group
// (group 0: the nyu u-planes, group 1: the nyv v-planes) as line = slot-in-group * nkx + kx,
// and a CTA takes CH = 1 << lb consecutive lines, so no CTA is left with a partial kx chunk.
// grid: x = line chunk, y = field, z = group.
//
// Pass 1 source of every line: ca * A[col] + cb * B[col] with planes A, B and weights fixed
// per line, so the element loop has no branches and its loads issue back to back.  On the
// two wall centres the ghost extrapolation of v (FOU3D.f90:261-283) is folded into the
// two weights (A = v(1), B = v(0) at the bottom; A = v(ny), B = v(ny-1) at the top; the
// u and v index ranges start at the same j).
template <typename T2, int TN1, int TN2>
__global__ void k_zinv2(Dims d, Geo g, const double2* __restrict__ u1, const double2* __restrict__ u2,
                        const double2* __restrict__ u3, T2* __restrict__ H0, T2* __restrict__ H1,
                        T2* __restrict__ H2, const T2* __restrict__ twz, int lb) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    const int grp = blockIdx.z, f = blockIdx.y;
    const int nsl = grp ? d.nsv : d.nsu;
    const int nlines = nsl * d.nkx;
    const int line0 = blockIdx.x << lb;
    if (line0 >= nlines) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twz);
    const int b = threadIdx.x & ((1 << lb) - 1);
    const bool live = line0 + b < nlines;
    const int line = live ? line0 + b : nlines - 1;
    const int sl = (line / d.nkx) + (grp ? d.sv0 : d.su0), i = line - (line / d.nkx) * d.nkx;
    const size_t nc = d.pstride;
    const double2* pa;
    const double2* pb;
    double ca = 1.0, cb = 0.0;
    bool two;
    if (grp == 0) {
        two = f == 2;
        if (!two) {
            pa = (f == 0 ? u1 : u3) + (size_t)sl * nc;
        } else if (sl == 0) {
            pa = u2 + nc;
            ca = (1.0 - g.gwib) * g.vca[1];
            cb = g.gwib + (1.0 - g.gwib) * g.vcb[1];
        } else if (sl == d.nyu - 1) {
            pa = u2 + (size_t)(sl - 1) * nc;
            ca = g.gwit + (1.0 - g.gwit) * g.vca[sl - 1];
            cb = (1.0 - g.gwit) * g.vcb[sl - 1];
        } else {
            pa = u2 + (size_t)sl * nc;
            ca = g.vca[sl];
            cb = g.vcb[sl];
        }
    } else {
        two = f != 2;
        if (!two) {
            pa = u2 + (size_t)sl * nc;
        } else {
            pa = (f == 0 ? u1 : u3) + (size_t)(sl + 1) * nc;
            ca = g.ufa[sl];
            cb = g.ufb[sl];
        }
    }
    pa += i;
    pb = two ? pa - nc : pa;
    const int r = threadIdx.x >> lb;
    T2* H = (f == 0 ? H0 : (f == 1 ? H1 : H2)) + (size_t)(grp ? d.nyu + sl : sl) * d.hstride + i;
    __syncthreads();
    auto qof = [&](int e) { return zrow_q<N, TN2>(e, r); };
    auto store = [&](int z, int, T2 v) {
        if (live) H[(size_t)z * d.nkx] = v;
    };
    if (two) {
        auto load = [&](int e, int) -> T2 {
            const int q = qof(e);
            double2 va = dc(0.0, 0.0), vb = dc(0.0, 0.0);
            if (q >= 0) {
                va = pa[scol(d, 0, q)];
                vb = pb[scol(d, 0, q)];
            }
            return to_t2<T2>(dc(ca * va.x + cb * vb.x, ca * va.y + cb * vb.y));
        };
        two_step_lines<T2, TN1, TN2, +1>(lb, ex, twt, load, store);
    } else {
        auto load = [&](int e, int) -> T2 {
            const int q = qof(e);
            return q >= 0 ? to_t2<T2>(pa[scol(d, 0, q)]) : cx<T2>((R)0, (R)0);
        };
        two_step_lines<T2, TN1, TN2, +1>(lb, ex, twt, load, store);
    }
}

// Pass 1 for the x-line kernel that interpolates in y itself: every field is transformed
// once on its own planes, Hx = [u planes ju0..ju1 | w planes ju0..ju1 | v planes jv0..jv1].
// Interpolation in y and the z transform are both linear, so interpolating the transformed
// planes gives the transform of the interpolated planes (FOU3D.f90:261-308).
// grid: x = line chunk (line = plane * nkx + kx), y = field (u, w, v).
template <typename T2, int TN1, int TN2>
__device__ __forceinline__ void zinv2s_body(Dims d, const double2* __restrict__ u1, const double2* __restrict__ u2,
                         const double2* __restrict__ u3, T2* __restrict__ Hx, const T2* __restrict__ twz, int lb) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    const int f = blockIdx.y;
    const int npl = f == 2 ? d.nyv : d.nyu;
    const int nlines = npl * d.nkx;
    const int line0 = blockIdx.x << lb;
    if (line0 >= nlines) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twz);
    const int b = threadIdx.x & ((1 << lb) - 1);
    const bool live = line0 + b < nlines;
    const int line = live ? line0 + b : nlines - 1;
    const int pl = line / d.nkx, i = line - pl * d.nkx;
    const double2* src = (f == 0 ? u1 : (f == 1 ? u3 : u2)) + (size_t)pl * d.ncol + i;
    T2* H = Hx + ((size_t)(f == 0 ? 0 : (f == 1 ? d.nyu : 2 * d.nyu)) + pl) * N * d.nkx + i;
    const int r = threadIdx.x >> lb;
    __syncthreads();
    auto load = [&](int e, int) -> T2 {
        const int q = zrow_q<N, TN2>(e, r);
        return q >= 0 ? to_t2<T2>(src[(size_t)q * d.nkx]) : cx<T2>((R)0, (R)0);
    };
    auto store = [&](int z, int, T2 v) {
        if (live) H[(size_t)z * d.nkx] = v;
    };
    two_step_lines<T2, TN1, TN2, +1>(lb, ex, twt, load, store);
}

template <typename T2, int TN1, int TN2>
__global__ void __launch_bounds__(16 * (TN1 > TN2 ? TN1 : TN2), (sizeof(T2) == 8 && (TN1 > TN2 ? TN1 : TN2) <= 24) ? 3 : 1) k_zinv2s(Dims d, const double2* __restrict__ u1, const double2* __restrict__ u2,
                         const double2* __restrict__ u3, T2* __restrict__ Hx, const T2* __restrict__ twz, int lb) {
    zinv2s_body<T2, TN1, TN2>(d, u1, u2, u3, Hx, twz, lb);
}

// Pass 3: grid x = line chunk, y = field 0..3, z = group (v-planes carry fields 0, 1 only).
template <typename T2, int TN1, int TN2>
__device__ __forceinline__ void zfwd2_body(Dims d, const T2* __restrict__ H0, const T2* __restrict__ H1, const T2* __restrict__ H2,
                        const T2* __restrict__ H3, T2* __restrict__ S0, T2* __restrict__ S1, T2* __restrict__ S2,
                        T2* __restrict__ S3, const T2* __restrict__ twz, int lb) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    const int grp = blockIdx.z, f = blockIdx.y;
    if (grp == 1 && f >= 2) return;
    const int nsl = grp ? d.nsv : d.nsu;
    const int nlines = nsl * d.nkx;
    const int line0 = blockIdx.x << lb;
    if (line0 >= nlines) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twz);
    const int b = threadIdx.x & ((1 << lb) - 1);
    const bool live = line0 + b < nlines;
    const int line = live ? line0 + b : nlines - 1;
    const int sl = line / d.nkx, i = line - sl * d.nkx;
    const int slot = grp ? d.nyu + d.sv0 + sl : d.su0 + sl;
    const T2* H = (f == 0 ? H0 : (f == 1 ? H1 : (f == 2 ? H2 : H3))) + (size_t)slot * d.hstride + i;
    T2* S = (f == 0 ? S0 : (f == 1 ? S1 : (f == 2 ? S2 : S3))) + (size_t)slot * d.pstride + i;
    const int r = threadIdx.x >> lb;
    const R sc = (R)1 / (R)N;
    __syncthreads();
    auto load = [&](int z, int) -> T2 { return H[(size_t)z * d.nkx]; };
    auto store = [&](int e, int, T2 v) {
        const int q = zrow_q<N, TN1>(e, r);
        if (q >= 0 && live) S[scol(d, 0, q)] = cscale(v, sc);
    };
    two_step_lines<T2, TN1, TN2, -1>(lb, ex, twt, load, store);
}

template <typename T2, int TN1, int TN2>
__global__ void __launch_bounds__(16 * (TN1 > TN2 ? TN1 : TN2), (sizeof(T2) == 8 && (TN1 > TN2 ? TN1 : TN2) <= 24) ? 3 : 1) k_zfwd2(Dims d, const T2* __restrict__ H0, const T2* __restrict__ H1, const T2* __restrict__ H2,
                        const T2* __restrict__ H3, T2* __restrict__ S0, T2* __restrict__ S1, T2* __restrict__ S2,
                        T2* __restrict__ S3, const T2* __restrict__ twz, int lb) {
    zfwd2_body<T2, TN1, TN2>(d, H0, H1, H2, H3, S0, S1, S2, S3, twz, lb);
}


// The FP64 z kernels of the nonlinear pass held to 112 registers per thread: with 8 lines
// per CTA (192 threads at the 384-point splits) three CTAs fit on an SM instead of two.
template <int TN1, int TN2>
__global__ void __maxnreg__(112) k_zinv2sd(Dims d, const double2* __restrict__ u1, const double2* __restrict__ u2,
                         const double2* __restrict__ u3, double2* __restrict__ Hx, const double2* __restrict__ twz, int lb) {
    zinv2s_body<double2, TN1, TN2>(d, u1, u2, u3, Hx, twz, lb);
}
template <int TN1, int TN2>
__global__ void __maxnreg__(112) k_zfwd2d(Dims d, const double2* __restrict__ H0, const double2* __restrict__ H1, const double2* __restrict__ H2,
                        const double2* __restrict__ H3, double2* __restrict__ S0, double2* __restrict__ S1, double2* __restrict__ S2,
                        double2* __restrict__ S3, const double2* __restrict__ twz, int lb) {
    zfwd2_body<double2, TN1, TN2>(d, H0, H1, H2, H3, S0, S1, S2, S3, twz, lb);
}

// --------------------------------------------------------------------------------------
// Column kernel: RHS0_u1/u2/u3 (littleharsh.f90:613-730), the tail of nonlinear
// (der_x/der_z FOU3D.f90:310-414 as ik products with the kz = -N2/2 row zeroed,
// der_yu_h/der_yv_h :453-493, du += -g Nu :233-244) and the solveU/solveV prologue
// (du = u + dt du, wall/ghost rows 0; littleharsh.f90:744-786).
// MODE bits: 1 = RHS0, 2 = nonlinear tail, 4 = solve prologue.
// --------------------------------------------------------------------------------------
struct RKCoef {
    double C1;    // a/Re
    double C2;    // -c
    double dRK;   // d = g + c
    double mg;    // -g
    double dt;
    int krk;
    // 1: the x/z advective derivatives of every interior plane are those of the last plane
    // of the grid (top ghost centre for u/w, top wall face for v), as the reference computes
    // them with one plane slab (2-D scratch summed after the plane loop, FOU3D.f90:1541,
    // 1571-1585, 1602-1613); 0: per plane
    int lastplane;
};

template <typename T2> __device__ __forceinline__ T2 ldT(const T2* p) { return *p; }

template <typename T2, int MODE>
__global__ void __launch_bounds__(256, sizeof(T2) == 8 ? 3 : 0) k_rhs(Dims d, Geo g, RKCoef c, const double* __restrict__ scal,
                                             const double2* __restrict__ u1, const double2* __restrict__ u2,
                                             const double2* __restrict__ u3, const double2* __restrict__ p,
                                             T2* __restrict__ Nu1, T2* __restrict__ Nu2, T2* __restrict__ Nu3,
                                             double2* __restrict__ du1, double2* __restrict__ du2,
                                             double2* __restrict__ du3, const T2* __restrict__ S0,
                                             const T2* __restrict__ S1, const T2* __restrict__ S2,
                                             const T2* __restrict__ S3, int JC) {
    // one thread = one column and a chunk of JC planes (blockIdx.y); no recurrence in y
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const double k2 = (-kxv * kxv) + (-kzv * kzv);
    const bool zrow = (q == d.n2 / 2);  // der_x/der_z zero the kz = -N2/2 mode
    const size_t nc = d.ncol;
    const double mpgx = scal[0];
    constexpr bool RHS0 = (MODE & 1) != 0, NL = (MODE & 2) != 0, PRO = (MODE & 4) != 0;
    const int cb = blockIdx.y;

    // ---- u and w (ugrid), j = ju0+1 .. ju1-1
    {
        const int jb = d.ju0 + 1 + cb * JC;
        const int je = min(jb + JC, d.ju1);
        if (jb < je) {
            const size_t ju = (size_t)(jb - d.ju0);
            double2 a_m = u1[(ju - 1) * nc + col], a_0 = u1[ju * nc + col];
            double2 w_m = u3[(ju - 1) * nc + col], w_0 = u3[ju * nc + col];
            const size_t vs = (size_t)d.nyu * nc;  // first v-slot
            double2 uv_m = NL ? to_d2(S0[vs + (size_t)(jb - 1 - d.jv0) * nc + col]) : dc(0, 0);
            double2 vw_m = NL ? to_d2(S1[vs + (size_t)(jb - 1 - d.jv0) * nc + col]) : dc(0, 0);
            for (int j = jb; j < je; ++j) {
                const size_t ju = (size_t)(j - d.ju0);
                const double2 a_p = u1[(ju + 1) * nc + col];
                const double2 w_p = u3[(ju + 1) * nc + col];
                const size_t jp = (size_t)(j - d.jp0);
                double2 r1, r3;
                if (RHS0) {
                    const double c0 = g.dyu2i[3 * ju + 0], c1 = g.dyu2i[3 * ju + 1], c2 = g.dyu2i[3 * ju + 2];
                    const double dg = k2 + c1;
                    const double2 Lu = dadd(dadd(dscl(c0, a_m), dscl(dg, a_0)), dscl(c2, a_p));
                    const double2 Lw = dadd(dadd(dscl(c0, w_m), dscl(dg, w_0)), dscl(c2, w_p));
                    const double2 pp = p[jp * nc + col];
                    const double2 n1o = to_d2(Nu1[ju * nc + col]);
                    const double2 n3o = to_d2(Nu3[ju * nc + col]);
                    r1 = dadd(dadd(dscl(c.C1, Lu), dscl(c.C2, n1o)), dik(-c.dRK * kxv, pp));
                    r3 = dadd(dadd(dscl(c.C1, Lw), dscl(c.C2, n3o)), dik(-c.dRK * kzv, pp));
                    if (col == 0) r1.x += -c.dRK * mpgx;
                } else {
                    r1 = du1[ju * nc + col];
                    r3 = du3[ju * nc + col];
                }
                if (NL) {
                    const size_t su = ju * nc + col;
                    const size_t sx = c.lastplane ? (size_t)(d.nyu - 1) * nc + col : su;  // x/z products
                    const size_t sv = vs + (size_t)(j - d.jv0) * nc + col;
                    const double2 uv_p = to_d2(S0[sv]), vw_p = to_d2(S1[sv]);
                    const double dth = g.dthdyu[ju];
                    double2 n1 = zrow ? dc(0, 0) : dadd(dik(kxv, to_d2(S0[sx])), dik(kzv, to_d2(S1[sx])));
                    double2 n3 = zrow ? dc(0, 0) : dadd(dik(kxv, to_d2(S1[sx])), dik(kzv, to_d2(S3[sx])));
                    n1 = dadd(n1, dscl(dth, dsub(uv_p, uv_m)));
                    n3 = dadd(n3, dscl(dth, dsub(vw_p, vw_m)));
                    Nu1[su] = to_t2<T2>(n1);
                    Nu3[su] = to_t2<T2>(n3);
                    r1 = dadd(r1, dscl(c.mg, n1));
                    r3 = dadd(r3, dscl(c.mg, n3));
                    uv_m = uv_p;
                    vw_m = vw_p;
                }
                if (PRO) {
                    r1 = dadd(a_0, dscl(c.dt, r1));
                    r3 = dadd(w_0, dscl(c.dt, r3));
                }
                du1[ju * nc + col] = r1;
                du3[ju * nc + col] = r3;
                a_m = a_0; a_0 = a_p;
                w_m = w_0; w_0 = w_p;
            }
        }
    }
    // ---- v (vgrid), j = jv0+1 .. jv1-1
    {
        const int jb = d.jv0 + 1 + cb * JC;
        const int je = min(jb + JC, d.jv1);
        if (jb < je) {
            const size_t jv = (size_t)(jb - d.jv0);
            double2 v_m = u2[(jv - 1) * nc + col], v_0 = u2[jv * nc + col];
            double2 vv_0 = NL ? to_d2(S2[(size_t)(jb - d.ju0) * nc + col]) : dc(0, 0);
            const size_t vs = (size_t)d.nyu * nc;
            for (int j = jb; j < je; ++j) {
                const size_t jv = (size_t)(j - d.jv0);
                const double2 v_p = u2[(jv + 1) * nc + col];
                double2 r2;
                if (RHS0) {
                    const double c0 = g.dyv2i[3 * jv + 0], c1 = g.dyv2i[3 * jv + 1], c2 = g.dyv2i[3 * jv + 2];
                    const double2 Lv = dadd(dadd(dscl(c0, v_m), dscl(k2 + c1, v_0)), dscl(c2, v_p));
                    const double C3 = -c.dRK * g.dthdyv[jv];
                    const double2 pa = p[(size_t)(j + 1 - d.jp0) * nc + col];
                    const double2 pb = p[(size_t)(j - d.jp0) * nc + col];
                    const double2 n2o = to_d2(Nu2[jv * nc + col]);
                    r2 = dadd(dadd(dscl(c.C1, Lv), dscl(c.C2, n2o)), dscl(C3, dsub(pa, pb)));
                } else {
                    r2 = du2[jv * nc + col];
                }
                if (NL) {
                    const size_t sv = vs + (c.lastplane ? (size_t)(d.nyv - 1) : jv) * nc + col;
                    const double2 vv_p = to_d2(S2[(size_t)(j + 1 - d.ju0) * nc + col]);
                    double2 n2 = zrow ? dc(0, 0) : dadd(dik(kxv, to_d2(S0[sv])), dik(kzv, to_d2(S1[sv])));
                    n2 = dadd(n2, dscl(g.dthdyv[jv], dsub(vv_p, vv_0)));
                    Nu2[jv * nc + col] = to_t2<T2>(n2);
                    r2 = dadd(r2, dscl(c.mg, n2));
                    vv_0 = vv_p;
                }
                if (PRO) r2 = dadd(v_0, dscl(c.dt, r2));
                du2[jv * nc + col] = r2;
                v_m = v_0; v_0 = v_p;
            }
        }
    }
    if (PRO && cb == 0) {
        du1[col] = dc(0, 0);
        du3[col] = dc(0, 0);
        du1[(size_t)(d.nyu - 1) * nc + col] = dc(0, 0);
        du3[(size_t)(d.nyu - 1) * nc + col] = dc(0, 0);
        du2[col] = dc(0, 0);
        du2[(size_t)(d.nyv - 1) * nc + col] = dc(0, 0);
    }
}

// --------------------------------------------------------------------------------------
// Immersed-boundary forcing (immersed_boundaries_U/V, tridLU_3D_IB.f90:163-281) on the
// canopy planes only: inverse 2-D transform of rhs and u, point forcing, forward
// transform of rhs back to every column of those planes.
// Sources are (rhs, u) pairs; src[2*fb] = rhs of batch fb, src[2*fb+1] = its u.
// --------------------------------------------------------------------------------------
struct IBSrc {
    const double2* f[4];
};
struct IBDst {
    double2* f[2];
};

// inverse z transform of the IB planes of every source.  grid: x = kx chunk, y = plane,
// z = source.  Hib[(s*npl + p)][z][kx]
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_ib_zinv(Dims d, IBSrc src, int j0, const int* __restrict__ planes, int npl,
                                                 T2* __restrict__ Hib, FFTDesc fz, const T2* __restrict__ twz, int CH, int bshift) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal2;
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * CH;
    T2* tw = buf1 + (size_t)n * CH;
    const int kx0 = blockIdx.x * CH, p = blockIdx.y, s = blockIdx.z;
    const int j = planes[p];
    const double2* f = src.f[s];
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
    for (int t = threadIdx.x; t < n * CH; t += blockDim.x) buf0[t] = cx<T2>(0, 0);
    __syncthreads();
    for (int t = threadIdx.x; t < (d.n2 << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), q = t >> bshift, i = kx0 + b;
        if (i >= d.nkx) continue;
        buf0[swz(row_of(d, q), b, bshift)] = to_t2<T2>(f[(size_t)(j - j0) * d.ncol + (size_t)q * d.nkx + i]);
    }
    __syncthreads();
    T2* res = fft_batch<T2, NF, +1>(buf0, buf1, CH, bshift, fz, tw);
    const size_t base = ((size_t)s * npl + p) * n * d.nkx;
    for (int t = threadIdx.x; t < (n << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), z = t >> bshift, i = kx0 + b;
        if (i < d.nkx) Hib[base + (size_t)z * d.nkx + i] = res[swz(z, b, bshift)];
    }
}

// inverse x transform: line (rhs + i u) of one row -> physical rhs, u.
// grid: x = row chunk (RW rows), y = plane, z = batch fb.  Phys[(fb*2+which)*npl + p][z][x]
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_ib_xinv(Dims d, const T2* __restrict__ Hib, int npl, decltype(T2::x)* __restrict__ phys,
                                                 FFTDesc fx, const T2* __restrict__ twx, int RW, int bshift) {
    using R = decltype(T2::x);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal1;
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * RW;
    T2* tw = buf1 + (size_t)n * RW;
    const int z0 = blockIdx.x * RW, p = blockIdx.y, fb = blockIdx.z;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twx[t];
    const size_t pl = (size_t)d.ngal2 * d.nkx;
    const T2* Hr = Hib + ((size_t)(2 * fb) * npl + p) * pl;
    const T2* Hu = Hib + ((size_t)(2 * fb + 1) * npl + p) * pl;
    // line (rhs + i u) per row, k fastest across threads (coalesced rows); gap modes zero
    const int h = d.n1 / 2, nk = d.nkx;
    for (int t = threadIdx.x; t < (n - 2 * h - 1) * RW; t += blockDim.x) {
        const int b = t & (RW - 1), k = h + 1 + (t >> bshift);
        buf0[swz(k, b, bshift)] = cx<T2>((R)0, (R)0);
    }
    for (int t = threadIdx.x; t < nk * RW; t += blockDim.x) {
        const int k = t % nk, b = t / nk;
        const size_t o = (size_t)(z0 + b) * nk + k;
        T2 a = Hr[o], c = Hu[o];
        if (k == 0) { a.y = 0; c.y = 0; }
        buf0[swz(k, b, bshift)] = cx<T2>(a.x - c.y, a.y + c.x);
        if (k > 0) buf0[swz(n - k, b, bshift)] = cx<T2>(a.x + c.y, -a.y + c.x);
    }
    __syncthreads();
    T2* res = fft_batch<T2, NF, +1>(buf0, buf1, RW, bshift, fx, tw);
    const size_t ppl = (size_t)d.ngal2 * n;
    R* pr = phys + ((size_t)(2 * fb) * npl + p) * ppl;
    R* pu = phys + ((size_t)(2 * fb + 1) * npl + p) * ppl;
    for (int t = threadIdx.x; t < n * RW; t += blockDim.x) {
        const int k = t % n, b = t / n;
        const T2 v = res[swz(k, b, bshift)];
        pr[(size_t)(z0 + b) * n + k] = v.x;
        pu[(size_t)(z0 + b) * n + k] = v.y;
    }
}

// point forcing rhs(p) = Lap*(w2 u(p2) + w3 u(p3) - u(p) + rhs(p)) (tridLU_3D_IB.f90:193-211);
// points are sorted by (j,k,i): the first point of a run of equal targets applies the
// whole run in list order, so repeated targets behave as the reference's serial loop.
// grid: x = points, y = batch fb
template <typename R>
__global__ void k_ib_force(Dims d, const int* __restrict__ idx, const double* __restrict__ w, int npts,
                           const int* __restrict__ slot_of_j, int j0, int npl, R* __restrict__ phys) {
    const int pt = blockIdx.x * blockDim.x + threadIdx.x;
    if (pt >= npts) return;
    const int fb = blockIdx.y;
    const int* id = idx + 9 * (size_t)pt;
    if (pt > 0) {
        const int* pv = id - 9;
        if (pv[0] == id[0] && pv[1] == id[1] && pv[2] == id[2]) return;
    }
    const size_t ppl = (size_t)d.ngal2 * d.ngal1;
    R* pr = phys + (size_t)(2 * fb) * npl * ppl;
    const R* pu = phys + (size_t)(2 * fb + 1) * npl * ppl;
    auto off = [&](int i, int k, int j) -> size_t {
        return (size_t)slot_of_j[j - j0] * ppl + (size_t)(k - 1) * d.ngal1 + (i - 1);
    };
    const size_t tgt = off(id[0], id[1], id[2]);
    R r = pr[tgt];
    const R u0 = pu[tgt];
    for (int q = pt; q < npts; ++q) {
        const int* iq = idx + 9 * (size_t)q;
        if (q > pt && !(iq[0] == id[0] && iq[1] == id[1] && iq[2] == id[2])) break;
        const double* wq = w + 3 * (size_t)q;
        const R vf = (R)wq[1] * pu[off(iq[3], iq[4], iq[5])] + (R)wq[2] * pu[off(iq[6], iq[7], iq[8])];
        r = (R)wq[0] * (vf - u0 + r);
    }
    pr[tgt] = r;
}

// forward x transform of physical rhs rows (two rows per complex line), truncated to
// kx <= N1/2, x 1/Ngal1.  grid: x = row chunk (RW rows, RW even), y = plane, z = batch.
// Output into Hib[(fb*2)*npl + p] (the rhs slot).
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_ib_xfwd(Dims d, T2* __restrict__ Hib, int npl, const decltype(T2::x)* __restrict__ phys,
                                                 FFTDesc fx, const T2* __restrict__ twx, int RW, int bshift) {
    using R = decltype(T2::x);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal1;
    const int B = RW / 2;
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * B;
    T2* tw = buf1 + (size_t)n * B;
    const int z0 = blockIdx.x * RW, p = blockIdx.y, fb = blockIdx.z;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twx[t];
    const size_t ppl = (size_t)d.ngal2 * n;
    const R* pr = phys + ((size_t)(2 * fb) * npl + p) * ppl;
    for (int t = threadIdx.x; t < n * B; t += blockDim.x) {
        const int k = t % n, b = t / n;
        buf0[swz(k, b, bshift)] = cx<T2>(pr[(size_t)(z0 + 2 * b) * n + k], pr[(size_t)(z0 + 2 * b + 1) * n + k]);
    }
    __syncthreads();
    T2* F = fft_batch<T2, NF, -1>(buf0, buf1, B, bshift, fx, tw);
    const R s = (R)1 / (R)n;
    T2* Hr = Hib + ((size_t)(2 * fb) * npl + p) * (size_t)d.ngal2 * d.nkx;
    for (int t = threadIdx.x; t < d.nkx * B; t += blockDim.x) {
        const int k = t % d.nkx, b = t / d.nkx;
        const T2 Pk = F[swz(k, b, bshift)];
        const T2 Qc = cconj(F[swz((n - k) % n, b, bshift)]);
        Hr[(size_t)(z0 + 2 * b) * d.nkx + k] = cx<T2>((Pk.x + Qc.x) * (R)0.5 * s, (Pk.y + Qc.y) * (R)0.5 * s);
        Hr[(size_t)(z0 + 2 * b + 1) * d.nkx + k] = cx<T2>((Pk.y - Qc.y) * (R)0.5 * s, -(Pk.x - Qc.x) * (R)0.5 * s);
    }
}

// forward z transform of the rhs slot and write-back to every column of the plane
// (planes_to_modes_dU/dV).  grid: x = kx chunk, y = plane, z = batch fb
template <typename T2, int NF>
__global__ void __launch_bounds__(256) k_ib_zfwd(Dims d, const T2* __restrict__ Hib, int npl, IBDst dst, int j0,
                                                 const int* __restrict__ planes, FFTDesc fz, const T2* __restrict__ twz,
                                                 int CH, int bshift) {
    using R = decltype(T2::x);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = d.ngal2;
    T2* buf0 = reinterpret_cast<T2*>(smem_raw);
    T2* buf1 = buf0 + (size_t)n * CH;
    T2* tw = buf1 + (size_t)n * CH;
    const int kx0 = blockIdx.x * CH, p = blockIdx.y, fb = blockIdx.z;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = twz[t];
    const T2* H = Hib + ((size_t)(2 * fb) * npl + p) * (size_t)n * d.nkx;
    for (int t = threadIdx.x; t < (n << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), z = t >> bshift, i = kx0 + b;
        buf0[swz(z, b, bshift)] = i < d.nkx ? H[(size_t)z * d.nkx + i] : cx<T2>((R)0, (R)0);
    }
    __syncthreads();
    T2* res = fft_batch<T2, NF, -1>(buf0, buf1, CH, bshift, fz, tw);
    const R s = (R)1 / (R)n;
    double2* out = dst.f[fb] + (size_t)(planes[p] - j0) * d.ncol;
    for (int t = threadIdx.x; t < (d.n2 << bshift); t += blockDim.x) {
        const int b = t & (CH - 1), q = t >> bshift, i = kx0 + b;
        if (i < d.nkx) out[(size_t)q * d.nkx + i] = to_d2(cscale(res[swz(row_of(d, q), b, bshift)], s));
    }
}

// IB round trip with the two-step transform (same data flow as k_ib_zinv/xinv/xfwd/zfwd).
template <typename T2, int TN1, int TN2>
__global__ void __launch_bounds__(16 * (TN1 > TN2 ? TN1 : TN2), (sizeof(T2) == 8 && (TN1 > TN2 ? TN1 : TN2) <= 24) ? 3 : 1) k_ib_zinv2(Dims d, IBSrc src, int j0, const int* __restrict__ planes, int npl, T2* __restrict__ Hib,
                           const T2* __restrict__ twz, int lb, int sstep) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    const int nlines = npl * d.nkx;
    // sstep 2: the right-hand sides only (the velocities come from the nonlinear pass)
    const int line0 = blockIdx.x << lb, sidx = blockIdx.z * sstep;
    if (line0 >= nlines) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twz);
    const int b = threadIdx.x & ((1 << lb) - 1);
    const bool live = line0 + b < nlines;
    const int line = live ? line0 + b : nlines - 1;
    const int p = line / d.nkx, i = line - p * d.nkx;
    const double2* f = src.f[sidx] + (size_t)(planes[p] - j0) * d.ncol + i;
    T2* H = Hib + ((size_t)sidx * npl + p) * N * d.nkx + i;
    const int r = threadIdx.x >> lb;
    __syncthreads();
    auto load = [&](int e, int) -> T2 {
        const int q = zrow_q<N, TN2>(e, r);
        return q >= 0 ? to_t2<T2>(f[(size_t)q * d.nkx]) : cx<T2>((R)0, (R)0);
    };
    auto store = [&](int z, int, T2 v) {
        if (live) H[(size_t)z * d.nkx] = v;
    };
    two_step_lines<T2, TN1, TN2, +1>(lb, ex, twt, load, store);
}

// inverse x: line (rhs + i u) of each of RW rows -> physical rhs, u (rows coalesced in x)
// With Hvel, the velocity of batch fb is read from the z-transformed field planes of the
// nonlinear pass (k_zinv2s, the same transform of the same state): plane voff[fb] + (j - j0)
// of Hvel for the IB plane j = planes[p].
struct IBVel {
    const void* H;
    int voff[2];
    const int* planes;
    int j0;
};

template <typename T2, int TN1, int TN2>
__global__ void k_ib_xinv2(Dims d, const T2* __restrict__ Hib, int npl, decltype(T2::x)* __restrict__ phys,
                           const int* __restrict__ arow, int nact, const T2* __restrict__ twx, int RW, IBVel vel) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    constexpr int HX = N / 3;   // highest retained kx (N1 = 2*(Ngal1/3))
    constexpr int NK = HX + 1;  // kx columns per row (= d.nkx)
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twx);
    const int z0 = blockIdx.x * RW, p = blockIdx.y, fb = blockIdx.z;
    const size_t pl = (size_t)d.ngal2 * NK;
    // line b of the CTA is active row arow[z0 + b] (the last one repeated past the end: the
    // repeated line writes the same values again)
    const T2* Hr = Hib + ((size_t)(2 * fb) * npl + p) * pl;
    const T2* Hu = vel.H ? (const T2*)vel.H + (size_t)(vel.voff[fb] + vel.planes[p] - vel.j0) * pl
                         : Hib + ((size_t)(2 * fb + 1) * npl + p) * pl;
    auto row_of_line = [&](int b) { return arow[min(z0 + b, nact - 1)]; };
    // this thread's offset within its stride-TN2 subsequence, computed as two_step_lines
    // does, so that e - n2 is a compile-time constant in the unrolled element loop
    const int tt = threadIdx.x;
    const int n2me = tt - (tt / TN2) * TN2;
    __syncthreads();
    // rows are read straight from global memory (consecutive threads, consecutive kx)
    auto load = [&](int e, int b) -> T2 {
        const int e0 = e - n2me;
        const bool lo = (e0 + TN2 - 1 <= HX) || (e0 <= HX && e <= HX);
        const bool hi = (e0 >= N - HX) || (e0 + TN2 - 1 >= N - HX && e >= N - HX);
        const size_t ro = (size_t)row_of_line(b) * NK;
        const T2* A = Hr + ro;
        const T2* C = Hu + ro;
        if (lo) {
            T2 a = A[e], c = C[e];
            if (e == 0) { a.y = 0; c.y = 0; }
            return cx<T2>(a.x - c.y, a.y + c.x);
        }
        if (hi) {
            const T2 a = A[N - e], c = C[N - e];
            return cx<T2>(a.x + c.y, -a.y + c.x);
        }
        return cx<T2>((R)0, (R)0);
    };
    const size_t ppl = (size_t)d.ngal2 * N;
    R* pr = phys + ((size_t)(2 * fb) * npl + p) * ppl;
    R* pu = phys + ((size_t)(2 * fb + 1) * npl + p) * ppl;
    auto store = [&](int x, int b, T2 v) {
        const size_t o = (size_t)row_of_line(b) * N + x;
        pr[o] = v.x;
        pu[o] = v.y;
    };
    two_step_lines<T2, TN1, TN2, +1, false>(0, ex, twt, load, store, RW);
}

// forward x of physical rhs rows (two rows per complex line), unpack, truncate, x 1/Ngal1
template <typename T2, int TN1, int TN2>
__global__ void k_ib_xfwd2(Dims d, T2* __restrict__ Hib, int npl, const decltype(T2::x)* __restrict__ phys,
                           const int* __restrict__ arow, int nact, const T2* __restrict__ twx, int RW) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    constexpr int LU = N + 1;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int nl = RW / 2;
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ub = twt + N;                                  // [nl][LU]
    T2* ex = ub + (size_t)nl * LU;
    load_twiddles<T2, TN1, TN2>(twt, twx);
    const int z0 = blockIdx.x * RW, p = blockIdx.y, fb = blockIdx.z;
    const size_t ppl = (size_t)d.ngal2 * N;
    const R* pr = phys + ((size_t)(2 * fb) * npl + p) * ppl;
    // line b packs active rows arow[z0 + 2b] and arow[z0 + 2b + 1] (the last repeated)
    auto row_of = [&](int r) { return arow[min(z0 + r, nact - 1)]; };
    __syncthreads();
    auto load = [&](int x, int b) -> T2 {
        return cx<T2>(pr[(size_t)row_of(2 * b) * N + x], pr[(size_t)row_of(2 * b + 1) * N + x]);
    };
    auto store = [&](int k, int b, T2 v) { ub[(size_t)b * LU + k] = v; };
    two_step_lines<T2, TN1, TN2, -1, false>(0, ex, twt, load, store, nl);
    const R hs = (R)0.5 / (R)N;
    constexpr int NK = N / 3 + 1;  // kx columns per row (= d.nkx)
    T2* Hr = Hib + ((size_t)(2 * fb) * npl + p) * (size_t)d.ngal2 * NK;
    // work items (line, k) flattened so that no lane idles on a partial last chunk
    for (int it = threadIdx.x; it < nl * NK; it += blockDim.x) {
        const int b = (unsigned)it / NK, k = it - b * NK;
        const T2* line = ub + (size_t)b * LU;
        const T2 Pk = line[k];
        const T2 Qc = cconj(line[k == 0 ? 0 : N - k]);
        Hr[(size_t)row_of(2 * b) * NK + k] = cx<T2>((Pk.x + Qc.x) * hs, (Pk.y + Qc.y) * hs);
        Hr[(size_t)row_of(2 * b + 1) * NK + k] = cx<T2>((Pk.y - Qc.y) * hs, -(Pk.x - Qc.x) * hs);
    }
}

template <typename T2, int TN1, int TN2>
__global__ void __launch_bounds__(16 * (TN1 > TN2 ? TN1 : TN2), (sizeof(T2) == 8 && (TN1 > TN2 ? TN1 : TN2) <= 24) ? 3 : 1) k_ib_zfwd2(Dims d, const T2* __restrict__ Hib, int npl, IBDst dst, int j0,
                           const int* __restrict__ planes, const unsigned char* __restrict__ rowflag,
                           const T2* __restrict__ twz, int lb) {
    using R = decltype(T2::x);
    constexpr int N = TN1 * TN2;
    const int nlines = npl * d.nkx;
    const int line0 = blockIdx.x << lb, fb = blockIdx.z;
    if (line0 >= nlines) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* twt = reinterpret_cast<T2*>(smem_raw);
    T2* ex = twt + N;
    load_twiddles<T2, TN1, TN2>(twt, twz);
    const int b = threadIdx.x & ((1 << lb) - 1);
    const bool live = line0 + b < nlines;
    const int line = live ? line0 + b : nlines - 1;
    const int p = line / d.nkx, i = line - p * d.nkx;
    const T2* H = Hib + ((size_t)(2 * fb) * npl + p) * (size_t)N * d.nkx + i;
    double2* out = dst.f[fb] + (size_t)(planes[p] - j0) * d.ncol + i;
    const int r = threadIdx.x >> lb;
    const R sc = (R)1 / (R)N;
    __syncthreads();
    // rows left out of the x round trip still get its one effect: the inverse real transform
    // ignores Im of the kx = 0 entry (rft_buff.f:78-80), so that entry leaves real
    const bool zero_im = rowflag && i == 0;
    auto load = [&](int z, int) -> T2 {
        T2 v = H[(size_t)z * d.nkx];
        if (zero_im && !rowflag[z]) v.y = (decltype(T2::x))0;
        return v;
    };
    auto store = [&](int e, int, T2 v) {
        const int q = zrow_q<N, TN1>(e, r);
        if (q >= 0 && live) out[(size_t)q * d.nkx] = to_d2(cscale(v, sc));
    };
    two_step_lines<T2, TN1, TN2, -1>(lb, ex, twt, load, store);
}

// --------------------------------------------------------------------------------------
// Implicit Helmholtz solves: LUsolU/LUsolV with LU_buildU/V + LU_dec computed on the fly
// (tridLU_3D_IB.f90:50-160, 349-413, 521-559).  One thread per (kx,kz) column; the
// forward sweep leaves y_j in the solution array and the scaled upper diagonal in `cs`.
// u and w share the matrix and its factorisation.
// --------------------------------------------------------------------------------------
// Loads of the sweeps are batched UB planes at a time so that each thread keeps several
// independent loads in flight while the recurrence runs on registers.
#define CFD_UB 8

__global__ void __launch_bounds__(256) k_solve_uvw(Dims d, Geo g, double beta, double2* __restrict__ u1,
                                                   double2* __restrict__ u2, double2* __restrict__ u3,
                                                   const double2* __restrict__ r1, const double2* __restrict__ r2,
                                                   const double2* __restrict__ r3, double* __restrict__ cs_uw,
                                                   double* __restrict__ cs_v, int part0) {
    // blockIdx.y + part0: 0 = the u/w systems, 1 = the v system
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double k2x = -g.kx[i] * g.kx[i], k2z = -g.kz[q] * g.kz[q];
    const size_t nc = d.ncol;
    if (blockIdx.y + part0 == 0) {
        // u and w share the matrix: rows (0,1,gwb), interior, (gwt,1,0)
        const int n = d.nyu;
        double dprev = 1.0, a3prev = g.gwb;
        double2 y1 = r1[col], y3 = r3[col];
        u1[col] = y1;
        u3[col] = y3;
        for (int j0 = 1; j0 < n; j0 += CFD_UB) {
            double2 ra[CFD_UB], rc[CFD_UB];
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t)
                if (j0 + t < n) { ra[t] = r1[(size_t)(j0 + t) * nc + col]; rc[t] = r3[(size_t)(j0 + t) * nc + col]; }
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t) {
                const int jj = j0 + t;
                if (jj >= n) break;
                double a1, a2, a3;
                if (jj < n - 1) {
                    a1 = -beta * g.dyu2i[3 * jj + 0];
                    a2 = 1.0 - beta * (g.dyu2i[3 * jj + 1] + k2x + k2z);
                    a3 = -beta * g.dyu2i[3 * jj + 2];
                } else {
                    a1 = g.gwt; a2 = 1.0; a3 = 0.0;
                }
                const double csm = a3prev * dprev;  // a(3,j-1) * a(2,j-1)
                cs_uw[(size_t)(jj - 1) * nc + col] = csm;
                const double dj = 1.0 / (a2 - a1 * csm);
                y1 = dscl(dj, dsub(ra[t], dscl(a1, y1)));
                y3 = dscl(dj, dsub(rc[t], dscl(a1, y3)));
                u1[(size_t)jj * nc + col] = y1;
                u3[(size_t)jj * nc + col] = y3;
                dprev = dj;
                a3prev = a3;
            }
        }
        double2 x1 = y1, x3 = y3;
        for (int j0 = n - 2; j0 >= 0; j0 -= CFD_UB) {
            double cc[CFD_UB];
            double2 ya[CFD_UB], yc[CFD_UB];
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t)
                if (j0 - t >= 0) {
                    const size_t o = (size_t)(j0 - t) * nc + col;
                    cc[t] = cs_uw[o]; ya[t] = u1[o]; yc[t] = u3[o];
                }
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t) {
                if (j0 - t < 0) break;
                const size_t o = (size_t)(j0 - t) * nc + col;
                x1 = dsub(ya[t], dscl(cc[t], x1));
                x3 = dsub(yc[t], dscl(cc[t], x3));
                u1[o] = x1;
                u3[o] = x3;
            }
        }
    } else {
        // v: identity wall rows
        const int n = d.nyv;
        double dprev = 1.0, a3prev = 0.0;
        double2 y = r2[col];
        u2[col] = y;
        for (int j0 = 1; j0 < n; j0 += CFD_UB) {
            double2 ra[CFD_UB];
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t)
                if (j0 + t < n) ra[t] = r2[(size_t)(j0 + t) * nc + col];
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t) {
                const int jj = j0 + t;
                if (jj >= n) break;
                double a1, a2, a3;
                if (jj < n - 1) {
                    a1 = -beta * g.dyv2i[3 * jj + 0];
                    a2 = 1.0 - beta * (g.dyv2i[3 * jj + 1] + k2x + k2z);
                    a3 = -beta * g.dyv2i[3 * jj + 2];
                } else {
                    a1 = 0.0; a2 = 1.0; a3 = 0.0;
                }
                const double csm = a3prev * dprev;
                cs_v[(size_t)(jj - 1) * nc + col] = csm;
                const double dj = 1.0 / (a2 - a1 * csm);
                y = dscl(dj, dsub(ra[t], dscl(a1, y)));
                u2[(size_t)jj * nc + col] = y;
                dprev = dj;
                a3prev = a3;
            }
        }
        double2 x = y;
        for (int j0 = n - 2; j0 >= 0; j0 -= CFD_UB) {
            double cc[CFD_UB];
            double2 ya[CFD_UB];
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t)
                if (j0 - t >= 0) {
                    const size_t o = (size_t)(j0 - t) * nc + col;
                    cc[t] = cs_v[o]; ya[t] = u2[o];
                }
#pragma unroll
            for (int t = 0; t < CFD_UB; ++t) {
                if (j0 - t < 0) break;
                x = dsub(ya[t], dscl(cc[t], x));
                u2[(size_t)(j0 - t) * nc + col] = x;
            }
        }
    }
}

// --------------------------------------------------------------------------------------
// solveP (littleharsh.f90:556-611): divergence (:209-244), psi = div/(dt(a+b)),
// psi(mean, bottom) = 0, LUsolP with the D.G matrix of LU_buildP/LU_decP computed on
// the fly (tridLU_3D_IB.f90:284-318, 417-491, 562-603), p += psi.
// --------------------------------------------------------------------------------------
template <bool FUSE>
__global__ void __launch_bounds__(256) k_solve_p(Dims d, Geo g, double dtirk, double2* __restrict__ u1,
                                                 double2* __restrict__ u2, double2* __restrict__ u3,
                                                 double2* __restrict__ p, double2* __restrict__ psi,
                                                 double2* __restrict__ divo, double* __restrict__ cs, double mean_diag,
                                                 double dtrk) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const double k2x = -kxv * kxv, k2z = -kzv * kzv;
    const size_t nc = d.ncol;
    const int n = d.nyp;
    // D.G coefficients: D_b(m) = -dthdyu(m+1), G_b(m) = -dthdyv(m), D_t(m) = dthdyu(m), G_t(m) = dthdyv(m-1)
    auto DTHU = [&](int j) { return g.dthdyu[j - d.ju0]; };
    auto DTHV = [&](int j) { return g.dthdyv[j - d.jv0]; };
    double dprev = 0.0, a3prev = 0.0;
    double2 y = dc(0, 0);
    double2 vb = u2[(size_t)(d.jp0 - 1 - d.jv0) * nc + col];
    for (int jj0 = 0; jj0 < n; jj0 += CFD_UB) {
        double2 A[CFD_UB], W[CFD_UB], VA[CFD_UB];
#pragma unroll
        for (int t = 0; t < CFD_UB; ++t)
            if (jj0 + t < n) {
                const int j = d.jp0 + jj0 + t;
                A[t] = u1[(size_t)(j - d.ju0) * nc + col];
                W[t] = u3[(size_t)(j - d.ju0) * nc + col];
                VA[t] = u2[(size_t)(j - d.jv0) * nc + col];
            }
#pragma unroll
        for (int t = 0; t < CFD_UB; ++t) {
            const int jj = jj0 + t;
            if (jj >= n) break;
            const int j = d.jp0 + jj;
            // divergence at p-point j
            const double2 dv = dadd(dadd(dik(kxv, A[t]), dik(kzv, W[t])), dscl(DTHU(j), dsub(VA[t], vb)));
            vb = VA[t];
            if (divo) divo[(size_t)jj * nc + col] = dv;
            double2 r = dscl(dtirk, dv);
            double a1, a2, a3;
            if (jj == 0) {
                a1 = 0.0;
                a2 = (DTHU(j) * -DTHV(j)) + k2x + k2z;
                a3 = (DTHU(j) * DTHV(j));
                if (col == 0) { a2 = mean_diag; a3 = 0.0; r = dc(0, 0); }
            } else if (jj == n - 1) {
                a1 = (-DTHU(j)) * (-DTHV(j - 1));
                a2 = ((-DTHU(j)) * DTHV(j - 1)) + k2x + k2z;
                a3 = 0.0;
            } else {
                a2 = ((-DTHU(j)) * DTHV(j - 1)) + (DTHU(j) * -DTHV(j)) + k2x + k2z;
                a1 = ((-DTHU(j)) * (-DTHV(j - 1)));
                a3 = (DTHU(j) * DTHV(j));
            }
            double dj;
            if (jj == 0) {
                dj = 1.0 / a2;
                y = dscl(dj, r);
            } else {
                const double csm = a3prev * dprev;
                cs[(size_t)(jj - 1) * nc + col] = csm;
                dj = 1.0 / (a2 - a1 * csm);
                y = dscl(dj, dsub(r, dscl(a1, y)));
            }
            psi[(size_t)jj * nc + col] = y;
            dprev = dj;
            a3prev = a3;
        }
    }
    double2 x = y;
    p[(size_t)(n - 1) * nc + col] = dadd(p[(size_t)(n - 1) * nc + col], x);
    if (FUSE) {
        // v_corr (littleharsh.f90:796-907) in the back sweep: centre j = jp0 + jj takes
        // psi(j); face j takes psi(j+1) - psi(j) (faces jv0+1..jv1-1); ghost/wall rows last
        const size_t ju = (size_t)(d.jp1 - d.ju0);
        u1[ju * nc + col] = dsub(u1[ju * nc + col], dik(dtrk * kxv, x));
        u3[ju * nc + col] = dsub(u3[ju * nc + col], dik(dtrk * kzv, x));
        u1[(ju + 1) * nc + col] = dscl(-g.gwt, u1[ju * nc + col]);
        u3[(ju + 1) * nc + col] = dscl(-g.gwt, u3[ju * nc + col]);
    }
    for (int jj0 = n - 2; jj0 >= 0; jj0 -= CFD_UB) {
        double cc[CFD_UB];
        double2 ya[CFD_UB], pa[CFD_UB], ua[CFD_UB], wa[CFD_UB], va[CFD_UB];
#pragma unroll
        for (int t = 0; t < CFD_UB; ++t)
            if (jj0 - t >= 0) {
                const size_t o = (size_t)(jj0 - t) * nc + col;
                cc[t] = cs[o]; ya[t] = psi[o]; pa[t] = p[o];
                if (FUSE) {
                    const int j = d.jp0 + jj0 - t;
                    ua[t] = u1[(size_t)(j - d.ju0) * nc + col];
                    wa[t] = u3[(size_t)(j - d.ju0) * nc + col];
                    va[t] = u2[(size_t)(j - d.jv0) * nc + col];
                }
            }
#pragma unroll
        for (int t = 0; t < CFD_UB; ++t) {
            if (jj0 - t < 0) break;
            const size_t o = (size_t)(jj0 - t) * nc + col;
            const double2 xp = x;  // psi(j+1)
            x = dsub(ya[t], dscl(cc[t], x));
            if (!FUSE) psi[o] = x;
            p[o] = dadd(pa[t], x);
            if (FUSE) {
                const int j = d.jp0 + jj0 - t;
                u1[(size_t)(j - d.ju0) * nc + col] = dsub(ua[t], dik(dtrk * kxv, x));
                u3[(size_t)(j - d.ju0) * nc + col] = dsub(wa[t], dik(dtrk * kzv, x));
                const size_t jv = (size_t)(j - d.jv0);
                u2[jv * nc + col] = dsub(va[t], dscl(dtrk * g.dthdyv[jv], dsub(xp, x)));
            }
        }
    }
    if (FUSE) {
        u1[col] = dscl(-g.gwb, u1[nc + col]);
        u3[col] = dscl(-g.gwb, u3[nc + col]);
        u2[col] = dc(0, 0);
        u2[(size_t)(d.nyv - 1) * nc + col] = dc(0, 0);
    }
}

// v_corr without the closing divergence, one thread per column and a chunk of JC planes
// (the fused substep; cfd_vcorr keeps the sequential k_vcorr that also returns div).
__global__ void __launch_bounds__(256) k_vcorr_chunk(Dims d, Geo g, double dtrk, double2* __restrict__ u1,
                                                     double2* __restrict__ u2, double2* __restrict__ u3,
                                                     const double2* __restrict__ psi, int JC) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const size_t nc = d.ncol;
    const int cb = blockIdx.y;
    // u, w at centres j = ju0+1..ju1-1 (= p-points)
    const int jb = d.ju0 + 1 + cb * JC, je = min(jb + JC, d.ju1);
    for (int j = jb; j < je; ++j) {
        const size_t ju = (size_t)(j - d.ju0);
        const double2 ps = psi[(size_t)(j - d.jp0) * nc + col];
        u1[ju * nc + col] = dsub(u1[ju * nc + col], dik(dtrk * kxv, ps));
        u3[ju * nc + col] = dsub(u3[ju * nc + col], dik(dtrk * kzv, ps));
    }
    // v at faces j = jv0+1..jv1-1: psi(j+1) - psi(j)
    const int vb = d.jv0 + 1 + cb * JC, ve = min(vb + JC, d.jv1);
    for (int j = vb; j < ve; ++j) {
        const size_t jv = (size_t)(j - d.jv0);
        const double2 pa = psi[(size_t)(j + 1 - d.jp0) * nc + col], pb = psi[(size_t)(j - d.jp0) * nc + col];
        u2[jv * nc + col] = dsub(u2[jv * nc + col], dscl(dtrk * g.dthdyv[jv], dsub(pa, pb)));
    }
    if (cb == 0) {
        u2[col] = dc(0, 0);
        u2[(size_t)(d.nyv - 1) * nc + col] = dc(0, 0);
        // chunk 0 has just corrected u(ju0+1), the row the bottom ghost extrapolates from
        u1[col] = dscl(-g.gwb, u1[nc + col]);
        u3[col] = dscl(-g.gwb, u3[nc + col]);
    }
    if (je == d.ju1 && jb < je) {
        u1[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u1[(size_t)(d.nyu - 2) * nc + col]);
        u3[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u3[(size_t)(d.nyu - 2) * nc + col]);
    }
}

// v_corr (littleharsh.f90:796-907): u -= dt(a+b) ikx psi, w -= dt(a+b) ikz psi,
// v -= dt(a+b) dthdyv (psi(j+1)-psi(j)), ghost rows by gridweighting, v walls 0, and the
// closing divergence (optional).
__global__ void __launch_bounds__(256) k_vcorr(Dims d, Geo g, double dtrk, double2* __restrict__ u1,
                                               double2* __restrict__ u2, double2* __restrict__ u3,
                                               const double2* __restrict__ psi, double2* __restrict__ divo) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const size_t nc = d.ncol;
    double2 psim = dc(0, 0);
    double2 vprev = dc(0, 0);
    for (int j = d.ju0 + 1; j <= d.ju1 - 1; ++j) {
        const size_t ju = (size_t)(j - d.ju0), jp = (size_t)(j - d.jp0), jv = (size_t)(j - d.jv0);
        const double2 ps = psi[jp * nc + col];
        const double2 a = dsub(u1[ju * nc + col], dik(dtrk * kxv, ps));
        const double2 w = dsub(u3[ju * nc + col], dik(dtrk * kzv, ps));
        u1[ju * nc + col] = a;
        u3[ju * nc + col] = w;
        // v at face j-1 (interior faces jv0+1..jv1-1) uses psi(j) - psi(j-1)
        if (j - 1 >= d.jv0 + 1) {
            const size_t jvm = jv - 1;
            const double2 vn = dsub(u2[jvm * nc + col], dscl(dtrk * g.dthdyv[jvm], dsub(ps, psim)));
            u2[jvm * nc + col] = vn;
            if (divo) {
                // divergence at p-point j-1 now that u(j-1), w(j-1), v(j-1), v(j-2) are final
                const double2 am = u1[(ju - 1) * nc + col], wm = u3[(ju - 1) * nc + col];
                divo[(jp - 1) * nc + col] = dadd(dadd(dik(kxv, am), dik(kzv, wm)), dscl(g.dthdyu[ju - 1], dsub(vn, vprev)));
            }
            vprev = vn;
        } else {
            vprev = dc(0, 0);  // wall v(jv0) = 0
        }
        psim = ps;
    }
    u2[col] = dc(0, 0);
    u2[(size_t)(d.nyv - 1) * nc + col] = dc(0, 0);
    u1[col] = dscl(-g.gwb, u1[nc + col]);
    u3[col] = dscl(-g.gwb, u3[nc + col]);
    u1[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u1[(size_t)(d.nyu - 2) * nc + col]);
    u3[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u3[(size_t)(d.nyu - 2) * nc + col]);
    if (divo) {
        // last p-point j = jp1: v(jv1) = 0 (wall)
        const int j = d.jp1;
        const size_t ju = (size_t)(j - d.ju0), jp = (size_t)(j - d.jp0);
        const double2 am = u1[ju * nc + col], wm = u3[ju * nc + col];
        divo[jp * nc + col] = dadd(dadd(dik(kxv, am), dik(kzv, wm)), dscl(g.dthdyu[ju], dsub(dc(0, 0), vprev)));
    }
}

// --------------------------------------------------------------------------------------
// Mean mode: flowrate_corr with LUsol0/LU_build0/LU_dec0 (littleharsh.f90:452-484,
// tridLU_3D_IB.f90:320-346, 493-519, 605-622) and flowrateIm (littleharsh.f90:411-430).
// scal[0] = mpgx, scal[1] = Qx, scal[2] = dgx.  One thread.  The unit-response column
// spans j = 0..ny (cells between the crests plus one each side), as in the reference.
// --------------------------------------------------------------------------------------
__global__ void k_meanflow(Dims d, Geo g, double beta, double bdt, double qxt, int ctpress, double2* __restrict__ u1,
                           double* __restrict__ scal, double* __restrict__ work) {
    // one warp: the flow-rate sums and the final update spread over the lanes (strided
    // reads of the mean-mode column), the tridiagonal solve of the mean mode on lane 0
    if (blockIdx.x != 0) return;
    const int lane = threadIdx.x & 31;
    const int nn = d.ny - 2;
    auto YV = [&](int j) { return g.yv[j - d.jv0]; };
    auto wsum = [](double v) {
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    };
    double Qx0 = 0.0;
    for (int j = 1 + lane; j <= nn + 1; j += 32) Qx0 += (YV(j) - YV(j - 1)) * u1[(size_t)(j - d.ju0) * d.ncol].x;
    Qx0 = wsum(Qx0);
    if (ctpress == 1) {
        if (lane == 0) scal[1] = Qx0;
        return;
    }
    const int n = nn + 3;
    double* a1 = work;
    double* a2 = work + n;
    double* a3 = work + 2 * n;
    double* x = work + 3 * n;
    for (int j = 1 + lane; j <= nn + 1; j += 32) {
        const int jj = j - d.ju0;
        a1[j] = -beta * g.dyu2i[3 * jj + 0];
        a2[j] = 1.0 - beta * g.dyu2i[3 * jj + 1];
        a3[j] = -beta * g.dyu2i[3 * jj + 2];
    }
    __syncwarp();
    if (lane == 0) {
        a1[0] = 0.0; a2[0] = 1.0; a3[0] = g.gwb;
        a1[nn + 2] = g.gwt; a2[nn + 2] = 1.0; a3[nn + 2] = 0.0;
        a2[0] = 1.0 / a2[0];
        for (int j = 1; j < n; ++j) {
            a3[j - 1] = a3[j - 1] * a2[j - 1];
            a2[j] = 1.0 / (a2[j] - a1[j] * a3[j - 1]);
        }
        x[0] = 0.0 * a2[0];
        for (int j = 1; j < n; ++j) {
            const double rj = (j <= nn + 1) ? bdt : 0.0;
            x[j] = (rj - a1[j] * x[j - 1]) * a2[j];
        }
        for (int j = n - 2; j >= 0; --j) x[j] = x[j] - a3[j] * x[j + 1];
    }
    __syncwarp();
    double Qx1 = 0.0;
    for (int j = 1 + lane; j <= nn + 1; j += 32) Qx1 += (YV(j) - YV(j - 1)) * x[j];
    Qx1 = wsum(Qx1);
    const double gg = (qxt - Qx0) / Qx1;
    if (lane == 0) {
        scal[0] = scal[0] + gg;
        scal[2] = gg;
    }
    for (int j = lane; j <= nn + 2; j += 32) u1[(size_t)(j - d.ju0) * d.ncol].x += gg * x[j];
}

// --------------------------------------------------------------------------------------
// Layout conversion f(j,column) <-> [j][column] (32x32 tiles through shared memory).
// --------------------------------------------------------------------------------------
__global__ void k_transpose(const double2* __restrict__ in, double2* __restrict__ out, int rows, int cols,
                            int ldi, int ldo) {
    // in: [rows][cols] with row stride ldi -> out: [cols][rows] with row stride ldo
    __shared__ double2 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const int r = by + yy, c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[yy][threadIdx.x] = in[(size_t)r * ldi + c];
    }
    __syncthreads();
    for (int yy = threadIdx.y; yy < 32; yy += blockDim.y) {
        const int c = bx + yy, r = by + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * ldo + r] = tile[threadIdx.x][yy];
    }
}

// divergence at every p-point (littleharsh.f90:209-244), no state change
__global__ void __launch_bounds__(256) k_divergence(Dims d, Geo g, const double2* __restrict__ u1,
                                                    const double2* __restrict__ u2, const double2* __restrict__ u3,
                                                    double2* __restrict__ divo) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const double kxv = g.kx[col % d.nkx], kzv = g.kz[col / d.nkx];
    const size_t nc = d.ncol;
    for (int j = d.jp0; j <= d.jp1; ++j) {
        const size_t ju = (size_t)(j - d.ju0), jv = (size_t)(j - d.jv0);
        divo[(size_t)(j - d.jp0) * nc + col] =
            dadd(dadd(dik(kxv, u1[ju * nc + col]), dik(kzv, u3[ju * nc + col])),
                 dscl(g.dthdyu[ju], dsub(u2[jv * nc + col], u2[(jv - 1) * nc + col])));
    }
}

// per-block max |z| of a complex array (error(), littleharsh.f90:322-351)
__global__ void k_absmax(const double2* __restrict__ a, size_t n, double* __restrict__ part) {
    __shared__ double sm[256];
    double m = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const double2 v = a[t];
        m = nan_max(m, sqrt(v.x * v.x + v.y * v.y));
    }
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sm[threadIdx.x] = nan_max(sm[threadIdx.x], sm[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// --------------------------------------------------------------------------------------
// Generic strided transforms with the reference wrapper semantics (cft_buff.f:1-65,
// rft_buff.f:24-86), FP64.  Lines are gathered into shared memory, transformed, scattered.
// grid: x = chunk of CH lines, y = batch (plane) with stride `bstride` doubles.
// --------------------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_cft_strided(double* __restrict__ c, int ise, int isa, int m, long long bstride,
                                                     FFTDesc fd, const double2* __restrict__ tw_g, int iopt, int CH) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = fd.n;
    double2* buf0 = reinterpret_cast<double2*>(smem_raw);
    double2* buf1 = buf0 + (size_t)n * CH;
    double2* tw = buf1 + (size_t)n * CH;
    double* base = c + (size_t)blockIdx.y * bstride;
    const int l0 = blockIdx.x * CH;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = tw_g[t];
    for (int t = threadIdx.x; t < n * CH; t += blockDim.x) {
        const int b = t % CH, e = t / CH, l = l0 + b;
        buf0[swz(e, b, __ffs(CH) - 1)] =
            l < m ? dc(base[(size_t)l * isa + (size_t)e * ise], base[(size_t)l * isa + (size_t)e * ise + 1]) : dc(0, 0);
    }
    __syncthreads();
    double2* res = fft_lines<double2>(buf0, buf1, CH, fd, tw, iopt < 0 ? -1 : +1);
    const double s = iopt < 0 ? 1.0 / n : 1.0;
    for (int t = threadIdx.x; t < n * CH; t += blockDim.x) {
        const int b = t % CH, e = t / CH, l = l0 + b;
        if (l < m) {
            const double2 v = res[swz(e, b, __ffs(CH) - 1)];
            base[(size_t)l * isa + (size_t)e * ise] = s * v.x;
            base[(size_t)l * isa + (size_t)e * ise + 1] = s * v.y;
        }
    }
}

__global__ void __launch_bounds__(256) k_rft_strided(double* __restrict__ c, int isa, int m, long long bstride,
                                                     FFTDesc fd, const double2* __restrict__ tw_g, int iopt, int CH) {
    // forward: each line a complex transform of length n of (real, 0) data, FFTPACK
    // storage; inverse: two lines per complex transform
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int n = fd.n;
    double2* buf0 = reinterpret_cast<double2*>(smem_raw);
    double2* buf1 = buf0 + (size_t)n * CH;
    double2* tw = buf1 + (size_t)n * CH;
    double* base = c + (size_t)blockIdx.y * bstride;
    const int l0 = blockIdx.x * CH;
    for (int t = threadIdx.x; t < n; t += blockDim.x) tw[t] = tw_g[t];
    if (iopt > 0) {
        // inverse: CTA line slot b carries the line pair (2(l0+b), 2(l0+b)+1) as one complex
        // transform of X_a + i X_b (both Hermitian extensions of cc(0..n/2), Im cc(0) and
        // Im cc(n/2) ignored), whose output is x_a + i x_b
        for (int t = threadIdx.x; t < n * CH; t += blockDim.x) {
            const int b = t % CH, k = t / CH, la = 2 * (l0 + b), lb = la + 1;
            double2 A = dc(0, 0), B = dc(0, 0);
            const int kk = k <= n / 2 ? k : n - k;
            const bool edge = kk == 0 || kk == n / 2;
            if (la < m) { const double* x = base + (size_t)la * isa; A = dc(x[2 * kk], edge ? 0.0 : x[2 * kk + 1]); }
            if (lb < m) { const double* x = base + (size_t)lb * isa; B = dc(x[2 * kk], edge ? 0.0 : x[2 * kk + 1]); }
            if (k > n / 2) { A.y = -A.y; B.y = -B.y; }
            buf0[swz(k, b, __ffs(CH) - 1)] = dc(A.x - B.y, A.y + B.x);
        }
        __syncthreads();
        double2* res = fft_lines<double2>(buf0, buf1, CH, fd, tw, +1);
        for (int t = threadIdx.x; t < n * CH; t += blockDim.x) {
            const int b = t % CH, e = t / CH, la = 2 * (l0 + b), lb = la + 1;
            const double2 v = res[swz(e, b, __ffs(CH) - 1)];
            if (la < m) base[(size_t)la * isa + e] = v.x;
            if (lb < m) base[(size_t)lb * isa + e] = v.y;
        }
        return;
    }
    for (int t = threadIdx.x; t < n * CH; t += blockDim.x) {
        const int b = t % CH, k = t / CH, l = l0 + b;
        double2 v = dc(0, 0);
        if (l < m) v = dc(base[(size_t)l * isa + k], 0.0);
        buf0[swz(k, b, __ffs(CH) - 1)] = v;
    }
    __syncthreads();
    double2* res = fft_lines<double2>(buf0, buf1, CH, fd, tw, -1);
    for (int t = threadIdx.x; t < (n + 2) * CH; t += blockDim.x) {
        const int b = t % CH, e = t / CH, l = l0 + b;
        if (l >= m) continue;
        double* x = base + (size_t)l * isa;
        const int k = e >> 1;
        const double2 v = res[swz(k, b, __ffs(CH) - 1)];
        double val = (e & 1) ? v.y : v.x;
        if ((e & 1) && (k == 0 || k == n / 2)) val = 0.0;
        x[e] = val / n;
    }
}

}  // namespace cfd
