// stats_kernels.cuh - FP64 statistics and CFL maxima on physical planes (sm_100a).
//
// The statistics pass of the reference (stats.f90:1-253, called from nonlinear at kRK = 1,
// FOU3D.f90:187-217) and dtc_calc (FOU3D.f90:516-544) work on physical planes of
// u, v, w, the y-interpolated v (u planes) and w (v planes), p and omega_x.  The pass
// builds those planes chunk by chunk in the reference's plane layout xPL(Ngal1+2, Ngal2),
// transforms them with the FP64 strided FFTs, and reduces them:
//   k_st_build   spectral columns -> plane layout, as a y-combination of up to two planes
//                plus an optional i*kz term (the interpolations of interp_u/interp_v and
//                omega_x = dw/dy - dv/dz at the faces)
//   k_st_sums    ns CTAs per plane: partial plane sums (deterministic tree) and |.| maxima
//   k_st_fin     the partials of each plane added in slice order into the accumulators
//   k_st_cond    one thread per tile point and segment of tile rows: the tile-folded
//                (conditional) sums of the segment in the reference's loop order
//   k_st_cond_fin the segments added in order to the band accumulators
#pragma once

#include "channel_kernels.cuh"

namespace cfd {

// out(column) = ca*a + cb*b + cc*(i kz) c; the kz term is zero on the kz = -N2/2 row
// (the dealiasing zero of der_z, FOU3D.f90:388-412).  b, c may be null.
struct PlaneSrc {
    const double2* a;
    const double2* b;
    const double2* c;
    double ca, cb, cc;
};

// grid: x = row blocks, y = output plane.  Each thread writes one (row, kx) complex slot
// of the plane (entries 2i, 2i+1 of the row); rows and kx slots with no mode get zero.
__global__ void __launch_bounds__(256) k_st_build(Dims d, Geo g, const PlaneSrc* __restrict__ src,
                                                  double* __restrict__ planes) {
    const int pl = blockIdx.y;
    const PlaneSrc s = src[pl];
    const int rowc = (d.ngal1 + 2) / 2;  // complex slots per row
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= rowc * d.ngal2) return;
    const int z = idx / rowc, i = idx - z * rowc;
    const int hq = d.n2 / 2;
    int q = -1;
    if (z < hq) q = z;
    else if (z >= d.ngal2 - hq) q = z - (d.ngal2 - d.n2);
    double2 v = dc(0.0, 0.0);
    if (q >= 0 && i < d.nkx) {
        const size_t col = (size_t)q * d.nkx + i;
        const double2 a = s.a[col];
        v = dc(s.ca * a.x, s.ca * a.y);
        if (s.b) {
            const double2 b = s.b[col];
            v = dc(v.x + s.cb * b.x, v.y + s.cb * b.y);
        }
        if (s.c && q != hq) v = dadd(v, dscl(s.cc, dik(g.kz[q], s.c[col])));
    }
    reinterpret_cast<double2*>(planes + (size_t)pl * (d.ngal1 + 2) * d.ngal2)[idx] = v;
}

// Per-plane reductions.  kind 0: u planes, fields (u, w, v_itp) -> Um U2m Wm W2m UVm UWm,
// maxima |u|, |w|.  kind 1: v planes, fields (v, w_itp, wx) -> Vm V2m wxm wx2m VWm (wx over
// the first N1 x N2 points, stats.f90:53-60), maximum |v| * dthdyv(j) on interior planes.
// kind 2: p planes -> Pm P2m.  Each plane j0+pl of the chunk adds its sums to acc[q][j]
// (one writer per entry) and stores its maxima in mx[q][j].
template <int KIND>
__global__ void __launch_bounds__(256) k_st_sums(Dims d, const double* __restrict__ planes, int nchunk,
                                                 double* __restrict__ part) {
    constexpr int NQ = KIND == 0 ? 6 : (KIND == 1 ? 5 : 2);
    const int sl = blockIdx.x, ns = gridDim.x;   // slice of the plane
    const int pl = blockIdx.y;
    const size_t ps = (size_t)(d.ngal1 + 2) * d.ngal2;
    const double* f0 = planes + (size_t)pl * ps;
    const double* f1 = planes + (size_t)(nchunk + pl) * ps;
    const double* f2 = planes + (size_t)(2 * nchunk + pl) * ps;
    double s[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) s[k] = 0.0;
    double m0 = 0.0, m1 = 0.0;
    const int L = d.ngal1 + 2;
    const int npts = d.ngal1 * d.ngal2;
    for (int t = sl * blockDim.x + threadIdx.x; t < npts; t += ns * blockDim.x) {
        const int k = t / d.ngal1, i = t - k * d.ngal1;
        const size_t o = (size_t)k * L + i;
        const double x0 = f0[o];
        if (KIND == 0) {
            const double x1 = f1[o], x2 = f2[o];
            s[0] += x0; s[1] += x0 * x0; s[2] += x1; s[3] += x1 * x1; s[4] += x0 * x2; s[5] += x0 * x1;
            m0 = nan_max(m0, fabs(x0)); m1 = nan_max(m1, fabs(x1));
        } else if (KIND == 1) {
            const double x1 = f1[o];
            s[0] += x0; s[1] += x0 * x0; s[4] += x0 * x1;
            if (i < d.n1 && k < d.n2) { const double x2 = f2[o]; s[2] += x2; s[3] += x2 * x2; }
            m0 = nan_max(m0, fabs(x0));
        } else {
            s[0] += x0; s[1] += x0 * x0;
        }
    }
    __shared__ double red[(NQ + 2) * 256];
#pragma unroll
    for (int k = 0; k < NQ; ++k) red[k * 256 + threadIdx.x] = s[k];
    red[NQ * 256 + threadIdx.x] = m0;
    red[(NQ + 1) * 256 + threadIdx.x] = m1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
#pragma unroll
            for (int k = 0; k < NQ; ++k) red[k * 256 + threadIdx.x] += red[k * 256 + threadIdx.x + w];
            red[NQ * 256 + threadIdx.x] = nan_max(red[NQ * 256 + threadIdx.x], red[NQ * 256 + threadIdx.x + w]);
            red[(NQ + 1) * 256 + threadIdx.x] =
                nan_max(red[(NQ + 1) * 256 + threadIdx.x], red[(NQ + 1) * 256 + threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x < NQ + 2) part[((size_t)pl * ns + sl) * (NQ + 2) + threadIdx.x] = red[threadIdx.x * 256];
}

// The partial sums of the slices of each plane, added in slice order (deterministic), into
// the plane accumulators; the maxima of |.| per plane for the CFL query.  One thread per plane.
template <int KIND>
__global__ void k_st_fin(Dims d, Geo g, const double* __restrict__ part, int nchunk, int ns, int jrel0,
                         double* __restrict__ acc, int nyg, double* __restrict__ mx) {
    constexpr int NQ = KIND == 0 ? 6 : (KIND == 1 ? 5 : 2);
    constexpr int NM = KIND == 0 ? 2 : (KIND == 1 ? 1 : 0);
    const int pl = blockIdx.x * blockDim.x + threadIdx.x;
    if (pl >= nchunk) return;
    const int jr = jrel0 + pl;  // plane index within its grid (j - j0 of the grid)
    double s[NQ + 2];
#pragma unroll
    for (int k = 0; k < NQ + 2; ++k) s[k] = 0.0;
    for (int sl = 0; sl < ns; ++sl) {
        const double* q = part + ((size_t)pl * ns + sl) * (NQ + 2);
#pragma unroll
        for (int k = 0; k < NQ; ++k) s[k] += q[k];
        s[NQ] = nan_max(s[NQ], q[NQ]);
        s[NQ + 1] = nan_max(s[NQ + 1], q[NQ + 1]);
    }
    if (acc)
#pragma unroll
        for (int k = 0; k < NQ; ++k) acc[(size_t)k * nyg + jr] += s[k];
    if (NM >= 1) {
        double v = s[NQ];
        if (KIND == 1) v = (jr > 0 && jr < nyg - 1) ? v * g.dthdyv[jr] : 0.0;
        mx[jr] = v;
    }
    if (NM >= 2) mx[nyg + jr] = s[NQ + 1];
}

// Conditional sums of one chunk.  grid: x = blocks of (segment, tile point), y = plane of
// the chunk.  Plane j (index jr in its grid) is a bottom-band plane when jr < nb (j1 = jr)
// and a top-band plane when nyg-1-jr < nb (j1 = nyg-1-jr, v sign-flipped: condup1/condup2).
// The nseg segments split the tile rows iz; each thread adds the points of its tile point
// in its segment in the reference's loop order (iz, then ix) and writes the partial sums
// part[((pl*2 + side)*nseg + seg)*NQ + k][t]; k_st_cond_fin adds the segments in order to
// the accumulators cb/ct [NQ][nb][dnz][dnx] of the bottom and the top band.  With one
// segment the thread adds straight onto the accumulator.
template <int KIND>
__global__ void __launch_bounds__(256) k_st_cond(Dims d, const double* __restrict__ planes, int nchunk, int jrel0,
                                                 int nyg, int nb, int dnx, int dnz, int nseg,
                                                 double* __restrict__ part, double* __restrict__ cbot,
                                                 double* __restrict__ ctop) {
    constexpr int NQ = KIND == 0 ? 6 : (KIND == 1 ? 5 : 2);
    const int pl = blockIdx.y;
    const int jr = jrel0 + pl;
    const int tsz = dnx * dnz;
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= tsz * nseg) return;
    if (jr >= nb && nyg - 1 - jr >= nb) return;   // a plane of neither band
    const int seg = u / tsz, t = u - seg * tsz;
    const int tk = t / dnx, ti = t - tk * dnx;
    const int ntx = d.ngal1 / dnx, ntz = d.ngal2 / dnz;
    const int iz0 = (int)((long long)ntz * seg / nseg), iz1 = (int)((long long)ntz * (seg + 1) / nseg);
    const size_t ps = (size_t)(d.ngal1 + 2) * d.ngal2;
    const int L = d.ngal1 + 2;
    const double* f0 = planes + (size_t)pl * ps;
    const double* f1 = planes + (size_t)(nchunk + pl) * ps;
    const double* f2 = planes + (size_t)(2 * nchunk + pl) * ps;
    for (int side = 0; side < 2; ++side) {
        const int j1 = side == 0 ? jr : nyg - 1 - jr;
        if (j1 < 0 || j1 >= nb) continue;
        // sign of v in the top band (condup1 xsign = -1 for v, condup2 -1 on the v factor)
        const double sv = (side == 1) ? -1.0 : 1.0;
        // one segment: add straight onto the accumulator (the reference's order throughout)
        double* C = (side == 0 ? cbot : ctop) + (size_t)j1 * tsz + t;
        const size_t qs = (size_t)nb * tsz;  // stride between quantities
        double a[NQ];
#pragma unroll
        for (int k = 0; k < NQ; ++k) a[k] = nseg == 1 ? C[k * qs] : 0.0;
        for (int iz = iz0; iz < iz1; ++iz) {
            const size_t ro = (size_t)(tk + dnz * iz) * L + ti;
            for (int ix = 0; ix < ntx; ++ix) {
                const size_t o = ro + (size_t)dnx * ix;
                const double x0 = f0[o];
                if (KIND == 0) {  // u, w, v_itp: U U2 W W2 UV UW
                    const double x1 = f1[o], x2 = f2[o];
                    a[0] += x0;
                    a[1] += x0 * x0;
                    a[2] += x1;
                    a[3] += x1 * x1;
                    a[4] += x0 * (x2 * sv);
                    a[5] += x0 * x1;
                } else if (KIND == 1) {  // v, w_itp, wx: V V2 wx wx2 VW
                    const double x1 = f1[o], x2 = f2[o];
                    a[0] += x0 * sv;
                    a[1] += x0 * x0;
                    a[2] += x2;
                    a[3] += x2 * x2;
                    a[4] += (x0 * sv) * x1;
                } else {
                    a[0] += x0;
                    a[1] += x0 * x0;
                }
            }
        }
        if (nseg == 1) {
#pragma unroll
            for (int k = 0; k < NQ; ++k) C[k * qs] = a[k];
        } else {
            double* P = part + ((size_t)(pl * 2 + side) * nseg + seg) * NQ * tsz + t;
#pragma unroll
            for (int k = 0; k < NQ; ++k) P[(size_t)k * tsz] = a[k];
        }
    }
}

// The segments of k_st_cond added in segment order to the band accumulators.  grid: x =
// tile-point blocks, y = plane of the chunk.
template <int KIND>
__global__ void __launch_bounds__(256) k_st_cond_fin(const double* __restrict__ part, int jrel0, int nyg, int nb,
                                                     int tsz, int nseg, double* __restrict__ cbot,
                                                     double* __restrict__ ctop) {
    constexpr int NQ = KIND == 0 ? 6 : (KIND == 1 ? 5 : 2);
    const int pl = blockIdx.y;
    const int jr = jrel0 + pl;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= tsz) return;
    for (int side = 0; side < 2; ++side) {
        const int j1 = side == 0 ? jr : nyg - 1 - jr;
        if (j1 < 0 || j1 >= nb) continue;
        double* C = (side == 0 ? cbot : ctop) + (size_t)j1 * tsz + t;
        const size_t qs = (size_t)nb * tsz;  // stride between quantities
        const double* P = part + (size_t)(pl * 2 + side) * nseg * NQ * tsz + t;
#pragma unroll
        for (int k = 0; k < NQ; ++k) {
            double sum = P[(size_t)k * tsz];
            for (int seg = 1; seg < nseg; ++seg) sum += P[((size_t)seg * NQ + k) * tsz];
            C[k * qs] += sum;
        }
    }
}

// Spectra (spectra.f90:1-56): buildsp / buildspUV on the spectral columns of every plane.
// grid: x = column blocks, y = u plane (index j - ju0; v and p planes are the leading
// nyv, nyp of them).  sp arrays are [plane][column] in FP64.  v_itp is interp_v
// (FOU3D.f90:285-308): vca v(j) + vcb v(j-1) at the interior centres, the ghost centres
// extrapolated with gridweighting_interp.  Each sum is added in the reference's order,
// (sp + re^2) + im^2, with no fused multiply-adds.
__device__ __forceinline__ double sp_add2(double s, double2 a) {
    return __dadd_rn(__dadd_rn(s, __dmul_rn(a.x, a.x)), __dmul_rn(a.y, a.y));
}

__global__ void __launch_bounds__(256) k_spectra(Dims d, Geo g, const double2* __restrict__ u1,
                                                 const double2* __restrict__ u2, const double2* __restrict__ u3,
                                                 const double2* __restrict__ p, double* __restrict__ spu,
                                                 double* __restrict__ spv, double* __restrict__ spw,
                                                 double* __restrict__ spuv, double* __restrict__ spp) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    const int jr = blockIdx.y;
    if (col >= d.ncol) return;
    const size_t nc = d.ncol, o = (size_t)jr * nc + col;
    const double2 a = u1[o];
    spu[o] = sp_add2(spu[o], a);
    spw[o] = sp_add2(spw[o], u3[o]);
    if (jr < d.nyv) spv[o] = sp_add2(spv[o], u2[o]);
    if (jr < d.nyp) spp[o] = sp_add2(spp[o], p[o]);
    // u and v planes share their first index (ju0 = jv0): face r is v index r
    auto itp = [&](int r) {
        const double2 va = u2[(size_t)r * nc + col], vb = u2[(size_t)(r - 1) * nc + col];
        const double wa = g.vca[r], wb = g.vcb[r];
        return make_double2(wa * va.x + wb * vb.x, wa * va.y + wb * vb.y);
    };
    double2 vi;
    if (jr == 0) {
        const double2 v1 = itp(1), vw = u2[col];
        vi = make_double2(g.gwib * (vw.x - v1.x) + v1.x, g.gwib * (vw.y - v1.y) + v1.y);
    } else if (jr == d.nyu - 1) {
        const double2 v1 = itp(jr - 1), vw = u2[(size_t)(d.nyv - 1) * nc + col];
        vi = make_double2(g.gwit * (vw.x - v1.x) + v1.x, g.gwit * (vw.y - v1.y) + v1.y);
    } else {
        vi = itp(jr);
    }
    spuv[o] = __dadd_rn(__dadd_rn(spuv[o], __dmul_rn(a.x, vi.x)), __dmul_rn(a.y, vi.y));
}

}  // namespace cfd
