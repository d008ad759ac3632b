// bands_kernels.cuh - column stages of a three-band channel (start.f90:76-111, 1382-1651).
//
// The wall bands run at Ngal1 x Ngal2 and the middle band coarser.  The modes of the middle
// band ("long" columns) span the channel; the others ("short" columns) exist in the wall
// bands only, as two independent segments whose ends are boundary rows: the band-interface
// rows of LU_buildU/V (gridweighting(1,2) above the bottom segment, gridweighting(3,1) below
// the top one, identity rows for v; tridLU_3D_IB.f90:349-413) and the truncated D.G rows of
// LU_buildP (:417-491).  A short column holds zero outside its segments.  The spectral
// products of a plane that does not carry a column read as zero, as the reference's module
// arrays do (allocated to zero, start.f90:613, and never transposed there).
//
// One thread per column walks its segments in turn; the one-band contexts keep the tuned
// kernels of channel_kernels.cuh and never launch these.
#pragma once

#include "channel_kernels.cuh"

namespace cfd {

// y rows of one column segment (jlim(:,grid,band), start.f90:1538-1557) and the
// gridweighting of its ends (start.f90:494-500)
struct MBSeg {
    int u0, u1, v0, v1, p0, p1;
    double gwb, gwt;
};

__device__ __forceinline__ bool mb_long(const Dims& d, int i, int q) {
    return i <= d.n1m / 2 && (q < d.n2m / 2 || q >= d.n2 - d.n2m / 2);
}
__device__ __forceinline__ MBSeg mb_seg(const Dims& d, const Geo& g, bool lng, int s) {
    const int m = d.ny - 2 - d.jb;  // N(3,2) = N(4,2)
    if (lng) return MBSeg{d.ju0, d.ju1, d.jv0, d.jv1, d.jp0, d.jp1, g.gwb, g.gwt};
    if (s == 0) return MBSeg{d.ju0, d.jb + 2, d.jv0, d.jb + 1, d.ju0 + 1, d.jb + 1, g.gwb, g.gw1t};
    return MBSeg{m, d.ju1, m, d.jv1, m + 1, d.jp1, g.gw3b, g.gwt};
}
// the planes of the middle band (planelim, start.f90:1778-1800)
__device__ __forceinline__ bool mb_umid(const Dims& d, int j) { return j > d.jb + 1 && j <= d.ny - 2 - d.jb; }
__device__ __forceinline__ bool mb_vmid(const Dims& d, int j) { return j > d.jb && j <= d.ny - 2 - d.jb; }

// RHS0 (MODE & 1), the nonlinear tail (MODE & 2) and the solve prologue (MODE & 4) of
// k_rhs, per column segment.  The x/z derivatives zero the kz = -N2/2 mode of the band of
// the plane they come from (der_x/der_z, FOU3D.f90:329-346).
template <typename T2, int MODE>
__global__ void __launch_bounds__(256) k_mb_rhs(Dims d, Geo g, RKCoef c, const double* __restrict__ scal,
                                                const double2* __restrict__ u1, const double2* __restrict__ u2,
                                                const double2* __restrict__ u3, const double2* __restrict__ p,
                                                T2* __restrict__ Nu1, T2* __restrict__ Nu2, T2* __restrict__ Nu3,
                                                double2* __restrict__ du1, double2* __restrict__ du2,
                                                double2* __restrict__ du3, const T2* __restrict__ S0,
                                                const T2* __restrict__ S1, const T2* __restrict__ S2,
                                                const T2* __restrict__ S3) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const double k2 = (-kxv * kxv) + (-kzv * kzv);
    const bool lng = mb_long(d, i, q);
    const bool zrow_w = q == d.n2 / 2, zrow_m = q == d.n2 - d.n2m / 2;
    const size_t nc = d.ncol, vs = (size_t)d.nyu * nc;
    const double mpgx = scal[0];
    constexpr bool RHS0 = (MODE & 1) != 0, NL = (MODE & 2) != 0, PRO = (MODE & 4) != 0;
    for (int s = 0; s < (lng ? 1 : 2); ++s) {
        const MBSeg S = mb_seg(d, g, lng, s);
        for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
            const size_t ju = (size_t)(j - d.ju0);
            const double2 a_m = u1[(ju - 1) * nc + col], a_0 = u1[ju * nc + col], a_p = u1[(ju + 1) * nc + col];
            const double2 w_m = u3[(ju - 1) * nc + col], w_0 = u3[ju * nc + col], w_p = u3[(ju + 1) * nc + col];
            double2 r1, r3;
            if (RHS0) {
                const double c0 = g.dyu2i[3 * ju + 0], c1 = g.dyu2i[3 * ju + 1], c2 = g.dyu2i[3 * ju + 2];
                const double dg = k2 + c1;
                const double2 Lu = dadd(dadd(dscl(c0, a_m), dscl(dg, a_0)), dscl(c2, a_p));
                const double2 Lw = dadd(dadd(dscl(c0, w_m), dscl(dg, w_0)), dscl(c2, w_p));
                const double2 pp = p[(size_t)(j - d.jp0) * nc + col];
                const double2 n1o = to_d2(Nu1[ju * nc + col]), n3o = to_d2(Nu3[ju * nc + col]);
                r1 = dadd(dadd(dscl(c.C1, Lu), dscl(c.C2, n1o)), dik(-c.dRK * kxv, pp));
                r3 = dadd(dadd(dscl(c.C1, Lw), dscl(c.C2, n3o)), dik(-c.dRK * kzv, pp));
                if (col == 0) r1.x += -c.dRK * mpgx;
            } else {
                r1 = du1[ju * nc + col];
                r3 = du3[ju * nc + col];
            }
            if (NL) {
                const size_t su = ju * nc + col;
                const size_t sp = vs + (size_t)(j - d.jv0) * nc + col, sm = sp - nc;  // faces j, j-1
                const bool zr = mb_umid(d, j) ? zrow_m : zrow_w;
                double2 n1 = zr ? dc(0, 0) : dadd(dik(kxv, to_d2(S0[su])), dik(kzv, to_d2(S1[su])));
                double2 n3 = zr ? dc(0, 0) : dadd(dik(kxv, to_d2(S1[su])), dik(kzv, to_d2(S3[su])));
                const double dth = g.dthdyu[ju];
                n1 = dadd(n1, dscl(dth, dsub(to_d2(S0[sp]), to_d2(S0[sm]))));
                n3 = dadd(n3, dscl(dth, dsub(to_d2(S1[sp]), to_d2(S1[sm]))));
                Nu1[su] = to_t2<T2>(n1);
                Nu3[su] = to_t2<T2>(n3);
                r1 = dadd(r1, dscl(c.mg, n1));
                r3 = dadd(r3, dscl(c.mg, n3));
            }
            if (PRO) {
                r1 = dadd(a_0, dscl(c.dt, r1));
                r3 = dadd(w_0, dscl(c.dt, r3));
            }
            du1[ju * nc + col] = r1;
            du3[ju * nc + col] = r3;
        }
        for (int j = S.v0 + 1; j <= S.v1 - 1; ++j) {
            const size_t jv = (size_t)(j - d.jv0);
            const double2 v_m = u2[(jv - 1) * nc + col], v_0 = u2[jv * nc + col], v_p = u2[(jv + 1) * nc + col];
            double2 r2;
            if (RHS0) {
                const double c0 = g.dyv2i[3 * jv + 0], c1 = g.dyv2i[3 * jv + 1], c2 = g.dyv2i[3 * jv + 2];
                const double2 Lv = dadd(dadd(dscl(c0, v_m), dscl(k2 + c1, v_0)), dscl(c2, v_p));
                const double C3 = -c.dRK * g.dthdyv[jv];
                const double2 pa = p[(size_t)(j + 1 - d.jp0) * nc + col], pb = p[(size_t)(j - d.jp0) * nc + col];
                const double2 n2o = to_d2(Nu2[jv * nc + col]);
                r2 = dadd(dadd(dscl(c.C1, Lv), dscl(c.C2, n2o)), dscl(C3, dsub(pa, pb)));
            } else {
                r2 = du2[jv * nc + col];
            }
            if (NL) {
                const size_t sv = vs + jv * nc + col;
                const bool zr = mb_vmid(d, j) ? zrow_m : zrow_w;
                double2 n2 = zr ? dc(0, 0) : dadd(dik(kxv, to_d2(S0[sv])), dik(kzv, to_d2(S1[sv])));
                const double2 vv_p = to_d2(S2[(size_t)(j + 1 - d.ju0) * nc + col]);
                const double2 vv_0 = to_d2(S2[(size_t)(j - d.ju0) * nc + col]);
                n2 = dadd(n2, dscl(g.dthdyv[jv], dsub(vv_p, vv_0)));
                Nu2[jv * nc + col] = to_t2<T2>(n2);
                r2 = dadd(r2, dscl(c.mg, n2));
            }
            if (PRO) r2 = dadd(v_0, dscl(c.dt, r2));
            du2[jv * nc + col] = r2;
        }
        if (PRO) {
            du1[(size_t)(S.u0 - d.ju0) * nc + col] = dc(0, 0);
            du3[(size_t)(S.u0 - d.ju0) * nc + col] = dc(0, 0);
            du1[(size_t)(S.u1 - d.ju0) * nc + col] = dc(0, 0);
            du3[(size_t)(S.u1 - d.ju0) * nc + col] = dc(0, 0);
            du2[(size_t)(S.v0 - d.jv0) * nc + col] = dc(0, 0);
            du2[(size_t)(S.v1 - d.jv0) * nc + col] = dc(0, 0);
        }
    }
}

// LUsolU/LUsolV per band (tridLU_3D_IB.f90:50-160): LU_buildU/V + LU_dec computed on the
// fly over each segment, the scaled upper diagonals in cs_uw / cs_v
__global__ void __launch_bounds__(256) k_mb_solve_uvw(Dims d, Geo g, double beta, double2* __restrict__ u1,
                                                      double2* __restrict__ u2, double2* __restrict__ u3,
                                                      const double2* __restrict__ r1, const double2* __restrict__ r2,
                                                      const double2* __restrict__ r3, double* __restrict__ cs_uw,
                                                      double* __restrict__ cs_v) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double k2x = -g.kx[i] * g.kx[i], k2z = -g.kz[q] * g.kz[q];
    const bool lng = mb_long(d, i, q);
    const size_t nc = d.ncol;
    for (int s = 0; s < (lng ? 1 : 2); ++s) {
        const MBSeg S = mb_seg(d, g, lng, s);
        {   // u and w share the matrix: rows (0,1,gwb), interior, (gwt,1,0)
            const size_t o0 = (size_t)(S.u0 - d.ju0);
            double dprev = 1.0, a3prev = S.gwb;
            double2 y1 = r1[o0 * nc + col], y3 = r3[o0 * nc + col];
            u1[o0 * nc + col] = y1;
            u3[o0 * nc + col] = y3;
            for (int j = S.u0 + 1; j <= S.u1; ++j) {
                const size_t ju = (size_t)(j - d.ju0);
                double a1, a2, a3;
                if (j < S.u1) {
                    a1 = -beta * g.dyu2i[3 * ju + 0];
                    a2 = 1.0 - beta * (g.dyu2i[3 * ju + 1] + k2x + k2z);
                    a3 = -beta * g.dyu2i[3 * ju + 2];
                } else {
                    a1 = S.gwt; a2 = 1.0; a3 = 0.0;
                }
                const double csm = a3prev * dprev;
                cs_uw[(ju - 1) * nc + col] = csm;
                const double dj = 1.0 / (a2 - a1 * csm);
                y1 = dscl(dj, dsub(r1[ju * nc + col], dscl(a1, y1)));
                y3 = dscl(dj, dsub(r3[ju * nc + col], dscl(a1, y3)));
                u1[ju * nc + col] = y1;
                u3[ju * nc + col] = y3;
                dprev = dj;
                a3prev = a3;
            }
            double2 x1 = y1, x3 = y3;
            for (int j = S.u1 - 1; j >= S.u0; --j) {
                const size_t o = (size_t)(j - d.ju0) * nc + col;
                const double cc = cs_uw[o];
                x1 = dsub(u1[o], dscl(cc, x1));
                x3 = dsub(u3[o], dscl(cc, x3));
                u1[o] = x1;
                u3[o] = x3;
            }
        }
        {   // v: identity end rows
            const size_t o0 = (size_t)(S.v0 - d.jv0);
            double dprev = 1.0, a3prev = 0.0;
            double2 y = r2[o0 * nc + col];
            u2[o0 * nc + col] = y;
            for (int j = S.v0 + 1; j <= S.v1; ++j) {
                const size_t jv = (size_t)(j - d.jv0);
                double a1, a2, a3;
                if (j < S.v1) {
                    a1 = -beta * g.dyv2i[3 * jv + 0];
                    a2 = 1.0 - beta * (g.dyv2i[3 * jv + 1] + k2x + k2z);
                    a3 = -beta * g.dyv2i[3 * jv + 2];
                } else {
                    a1 = 0.0; a2 = 1.0; a3 = 0.0;
                }
                const double csm = a3prev * dprev;
                cs_v[(jv - 1) * nc + col] = csm;
                const double dj = 1.0 / (a2 - a1 * csm);
                y = dscl(dj, dsub(r2[jv * nc + col], dscl(a1, y)));
                u2[jv * nc + col] = y;
                dprev = dj;
                a3prev = a3;
            }
            double2 x = y;
            for (int j = S.v1 - 1; j >= S.v0; --j) {
                const size_t o = (size_t)(j - d.jv0) * nc + col;
                x = dsub(u2[o], dscl(cs_v[o], x));
                u2[o] = x;
            }
        }
    }
}

// divergence at the p rows of a segment (littleharsh.f90:209-244)
__device__ __forceinline__ double2 mb_div(const Dims& d, const Geo& g, double kxv, double kzv,
                                          const double2* u1, const double2* u2, const double2* u3, int col, int j) {
    const size_t nc = d.ncol;
    const double2 a = u1[(size_t)(j - d.ju0) * nc + col], w = u3[(size_t)(j - d.ju0) * nc + col];
    const double2 va = u2[(size_t)(j - d.jv0) * nc + col], vb = u2[(size_t)(j - 1 - d.jv0) * nc + col];
    return dadd(dadd(dik(kxv, a), dik(kzv, w)), dscl(g.dthdyu[j - d.ju0], dsub(va, vb)));
}

// v_corr per band (littleharsh.f90:796-907): u, w at the p rows and v at the inner faces of
// each segment; the ghost rows are set from the channel's gridweighting at the bottom of
// bands 1-2 and the top of bands 2-3 only (the interface ghosts of the short segments keep
// the solve's values); v = 0 on every segment end
__device__ __forceinline__ void mb_vcorr_seg(const Dims& d, const Geo& g, const MBSeg& S, double dtrk, double kxv,
                                             double kzv, double2* u1, double2* u2, double2* u3,
                                             const double2* psi, int col) {
    const size_t nc = d.ncol;
    for (int j = S.p0; j <= S.p1; ++j) {
        const size_t ju = (size_t)(j - d.ju0);
        const double2 ps = psi[(size_t)(j - d.jp0) * nc + col];
        u1[ju * nc + col] = dsub(u1[ju * nc + col], dik(dtrk * kxv, ps));
        u3[ju * nc + col] = dsub(u3[ju * nc + col], dik(dtrk * kzv, ps));
    }
    for (int j = S.v0 + 1; j <= S.v1 - 1; ++j) {
        const size_t jv = (size_t)(j - d.jv0);
        const double2 pa = psi[(size_t)(j + 1 - d.jp0) * nc + col], pb = psi[(size_t)(j - d.jp0) * nc + col];
        u2[jv * nc + col] = dsub(u2[jv * nc + col], dscl(dtrk * g.dthdyv[jv], dsub(pa, pb)));
    }
    if (S.u0 == d.ju0) {
        u1[col] = dscl(-g.gwb, u1[nc + col]);
        u3[col] = dscl(-g.gwb, u3[nc + col]);
    }
    if (S.u1 == d.ju1) {
        u1[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u1[(size_t)(d.nyu - 2) * nc + col]);
        u3[(size_t)(d.nyu - 1) * nc + col] = dscl(-g.gwt, u3[(size_t)(d.nyu - 2) * nc + col]);
    }
    u2[(size_t)(S.v0 - d.jv0) * nc + col] = dc(0, 0);
    u2[(size_t)(S.v1 - d.jv0) * nc + col] = dc(0, 0);
}

// solveP per band (littleharsh.f90:556-611): divergence, psi = div*dti/(a+b), LUsolP with
// LU_buildP over the segment's p rows (tridLU_3D_IB.f90:417-491; the mean mode's bottom row
// of the middle band replaced), p += psi; FUSE: v_corr after the segment's back sweep
template <bool FUSE>
__global__ void __launch_bounds__(256) k_mb_solve_p(Dims d, Geo g, double dtirk, double2* __restrict__ u1,
                                                    double2* __restrict__ u2, double2* __restrict__ u3,
                                                    double2* __restrict__ p, double2* __restrict__ psi,
                                                    double2* __restrict__ divo, double* __restrict__ cs,
                                                    double mean_diag, double dtrk) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const double k2x = -kxv * kxv, k2z = -kzv * kzv;
    const bool lng = mb_long(d, i, q);
    const size_t nc = d.ncol;
    auto DTHU = [&](int j) { return g.dthdyu[j - d.ju0]; };
    auto DTHV = [&](int j) { return g.dthdyv[j - d.jv0]; };
    for (int s = 0; s < (lng ? 1 : 2); ++s) {
        const MBSeg S = mb_seg(d, g, lng, s);
        double dprev = 0.0, a3prev = 0.0;
        double2 y = dc(0, 0);
        for (int j = S.p0; j <= S.p1; ++j) {
            const size_t jp = (size_t)(j - d.jp0);
            const double2 dv = mb_div(d, g, kxv, kzv, u1, u2, u3, col, j);
            if (divo) divo[jp * nc + col] = dv;
            double2 r = dscl(dtirk, dv);
            double a1, a2, a3;
            if (j == S.p0) {
                a1 = 0.0;
                a2 = (DTHU(j) * -DTHV(j)) + k2x + k2z;
                a3 = (DTHU(j) * DTHV(j));
                if (col == 0) { a2 = mean_diag; a3 = 0.0; r = dc(0, 0); }
            } else if (j == S.p1) {
                a1 = (-DTHU(j)) * (-DTHV(j - 1));
                a2 = ((-DTHU(j)) * DTHV(j - 1)) + k2x + k2z;
                a3 = 0.0;
            } else {
                a2 = ((-DTHU(j)) * DTHV(j - 1)) + (DTHU(j) * -DTHV(j)) + k2x + k2z;
                a1 = ((-DTHU(j)) * (-DTHV(j - 1)));
                a3 = (DTHU(j) * DTHV(j));
            }
            double dj;
            if (j == S.p0) {
                dj = 1.0 / a2;
                y = dscl(dj, r);
            } else {
                const double csm = a3prev * dprev;
                cs[(jp - 1) * nc + col] = csm;
                dj = 1.0 / (a2 - a1 * csm);
                y = dscl(dj, dsub(r, dscl(a1, y)));
            }
            psi[jp * nc + col] = y;
            dprev = dj;
            a3prev = a3;
        }
        double2 x = y;
        {
            const size_t o = (size_t)(S.p1 - d.jp0) * nc + col;
            p[o] = dadd(p[o], x);
        }
        for (int j = S.p1 - 1; j >= S.p0; --j) {
            const size_t o = (size_t)(j - d.jp0) * nc + col;
            x = dsub(psi[o], dscl(cs[o], x));
            psi[o] = x;
            p[o] = dadd(p[o], x);
        }
        if (FUSE) mb_vcorr_seg(d, g, S, dtrk, kxv, kzv, u1, u2, u3, psi, col);
    }
}

// v_corr alone (the stage entry point), with the closing divergence of every segment
__global__ void __launch_bounds__(256) k_mb_vcorr(Dims d, Geo g, double dtrk, double2* __restrict__ u1,
                                                  double2* __restrict__ u2, double2* __restrict__ u3,
                                                  const double2* __restrict__ psi, double2* __restrict__ divo) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const bool lng = mb_long(d, i, q);
    for (int s = 0; s < (lng ? 1 : 2); ++s) {
        const MBSeg S = mb_seg(d, g, lng, s);
        mb_vcorr_seg(d, g, S, dtrk, kxv, kzv, u1, u2, u3, psi, col);
        if (divo)
            for (int j = S.p0; j <= S.p1; ++j)
                divo[(size_t)(j - d.jp0) * d.ncol + col] = mb_div(d, g, kxv, kzv, u1, u2, u3, col, j);
    }
}

// divergence of every segment (zero on the p rows a short column does not have)
__global__ void __launch_bounds__(256) k_mb_divergence(Dims d, Geo g, const double2* __restrict__ u1,
                                                       const double2* __restrict__ u2, const double2* __restrict__ u3,
                                                       double2* __restrict__ divo) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= d.ncol) return;
    const int i = col % d.nkx, q = col / d.nkx;
    const double kxv = g.kx[i], kzv = g.kz[q];
    const bool lng = mb_long(d, i, q);
    const int m = d.ny - 2 - d.jb;
    for (int j = d.jp0; j <= d.jp1; ++j) {
        const bool in = lng || j <= d.jb + 1 || j >= m + 1;
        divo[(size_t)(j - d.jp0) * d.ncol + col] = in ? mb_div(d, g, kxv, kzv, u1, u2, u3, col, j) : dc(0, 0);
    }
}

}  // namespace cfd
