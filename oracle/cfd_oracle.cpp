// cfd_oracle.cpp - TEST INFRASTRUCTURE, not the product.
//
// FP64 CPU restatement of the LittleHarsh per-substep hot path, used only by tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg as the checker and the timed
// CPU baseline.  Parity is unpinned by the reference itself (the Fortran/MPI reference
// cannot be compiled without a Fortran compiler, and it ships no tests or golden data);
// this restatement is pinned by independent checks instead: numpy.fft for the
// transforms, scipy banded solves for the Thomas sweeps, an independent numpy
// restatement of the substep (tests/golden), and discrete invariants.
//
// One process: the reference's MPI transposes become per-plane gathers/scatters and its
// ranks become OpenMP threads over planes or columns.  Every function cites the reference
// routine it restates.
//
// y-bands (start.f90:76-111, 1382-1651): with one band every (kx,kz) column spans the whole
// channel.  With three (cfd_config.band_vface > 0) the two wall bands keep the x/z
// resolution Ngal1 x Ngal2 and the middle band runs at ngal1_mid x ngal2_mid: the modes of
// the middle band ("long" columns) span the channel, the others ("short" columns) exist in
// the wall bands only, as two independent segments with their own boundary rows at the
// band interfaces (jlim, start.f90:1538-1557; gridweighting(band,:), start.f90:494-508).
// Every plane is transformed at its band's resolution and carries the columns that exist
// there (modes_to_planes_UVP/planes_to_modes_UVP, FOU3D.f90:808-906, 1662-1758).
//
// Data layout mirrors the reference: a spectral field is f[column][j-j0] (Fortran
// f(j,column)), a physical plane is xPL[k][i] with row length Ngal1+2.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/cfd_b200.h"

using cplx = std::complex<double>;
static const double PI = 3.14159265358979323846264338327950288;

// ------------------------------------------------------------------------------------
// Complex FFT: mixed-radix (4, 2, 3) Stockham autosort.  Twiddles are evaluated directly
// (the reference's cffti1 builds them by angle-addition recurrence, cft_buff.f:169-180;
// the difference is far below 1e-10 at these lengths).
// ------------------------------------------------------------------------------------
struct FFTPlan {
    int n = 0;
    std::vector<int> rad;
    std::vector<cplx> w;  // w[m] = exp(-2 pi i m / n)
    void init(int n_) {
        n = n_;
        rad.clear();
        int m = n;
        while (m % 4 == 0) { rad.push_back(4); m /= 4; }
        while (m % 2 == 0) { rad.push_back(2); m /= 2; }
        while (m % 3 == 0) { rad.push_back(3); m /= 3; }
        if (m != 1) throw std::runtime_error("FFT length must be 2^a*3^b");
        w.resize(n);
        for (int k = 0; k < n; ++k) {
            long double a = -2.0L * (long double)PI * (long double)k / (long double)n;
            w[k] = cplx((double)std::cos(a), (double)std::sin(a));
        }
    }
    // sign = -1 forward, +1 inverse; unnormalised; result in `x`; `t` is scratch [n].
    void exec(cplx* x, cplx* t, int sign) const {
        cplx* in = x;
        cplx* out = t;
        int Ns = 1;
        for (int R : rad) {
            const int nr = n / R;
            const int tstep = n / (Ns * R);
            for (int i = 0; i < nr; ++i) {
                const int k = i % Ns;
                cplx v[4];
                for (int r = 0; r < R; ++r) {
                    cplx a = in[i + r * nr];
                    if (Ns > 1 && r > 0) {
                        cplx tw = w[(size_t)(r * k * tstep) % n];
                        if (sign > 0) tw = std::conj(tw);
                        a *= tw;
                    }
                    v[r] = a;
                }
                if (R == 2) {
                    cplx a0 = v[0] + v[1], a1 = v[0] - v[1];
                    v[0] = a0; v[1] = a1;
                } else if (R == 3) {
                    const double s3 = 0.86602540378443864676 * (double)sign;
                    cplx t1 = v[1] + v[2];
                    cplx t2 = v[0] - 0.5 * t1;
                    cplx d = v[1] - v[2];
                    cplx t3(-s3 * d.imag(), s3 * d.real());  // i * s3 * d
                    v[0] = v[0] + t1;
                    v[1] = t2 + t3;
                    v[2] = t2 - t3;
                } else {  // R == 4
                    cplx a0 = v[0] + v[2], a1 = v[0] - v[2];
                    cplx b0 = v[1] + v[3], b1 = v[1] - v[3];
                    cplx ib1((double)(-sign) * b1.imag(), (double)sign * b1.real());  // sign*i*b1
                    v[0] = a0 + b0;
                    v[1] = a1 + ib1;
                    v[2] = a0 - b0;
                    v[3] = a1 - ib1;
                }
                const int idxD = (i / Ns) * Ns * R + k;
                for (int r = 0; r < R; ++r) out[idxD + r * Ns] = v[r];
            }
            std::swap(in, out);
            Ns *= R;
        }
        if (in != x) std::memcpy((void*)x, (const void*)in, sizeof(cplx) * n);
    }
};

// Real transform of even length n via a complex transform of length n/2, with the
// FFTPACK storage of the reference's rft (rft_buff.f:24-86): c[2k], c[2k+1] = Re, Im of
// cc(k), k = 0..n/2.  Forward: cc(k) = (1/n) sum x_j e^{-2 pi i jk/n}, Im cc(0) =
// Im cc(n/2) = 0.  Inverse (unscaled): x_j = sum_k cc(k) e^{2 pi i jk/n} over the
// Hermitian extension, imaginary parts of cc(0), cc(n/2) ignored.
struct RFFTPlan {
    int n = 0, h = 0;
    FFTPlan half;
    std::vector<cplx> wn;  // exp(-2 pi i k / n), k = 0..h
    void init(int n_) {
        n = n_;
        if (n % 2) throw std::runtime_error("real FFT length must be even");
        h = n / 2;
        half.init(h);
        wn.resize(h + 1);
        for (int k = 0; k <= h; ++k) {
            long double a = -2.0L * (long double)PI * k / n;
            wn[k] = cplx((double)std::cos(a), (double)std::sin(a));
        }
    }
    // forward: x (real, n values at c[0..n-1]) -> c[0..n+1] spectral; z, t scratch [h+1]
    void forward(double* c, cplx* z, cplx* t) const {
        for (int m = 0; m < h; ++m) z[m] = cplx(c[2 * m], c[2 * m + 1]);
        half.exec(z, t, -1);
        const double s = 1.0 / n;
        // X_k = E_k + W^k O_k, E_k = (Z_k + conj Z_{h-k})/2, O_k = (Z_k - conj Z_{h-k})/(2i)
        cplx* X = t;  // scratch is free after exec
        for (int k = 0; k <= h; ++k) {
            cplx Zk = z[k % h], Zc = std::conj(z[(h - k) % h]);
            cplx E = 0.5 * (Zk + Zc);
            cplx D = 0.5 * (Zk - Zc);
            cplx O(D.imag(), -D.real());  // D / i
            X[k] = E + wn[k] * O;
        }
        for (int k = 0; k <= h; ++k) {
            c[2 * k] = s * X[k].real();
            c[2 * k + 1] = s * X[k].imag();
        }
        c[1] = 0.0;
        c[n + 1] = 0.0;
    }
    void inverse(double* c, cplx* z, cplx* t) const {
        // Z'_k = (X_k + conj X_{h-k}) + i (X_k - conj X_{h-k}) W^{-k}, k = 0..h-1
        for (int k = 0; k < h; ++k) {
            cplx Xk(c[2 * k], (k == 0) ? 0.0 : c[2 * k + 1]);
            int kk = h - k;
            cplx Xm(c[2 * kk], (kk == h || kk == 0) ? 0.0 : c[2 * kk + 1]);
            cplx Xc = std::conj(Xm);
            cplx S = Xk + Xc;
            cplx D = (Xk - Xc) * std::conj(wn[k]);
            z[k] = S + cplx(-D.imag(), D.real());
        }
        half.exec(z, t, +1);
        for (int m = 0; m < h; ++m) {
            c[2 * m] = z[m].real();
            c[2 * m + 1] = z[m].imag();
        }
    }
};

// ------------------------------------------------------------------------------------
struct IBData {
    int n = 0;
    std::vector<int32_t> idx;
    std::vector<double> w;
    int jlo[2] = {0, 0}, jhi[2] = {-1, -1};
};

// one column segment: the y rows of a column in one band (jlim(:,grid,band)) and the
// gridweighting / gridweighting_interp of its two ends
struct Seg {
    int u0, u1, v0, v1, p0, p1;
    double gwb, gwt, gwib, gwit;
};

// x/z size of a plane's band and its transforms
struct PlaneGeom {
    int ngal1, ngal2, n1, n2, rowlen;
    bool mid;  // the middle band of a three-band run
    const struct RFFTPlan* px;
    const struct FFTPlan* pz;
};

struct Oracle {
    // sizes (the wall bands' with three bands)
    int ngal1, ngal2, n1, n2, nkx, ncol, ny, dny;
    // three bands: middle band size and the last v face of the bottom band (N(3,1));
    // mb = 0 for one band
    int mb = 0, jb = 0, ngal1m = 0, ngal2m = 0, n1m = 0, n2m = 0;
    std::vector<unsigned char> islong;  // column exists in the middle band
    Seg segL{}, segS[2]{};              // long columns; bottom and top segments of short ones
    int ju0, ju1, jv0, jv1, jp0, jp1, nyu, nyv, nyp;
    int rowlen;  // Ngal1 + 2
    // parameters
    double Re, alp, bet, dt, mpgx, QxT, Qx = 0.0, dgx = 0.0;
    int ctpress;
    // grid (array index = j - ju0 for u, j - jv0 for v)
    std::vector<double> yu, yv, dthdyu, dthdyv, dyu2i, dyv2i;
    double gwb, gwt, gwib, gwit;
    std::vector<double> kx, kz;
    IBData ibu, ibv;
    // spectral fields [col*ny + (j - j0)]
    std::vector<cplx> u1, u2, u3, p, psi, div, Nu1, Nu2, Nu3, du1, du2, du3;
    std::vector<cplx> u1i, u2i, u3i, uvf, vvc, vwf;
    RFFTPlan px, pxm;
    FFTPlan pz, pzm;
    int quirk_lastplane = 0;
    // statistics accumulators (stats.f90:1-253, allocated as start.f90:2705-2793):
    // plane sums [q][j - j0]; conditional sums of the bottom (b) and top (t) band
    // [q][j1][k][i] (Fortran YmC(i,k,j1))
    struct {
        bool on = false;
        int jband = 0, dnx = 0, dnz = 0, nbu = 0, nbv = 0, nbp = 0, istat = 0;
        std::vector<double> su, sv, sp, cub, cut, cvb, cvt, cpb, cpt;
        // spectra (spectra.f90:1-56), sp(j,column): [col][j - j0]; empty when not asked for
        std::vector<double> spu, spv, spw, spuv, spp;
    } st;

    // RK coefficients, Le & Moin (start.f90:395-409)
    static constexpr double aRK[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
    static constexpr double bRK[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
    static constexpr double gRK[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
    static constexpr double cRK[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
    static constexpr double dRK[3] = {8.0 / 15.0, 2.0 / 15.0, 1.0 / 3.0};

    double YU(int j) const { return yu[j - ju0]; }
    double YV(int j) const { return yv[j - jv0]; }
    double DTHU(int j) const { return dthdyu[j - ju0]; }
    double DTHV(int j) const { return dthdyv[j - jv0]; }
    double DU2(int c, int j) const { return dyu2i[3 * (j - ju0) + c]; }
    double DV2(int c, int j) const { return dyv2i[3 * (j - jv0) + c]; }

    // field accessors
    cplx& U(std::vector<cplx>& f, int col, int j) { return f[(size_t)col * nyu + (j - ju0)]; }
    cplx& V(std::vector<cplx>& f, int col, int j) { return f[(size_t)col * nyv + (j - jv0)]; }
    cplx& P(std::vector<cplx>& f, int col, int j) { return f[(size_t)col * nyp + (j - jp0)]; }

    int col_i(int col) const { return col % nkx; }
    int col_q(int col) const { return col / nkx; }
    // physical row (0-based) of spectral kz index q (0-based): start.f90:1561-1573
    int row_of(int q) const { return q < n2 / 2 ? q : q + (ngal2 - n2); }
    // segments of a column
    bool is_long(int col) const { return !mb || islong[col]; }
    int nseg(int col) const { return is_long(col) ? 1 : 2; }
    const Seg& seg(int col, int s) const { return is_long(col) ? segL : segS[s]; }
    // band of a u/w plane and of a v plane (planelim, start.f90:1778-1800): 2 = middle
    bool u_mid(int j) const { return mb && j > jb + 1 && j <= ny - 2 - jb; }
    bool v_mid(int j) const { return mb && j > jb && j <= ny - 2 - jb; }
    PlaneGeom geom(bool mid) const {
        return mid ? PlaneGeom{ngal1m, ngal2m, n1m, n2m, ngal1m + 2, true, &pxm, &pzm}
                   : PlaneGeom{ngal1, ngal2, n1, n2, ngal1 + 2, false, &px, &pz};
    }
    // a column is carried by a plane of the middle band only if it is long
    bool on_plane(int col, bool mid) const { return !mid || is_long(col); }
    // physical row of column q in a plane of geometry g (dk shift, start.f90:1625-1637)
    int row_in(const PlaneGeom& g, int q) const { return q < g.n2 / 2 ? q : q + (g.ngal2 - n2); }
    // spectral kz index of the plane's dealiasing row kz = -N2(band)/2 (der_x/der_z zero it)
    int zrow_q(const PlaneGeom& g) const { return n2 - g.n2 / 2; }
};

// ------------------------------------------------------------------------------------
// 2-D plane transforms: four_to_phys_du / phys_to_four_du (FOU3D.f90:574-592, 1619-1639)
// ------------------------------------------------------------------------------------
struct PlaneWork {
    std::vector<cplx> z, t, zl;
    void init(const Oracle& o) {
        int m = std::max(o.ngal1, o.ngal2) + 2;
        z.resize(m);
        t.resize(m);
        zl.resize(o.ngal2);
    }
};

static void cft_plane(const PlaneGeom& g, double* pl, int iopt, PlaneWork& w) {
    // cft(pl, ise=Ngal1+2, isa=2, m=(N1+2)/2, iopt): z-transform of kx-modes 0..N1/2
    const int L = g.rowlen;
    for (int i = 0; i <= g.n1 / 2; ++i) {
        for (int k = 0; k < g.ngal2; ++k) w.zl[k] = cplx(pl[k * L + 2 * i], pl[k * L + 2 * i + 1]);
        g.pz->exec(w.zl.data(), w.t.data(), iopt < 0 ? -1 : +1);
        const double s = iopt < 0 ? 1.0 / g.ngal2 : 1.0;
        for (int k = 0; k < g.ngal2; ++k) {
            pl[k * L + 2 * i] = s * w.zl[k].real();
            pl[k * L + 2 * i + 1] = s * w.zl[k].imag();
        }
    }
}

static void rft_plane(const PlaneGeom& g, double* pl, int iopt, PlaneWork& w) {
    const int L = g.rowlen;
    for (int k = 0; k < g.ngal2; ++k) {
        if (iopt < 0) g.px->forward(pl + (size_t)k * L, w.z.data(), w.t.data());
        else g.px->inverse(pl + (size_t)k * L, w.z.data(), w.t.data());
    }
}

static void four_to_phys(const PlaneGeom& g, double* pl, bool zero_oddball, PlaneWork& w) {
    if (zero_oddball)
        for (int i = 0; i < g.rowlen; ++i) pl[(g.ngal2 / 2) * g.rowlen + i] = 0.0;
    cft_plane(g, pl, +1, w);
    rft_plane(g, pl, +1, w);
}

static void phys_to_four(const PlaneGeom& g, double* pl, PlaneWork& w) {
    rft_plane(g, pl, -1, w);
    cft_plane(g, pl, -1, w);
}
static void four_to_phys(const Oracle& o, double* pl, bool zero_oddball, PlaneWork& w) {
    four_to_phys(o.geom(false), pl, zero_oddball, w);
}
static void phys_to_four(const Oracle& o, double* pl, PlaneWork& w) { phys_to_four(o.geom(false), pl, w); }

// modes_to_planes for one plane (FOU3D.f90:842-848): zero, then scatter the spectral
// columns the plane's band carries
static void gather_plane(Oracle& o, const PlaneGeom& g, std::vector<cplx>& f, int nyf, int j0, int j, double* pl) {
    std::memset(pl, 0, sizeof(double) * (size_t)g.rowlen * g.ngal2);
    for (int col = 0; col < o.ncol; ++col) {
        if (!o.on_plane(col, g.mid)) continue;
        int i = o.col_i(col), row = o.row_in(g, o.col_q(col));
        cplx v = f[(size_t)col * nyf + (j - j0)];
        pl[(size_t)row * g.rowlen + 2 * i] = v.real();
        pl[(size_t)row * g.rowlen + 2 * i + 1] = v.imag();
    }
}
static void gather_plane(Oracle& o, std::vector<cplx>& f, int nyf, int j0, int j, double* pl) {
    gather_plane(o, o.geom(false), f, nyf, j0, j, pl);
}

// ------------------------------------------------------------------------------------
// RHS0_u1/u2/u3 with laplacian_U/V (littleharsh.f90:246-320, 613-730)
// ------------------------------------------------------------------------------------
static void rhs0(Oracle& o, int krk) {
    const int r = krk - 1;
    const double C1 = Oracle::aRK[r] / o.Re;
    const double C2 = -Oracle::cRK[r];
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        const int i = o.col_i(col), q = o.col_q(col);
        const double k2x = -o.kx[i] * o.kx[i], k2z = -o.kz[q] * o.kz[q];
        const cplx C3x = -Oracle::dRK[r] * cplx(0.0, o.kx[i]);
        const cplx C3z = -Oracle::dRK[r] * cplx(0.0, o.kz[q]);
        for (int sg = 0; sg < o.nseg(col); ++sg) {
        const Seg& S = o.seg(col, sg);
        for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
            cplx Lu = o.DU2(0, j) * o.U(o.u1, col, j - 1) + (k2x + k2z + o.DU2(1, j)) * o.U(o.u1, col, j) +
                      o.DU2(2, j) * o.U(o.u1, col, j + 1);
            o.U(o.du1, col, j) = C1 * Lu + C2 * o.U(o.Nu1, col, j) + C3x * o.P(o.p, col, j);
            cplx Lw = o.DU2(0, j) * o.U(o.u3, col, j - 1) + (k2x + k2z + o.DU2(1, j)) * o.U(o.u3, col, j) +
                      o.DU2(2, j) * o.U(o.u3, col, j + 1);
            o.U(o.du3, col, j) = C1 * Lw + C2 * o.U(o.Nu3, col, j) + C3z * o.P(o.p, col, j);
        }
        for (int j = S.v0 + 1; j <= S.v1 - 1; ++j) {
            const double C3 = -Oracle::dRK[r] * o.DTHV(j);
            cplx Lv = o.DV2(0, j) * o.V(o.u2, col, j - 1) + (k2x + k2z + o.DV2(1, j)) * o.V(o.u2, col, j) +
                      o.DV2(2, j) * o.V(o.u2, col, j + 1);
            o.V(o.du2, col, j) = C1 * Lv + C2 * o.V(o.Nu2, col, j) + C3 * (o.P(o.p, col, j + 1) - o.P(o.p, col, j));
        }
        }
    }
    // mean pressure gradient on mode (0,0), j = N(4,0)+1..N(4,nband) (littleharsh.f90:650-656)
    const double C1m = -Oracle::dRK[r] * o.mpgx;
    for (int j = o.ju0 + 1; j <= o.ju1 - 1; ++j) o.U(o.du1, 0, j) += C1m;
}

// ------------------------------------------------------------------------------------
// nonlinear (FOU3D.f90:41-259) with interp_u/v (:261-308), ops_in_planes (:1529-1617),
// der_x/der_z (:310-414), der_yu_h/der_yv_h (:453-493).  The x/z advective derivatives
// are taken per plane (the reference keeps them in 2-D scratch so every plane of a rank
// receives its last plane's value, FOU3D.f90:1541,1571-1585; with quirk_lastplane set the
// oracle reproduces that for a single slab).
// ------------------------------------------------------------------------------------
static void interp(Oracle& o) {
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        for (int sg = 0; sg < o.nseg(col); ++sg) {
        const Seg& S = o.seg(col, sg);
        for (int j = S.v0; j <= S.v1; ++j) {
            const double den = o.YU(j + 1) - o.YU(j);
            o.V(o.u1i, col, j) = ((o.YV(j) - o.YU(j)) * o.U(o.u1, col, j + 1) + (o.YU(j + 1) - o.YV(j)) * o.U(o.u1, col, j)) / den;
            o.V(o.u3i, col, j) = ((o.YV(j) - o.YU(j)) * o.U(o.u3, col, j + 1) + (o.YU(j + 1) - o.YV(j)) * o.U(o.u3, col, j)) / den;
        }
        for (int j = S.u0 + 1; j <= S.u1 - 1; ++j)
            o.U(o.u2i, col, j) = ((o.YU(j) - o.YV(j - 1)) * o.V(o.u2, col, j) + (o.YV(j) - o.YU(j)) * o.V(o.u2, col, j - 1)) /
                                 (o.YV(j) - o.YV(j - 1));
        o.U(o.u2i, col, S.u0) = S.gwib * (o.V(o.u2, col, S.v0) - o.U(o.u2i, col, S.u0 + 1)) + o.U(o.u2i, col, S.u0 + 1);
        o.U(o.u2i, col, S.u1) = S.gwit * (o.V(o.u2, col, S.v1) - o.U(o.u2i, col, S.u1 - 1)) + o.U(o.u2i, col, S.u1 - 1);
        }
    }
}

// derivative value of one spectral entry with the dealiasing zero of der_x/der_z: the
// kz = -N2/2 mode of the plane's band (physical row Ngal2-N2/2) is zeroed (FOU3D.f90:334-338)
static inline cplx dxdz(const Oracle& o, int i, int q, int qzero, cplx a, cplx b) {
    if (q == qzero) return cplx(0.0, 0.0);
    return cplx(0.0, o.kx[i]) * a + cplx(0.0, o.kz[q]) * b;
}

static void ops_in_planes(Oracle& o) {
    const size_t psz = (size_t)o.rowlen * o.ngal2;  // the largest plane
    // u planes (ugrid, incl. ghosts): uu, uw, vv, ww
#pragma omp parallel
    {
        PlaneWork w;
        w.init(o);
        std::vector<double> a(psz), b(psz), c(psz), uu(psz), uw(psz), vv(psz), ww(psz);
#pragma omp for schedule(dynamic)
        for (int j = o.ju0; j <= o.ju1; ++j) {
            const PlaneGeom g = o.geom(o.u_mid(j));
            const size_t gsz = (size_t)g.rowlen * g.ngal2;
            gather_plane(o, g, o.u1, o.nyu, o.ju0, j, a.data());
            gather_plane(o, g, o.u2i, o.nyu, o.ju0, j, b.data());
            gather_plane(o, g, o.u3, o.nyu, o.ju0, j, c.data());
            four_to_phys(g, a.data(), true, w);
            four_to_phys(g, b.data(), true, w);
            four_to_phys(g, c.data(), true, w);
            std::fill(uu.begin(), uu.begin() + gsz, 0.0);
            std::fill(uw.begin(), uw.begin() + gsz, 0.0);
            std::fill(vv.begin(), vv.begin() + gsz, 0.0);
            std::fill(ww.begin(), ww.begin() + gsz, 0.0);
            for (int k = 0; k < g.ngal2; ++k)
                for (int i = 0; i < g.ngal1; ++i) {
                    size_t e = (size_t)k * g.rowlen + i;
                    uu[e] = a[e] * a[e];
                    uw[e] = a[e] * c[e];
                    vv[e] = b[e] * b[e];
                    ww[e] = c[e] * c[e];
                }
            phys_to_four(g, uu.data(), w);
            phys_to_four(g, uw.data(), w);
            phys_to_four(g, vv.data(), w);
            phys_to_four(g, ww.data(), w);
            const bool interior = (j > o.ju0 && j < o.ju1);
            const int qz = o.zrow_q(g);
            for (int col = 0; col < o.ncol; ++col) {
                if (!o.on_plane(col, g.mid)) continue;
                const int i = o.col_i(col), q = o.col_q(col);
                const size_t e = (size_t)o.row_in(g, q) * g.rowlen + 2 * i;
                cplx UU(uu[e], uu[e + 1]), UW(uw[e], uw[e + 1]), VV(vv[e], vv[e + 1]), WW(ww[e], ww[e + 1]);
                o.U(o.vvc, col, j) = VV;
                if (interior || o.quirk_lastplane) {
                    o.U(o.Nu1, col, j) = dxdz(o, i, q, qz, UU, UW);
                    o.U(o.Nu3, col, j) = dxdz(o, i, q, qz, UW, WW);
                }
            }
        }
        // v planes (vgrid, incl. walls): uv, vw
#pragma omp for schedule(dynamic)
        for (int j = o.jv0; j <= o.jv1; ++j) {
            const PlaneGeom g = o.geom(o.v_mid(j));
            const size_t gsz = (size_t)g.rowlen * g.ngal2;
            gather_plane(o, g, o.u1i, o.nyv, o.jv0, j, a.data());
            gather_plane(o, g, o.u2, o.nyv, o.jv0, j, b.data());
            gather_plane(o, g, o.u3i, o.nyv, o.jv0, j, c.data());
            four_to_phys(g, a.data(), true, w);
            four_to_phys(g, b.data(), true, w);
            four_to_phys(g, c.data(), true, w);
            std::fill(uu.begin(), uu.begin() + gsz, 0.0);
            std::fill(uw.begin(), uw.begin() + gsz, 0.0);
            for (int k = 0; k < g.ngal2; ++k)
                for (int i = 0; i < g.ngal1; ++i) {
                    size_t e = (size_t)k * g.rowlen + i;
                    uu[e] = a[e] * b[e];  // uv
                    uw[e] = c[e] * b[e];  // vw
                }
            phys_to_four(g, uu.data(), w);
            phys_to_four(g, uw.data(), w);
            const bool interior = (j > o.jv0 && j < o.jv1);
            const int qz = o.zrow_q(g);
            for (int col = 0; col < o.ncol; ++col) {
                if (!o.on_plane(col, g.mid)) continue;
                const int i = o.col_i(col), q = o.col_q(col);
                const size_t e = (size_t)o.row_in(g, q) * g.rowlen + 2 * i;
                cplx UV(uu[e], uu[e + 1]), VW(uw[e], uw[e + 1]);
                o.V(o.uvf, col, j) = UV;
                o.V(o.vwf, col, j) = VW;
                if (interior || o.quirk_lastplane) o.V(o.Nu2, col, j) = dxdz(o, i, q, qz, UV, VW);
            }
        }
    }
    if (o.quirk_lastplane) {
        // one slab holding every plane: the 2-D scratch keeps the last plane of the
        // loop over limPL_incw, i.e. the top ghost (u/w) and the top wall (v), and every
        // interior plane receives it (FOU3D.f90:1553-1585, 1588-1613)
        for (int col = 0; col < o.ncol; ++col) {
            cplx a1 = o.U(o.Nu1, col, o.ju1), a3 = o.U(o.Nu3, col, o.ju1), a2 = o.V(o.Nu2, col, o.jv1);
            for (int j = o.ju0 + 1; j <= o.ju1 - 1; ++j) { o.U(o.Nu1, col, j) = a1; o.U(o.Nu3, col, j) = a3; }
            for (int j = o.jv0 + 1; j <= o.jv1 - 1; ++j) o.V(o.Nu2, col, j) = a2;
            o.U(o.Nu1, col, o.ju0) = o.U(o.Nu1, col, o.ju1) = 0.0;
            o.U(o.Nu3, col, o.ju0) = o.U(o.Nu3, col, o.ju1) = 0.0;
            o.V(o.Nu2, col, o.jv0) = o.V(o.Nu2, col, o.jv1) = 0.0;
        }
    }
}

static void nonlinear(Oracle& o, int krk) {
    interp(o);
    ops_in_planes(o);
    const double C1 = -Oracle::gRK[krk - 1];
    // der_yu_h / der_yv_h over each column segment (FOU3D.f90:158-173); a short column reads
    // the products of the interface plane it is not carried on as the zero they were
    // allocated with (start.f90:613), as the reference does
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        for (int sg = 0; sg < o.nseg(col); ++sg) {
            const Seg& S = o.seg(col, sg);
            for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
                o.U(o.Nu1, col, j) = o.U(o.Nu1, col, j) + (o.V(o.uvf, col, j) - o.V(o.uvf, col, j - 1)) * o.DTHU(j);
                o.U(o.Nu3, col, j) = o.U(o.Nu3, col, j) + (o.V(o.vwf, col, j) - o.V(o.vwf, col, j - 1)) * o.DTHU(j);
            }
            for (int j = S.v0 + 1; j <= S.v1 - 1; ++j)
                o.V(o.Nu2, col, j) = o.V(o.Nu2, col, j) + (o.U(o.vvc, col, j + 1) - o.U(o.vvc, col, j)) * o.DTHV(j);
            for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
                o.U(o.du1, col, j) = o.U(o.du1, col, j) + C1 * o.U(o.Nu1, col, j);
                o.U(o.du3, col, j) = o.U(o.du3, col, j) + C1 * o.U(o.Nu3, col, j);
            }
            for (int j = S.v0 + 1; j <= S.v1 - 1; ++j)
                o.V(o.du2, col, j) = o.V(o.du2, col, j) + C1 * o.V(o.Nu2, col, j);
        }
    }
}

// ------------------------------------------------------------------------------------
// immersed_boundaries_U/V (tridLU_3D_IB.f90:163-281)
// ------------------------------------------------------------------------------------
static void immersed_boundaries(Oracle& o, std::vector<cplx>& u, std::vector<cplx>& rhs, int nyf, int j0,
                                int j1, const IBData& ib) {
    // planes that go through the round trip: interior planes of the two ranges
    std::vector<int> planes;
    for (int s = 0; s < 2; ++s)
        for (int j = std::max(ib.jlo[s], j0 + 1); j <= std::min(ib.jhi[s], j1 - 1); ++j) planes.push_back(j);
    if (planes.empty()) return;
    const size_t psz = (size_t)o.rowlen * o.ngal2;
    const int np = (int)planes.size();
    std::vector<int> slot(j1 - j0 + 1, -1);
    for (int s = 0; s < np; ++s) slot[planes[s] - j0] = s;
    std::vector<double> rpl(psz * np), upl(psz * np);
#pragma omp parallel
    {
        PlaneWork w;
        w.init(o);
#pragma omp for schedule(dynamic)
        for (int s = 0; s < np; ++s) {
            gather_plane(o, rhs, nyf, j0, planes[s], rpl.data() + psz * s);
            gather_plane(o, u, nyf, j0, planes[s], upl.data() + psz * s);
            four_to_phys(o, rpl.data() + psz * s, false, w);
            four_to_phys(o, upl.data() + psz * s, false, w);
        }
    }
    // forcing loop in list order (:193-211)
    for (int p = 0; p < ib.n; ++p) {
        const int32_t* id = &ib.idx[9 * p];
        const double* wt = &ib.w[3 * p];
        auto at = [&](std::vector<double>& pl, int i, int k, int j) -> double& {
            int s = slot[j - j0];
            return pl[psz * s + (size_t)(k - 1) * o.rowlen + (i - 1)];
        };
        const double vf = wt[1] * at(upl, id[3], id[4], id[5]) + wt[2] * at(upl, id[6], id[7], id[8]);
        double& r = at(rpl, id[0], id[1], id[2]);
        r = wt[0] * (vf - at(upl, id[0], id[1], id[2]) + r);
    }
#pragma omp parallel
    {
        PlaneWork w;
        w.init(o);
#pragma omp for schedule(dynamic)
        for (int s = 0; s < np; ++s) {
            double* pl = rpl.data() + psz * s;
            phys_to_four(o, pl, w);
            const int j = planes[s];
            for (int col = 0; col < o.ncol; ++col) {
                const size_t e = (size_t)o.row_of(o.col_q(col)) * o.rowlen + 2 * o.col_i(col);
                rhs[(size_t)col * nyf + (j - j0)] = cplx(pl[e], pl[e + 1]);
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// Thomas solves: LU_buildU/LU_buildV + LU_dec + substitution (tridLU_3D_IB.f90:50-160,
// 349-413, 521-559)
// ------------------------------------------------------------------------------------
static void thomas(int n, double* a1, double* a2, double* a3, const cplx* rhs, cplx* x) {
    // LU_dec
    a2[0] = 1.0 / a2[0];
    for (int j = 1; j < n; ++j) {
        a3[j - 1] = a3[j - 1] * a2[j - 1];
        a2[j] = 1.0 / (a2[j] - a1[j] * a3[j - 1]);
    }
    x[0] = rhs[0] * a2[0];
    for (int j = 1; j < n; ++j) x[j] = (rhs[j] - a1[j] * x[j - 1]) * a2[j];
    for (int j = n - 2; j >= 0; --j) x[j] = x[j] - a3[j] * x[j + 1];
}

static void solve_u(Oracle& o, std::vector<cplx>& u, std::vector<cplx>& du, int krk) {
    // solveU prologue (littleharsh.f90:744-755), per column segment
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        for (int sg = 0; sg < o.nseg(col); ++sg) {
            const Seg& S = o.seg(col, sg);
            o.U(du, col, S.u0) = 0.0;
            for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) o.U(du, col, j) = o.U(u, col, j) + o.dt * o.U(du, col, j);
            o.U(du, col, S.u1) = 0.0;
        }
    }
    immersed_boundaries(o, u, du, o.nyu, o.ju0, o.ju1, o.ibu);
    const double beta = Oracle::bRK[krk - 1] * o.dt / o.Re;
    // LUsolU per band: LU_buildU over jlim with the band's gridweighting rows (tridLU_3D_IB.f90:
    // 50-103, 349-380)
#pragma omp parallel
    {
        std::vector<double> a1(o.nyu), a2(o.nyu), a3(o.nyu);
#pragma omp for schedule(static)
        for (int col = 0; col < o.ncol; ++col) {
            const int i = o.col_i(col), q = o.col_q(col);
            const double k2x = -o.kx[i] * o.kx[i], k2z = -o.kz[q] * o.kz[q];
            for (int sg = 0; sg < o.nseg(col); ++sg) {
                const Seg& S = o.seg(col, sg);
                const int n = S.u1 - S.u0 + 1;
                a1[0] = 0.0; a2[0] = 1.0; a3[0] = S.gwb;
                for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
                    int jj = j - S.u0;
                    a1[jj] = -beta * o.DU2(0, j);
                    a2[jj] = 1.0 - beta * (o.DU2(1, j) + k2x + k2z);
                    a3[jj] = -beta * o.DU2(2, j);
                }
                a1[n - 1] = S.gwt; a2[n - 1] = 1.0; a3[n - 1] = 0.0;
                const size_t off = (size_t)col * o.nyu + (S.u0 - o.ju0);
                thomas(n, a1.data(), a2.data(), a3.data(), &du[off], &u[off]);
            }
        }
    }
}

static void solve_v(Oracle& o, int krk) {
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        for (int sg = 0; sg < o.nseg(col); ++sg) {
            const Seg& S = o.seg(col, sg);
            o.V(o.du2, col, S.v0) = 0.0;
            for (int j = S.v0 + 1; j <= S.v1 - 1; ++j) o.V(o.du2, col, j) = o.V(o.u2, col, j) + o.dt * o.V(o.du2, col, j);
            o.V(o.du2, col, S.v1) = 0.0;
        }
    }
    immersed_boundaries(o, o.u2, o.du2, o.nyv, o.jv0, o.jv1, o.ibv);
    const double beta = Oracle::bRK[krk - 1] * o.dt / o.Re;
#pragma omp parallel
    {
        std::vector<double> a1(o.nyv), a2(o.nyv), a3(o.nyv);
#pragma omp for schedule(static)
        for (int col = 0; col < o.ncol; ++col) {
            const int i = o.col_i(col), q = o.col_q(col);
            const double k2x = -o.kx[i] * o.kx[i], k2z = -o.kz[q] * o.kz[q];
            for (int sg = 0; sg < o.nseg(col); ++sg) {
                const Seg& S = o.seg(col, sg);
                const int n = S.v1 - S.v0 + 1;
                a1[0] = 0.0; a2[0] = 1.0; a3[0] = 0.0;
                for (int j = S.v0 + 1; j <= S.v1 - 1; ++j) {
                    int jj = j - S.v0;
                    a1[jj] = -beta * o.DV2(0, j);
                    a2[jj] = 1.0 - beta * (o.DV2(1, j) + k2x + k2z);
                    a3[jj] = -beta * o.DV2(2, j);
                }
                a1[n - 1] = 0.0; a2[n - 1] = 1.0; a3[n - 1] = 0.0;
                const size_t off = (size_t)col * o.nyv + (S.v0 - o.jv0);
                thomas(n, a1.data(), a2.data(), a3.data(), &o.du2[off], &o.u2[off]);
            }
        }
    }
}

// ------------------------------------------------------------------------------------
// mean flow: flowrateIm/flowrateRe/flowrate_corr/LUsol0/LU_build0 (littleharsh.f90:411-537,
// tridLU_3D_IB.f90:320-346, 493-519, 605-622).  The u11 column spans j = 0..nn+2
// (nn = ny-2), the cells between the crests plus one on each side, as in the reference.
// ------------------------------------------------------------------------------------
static double flowrate(const Oracle& o, const std::vector<cplx>& u1) {
    const int nn = o.ny - 2;
    double Qu = 0.0;
    for (int j = 1; j <= nn + 1; ++j) Qu += (o.YV(j) - o.YV(j - 1)) * u1[(size_t)(j - o.ju0)].real();
    return Qu;
}

static void meanflow(Oracle& o, int krk) {
    const int nn = o.ny - 2;
    if (o.ctpress == 1) {
        o.Qx = flowrate(o, o.u1);
        return;
    }
    const int n = nn + 3;
    std::vector<double> a1(n), a2(n), a3(n);
    std::vector<cplx> u11(n), x(n);
    const double beta = Oracle::bRK[krk - 1] * o.dt / o.Re;
    a1[0] = 0.0; a2[0] = 1.0; a3[0] = o.gwb;
    for (int j = 1; j <= nn + 1; ++j) {
        a1[j] = -beta * o.DU2(0, j);
        a2[j] = 1.0 - beta * o.DU2(1, j);
        a3[j] = -beta * o.DU2(2, j);
    }
    a1[nn + 2] = o.gwt; a2[nn + 2] = 1.0; a3[nn + 2] = 0.0;
    const double bdt = -Oracle::dRK[krk - 1] * o.dt;
    u11[0] = 0.0;
    for (int j = 1; j <= nn + 1; ++j) u11[j] = bdt;
    u11[nn + 2] = 0.0;
    thomas(n, a1.data(), a2.data(), a3.data(), u11.data(), x.data());
    double Qx1 = 0.0;
    for (int j = 1; j <= nn + 1; ++j) Qx1 += (o.YV(j) - o.YV(j - 1)) * x[j].real();
    const double Qx0 = flowrate(o, o.u1);
    const double g = (o.QxT - Qx0) / Qx1;
    o.mpgx += g;
    o.dgx = g;
    for (int j = 0; j <= nn + 2; ++j) o.U(o.u1, 0, j) = o.U(o.u1, 0, j) + g * x[j];
}

// ------------------------------------------------------------------------------------
// divergence, solveP, LUsolP, LU_buildP/LU_decP, v_corr (littleharsh.f90:209-244, 556-611,
// 796-907; tridLU_3D_IB.f90:284-318, 417-491, 562-603)
// ------------------------------------------------------------------------------------
static void divergence(Oracle& o) {
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        const cplx kx(0.0, o.kx[o.col_i(col)]), kz(0.0, o.kz[o.col_q(col)]);
        for (int sg = 0; sg < o.nseg(col); ++sg) {
            const Seg& S = o.seg(col, sg);
            for (int j = S.p0; j <= S.p1; ++j)
                o.P(o.div, col, j) = kx * o.U(o.u1, col, j) + kz * o.U(o.u3, col, j) +
                                     o.DTHU(j) * (o.V(o.u2, col, j) - o.V(o.u2, col, j - 1));
        }
    }
}

static void solve_p(Oracle& o, int krk) {
    const double dtirk = (1.0 / o.dt) / (Oracle::aRK[krk - 1] + Oracle::bRK[krk - 1]);
    divergence(o);
    // per band (solveP, littleharsh.f90:569-609): LU_buildP over jlim(:,pgrid,band), the mean
    // mode's bottom row replaced in the middle band only (tridLU_3D_IB.f90:468-474)
#pragma omp parallel
    {
        std::vector<double> a1(o.nyp), a2(o.nyp), a3(o.nyp);
        std::vector<cplx> x(o.nyp), r(o.nyp);
#pragma omp for schedule(static)
        for (int col = 0; col < o.ncol; ++col) {
            const int i = o.col_i(col), q = o.col_q(col);
            const double k2x = -o.kx[i] * o.kx[i], k2z = -o.kz[q] * o.kz[q];
            // D_vec/G_vec (tridLU_3D_IB.f90:434-439)
            auto Db = [&](int m) { return -o.DTHU(m + 1); };
            auto Gb = [&](int m) { return -o.DTHV(m); };
            auto Dt = [&](int m) { return o.DTHU(m); };
            auto Gt = [&](int m) { return o.DTHV(m - 1); };
            for (int sg = 0; sg < o.nseg(col); ++sg) {
                const Seg& S = o.seg(col, sg);
                const int n = S.p1 - S.p0 + 1;
                for (int j = S.p0; j <= S.p1; ++j) r[j - S.p0] = dtirk * o.P(o.div, col, j);
                if (col == 0) r[0] = 0.0;
                a2[0] = (Dt(S.p0) * Gb(S.p0)) + k2x + k2z;
                a3[0] = (Dt(S.p0) * Gt(S.p0 + 1));
                a1[0] = 0.0;
                a2[n - 1] = (Db(S.p1 - 1) * Gt(S.p1)) + k2x + k2z;
                a1[n - 1] = (Db(S.p1 - 1) * Gb(S.p1 - 1));
                a3[n - 1] = 0.0;
                for (int j = S.p0 + 1; j <= S.p1 - 1; ++j) {
                    int jj = j - S.p0;
                    a2[jj] = (Db(j - 1) * Gt(j)) + (Dt(j) * Gb(j)) + k2x + k2z;
                    a1[jj] = (Db(j - 1) * Gb(j - 1));
                    a3[jj] = (Dt(j) * Gt(j + 1));
                }
                if (col == 0) {
                    a1[0] = 0.0;
                    a2[0] = 1.0 / ((o.YU(2) - o.YU(1)) * (o.YU(2) - o.YU(1)));
                    a3[0] = 0.0;
                }
                thomas(n, a1.data(), a2.data(), a3.data(), r.data(), x.data());
                for (int j = S.p0; j <= S.p1; ++j) {
                    o.P(o.psi, col, j) = x[j - S.p0];
                    o.P(o.p, col, j) = o.P(o.p, col, j) + x[j - S.p0];
                }
            }
        }
    }
}

static void v_corr(Oracle& o, int krk) {
    const double dtrk = o.dt * (Oracle::aRK[krk - 1] + Oracle::bRK[krk - 1]);
    // per band (littleharsh.f90:816-899): the ghost rows are set from the channel's own
    // gridweighting at the bottom of bands 1-2 and the top of bands 2-3 only; the ghost
    // rows of the short segments at the band interfaces keep what the solve left there
#pragma omp parallel for schedule(static)
    for (int col = 0; col < o.ncol; ++col) {
        const cplx kx = dtrk * cplx(0.0, o.kx[o.col_i(col)]);
        const cplx kz = dtrk * cplx(0.0, o.kz[o.col_q(col)]);
        for (int sg = 0; sg < o.nseg(col); ++sg) {
            const Seg& S = o.seg(col, sg);
            for (int j = S.u0 + 1; j <= S.u1 - 1; ++j) {
                o.U(o.u1, col, j) = o.U(o.u1, col, j) - kx * o.P(o.psi, col, j);
                o.U(o.u3, col, j) = o.U(o.u3, col, j) - kz * o.P(o.psi, col, j);
            }
            if (S.u0 == o.ju0) {
                o.U(o.u1, col, o.ju0) = -o.gwb * o.U(o.u1, col, o.ju0 + 1);
                o.U(o.u3, col, o.ju0) = -o.gwb * o.U(o.u3, col, o.ju0 + 1);
            }
            if (S.u1 == o.ju1) {
                o.U(o.u1, col, o.ju1) = -o.gwt * o.U(o.u1, col, o.ju1 - 1);
                o.U(o.u3, col, o.ju1) = -o.gwt * o.U(o.u3, col, o.ju1 - 1);
            }
            for (int j = S.v0 + 1; j <= S.v1 - 1; ++j)
                o.V(o.u2, col, j) = o.V(o.u2, col, j) - dtrk * o.DTHV(j) * (o.P(o.psi, col, j + 1) - o.P(o.psi, col, j));
            o.V(o.u2, col, S.v0) = 0.0;
            o.V(o.u2, col, S.v1) = 0.0;
        }
    }
    divergence(o);
}

static void rk_substep(Oracle& o, int krk) {
    rhs0(o, krk);
    nonlinear(o, krk);
    solve_u(o, o.u1, o.du1, krk);
    solve_v(o, krk);
    solve_u(o, o.u3, o.du3, krk);
    if (o.ctpress == 0) meanflow(o, krk);
    solve_p(o, krk);
    v_corr(o, krk);
}

// ------------------------------------------------------------------------------------
// extern "C" API (ctypes)
// ------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------
// stats (stats.f90:1-106) with conddown1/2, condup1/2 (:110-253) and the omega_x planes of
// nonlinear (FOU3D.f90:187-207); dtc_calc (FOU3D.f90:516-544).  Physical planes come from
// the same plane transforms as ops_in_planes: u, w, v_itp on u planes, v, w_itp, wx on v
// planes (four_to_phys_u for velocities, four_to_phys_du for wx and p).
// ------------------------------------------------------------------------------------
static void stats_configure(Oracle& o, int jband, int dnx, int dnz, int spectra) {
    auto& st = o.st;
    const size_t nc = o.ncol;
    st.spu.assign(spectra ? nc * o.nyu : 0, 0.0);
    st.spv.assign(spectra ? nc * o.nyv : 0, 0.0);
    st.spw.assign(spectra ? nc * o.nyu : 0, 0.0);
    st.spuv.assign(spectra ? nc * o.nyu : 0, 0.0);
    st.spp.assign(spectra ? nc * o.nyp : 0, 0.0);
    const bool cond = jband >= o.jv0;
    st.jband = jband;
    st.dnx = cond ? dnx : 0;
    st.dnz = cond ? dnz : 0;
    st.nbu = cond ? jband + 1 - o.ju0 + 1 : 0;
    st.nbv = cond ? jband - o.jv0 + 1 : 0;
    st.nbp = cond ? jband - o.jp0 + 1 : 0;
    const size_t t = (size_t)st.dnx * st.dnz;
    st.su.assign((size_t)6 * o.nyu, 0.0);
    st.sv.assign((size_t)5 * o.nyv, 0.0);
    st.sp.assign((size_t)2 * o.nyp, 0.0);
    st.cub.assign(6 * st.nbu * t, 0.0); st.cut.assign(6 * st.nbu * t, 0.0);
    st.cvb.assign(5 * st.nbv * t, 0.0); st.cvt.assign(5 * st.nbv * t, 0.0);
    st.cpb.assign(2 * st.nbp * t, 0.0); st.cpt.assign(2 * st.nbp * t, 0.0);
    st.istat = 0;
    st.on = true;
}

// conddown1/condup1 (YmC, Y2mC from x) and conddown2/condup2 (YmC from x1*x2) of one plane
static void cond1(const Oracle& o, double* Ym, double* Y2m, const double* x, double sign) {
    const int ntx = o.ngal1 / o.st.dnx, ntz = o.ngal2 / o.st.dnz;
    for (int k = 0; k < o.st.dnz; ++k)
        for (int i = 0; i < o.st.dnx; ++i) {
            double& a = Ym[k * o.st.dnx + i];
            double& b = Y2m[k * o.st.dnx + i];
            for (int iz = 0; iz < ntz; ++iz)
                for (int ix = 0; ix < ntx; ++ix) {
                    const double v = x[(size_t)(k + o.st.dnz * iz) * o.rowlen + i + o.st.dnx * ix];
                    a = a + v * sign;
                    b = b + v * v;
                }
        }
}
static void cond2(const Oracle& o, double* Ym, const double* x1, const double* x2, double s1, double s2) {
    const int ntx = o.ngal1 / o.st.dnx, ntz = o.ngal2 / o.st.dnz;
    for (int k = 0; k < o.st.dnz; ++k)
        for (int i = 0; i < o.st.dnx; ++i) {
            double& a = Ym[k * o.st.dnx + i];
            for (int iz = 0; iz < ntz; ++iz)
                for (int ix = 0; ix < ntx; ++ix) {
                    const size_t e = (size_t)(k + o.st.dnz * iz) * o.rowlen + i + o.st.dnx * ix;
                    a = a + x1[e] * s1 * x2[e] * s2;
                }
        }
}

static void stats_accumulate(Oracle& o) {
    auto& st = o.st;
    interp(o);
    const size_t psz = (size_t)o.rowlen * o.ngal2;
    const size_t tsz = (size_t)st.dnx * st.dnz;
    const bool cond = tsz > 0;
#pragma omp parallel
    {
        PlaneWork w;
        w.init(o);
        std::vector<double> a(psz), b(psz), c(psz);
#pragma omp for schedule(dynamic)
        for (int j = o.ju0; j <= o.ju1; ++j) {  // u1PL, u3PL, u2PL_itp
            const int jr = j - o.ju0;
            gather_plane(o, o.u1, o.nyu, o.ju0, j, a.data());
            gather_plane(o, o.u3, o.nyu, o.ju0, j, b.data());
            gather_plane(o, o.u2i, o.nyu, o.ju0, j, c.data());
            four_to_phys(o, a.data(), true, w);
            four_to_phys(o, b.data(), true, w);
            four_to_phys(o, c.data(), true, w);
            double s0 = st.su[0 * o.nyu + jr], s1 = st.su[1 * o.nyu + jr], s2 = st.su[2 * o.nyu + jr];
            double s3 = st.su[3 * o.nyu + jr], s4 = st.su[4 * o.nyu + jr], s5 = st.su[5 * o.nyu + jr];
            for (int k = 0; k < o.ngal2; ++k)
                for (int i = 0; i < o.ngal1; ++i) {
                    const size_t e = (size_t)k * o.rowlen + i;
                    s0 = s0 + a[e]; s1 = s1 + a[e] * a[e];
                    s2 = s2 + b[e]; s3 = s3 + b[e] * b[e];
                    s4 = s4 + a[e] * c[e]; s5 = s5 + a[e] * b[e];
                }
            st.su[0 * o.nyu + jr] = s0; st.su[1 * o.nyu + jr] = s1; st.su[2 * o.nyu + jr] = s2;
            st.su[3 * o.nyu + jr] = s3; st.su[4 * o.nyu + jr] = s4; st.su[5 * o.nyu + jr] = s5;
            if (!cond) continue;
            for (int side = 0; side < 2; ++side) {
                const int j1 = side == 0 ? jr : o.ju1 - j;
                if (j1 >= st.nbu) continue;
                double* C = (side == 0 ? st.cub : st.cut).data();
                const size_t qs = (size_t)st.nbu * tsz;
                double* at = C + (size_t)j1 * tsz;
                const double sv = side == 0 ? 1.0 : -1.0;
                cond1(o, at + 0 * qs, at + 1 * qs, a.data(), 1.0);
                cond1(o, at + 2 * qs, at + 3 * qs, b.data(), 1.0);
                cond2(o, at + 4 * qs, a.data(), c.data(), 1.0, sv);
                cond2(o, at + 5 * qs, a.data(), b.data(), 1.0, 1.0);
            }
        }
#pragma omp for schedule(dynamic)
        for (int j = o.jv0; j <= o.jv1; ++j) {  // u2PL, u3PL_itp, wx
            const int jr = j - o.jv0;
            gather_plane(o, o.u2, o.nyv, o.jv0, j, a.data());
            gather_plane(o, o.u3i, o.nyv, o.jv0, j, b.data());
            // wx = -der_z(v) + der_yv_h_wx(w): dw/dy - dv/dz at the face (FOU3D.f90:187-204)
            std::memset(c.data(), 0, sizeof(double) * psz);
            for (int col = 0; col < o.ncol; ++col) {
                const int i = o.col_i(col), q = o.col_q(col);
                cplx dz = (q == o.n2 / 2) ? cplx(0.0, 0.0) : cplx(0.0, o.kz[q]) * o.V(o.u2, col, j);
                cplx dy = (o.U(o.u3, col, j + 1) - o.U(o.u3, col, j)) * o.DTHV(j);
                cplx v = -dz + dy;
                const size_t e = (size_t)o.row_of(q) * o.rowlen + 2 * i;
                c[e] = v.real();
                c[e + 1] = v.imag();
            }
            four_to_phys(o, a.data(), true, w);
            four_to_phys(o, b.data(), true, w);
            four_to_phys(o, c.data(), false, w);
            double s0 = st.sv[0 * o.nyv + jr], s1 = st.sv[1 * o.nyv + jr], s2 = st.sv[2 * o.nyv + jr];
            double s3 = st.sv[3 * o.nyv + jr], s4 = st.sv[4 * o.nyv + jr];
            for (int k = 0; k < o.ngal2; ++k)
                for (int i = 0; i < o.ngal1; ++i) {
                    const size_t e = (size_t)k * o.rowlen + i;
                    s0 = s0 + a[e]; s1 = s1 + a[e] * a[e];
                    s4 = s4 + a[e] * b[e];
                }
            // wx over the first N1 x N2 points only (stats.f90:53-60)
            for (int k = 0; k < o.n2; ++k)
                for (int i = 0; i < o.n1; ++i) {
                    const size_t e = (size_t)k * o.rowlen + i;
                    s2 = s2 + c[e]; s3 = s3 + c[e] * c[e];
                }
            st.sv[0 * o.nyv + jr] = s0; st.sv[1 * o.nyv + jr] = s1; st.sv[2 * o.nyv + jr] = s2;
            st.sv[3 * o.nyv + jr] = s3; st.sv[4 * o.nyv + jr] = s4;
            if (!cond) continue;
            for (int side = 0; side < 2; ++side) {
                const int j1 = side == 0 ? jr : o.jv1 - j;
                if (j1 >= st.nbv) continue;
                double* C = (side == 0 ? st.cvb : st.cvt).data();
                const size_t qs = (size_t)st.nbv * tsz;
                double* at = C + (size_t)j1 * tsz;
                const double sv = side == 0 ? 1.0 : -1.0;
                cond1(o, at + 0 * qs, at + 1 * qs, a.data(), sv);
                cond1(o, at + 2 * qs, at + 3 * qs, c.data(), 1.0);
                cond2(o, at + 4 * qs, a.data(), b.data(), sv, 1.0);
            }
        }
#pragma omp for schedule(dynamic)
        for (int j = o.jp0; j <= o.jp1; ++j) {  // ppPL
            const int jr = j - o.jp0;
            gather_plane(o, o.p, o.nyp, o.jp0, j, a.data());
            four_to_phys(o, a.data(), false, w);
            double s0 = st.sp[jr], s1 = st.sp[o.nyp + jr];
            for (int k = 0; k < o.ngal2; ++k)
                for (int i = 0; i < o.ngal1; ++i) {
                    const size_t e = (size_t)k * o.rowlen + i;
                    s0 = s0 + a[e]; s1 = s1 + a[e] * a[e];
                }
            st.sp[jr] = s0; st.sp[o.nyp + jr] = s1;
            if (!cond) continue;
            for (int side = 0; side < 2; ++side) {
                const int j1 = side == 0 ? jr : o.jp1 - j;
                if (j1 >= st.nbp) continue;
                double* C = (side == 0 ? st.cpb : st.cpt).data();
                const size_t qs = (size_t)st.nbp * tsz;
                cond1(o, C + (size_t)j1 * tsz, C + qs + (size_t)j1 * tsz, a.data(), 1.0);
            }
        }
    }
    // spectra (spectra.f90:1-56, called at FOU3D.f90:107-110 with u2_itp of interp_v):
    // buildsp sp = sp + Re(u)^2 + Im(u)^2, buildspUV sp = sp + Re(u) Re(v) + Im(u) Im(v)
    if (!st.spu.empty()) {
#pragma omp parallel for schedule(static)
        for (int col = 0; col < o.ncol; ++col) {
            auto sq = [](double& sp, cplx a) { sp = sp + a.real() * a.real() + a.imag() * a.imag(); };
            for (int j = o.ju0; j <= o.ju1; ++j) {
                const size_t e = (size_t)col * o.nyu + (j - o.ju0);
                sq(st.spu[e], o.U(o.u1, col, j));
                sq(st.spw[e], o.U(o.u3, col, j));
                const cplx a = o.U(o.u1, col, j), b = o.U(o.u2i, col, j);
                st.spuv[e] = st.spuv[e] + a.real() * b.real() + a.imag() * b.imag();
            }
            for (int j = o.jv0; j <= o.jv1; ++j) sq(st.spv[(size_t)col * o.nyv + (j - o.jv0)], o.V(o.u2, col, j));
            for (int j = o.jp0; j <= o.jp1; ++j) sq(st.spp[(size_t)col * o.nyp + (j - o.jp0)], o.P(o.p, col, j));
        }
    }
    st.istat += 1;
}

static void dtc_calc(Oracle& o, double* terms) {
    // maxima per band (index 0: wall bands, 1: middle band); each band's x/z terms use its
    // own N (dtc_calc runs per rank with bandPL, the MPI MIN combines them, FOU3D.f90:177-180)
    double um[2] = {0.0, 0.0}, wm[2] = {0.0, 0.0}, vm = 1e-6;
#pragma omp parallel
    {
        PlaneWork w;
        w.init(o);
        const size_t psz = (size_t)o.rowlen * o.ngal2;
        std::vector<double> a(psz);
        double lu[2] = {0.0, 0.0}, lw[2] = {0.0, 0.0}, lv = 0.0;
#pragma omp for schedule(dynamic) nowait
        for (int j = o.ju0; j <= o.ju1; ++j) {
            const bool mid = o.u_mid(j);
            const PlaneGeom g = o.geom(mid);
            const size_t gsz = (size_t)g.rowlen * g.ngal2;
            gather_plane(o, g, o.u1, o.nyu, o.ju0, j, a.data());
            four_to_phys(g, a.data(), true, w);
            for (size_t e = 0; e < gsz; ++e) lu[mid] = std::max(lu[mid], std::fabs(a[e]));
            gather_plane(o, g, o.u3, o.nyu, o.ju0, j, a.data());
            four_to_phys(g, a.data(), true, w);
            for (size_t e = 0; e < gsz; ++e) lw[mid] = std::max(lw[mid], std::fabs(a[e]));
        }
#pragma omp for schedule(dynamic) nowait
        for (int j = o.jv0 + 1; j <= o.jv1 - 1; ++j) {
            const PlaneGeom g = o.geom(o.v_mid(j));
            gather_plane(o, g, o.u2, o.nyv, o.jv0, j, a.data());
            four_to_phys(g, a.data(), true, w);
            for (int k = 0; k < g.ngal2; ++k)
                for (int i = 0; i < g.ngal1; ++i)
                    lv = std::max(lv, std::fabs(a[(size_t)k * g.rowlen + i]) * o.DTHV(j));
        }
#pragma omp critical
        {
            for (int b = 0; b < 2; ++b) {
                um[b] = std::max(um[b], lu[b]);
                wm[b] = std::max(wm[b], lw[b]);
            }
            vm = std::max(vm, lv);
        }
    }
    terms[0] = 1.0 / (o.alp * (o.n1 / 2) * um[0]);
    terms[1] = 1.0 / (o.bet * (o.n2 / 2) * wm[0]);
    if (o.mb) {
        terms[0] = std::min(terms[0], 1.0 / (o.alp * (o.n1m / 2) * um[1]));
        terms[1] = std::min(terms[1], 1.0 / (o.bet * (o.n2m / 2) * wm[1]));
    }
    terms[2] = 1.0 / vm;
}

static thread_local std::string g_err;

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_create(const cfd_config* c, const cfd_ib_list* ibu, const cfd_ib_list* ibv) {
    try {
        Oracle* o = new Oracle();
        o->ngal1 = c->ngal1; o->ngal2 = c->ngal2;
        o->n1 = 2 * (c->ngal1 / 3); o->n2 = 2 * (c->ngal2 / 3);
        o->nkx = o->n1 / 2 + 1; o->ncol = o->nkx * o->n2;
        o->ny = c->ny; o->dny = c->dsty;
        o->ju0 = -o->dny; o->ju1 = o->ny + o->dny;
        o->jv0 = -o->dny; o->jv1 = o->ny + o->dny - 1;
        o->jp0 = -o->dny + 1; o->jp1 = o->ny + o->dny - 1;
        o->nyu = o->ju1 - o->ju0 + 1; o->nyv = o->jv1 - o->jv0 + 1; o->nyp = o->jp1 - o->jp0 + 1;
        o->rowlen = o->ngal1 + 2;
        o->Re = c->re; o->alp = c->alp; o->bet = c->bet; o->dt = c->dt; o->mpgx = c->mpgx;
        o->QxT = c->qxt; o->ctpress = c->flag_ctpress;
        o->yu.assign(c->yu, c->yu + o->nyu);
        o->yv.assign(c->yv, c->yv + o->nyv);
        o->dthdyu.assign(c->dthdyu, c->dthdyu + o->nyu);
        o->dthdyv.assign(c->dthdyv, c->dthdyv + o->nyv);
        o->dyu2i.assign(c->dyu2i, c->dyu2i + 3 * o->nyu);
        o->dyv2i.assign(c->dyv2i, c->dyv2i + 3 * o->nyv);
        // gridweighting / gridweighting_interp of the single band (start.f90:495-508)
        o->gwb = -(o->YV(o->jv0) - o->YU(o->ju0)) / (o->YV(o->jv0) - o->YU(o->ju0 + 1));
        o->gwt = (o->YU(o->ju1) - o->YV(o->jv1)) / (o->YV(o->jv1) - o->YU(o->ju1 - 1));
        o->gwib = (o->YU(o->ju0) - o->YU(o->ju0 + 1)) / (o->YV(o->jv0) - o->YU(o->ju0 + 1));
        o->gwit = (o->YU(o->ju1) - o->YU(o->ju1 - 1)) / (o->YV(o->jv1) - o->YU(o->ju1 - 1));
        // column segments: the channel (long columns) and, with three bands, the bottom and
        // top segments of the short columns (jlim, start.f90:1538-1557) with their
        // gridweighting / gridweighting_interp (start.f90:494-508)
        o->segL = Seg{o->ju0, o->ju1, o->jv0, o->jv1, o->jp0, o->jp1, o->gwb, o->gwt, o->gwib, o->gwit};
        if (c->band_vface > 0) {
            const int jb = c->band_vface, m = o->ny - 2 - jb;  // N(3,1), N(3,2) = N(4,2)
            if (jb + 2 >= m || jb + 1 <= o->jv0 + 1)
                throw std::runtime_error("band_vface leaves no middle band of two planes");
            if (c->ngal1_mid > c->ngal1 || c->ngal2_mid > c->ngal2 || c->ngal1_mid < 6 || c->ngal2_mid < 6)
                throw std::runtime_error("middle-band sizes must lie between 6 and the wall bands' sizes");
            o->mb = 1;
            o->jb = jb;
            o->ngal1m = c->ngal1_mid; o->ngal2m = c->ngal2_mid;
            o->n1m = 2 * (o->ngal1m / 3); o->n2m = 2 * (o->ngal2m / 3);
            const double gw1t = (o->YU(jb + 2) - o->YV(jb + 1)) / (o->YV(jb + 1) - o->YU(jb + 1));
            const double gwi1t = (o->YU(jb + 2) - o->YU(jb + 1)) / (o->YV(jb + 1) - o->YU(jb + 1));
            const double gw3b = -(o->YV(m) - o->YU(m)) / (o->YV(m) - o->YU(m + 1));
            const double gwi3b = (o->YU(m) - o->YU(m + 1)) / (o->YV(m) - o->YU(m + 1));
            o->segS[0] = Seg{o->ju0, jb + 2, o->jv0, jb + 1, o->ju0 + 1, jb + 1, o->gwb, gw1t, o->gwib, gwi1t};
            o->segS[1] = Seg{m, o->ju1, m, o->jv1, m + 1, o->jp1, gw3b, o->gwt, gwi3b, o->gwit};
            o->islong.assign(o->ncol, 0);
            for (int col = 0; col < o->ncol; ++col) {
                const int i = col % o->nkx, q = col / o->nkx;
                o->islong[col] = i <= o->n1m / 2 && (q < o->n2m / 2 || q >= o->n2 - o->n2m / 2);
            }
            for (const cfd_ib_list* l : {ibu, ibv})
                if (l)
                    for (int s = 0; s < 2; ++s)
                        if (l->jhi[s] >= l->jlo[s] && !(l->jhi[s] <= jb || l->jlo[s] > m))
                            throw std::runtime_error("immersed-boundary planes must lie in the wall bands");
        }
        o->kx.resize(o->nkx);
        for (int i = 0; i < o->nkx; ++i) o->kx[i] = o->alp * i;
        o->kz.resize(o->n2);
        for (int q = 0; q < o->n2; ++q) o->kz[q] = q < o->n2 / 2 ? o->bet * q : -o->bet * (o->n2 - q);
        auto setib = [](IBData& d, const cfd_ib_list* l) {
            if (!l) return;
            d.n = l->n;
            d.idx.assign(l->idx, l->idx + 9 * (size_t)l->n);
            d.w.assign(l->w, l->w + 3 * (size_t)l->n);
            for (int s = 0; s < 2; ++s) { d.jlo[s] = l->jlo[s]; d.jhi[s] = l->jhi[s]; }
        };
        setib(o->ibu, ibu);
        setib(o->ibv, ibv);
        size_t su = (size_t)o->ncol * o->nyu, sv = (size_t)o->ncol * o->nyv, sp = (size_t)o->ncol * o->nyp;
        for (auto* f : {&o->u1, &o->u3, &o->Nu1, &o->Nu3, &o->du1, &o->du3, &o->u2i, &o->vvc}) f->assign(su, 0.0);
        for (auto* f : {&o->u2, &o->Nu2, &o->du2, &o->u1i, &o->u3i, &o->uvf, &o->vwf}) f->assign(sv, 0.0);
        for (auto* f : {&o->p, &o->psi, &o->div}) f->assign(sp, 0.0);
        o->px.init(o->ngal1);
        o->pz.init(o->ngal2);
        if (o->mb) {
            o->pxm.init(o->ngal1m);
            o->pzm.init(o->ngal2m);
        }
        return o;
    } catch (std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_destroy(void* h) { delete (Oracle*)h; }

static std::vector<cplx>* field_of(Oracle* o, int f) {
    switch (f) {
        case CFD_FIELD_U1: return &o->u1;
        case CFD_FIELD_U2: return &o->u2;
        case CFD_FIELD_U3: return &o->u3;
        case CFD_FIELD_P: return &o->p;
        case CFD_FIELD_NU1: return &o->Nu1;
        case CFD_FIELD_NU2: return &o->Nu2;
        case CFD_FIELD_NU3: return &o->Nu3;
        case CFD_FIELD_DIV: return &o->div;
        case CFD_FIELD_PSI: return &o->psi;
        case CFD_FIELD_DU1: return &o->du1;
        case CFD_FIELD_DU2: return &o->du2;
        case CFD_FIELD_DU3: return &o->du3;
    }
    return nullptr;
}

// host arrays in CFD_LAYOUT_REF order (f(j,column), j fastest) = the oracle's own layout
int orc_set_field(void* h, int f, const double* src) {
    auto* v = field_of((Oracle*)h, f);
    if (!v) return CFD_ERR_ARG;
    std::memcpy((void*)v->data(), (const void*)src, sizeof(cplx) * v->size());
    return CFD_OK;
}
int orc_get_field(void* h, int f, double* dst) {
    auto* v = field_of((Oracle*)h, f);
    if (!v) return CFD_ERR_ARG;
    std::memcpy((void*)dst, (const void*)v->data(), sizeof(cplx) * v->size());
    return CFD_OK;
}

int orc_rhs0(void* h, int krk) { rhs0(*(Oracle*)h, krk); return 0; }
int orc_nonlinear(void* h, int krk) { nonlinear(*(Oracle*)h, krk); return 0; }
int orc_solve_uvw(void* h, int krk) {
    Oracle& o = *(Oracle*)h;
    solve_u(o, o.u1, o.du1, krk);
    solve_v(o, krk);
    solve_u(o, o.u3, o.du3, krk);
    return 0;
}
int orc_meanflow(void* h, int krk) { meanflow(*(Oracle*)h, krk); return 0; }
int orc_solve_p(void* h, int krk) { solve_p(*(Oracle*)h, krk); return 0; }
int orc_vcorr(void* h, int krk) { v_corr(*(Oracle*)h, krk); return 0; }
int orc_rk_substep(void* h, int krk) { rk_substep(*(Oracle*)h, krk); return 0; }
int orc_step(void* h, int nsteps) {
    Oracle& o = *(Oracle*)h;
    for (int s = 0; s < nsteps; ++s) {
        for (int k = 1; k <= 3; ++k) rk_substep(o, k);
        if (o.ctpress == 1) meanflow(o, 1);
    }
    return 0;
}
int orc_stats_configure(void* h, int jband, int dnx, int dnz, int spectra) {
    if (((Oracle*)h)->mb) return CFD_ERR_ARG;  // statistics of one band only
    Oracle& o = *(Oracle*)h;
    if (jband >= o.jv0 && (dnx <= 0 || dnz <= 0 || o.ngal1 % dnx || o.ngal2 % dnz)) return 1;
    stats_configure(o, jband, dnx, dnz, spectra);
    return 0;
}
// same layout as cfd_spectra_read: sp(j,column), j fastest
int orc_spectra_read(void* h, double* spu, double* spv, double* spw, double* spuv, double* spp) {
    Oracle& o = *(Oracle*)h;
    auto& st = o.st;
    if (!st.on || st.spu.empty()) return 5;
    auto cp_ = [](double* dst, const std::vector<double>& a) { if (dst) std::copy(a.begin(), a.end(), dst); };
    cp_(spu, st.spu); cp_(spv, st.spv); cp_(spw, st.spw); cp_(spuv, st.spuv); cp_(spp, st.spp);
    return 0;
}
int orc_stats_accumulate(void* h) {
    Oracle& o = *(Oracle*)h;
    if (!o.st.on) return 5;
    stats_accumulate(o);
    return 0;
}
// same layout as cfd_stats_read: bottom + top band combined
int orc_stats_read(void* h, double* su, double* sv, double* sp, double* cu, double* cv, double* cp, int* istat) {
    Oracle& o = *(Oracle*)h;
    auto& st = o.st;
    if (!st.on) return 5;
    auto cp_ = [](double* dst, const std::vector<double>& a) { if (dst) std::copy(a.begin(), a.end(), dst); };
    auto comb = [](double* dst, const std::vector<double>& b, const std::vector<double>& t) {
        if (dst) for (size_t i = 0; i < b.size(); ++i) dst[i] = b[i] + t[i];
    };
    cp_(su, st.su); cp_(sv, st.sv); cp_(sp, st.sp);
    comb(cu, st.cub, st.cut); comb(cv, st.cvb, st.cvt); comb(cp, st.cpb, st.cpt);
    if (istat) *istat = st.istat;
    return 0;
}
int orc_cfl(void* h, double* dtc, double* terms) {
    double t[3];
    dtc_calc(*(Oracle*)h, t);
    if (terms) { terms[0] = t[0]; terms[1] = t[1]; terms[2] = t[2]; }
    *dtc = std::min(t[0], t[1]);
    return 0;
}
int orc_set_dt(void* h, double dt) {
    if (!(dt > 0)) return 1;
    ((Oracle*)h)->dt = dt;
    return 0;
}
int orc_set_quirk(void* h, int lastplane) {
    if (((Oracle*)h)->mb && lastplane) return CFD_ERR_ARG;  // a single slab has one band
    ((Oracle*)h)->quirk_lastplane = lastplane;
    return 0;
}
void orc_get_scalars(void* h, double* mpgx, double* qx, double* dgx) {
    Oracle& o = *(Oracle*)h;
    *mpgx = o.mpgx; *qx = o.Qx; *dgx = o.dgx;
}
int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// stand-alone transforms with the reference's rft/cft semantics (unit-tested against numpy)
int orc_rft(double* c, int n, int isa, int m, int iopt) {
    try {
        RFFTPlan p; p.init(n);
        std::vector<cplx> z(n), t(n);
        for (int j = 0; j < m; ++j) {
            if (iopt < 0) p.forward(c + (size_t)j * isa, z.data(), t.data());
            else p.inverse(c + (size_t)j * isa, z.data(), t.data());
        }
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return CFD_ERR_SIZE; }
}
int orc_cft(double* c, int n, int ise, int isa, int m, int iopt) {
    try {
        FFTPlan p; p.init(n);
        std::vector<cplx> z(n), t(n);
        for (int b = 0; b < m; ++b) {
            double* base = c + (size_t)b * isa;
            for (int j = 0; j < n; ++j) z[j] = cplx(base[(size_t)j * ise], base[(size_t)j * ise + 1]);
            p.exec(z.data(), t.data(), iopt < 0 ? -1 : +1);
            const double s = iopt < 0 ? 1.0 / n : 1.0;
            for (int j = 0; j < n; ++j) {
                base[(size_t)j * ise] = s * z[j].real();
                base[(size_t)j * ise + 1] = s * z[j].imag();
            }
        }
        return 0;
    } catch (std::exception& e) { g_err = e.what(); return CFD_ERR_SIZE; }
}
// four_to_phys_du / phys_to_four_du on host planes (Ngal1+2, Ngal2) of the context's size
int orc_four_to_phys(void* h, double* planes, int nplanes, int zero_oddball) {
    Oracle& o = *(Oracle*)h;
    PlaneWork w; w.init(o);
    for (int s = 0; s < nplanes; ++s) four_to_phys(o, planes + (size_t)s * o.rowlen * o.ngal2, zero_oddball != 0, w);
    return 0;
}
int orc_phys_to_four(void* h, double* planes, int nplanes) {
    Oracle& o = *(Oracle*)h;
    PlaneWork w; w.init(o);
    for (int s = 0; s < nplanes; ++s) phys_to_four(o, planes + (size_t)s * o.rowlen * o.ngal2, w);
    return 0;
}

}  // extern "C"
