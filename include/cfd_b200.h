/*
 * cfd_b200.h - C ABI of the B200 (sm_100a) hot path of the LittleHarsh channel DNS
 * (Fourier x/z, staggered 2nd-order finite differences in y, Kim & Moin fractional
 * step with low-storage RK3 / Crank-Nicolson, direct-forcing immersed boundaries).
 *
 * Every entry point takes plain pointers, sizes and int32/int64/double scalars so it can
 * be bound from Fortran with iso_c_binding, from C, or from Python ctypes.  All
 * functions return an int status (CFD_OK = 0) and never abort the process; the text of
 * the last error of a context is available from cfd_last_error().
 *
 * Citations are file:line in the reference Fortran tree (Mel222/CFD).
 *
 * Conventions shared with the reference
 *  - A spectral field is the reference's cfield%f(j,column) (declaration.f90:140-142):
 *    complex(8), one y-profile per (kx,kz) column.  With a single y-band the column list
 *    is k-major, i-minor: column = (k-1)*(N1/2+1) + i + 1, i = 0..N1/2 (kx = alp*i),
 *    k = 1..N2 (kz = bet*(k-1) for k <= N2/2, -bet*(N2-k+1) above; start.f90:965-986,
 *    start.f90:1488-1501).  N1 = 2*(Ngal1/3), N2 = 2*(Ngal2/3) (start.f90:108-111).
 *  - y indices are absolute as in the reference: u/w live on j = -dsty .. ny+dsty
 *    (ghosts included), v on j = -dsty .. ny+dsty-1 (walls included), p on
 *    j = -dsty+1 .. ny+dsty-1 (start.f90:1538-1557 with y_grid_rough.f90:46-52).
 *  - Host arrays passed to cfd_upload_field/cfd_download_field are interleaved
 *    (re,im) doubles in one of two orders: CFD_LAYOUT_REF is f(j,column) with j fastest
 *    (the Fortran array itself), CFD_LAYOUT_PLANE is [j][column] with column fastest
 *    (the device layout, no reordering needed).
 *  - A physical plane is the reference's xPL(Ngal1+2, Ngal2): Re/Im of kx-mode i at
 *    entries 2i+1/2i+2 of row k (FOU3D.f90:842-848); after the inverse transform entries
 *    1..Ngal1 of each row are samples at x=(i-1)Lx/Ngal1.  Forward transforms scale by
 *    1/(Ngal1*Ngal2), inverse transforms do not (rft_buff.f:60-70, cft_buff.f:41-51).
 */
#ifndef CFD_B200_H
#define CFD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CFD_OK              0
#define CFD_ERR_ARG         1   /* null pointer, bad enum, out-of-range index           */
#define CFD_ERR_SIZE        2   /* FFT length not 2^a*3^b, grid too small, list too big  */
#define CFD_ERR_CUDA        3   /* a CUDA runtime call failed                            */
#define CFD_ERR_NONFINITE   4   /* NaN/Inf found by the watchdog                         */
#define CFD_ERR_STATE       5   /* call out of order (e.g. before state upload)          */
#define CFD_ERR_NOMEM       6   /* device allocation failed at create                    */

/* arithmetic of the transforms and nonlinear products */
#define CFD_PREC_FP64   0       /* everything in FP64 (the reference's real(8))          */
#define CFD_PREC_MIXED  1       /* FFTs/products/Nu history in FP32; y-solves, state,
                                   mean mode, bulk correction in FP64                   */

/* field identifiers */
#define CFD_FIELD_U1    0       /* u  (ugrid)                       */
#define CFD_FIELD_U2    1       /* v  (vgrid)                       */
#define CFD_FIELD_U3    2       /* w  (ugrid)                       */
#define CFD_FIELD_P     3       /* p  (pgrid)                       */
#define CFD_FIELD_NU1   4       /* RK nonlinear history, ugrid      */
#define CFD_FIELD_NU2   5       /* RK nonlinear history, vgrid      */
#define CFD_FIELD_NU3   6       /* RK nonlinear history, ugrid      */
#define CFD_FIELD_DIV   7       /* divergence (pgrid, diagnostic)   */
#define CFD_FIELD_PSI   8       /* pressure increment (pgrid)       */
#define CFD_FIELD_DU1   9       /* RHS / Helmholtz right-hand side  */
#define CFD_FIELD_DU2   10
#define CFD_FIELD_DU3   11

#define CFD_LAYOUT_REF   0      /* f(j,column), j fastest (Fortran cfield%f)             */
#define CFD_LAYOUT_PLANE 1      /* [j][column], column fastest                           */

/* Problem definition.  Replaces the module globals of declaration.f90 that the hot path
 * reads (Re, alp, bet, dt, mpgx, QxT, flag_ctpress, N/Ngal, yu, yv, dthdyu, dthdyv,
 * dyu2i, dyv2i).  Grid arrays start at j = -dsty. */
typedef struct cfd_config {
    int32_t ngal1;          /* Ngal(1,1): collocation points in x (2^a*3^b)         */
    int32_t ngal2;          /* Ngal(2,1): collocation points in z (2^a*3^b)         */
    int32_t ny;             /* input.in ny: faces from y=-1 to y=1                 */
    int32_t dsty;           /* in-canopy planes below each crest (dny)             */
    double  re;             /* Re (bulk)                                           */
    double  alp, bet;       /* Lx = 2*pi/alp, Lz = 2*pi/bet                        */
    double  dt;             /* fixed time step                                     */
    double  mpgx;           /* mean pressure gradient (initial value if ctpress=0) */
    double  qxt;            /* target flow rate QxT (flag_ctpress = 0)             */
    int32_t flag_ctpress;   /* 1 = constant pressure gradient, 0 = constant flow   */
    int32_t precision;      /* CFD_PREC_FP64 or CFD_PREC_MIXED                     */
    const double *yu;       /* [ny+2*dsty+1]                                       */
    const double *yv;       /* [ny+2*dsty]                                         */
    const double *dthdyu;   /* [ny+2*dsty+1]                                       */
    const double *dthdyv;   /* [ny+2*dsty]                                         */
    const double *dyu2i;    /* [ny+2*dsty+1][3]  (Fortran dyu2i(3,j))              */
    const double *dyv2i;    /* [ny+2*dsty][3]                                      */
    /* Three y-bands (start.f90:76-111) when band_vface > 0: band_vface is the reference's
     * N(3,1), the last v face of the bottom band.  The wall bands (u/w centres up to
     * band_vface+1 and from ny-1-band_vface, v faces up to band_vface and from
     * ny-1-band_vface) run at ngal1 x ngal2, the middle band at ngal1_mid x ngal2_mid
     * (2^a*3^b, at most the wall bands' size); the modes of the wall bands that the middle
     * band lacks are "short" columns, solved in each wall band separately with the band
     * interface rows of LU_buildU/V/P (tridLU_3D_IB.f90:349-413, 417-491).  band_vface = 0:
     * one band, ngal*_mid ignored.  The column list and the field layout are those of the
     * wall bands; a short column is zero outside its two segments. */
    int32_t ngal1_mid, ngal2_mid, band_vface;
} cfd_config;

/* Immersed-boundary forcing list of one grid (start.f90:1133-1145 f_list_ib_u/w_list_ib_u).
 * idx[p*9 + 0..8] = i,k,j,i2,k2,j2,i3,k3,j3 (i,k 1-based physical indices, j absolute);
 * w[p*3 + 0..2] = Lap coefficient, w2, w3.  Points act in list order: the reference sorts
 * them by (j,k,i) (geom_circ_rough_mixed_forcing_24pt.f90:578-606).  jlo/jhi are the plane
 * ranges that go through the physical round trip (nyuIB1..nyuIB2 / nyvIB1..nyvIB2 of the
 * bottom [0] and top [1] canopy, start.f90:1091-1101); a range with jhi < jlo is empty.
 * Every j, j2, j3 must lie inside one of the ranges. */
typedef struct cfd_ib_list {
    int32_t        n;
    const int32_t *idx;
    const double  *w;
    int32_t        jlo[2];
    int32_t        jhi[2];
} cfd_ib_list;

typedef struct cfd_ctx cfd_ctx;

/* ---- lifetime ------------------------------------------------------------------- */

/* Build a context on CUDA device `device`: validates sizes, uploads the grid, the
 * wavenumbers and the IB lists, and allocates every device buffer the step needs (no
 * allocation happens inside a step).  Replaces start() + getbounds() + LU_buildP()
 * set-up (start.f90:36-649, start.f90:1020-1380, tridLU_3D_IB.f90:417-491).
 * ibu: list for u and w (ugrid), ibv: list for v (vgrid); either may be NULL. */
int cfd_create(const cfd_config *cfg, const cfd_ib_list *ibu, const cfd_ib_list *ibv,
               int32_t device, cfd_ctx **out);
int cfd_destroy(cfd_ctx *ctx);
const char *cfd_last_error(const cfd_ctx *ctx);

/* Launch shapes of the kernels (no counterpart in the reference).  A zero field keeps the
 * library's choice (or the CFD_* environment override of the same name); cfd_b200/autotune.py
 * picks them by timing the candidates on the device.
 *   xline_path   1: register two-step x-line kernel with one z transform per field plane,
 *                2: shared-memory Stockham x-line kernel with the per-slot z pass,
 *                3: as 1 with three real inputs packed into 1.5 complex lines per row,
 *                4: as 1 with the two lines of a row in packed FP32 pairs (.f32x2
 *                   instructions; FP32-mixed only, FP64 contexts run path 1),
 *                5: as 1 with the kernel held to 64 registers per thread (more CTAs per
 *                   SM; FP32-mixed only, FP64 contexts run path 1),
 *                6: x-line pass marching in y: a CTA walks a pair of z rows up the channel,
 *                   transforms u, w and v of each plane pair once and interpolates in
 *                   physical space (1.5 inverse and 3 forward lines per row and plane pair
 *                   instead of 4 and 3); FP32-mixed one-band contexts with x lengths 64,
 *                   96, 128, 192, 384 (the default at 384; FP64 contexts, other lengths
 *                   and three-band channels run path 1); CFD_XMARCH_STEPS sets its y-chunk
 *   xline_rows   rows per CTA of the two-step x-line kernel: 2, 4 or 8 (path 6: 2 or 4)
 *   zlines       lines per CTA of the two-step z kernels: 4, 8 or 16
 *   solve_kind   1: thread-per-column Thomas sweeps (the only kind; other values fall back
 *                to it)
 *   solve_cols   threads (columns) per CTA of the column sweeps k_solve_uvw and k_solve_p:
 *                32, 64, 128 or 256
 *   rhs_chunk    y-planes per thread of the right-hand-side kernel: 2 .. 64
 *   xsplit       radix order of the x-line transforms (x-line paths 1, 5): 1 = the split
 *                N = N1*N2 of 64 = 8*8, 96 = 8*12, 128 = 8*16, 192 = 16*12, 384 = 16*24,
 *                768 = 32*24 (first step N1 points); 2 = the transposed split (16*4, 12*8,
 *                16*8, 12*16, 24*16, 24*32)
 *   zsplit       the same for the z transforms of the nonlinear pass (x-line path 1) */
typedef struct cfd_tuning {
    int32_t xline_path, xline_rows, zlines, solve_kind, solve_cols, rhs_chunk, xsplit, zsplit;
} cfd_tuning;
/* cfd_create with explicit launch shapes (tuning may be NULL: as cfd_create). */
int cfd_create_tuned(const cfd_config *cfg, const cfd_ib_list *ibu, const cfd_ib_list *ibv,
                     int32_t device, const cfd_tuning *tuning, cfd_ctx **out);
/* The launch shapes a context runs with (every field filled in). */
int cfd_get_tuning(const cfd_ctx *ctx, cfd_tuning *tuning);

/* Work on a caller-provided cudaStream_t (NULL = the context's own stream). */
int cfd_set_stream(cfd_ctx *ctx, void *stream);
int cfd_synchronize(cfd_ctx *ctx);

/* Sizes: number of complex values of a field (columns * planes), its first absolute j
 * and its plane count. */
int cfd_field_shape(const cfd_ctx *ctx, int32_t field, int64_t *ncomplex,
                    int32_t *j0, int32_t *nplanes, int32_t *ncolumns);

/* ---- state transfer (littleharsh.f90:103-147 arrays) ---------------------------- */

/* Host <-> device copy of one field (complex(8) interleaved).  host must hold
 * ncomplex complex values in `layout` order.  Stream-ordered; call cfd_synchronize
 * before reading a downloaded buffer.  Pinned host memory makes the copy async.
 * U1, U2, U3 and P in CFD_LAYOUT_REF go through a staging buffer per field, in 8 column
 * chunks, on two copy streams of their own (one per direction): the upload of a chunk
 * waits only for the download that last used that chunk of the buffer, so a loop of
 * upload / cfd_step / download without host synchronisation overlaps the next step's
 * uploads with this step's downloads.  The first such transfer of a field allocates its
 * buffer (one field's size). */
int cfd_upload_field(cfd_ctx *ctx, int32_t field, const double *host, int32_t layout);
int cfd_download_field(cfd_ctx *ctx, int32_t field, double *host, int32_t layout);
/* Device pointer of a field (FP64 [j][column] complex; NU* are FP32 complex in
 * CFD_PREC_MIXED).  Lets a caller fill state in place.  The immersed-boundary forcing of
 * cfd_solve_uvw reuses the z transforms of u, v, w made by the preceding cfd_nonlinear;
 * uploads and this call mark them stale, so a caller that writes u, v or w through an
 * earlier pointer between cfd_nonlinear and cfd_solve_uvw calls it again after writing. */
int cfd_field_device_ptr(cfd_ctx *ctx, int32_t field, void **dev_ptr);

/* ---- one RK substep, stage by stage (littleharsh.f90:163-189) -------------------- */
/* krk = 1, 2, 3 selects the Le & Moin coefficients (start.f90:395-409). */

/* RHS0_u1/u2/u3 (littleharsh.f90:613-730): du = a/Re*L(u) - c*Nu_old - d*grad p
 * (+ -d*mpgx on the (0,0) mode). */
int cfd_rhs0(cfd_ctx *ctx, int32_t krk);
/* nonlinear (FOU3D.f90:41-259): y-interpolation, inverse FFTs, products, forward FFTs,
 * x/z and y derivatives; Nu <- new advective term; du += -g*Nu. */
int cfd_nonlinear(cfd_ctx *ctx, int32_t krk);
/* solveU(u1), solveV(u2), solveU(u3) (littleharsh.f90:172-174, 732-794): du = u + dt*du,
 * immersed_boundaries_U/V (tridLU_3D_IB.f90:163-281), LUsolU/LUsolV (:50-160). */
int cfd_solve_uvw(cfd_ctx *ctx, int32_t krk);
/* meanflow_ctU / flowrate_corr (littleharsh.f90:452-484, 522-537) if flag_ctpress = 0;
 * meanflow_ctP (littleharsh.f90:504-520) otherwise. */
int cfd_meanflow(cfd_ctx *ctx, int32_t krk);
/* solveP (littleharsh.f90:556-611): divergence, psi = div/(dt(a+b)), LUsolP, p += psi. */
int cfd_solve_p(cfd_ctx *ctx, int32_t krk);
/* v_corr (littleharsh.f90:796-907): u -= dt(a+b) grad psi, ghost/wall rows. */
int cfd_vcorr(cfd_ctx *ctx, int32_t krk);

/* The whole substep (all of the above in order) and whole RK3 steps.  cfd_step captures
 * one RK3 step in a CUDA graph on first use and replays it. */
int cfd_rk_substep(cfd_ctx *ctx, int32_t krk);
int cfd_step(cfd_ctx *ctx, int32_t nsteps);

/* Scalars of the mean mode: mpgx, Qx (flow rate between the crests), dgx (last
 * correction).  Synchronises the context stream.  These are the cheap watchdog of a run: a
 * NaN or Inf anywhere in the flow reaches the mean mode through the nonlinear term within
 * one step, and the call then returns CFD_ERR_NONFINITE (the values are still written). */
int cfd_get_scalars(cfd_ctx *ctx, double *mpgx, double *qx, double *dgx);

/* Largest |div| over all columns and p-planes (error(), littleharsh.f90:322-351).
 * Synchronises. */
int cfd_divergence_max(cfd_ctx *ctx, double *errmax);

/* ---- transforms (four_to_phys_du / phys_to_four_du, FOU3D.f90:574-592, 1619-1639) -- */

/* In-place batched 2-D transforms of `nplanes` device planes laid out as the reference's
 * xPL(Ngal1+2, Ngal2) (plane stride (Ngal1+2)*Ngal2 doubles).  Inverse: complex z
 * transform of kx-modes 0..N1/2 then real x transform of every row; forward: the reverse,
 * scaled by 1/(Ngal1*Ngal2).  If zero_oddball, row Ngal2/2+1 is zeroed first
 * (four_to_phys_u, FOU3D.f90:561-563). */
int cfd_four_to_phys(cfd_ctx *ctx, double *planes_dev, int32_t nplanes, int32_t zero_oddball);
int cfd_phys_to_four(cfd_ctx *ctx, double *planes_dev, int32_t nplanes);

/* Batched strided transforms with the FFTPACK-wrapper semantics of the reference, on
 * device memory.  rft: m real vectors of length Ngal1 at stride isa (rft_buff.f:24-86);
 * cft: m complex vectors of length Ngal2, element stride ise, vector stride isa, both in
 * doubles (cft_buff.f:1-65).  iopt >= 0 inverse (unscaled), iopt < 0 forward (x 1/n).
 * n must be the context's Ngal1 (rft) or Ngal2 (cft). */
int cfd_rft(cfd_ctx *ctx, double *c_dev, int32_t isa, int32_t m, int32_t iopt);
int cfd_cft(cfd_ctx *ctx, double *c_dev, int32_t ise, int32_t isa, int32_t m, int32_t iopt);

/* ---- statistics and CFL ------------------------------------------------------------- */

/* Statistics accumulation of stats.f90:1-106, called by the reference from nonlinear at
 * kRK = 1 every nstat steps (FOU3D.f90:58-62, 187-217), on the current state.  All sums
 * are FP64 on the device whatever the context precision; the physical fields come from
 * FP64 transforms of the FP64 state.
 *   plane sums over the Ngal1 x Ngal2 points of each plane, every plane of its grid:
 *     u planes (j = -dsty..ny+dsty):   Um U2m Wm W2m UVm UWm   (UV: u * v interpolated)
 *     v planes (j = -dsty..ny+dsty-1): Vm V2m wxm wx2m VWm      (VW: v * w interpolated;
 *       wx = dw/dy - dv/dz at the faces, FOU3D.f90:187-207, summed over the first N1 x N2
 *       points of the plane only, as stats.f90:53-60 does)
 *     p planes (j = -dsty+1..ny+dsty-1): Pm P2m
 *   conditional (tile-folded) sums, conddown1/2 and condup1/2 (stats.f90:110-253): each
 *     plane of the bottom band (index j1 counted from the first plane of its grid) and of
 *     the top band (j1 counted down from the last plane, v and its products sign-flipped)
 *     is folded onto one dnx x dnz tile, ntilex = Ngal1/dnx by ntilez = Ngal2/dnz copies.
 *     The bottom band ends at the v plane jband (the reference's N(3,1)); it holds
 *     jband+dsty+2 u planes, jband+dsty+1 v planes and jband+dsty p planes.
 */
typedef struct cfd_stats_config {
    int32_t jband;      /* last v plane of the bottom band; < -dsty: no conditional sums */
    int32_t dnx, dnz;   /* tile size in points; must divide Ngal1, Ngal2 */
    int32_t spectra;    /* nonzero: each accumulation also adds the spectra below */
} cfd_stats_config;

/* Sets the band and tile, allocates the accumulators (and the plane scratch) and zeroes
 * them (the reference's allocation in start.f90:2705-2793). */
int cfd_stats_configure(cfd_ctx *ctx, const cfd_stats_config *sc);
/* stats() on the current u, v, w, p: istat += 1 and every sum above updated. */
int cfd_stats_accumulate(cfd_ctx *ctx);
/* Zeroes every sum and istat (write_stats' reset, stats.f90:411-441). */
int cfd_stats_reset(cfd_ctx *ctx);
/* Copies the sums to host arrays (any pointer may be NULL to skip it):
 *   u_sums [6][nyu]  Um U2m Wm W2m UVm UWm        (nyu = ny+2*dsty+1)
 *   v_sums [5][nyv]  Vm V2m wxm wx2m VWm          (nyv = ny+2*dsty)
 *   p_sums [2][nyp]  Pm P2m                       (nyp = ny+2*dsty-1)
 *   cu [6][nbu][dnz][dnx], cv [5][nbv][dnz][dnx], cp [2][nbp][dnz][dnx]: conditional sums
 *     in the same quantity order, bottom band plus mirrored top band as write_stats
 *     stores them (recvXC, stats.f90:473-512); dnx fastest (the Fortran YmC(i,k,j1)).
 *   istat: number of accumulated calls. */
int cfd_stats_read(cfd_ctx *ctx, double *u_sums, double *v_sums, double *p_sums,
                   double *cu, double *cv, double *cp, int32_t *istat);
/* Spectra of spectra.f90:1-56, accumulated by cfd_stats_accumulate when the configuration
 * asks for them (the reference calls spectra at the same kRK = 1 steps as stats,
 * FOU3D.f90:107-110): per plane j and column, in FP64,
 *   spU += |u|^2, spV += |v|^2, spW += |w|^2, spP += |p|^2          (buildsp)
 *   spUV += Re(u) Re(v_itp) + Im(u) Im(v_itp)                       (buildspUV)
 * over every plane of the field's grid (the reference's midband holds the whole channel),
 * v_itp being v interpolated to the u planes (interp_v, FOU3D.f90:285-308).  cfd_stats_reset
 * zeroes them with the statistics (write_spect and write_stats run together,
 * FOU3D.f90:222-225).  Copies them to host arrays in the reference's sp(j,column) layout,
 * j fastest (any pointer may be NULL):
 *   spu, spw, spuv [ncol][nyu], spv [ncol][nyv], spp [ncol][nyp] */
int cfd_spectra_read(cfd_ctx *ctx, double *spu, double *spv, double *spw, double *spuv, double *spp);

/* dtc_calc (FOU3D.f90:516-544) on the current state.  terms (may be NULL) receives
 *   [0] 1/(alp*(N1/2)*max|u|), [1] 1/(bet*(N2/2)*max|w|), [2] 1/max(1e-6, max|v|*dthdyv)
 * with the maxima over the physical u, w planes (all) and v planes (walls excluded).
 * *dtc is the reference's result min(terms[0], terms[1]): its v term divides by
 * dthetavi, a module variable that nothing assigns (declaration.f90:72; only ddthetavi is
 * set, start.f90:684), so that term is 1/0 = +Inf and never limits the step.
 * A NaN or Inf in the physical u, v, w planes gives CFD_ERR_NONFINITE with NaN results. */
int cfd_cfl(cfd_ctx *ctx, double *dtc, double *terms);

/* Changes the time step used by every following stage and step (the reference's
 * dt = min(2.5*dtv, CFL*dtc) update at kRK = 1, FOU3D.f90:177-183).  The captured RK3 graph
 * holds dt in its kernel arguments, so it is dropped here and captured again by the next
 * cfd_step. */
int cfd_set_dt(cfd_ctx *ctx, double dt);

/* Bug-compatible x/z advective term of a single-slab run (on = 1) or the per-plane term
 * (on = 0, the default).  ops_in_planes (FOU3D.f90:1529-1617) forms der_x/der_z of each
 * plane's products into 2-D scratch inside its plane loop and adds the scratch into
 * Nu1PL/Nu3PL/Nu2PL after the loop (FOU3D.f90:1541, 1571-1585, 1602-1613), so every interior
 * plane of a rank receives the term of the rank's last plane.  With on = 1 the whole channel
 * behaves as one rank's slab: every interior plane takes the term of the top ghost centre
 * (u, w) and of the top wall face (v, where it is zero), for comparisons with an unpatched
 * reference run on one rank.  Drops the captured RK3 graph like cfd_set_dt. */
int cfd_set_lastplane(cfd_ctx *ctx, int32_t on);

/* ---- batched ensemble -------------------------------------------------------------- */

/* No counterpart in the reference, which runs one channel per MPI job.  An ensemble
 * advances several independent contexts of one device together: their RK3 steps (of any
 * sizes, IB geometries and precisions) are captured as parallel branches of one CUDA graph,
 * so one graph launch per step advances every member and small members share the GPU.
 * Members stay owned by the caller (upload and download through their own entry points);
 * each must hold a state before the first cfd_ensemble_step.  Work issued on a member's
 * stream before cfd_ensemble_step completes before the ensemble step starts, and work
 * issued after it waits for it.  A member whose dt or stream changes (cfd_set_dt,
 * cfd_set_stream) is captured again at the next step. */
typedef struct cfd_ensemble cfd_ensemble;
int cfd_ensemble_create(cfd_ctx *const *members, int32_t nmembers, cfd_ensemble **out);
int cfd_ensemble_step(cfd_ensemble *ens, int32_t nsteps);
int cfd_ensemble_synchronize(cfd_ensemble *ens);
/* The stream the ensemble's graph is launched on (to order or time work around it). */
int cfd_ensemble_stream(cfd_ensemble *ens, void **stream);
const char *cfd_ensemble_last_error(const cfd_ensemble *ens);
int cfd_ensemble_destroy(cfd_ensemble *ens);

/* ---- allocation-free solve ----------------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot call cudaMalloc/cudaFree: a
 * driver whose device memory belongs to another allocator or sits under a hard cap, or a
 * loop that must not take cudaFree's implicit device synchronisation.  Solves, per
 * (kx,kz) column, the tridiagonal u/w Helmholtz system with the ghost rows (0,1,gw_bot)
 * and (gw_top,1,0) and the interior rows -beta*dyu2i(1), 1-beta*(dyu2i(2)+k2x+k2z),
 * -beta*dyu2i(3), for one complex right-hand side on caller-owned device memory, with no
 * context and no allocation.
 *   rhs_dev, u_dev : [nplanes][nkx*n2] complex (interleaved doubles, CFD_LAYOUT_PLANE order);
 *                    they may be the same buffer (an in-place solve)
 *   kx_dev [nkx], kz_dev [n2], dyu2i_dev [nplanes][3] : device arrays
 * Its Thomas scratch is one file-scope device array of CFD_NOALLOC_MAX_SCRATCH doubles
 * (128 MiB) that every GPU loading the library holds until exit; (nplanes-1)*nkx*n2 above
 * that returns CFD_ERR_SIZE before any GPU work.  The first call on a device looks up that
 * device's copy of the array (with the device current) and keeps its address for the life
 * of the process, so make it before any stream capture; after a cudaDeviceReset the
 * library must be unloaded and loaded again before the next call.  All calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race on it and give wrong results.  Nothing in it needs to start at zero.
 * Enqueued on `stream` (NULL = legacy default stream); returns CFD_ERR_CUDA on a launch
 * failure. */
#define CFD_NOALLOC_MAX_SCRATCH (16u * 1024u * 1024u)
int cfd_lusol_u_noalloc(int32_t nkx, int32_t n2, int32_t nplanes, double beta,
                        double gw_bot, double gw_top, const double *kx_dev,
                        const double *kz_dev, const double *dyu2i_dev,
                        const double *rhs_dev, double *u_dev, void *stream);

/* ---- introspection ---------------------------------------------------------------- */

/* Per-kernel timing: while enabled, every kernel launched by a stage entry point (not by
 * a graph replay) is bracketed by CUDA events on the context stream.  cfd_profile_read
 * synchronises and writes one line "name calls total_ms" per kernel into buf (NUL
 * terminated, truncated to buflen) and clears the records. */
int cfd_profile(cfd_ctx *ctx, int32_t enable);
int cfd_profile_read(cfd_ctx *ctx, char *buf, int32_t buflen);

/* Number of kernel launches issued by this context since creation (all entry points). */
int cfd_launch_count(const cfd_ctx *ctx, int64_t *count);
/* Library version string. */
const char *cfd_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CFD_B200_H */
