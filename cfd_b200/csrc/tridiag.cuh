// tridiag.cuh - warp-cooperative tridiagonal substitutions (sm_100a).
//
// The reference solves each (kx,kz) column with a sequential Thomas algorithm: LU_dec
// (tridLU_3D_IB.f90:521-559) stores the pivot d_j and the scaled upper diagonal e_j of every
// row, LUsolU/V/P (:50-160, :284-318) run the substitutions
//   y_j = d_j (r_j - a1_j y_{j-1})      forward, affine in y_{j-1}
//   x_j = y_j - e_j x_{j+1}             backward, affine in x_{j+1}
// Here one warp solves one column: lane p owns the m consecutive rows [p*m, p*m + m).  The
// pivot recurrence e_j = a3_j / (a2_j - a1_j e_{j-1}) is a linear fractional map of e_{j-1}:
// the lanes compose their rows' maps, a warp scan hands every lane its incoming e, and each
// lane replays its rows with d_j = 1 / (a2_j - a1_j e_{j-1}).  The two substitutions are
// affine maps, composed and scanned the same way, then replayed with the reference's
// formulas.  The column stays in the warp, so the right-hand side is read once and the
// solution written once; only the grouping of the chained maps differs from the sequential
// sweep, so results agree to round-off.
#pragma once

#include <cuda_runtime.h>

namespace cfd {

__device__ __forceinline__ double shfl_up_d(double v, int off) { return __shfl_up_sync(0xffffffffu, v, off); }
__device__ __forceinline__ double shfl_dn_d(double v, int off) { return __shfl_down_sync(0xffffffffu, v, off); }

// rows of one lane for an n-row system spread over the 32 lanes
struct LaneRows {
    int s, mp;
};
__device__ __forceinline__ LaneRows lane_rows(int n, int lane) {
    const int m = (n + 31) >> 5;
    const int s = lane * m;
    return LaneRows{s, max(0, min(m, n - s))};
}

// Substitutions of one column: y[t] holds the lane's right-hand side on entry and the
// solution on exit; dd[t] are the pivots d of the lane's rows, a1(t) their sub-diagonal and
// e(t) their scaled upper diagonal.
template <int MAXM, typename A1F, typename EF>
__device__ __forceinline__ void warp_substitute(const LaneRows& lr, int lane, const double (&dd)[MAXM], A1F a1,
                                                EF e, double2 (&y)[MAXM]) {
    double A = 1.0;  // y_last = A * y_in + B over the lane's rows
    double2 B = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < MAXM; ++t)
        if (t < lr.mp) {
            const double dj = dd[t], al = -a1(t) * dj;
            B = make_double2(al * B.x + dj * y[t].x, al * B.y + dj * y[t].y);
            A *= al;
        }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double oA = shfl_up_d(A, off), oBx = shfl_up_d(B.x, off), oBy = shfl_up_d(B.y, off);
        if (lane >= off) {
            B = make_double2(A * oBx + B.x, A * oBy + B.y);
            A *= oA;
        }
    }
    double2 yp = make_double2(shfl_up_d(B.x, 1), shfl_up_d(B.y, 1));
    if (lane == 0) yp = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < MAXM; ++t)
        if (t < lr.mp) {
            const double dj = dd[t];
            const double a = a1(t);
            y[t] = make_double2(dj * (y[t].x - a * yp.x), dj * (y[t].y - a * yp.y));
            yp = y[t];
        }
    double G = 1.0;  // x_first = G * x_next + H over the lane's rows
    double2 H = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = MAXM - 1; t >= 0; --t)
        if (t < lr.mp) {
            const double et = e(t);
            H = make_double2(y[t].x - et * H.x, y[t].y - et * H.y);
            G *= -et;
        }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double oG = shfl_dn_d(G, off), oHx = shfl_dn_d(H.x, off), oHy = shfl_dn_d(H.y, off);
        if (lane + off < 32) {
            H = make_double2(G * oHx + H.x, G * oHy + H.y);
            G *= oG;
        }
    }
    double2 xn = make_double2(shfl_dn_d(H.x, 1), shfl_dn_d(H.y, 1));
    if (lane == 31) xn = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = MAXM - 1; t >= 0; --t)
        if (t < lr.mp) {
            const double et = e(t);
            y[t] = make_double2(y[t].x - et * xn.x, y[t].y - et * xn.y);
            xn = y[t];
        }
}

// Linear fractional maps x -> (a x + b) / (c x + d) as 2x2 matrices.  Only the ratios
// matter, so products are rescaled by a power of two (exact) to keep the entries near 1.
struct Mob {
    double a, b, c, d;
};
__device__ __forceinline__ Mob mob_identity() { return Mob{1.0, 0.0, 0.0, 1.0}; }
// x after y
__device__ __forceinline__ Mob mob_mul(const Mob& x, const Mob& y) {
    return Mob{x.a * y.a + x.b * y.c, x.a * y.b + x.b * y.d, x.c * y.a + x.d * y.c, x.c * y.b + x.d * y.d};
}
__device__ __forceinline__ Mob mob_norm(const Mob& m) {
    const double mx = fmax(fmax(fabs(m.a), fabs(m.b)), fmax(fabs(m.c), fabs(m.d)));
    // 2^-(E - 1023) for the biased exponent E of mx (a normal number): biased 2046 - E
    const long long eb = (__double_as_longlong(mx) >> 52) & 0x7ff;
    const double s = __longlong_as_double((2046 - eb) << 52);
    return Mob{m.a * s, m.b * s, m.c * s, m.d * s};
}
// composition of the maps of all lanes below this one (lane 0: identity)
__device__ __forceinline__ Mob mob_scan_exclusive(Mob P, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Mob O{shfl_up_d(P.a, off), shfl_up_d(P.b, off), shfl_up_d(P.c, off), shfl_up_d(P.d, off)};
        if (lane >= off) P = mob_norm(mob_mul(P, O));
    }
    Mob E{shfl_up_d(P.a, 1), shfl_up_d(P.b, 1), shfl_up_d(P.c, 1), shfl_up_d(P.d, 1)};
    return lane == 0 ? mob_identity() : E;
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

}  // namespace cfd
