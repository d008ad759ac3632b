// tridiag.cuh - warp-cooperative tridiagonal substitutions (sm_100a).
//
// The reference solves each (kx,kz) column with a sequential Thomas algorithm: LU_dec
// (tridLU_3D_IB.f90:521-559) stores the pivot d_j and the scaled upper diagonal e_j of every
// row, LUsolU/V/P (:50-160, :284-318) run the substitutions
//   y_j = d_j (r_j - a1_j y_{j-1})      forward, affine in y_{j-1}
//   x_j = y_j - e_j x_{j+1}             backward, affine in x_{j+1}
// Here the factors are computed once per time step size (they depend on kx, kz, the y-grid
// and the RK coefficient only) and stored column-major, and one warp substitutes one column:
// lane p owns the m consecutive rows [p*m, p*m + m), composes the affine maps of its rows,
// a warp scan hands every lane its incoming value, and the lane replays its rows with the
// reference's formulas.  The column stays in registers, so the right-hand side is read once
// and the solution written once; only the grouping of the chained maps differs from the
// sequential sweep, so results agree to round-off.
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
// solution on exit; ed[t] = {e, d} of the lane's rows, a1(t) their sub-diagonal.
template <int MAXM, typename A1F>
__device__ __forceinline__ void warp_substitute(const LaneRows& lr, int lane, const double2 (&ed)[MAXM], A1F a1,
                                                double2 (&y)[MAXM]) {
    double A = 1.0;  // y_last = A * y_in + B over the lane's rows
    double2 B = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = 0; t < MAXM; ++t)
        if (t < lr.mp) {
            const double dj = ed[t].y, al = -a1(t) * dj;
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
            const double dj = ed[t].y;
            const double a = a1(t);
            y[t] = make_double2(dj * (y[t].x - a * yp.x), dj * (y[t].y - a * yp.y));
            yp = y[t];
        }
    double G = 1.0;  // x_first = G * x_next + H over the lane's rows
    double2 H = make_double2(0.0, 0.0);
#pragma unroll
    for (int t = MAXM - 1; t >= 0; --t)
        if (t < lr.mp) {
            H = make_double2(y[t].x - ed[t].x * H.x, y[t].y - ed[t].x * H.y);
            G *= -ed[t].x;
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
            y[t] = make_double2(y[t].x - ed[t].x * xn.x, y[t].y - ed[t].x * xn.y);
            xn = y[t];
        }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace cfd
