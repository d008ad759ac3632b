// xmarch.cuh - the x-line pass of the nonlinear term marching in y (x-line path 6, FP32).
//
// The products of ops_in_planes (FOU3D.f90:1529-1617) need, on every u-plane, u and w and v
// interpolated to the centre, and on every v-plane, v and u, w interpolated to the face
// (interp_u/interp_v, FOU3D.f90:261-308).  The per-slot kernels (k_xline2) transform the
// interpolated spectra, i.e. four inverse lines per row of a u-plane/v-plane pair.  The
// interpolation is linear in y and commutes with the x transform, so here a CTA holds a
// pair of z-rows and walks up the channel: each step transforms u, w of u-plane t and v of
// v-plane t once (1.5 complex lines per row), keeps the previous step's physical values in
// shared memory, and forms the products of u-plane t and v-plane t-1 from the two steps'
// values in physical space: 1.5 inverse + 3 forward complex lines per row and step instead
// of 4 + 3, and each spectral plane is read once.
//
// Lines of a row pair (rows r, r+1) and their lanes:
//   inverse: A = u_r + i v_r, B = u_r+1 + i v_r+1, C = w_r + i w_r+1
//   forward: A: (uu + i vv)_r [u-plane t], (uv + i vw)_r [v-plane t-1]; B: the same on r+1;
//            C: (ww_r + i ww_r+1), (uw_r + i uw_r+1) [u-plane t]
// In the physical phase the three lanes of a (pair, k1) triple are adjacent (10 triples per
// warp, lanes 30 and 31 idle) and pass u (A, B -> C) and the face value of w (C -> A, B)
// with two shuffles, so every lane runs two forward lines, as one packed-pair transform
// (fft_pair.cuh: each .f32x2 instruction serves both lines).  The forward N1-point step holds
// X[kb + N2 ka] in registers; the unpack of the two real spectra pairs X_k with X_N-k, which
// lane N2 - kb of the same warp holds (N2 divides 32), so it needs no shared memory.
//
// Sequence of a CTA over emission steps t = ta..tb-1 (u-plane t and v-plane t-1):
//   chunk 0: step "0a" (u-plane 0 with v interpolated to its ghost centre in spectral space,
//            u-plane lines only), step 0 (fills the history), then t = 1..tb-1
//   chunk c: step ta-1 (fills the history), then t = ta..tb-1
// The top u-plane (t = nyu-1) is transformed with v interpolated to its ghost centre in
// spectral space, since no v-plane t exists; the weights are those of the per-slot kernels.
#pragma once

#include <type_traits>

#include "fft_reg.cuh"
#include "fft_pair.cuh"
#include "xmarch_plan.cuh"

namespace cfd {

template <typename T2, int N1, int N2>
__global__ void __launch_bounds__(256) k_xmarch(Dims d, Geo g, const T2* __restrict__ Hx, T2* __restrict__ H0,
                                                 T2* __restrict__ H1, T2* __restrict__ H2, T2* __restrict__ H3,
                                                 const T2* __restrict__ twx, int RW, int csteps) {
    using R = decltype(T2::x);
    static_assert(N2 == 8 || N2 == 16, "the shuffle unpack pairs lanes kb and N2-kb inside a warp");
    static_assert(std::is_same<T2, float2>::value, "FP32 only: the forward step runs on packed FP32 pairs");
    constexpr int N = N1 * N2;
    constexpr int HX = N / 3;               // highest retained kx
    constexpr int NK = HX + 1;              // kx columns per row
    constexpr int L1 = xmarch_l1(N1, N2);  // inverse exchange per line: [k1][n2]
    constexpr int L2 = xmarch_l2(N1, N2);  // forward exchange per line: [kb][na]
    constexpr int TP = N2 + 1;              // twiddle row pitch
    constexpr int KA = HX / N2 + 1;         // output blocks ka holding some k <= HX
    const int NT = blockDim.x;
    const int pairs = RW >> 1;
    const int NLI = 3 * pairs, NLF = 6 * pairs;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T2* exi = reinterpret_cast<T2*>(smem_raw);
    T2* exf = exi + (size_t)NLI * L1;
    T2* hist = exf + (size_t)NLF * L2;      // hist[k2 * NT + thread]
    T2* twt = hist + (size_t)N2 * NT;       // twt[b * TP + a] = w^(a*b)
    const int t = threadIdx.x;
    for (int i = t; i < N; i += NT) {
        const int b = i / N2, a = i - b * N2;
        twt[b * TP + a] = twx[(a * b) % N];
    }
    for (int i = t; i < N2 * NT; i += NT) hist[i] = cx<T2>((R)0, (R)0);

    const int z0 = blockIdx.x * RW;
    const size_t pls = (size_t)d.ngal2 * NK;
    const T2* Hu = Hx;
    const T2* Hw = Hx + (size_t)d.nyu * pls;
    const T2* Hv = Hx + (size_t)(2 * d.nyu) * pls;
    int it0, ta, tb;
    xmarch_chunk(blockIdx.y, csteps, d.nyu, it0, ta, tb);

    // thread roles of step 1 (line b1, column n2), the physical phase (lane triples) and
    // step 2' (forward line bf, column kb)
    const XMRoles ro = xmarch_roles(t, RW, N1, N2);
    const bool act1 = ro.act1, act2 = ro.act2, act3 = ro.act3;
    const int b1 = ro.b1, n2 = ro.n2, p1 = ro.p1, role1 = ro.role1;
    const int role = ro.role, p2 = ro.p2, k1 = ro.k1, b2 = ro.b2, src1 = ro.src1, src2 = ro.src2;
    const bool isA = role == 0, isC = role == 2;
    const int kb = ro.kb, bfc = ro.bfc, partner = ro.partner, p3 = ro.p3, role3 = ro.role3, j3 = ro.j3;
    __syncthreads();

    for (int it = it0; it < tb; ++it) {
        // ---- step parameters (uniform over the CTA)
        const XMStep sp = xmarch_step(it, ta, d.nyu);
        const bool emit = sp.emit, emit_v = sp.emit_v, combo = sp.combo != 0;
        const int tu = sp.tu, va = sp.va, vb = sp.vb;
        R ca = 1, cb = 0, pa = 1, pb = 0, fa = 0, fb = 0;
        if (sp.combo < 0) {  // u-plane 0: v at the bottom ghost centre
            ca = (R)((1.0 - g.gwib) * g.vca[1]);
            cb = (R)(g.gwib + (1.0 - g.gwib) * g.vcb[1]);
        } else if (sp.combo > 0) {  // u-plane nyu-1: v at the top ghost centre
            ca = (R)(g.gwit + (1.0 - g.gwit) * g.vca[it - 1]);
            cb = (R)((1.0 - g.gwit) * g.vcb[it - 1]);
        }
        if (emit_v) {
            fa = (R)g.ufa[tu - 1];
            fb = (R)g.ufb[tu - 1];
        }
        if (sp.vc >= 0) { pa = (R)g.vca[sp.vc]; pb = (R)g.vcb[sp.vc]; }

        // ---- step 1: inverse N1-point DFTs of the Hermitian-extended spectra, thread (b1, n2)
        if (act1) {
            const T2 *A0, *C0, *C1;
            bool cmb = false;
            if (role1 == 2) {
                A0 = Hw + tu * pls + (size_t)(z0 + 2 * p1) * NK;
                C0 = A0 + NK;
                C1 = C0;
            } else {
                const size_t ro = (size_t)(z0 + 2 * p1 + role1) * NK;
                A0 = Hu + tu * pls + ro;
                C0 = Hv + va * pls + ro;
                C1 = Hv + vb * pls + ro;
                cmb = combo;
            }
            T2 v[N1];
            auto fill = [&](auto cm) {
                constexpr bool CM = decltype(cm)::value;
                auto fetch = [&](int k, T2& a, T2& c) {
                    a = A0[k];
                    if (CM) {
                        const T2 c0 = C0[k], c1 = C1[k];
                        c = cx<T2>(ca * c0.x + cb * c1.x, ca * c0.y + cb * c1.y);
                    } else {
                        c = C0[k];
                    }
                };
#pragma unroll
                for (int n1 = 0; n1 < N1; ++n1) {
                    const int e0 = n1 * N2, e = e0 + n2;
                    const bool lo = (e0 + N2 - 1 <= HX) || (e0 <= HX && e <= HX);
                    const bool hi = (e0 >= N - HX) || (e0 + N2 - 1 >= N - HX && e >= N - HX);
                    T2 val = cx<T2>((R)0, (R)0);
                    T2 a, c;
                    if (lo) {  // A_e + i C_e; the inverse real transform ignores Im of kx = 0
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
            if (cmb) fill(std::true_type{});
            else fill(std::false_type{});
            rdft_z<N1, +1, gap_blocks<N1, N2, HX>()>(v);
            T2* o = exi + (size_t)b1 * L1 + n2;
#pragma unroll
            for (int q = 0; q < N1; ++q) o[q * (N2 + 1)] = q == 0 ? v[0] : cmulc(v[q], twt[q * TP + n2]);
        }
        __syncthreads();

        // ---- step 2: inverse N2-point DFT -> physical x = k1 + N1*k2; products with the
        // previous step's values; the forward N2-point DFT of the lane's two output lines, la
        // and lb, as one transform on packed FP32 pairs
        {
            T2 y[N2];
            const T2* o = exi + (size_t)b2 * L1 + k1 * (N2 + 1);
#pragma unroll
            for (int q = 0; q < N2; ++q) y[q] = o[q];
            rdft<N2, +1>(y);
            if (!emit) {
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) hist[k2 * NT + t] = y[k2];
            } else {
                cpair P[N2];  // the lane's two forward lines: x = (Re la, Re lb), y = (Im la, Im lb)
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) {
                    const T2 h = hist[k2 * NT + t];
                    hist[k2 * NT + t] = y[k2];
                    // A/B: f = u at the face of v-plane t-1; C: f, f2 = w, w' at that face
                    const R f = fa * y[k2].x + fb * h.x, f2 = fa * y[k2].y + fb * h.y;
                    const R r1 = __shfl_sync(0xffffffffu, isC ? f : y[k2].x, src1);
                    const R r2 = __shfl_sync(0xffffffffu, isC ? f2 : y[k2].x, src2);
                    // la: A/B (u u, vc vc) with vc = pa v + pb v(t-1); C (w w, w' w')
                    const R x2 = isC ? y[k2].y : pa * y[k2].y + pb * h.y;
                    // lb: A/B (uf v(t-1), v(t-1) wf); C (u w, u' w')
                    const R lbx = (isC ? r1 : f) * (isC ? y[k2].x : h.y);
                    const R lby = (isC ? r2 : h.y) * (isC ? y[k2].y : (isA ? r1 : r2));
                    P[k2] = cpair{f2p(y[k2].x * y[k2].x, lbx), f2p(x2 * x2, lby)};
                }
                rdft<N2, -1>(P);
                if (act2) {
                    T2* oa = exf + (size_t)(6 * p2 + 2 * role) * L2 + k1;
                    T2* ob = oa + L2;
#pragma unroll
                    for (int q = 0; q < N2; ++q) {
                        cpair v = P[q];
                        if (q > 0) {
                            const T2 w = twt[k1 * TP + q];
                            v = cmul(v, cpair{f2b(w.x), f2b(w.y)});
                        }
                        oa[q * (N1 + 1)] = cx<T2>(v.x.v.x, v.y.v.x);
                        ob[q * (N1 + 1)] = cx<T2>(v.x.v.y, v.y.v.y);
                    }
                }
            }
        }
        __syncthreads();

        // ---- step 2': forward N1-point DFT, thread (bf, kb) -> X[kb + N2*ka]; unpack
        // A_k = (P_k + conj P_N-k)/2, B_k = (P_k - conj P_N-k)/(2i), x 1/N, with P_N-k from
        // lane N2 - kb; stores of k <= HX
        if (emit) {
            T2 z[N1];
            const T2* o = exf + (size_t)bfc * L2 + kb * (N1 + 1);
#pragma unroll
            for (int q = 0; q < N1; ++q) z[q] = o[q];
            rdft<N1, -1>(z);
            const size_t ub = (size_t)tu * d.ngal2 * NK;
            const size_t vsb = (size_t)(d.nyu + tu - 1) * d.ngal2 * NK;
            T2 *da = nullptr, *db = nullptr;
            if (role3 < 2) {
                const size_t ro = (size_t)(z0 + 2 * p3 + role3) * NK;
                if (j3 == 0) { da = H0 + ub + ro; db = H2 + ub + ro; }
                else if (emit_v) { da = H0 + vsb + ro; db = H1 + vsb + ro; }
            } else {
                const size_t ro = (size_t)(z0 + 2 * p3) * NK;
                T2* hh = j3 == 0 ? H3 : H1;
                da = hh + ub + ro;
                db = da + NK;
            }
            const R hs = (R)0.5 / (R)N;
#pragma unroll
            for (int ka = 0; ka < KA; ++ka) {
                const T2 zs = z[N1 - 1 - ka];
                T2 q = cx<T2>(__shfl_sync(0xffffffffu, zs.x, partner), __shfl_sync(0xffffffffu, zs.y, partner));
                if (kb == 0) q = z[(N1 - ka) % N1];
                const int k = kb + N2 * ka;
                if (act3 && da != nullptr && k <= HX) {
                    const T2 Pk = z[ka];
                    const T2 Qc = cconj(q);
                    da[k] = cx<T2>((Pk.x + Qc.x) * hs, (Pk.y + Qc.y) * hs);
                    db[k] = cx<T2>((Pk.y - Qc.y) * hs, -(Pk.x - Qc.x) * hs);
                }
            }
        }
    }
}

}  // namespace cfd
