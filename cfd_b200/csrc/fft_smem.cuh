// fft_smem.cuh - batched mixed-radix (4/2/3) Stockham FFT in shared memory, sm_100a.
//
// Replaces the FFTPACK kernels the reference vendors (cfftf1/cfftb1 + passf*/passb*,
// cft_buff.f:247-274, 693-720, 279-1073): lengths 2^a*3^b, complex, unnormalised.
// One CTA transforms B lines at once; element e of line b sits at buf[e*B + b] so that
// consecutive threads touch consecutive words.  Each radix pass reads one buffer and
// writes the other (autosort, no bit reversal); the caller owns both buffers.
//
// Twiddles are a table tw[m] = exp(-2 pi i m/n), m < n, evaluated once on the host in
// extended precision and rounded to the working type (the FP32 path therefore uses
// correctly-rounded twiddles rather than a recurrence, which would drift as O(n eps)).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace cfd {

template <typename R> struct CxT;
template <> struct CxT<float> { using T = float2; };
template <> struct CxT<double> { using T = double2; };

template <typename T2> __host__ __device__ __forceinline__ T2 cx(decltype(T2::x) a, decltype(T2::x) b) {
    T2 r; r.x = a; r.y = b; return r;
}
template <typename T2> __host__ __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return cx<T2>(a.x + b.x, a.y + b.y); }
template <typename T2> __host__ __device__ __forceinline__ T2 csub(T2 a, T2 b) { return cx<T2>(a.x - b.x, a.y - b.y); }
template <typename T2> __host__ __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    return cx<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T2> __device__ __forceinline__ T2 cmulc(T2 a, T2 b) {
    return cx<T2>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T2> __device__ __forceinline__ T2 cconj(T2 a) { return cx<T2>(a.x, -a.y); }
template <typename T2> __host__ __device__ __forceinline__ T2 cscale(T2 a, decltype(T2::x) s) { return cx<T2>(a.x * s, a.y * s); }
// i * a
template <typename T2> __device__ __forceinline__ T2 cmuli(T2 a) { return cx<T2>(-a.y, a.x); }

// Radix plan of one length (filled on the host).
struct FFTDesc {
    int n;
    int nrad;
    int rad[10];
};

// Shared-memory address of element e of line b in a batch of B = 1 << bshift lines:
// element-major with the line index XOR-swizzled by the low bits of e, so that both
// "consecutive lines, same element" and "consecutive elements, same line" accesses of a
// warp spread over all banks.
__device__ __forceinline__ int swz(int e, int b, int bshift) {
    return (e << bshift) + (b ^ (e & ((1 << bshift) - 1)));
}

// sign = -1: forward (e^{-i..}), +1: inverse.
template <typename T2>
__device__ __forceinline__ void butterfly(T2* v, int R, int sign) {
    using R_t = decltype(T2::x);
    if (R == 2) {
        T2 a0 = cadd(v[0], v[1]), a1 = csub(v[0], v[1]);
        v[0] = a0; v[1] = a1;
    } else if (R == 3) {
        const R_t s3 = (R_t)0.86602540378443864676 * (R_t)sign;
        T2 t1 = cadd(v[1], v[2]);
        T2 t2 = csub(v[0], cscale(t1, (R_t)0.5));
        T2 d = csub(v[1], v[2]);
        T2 t3 = cx<T2>(-s3 * d.y, s3 * d.x);
        v[0] = cadd(v[0], t1);
        v[1] = cadd(t2, t3);
        v[2] = csub(t2, t3);
    } else {
        T2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
        T2 b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
        T2 ib1 = sign < 0 ? cx<T2>(b1.y, -b1.x) : cx<T2>(-b1.y, b1.x);
        v[0] = cadd(a0, b0);
        v[1] = cadd(a1, ib1);
        v[2] = csub(a0, b0);
        v[3] = csub(a1, ib1);
    }
}

// Transform B lines of length d.n held in `a` (layout [e][b]); `b` is scratch of the
// same size.  All threads of the CTA must call it; it ends with __syncthreads() and
// returns the buffer that holds the result.
template <typename T2>
__device__ T2* fft_lines(T2* a, T2* b, int B, const FFTDesc& d, const T2* __restrict__ tw, int sign) {
    T2* in = a;
    T2* out = b;
    const int n = d.n;
    const int bshift = __ffs(B) - 1;  // B is a power of two
    int Ns = 1;
    for (int p = 0; p < d.nrad; ++p) {
        const int R = d.rad[p];
        const int nr = n / R;
        const int tstep = n / (Ns * R);
        const int ntask = nr * B;
        for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
            const int bb = t & (B - 1);
            const int i = t >> bshift;
            const int k = i % Ns;
            T2 v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r < R) {
                    T2 x = in[swz(i + r * nr, bb, bshift)];
                    if (r > 0 && Ns > 1) {
                        const T2 w = tw[r * k * tstep];
                        x = sign < 0 ? cmul(x, w) : cmulc(x, w);
                    }
                    v[r] = x;
                }
            }
            butterfly(v, R, sign);
            const int idxD = (i / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < 4; ++r)
                if (r < R) out[swz(idxD + r * Ns, bb, bshift)] = v[r];
        }
        __syncthreads();
        T2* tmp = in; in = out; out = tmp;
        Ns *= R;
    }
    return in;
}

}  // namespace cfd

// ======================================================================================
// Fixed-length engine for the production lengths (64, 96, 128, 192, 384, 768): the radix
// plan is a compile-time constant (radix 8 first, then 4/6/3), so every index of a pass is
// a constant-folded multiply/shift; the batch count B is a power of two (B = 1 << bshift).
// ======================================================================================
namespace cfd {

template <int N> struct RadixPlan { static constexpr int P = 0; static constexpr int R[1] = {1}; };
template <> struct RadixPlan<64> { static constexpr int P = 2; static constexpr int R[2] = {8, 8}; };
template <> struct RadixPlan<96> { static constexpr int P = 3; static constexpr int R[3] = {8, 4, 3}; };
template <> struct RadixPlan<128> { static constexpr int P = 3; static constexpr int R[3] = {8, 4, 4}; };
template <> struct RadixPlan<192> { static constexpr int P = 3; static constexpr int R[3] = {8, 8, 3}; };
template <> struct RadixPlan<384> { static constexpr int P = 3; static constexpr int R[3] = {8, 8, 6}; };
template <> struct RadixPlan<768> { static constexpr int P = 4; static constexpr int R[4] = {8, 8, 4, 3}; };

template <int N> struct IsFixed { static constexpr bool value = RadixPlan<N>::P > 0; };

// multiply by SIGN*i
template <int SIGN, typename T2> __host__ __device__ __forceinline__ T2 mul_si(T2 a) {
    return SIGN < 0 ? cx<T2>(a.y, -a.x) : cx<T2>(-a.y, a.x);
}

template <int SIGN, typename T2> __host__ __device__ __forceinline__ void dft2(T2& a, T2& b) {
    T2 t = csub(a, b);
    a = cadd(a, b);
    b = t;
}

template <int SIGN, typename T2> __host__ __device__ __forceinline__ void dft3(T2& x0, T2& x1, T2& x2) {
    using R_t = decltype(T2::x);
    const R_t s3 = (R_t)0.86602540378443864676 * (R_t)SIGN;
    T2 t1 = cadd(x1, x2);
    T2 t2 = csub(x0, cscale(t1, (R_t)0.5));
    T2 d = csub(x1, x2);
    T2 t3 = cx<T2>(-s3 * d.y, s3 * d.x);
    x0 = cadd(x0, t1);
    x1 = cadd(t2, t3);
    x2 = csub(t2, t3);
}

template <int SIGN, typename T2> __host__ __device__ __forceinline__ void dft4(T2& x0, T2& x1, T2& x2, T2& x3) {
    T2 a0 = cadd(x0, x2), a1 = csub(x0, x2);
    T2 b0 = cadd(x1, x3), b1 = mul_si<SIGN>(csub(x1, x3));
    x0 = cadd(a0, b0);
    x2 = csub(a0, b0);
    x1 = cadd(a1, b1);
    x3 = csub(a1, b1);
}

// radix-6 = even/odd split into two DFT3: X_k = E_{k%3} + w6^k O_{k%3}
template <int SIGN, typename T2> __host__ __device__ __forceinline__ void dft6(T2* v) {
    using R_t = decltype(T2::x);
    T2 e0 = v[0], e1 = v[2], e2 = v[4], o0 = v[1], o1 = v[3], o2 = v[5];
    dft3<SIGN>(e0, e1, e2);
    dft3<SIGN>(o0, o1, o2);
    const R_t h = (R_t)0.5, s = (R_t)0.86602540378443864676 * (R_t)SIGN;
    const T2 w1 = cx<T2>(h, s), w2 = cx<T2>(-h, s);  // w6^1, w6^2
    const T2 p1 = cmul(o1, w1), p2 = cmul(o2, w2);
    v[0] = cadd(e0, o0); v[3] = csub(e0, o0);
    v[1] = cadd(e1, p1); v[4] = csub(e1, p1);
    v[2] = cadd(e2, p2); v[5] = csub(e2, p2);
}

// radix-8 = even/odd split into two DFT4: X_k = A_{k%4} + w8^k B_{k%4}
template <int SIGN, typename T2> __host__ __device__ __forceinline__ void dft8(T2* v) {
    using R_t = decltype(T2::x);
    T2 a0 = v[0], a1 = v[2], a2 = v[4], a3 = v[6];
    T2 b0 = v[1], b1 = v[3], b2 = v[5], b3 = v[7];
    dft4<SIGN>(a0, a1, a2, a3);
    dft4<SIGN>(b0, b1, b2, b3);
    const R_t r = (R_t)0.70710678118654752440;
    // w8^1 = r(1 + SIGN i), w8^2 = SIGN i, w8^3 = r(-1 + SIGN i)
    const T2 q1 = cmul(b1, cx<T2>(r, (R_t)SIGN * r));
    const T2 q2 = mul_si<SIGN>(b2);
    const T2 q3 = cmul(b3, cx<T2>(-r, (R_t)SIGN * r));
    v[0] = cadd(a0, b0); v[4] = csub(a0, b0);
    v[1] = cadd(a1, q1); v[5] = csub(a1, q1);
    v[2] = cadd(a2, q2); v[6] = csub(a2, q2);
    v[3] = cadd(a3, q3); v[7] = csub(a3, q3);
}

template <int R, int SIGN, typename T2> __device__ __forceinline__ void dftR(T2* v) {
    if constexpr (R == 2) dft2<SIGN>(v[0], v[1]);
    else if constexpr (R == 3) dft3<SIGN>(v[0], v[1], v[2]);
    else if constexpr (R == 4) dft4<SIGN>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 6) dft6<SIGN>(v);
    else dft8<SIGN>(v);
}

// one Stockham pass: B lines at buf[e*B + b], Ns = product of the previous radices
template <typename T2, int N, int PASS, int NS, int SIGN>
__device__ __forceinline__ void fixed_pass(const T2* __restrict__ in, T2* __restrict__ out, int bshift,
                                           const T2* __restrict__ tw) {
    constexpr int R = RadixPlan<N>::R[PASS];
    constexpr int NR = N / R;
    constexpr int TSTEP = N / (NS * R);
    const int B = 1 << bshift;
    const int ntask = NR << bshift;
    for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
        const int bb = t & (B - 1);
        const int i = t >> bshift;
        const int k = i % NS;
        T2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[swz(i + r * NR, bb, bshift)];
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) {
                const T2 w = tw[r * k * TSTEP];
                v[r] = SIGN < 0 ? cmul(v[r], w) : cmulc(v[r], w);
            }
        }
        dftR<R, SIGN>(v);
        const int idxD = (i / NS) * NS * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[swz(idxD + r * NS, bb, bshift)] = v[r];
    }
    __syncthreads();
}

template <typename T2, int N, int PASS, int NS, int SIGN>
__device__ __forceinline__ T2* fixed_passes(T2* a, T2* b, int bshift, const T2* tw) {
    if constexpr (PASS == RadixPlan<N>::P) {
        return a;
    } else {
        fixed_pass<T2, N, PASS, NS, SIGN>(a, b, bshift, tw);
        return fixed_passes<T2, N, PASS + 1, NS * RadixPlan<N>::R[PASS], SIGN>(b, a, bshift, tw);
    }
}

// Batched transform dispatch: NF = 0 uses the runtime plan `d` (any 2^a*3^b), otherwise
// the fixed engine for length NF (B must then be a power of two, B = 1 << bshift).
template <typename T2, int NF, int SIGN>
__device__ __forceinline__ T2* fft_batch(T2* a, T2* b, int B, int bshift, const FFTDesc& d, const T2* tw) {
    if constexpr (NF == 0) {
        (void)bshift;
        return fft_lines<T2>(a, b, B, d, tw, SIGN);
    } else {
        (void)d;
        (void)B;
        return fixed_passes<T2, NF, 0, 1, SIGN>(a, b, bshift, tw);
    }
}

}  // namespace cfd
