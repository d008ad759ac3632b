// fft_reg.cuh - register-resident DFTs of compile-time length and the two-step transform
// of B lines of length N = N1*N2 across a CTA (sm_100a).
//
// A length-N transform is split as X[k1 + N1 k2] = sum_{n2} w_N^{n2 k1} w_N2^{n2 k2}
// sum_{n1} x[n1 N2 + n2] w_N1^{n1 k1}: a thread first transforms one stride-N2 subsequence
// (N1 points) in registers, multiplies by w_N^{n2 k1}, exchanges once through padded shared
// memory, and a second thread transforms N2 points in registers.  Compared with a
// radix-by-radix Stockham this touches shared memory once per element instead of once per
// pass and spends almost no integer instructions on addressing: every register index is a
// compile-time constant.
//
// Twiddles inside a register DFT are compile-time constants (exact at multiples of pi/4,
// otherwise a 10-term Taylor series on |x| <= pi/4, i.e. correctly rounded to double).
#pragma once

#include "fft_smem.cuh"

namespace cfd {

__host__ __device__ constexpr double k_poly_sin(double x) {
    double x2 = x * x, t = x, s = x;
    for (int i = 1; i <= 11; ++i) {
        t *= -x2 / (double)((2 * i) * (2 * i + 1));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double k_poly_cos(double x) {
    double x2 = x * x, t = 1.0, s = 1.0;
    for (int i = 1; i <= 11; ++i) {
        t *= -x2 / (double)((2 * i - 1) * (2 * i));
        s += t;
    }
    return s;
}
// cos and sin of 2*pi*m/n
__host__ __device__ constexpr double k_tw_c(int m, int n) {
    m = ((m % n) + n) % n;
    const int qd = (4 * m) / n;         // quadrant
    const int num = 4 * m - qd * n;     // alpha = (pi/2) num/n in [0, pi/2)
    const double a = 1.5707963267948966192 * ((double)num / (double)n);
    double c0 = 0, s0 = 0;
    if (2 * num <= n) { c0 = k_poly_cos(a); s0 = k_poly_sin(a); }
    else { const double b = 1.5707963267948966192 * ((double)(n - num) / (double)n); c0 = k_poly_sin(b); s0 = k_poly_cos(b); }
    return qd == 0 ? c0 : (qd == 1 ? -s0 : (qd == 2 ? -c0 : s0));
}
__host__ __device__ constexpr double k_tw_s(int m, int n) {
    m = ((m % n) + n) % n;
    const int qd = (4 * m) / n;
    const int num = 4 * m - qd * n;
    const double a = 1.5707963267948966192 * ((double)num / (double)n);
    double c0 = 0, s0 = 0;
    if (2 * num <= n) { c0 = k_poly_cos(a); s0 = k_poly_sin(a); }
    else { const double b = 1.5707963267948966192 * ((double)(n - num) / (double)n); c0 = k_poly_sin(b); s0 = k_poly_cos(b); }
    return qd == 0 ? s0 : (qd == 1 ? c0 : (qd == 2 ? -s0 : -c0));
}

// w_N^m = exp(SIGN 2 pi i m / N) as a compile-time constant
template <int M, int N, int SIGN> struct TwC {
    static constexpr double c = k_tw_c(M, N);
    static constexpr double s = (double)SIGN * k_tw_s(M, N);
    static constexpr bool one = (M % N) == 0;
};

// multiplication by the compile-time twiddle TW (overloaded for packed line pairs)
template <typename TW, typename T2> __host__ __device__ __forceinline__ T2 cmul_k(T2 v) {
    using R = decltype(T2::x);
    constexpr R c = (R)TW::c, s = (R)TW::s;
    return cx<T2>(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <typename T2, int M, int N, int SIGN>
__host__ __device__ __forceinline__ T2 twmul(T2 v) {
    if constexpr (TwC<M, N, SIGN>::one) {
        return v;
    } else {
        return cmul_k<TwC<M, N, SIGN>>(v);
    }
}

template <int N> struct FirstFactor {
    static constexpr int value = (N % 4 == 0 && N > 4) ? 4 : ((N % 3 == 0 && N > 3) ? 3 : ((N % 2 == 0 && N > 2) ? 2 : N));
};

template <int N, int SIGN, typename T2> __host__ __device__ __forceinline__ void rdft(T2* v);

// one column of the composite step: DFT_P of v[Q*n1 + n2] (n1 = 0..P-1), twiddled, into y
template <int P, int Q, int N2I, int SIGN, typename T2>
__host__ __device__ __forceinline__ void rdft_col(const T2* v, T2* y) {
    T2 t[P];
#pragma unroll
    for (int n1 = 0; n1 < P; ++n1) t[n1] = v[Q * n1 + N2I];
    rdft<P, SIGN>(t);
    y[N2I * P + 0] = t[0];
    if constexpr (P > 1) y[N2I * P + 1] = twmul<T2, N2I * 1, P * Q, SIGN>(t[1]);
    if constexpr (P > 2) y[N2I * P + 2] = twmul<T2, N2I * 2, P * Q, SIGN>(t[2]);
    if constexpr (P > 3) y[N2I * P + 3] = twmul<T2, N2I * 3, P * Q, SIGN>(t[3]);
}

template <int P, int Q, int N2I, int SIGN, typename T2>
__host__ __device__ __forceinline__ void rdft_cols(const T2* v, T2* y) {
    if constexpr (N2I < Q) {
        rdft_col<P, Q, N2I, SIGN>(v, y);
        rdft_cols<P, Q, N2I + 1, SIGN>(v, y);
    }
}

// in-place DFT of N registers, natural order in and out
template <int N, int SIGN, typename T2> __host__ __device__ __forceinline__ void rdft(T2* v) {
    if constexpr (N == 1) {
    } else if constexpr (N == 2) {
        dft2<SIGN>(v[0], v[1]);
    } else if constexpr (N == 3) {
        dft3<SIGN>(v[0], v[1], v[2]);
    } else if constexpr (N == 4) {
        dft4<SIGN>(v[0], v[1], v[2], v[3]);
    } else {
        constexpr int P = FirstFactor<N>::value;  // P <= 4
        constexpr int Q = N / P;
        T2 y[N];
        rdft_cols<P, Q, 0, SIGN>(v, y);  // y[n2*P + k1]
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            T2 t[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) t[n2] = y[n2 * P + k1];
            rdft<Q, SIGN>(t);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = t[k2];
        }
    }
}

// ---- inputs known to be zero --------------------------------------------------------
// The zero-padded inverse transforms get whole stride-N2 subsequences of zeros (the
// dealiasing gap).  IEEE rules keep the compiler from dropping x + 0.0, so the first
// radix-4 stage below skips the additions with inputs flagged in a compile-time mask.  Its
// values equal rdft's, except that a zero may keep a negative sign that rdft's x + 0 would
// have made positive (checked on the host for every production length by
// tests/fft_prune_check.cu).
template <int SIGN, int ZM, typename T2>
__host__ __device__ __forceinline__ void dft4_z(T2& x0, T2& x1, T2& x2, T2& x3) {
    if constexpr (ZM == 0) {
        dft4<SIGN>(x0, x1, x2, x3);
    } else {
        auto neg = [](T2 a) { return cx<T2>(-a.x, -a.y); };
        T2 a0, a1, b0, d;
        if constexpr ((ZM & 4) != 0) { a0 = x0; a1 = x0; }
        else if constexpr ((ZM & 1) != 0) { a0 = x2; a1 = neg(x2); }
        else { a0 = cadd(x0, x2); a1 = csub(x0, x2); }
        if constexpr ((ZM & 8) != 0) { b0 = x1; d = x1; }
        else if constexpr ((ZM & 2) != 0) { b0 = x3; d = neg(x3); }
        else { b0 = cadd(x1, x3); d = csub(x1, x3); }
        const T2 b1 = mul_si<SIGN>(d);
        x0 = cadd(a0, b0);
        x2 = csub(a0, b0);
        x1 = cadd(a1, b1);
        x3 = csub(a1, b1);
    }
}

template <int Q, int N2I, int SIGN, unsigned long long ZM, typename T2>
__host__ __device__ __forceinline__ void rdft_cols_z(const T2* v, T2* y) {
    if constexpr (N2I < Q) {
        constexpr int m = (int)(((ZM >> N2I) & 1) | (((ZM >> (Q + N2I)) & 1) << 1) |
                                (((ZM >> (2 * Q + N2I)) & 1) << 2) | (((ZM >> (3 * Q + N2I)) & 1) << 3));
        T2 t0 = v[N2I], t1 = v[Q + N2I], t2 = v[2 * Q + N2I], t3 = v[3 * Q + N2I];
        dft4_z<SIGN, m>(t0, t1, t2, t3);
        y[N2I * 4 + 0] = t0;
        y[N2I * 4 + 1] = twmul<T2, N2I * 1, 4 * Q, SIGN>(t1);
        y[N2I * 4 + 2] = twmul<T2, N2I * 2, 4 * Q, SIGN>(t2);
        y[N2I * 4 + 3] = twmul<T2, N2I * 3, 4 * Q, SIGN>(t3);
        rdft_cols_z<Q, N2I + 1, SIGN, ZM>(v, y);
    }
}

// rdft<N, SIGN> for inputs whose zeros are flagged in ZM (bit n: v[n] == 0)
template <int N, int SIGN, unsigned long long ZM, typename T2>
__host__ __device__ __forceinline__ void rdft_z(T2* v) {
    if constexpr (ZM == 0 || N <= 4 || FirstFactor<N>::value != 4) {
        rdft<N, SIGN>(v);
    } else {
        constexpr int P = 4, Q = N / 4;
        T2 y[N];
        rdft_cols_z<Q, 0, SIGN, ZM>(v, y);  // y[n2*P + k1], as rdft_cols
#pragma unroll
        for (int k1 = 0; k1 < P; ++k1) {
            T2 t[Q];
#pragma unroll
            for (int n2 = 0; n2 < Q; ++n2) t[n2] = y[n2 * P + k1];
            rdft<Q, SIGN>(t);
#pragma unroll
            for (int k2 = 0; k2 < Q; ++k2) v[k1 + P * k2] = t[k2];
        }
    }
}

// stride-N2 subsequences n1 (elements n1*N2 .. n1*N2+N2-1) wholly inside the gap between
// the retained modes 0..HX and N-HX..N-1
template <int N1, int N2, int HX>
__host__ __device__ constexpr unsigned long long gap_blocks() {
    unsigned long long m = 0;
    for (int n1 = 0; n1 < N1; ++n1)
        if (n1 * N2 > HX && n1 * N2 + N2 - 1 < N1 * N2 - HX) m |= 1ull << n1;
    return m;
}

// (N1, N2) split of the production lengths
template <int N> struct TwoStep { static constexpr int N1 = 0, N2 = 0; };
template <> struct TwoStep<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct TwoStep<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct TwoStep<128> { static constexpr int N1 = 8, N2 = 16; };
template <> struct TwoStep<192> { static constexpr int N1 = 16, N2 = 12; };
template <> struct TwoStep<384> { static constexpr int N1 = 16, N2 = 24; };
template <> struct TwoStep<768> { static constexpr int N1 = 32, N2 = 24; };

// Two-step transform of `nl` lines (nl = 1 << lb) of length N = TN1*TN2 across the CTA.
// Line b, element e: load(e, b) supplies the input, store(e, b, v) receives the output in
// natural order.  Threads map line-fastest in both steps (b = t & (nl-1)), so global
// loads/stores of kx-columns stay coalesced; the exchange rows are an odd number of
// elements apart, which keeps a warp's shared accesses at the minimum wavefront count for
// 16 FP32 lines or 8 FP64 lines.  `ex` holds nl * exch_elems<TN1,TN2>() elements; `twt` is
// the table twt[b*TN2 + a] = w^(a*b) (forward sign).  Ends with __syncthreads().
template <int TN1, int TN2> __host__ __device__ constexpr int exch_row() { return (TN1 * (TN2 + 1)) | 1; }

// BFAST = false maps threads element-fastest instead (n2, then k1, vary fastest), for
// lines that are contiguous in global memory (x-lines); nl need not be a power of two then.
template <typename T2, int TN1, int TN2, int SIGN, bool BFAST = true, typename LoadF, typename StoreF>
__device__ __forceinline__ void two_step_lines(int lb, T2* ex, const T2* twt, LoadF load, StoreF store, int nlines = 0) {
    constexpr int L1 = exch_row<TN1, TN2>();
    const int nl = BFAST ? (1 << lb) : nlines;
    const int t = threadIdx.x;
    if (t < TN2 * nl) {
        const int b = BFAST ? (t & (nl - 1)) : t / TN2;
        const int n2 = BFAST ? (t >> lb) : t - b * TN2;
        T2 v[TN1];
#pragma unroll
        for (int n1 = 0; n1 < TN1; ++n1) v[n1] = load(n1 * TN2 + n2, b);
        rdft<TN1, SIGN>(v);
        T2* o = ex + (size_t)b * L1 + n2;
#pragma unroll
        for (int k1 = 0; k1 < TN1; ++k1) {
            const T2 w = twt[k1 * TN2 + n2];
            o[k1 * (TN2 + 1)] = k1 == 0 ? v[0] : (SIGN < 0 ? cmul(v[k1], w) : cmulc(v[k1], w));
        }
    }
    __syncthreads();
    if (t < TN1 * nl) {
        const int b = BFAST ? (t & (nl - 1)) : t / TN1;
        const int k1 = BFAST ? (t >> lb) : t - b * TN1;
        T2 y[TN2];
        const T2* o = ex + (size_t)b * L1 + k1 * (TN2 + 1);
#pragma unroll
        for (int n2 = 0; n2 < TN2; ++n2) y[n2] = o[n2];
        rdft<TN2, SIGN>(y);
#pragma unroll
        for (int k2 = 0; k2 < TN2; ++k2) store(k1 + TN1 * k2, b, y[k2]);
    }
    __syncthreads();
}

template <typename T2, int TN1, int TN2>
__device__ __forceinline__ void load_twiddles(T2* twt, const T2* __restrict__ tw) {
    constexpr int N = TN1 * TN2;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const int b = i / TN2, a = i - b * TN2;
        twt[i] = tw[(a * b) % N];
    }
}

}  // namespace cfd
