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

template <typename T2> __device__ __forceinline__ T2 cx(decltype(T2::x) a, decltype(T2::x) b) {
    T2 r; r.x = a; r.y = b; return r;
}
template <typename T2> __device__ __forceinline__ T2 cadd(T2 a, T2 b) { return cx<T2>(a.x + b.x, a.y + b.y); }
template <typename T2> __device__ __forceinline__ T2 csub(T2 a, T2 b) { return cx<T2>(a.x - b.x, a.y - b.y); }
template <typename T2> __device__ __forceinline__ T2 cmul(T2 a, T2 b) {
    return cx<T2>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T2> __device__ __forceinline__ T2 cmulc(T2 a, T2 b) {
    return cx<T2>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T2> __device__ __forceinline__ T2 cconj(T2 a) { return cx<T2>(a.x, -a.y); }
template <typename T2> __device__ __forceinline__ T2 cscale(T2 a, decltype(T2::x) s) { return cx<T2>(a.x * s, a.y * s); }
// i * a
template <typename T2> __device__ __forceinline__ T2 cmuli(T2 a) { return cx<T2>(-a.y, a.x); }

// Radix plan of one length (filled on the host).
struct FFTDesc {
    int n;
    int nrad;
    int rad[10];
};

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
    int Ns = 1;
    for (int p = 0; p < d.nrad; ++p) {
        const int R = d.rad[p];
        const int nr = n / R;
        const int tstep = n / (Ns * R);
        const int ntask = nr * B;
        for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
            const int bb = t % B;
            const int i = t / B;
            const int k = i % Ns;
            T2 v[4];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (r < R) {
                    T2 x = in[(i + r * nr) * B + bb];
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
                if (r < R) out[(idxD + r * Ns) * B + bb] = v[r];
        }
        __syncthreads();
        T2* tmp = in; in = out; out = tmp;
        Ns *= R;
    }
    return in;
}

}  // namespace cfd
