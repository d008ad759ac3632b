// fft_pair.cuh - complex values of two lines in packed FP32 pairs for the register DFTs
// of fft_reg.cuh (sm_100a).
//
// sm_100 executes add, sub, mul and fma on two FP32 values held in one 64-bit register
// pair with a single instruction (.f32x2).  A cpair carries element e of two lines A and B
// as x = (Re A_e, Re B_e), y = (Im A_e, Im B_e), so every operation of a DFT on the two
// lines is one packed instruction where the scalar form issues two.  The register DFTs of
// fft_reg.cuh are generic in the complex type; the overloads below give them the packed
// forms and avoid negations, which the scalar instructions fold into their operands for
// free but the packed ones would pay for.
#pragma once

#include "fft_reg.cuh"

namespace cfd {

struct f2x {
    float2 v;
};
struct cpair {
    f2x x, y;
};

__host__ __device__ __forceinline__ f2x f2p(float a, float b) {
    f2x r;
    r.v = make_float2(a, b);
    return r;
}
__host__ __device__ __forceinline__ f2x f2b(float a) { return f2p(a, a); }

#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
__device__ __forceinline__ f2x add2(f2x a, f2x b) { return f2x{__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2x mul2(f2x a, f2x b) { return f2x{__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ f2x fma2(f2x a, f2x b, f2x c) { return f2x{__ffma2_rn(a.v, b.v, c.v)}; }
__device__ __forceinline__ f2x sub2(f2x a, f2x b) {
    unsigned long long ra, rb, rd;
    memcpy(&ra, &a.v, 8);
    memcpy(&rb, &b.v, 8);
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(rd) : "l"(ra), "l"(rb));
    f2x r;
    memcpy(&r.v, &rd, 8);
    return r;
}
#else  // host (and the host-side check of these forms): the same operations lane by lane
__host__ __device__ inline f2x add2(f2x a, f2x b) { return f2p(a.v.x + b.v.x, a.v.y + b.v.y); }
__host__ __device__ inline f2x sub2(f2x a, f2x b) { return f2p(a.v.x - b.v.x, a.v.y - b.v.y); }
__host__ __device__ inline f2x mul2(f2x a, f2x b) { return f2p(a.v.x * b.v.x, a.v.y * b.v.y); }
__host__ __device__ inline f2x fma2(f2x a, f2x b, f2x c) { return f2p(fmaf(a.v.x, b.v.x, c.v.x), fmaf(a.v.y, b.v.y, c.v.y)); }
#endif
__host__ __device__ __forceinline__ f2x neg2(f2x a) { return mul2(a, f2b(-1.0f)); }

__host__ __device__ __forceinline__ cpair cadd(cpair a, cpair b) { return cpair{add2(a.x, b.x), add2(a.y, b.y)}; }
__host__ __device__ __forceinline__ cpair csub(cpair a, cpair b) { return cpair{sub2(a.x, b.x), sub2(a.y, b.y)}; }
// a * w and a * conj(w) for a twiddle w shared by both lines: w.x = (Re w, Re w),
// w.y = (Im w, Im w)
__host__ __device__ __forceinline__ cpair cmul(cpair a, cpair w) {
    return cpair{sub2(mul2(a.x, w.x), mul2(a.y, w.y)), fma2(a.x, w.y, mul2(a.y, w.x))};
}
__host__ __device__ __forceinline__ cpair cmulc(cpair a, cpair w) {
    return cpair{fma2(a.y, w.y, mul2(a.x, w.x)), sub2(mul2(a.y, w.x), mul2(a.x, w.y))};
}

template <int SIGN> __host__ __device__ __forceinline__ void dft2(cpair& a, cpair& b) {
    const cpair t = csub(a, b);
    a = cadd(a, b);
    b = t;
}

template <int SIGN> __host__ __device__ __forceinline__ void dft3(cpair& x0, cpair& x1, cpair& x2) {
    const float s3 = 0.86602540378443864676f * (float)SIGN;
    const cpair t1 = cadd(x1, x2), d = csub(x1, x2);
    const cpair t2 = cpair{fma2(t1.x, f2b(-0.5f), x0.x), fma2(t1.y, f2b(-0.5f), x0.y)};
    x0 = cadd(x0, t1);
    // t3 = (-s3 d.y, s3 d.x); x1 = t2 + t3, x2 = t2 - t3
    x1 = cpair{fma2(d.y, f2b(-s3), t2.x), fma2(d.x, f2b(s3), t2.y)};
    x2 = cpair{fma2(d.y, f2b(s3), t2.x), fma2(d.x, f2b(-s3), t2.y)};
}

template <int SIGN> __host__ __device__ __forceinline__ void dft4(cpair& x0, cpair& x1, cpair& x2, cpair& x3) {
    const cpair a0 = cadd(x0, x2), a1 = csub(x0, x2), b0 = cadd(x1, x3), d = csub(x1, x3);
    x0 = cadd(a0, b0);
    x2 = csub(a0, b0);
    // b1 = SIGN * i * d folded into the last two sums
    if constexpr (SIGN < 0) {
        x1 = cpair{add2(a1.x, d.y), sub2(a1.y, d.x)};
        x3 = cpair{sub2(a1.x, d.y), add2(a1.y, d.x)};
    } else {
        x1 = cpair{sub2(a1.x, d.y), add2(a1.y, d.x)};
        x3 = cpair{add2(a1.x, d.y), sub2(a1.y, d.x)};
    }
}

// multiplication by the compile-time twiddle TW (c + i s, not 1)
template <typename TW> __host__ __device__ __forceinline__ cpair cmul_k(cpair v) {
    constexpr float c = (float)TW::c, s = (float)TW::s;
    if constexpr (TW::c == 0.0) {
        // i s v: (-s v.y, s v.x), s = +-1
        if constexpr (TW::s > 0) return cpair{neg2(v.y), v.x};
        else return cpair{v.y, neg2(v.x)};
    } else if constexpr (TW::s == 0.0) {
        return cpair{neg2(v.x), neg2(v.y)};  // c = -1
    } else {
        return cpair{fma2(v.y, f2b(-s), mul2(v.x, f2b(c))), fma2(v.y, f2b(c), mul2(v.x, f2b(s)))};
    }
}

}  // namespace cfd
