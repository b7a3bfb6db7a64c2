// Host/device portability macros for the kernel bodies.
//
// Every kernel in this library is written as a sequence of barrier-separated phases in
// which thread `tid` of `nthr` walks a strided loop over independent work items.  The
// device build runs the phases with real threads and __syncthreads() between them.  The
// host-emulation build (ASARF_HOST_EMU, used only by the CPU test suite) runs the same
// code with tid = 0, nthr = 1, so a barrier is a no-op and shared memory is a host array.
#pragma once

#include <cuda_runtime.h>

#define ASARF_HD __host__ __device__

#if defined(__CUDA_ARCH__)
#define ASARF_INLINE __forceinline__
#define ASARF_SYNC() __syncthreads()
#define ASARF_LDG(p) __ldg(p)
#else
#define ASARF_INLINE inline
#define ASARF_SYNC() \
    do {             \
    } while (0)
#define ASARF_LDG(p) (*(p))
#endif

namespace asarf {

// Integer add into an accumulator shared by many threads.  Integer sums are order
// independent, so the statistics are bit-reproducible run to run.
ASARF_HD ASARF_INLINE void atomic_add_u64(unsigned long long* p, unsigned long long v) {
#if defined(__CUDA_ARCH__)
    atomicAdd(p, v);
#else
    *p += v;
#endif
}

ASARF_HD ASARF_INLINE void atomic_add_i64(long long* p, long long v) {
#if defined(__CUDA_ARCH__)
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(v));
#else
    *p += v;
#endif
}

// IEEE round-to-nearest division and fused multiply-add, written explicitly so the host
// emulation and the device agree with each other and with nvcc's default contraction.
ASARF_HD ASARF_INLINE float fdiv_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}

ASARF_HD ASARF_INLINE float fma_rn(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return __builtin_fmaf(a, b, c);
#endif
}

ASARF_HD ASARF_INLINE float fmul_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}

ASARF_HD ASARF_INLINE float fadd_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}

ASARF_HD ASARF_INLINE float fsub_rn(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}

// a / b rounded to nearest, given rb = RN(1 / b): q0 = RN(a rb) is within one ulp of a / b,
// the residual a - b q0 is exact in one FMA, and RN(q0 + residual * rb) is the correctly
// rounded quotient (Markstein, IBM J. Res. Dev. 34(1), 1990; the theorem in round-to-nearest
// binary arithmetic, no overflow or underflow).  Three operations when b is reused.
ASARF_HD ASARF_INLINE float div_by_recip_rn(float a, float b, float rb) {
    const float q0 = fmul_rn(a, rb);
    const float r = fma_rn(-q0, b, a);
    return fma_rn(r, rb, q0);
}

// sin and cos of x in [-pi, pi] from the hardware approximation (absolute error below
// 2^-21.4 there on the device); the host emulation evaluates them in FP64.
ASARF_HD ASARF_INLINE void sincos_reduced(float x, float* s, float* c) {
#if defined(__CUDA_ARCH__)
    __sincosf(x, s, c);
#else
    *s = static_cast<float>(__builtin_sin(static_cast<double>(x)));
    *c = static_cast<float>(__builtin_cos(static_cast<double>(x)));
#endif
}

// Hardware reciprocal approximation (about 1 ulp, flush-to-zero); the host emulation divides.
ASARF_HD ASARF_INLINE float rcp_approx(float x) {
#if defined(__CUDA_ARCH__)
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
#else
    return 1.0f / x;
#endif
}

ASARF_HD ASARF_INLINE float rint_f(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return __builtin_rintf(x);
#endif
}

// exp(-j (a + b)) for float phases a, b in radians with |a + b| < 2^20.  The sum is kept
// exactly as a float pair (Knuth's two-sum), reduced by k = rint((a + b) / 2 pi) against a
// two-part 2 pi (Cody & Waite): s - k * A is exact (both are multiples of ulp(A) = 2^-21 once
// |s| >= 4, Sterbenz below that, and the difference is under 4), so the reduced angle carries
// only the roundings of the two small terms.
ASARF_HD ASARF_INLINE float2 expj_neg_sum(float a, float b) {
    constexpr double kTwoPi = 6.283185307179586476925286766559;
    constexpr float kTwoPiA = static_cast<float>(kTwoPi);
    constexpr float kTwoPiB = static_cast<float>(kTwoPi - static_cast<double>(kTwoPiA));
    constexpr float kInvTwoPi = static_cast<float>(1.0 / kTwoPi);
    const float s = fadd_rn(a, b);
    const float bb = fsub_rn(s, a);
    const float e = fadd_rn(fsub_rn(a, fsub_rn(s, bb)), fsub_rn(b, bb));
    const float k = rint_f(fmul_rn(s, kInvTwoPi));
    float r = fma_rn(-k, kTwoPiA, s);
    r = fma_rn(-k, kTwoPiB, r);
    r = fadd_rn(r, e);
    float sn, cs;
    sincos_reduced(r, &sn, &cs);
    return make_float2(cs, -sn);
}

// Division by a loop-invariant divisor d < 2^16 of n < 2^16 without a hardware divide:
// q = umulhi(n, ceil(2^32 / d)) (exact while n * (m d - 2^32) < 2^32), or a shift when d is
// a power of two.
struct FastDiv {
    unsigned int d;
    unsigned int m;      // 0: power of two, use shift
    unsigned int shift;
};

ASARF_HD ASARF_INLINE FastDiv make_fastdiv(unsigned int d) {
    FastDiv f{d, 0u, 0u};
    if ((d & (d - 1)) == 0) {
        unsigned int s = 0;
        while ((1u << s) < d) ++s;
        f.shift = s;
    } else {
        f.m = static_cast<unsigned int>((0x100000000ull + d - 1) / d);
    }
    return f;
}

ASARF_HD ASARF_INLINE unsigned int fdiv_u(unsigned int n, const FastDiv& f) {
    if (f.m == 0) return n >> f.shift;
#if defined(__CUDA_ARCH__)
    return __umulhi(n, f.m);
#else
    return static_cast<unsigned int>((static_cast<unsigned long long>(n) * f.m) >> 32);
#endif
}

ASARF_HD ASARF_INLINE float qnan_f() {
#if defined(__CUDA_ARCH__)
    return __int_as_float(0x7fc00000);
#else
    return __builtin_nanf("");
#endif
}

// sin(pi x) with exact argument reduction (CUDA sinpif; FP64 on the host).
ASARF_HD ASARF_INLINE float sinpi_f32(float x) {
#if defined(__CUDA_ARCH__)
    return sinpif(x);
#else
    return static_cast<float>(__builtin_sin(3.141592653589793238462643383279502884 * static_cast<double>(x)));
#endif
}

// Correctly rounded reciprocal.
ASARF_HD ASARF_INLINE float rcp_f32(float x) {
#if defined(__CUDA_ARCH__)
    return __frcp_rn(x);
#else
    return 1.0f / x;
#endif
}

}  // namespace asarf
