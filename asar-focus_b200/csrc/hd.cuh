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
