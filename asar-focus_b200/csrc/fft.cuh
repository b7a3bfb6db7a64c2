// Shared-memory mixed-radix FFT building blocks for sm_100a.
//
// Every transform here works IN PLACE on a tile held in shared memory, laid out as
// element (l, c) at s[l * ldc + c]: l in [0, n) runs along the transform, c in [0, ncol)
// indexes independent transforms (range lines, or range columns of an azimuth block).
//
//  * forward transforms are decimation-in-frequency: natural-order input, digit-reversed
//    output (position p holds frequency digit_reverse(p));
//  * inverse transforms are decimation-in-time: digit-reversed input, natural-order
//    output, unscaled.
//
// Pairing the two removes every reordering pass: a frequency-domain operation (chirp
// matched filter, RCMC, azimuth matched filter) only needs to know which frequency each
// position holds.  Radices 2, 3, 4, 5, 7 and 8 cover all 2^a 3^b 5^c 7^d lengths the
// range / azimuth padding rules produce; the register-resident range transforms add
// composite radices built from two of them (dft_any).  Twiddles come from a per-length table
// tw[m] = exp(-2*pi*i*m/n), m in [0, n), computed in FP64 on the host.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>
#include <utility>

#include "hd.cuh"

namespace asarf {

constexpr int kMaxStages = 16;

// Radix schedule of one transform length (host-built, passed by value to kernels).
struct FftPlan {
    int n;
    int nst;
    int radix[kMaxStages];
    int span[kMaxStages];  // S of stage i (block length M = S * radix)
    FastDiv sdiv[kMaxStages];
    const float2* tw;      // n entries
};

ASARF_HD ASARF_INLINE float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
ASARF_HD ASARF_INLINE float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
ASARF_HD ASARF_INLINE float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
ASARF_HD ASARF_INLINE float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
ASARF_HD ASARF_INLINE float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
ASARF_HD ASARF_INLINE float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// ----------------------------------------------------------------------------- packed complex ops
// Component-wise complex arithmetic: on sm_100 one f32x2 instruction per complex add, subtract,
// real scaling or real multiply-add (the instruction issue rate, not the FMA pipe, bounds the
// FFT kernels); the host emulation performs the same IEEE operations one lane at a time.
ASARF_HD ASARF_INLINE float2 padd(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __fadd2_rn(a, b);
#else
    return make_float2(a.x + b.x, a.y + b.y);
#endif
}

// a - b, as b * (-1) + a (one rounding of the exact difference)
ASARF_HD ASARF_INLINE float2 psub(float2 a, float2 b) {
#if defined(__CUDA_ARCH__)
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
#else
    return make_float2(a.x - b.x, a.y - b.y);
#endif
}

ASARF_HD ASARF_INLINE float2 pscale(float2 a, float c) {
#if defined(__CUDA_ARCH__)
    return __fmul2_rn(a, make_float2(c, c));
#else
    return make_float2(a.x * c, a.y * c);
#endif
}

// a * c + b
ASARF_HD ASARF_INLINE float2 pfma(float2 a, float c, float2 b) {
#if defined(__CUDA_ARCH__)
    return __ffma2_rn(a, make_float2(c, c), b);
#else
    return make_float2(__builtin_fmaf(a.x, c, b.x), __builtin_fmaf(a.y, c, b.y));
#endif
}

// r + mul_mi(p) and r - mul_mi(p): the swap of p's parts folded into two scalar adds
template <bool INV>
ASARF_HD ASARF_INLINE float2 add_mi(float2 r, float2 p) {
    return INV ? make_float2(r.x - p.y, r.y + p.x) : make_float2(r.x + p.y, r.y - p.x);
}
template <bool INV>
ASARF_HD ASARF_INLINE float2 sub_mi(float2 r, float2 p) {
    return INV ? make_float2(r.x + p.y, r.y - p.x) : make_float2(r.x - p.y, r.y + p.x);
}

// ----------------------------------------------------------------------------- small DFTs
// Sign convention: forward y_k = sum_m x_m exp(-2 pi i m k / R), inverse uses +.

template <bool INV>
ASARF_HD ASARF_INLINE void dft2(float2* v) {
    const float2 a = v[0];
    v[0] = padd(a, v[1]);
    v[1] = psub(a, v[1]);
}

template <bool INV>
ASARF_HD ASARF_INLINE void dft4(float2* v) {
    const float2 t0 = padd(v[0], v[2]);
    const float2 t1 = psub(v[0], v[2]);
    const float2 t2 = padd(v[1], v[3]);
    const float2 d = psub(v[1], v[3]);
    v[0] = padd(t0, t2);
    v[2] = psub(t0, t2);
    v[1] = add_mi<INV>(t1, d);
    v[3] = sub_mi<INV>(t1, d);
}

template <bool INV>
ASARF_HD ASARF_INLINE void dft8(float2* v) {
    constexpr float h = 0.7071067811865476f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    dft4<INV>(e);
    dft4<INV>(o);
    // o_k *= W8^k (forward W8 = exp(-i pi/4))
    const float2 o1 = INV ? make_float2(h * (o[1].x - o[1].y), h * (o[1].x + o[1].y))
                          : make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x));
    const float2 o3 = INV ? make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y))
                          : make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y));
    v[0] = padd(e[0], o[0]);
    v[4] = psub(e[0], o[0]);
    v[1] = padd(e[1], o1);
    v[5] = psub(e[1], o1);
    v[2] = add_mi<INV>(e[2], o[2]);
    v[6] = sub_mi<INV>(e[2], o[2]);
    v[3] = padd(e[3], o3);
    v[7] = psub(e[3], o3);
}

template <bool INV>
ASARF_HD ASARF_INLINE void dft3(float2* v) {
    constexpr float s3 = 0.8660254037844387f;
    const float2 a = padd(v[1], v[2]);
    const float2 b = psub(v[1], v[2]);
    const float2 t = pfma(a, -0.5f, v[0]);
    const float2 bs = pscale(b, s3);
    v[0] = padd(v[0], a);
    v[1] = add_mi<INV>(t, bs);
    v[2] = sub_mi<INV>(t, bs);
}

template <bool INV>
ASARF_HD ASARF_INLINE void dft5(float2* v) {
    constexpr float c1 = 0.30901699437494745f, s1 = 0.9510565162951535f;
    constexpr float c2 = -0.8090169943749473f, s2 = 0.5877852522924732f;
    const float2 a1 = padd(v[1], v[4]), b1 = psub(v[1], v[4]);
    const float2 a2 = padd(v[2], v[3]), b2 = psub(v[2], v[3]);
    const float2 x0 = v[0];
    const float2 r1 = pfma(a2, c2, pfma(a1, c1, x0));
    const float2 r2 = pfma(a2, c1, pfma(a1, c2, x0));
    const float2 p1 = pfma(b2, s2, pscale(b1, s1));
    const float2 p2 = pfma(b2, -s1, pscale(b1, s2));
    v[0] = padd(padd(x0, a1), a2);
    v[1] = add_mi<INV>(r1, p1);
    v[4] = sub_mi<INV>(r1, p1);
    v[2] = add_mi<INV>(r2, p2);
    v[3] = sub_mi<INV>(r2, p2);
}

template <bool INV>
ASARF_HD ASARF_INLINE void dft7(float2* v) {
    constexpr float c1 = 0.6234898018587336f, s1 = 0.7818314824680298f;
    constexpr float c2 = -0.22252093395631434f, s2 = 0.9749279121818236f;
    constexpr float c3 = -0.900968867902419f, s3 = 0.43388373911755823f;
    const float2 a1 = padd(v[1], v[6]), b1 = psub(v[1], v[6]);
    const float2 a2 = padd(v[2], v[5]), b2 = psub(v[2], v[5]);
    const float2 a3 = padd(v[3], v[4]), b3 = psub(v[3], v[4]);
    const float2 x0 = v[0];
    // k = 1..3: cos(2 pi m k / 7) pattern over m = 1..3; sin pattern with sign folding
    const float2 r1 = pfma(a3, c3, pfma(a2, c2, pfma(a1, c1, x0)));
    const float2 r2 = pfma(a3, c1, pfma(a2, c3, pfma(a1, c2, x0)));
    const float2 r3 = pfma(a3, c2, pfma(a2, c1, pfma(a1, c3, x0)));
    // sin(2 pi m k / 7): k=1: s1 s2 s3 ; k=2: s2 -s3 -s1 ; k=3: s3 -s1 s2
    const float2 p1 = pfma(b3, s3, pfma(b2, s2, pscale(b1, s1)));
    const float2 p2 = pfma(b3, -s1, pfma(b2, -s3, pscale(b1, s2)));
    const float2 p3 = pfma(b3, s2, pfma(b2, -s1, pscale(b1, s3)));
    v[0] = padd(padd(padd(x0, a1), a2), a3);
    v[1] = add_mi<INV>(r1, p1);
    v[6] = sub_mi<INV>(r1, p1);
    v[2] = add_mi<INV>(r2, p2);
    v[5] = sub_mi<INV>(r2, p2);
    v[3] = add_mi<INV>(r3, p3);
    v[4] = sub_mi<INV>(r3, p3);
}

template <int R, bool INV>
ASARF_HD ASARF_INLINE void dft(float2* v) {
    if constexpr (R == 2) dft2<INV>(v);
    else if constexpr (R == 3) dft3<INV>(v);
    else if constexpr (R == 4) dft4<INV>(v);
    else if constexpr (R == 5) dft5<INV>(v);
    else if constexpr (R == 7) dft7<INV>(v);
    else if constexpr (R == 8) dft8<INV>(v);
}

// ----------------------------------------------------------------------------- constants
// cos / sin of 2 pi num / den in double, evaluated at compile time from their Taylor series
// after reduction to [0, pi/4) by the symmetries of the circle (plain mathematics).
constexpr double ct_pi = 3.14159265358979323846264338327950288;

ASARF_HD constexpr double ct_taylor_cos(double x) {
    double term = 1.0, sum = 1.0;
    for (int k = 1; k < 24; ++k) {
        term *= -x * x / ((2 * k - 1) * (2 * k));
        sum += term;
    }
    return sum;
}
ASARF_HD constexpr double ct_taylor_sin(double x) {
    double term = x, sum = x;
    for (int k = 1; k < 24; ++k) {
        term *= -x * x / ((2 * k) * (2 * k + 1));
        sum += term;
    }
    return sum;
}
// 8 * num / den = octant + fraction; the fraction of the octant is exact in double
ASARF_HD constexpr double ct_cos2pi(long num, long den) {
    num %= den;
    if (num < 0) num += den;
    const long e = 8 * num;
    const long oct = e / den;
    const double frac = static_cast<double>(e - oct * den) / static_cast<double>(den);
    const double x = frac * ct_pi / 4;
    const double y = (1.0 - frac) * ct_pi / 4;
    switch (oct) {
        case 0: return ct_taylor_cos(x);
        case 1: return ct_taylor_sin(y);
        case 2: return -ct_taylor_sin(x);
        case 3: return -ct_taylor_cos(y);
        case 4: return -ct_taylor_cos(x);
        case 5: return -ct_taylor_sin(y);
        case 6: return ct_taylor_sin(x);
        default: return ct_taylor_cos(y);
    }
}
// sin(2 pi n / d) = cos(2 pi (4n - d) / 4d)
ASARF_HD constexpr double ct_sin2pi(long num, long den) { return ct_cos2pi(4 * num - den, 4 * den); }

// ----------------------------------------------------------------------------- composite DFTs
// Compile-time loop: f(std::integral_constant<int, I>) for I = 0 .. N-1, so that indices
// are constant expressions (twiddle constants evaluated by the compiler, never at run time).
template <class F, int... I>
ASARF_HD ASARF_INLINE void ct_static_for_impl(F& f, std::integer_sequence<int, I...>) {
    (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
ASARF_HD ASARF_INLINE void ct_static_for(F&& f) {
    ct_static_for_impl(f, std::make_integer_sequence<int, N>{});
}

// a * W_R^{e} (forward W = exp(-2 pi i / R), inverse conjugate) with constant factors
template <int R, long E, bool INV>
ASARF_HD ASARF_INLINE float2 ct_twiddle(float2 a) {
    if constexpr (E % R == 0) {
        return a;
    } else {
        constexpr float c = static_cast<float>(ct_cos2pi(E, R));
        constexpr float sn = static_cast<float>(INV ? ct_sin2pi(E, R) : -ct_sin2pi(E, R));
        return cmul(a, make_float2(c, sn));
    }
}

// X[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_R^{n2 k1} sum_n1 x[n1 R2 + n2] W_R1^{n1 k1}
// (forward W = exp(-2 pi i / R); inverse conjugate), natural order in and out.
template <int R1, int R2, bool INV>
ASARF_HD ASARF_INLINE void dft_composite(float2* v) {
    constexpr int R = R1 * R2;
    float2 t[R];
    ct_static_for<R2>([&](auto n2c) {
        constexpr int n2 = decltype(n2c)::value;
        float2 a[R1];
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) a[n1] = v[n1 * R2 + n2];
        dft<R1, INV>(a);
        ct_static_for<R1>([&](auto k1c) {
            constexpr int k1 = decltype(k1c)::value;
            t[k1 * R2 + n2] = ct_twiddle<R, static_cast<long>(n2) * k1, INV>(a[k1]);
        });
    });
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        float2 b[R2];
#pragma unroll
        for (int n2 = 0; n2 < R2; ++n2) b[n2] = t[k1 * R2 + n2];
        dft<R2, INV>(b);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = b[k2];
    }
}

// Any radix the schedules use: the direct small DFTs, or a composite of two of them.
template <int R, bool INV>
ASARF_HD ASARF_INLINE void dft_any(float2* v) {
    if constexpr (R == 9) dft_composite<3, 3, INV>(v);
    else if constexpr (R == 12) dft_composite<4, 3, INV>(v);
    else if constexpr (R == 16) dft_composite<4, 4, INV>(v);
    else if constexpr (R == 24) dft_composite<8, 3, INV>(v);
    else if constexpr (R == 32) dft_composite<8, 4, INV>(v);
    else dft<R, INV>(v);
}

// ----------------------------------------------------------------------------- one stage
// Butterfly item t -> (column c = t % ncol, butterfly bj = t / ncol); bj -> (block b, offset j).
// Forward (DIF): load R values at stride S, small DFT, multiply output q by W_M^{j q}.
// Inverse (DIT): multiply input q by conj(W_M^{j q}), small inverse DFT.
template <int R, bool INV>
ASARF_HD ASARF_INLINE void fft_stage(float2* s, int n, int S, const FastDiv& sdiv, int ncol, const FastDiv& cdiv, int ldc,
                                     const float2* __restrict__ tw, int tid, int nthr) {
    const int M = S * R;
    const int items = (n / R) * ncol;
    const int tw_step = n / M;
    for (int t = tid; t < items; t += nthr) {
        const int bj = ncol == 1 ? t : static_cast<int>(fdiv_u(t, cdiv));
        const int c = t - bj * ncol;
        const int b = static_cast<int>(fdiv_u(bj, sdiv));
        const int j = bj - b * S;
        float2* p = s + (b * M + j) * ldc + c;
        const int st = S * ldc;
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = p[m * st];
        if (INV) {
            if (j != 0) {
                // W^{j q}: one table load, higher powers by recurrence (error ~ q ulp)
                const float2 w1 = ASARF_LDG(tw + j * tw_step);
                float2 w = w1;
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    v[q] = cmulc(v[q], w);
                    w = cmul(w, w1);
                }
            }
            dft<R, true>(v);
        } else {
            dft<R, false>(v);
            if (j != 0) {
                const float2 w1 = ASARF_LDG(tw + j * tw_step);
                float2 w = w1;
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    v[q] = cmul(v[q], w);
                    w = cmul(w, w1);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m) p[m * st] = v[m];
    }
}

// Inverse transform in decimation-in-frequency form: small inverse DFT, then multiply output
// q by conj(W_M^{j q}).  Natural-order input, digit-reversed output (same map as the forward).
template <int R>
ASARF_HD ASARF_INLINE void fft_stage_dif_inv(float2* s, int n, int S, const FastDiv& sdiv, int ncol, const FastDiv& cdiv,
                                             int ldc, const float2* __restrict__ tw, int tid, int nthr) {
    const int M = S * R;
    const int items = (n / R) * ncol;
    const int tw_step = n / M;
    for (int t = tid; t < items; t += nthr) {
        const int bj = ncol == 1 ? t : static_cast<int>(fdiv_u(t, cdiv));
        const int c = t - bj * ncol;
        const int b = static_cast<int>(fdiv_u(bj, sdiv));
        const int j = bj - b * S;
        float2* p = s + (b * M + j) * ldc + c;
        const int st = S * ldc;
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = p[m * st];
        dft<R, true>(v);
        if (j != 0) {
            const float2 w1 = ASARF_LDG(tw + j * tw_step);
            float2 w = w1;
#pragma unroll
            for (int q = 1; q < R; ++q) {
                v[q] = cmulc(v[q], w);
                w = cmul(w, w1);
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m) p[m * st] = v[m];
    }
}

// ----------------------------------------------------------------------------- column pairs
// The same stages over PAIRS of adjacent columns: one 16-byte shared-memory access moves
// both columns' samples and one twiddle set serves both butterflies.  Needs ldc even, the
// tile base 16-byte aligned and an even column count.  TW_FIRST selects decimation in time
// (twiddle, then DFT); INV selects the inverse DFT sign and conjugated twiddles.
// Epilogue of a column-pair transform: the last stage hands each output (row l, column pair
// cp) to epi(l, cp, u, v) instead of storing it back to the tile.
struct NoEpi {
    static constexpr bool kActive = false;
    ASARF_HD ASARF_INLINE void operator()(int, int, float2, float2) const {}
};

// u * w from w and iw = i w: u.x w + u.y iw, two packed operations.
ASARF_HD ASARF_INLINE float2 cmul_rot(float2 u, float2 w, float2 iw) { return pfma(iw, u.y, pscale(w, u.x)); }
ASARF_HD ASARF_INLINE float2 rot90(float2 w) { return make_float2(-w.y, w.x); }

// Value q of both columns times W^q (INV: conj(W)^q), W = w1, q = 1 .. R-1.  PTW: packed
// products (one rotation of each power serves both columns); otherwise scalar complex products.
template <int R, bool INV, bool PTW>
ASARF_HD ASARF_INLINE void pair_twiddle(float2* u, float2* v, float2 w1) {
    if constexpr (PTW) {
        const float2 ws = INV ? make_float2(w1.x, -w1.y) : w1;
        const float2 is = rot90(ws);
        float2 w = ws, iw = is;
#pragma unroll
        for (int q = 1; q < R; ++q) {
            u[q] = cmul_rot(u[q], w, iw);
            v[q] = cmul_rot(v[q], w, iw);
            if (q + 1 < R) {
                w = cmul_rot(w, ws, is);
                iw = rot90(w);
            }
        }
    } else {
        float2 w = w1;
#pragma unroll
        for (int q = 1; q < R; ++q) {
            u[q] = INV ? cmulc(u[q], w) : cmul(u[q], w);
            v[q] = INV ? cmulc(v[q], w) : cmul(v[q], w);
            w = cmul(w, w1);
        }
    }
}

// One butterfly of a column-pair stage: block b, offset j (M = S * R), column pair cp.
// PRE: the loaded values of row l are first multiplied by conj(pre[l]) (a per-row table, here the
// input twiddles of the inverse strided pass), saving a separate pass over the tile.
template <int R, bool INV, bool TW_FIRST, bool PRE, class Epi, bool PTW>
ASARF_HD ASARF_INLINE void pair_item(float2* s, int b, int j, int cp, int M, int S, int ldc, int tw_step,
                                     const float2* __restrict__ tw, const float2* pre, const Epi& epi) {
    const int st = (S * ldc) >> 1;  // float4 units
    float4* p = reinterpret_cast<float4*>(s + (b * M + j) * ldc) + cp;
    float2 u[R], v[R];
#pragma unroll
    for (int m = 0; m < R; ++m) {
        const float4 q = p[m * st];
        u[m] = make_float2(q.x, q.y);
        v[m] = make_float2(q.z, q.w);
        if constexpr (PRE) {
            const float2 w = pre[b * M + j + m * S];
            u[m] = cmulc(u[m], w);
            v[m] = cmulc(v[m], w);
        }
    }
    // W_M^{j q}: one table load, higher powers by recurrence (error ~ q ulp); a table load
    // per q is exact but measured slower
    const float2 w1 = j != 0 ? ASARF_LDG(tw + j * tw_step) : make_float2(1.0f, 0.0f);
    if (TW_FIRST && j != 0) pair_twiddle<R, INV, PTW>(u, v, w1);
    dft_any<R, INV>(u);
    dft_any<R, INV>(v);
    if (!TW_FIRST && j != 0) pair_twiddle<R, INV, PTW>(u, v, w1);
    if constexpr (Epi::kActive) {
#pragma unroll
        for (int m = 0; m < R; ++m) epi(b * M + j + m * S, cp, u[m], v[m]);
    } else {
#pragma unroll
        for (int m = 0; m < R; ++m) p[m * st] = make_float4(u[m].x, u[m].y, v[m].x, v[m].y);
    }
}

template <int R, bool INV, bool TW_FIRST, bool PRE = false, class Epi = NoEpi, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_stage_pair(float2* s, int n, int S, const FastDiv& sdiv, int npair, const FastDiv& pdiv,
                                          int ldc, const float2* __restrict__ tw, int tid, int nthr,
                                          const float2* pre = nullptr, const Epi& epi = Epi()) {
    const int M = S * R;
    const int items = (n / R) * npair;
    const int tw_step = n / M;
    for (int t = tid; t < items; t += nthr) {
        const int bj = static_cast<int>(fdiv_u(t, pdiv));
        const int cp = t - bj * npair;
        const int b = static_cast<int>(fdiv_u(bj, sdiv));
        const int j = bj - b * S;
        pair_item<R, INV, TW_FIRST, PRE, Epi, PTW>(s, b, j, cp, M, S, ldc, tw_step, tw, pre, epi);
    }
}

// The same stage with every size a compile-time constant (length N, span S, NPAIR column pairs
// of row stride LDC): the index arithmetic folds into constant multiplies and shifts.
template <int R, bool INV, bool TW_FIRST, int N, int S, int NPAIR, int LDC, bool PRE = false, class Epi = NoEpi,
          bool PTW = false>
ASARF_HD ASARF_INLINE void fft_stage_pair_ct(float2* s, const float2* __restrict__ tw, int tid, int nthr,
                                             const float2* pre = nullptr, const Epi& epi = Epi()) {
    constexpr int M = S * R;
    constexpr int ITEMS = (N / R) * NPAIR;
    constexpr int TW_STEP = N / M;
    for (int t = tid; t < ITEMS; t += nthr) {
        const int bj = t / NPAIR;
        const int cp = t - bj * NPAIR;
        const int b = bj / S;
        const int j = bj - b * S;
        pair_item<R, INV, TW_FIRST, PRE, Epi, PTW>(s, b, j, cp, M, S, LDC, TW_STEP, tw, pre, epi);
    }
}

// The same stage with the length N and span S compile-time constants and the column count
// run-time (npair pairs, divider pdiv, row stride ldc): the range-Doppler block, whose tile
// width follows the scene's range walk.  PTW: packed twiddle products.
template <int R, bool INV, bool TW_FIRST, int N, int S, class Epi = NoEpi, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_stage_pair_cs(float2* s, int npair, const FastDiv& pdiv, int ldc,
                                             const float2* __restrict__ tw, int tid, int nthr,
                                             const Epi& epi = Epi()) {
    constexpr int M = S * R;
    const int items = (N / R) * npair;
    for (int t = tid; t < items; t += nthr) {
        const int bj = static_cast<int>(fdiv_u(t, pdiv));
        const int cp = t - bj * npair;
        const int b = bj / S;
        const int j = bj - b * S;
        pair_item<R, INV, TW_FIRST, false, Epi, PTW>(s, b, j, cp, M, S, ldc, N / M, tw, nullptr, epi);
    }
}

// Column-pair stages take the prime-power radices: a larger composite radix holds twice its
// length in registers per column pair, which lifts the azimuth kernels from 64 to 128
// registers per thread and halves their resident CTAs (measured slower despite fewer passes).
// NINE adds radix 9 (two radix-3 DFTs in registers, 36 values per column pair: 71 registers
// in the strided kernel, whose occupancy shared memory limits anyway) for plans that merge
// factors 3 * 3; it is compiled only where such plans run, since every extra case costs the
// other kernels registers.  PTW selects the packed twiddle products: the strided kernel uses them,
// the range-Doppler block for radix <= 5 schedules only (az_rd_packed_twiddles).
template <bool INV, bool TW_FIRST, bool NINE = false, bool PRE = false, class Epi = NoEpi, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_stage_pair_dispatch(int R, float2* s, int n, int S, const FastDiv& sdiv, int npair,
                                                   const FastDiv& pdiv, int ldc, const float2* __restrict__ tw,
                                                   int tid, int nthr, const float2* pre = nullptr,
                                                   const Epi& epi = Epi()) {
#define ASARF_PAIR(RR) \
    fft_stage_pair<RR, INV, TW_FIRST, PRE, Epi, PTW>(s, n, S, sdiv, npair, pdiv, ldc, tw, tid, nthr, pre, epi)
    if constexpr (NINE) {
        if (R == 9) {
            ASARF_PAIR(9);
            return;
        }
    }
    switch (R) {
        case 2: ASARF_PAIR(2); break;
        case 3: ASARF_PAIR(3); break;
        case 4: ASARF_PAIR(4); break;
        case 5: ASARF_PAIR(5); break;
        case 7: ASARF_PAIR(7); break;
        default: ASARF_PAIR(8); break;
    }
#undef ASARF_PAIR
}

// Column-pair forms of fft_forward / fft_inverse / fft_inverse_dif (ncol and ldc even).
template <bool NINE = false, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_forward_pairs(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr) {
    const int npair = ncol >> 1;
    const FastDiv pdiv = make_fastdiv(static_cast<unsigned int>(npair));
    for (int i = 0; i < p.nst; ++i) {
        fft_stage_pair_dispatch<false, false, NINE, false, NoEpi, PTW>(p.radix[i], s, p.n, p.span[i], p.sdiv[i], npair,
                                                                      pdiv, ldc, p.tw, tid, nthr);
        ASARF_SYNC();
    }
}

// With an active epilogue the last stage writes through it and the tile is left unfinished.
template <class Epi = NoEpi, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_inverse_pairs(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr,
                                             const Epi& epi = Epi()) {
    const int npair = ncol >> 1;
    const FastDiv pdiv = make_fastdiv(static_cast<unsigned int>(npair));
    for (int i = p.nst - 1; i >= 0; --i) {
        if (Epi::kActive && i == 0)
            fft_stage_pair_dispatch<true, true, false, false, Epi, PTW>(p.radix[i], s, p.n, p.span[i], p.sdiv[i],
                                                                        npair, pdiv, ldc, p.tw, tid, nthr, nullptr, epi);
        else
            fft_stage_pair_dispatch<true, true, false, false, NoEpi, PTW>(p.radix[i], s, p.n, p.span[i], p.sdiv[i],
                                                                          npair, pdiv, ldc, p.tw, tid, nthr);
        ASARF_SYNC();
    }
}

// pre (optional): per-row table whose conjugate multiplies the input (folded into stage 0).
template <bool NINE = false, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_inverse_dif_pairs(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr,
                                                 const float2* pre = nullptr) {
    const int npair = ncol >> 1;
    const FastDiv pdiv = make_fastdiv(static_cast<unsigned int>(npair));
    for (int i = 0; i < p.nst; ++i) {
        if (i == 0 && pre)
            fft_stage_pair_dispatch<true, false, NINE, true, NoEpi, PTW>(p.radix[i], s, p.n, p.span[i], p.sdiv[i],
                                                                        npair, pdiv, ldc, p.tw, tid, nthr, pre);
        else
            fft_stage_pair_dispatch<true, false, NINE, false, NoEpi, PTW>(p.radix[i], s, p.n, p.span[i], p.sdiv[i],
                                                                         npair, pdiv, ldc, p.tw, tid, nthr);
        ASARF_SYNC();
    }
}

// Compile-time three-stage column-pair transforms (radices R0, R1, R2 first stage first, NPAIR
// column pairs of row stride LDC): the forward DIF and the inverse in DIF form of the strided
// azimuth pass, with the same stage sequence, twiddle tables and rounding as the run-time
// versions above (fft_forward_pairs / fft_inverse_dif_pairs), so the results are identical.
template <int R0, int R1, int R2, int NPAIR, int LDC, bool PTW>
ASARF_HD ASARF_INLINE void fft_forward_pairs_ct3(float2* s, const float2* __restrict__ tw, int tid, int nthr) {
    constexpr int N = R0 * R1 * R2;
    fft_stage_pair_ct<R0, false, false, N, N / R0, NPAIR, LDC, false, NoEpi, PTW>(s, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_ct<R1, false, false, N, N / (R0 * R1), NPAIR, LDC, false, NoEpi, PTW>(s, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_ct<R2, false, false, N, 1, NPAIR, LDC, false, NoEpi, PTW>(s, tw, tid, nthr);
    ASARF_SYNC();
}

template <int R0, int R1, int R2, int NPAIR, int LDC, bool PTW>
ASARF_HD ASARF_INLINE void fft_inverse_dif_pairs_ct3(float2* s, const float2* __restrict__ tw, int tid, int nthr,
                                                     const float2* pre) {
    constexpr int N = R0 * R1 * R2;
    fft_stage_pair_ct<R0, true, false, N, N / R0, NPAIR, LDC, true, NoEpi, PTW>(s, tw, tid, nthr, pre);
    ASARF_SYNC();
    fft_stage_pair_ct<R1, true, false, N, N / (R0 * R1), NPAIR, LDC, false, NoEpi, PTW>(s, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_ct<R2, true, false, N, 1, NPAIR, LDC, false, NoEpi, PTW>(s, tw, tid, nthr);
    ASARF_SYNC();
}

// Three-stage forward DIF (fft_forward_pairs) and inverse DIT with epilogue (fft_inverse_pairs)
// of a compile-time radix schedule R0, R1, R2 over a run-time number of columns: the same
// stages, twiddles and rounding as the run-time versions.
template <int R0, int R1, int R2, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_forward_pairs_cs3(float2* s, int ncol, int ldc, const float2* __restrict__ tw, int tid,
                                                 int nthr) {
    constexpr int N = R0 * R1 * R2;
    const int npair = ncol >> 1;
    const FastDiv pdiv = make_fastdiv(static_cast<unsigned int>(npair));
    fft_stage_pair_cs<R0, false, false, N, N / R0, NoEpi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_cs<R1, false, false, N, R2, NoEpi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_cs<R2, false, false, N, 1, NoEpi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr);
    ASARF_SYNC();
}

template <int R0, int R1, int R2, class Epi = NoEpi, bool PTW = false>
ASARF_HD ASARF_INLINE void fft_inverse_pairs_cs3(float2* s, int ncol, int ldc, const float2* __restrict__ tw, int tid,
                                                 int nthr, const Epi& epi = Epi()) {
    constexpr int N = R0 * R1 * R2;
    const int npair = ncol >> 1;
    const FastDiv pdiv = make_fastdiv(static_cast<unsigned int>(npair));
    fft_stage_pair_cs<R2, true, true, N, 1, NoEpi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_cs<R1, true, true, N, R2, NoEpi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr);
    ASARF_SYNC();
    fft_stage_pair_cs<R0, true, true, N, N / R0, Epi, PTW>(s, npair, pdiv, ldc, tw, tid, nthr, epi);
    ASARF_SYNC();
}

template <bool INV>
ASARF_HD ASARF_INLINE void fft_stage_dispatch(int R, float2* s, int n, int S, const FastDiv& sdiv, int ncol,
                                              const FastDiv& cdiv, int ldc, const float2* __restrict__ tw, int tid,
                                              int nthr) {
    switch (R) {
        case 2: fft_stage<2, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
        case 3: fft_stage<3, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
        case 4: fft_stage<4, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
        case 5: fft_stage<5, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
        case 7: fft_stage<7, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
        default: fft_stage<8, INV>(s, n, S, sdiv, ncol, cdiv, ldc, tw, tid, nthr); break;
    }
}

// Forward DIF transform of ncol independent columns; output digit-reversed.  The caller
// places a barrier after loading the tile; this returns after a final barrier.
ASARF_HD ASARF_INLINE void fft_forward(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr) {
    const FastDiv cdiv = make_fastdiv(static_cast<unsigned int>(ncol));
    for (int i = 0; i < p.nst; ++i) {
        fft_stage_dispatch<false>(p.radix[i], s, p.n, p.span[i], p.sdiv[i], ncol, cdiv, ldc, p.tw, tid, nthr);
        ASARF_SYNC();
    }
}

// Inverse DIT transform (digit-reversed input, natural output, unscaled).
ASARF_HD ASARF_INLINE void fft_inverse(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr) {
    const FastDiv cdiv = make_fastdiv(static_cast<unsigned int>(ncol));
    for (int i = p.nst - 1; i >= 0; --i) {
        fft_stage_dispatch<true>(p.radix[i], s, p.n, p.span[i], p.sdiv[i], ncol, cdiv, ldc, p.tw, tid, nthr);
        ASARF_SYNC();
    }
}

// Inverse transform, natural-order input, digit-reversed output, unscaled.
ASARF_HD ASARF_INLINE void fft_inverse_dif(const FftPlan& p, float2* s, int ncol, int ldc, int tid, int nthr) {
    const FastDiv cdiv = make_fastdiv(static_cast<unsigned int>(ncol));
    for (int i = 0; i < p.nst; ++i) {
        const FastDiv& sd = p.sdiv[i];
        switch (p.radix[i]) {
            case 2: fft_stage_dif_inv<2>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
            case 3: fft_stage_dif_inv<3>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
            case 4: fft_stage_dif_inv<4>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
            case 5: fft_stage_dif_inv<5>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
            case 7: fft_stage_dif_inv<7>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
            default: fft_stage_dif_inv<8>(s, p.n, p.span[i], sd, ncol, cdiv, ldc, p.tw, tid, nthr); break;
        }
        ASARF_SYNC();
    }
}

}  // namespace asarf
