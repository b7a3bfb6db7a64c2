// Compile-time-scheduled line FFTs for the range compression kernel.
//
// The range FFT length is a free choice (any L >= range size gives the same compressed
// samples), so the planner picks it from the lengths below and the whole transform is
// instantiated with constant radices, spans and per-thread item counts.
//
// Each length is three passes of composite radices (8, 12, 16, 24 or 32), each pass one
// register-resident DFT per item: three shared-memory round trips per transform instead
// of one per radix-2..8 stage.  The last forward pass, the matched-filter multiply and the
// first inverse pass touch the same R contiguous positions, so one thread does all three in
// registers (no shared-memory traffic between them).  The tile is padded with one element
// after every Q = (last radix) elements: every pass's R inputs stay at a constant stride,
// and lanes reading blocks of Q contiguous elements fall into different banks.
//
// Twiddles: a per-pass table tw_I[q][j] = exp(-2 pi i j q / M_I) (q = 1..R_I-1, j < S_I,
// M_I = R_I S_I), adjacent j adjacent in memory so a warp's loads coalesce; the matched
// filter is stored transposed, mf[q][b] for position b*R_last + q, for the same reason.
// The output order of the forward transform (and so the matched filter's order) is the
// digit reversal of this radix sequence, which the host builds from ct_radices().
#pragma once

#include "fft.cuh"
#include "hd.cuh"

namespace asarf {

// ----------------------------------------------------------------------------- schedules
template <int L>
struct CtSchedule {
    static constexpr int count = 0;
};
#define ASARF_CT_SCHEDULE(LEN, NT, R0, R1, R2)   \
    template <>                                  \
    struct CtSchedule<LEN> {                     \
        static constexpr int r[] = {R0, R1, R2}; \
        static constexpr int count = 3;          \
        static constexpr int nthr = NT;          \
    }
ASARF_CT_SCHEDULE(768, 96, 8, 8, 12);
ASARF_CT_SCHEDULE(1024, 128, 8, 8, 16);
ASARF_CT_SCHEDULE(1536, 192, 24, 8, 8);
ASARF_CT_SCHEDULE(2048, 128, 16, 16, 8);
ASARF_CT_SCHEDULE(3072, 256, 16, 16, 12);
ASARF_CT_SCHEDULE(4096, 256, 16, 16, 16);
ASARF_CT_SCHEDULE(6144, 384, 24, 16, 16);
ASARF_CT_SCHEDULE(8192, 256, 16, 16, 32);
#undef ASARF_CT_SCHEDULE

constexpr int kCtLengths[] = {768, 1024, 1536, 2048, 3072, 4096, 6144, 8192};

// Radix sequence of a compile-time length (host: digit reversal, matched filter, tables).
inline int ct_radices(int L, int* out) {
    auto put = [&](const int* r) {
        for (int i = 0; i < 3; ++i) out[i] = r[i];
        return 3;
    };
    switch (L) {
        case 768: return put(CtSchedule<768>::r);
        case 1024: return put(CtSchedule<1024>::r);
        case 1536: return put(CtSchedule<1536>::r);
        case 2048: return put(CtSchedule<2048>::r);
        case 3072: return put(CtSchedule<3072>::r);
        case 4096: return put(CtSchedule<4096>::r);
        case 6144: return put(CtSchedule<6144>::r);
        case 8192: return put(CtSchedule<8192>::r);
        default: return 0;
    }
}

template <int L, int I>
ASARF_HD constexpr int ct_span() {
    int m = L;
    for (int k = 0; k <= I; ++k) m /= CtSchedule<L>::r[k];
    return m;
}
// offset of pass I's twiddle table: sum over the earlier passes of (R - 1) * S
template <int L, int I>
ASARF_HD constexpr int ct_tw_offset() {
    int off = 0, m = L;
    for (int k = 0; k < I; ++k) {
        m /= CtSchedule<L>::r[k];
        off += (CtSchedule<L>::r[k] - 1) * m;
    }
    return off;
}
template <int L>
ASARF_HD constexpr int ct_padq() {
    return CtSchedule<L>::r[CtSchedule<L>::count - 1];
}
// padded shared-memory index of transform position e
template <int L>
ASARF_HD ASARF_INLINE int ct_pad(int e) {
    return e + e / ct_padq<L>();
}
// host: padded tile elements of a compile-time length
inline int ct_smem_elems_of(int L) {
    int r[3];
    return ct_radices(L, r) ? L + L / r[2] : 0;
}

// Run `phase(tid)` for this thread and barrier (device), or for every thread in turn (host
// emulation, where a phase must complete for all threads before the next one starts).
template <int NTHR, bool SYNC = true, class F>
ASARF_HD ASARF_INLINE void ct_phase(F&& phase, int tid) {
#if defined(__CUDA_ARCH__)
    phase(tid);
    if (SYNC) __syncthreads();
#else
    (void)tid;
    for (int t = 0; t < NTHR; ++t) phase(t);
#endif
}

// One pass I < count-1 (span S > 1, a multiple of Q): forward DIF (DFT, then twiddle output q
// by W_M^{jq}) or inverse DIT (conjugate twiddles on the inputs, then the inverse DFT).
// An active Epi receives each output (natural position, value) instead of the tile: the last
// inverse pass hands the line straight to its destination.
template <int L, int I, bool INV, class Epi = NoEpi>
ASARF_HD ASARF_INLINE void ct_pass(float2* s, const float2* __restrict__ ctw, int t, const Epi& epi = Epi{}) {
    constexpr int NTHR = CtSchedule<L>::nthr;
    constexpr int R = CtSchedule<L>::r[I];
    constexpr int S = ct_span<L, I>();
    constexpr int M = S * R;
    constexpr int Q = ct_padq<L>();
    constexpr int ITEMS = L / R;
    constexpr int PER = (ITEMS + NTHR - 1) / NTHR;
    constexpr int STRIDE = S + S / Q;  // padded distance between a butterfly's inputs
    constexpr int TWO = ct_tw_offset<L, I>();
    static_assert(S % Q == 0, "every pass but the last has a span divisible by the pad quotient");
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int it = t + k * NTHR;
        if (ITEMS % NTHR != 0 && it >= ITEMS) break;
        const int b = it / S;
        const int j = it - b * S;
        float2* p = s + ct_pad<L>(b * M + j);
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = p[m * STRIDE];
        if (INV) {
            if (j != 0) {
#pragma unroll
                for (int q = 1; q < R; ++q) v[q] = cmulc(v[q], ASARF_LDG(ctw + TWO + (q - 1) * S + j));
            }
            dft_any<R, true>(v);
        } else {
            dft_any<R, false>(v);
            if (j != 0) {
#pragma unroll
                for (int q = 1; q < R; ++q) v[q] = cmul(v[q], ASARF_LDG(ctw + TWO + (q - 1) * S + j));
            }
        }
        if constexpr (Epi::kActive) {
#pragma unroll
            for (int m = 0; m < R; ++m) epi(b * M + j + m * S, v[m]);
        } else {
#pragma unroll
            for (int m = 0; m < R; ++m) p[m * STRIDE] = v[m];
        }
    }
}

// Last forward pass, matched filter, first inverse pass: blocks of R contiguous positions
// (span 1, no twiddles), all in registers.  mf is transposed: position b*R + q at q*(L/R) + b.
template <int L>
ASARF_HD ASARF_INLINE void ct_middle(float2* s, const float2* __restrict__ mf, int t) {
    constexpr int NTHR = CtSchedule<L>::nthr;
    constexpr int R = ct_padq<L>();
    constexpr int ITEMS = L / R;
    constexpr int PER = (ITEMS + NTHR - 1) / NTHR;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int b = t + k * NTHR;
        if (ITEMS % NTHR != 0 && b >= ITEMS) break;
        float2* p = s + b * (R + 1);  // padded position of b * R
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = p[m];
        dft_any<R, false>(v);
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = cmul(v[q], ASARF_LDG(mf + q * ITEMS + b));
        dft_any<R, true>(v);
#pragma unroll
        for (int m = 0; m < R; ++m) p[m] = v[m];
    }
}

// Forward transform, matched filter, inverse transform of the padded tile s (natural order
// in, unscaled); the last pass hands its outputs to epi (natural position, value) and ends
// without a barrier, every other pass ends with one.
template <int L, class Epi>
ASARF_HD ASARF_INLINE void ct_fft_mf_ifft(float2* s, const float2* __restrict__ ctw, const float2* __restrict__ mf,
                                          int tid, const Epi& epi) {
    constexpr int NTHR = CtSchedule<L>::nthr;
    static_assert(CtSchedule<L>::count == 3, "three-pass schedules");
    static_assert(Epi::kActive, "the last pass writes through its epilogue");
    ct_phase<NTHR>([&](int t) { ct_pass<L, 0, false>(s, ctw, t); }, tid);
    ct_phase<NTHR>([&](int t) { ct_pass<L, 1, false>(s, ctw, t); }, tid);
    ct_phase<NTHR>([&](int t) { ct_middle<L>(s, mf, t); }, tid);
    ct_phase<NTHR>([&](int t) { ct_pass<L, 1, true>(s, ctw, t); }, tid);
    ct_phase<NTHR, false>([&](int t) { ct_pass<L, 0, true>(s, ctw, t, epi); }, tid);
}

}  // namespace asarf
