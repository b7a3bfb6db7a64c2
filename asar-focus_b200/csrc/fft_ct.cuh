// Compile-time-scheduled line FFTs for the range compression kernel.
//
// The range FFT length is a free choice (any L >= range size gives the same compressed
// samples), so the planner picks it from the lengths below and the whole transform is
// instantiated with constant radices, spans and per-thread item counts: every index
// computation folds to shifts and constant multiplies.  The radix order is the runtime
// factoriser's (host.cpp `factorize`), so the digit-reversed output order - and with it the
// matched-filter table - is identical to the generic path's.
#pragma once

#include "fft.cuh"
#include "hd.cuh"

namespace asarf {

template <int L>
struct CtSchedule {
    static constexpr int count = 0;
};
#define ASARF_CT_SCHEDULE(LEN, NT, ...)                   \
    template <>                                           \
    struct CtSchedule<LEN> {                              \
        static constexpr int r[] = {__VA_ARGS__};         \
        static constexpr int count = sizeof(r) / sizeof(int); \
        static constexpr int nthr = NT;                   \
    }
ASARF_CT_SCHEDULE(768, 256, 8, 8, 4, 3);
ASARF_CT_SCHEDULE(1024, 256, 8, 8, 8, 2);
ASARF_CT_SCHEDULE(1536, 256, 8, 8, 8, 3);
ASARF_CT_SCHEDULE(2048, 256, 8, 8, 8, 4);
ASARF_CT_SCHEDULE(3072, 384, 8, 8, 8, 2, 3);
ASARF_CT_SCHEDULE(4096, 512, 8, 8, 8, 8);
ASARF_CT_SCHEDULE(6144, 512, 8, 8, 8, 4, 3);
ASARF_CT_SCHEDULE(8192, 512, 8, 8, 8, 8, 2);
#undef ASARF_CT_SCHEDULE

constexpr int kCtLengths[] = {768, 1024, 1536, 2048, 3072, 4096, 6144, 8192};

template <int L, int I>
ASARF_HD constexpr int ct_span() {
    int m = L;
    for (int k = 0; k <= I; ++k) m /= CtSchedule<L>::r[k];
    return m;
}

// Run `phase(tid)` for this thread and barrier (device), or for every thread in turn (host
// emulation, where a phase must complete for all threads before the next one starts).
template <int NTHR, class F>
ASARF_HD ASARF_INLINE void ct_phase(F&& phase, int tid) {
#if defined(__CUDA_ARCH__)
    phase(tid);
    __syncthreads();
#else
    (void)tid;
    for (int t = 0; t < NTHR; ++t) phase(t);
#endif
}

template <int L, int NTHR, int R, int S, bool INV, bool DIT>
ASARF_HD ASARF_INLINE void ct_stage(float2* s, const float2* __restrict__ tw, int tid) {
    constexpr int M = S * R;
    constexpr int ITEMS = L / R;
    constexpr int TW_STEP = L / M;
    constexpr int PER = (ITEMS + NTHR - 1) / NTHR;
#pragma unroll
    for (int k = 0; k < PER; ++k) {
        const int t = tid + k * NTHR;
        if (ITEMS % NTHR != 0 && t >= ITEMS) break;
        const int b = t / S;
        const int j = t - b * S;
        float2* p = s + b * M + j;
        float2 v[R];
#pragma unroll
        for (int m = 0; m < R; ++m) v[m] = p[m * S];
        if (DIT) {  // inverse, decimation in time: twiddle inputs, then the small DFT
            if (j != 0) {
                const float2 w1 = ASARF_LDG(tw + j * TW_STEP);
                float2 w = w1;
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    v[q] = cmulc(v[q], w);
                    w = cmul(w, w1);
                }
            }
            dft<R, true>(v);
        } else {  // forward, decimation in frequency: small DFT, then twiddle outputs
            dft<R, INV>(v);
            if (j != 0) {
                const float2 w1 = ASARF_LDG(tw + j * TW_STEP);
                float2 w = w1;
#pragma unroll
                for (int q = 1; q < R; ++q) {
                    v[q] = INV ? cmulc(v[q], w) : cmul(v[q], w);
                    w = cmul(w, w1);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < R; ++m) p[m * S] = v[m];
    }
}

template <int L, int I>
ASARF_HD ASARF_INLINE void ct_forward_from(float2* s, const float2* __restrict__ tw, int tid) {
    if constexpr (I < CtSchedule<L>::count) {
        constexpr int NTHR = CtSchedule<L>::nthr;
        ct_phase<NTHR>([&](int t) { ct_stage<L, NTHR, CtSchedule<L>::r[I], ct_span<L, I>(), false, false>(s, tw, t); },
                       tid);
        ct_forward_from<L, I + 1>(s, tw, tid);
    }
}

template <int L, int I>
ASARF_HD ASARF_INLINE void ct_inverse_from(float2* s, const float2* __restrict__ tw, int tid) {
    if constexpr (I >= 0) {
        constexpr int NTHR = CtSchedule<L>::nthr;
        ct_phase<NTHR>([&](int t) { ct_stage<L, NTHR, CtSchedule<L>::r[I], ct_span<L, I>(), true, true>(s, tw, t); },
                       tid);
        ct_inverse_from<L, I - 1>(s, tw, tid);
    }
}

// Forward DIF (natural -> digit-reversed) and inverse DIT (digit-reversed -> natural).
template <int L>
ASARF_HD ASARF_INLINE void ct_fft_forward(float2* s, const float2* __restrict__ tw, int tid) {
    ct_forward_from<L, 0>(s, tw, tid);
}
template <int L>
ASARF_HD ASARF_INLINE void ct_fft_inverse(float2* s, const float2* __restrict__ tw, int tid) {
    ct_inverse_from<L, CtSchedule<L>::count - 1>(s, tw, tid);
}

}  // namespace asarf
