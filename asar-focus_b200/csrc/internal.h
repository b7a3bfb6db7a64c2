// Host-side helpers shared by the planner (host.cpp) and the per-stage entry points (stages.cpp).
#pragma once

#include <complex>
#include <vector>

#include "fft.cuh"

namespace asarf {

// FFT schedule of one length with its digit-reversal map and FP64-computed twiddles.
struct HostFft {
    FftPlan plan{};
    std::vector<int> drev;
    std::vector<float2> tw;
};

bool smooth(int n);
bool build_fft(int n, HostFft& h);
int choose_rc_len(int nr);
int32_t fft_size_above(int32_t v);
void matched_filter_table(const std::complex<float>* chirp, int nc, const HostFft& fft, std::vector<float2>& mf);

}  // namespace asarf
