// Host-side helpers shared by the planner (host.cpp) and the per-stage entry points (stages.cpp).
#pragma once

#include <complex>
#include <vector>

#include "asarf.h"
#include "fft.cuh"

namespace asarf {

// FFT schedule of one length with its digit-reversal map and FP64-computed twiddles.
struct HostFft {
    FftPlan plan{};
    std::vector<int> drev;
    std::vector<float2> tw;
};

bool smooth(int n);
// Longest synthetic aperture in lines over the range swath (CalcAperturePixels).
int max_aperture_pixels(const asarf_scene& s);
// Ground-to-slant SRGR polynomial (5 coefficients) and ground sample count for a multilooked
// block of azimuth_size lines at line interval lti (SlantRangeToGroundRangeInterpolation setup).
int srgr_poly(const asarf_scene& s, double slant_first, int range_size, int azimuth_size, double lti, double poly[5],
              int* ng);
bool build_fft(int n, HostFft& h);
// Same with an explicit radix sequence (product n), e.g. a compile-time schedule's.
bool build_fft_radices(int n, const std::vector<int>& radices, HostFft& h);
// radices of the strided azimuth pass: pairs of 3s merged into radix 9
std::vector<int> strided_radices(int n);
int choose_rc_len(int nr);
int32_t fft_size_above(int32_t v);
void matched_filter_table(const std::complex<float>* chirp, int nc, const HostFft& fft, std::vector<float2>& mf);

}  // namespace asarf
