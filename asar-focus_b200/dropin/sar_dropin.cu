// Header-compatible drop-in for the reference's GPU focusing stages.
//
// Defines the functions the reference declares in its sar/ headers, with the reference's own
// signatures and container types (DevicePaddedImage, CudaWorkspace, SARMetadata), on top of
// the per-stage entry points of libasarf (include/asarf.h).  A build of the reference that
// compiles this file in place of sar/iq_correction.cu, sar/fractional_doppler_centroid.cu,
// sar/range_compression.cu, sar/range_doppler_algorithm.cu, sar/az_multilook.cu,
// sar/range_spreading_loss.cu and sar/srgr.cu, and links libasarf.so instead of cuFFT, runs
// main.cc unchanged.  Everything else of the reference (decode, chirp generation, Vr
// estimation, the containers themselves) stays its own.
//
// Errors follow the reference: argument errors it throws as std::logic_error are thrown as
// std::logic_error with the same text, CUDA failures as alus::CudaErrorException, and the
// checks it makes with CHECK_BOOL use CHECK_BOOL.
#include <complex>
#include <stdexcept>
#include <string>
#include <vector>

#include "asarf.h"
#include "checks.h"
#include "cuda_util/cuda_util.h"
#include "cuda_util/cuda_workplace.h"
#include "cuda_util/device_padded_image.cuh"
#include "sar/az_multilook.cuh"
#include "sar/focussing_details.h"
#include "sar/fractional_doppler_centroid.cuh"
#include "sar/iq_correction.cuh"
#include "sar/range_compression.cuh"
#include "sar/range_doppler_algorithm.cuh"
#include "sar/range_spreading_loss.cuh"
#include "sar/sar_metadata.h"
#include "sar/srgr.cuh"

namespace {

void check(int rc) {
    if (rc == ASARF_OK) return;
    const std::string msg = asarf_last_error();
    if (rc == ASARF_ERR_CUDA || rc == ASARF_ERR_NOMEM) throw alus::CudaErrorException(msg);
    if (rc == ASARF_ERR_INVALID) throw std::logic_error(msg);
    throw std::runtime_error(msg);
}

}  // namespace

// sar/focussing_details.h:28: the RCMC interpolator length (16 taps, as the reference's)
namespace alus::sar::focus {
RcmcParameters GetRcmcParameters() {
    RcmcParameters params{};
    params.window_size = 16;
    return params;
}
}  // namespace alus::sar::focus

// sar/iq_correction.cuh:26
void RawDataCorrection(DevicePaddedImage& img, CorrectionParams par, SARResults& results) {
    asarf_iq_results r{};
    check(asarf_raw_data_correction(img.Data(), img.XSize(), img.YSize(), img.XStride(), img.YStride(),
                                    static_cast<int64_t>(par.n_total_samples), &r, nullptr));
    results.dc_i = r.dc_i;
    results.dc_q = r.dc_q;
    results.iq_gain = r.iq_gain;
    results.phase_error = r.phase_error;
    results.stddev_i = r.stddev_i;
    results.stddev_q = r.stddev_q;
}

// sar/fractional_doppler_centroid.cuh:23
std::vector<double> CalculateDopplerCentroid(const DevicePaddedImage& d_img, double prf) {
    double poly[3];
    check(asarf_doppler_centroid(d_img.Data(), d_img.XSize(), d_img.YSize(), d_img.XStride(), prf, poly, nullptr));
    return {poly[0], poly[1], poly[2]};
}

// sar/range_compression.cuh:27-28
void RangeCompression(DevicePaddedImage& data, const std::vector<std::complex<float>>& chirp_data, int chirp_samples,
                      CudaWorkspace& d_workspace) {
    (void)d_workspace;  // the transform runs in shared memory: no work area
    int32_t new_x = 0;
    check(asarf_range_compression(data.Data(), data.XSize(), data.YSize(), data.XStride(),
                                  reinterpret_cast<const float*>(chirp_data.data()),
                                  static_cast<int32_t>(chirp_data.size()), chirp_samples, &new_x, nullptr));
    data.SetXSize(new_x);
}

// sar/range_doppler_algorithm.cuh:28-29: out_img takes the workspace memory, and the
// workspace takes src_img's memory on return, as in the reference.
void RangeDopplerAlgorithm(const SARMetadata& metadata, DevicePaddedImage& src_img, DevicePaddedImage& out_img,
                           CudaWorkspace& d_workspace) {
    const auto& vr = metadata.results.Vr_poly;
    const auto& dc = metadata.results.doppler_centroid_poly;
    CHECK_BOOL(vr.size() == 3);
    CHECK_BOOL(dc.size() == 3);
    asarf_rda_params prm{};
    prm.prf = metadata.pulse_repetition_frequency;
    prm.wavelength = metadata.wavelength;
    prm.range_spacing = metadata.range_spacing;
    prm.slant_range_first = metadata.slant_range_first_sample;
    prm.az_bw_frac = metadata.azimuth_bandwidth_fraction;
    for (int k = 0; k < 3; ++k) {
        prm.vr_poly[k] = vr[k];
        prm.dc_poly[k] = dc[k];
    }
    out_img.InitExtPtr(src_img.XSize(), src_img.YSize(), src_img.XStride(), src_img.YStride(), d_workspace);
    check(asarf_range_doppler(&prm, src_img.Data(), out_img.Data(), src_img.XSize(), src_img.YSize(),
                              src_img.XStride(), src_img.YStride(), nullptr));
    d_workspace = src_img.ReleaseMemory();
}

// sar/az_multilook.cuh:24
void AzimuthMultiLook(const DevicePaddedImage& d_slc, CudaWorkspace& out, SARMetadata& sar_meta) {
    CHECK_BOOL(d_slc.XSize() == d_slc.XStride());
    const float ratio = 12.5f / sar_meta.azimuth_spacing;
    int32_t out_y = 0;
    check(asarf_azimuth_multilook(d_slc.Data(), d_slc.XSize(), d_slc.YSize(), sar_meta.azimuth_spacing,
                                  out.GetAs<float>(), &out_y, nullptr));
    sar_meta.azimuth_spacing *= ratio;
    sar_meta.line_time_interval *= ratio;
    sar_meta.img.azimuth_size = out_y;
}

// sar/range_spreading_loss.cuh:25
void RangeSpreadingLossCorrection(float* d_img_data, int range_size, int azimuth_size, RangeSpreadingLossParams params) {
    check(asarf_range_spreading_loss(d_img_data, range_size, azimuth_size, params.slant_range_first,
                                     params.range_spacing, params.reference_range, nullptr));
}

// sar/srgr.cuh:21: the slant-to-ground polynomial from the metadata's orbit and scene centre,
// the resampling, and the metadata updates the reference makes.
void SlantRangeToGroundRangeInterpolation(SARMetadata& sar_meta, const float* d_slant_in, float* d_gr_out) {
    CHECK_BOOL(!sar_meta.osv.empty());
    const auto t0 = sar_meta.osv.front().time;  // times are passed relative to the first state vector
    std::vector<asarf_osv> osv(sar_meta.osv.size());
    for (size_t i = 0; i < osv.size(); ++i) {
        const auto& v = sar_meta.osv[i];
        osv[i].time_us = (v.time - t0).total_microseconds();
        osv[i].pos[0] = v.x_pos;
        osv[i].pos[1] = v.y_pos;
        osv[i].pos[2] = v.z_pos;
        osv[i].vel[0] = v.x_vel;
        osv[i].vel[1] = v.y_vel;
        osv[i].vel[2] = v.z_vel;
    }
    asarf_scene sc{};
    sc.range_size = sar_meta.img.range_size;
    sc.azimuth_size = sar_meta.img.azimuth_size;
    sc.range_spacing = sar_meta.range_spacing;
    sc.slant_range_first = sar_meta.slant_range_first_sample;
    sc.n_osv = static_cast<int32_t>(osv.size());
    sc.osv = osv.data();
    sc.first_line_time_us = (sar_meta.first_line_time - t0).total_microseconds();
    sc.line_time_interval = sar_meta.line_time_interval;
    sc.center_point[0] = sar_meta.center_point.x;
    sc.center_point[1] = sar_meta.center_point.y;
    sc.center_point[2] = sar_meta.center_point.z;
    double poly[5];
    int32_t ng = 0;
    check(asarf_srgr_polynomial(&sc, sar_meta.slant_range_first_sample, sar_meta.img.range_size,
                                sar_meta.img.azimuth_size, sar_meta.line_time_interval, poly, &ng));
    check(asarf_srgr(d_slant_in, sar_meta.img.range_size, sar_meta.img.azimuth_size, poly, sar_meta.range_spacing, ng,
                     d_gr_out, nullptr));
    sar_meta.srgr.applied = true;
    sar_meta.srgr.grsr_poly.assign(poly, poly + 5);
    sar_meta.range_spacing = 12.5;
    sar_meta.img.range_size = ng;
}
