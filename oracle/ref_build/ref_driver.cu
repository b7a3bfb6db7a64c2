// Test harness around the REFERENCE's own focusing code (asar-focus sar/ + cuda_util/ +
// envisat_format_kernels.cu, compiled from their source files for sm_100a with cuFFT).
//
// TEST INFRASTRUCTURE ONLY: used to pin the CPU oracle and as the reference arm of the
// benchmark.  It replays the host flow of main.cc:176-327 for a synthetic ERS byte-I/Q
// scene, calling the reference functions; the steps main.cc takes through code that
// needs Boost/GDAL/Eigen (metadata assembly, results window, subsetting, polynomial fit,
// geolocation) are written here from the same rules.
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "asarf.h"  // asarf_scene: plain C description of the synthetic scene
#include "cuda_util/cuda_algorithm.h"
#include "cuda_util/cuda_workplace.h"
#include "cuda_util/cufft_plan.h"
#include "cuda_util/device_padded_image.cuh"
#include "envisat_format/include/envisat_format_kernels.h"
#include "sar/az_multilook.cuh"
#include "sar/focussing_details.h"
#include "sar/fractional_doppler_centroid.cuh"
#include "sar/iq_correction.cuh"
#include "sar/range_compression.cuh"
#include "sar/range_doppler_algorithm.cuh"
#include "sar/range_spreading_loss.cuh"
#include "sar/sar_chirp.h"
#include "sar/sar_metadata.h"
#include "sar/srgr.cuh"

// ---------------------------------------------------------------- Eigen-free helpers the
// reference sources link against (declared in util/include/math_utils.h, geo_tools.h)

std::vector<double> Polyfit(const std::vector<double>& x, const std::vector<double>& y, int degree) {
    // Householder QR least squares, coefficients highest power first
    const int m = static_cast<int>(x.size()), n = degree + 1;
    std::vector<double> A(static_cast<size_t>(m) * n), b(y);
    for (int r = 0; r < m; ++r) {
        double v = 1.0;
        for (int c = 0; c < n; ++c) {
            A[c * m + r] = v;
            v *= x[r];
        }
    }
    for (int k = 0; k < n; ++k) {
        double nrm = 0;
        for (int r = k; r < m; ++r) nrm += A[k * m + r] * A[k * m + r];
        nrm = std::sqrt(nrm);
        const double alpha = A[k * m + k] > 0 ? -nrm : nrm;
        std::vector<double> v(m, 0.0);
        for (int r = k; r < m; ++r) v[r] = A[k * m + r];
        v[k] -= alpha;
        double vn = 0;
        for (int r = k; r < m; ++r) vn += v[r] * v[r];
        for (int c = k; c < n; ++c) {
            double d = 0;
            for (int r = k; r < m; ++r) d += v[r] * A[c * m + r];
            for (int r = k; r < m; ++r) A[c * m + r] -= 2 * d / vn * v[r];
        }
        double d = 0;
        for (int r = k; r < m; ++r) d += v[r] * b[r];
        for (int r = k; r < m; ++r) b[r] -= 2 * d / vn * v[r];
    }
    std::vector<double> c(n);
    for (int k = n - 1; k >= 0; --k) {
        double s = b[k];
        for (int j = k + 1; j < n; ++j) s -= A[j * m + k] * c[j];
        c[k] = s / A[k * m + k];
    }
    return {c.rbegin(), c.rend()};
}

GeoPos3D RangeDopplerGeoLocate(Velocity3D v, GeoPos3D p, GeoPos3D g, double slant_range) {
    const double a = 6378137.0, b = 6356752.314245;
    double r[3] = {g.x, g.y, g.z};
    for (int it = 1; it <= 101; ++it) {
        double pv[3] = {r[0] - p.x, r[1] - p.y, r[2] - p.z};
        double M[3][4] = {{v.x, v.y, v.z, -(v.x * pv[0] + v.y * pv[1] + v.z * pv[2])},
                          {2 * pv[0], 2 * pv[1], 2 * pv[2],
                           -(pv[0] * pv[0] + pv[1] * pv[1] + pv[2] * pv[2] - slant_range * slant_range)},
                          {2 * r[0] / (a * a), 2 * r[1] / (a * a), 2 * r[2] / (b * b),
                           -(std::pow(r[0] / a, 2.0) + std::pow(r[1] / a, 2.0) + std::pow(r[2] / b, 2.0) - 1.0)}};
        for (int c = 0; c < 3; ++c) {
            int piv = c;
            for (int q = c + 1; q < 3; ++q)
                if (std::fabs(M[q][c]) > std::fabs(M[piv][c])) piv = q;
            for (int j = 0; j < 4; ++j) std::swap(M[c][j], M[piv][j]);
            for (int q = c + 1; q < 3; ++q) {
                const double f = M[q][c] / M[c][c];
                for (int j = c; j < 4; ++j) M[q][j] -= f * M[c][j];
            }
        }
        double dx[3];
        for (int i = 2; i >= 0; --i) {
            double s = M[i][3];
            for (int j = i + 1; j < 3; ++j) s -= M[i][j] * dx[j];
            dx[i] = s / M[i][i];
        }
        for (int k = 0; k < 3; ++k) r[k] += dx[k];
        if (std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) < 1e-6) return {r[0], r[1], r[2]};
    }
    throw std::runtime_error("Failed to converge for RangeDopplerGeoLocate");
}

// The reference's ERS decode kernel (envisat_format/src/envisat_format_kernels.cu:116-134),
// launched here directly on device-resident raw bytes with the grid its host wrapper uses
// (the wrapper itself always copies from host memory).
namespace alus::asar::envformat {
__global__ void ConvertErsImSamplesToComplexKernel(const uint8_t* samples, int samples_range_size_bytes, int packets,
                                                   const uint16_t* swst_codes, uint16_t min_swst,
                                                   cufftComplex* target_buf, int target_range_width);
}

// ---------------------------------------------------------------- harness entry point

extern "C" {

typedef struct ref_outputs {
    double dc_i, dc_q, iq_gain, phase_error, stddev_i, stddev_q;
    double dc_poly[3];
    double grsr_poly[5];
    int32_t first_line, n_lines, slc_cols, out_rows, out_cols, max_aperture;
    double ms_total;          // device time, host raw bytes -> SRGR output on the device (events)
    double ms_after_decode;   // same, from the end of the raw decode (its H2D excluded)
    double ms_wall;           // host wall clock of the whole call
    char error[256];
    // with ref_set_statistics(1): CalculateStatistics of the subset (main.cc:380) and
    // CalculateStatisticsImaged of the ground-range buffer (main.cc:327-333), unscaled
    double ims_stats[4];
    double imp_stats[4];
} ref_outputs;

static int g_statistics = 0;
void ref_set_statistics(int on) { g_statistics = on; }

// Runs the reference chain; optional host dumps (NULL to skip):
//   corrected [na][nr] complex (after RawDataCorrection + ZeroNaNs), rc [na][nk] complex,
//   slc [n_lines][nk-16] complex, ml [out_rows][nk-16] float (after RSL).
// d_raw (optional): device copy of the raw bytes; when given the timed region starts from
// device-resident input (decode kernel launched directly), otherwise from host memory
// through the reference's own ConvertErsImSamplesToComplex (which copies internally).
int ref_focus(const asarf_scene* s, const double vr_poly[3], const uint8_t* h_raw, const uint16_t* h_swst,
              float* h_out, int64_t out_capacity, ref_outputs* o, float* h_corrected, float* h_rc, float* h_slc,
              float* h_ml, const uint8_t* d_raw) {
    std::memset(o, 0, sizeof(*o));
    try {
        auto wall0 = std::chrono::steady_clock::now();
        const int nr = s->range_size, na = s->azimuth_size, nc = s->chirp_samples;
        SARMetadata meta{};
        meta.chirp.range_sampling_rate = s->range_sampling_rate;
        meta.chirp.pulse_duration = s->pulse_duration;
        meta.chirp.n_samples = nc;
        meta.chirp.Kr = s->chirp_kr;
        meta.chirp.apply_window = s->apply_window != 0;
        meta.img.range_size = nr;
        meta.img.azimuth_size = na;
        meta.pulse_repetition_frequency = s->prf;
        meta.line_time_interval = 1.0 / s->prf;
        meta.azimuth_bandwidth_fraction = s->az_bw_frac;
        meta.azimuth_window = false;
        meta.carrier_frequency = s->carrier_frequency;
        meta.wavelength = s->wavelength;
        meta.range_spacing = s->range_spacing;
        meta.azimuth_spacing = s->azimuth_spacing;
        meta.slant_range_first_sample = s->slant_range_first;
        meta.first_line_time.us = s->first_line_time_us;
        for (int i = 0; i < s->n_osv; ++i) {
            OrbitStateVector v{};
            v.time.us = s->osv[i].time_us;
            v.x_pos = s->osv[i].pos[0];
            v.y_pos = s->osv[i].pos[1];
            v.z_pos = s->osv[i].pos[2];
            v.x_vel = s->osv[i].vel[0];
            v.y_vel = s->osv[i].vel[1];
            v.z_vel = s->osv[i].vel[2];
            meta.osv.push_back(v);
        }
        meta.center_point = {s->center_point[0], s->center_point[1], s->center_point[2]};
        meta.total_raw_samples = static_cast<size_t>(s->total_raw_samples);
        meta.results.Vr_poly = {s->vr_poly_init[0], s->vr_poly_init[1], s->vr_poly_init[2]};

        std::vector<uint16_t> swst(na, 0);
        uint16_t min_swst = 0;
        if (h_swst) {
            swst.assign(h_swst, h_swst + na);
            min_swst = *std::min_element(swst.begin(), swst.end());
        }

        cudaEvent_t e0, e1, e2;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventCreate(&e2);
        uint16_t* d_swst = nullptr;
        if (d_raw) {
            CHECK_CUDA_ERR(cudaMalloc(&d_swst, sizeof(uint16_t) * na));
            CHECK_CUDA_ERR(cudaMemcpy(d_swst, swst.data(), sizeof(uint16_t) * na, cudaMemcpyHostToDevice));
        }
        cudaEventRecord(e0);
        // ConvertRawSampleSetsToComplex (main_flow.cc:530-583), ERS path
        cufftComplex* d_parsed = nullptr;
        CHECK_CUDA_ERR(cudaMalloc(&d_parsed, sizeof(cufftComplex) * static_cast<size_t>(nr) * na));
        alus::cuda::algorithm::Fill(d_parsed, static_cast<size_t>(nr) * na, cufftComplex{NAN, NAN});
        if (s->raw_format == ASARF_RAW_ASAR_FBAQ4) {
            // ASA_IM0 branch of ConvertRawSampleSetsToComplex (main_flow.cc:566-575), host records
            alus::asar::envformat::ConvertAsarImBlocksToComplex(h_raw, s->raw_line_bytes, na, swst.data(), min_swst,
                                                               d_parsed, nr, s->fbaq_i_lut, s->fbaq_q_lut, 4096);
        } else if (d_raw) {
            const int x_size = 11232;  // ers::highrate::MEASUREMENT_DATA_SIZE_BYTES, as the wrapper sizes its grid
            dim3 block(16, 16), grid((x_size + 15) / 16, (na + 15) / 16);
            alus::asar::envformat::ConvertErsImSamplesToComplexKernel<<<grid, block>>>(
                d_raw, 2 * s->samples_per_line, na, d_swst, min_swst, d_parsed, nr);
            CHECK_CUDA_ERR(cudaGetLastError());
        } else {
            alus::asar::envformat::ConvertErsImSamplesToComplex(h_raw, s->samples_per_line, na, swst.data(),
                                                               min_swst, d_parsed, nr);
        }
        cudaEventRecord(e1);
        // main.cc:213-245
        const auto fft_sizes = GetOptimalFFTSizes();
        const int rg_padded = fft_sizes.upper_bound(nr + nc)->first;
        const int az_padded = fft_sizes.upper_bound(na)->first;
        DevicePaddedImage img;
        img.InitPadded(nr, na, rg_padded, az_padded);
        img.ZeroMemory();
        CHECK_CUDA_ERR(cudaMemcpy2D(img.Data(), rg_padded * 8, d_parsed, nr * 8, nr * 8, na, cudaMemcpyDeviceToDevice));
        CHECK_CUDA_ERR(cudaFree(d_parsed));
        RawDataCorrection(img, {meta.total_raw_samples}, meta.results);
        img.ZeroNaNs();
        if (h_corrected)
            CHECK_CUDA_ERR(cudaMemcpy2D(h_corrected, nr * 8, img.Data(), rg_padded * 8, nr * 8, na, cudaMemcpyDeviceToHost));
        // main.cc:251-259: aperture (initial Vr guess, DC not yet known), Vr, chirp, DC
        auto aperture_pixels = CalcAperturePixels(meta);
        meta.results.Vr_poly = {vr_poly[0], vr_poly[1], vr_poly[2]};
        GenerateChirpData(meta.chirp, rg_padded);
        meta.results.doppler_centroid_poly = CalculateDopplerCentroid(img, meta.pulse_repetition_frequency);
        // main.cc:269-287
        CudaWorkspace d_workspace(img.TotalByteSize());
        RangeCompression(img, meta.chirp.padded_windowed_data, meta.chirp.n_samples, d_workspace);
        meta.img.range_size = img.XSize();
        const int nk = img.XSize();
        if (h_rc)
            CHECK_CUDA_ERR(cudaMemcpy2D(h_rc, nk * 8, img.Data(), rg_padded * 8, nk * 8, na, cudaMemcpyDeviceToHost));
        DevicePaddedImage az_img;
        RangeDopplerAlgorithm(meta, img, az_img, d_workspace);
        const auto rcmc = alus::sar::focus::GetRcmcParameters();
        az_img.ZeroFillPaddings();
        // CalcResultsWindow (main_flow.cc:155-201)
        size_t max_ap = 0;
        for (auto a : aperture_pixels) max_ap = std::max(max_ap, a);
        const double dc0 = meta.results.doppler_centroid_poly.back();
        const size_t before = s->lines_before, after = s->lines_after;
        size_t after_start = 0, before_stop = 0;
        if (dc0 > 0) {
            if (before < max_ap) after_start = max_ap - before;
        } else {
            if (after < max_ap) before_stop = max_ap - after;
        }
        const int near = static_cast<int>(rcmc.window_size / 2), far = static_cast<int>(rcmc.window_size / 2);
        CHECK_CUDA_ERR(cudaDeviceSynchronize());
        // SubsetResultsAndReassembleMeta (main_flow.cc:585-632)
        const int first = static_cast<int>(before + after_start);
        const int lines = na - first - static_cast<int>(before_stop + after);
        const int cols = az_img.XSize() - (near + far);
        DevicePaddedImage sub;
        CHECK_CUDA_ERR(cudaMemcpy2D(d_workspace.Get(), cols * 8,
                                    az_img.Data() + static_cast<size_t>(first) * az_img.XStride() + near,
                                    az_img.XStride() * 8, cols * 8, lines, cudaMemcpyDeviceToDevice));
        sub.InitExtPtr(cols, lines, cols, lines, d_workspace);
        d_workspace = az_img.ReleaseMemory();
        if (h_slc) CHECK_CUDA_ERR(cudaMemcpy(h_slc, sub.Data(), static_cast<size_t>(cols) * lines * 8, cudaMemcpyDeviceToHost));
        if (g_statistics) {
            // CalculateStatistics (main_flow.cc:666-670)
            const auto m = sub.CalcMean();
            const auto d = sub.CalcStdDev(m.x, m.y);
            o->ims_stats[0] = m.x;
            o->ims_stats[1] = m.y;
            o->ims_stats[2] = d.x;
            o->ims_stats[3] = d.y;
        }
        // AssembleMetadataFrom(..., range_pixels_recalib = near): slant range of the new first sample
        meta.slant_range_first_sample = CalcSlantRange(meta, near);
        meta.img.range_size = cols;
        meta.img.azimuth_size = lines;
        meta.line_time_interval = 1.0 / meta.pulse_repetition_frequency;
        // IMP tail (main.cc:320-327)
        AzimuthMultiLook(sub, d_workspace, meta);
        RangeSpreadingLossCorrection(d_workspace.GetAs<float>(), meta.img.range_size, meta.img.azimuth_size,
                                     {meta.slant_range_first_sample, meta.range_spacing, 800000.0});
        if (h_ml)
            CHECK_CUDA_ERR(cudaMemcpy(h_ml, d_workspace.GetAs<float>(),
                                      sizeof(float) * meta.img.range_size * meta.img.azimuth_size,
                                      cudaMemcpyDeviceToHost));
        auto srgr_dest = sub.ReleaseMemory();
        SlantRangeToGroundRangeInterpolation(meta, d_workspace.GetAs<float>(), srgr_dest.GetAs<float>());
        if (g_statistics) {
            // main.cc:327-333: the ground-range buffer viewed as a complex image of its size
            DevicePaddedImage stats_image;
            stats_image.InitExtPtr(meta.img.range_size, meta.img.azimuth_size, meta.img.range_size,
                                   meta.img.azimuth_size, srgr_dest);
            const auto m = stats_image.CalcMean();
            const auto d = stats_image.CalcStdDev(m.x, m.y);
            o->imp_stats[0] = (m.x + m.y) / 2;
            o->imp_stats[2] = (d.x + d.y) / 2;
            srgr_dest = stats_image.ReleaseMemory();
        }
        cudaEventRecord(e2);
        CHECK_CUDA_ERR(cudaEventSynchronize(e2));
        float ms0 = 0, ms1 = 0;
        cudaEventElapsedTime(&ms0, e0, e2);
        cudaEventElapsedTime(&ms1, e1, e2);
        const int64_t n_out = static_cast<int64_t>(meta.img.range_size) * meta.img.azimuth_size;
        if (h_out && n_out <= out_capacity)
            CHECK_CUDA_ERR(cudaMemcpy(h_out, srgr_dest.GetAs<float>(), sizeof(float) * n_out, cudaMemcpyDeviceToHost));
        auto wall1 = std::chrono::steady_clock::now();
        o->dc_i = meta.results.dc_i;
        o->dc_q = meta.results.dc_q;
        o->iq_gain = meta.results.iq_gain;
        o->phase_error = meta.results.phase_error;
        o->stddev_i = meta.results.stddev_i;
        o->stddev_q = meta.results.stddev_q;
        for (int k = 0; k < 3; ++k) o->dc_poly[k] = meta.results.doppler_centroid_poly[k];
        for (int k = 0; k < 5 && k < static_cast<int>(meta.srgr.grsr_poly.size()); ++k) o->grsr_poly[k] = meta.srgr.grsr_poly[k];
        o->first_line = first;
        o->n_lines = lines;
        o->slc_cols = cols;
        o->out_rows = meta.img.azimuth_size;
        o->out_cols = meta.img.range_size;
        o->max_aperture = static_cast<int>(max_ap);
        o->ms_total = ms0;
        o->ms_after_decode = ms1;
        o->ms_wall = std::chrono::duration<double, std::milli>(wall1 - wall0).count();
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        if (d_swst) cudaFree(d_swst);
        if (h_out && n_out > out_capacity) {
            std::snprintf(o->error, sizeof(o->error), "output needs %lld floats", static_cast<long long>(n_out));
            return -1;
        }
        return 0;
    } catch (const std::exception& e) {
        std::snprintf(o->error, sizeof(o->error), "%s", e.what());
        return -2;
    }
}

// The reference's level-1 record conditioning on host inputs: ConditionResultsSLC over a padded
// complex image [y_size][x_stride] (XSize x_size) and ConditionResultsDetected over a float
// image [azimuth_size][range_size]; the records are copied back.
int ref_condition_slc(const float* h_img, int32_t x_size, int32_t y_size, int32_t x_stride, int32_t hdr, float cal,
                      uint8_t* h_out) {
    try {
        const size_t in_bytes = sizeof(cufftComplex) * static_cast<size_t>(x_stride) * y_size;
        const size_t out_bytes = static_cast<size_t>(y_size) * (static_cast<size_t>(hdr) + 4ull * x_size);
        CudaWorkspace ws(in_bytes);
        CHECK_CUDA_ERR(cudaMemcpy(ws.Get(), h_img, in_bytes, cudaMemcpyHostToDevice));
        DevicePaddedImage img;
        img.InitExtPtr(x_size, y_size, x_stride, y_size, ws);
        char* d_out = nullptr;
        CHECK_CUDA_ERR(cudaMalloc(&d_out, out_bytes));
        alus::asar::envformat::ConditionResultsSLC(img, d_out, hdr, cal);
        CHECK_CUDA_ERR(cudaMemcpy(h_out, d_out, out_bytes, cudaMemcpyDeviceToHost));
        CHECK_CUDA_ERR(cudaFree(d_out));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref_condition_detected(const float* h_img, int32_t range_size, int32_t azimuth_size, int32_t hdr, float cal,
                           uint8_t* h_out) {
    try {
        const size_t in_bytes = sizeof(float) * static_cast<size_t>(range_size) * azimuth_size;
        const size_t out_bytes = static_cast<size_t>(azimuth_size) * (static_cast<size_t>(hdr) + 2ull * range_size);
        float* d_in = nullptr;
        char* d_out = nullptr;
        CHECK_CUDA_ERR(cudaMalloc(&d_in, in_bytes));
        CHECK_CUDA_ERR(cudaMalloc(&d_out, out_bytes));
        CHECK_CUDA_ERR(cudaMemcpy(d_in, h_img, in_bytes, cudaMemcpyHostToDevice));
        alus::asar::envformat::ConditionResultsDetected(d_in, d_out, range_size, azimuth_size, hdr, cal);
        CHECK_CUDA_ERR(cudaMemcpy(h_out, d_out, out_bytes, cudaMemcpyDeviceToHost));
        CHECK_CUDA_ERR(cudaFree(d_in));
        CHECK_CUDA_ERR(cudaFree(d_out));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// The reference's ASAR FBAQ4 decode alone: NaN-filled device image (main_flow.cc:537-540),
// ConvertAsarImBlocksToComplex from host records and tables, copied back as [records][range_size].
int ref_convert_asar(const uint8_t* h_raw, int32_t record_bytes, int32_t records, const uint16_t* h_swst,
                     const float* i_lut, const float* q_lut, int32_t range_size, float* h_out) {
    try {
        std::vector<uint16_t> swst(records, 0);
        if (h_swst) swst.assign(h_swst, h_swst + records);
        const uint16_t min_swst = *std::min_element(swst.begin(), swst.end());
        const size_t n = static_cast<size_t>(range_size) * records;
        cufftComplex* d = nullptr;
        CHECK_CUDA_ERR(cudaMalloc(&d, sizeof(cufftComplex) * n));
        alus::cuda::algorithm::Fill(d, n, cufftComplex{NAN, NAN});
        alus::asar::envformat::ConvertAsarImBlocksToComplex(h_raw, record_bytes, records, swst.data(), min_swst, d,
                                                           range_size, i_lut, q_lut, 4096);
        CHECK_CUDA_ERR(cudaMemcpy(h_out, d, sizeof(cufftComplex) * n, cudaMemcpyDeviceToHost));
        CHECK_CUDA_ERR(cudaFree(d));
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

}  // extern "C"
