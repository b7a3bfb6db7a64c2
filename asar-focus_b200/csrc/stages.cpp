// Per-stage entry points: the reference's sar/ functions one by one, on its padded complex
// image layout (complex float [y_stride][x_stride], data block [0, y_size) x [0, x_size)
// top-left, cuda_util/device_padded_image.cuh:13-27).  Like the reference's functions they
// allocate what they need, copy results to the host where the reference does, and
// synchronise the stream before returning.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"
#include "internal.h"

using namespace asarf;

namespace {

struct DevBuf {
    void* p = nullptr;
    explicit DevBuf(size_t n) : p(mem_alloc(n)) {}
    ~DevBuf() { mem_free(p); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    template <class T>
    T* as() const {
        return static_cast<T*>(p);
    }
};

int nomem() { return set_error(ASARF_ERR_NOMEM, "device allocation failed"); }

// NaN-aware moments of the data block and of the padding columns, summed on the host in a
// fixed order.
int image_moments(const float2* img, int x_size, int y_size, int x_stride, float mean_i, float mean_q, int centered,
                  double out[12], void* stream) {
    const int rpb = 16;
    const int blocks = (y_size + rpb - 1) / rpb;
    DevBuf part(sizeof(double) * 12 * static_cast<size_t>(blocks));
    if (!part.p) return nomem();
    ImgMomentsArgs a{};
    a.img = img;
    a.x_size = x_size;
    a.y_size = y_size;
    a.x_stride = x_stride;
    a.rows_per_block = rpb;
    a.partial = part.as<double>();
    a.mean_i = mean_i;
    a.mean_q = mean_q;
    a.centered = centered;
    int rc = backend_img_moments(a, blocks, stream);
    if (rc) return rc;
    std::vector<double> h(12 * static_cast<size_t>(blocks));
    rc = mem_d2h(h.data(), part.p, sizeof(double) * h.size(), stream);
    if (rc) return rc;
    rc = stream_sync(stream);
    if (rc) return rc;
    for (int k = 0; k < 12; ++k) out[k] = 0.0;
    for (int b = 0; b < blocks; ++b)
        for (int k = 0; k < 12; ++k) out[k] += h[static_cast<size_t>(b) * 12 + k];
    return ASARF_OK;
}

}  // namespace

extern "C" {

int asarf_convert_ers_samples(const uint8_t* d_raw, int32_t raw_line_bytes, int32_t samples_per_line, int32_t lines,
                              const uint16_t* d_swst, int32_t min_swst, void* d_img, int64_t img_stride,
                              int32_t range_size, void* stream) {
    if (!d_raw || !d_img || lines <= 0 || samples_per_line <= 0 || range_size < samples_per_line ||
        img_stride < range_size || raw_line_bytes < 2 * samples_per_line || (raw_line_bytes & 1))
        return set_error(ASARF_ERR_INVALID, "convert_ers_samples: bad arguments");
    DecodeArgs a{};
    a.raw = d_raw;
    a.line_bytes = raw_line_bytes;
    a.spl = samples_per_line;
    a.lines = lines;
    a.nr = range_size;
    a.swst = d_swst;
    a.min_swst = min_swst;
    a.img = static_cast<float2*>(d_img);
    a.stride = img_stride;
    int rc = backend_decode(a, static_cast<long long>(lines) * range_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_convert_asar_blocks(const uint8_t* d_raw, int32_t record_bytes, int32_t records, const uint16_t* d_swst,
                              int32_t min_swst, const float* d_lut_i, const float* d_lut_q, void* d_img,
                              int64_t img_stride, int32_t range_size, void* stream) {
    if (!d_raw || !d_img || !d_lut_i || !d_lut_q || records <= 0 || record_bytes < 2 || range_size <= 0 ||
        img_stride < range_size)
        return set_error(ASARF_ERR_INVALID, "convert_asar_blocks: bad arguments");
    DecodeFbaqArgs a{};
    a.raw = d_raw;
    a.line_bytes = record_bytes;
    a.lines = records;
    a.nr = range_size;
    a.swst = d_swst;
    a.min_swst = min_swst;
    a.lut_i = d_lut_i;
    a.lut_q = d_lut_q;
    a.img = static_cast<float2*>(d_img);
    a.stride = img_stride;
    int rc = backend_decode_fbaq(a, static_cast<long long>(records) * range_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int32_t asarf_fbaq4_index(int32_t block, int32_t code) { return fbaq4_index(block, code); }

int asarf_condition_slc(const void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride,
                        int32_t record_header_bytes, float calibration, void* d_dest, void* stream) {
    if (!d_img || !d_dest || x_size <= 0 || y_size <= 0 || x_stride < x_size || record_header_bytes < 0)
        return set_error(ASARF_ERR_INVALID, "condition_slc: bad arguments");
    ConditionArgs c{};
    c.product = 2;
    c.slc = static_cast<const float2*>(d_img);
    c.stride = x_stride;
    c.x_size = x_size;
    c.y_size = y_size;
    c.hdr = record_header_bytes;
    c.cal = calibration;
    c.dest = static_cast<uint8_t*>(d_dest);
    int rc = backend_condition(c, y_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_condition_detected(const float* d_img, int32_t range_size, int32_t azimuth_size,
                             int32_t record_header_bytes, float calibration, void* d_dest, void* stream) {
    if (!d_img || !d_dest || range_size <= 0 || azimuth_size <= 0 || record_header_bytes < 0)
        return set_error(ASARF_ERR_INVALID, "condition_detected: bad arguments");
    ConditionArgs c{};
    c.product = 1;
    c.img = d_img;
    c.stride = range_size;
    c.x_size = range_size;
    c.y_size = azimuth_size;
    c.hdr = record_header_bytes;
    c.cal = calibration;
    c.dest = static_cast<uint8_t*>(d_dest);
    int rc = backend_condition(c, azimuth_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_raw_data_correction(void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, int32_t y_stride,
                              int64_t n_total_samples, asarf_iq_results* results, void* stream) {
    if (!d_img || !results || x_size <= 0 || y_size <= 0 || x_stride < x_size || y_stride < y_size)
        return set_error(ASARF_ERR_INVALID, "raw_data_correction: bad arguments");
    float2* img = static_cast<float2*>(d_img);
    double m[12];
    int rc = image_moments(img, x_size, y_size, x_stride, 0.0f, 0.0f, 0, m, stream);
    if (rc) return rc;
    const double total = n_total_samples > 0 ? static_cast<double>(n_total_samples) : static_cast<double>(x_size) * y_size;
    const float totf = static_cast<float>(total);
    // CalcMean: float(double sum) / float(total)
    const float dc_i = static_cast<float>(m[1]) / totf;
    const float dc_q = static_cast<float>(m[2]) / totf;
    double c[12];
    rc = image_moments(img, x_size, y_size, x_stride, dc_i, dc_q, 1, c, stream);
    if (rc) return rc;
    const float std_i = std::sqrt(static_cast<float>(c[3]) / totf);
    const float std_q = std::sqrt(static_cast<float>(c[4]) / totf);
    // gain / phase sums over x < XStride after the DC step, both regions (closed forms)
    const double di = dc_i, dq = dc_q;
    auto sq = [&](int o, int s1, int s2, double d) { return m[o + s2] - 2.0 * d * m[o + s1] + m[o] * d * d; };
    const double i1sq = sq(0, 1, 3, di) + sq(6, 1, 3, di);
    const double q1sq = sq(0, 2, 4, dq) + sq(6, 2, 4, dq);
    auto cross = [&](int o) { return m[o + 5] - dq * m[o + 1] - di * m[o + 2] + m[o] * di * dq; };
    const double i1q1 = cross(0) + cross(6);
    const double gain = std::sqrt(i1sq / q1sq);
    const float gf = static_cast<float>(gain);
    const double delta = (i1q1 / gf) / (i1sq / (static_cast<double>(gf) * gf));
    IqApplyArgs ap{};
    ap.img = img;
    ap.x_stride = x_stride;
    ap.y_size = y_size;
    ap.dc_i = dc_i;
    ap.dc_q = dc_q;
    ap.gain = gf;
    ap.sin_c = static_cast<float>(delta);
    ap.cos_c = static_cast<float>(1.0 - delta * delta);
    rc = backend_iq_apply(ap, static_cast<long long>(y_size) * x_stride, stream);
    if (rc) return rc;
    results->dc_i = dc_i;
    results->dc_q = dc_q;
    results->iq_gain = gain;
    results->phase_error = 360.0 * std::asin(delta) / (2.0 * 3.14159265358979323846);
    results->stddev_i = std_i;
    results->stddev_q = std_q;
    return stream_sync(stream);
}

int asarf_zero_nans(void* d_img, int32_t x_stride, int32_t y_stride, void* stream) {
    if (!d_img || x_stride <= 0 || y_stride <= 0) return set_error(ASARF_ERR_INVALID, "zero_nans: bad arguments");
    int rc = backend_zero_nans(static_cast<float2*>(d_img), static_cast<long long>(x_stride) * y_stride, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_doppler_centroid(const void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, double prf,
                           double poly[3], void* stream) {
    if (!d_img || !poly || x_size < 32 || y_size < 2 || x_stride < x_size)
        return set_error(ASARF_ERR_INVALID, "doppler_centroid: bad arguments");
    AcccArgs a{};
    a.img = static_cast<const float2*>(d_img);
    a.x_size = x_size;
    a.y_size = y_size;
    a.x_stride = x_stride;
    a.step = x_size / 32;
    a.nblk = (x_size + a.step - 1) / a.step;
    a.rows_per_block = 256;
    const int blocks = (y_size + a.rows_per_block - 1) / a.rows_per_block;
    const int xend = std::min(a.nblk * a.step, x_stride);
    DevBuf part(sizeof(double) * 2 * static_cast<size_t>(xend) * blocks);
    if (!part.p) return nomem();
    a.partial = part.as<double>();
    int rc = backend_accc(a, blocks, stream);
    if (rc) return rc;
    std::vector<double> h(2 * static_cast<size_t>(xend) * blocks);
    rc = mem_d2h(h.data(), part.p, sizeof(double) * h.size(), stream);
    if (rc) return rc;
    rc = stream_sync(stream);
    if (rc) return rc;
    std::vector<double> re(a.nblk, 0.0), im(a.nblk, 0.0), xs(a.nblk), ys(a.nblk);
    for (int b = 0; b < blocks; ++b)
        for (int x = 0; x < xend; ++x) {
            re[x / a.step] += h[(static_cast<size_t>(b) * xend + x) * 2];
            im[x / a.step] += h[(static_cast<size_t>(b) * xend + x) * 2 + 1];
        }
    for (int k = 0; k < a.nblk; ++k) {
        ys[k] = prf * (std::atan2(im[k], re[k]) / (2.0 * 3.14159265358979323846));
        xs[k] = static_cast<double>((k * a.step + (k + 1) * a.step) / 2);
    }
    if (a.nblk > kMaxDcBlocks || !polyfit_qr<kMaxDcBlocks, 3>(xs.data(), ys.data(), a.nblk, 2, poly))
        return set_error(ASARF_ERR_NUMERIC, "doppler_centroid: fit failed");
    return ASARF_OK;
}

int asarf_range_compression(void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, const float* chirp_padded,
                            int32_t chirp_len, int32_t chirp_samples, int32_t* new_x_size, void* stream) {
    if (!d_img || !chirp_padded || x_size <= 0 || y_size <= 0 || chirp_samples <= 0 || chirp_samples >= x_size)
        return set_error(ASARF_ERR_INVALID, "range_compression: bad arguments");
    if (chirp_len != x_stride) return set_error(ASARF_ERR_INVALID, "Range padding and chirp size mismatch");
    HostFft fft;
    const int L = choose_rc_len(x_size);
    if (L < x_size || !build_fft(L, fft)) return set_error(ASARF_ERR_INVALID, "range_compression: no FFT length");
    std::vector<std::complex<float>> chirp(chirp_samples);
    for (int i = 0; i < chirp_samples; ++i) chirp[i] = {chirp_padded[2 * i], chirp_padded[2 * i + 1]};
    std::vector<float2> mf;
    matched_filter_table(chirp.data(), chirp_samples, fft, mf);
    DevBuf tw(sizeof(float2) * L), mfd(sizeof(float2) * L);
    if (!tw.p || !mfd.p) return nomem();
    int rc = mem_h2d(tw.p, fft.tw.data(), sizeof(float2) * L, stream);
    if (!rc) rc = mem_h2d(mfd.p, mf.data(), sizeof(float2) * L, stream);
    if (rc) return rc;
    RcRowsArgs a{};
    a.img = static_cast<float2*>(d_img);
    a.stride = x_stride;
    a.nr = x_size;
    a.nk = x_size - chirp_samples;
    a.x_zero_end = x_stride;
    a.plan = fft.plan;
    a.plan.tw = tw.as<float2>();
    a.mf = mfd.as<float2>();
    const LaunchShape sh{512, sizeof(float2) * static_cast<size_t>(L)};
    if (sh.smem > smem_optin_limit())
        return set_error(ASARF_ERR_INVALID, "range_compression: range FFT of %d samples exceeds shared memory", L);
    rc = backend_rc_rows(a, y_size, sh, stream);
    if (rc) return rc;
    if (new_x_size) *new_x_size = a.nk;
    return stream_sync(stream);
}

int asarf_range_doppler(const asarf_rda_params* prm, void* d_src, void* d_out, int32_t x_size, int32_t y_size,
                        int32_t x_stride, int32_t y_stride, void* stream) {
    if (!prm || !d_src || !d_out || x_size < 17 || y_size <= 1 || x_stride < x_size || y_stride < y_size)
        return set_error(ASARF_ERR_INVALID, "range_doppler: bad arguments");
    const int N = y_stride;
    int n2 = 1;
    for (int d = 1; static_cast<long long>(d) * d <= N; ++d)
        if (N % d == 0) n2 = d;
    const int n1 = N / n2;
    HostFft f1, f2, fN;
    if (n2 < 2 || !build_fft_radices(n1, strided_radices(n1), f1) || !build_fft(n2, f2) || !build_fft(N, fN))
        return set_error(ASARF_ERR_INVALID, "range_doppler: azimuth size %d is not 2^a3^b5^c7^d", N);
    // tables + a finalised state carrying the Doppler polynomial
    DevBuf tw1(sizeof(float2) * n1), dr1(sizeof(int) * n1), tw2(sizeof(float2) * n2), dr2(sizeof(int) * n2),
        twN(sizeof(float2) * N), st(sizeof(FocusState));
    if (!tw1.p || !dr1.p || !tw2.p || !dr2.p || !twN.p || !st.p) return nomem();
    FocusState hs{};
    for (int k = 0; k < 3; ++k) {
        hs.dc_poly[k] = prm->dc_poly[k];
        hs.dc_poly32[k] = static_cast<float>(prm->dc_poly[k]);
    }
    hs.first_line = 0;
    hs.n_lines = y_size;  // inverse pass stores the data rows only
    int rc = mem_h2d(tw1.p, f1.tw.data(), sizeof(float2) * n1, stream);
    if (!rc) rc = mem_h2d(dr1.p, f1.drev.data(), sizeof(int) * n1, stream);
    if (!rc) rc = mem_h2d(tw2.p, f2.tw.data(), sizeof(float2) * n2, stream);
    if (!rc) rc = mem_h2d(dr2.p, f2.drev.data(), sizeof(int) * n2, stream);
    if (!rc) rc = mem_h2d(twN.p, fN.tw.data(), sizeof(float2) * N, stream);
    if (!rc) rc = mem_h2d(st.p, &hs, sizeof(hs), stream);
    if (!rc) rc = mem_zero(d_out, sizeof(float2) * static_cast<size_t>(x_stride) * y_stride, stream);
    if (rc) return rc;
    f1.plan.tw = tw1.as<float2>();
    f2.plan.tw = tw2.as<float2>();
    FocusState* dstate = st.as<FocusState>();
    float2* src = static_cast<float2*>(d_src);
    float2* out = static_cast<float2*>(d_out);
    const int xt1 = (n1 * 32 * 8 <= 160 * 1024) ? 32 : 16;
    AzStridedArgs fwd{};
    fwd.in = src;
    fwd.out = src;
    fwd.pitch = x_stride;
    fwd.n1 = n1;
    fwd.n2 = n2;
    fwd.plan1 = f1.plan;
    fwd.drev1 = dr1.as<int>();
    fwd.twn = twN.as<float2>();
    fwd.nk = x_size;
    fwd.xt = xt1;
    fwd.valid_rows = N;  // the reference transforms every row of the padded image
    fwd.state = dstate;
    fwd.scale = 1.0f;
    AzStridedArgs inv = fwd;
    inv.in = out;
    inv.out = out;
    inv.valid_rows = N;
    inv.scale = 1.0f / static_cast<float>(N);
    inv.inverse = 1;
    // RCMC halo from the largest walk at |f| <= PRF
    double vr_min = 1e30;
    for (int x = 0; x < x_size; x += std::max(1, x_size / 64)) {
        const double v = (prm->vr_poly[0] * x + prm->vr_poly[1]) * x + prm->vr_poly[2];
        vr_min = std::min(vr_min, std::fabs(v));
    }
    const double rmax = prm->slant_range_first + x_size * prm->range_spacing;
    const double walk =
        prm->wavelength * prm->wavelength * prm->prf * prm->prf * rmax / (8 * vr_min * vr_min) / prm->range_spacing;
    AzRdArgs d{};
    d.in = src;
    d.out = out;
    d.pitch = x_stride;
    d.n1 = n1;
    d.n2 = n2;
    d.az_pad = N;
    d.plan2 = f2.plan;
    d.drev2 = dr2.as<int>();
    d.nk = x_size;
    d.hl = kRcmcTaps / 2;
    d.hr = rcmc_right_halo(walk);
    if ((d.hl + d.hr) & 1) ++d.hr;  // column-pair transforms need an even tile width
    d.xt = az_rd_tile_width(n2, d.hl, d.hr);
    d.wt = d.xt + d.hl + d.hr;
    d.prf = static_cast<float>(prm->prf);
    d.bin_step = d.prf / static_cast<float>(N);
    d.half_prf = d.prf * 0.5f;
    d.lambda = static_cast<float>(prm->wavelength);
    d.frac = static_cast<float>(prm->az_bw_frac);
    d.slant = prm->slant_range_first;
    d.range_spacing = prm->range_spacing;
    for (int k = 0; k < 3; ++k) d.vr_poly[k] = static_cast<float>(prm->vr_poly[k]);
    d.state = dstate;
    const LaunchShape sh_st{256, az_strided_smem(n1, xt1)};
    const LaunchShape sh_rd{512, az_rd_smem(n2, d.wt, d.xt)};
    if (sh_st.smem > smem_optin_limit() || sh_rd.smem > smem_optin_limit())
        return set_error(ASARF_ERR_INVALID, "range_doppler: tiles exceed shared memory (n1 %d, n2 %d)", n1, n2);
    const int tiles1 = (x_size + xt1 - 1) / xt1, tiles2 = (x_size + d.xt - 1) / d.xt;
    rc = backend_az_strided(fwd, nullptr, tiles1, n2, sh_st, stream);
    if (!rc) rc = backend_az_rd(d, nullptr, tiles2, n1, sh_rd, &dstate->errors, stream);
    if (!rc) rc = backend_az_strided(inv, nullptr, tiles1, n2, sh_st, stream);
    // rows past the data block still hold the spectrum stage's values: clear them
    if (!rc && y_size < N)
        rc = mem_zero(out + static_cast<size_t>(y_size) * x_stride,
                      sizeof(float2) * static_cast<size_t>(N - y_size) * x_stride, stream);
    if (rc) return rc;
    unsigned int err = 0;
    rc = mem_d2h(&err, &dstate->errors, sizeof(err), stream);
    if (!rc) rc = stream_sync(stream);
    if (rc) return rc;
    if (err) return set_error(ASARF_ERR_NUMERIC, "range_doppler: kernel error flags %#x", err);
    return ASARF_OK;
}

int asarf_azimuth_multilook(const void* d_slc, int32_t x_size, int32_t y_size, double azimuth_spacing, float* d_out,
                            int32_t* out_y, void* stream) {
    if (!d_slc || !d_out || x_size <= 0 || y_size <= 0 || !(azimuth_spacing > 0))
        return set_error(ASARF_ERR_INVALID, "azimuth_multilook: bad arguments");
    MultilookArgs a{};
    a.slc = static_cast<const float2*>(d_slc);
    a.x_size = x_size;
    a.in_y = y_size;
    a.ratio = static_cast<float>(12.5f / azimuth_spacing);
    a.out_y = static_cast<int>(std::round(static_cast<float>(y_size) / a.ratio));
    a.out = d_out;
    if (a.out_y <= 0) return set_error(ASARF_ERR_INVALID, "azimuth_multilook: no output lines");
    if (out_y) *out_y = a.out_y;
    int rc = backend_multilook(a, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_range_spreading_loss(float* d_img, int32_t range_size, int32_t azimuth_size, double slant_range_first,
                               double range_spacing, double reference_range, void* stream) {
    if (!d_img || range_size <= 0 || azimuth_size <= 0)
        return set_error(ASARF_ERR_INVALID, "range_spreading_loss: bad arguments");
    RslArgs a{};
    a.img = d_img;
    a.range_size = range_size;
    a.az_size = azimuth_size;
    a.slant_first = slant_range_first;
    a.range_spacing = range_spacing;
    a.ref_range = reference_range;
    int rc = backend_rsl(a, static_cast<long long>(range_size) * azimuth_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

static int srgr_common(const float* d_in, int32_t in_x, int32_t y_size, const double poly[5], double range_spacing,
                       int32_t out_x, float* d_out, int32_t* d_start, float* d_frac, void* stream) {
    SrgrArgs a{};
    a.in = d_in;
    a.in_x = in_x;
    a.y_size = y_size;
    a.out_x = out_x;
    for (int k = 0; k < 5; ++k) a.grsr[k] = static_cast<float>(poly[k]);
    a.range_spacing = static_cast<float>(range_spacing);
    a.ground_spacing = 12.5f;
    a.out = d_out;
    a.start = d_start;
    a.frac = d_frac;
    int rc = backend_srgr(a, static_cast<long long>(out_x) * y_size, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_srgr(const float* d_in, int32_t in_x, int32_t y_size, const double grsr_poly[5], double range_spacing,
               int32_t out_x, float* d_out, void* stream) {
    if (!d_in || !d_out || !grsr_poly || in_x < 2 || y_size <= 0 || out_x <= 0)
        return set_error(ASARF_ERR_INVALID, "srgr: bad arguments");
    return srgr_common(d_in, in_x, y_size, grsr_poly, range_spacing, out_x, d_out, nullptr, nullptr, stream);
}

int asarf_srgr_index(const double grsr_poly[5], double range_spacing, int32_t out_x, int32_t* d_start, float* d_frac,
                     void* stream) {
    if (!grsr_poly || !d_start || !d_frac || out_x <= 0) return set_error(ASARF_ERR_INVALID, "srgr_index: bad arguments");
    return srgr_common(nullptr, 2, 1, grsr_poly, range_spacing, out_x, nullptr, d_start, d_frac, stream);
}

}  // extern "C"
