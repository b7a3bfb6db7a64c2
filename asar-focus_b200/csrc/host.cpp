// Host side of the focusing path: FP64 geometry, FFT schedules, chirp matched filter,
// planning, the launch sequence, and the C ABI of include/asarf.h.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"
#include "fft_ct.cuh"
#include "internal.h"
#include "plan.h"

namespace asarf {

namespace {
thread_local std::string g_last_error;
constexpr double kPi = 3.14159265358979323846;
constexpr double kSol = 299792458.0;
constexpr double kReferenceRange = 800000.0;  // envisat_format/include/asar_constants.h:37
constexpr float kGroundSpacing = 12.5f;        // sar/srgr.cu:84, sar/az_multilook.cu:83
}  // namespace

int set_error(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

// ============================================================================ geometry (FP64)

static asarf_osv interpolate_orbit(const asarf_osv* osv, int n, int64_t time_us) {
    // Lagrange over all vectors (sar/orbit_state_vector.cc:23-48)
    asarf_osv r{};
    r.time_us = time_us;
    const double tp = static_cast<double>(time_us - osv[0].time_us) * 1e-6;
    for (int i = 0; i < n; ++i) {
        double mult = 1.0;
        const double xi = static_cast<double>(osv[i].time_us - osv[0].time_us) * 1e-6;
        for (int j = 0; j < n; ++j) {
            if (i == j) continue;
            const double xj = static_cast<double>(osv[j].time_us - osv[0].time_us) * 1e-6;
            mult *= (tp - xj) / (xi - xj);
        }
        for (int k = 0; k < 3; ++k) {
            r.pos[k] += mult * osv[i].pos[k];
            r.vel[k] += mult * osv[i].vel[k];
        }
    }
    return r;
}

static int64_t azimuth_time_us(int64_t first, double lti, int idx) {
    // CalcAzimuthTime (sar/sar_metadata.h:90-93): uint32 microseconds
    const uint32_t us = static_cast<uint32_t>(static_cast<int64_t>(lti * idx * 1e6));
    return first + us;
}

static bool solve3(double A[3][3], const double b[3], double x[3]) {
    // Gaussian elimination with partial pivoting
    double M[3][4];
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) M[i][j] = A[i][j];
        M[i][3] = b[i];
    }
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(M[r][c]) > std::fabs(M[piv][c])) piv = r;
        if (M[piv][c] == 0.0) return false;
        if (piv != c)
            for (int j = 0; j < 4; ++j) std::swap(M[c][j], M[piv][j]);
        for (int r = c + 1; r < 3; ++r) {
            const double f = M[r][c] / M[c][c];
            for (int j = c; j < 4; ++j) M[r][j] -= f * M[c][j];
        }
    }
    for (int i = 2; i >= 0; --i) {
        double s = M[i][3];
        for (int j = i + 1; j < 3; ++j) s -= M[i][j] * x[j];
        x[i] = s / M[i][i];
    }
    return true;
}

static bool geolocate(const double vel[3], const double pos[3], const double guess[3], double slant, double out[3]) {
    // zero-Doppler Newton iteration on the ellipsoid (util/src/geo_tools.cc:27-85)
    const double a = 6378137.0, b = 6356752.314245;
    double r[3] = {guess[0], guess[1], guess[2]};
    for (int it = 1; it <= 101; ++it) {
        double pv[3] = {r[0] - pos[0], r[1] - pos[1], r[2] - pos[2]};
        double A[3][3] = {{vel[0], vel[1], vel[2]},
                          {2 * pv[0], 2 * pv[1], 2 * pv[2]},
                          {2 * r[0] / (a * a), 2 * r[1] / (a * a), 2 * r[2] / (b * b)}};
        double B[3] = {-(vel[0] * pv[0] + vel[1] * pv[1] + vel[2] * pv[2]),
                       -(pv[0] * pv[0] + pv[1] * pv[1] + pv[2] * pv[2] - slant * slant),
                       -((r[0] / a) * (r[0] / a) + (r[1] / a) * (r[1] / a) + (r[2] / b) * (r[2] / b) - 1.0)};
        double dx[3];
        if (!solve3(A, B, dx)) return false;
        for (int k = 0; k < 3; ++k) r[k] += dx[k];
        if (std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]) < 1e-6) {
            for (int k = 0; k < 3; ++k) out[k] = r[k];
            return true;
        }
    }
    return false;
}

static double polyval_d(const double* p, int n, double x) {
    double v = 0.0;
    for (int i = 0; i < n; ++i) v = v * x + p[i];
    return v;
}

static double round_half_away(double v) { return v >= 0 ? std::floor(v + 0.5) : -std::floor(-v + 0.5); }

static int aperture_pixels_at(const asarf_scene& s, const double* vr_poly, int px) {
    // CalcKa + CalcAperturePixels (sar/sar_metadata.h:110-124) with an empty Doppler polynomial
    const double vr = polyval_d(vr_poly, 3, px);
    const double r0 = s.slant_range_first + px * s.range_spacing;
    const double ka = (2 * s.carrier_frequency * vr * vr) / (kSol * r0);
    const double fmax = 0.0 + (s.prf * s.az_bw_frac) / 2;
    return static_cast<int>(round_half_away((fmax / ka) * s.prf));
}

int max_aperture_pixels(const asarf_scene& s) {
    // CalcAperturePixels(sar_meta) (sar/sar_metadata.h:126-141) as main.cc:251 calls it
    const int range_end = s.range_size - s.chirp_samples;
    const int step = range_end / 10;
    int mx = 0;
    if (step <= 0) return aperture_pixels_at(s, s.vr_poly_init, 0);
    for (int px = 0; px < range_end; px += step) mx = std::max(mx, aperture_pixels_at(s, s.vr_poly_init, px));
    return mx;
}

static int estimate_vr_poly(const asarf_scene& s, double out[3]) {
    // EstimateProcessingVelocity / EstimateVrAtRange (sar/processing_velocity_estimation.cc:56-148)
    if (s.n_osv < 2 || !s.osv) return set_error(ASARF_ERR_INVALID, "Vr estimation needs orbit state vectors");
    const int az_idx = s.azimuth_size / 2;
    const int range_end = s.range_size - s.chirp_samples;
    const int step = range_end / 10;
    if (step <= 0) return set_error(ASARF_ERR_INVALID, "range too short for Vr estimation");
    std::vector<double> xs, ys;
    for (int r = 0; r < range_end; r += step) {
        const double r0 = s.slant_range_first + r * s.range_spacing;
        const int aperture = aperture_pixels_at(s, s.vr_poly_init, r);
        const int N = 9;
        const asarf_osv c = interpolate_orbit(s.osv, s.n_osv, azimuth_time_us(s.first_line_time_us, s.line_time_interval, az_idx));
        double earth[3];
        if (!geolocate(c.vel, c.pos, s.center_point, r0, earth))
            return set_error(ASARF_ERR_NUMERIC, "geolocation did not converge (Vr estimation)");
        const int st = aperture / (N - 1);
        // least squares of y = c0 + c1 x^2 through the normal equations of a 2-column system
        double xv[N], yv[N];
        for (int i = 0; i < N; ++i) {
            const int idx = az_idx + (i - N / 2) * st;
            const asarf_osv o = interpolate_orbit(s.osv, s.n_osv, azimuth_time_us(s.first_line_time_us, s.line_time_interval, idx));
            const double dx = o.pos[0] - earth[0], dy = o.pos[1] - earth[1], dz = o.pos[2] - earth[2];
            yv[i] = dx * dx + dy * dy + dz * dz - r0 * r0;
            xv[i] = static_cast<double>(c.time_us - o.time_us) * 1e-6;
        }
        // QR solve of [1, x^2] c = y (SquareFitVr, :30-47)
        double xq[N];
        for (int i = 0; i < N; ++i) xq[i] = xv[i] * xv[i];
        double cf[2];
        if (!polyfit_qr<128, 5>(xq, yv, N, 1, cf)) return set_error(ASARF_ERR_NUMERIC, "Vr fit failed");
        // cf highest power first: cf[0] = slope (Vr^2), cf[1] = intercept
        xs.push_back(static_cast<double>(r));
        ys.push_back(std::sqrt(cf[0]));
    }
    if (!polyfit_qr<128, 5>(xs.data(), ys.data(), static_cast<int>(xs.size()), 2, out))
        return set_error(ASARF_ERR_NUMERIC, "Vr polynomial fit failed");
    return ASARF_OK;
}

int srgr_poly(const asarf_scene& s, double slant_first, int range_size, int azimuth_size, double lti,
                     double poly[5], int* ng) {
    // SlantRangeToGroundRangeInterpolation setup (sar/srgr.cu:73-121)
    const int N = 100;
    const int64_t t = azimuth_time_us(s.first_line_time_us, lti, azimuth_size / 2);
    const asarf_osv o = interpolate_orbit(s.osv, s.n_osv, t);
    double first[3];
    if (!geolocate(o.vel, o.pos, s.center_point, slant_first, first))
        return set_error(ASARF_ERR_NUMERIC, "geolocation did not converge (SRGR)");
    double gd[N], sr[N];
    for (int i = 0; i < N; ++i) {
        const double R = slant_first + (i * (range_size / 100)) * s.range_spacing;
        double g[3];
        if (!geolocate(o.vel, o.pos, s.center_point, R, g))
            return set_error(ASARF_ERR_NUMERIC, "geolocation did not converge (SRGR)");
        const double dx = g[0] - first[0], dy = g[1] - first[1], dz = g[2] - first[2];
        gd[i] = std::sqrt(dx * dx + dy * dy + dz * dz);
        sr[i] = R - slant_first;
    }
    *ng = static_cast<int>(gd[N - 1] / static_cast<double>(kGroundSpacing));
    if (!polyfit_qr<128, 5>(gd, sr, N, 4, poly)) return set_error(ASARF_ERR_NUMERIC, "SRGR polynomial fit failed");
    return ASARF_OK;
}

static void generate_chirp(double kr, double fs, int n, bool window, int padding, std::vector<std::complex<float>>& out) {
    // GenerateChirpData (sar/sar_chirp.cc:70-104); the windowed power scale sum|C_k|^2/N equals
    // sum|c_n|^2 (Parseval) and is taken in FP64 on the time-domain replica
    out.assign(padding, std::complex<float>(0.0f, 0.0f));
    const double dt = 1.0 / fs;
    for (int64_t i = 0; i < n; ++i) {
        const double t = static_cast<double>(i - n / 2) * dt;
        const double ph = kPi * kr * t * t;
        std::complex<float> iq(static_cast<float>(std::cos(ph)), static_cast<float>(std::sin(ph)));
        if (window) {
            const double m = 0.54 - 0.46 * std::cos((2 * kPi * i) / n);
            iq *= static_cast<float>(m);
        }
        out[i] = iq;
    }
    double scale;
    if (window) {
        scale = 0.0;
        for (int i = 0; i < n; ++i) {
            const double re = out[i].real(), im = out[i].imag();
            scale += re * re + im * im;
        }
    } else {
        scale = static_cast<double>(n);
    }
    const float inv = static_cast<float>(std::sqrt(scale));
    for (auto& e : out) e /= inv;
}

// ============================================================================ FFT schedules

static std::vector<int> factorize(int n) {
    std::vector<int> r;
    int m = n;
    while (m % 8 == 0) {
        r.push_back(8);
        m /= 8;
    }
    if (m % 4 == 0) {
        r.push_back(4);
        m /= 4;
    }
    if (m % 2 == 0) {
        r.push_back(2);
        m /= 2;
    }
    for (int p : {7, 5, 3}) {
        while (m % p == 0) {
            r.push_back(p);
            m /= p;
        }
    }
    if (m != 1) r.clear();
    return r;
}

static double fft_cost(int n) {
    auto f = factorize(n);
    if (f.empty()) return 1e30;
    double c = 0;
    for (int r : f) {
        switch (r) {
            case 8: c += 1.5; break;
            case 4: c += 1.35; break;
            case 2: c += 1.2; break;
            case 3: c += 1.4; break;
            case 5: c += 1.55; break;
            default: c += 1.7; break;
        }
    }
    return c * n;
}

bool smooth(int n) {
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

// bf16 of a float, round to nearest even (finite inputs).
static uint16_t bf16_rn(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(u >> 16);
}
static float bf16_to_float(uint16_t h) {
    const uint32_t u = static_cast<uint32_t>(h) << 16;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

// Tables of the split-precision forward transform of length n = R * m: the m-point DFT matrix
// as the B operand (rows = output (slot, re / im), K = input (mm, re / im)) in the canonical
// no-swizzle K-major layout, bf16 hi image then lo image; and the twiddles W_n^(r k1(s)),
// [r][s].  Output slot s holds frequency k1(s) = drev[R s] (the FP32 transform's order).
// FP64 throughout, rounded once.
void split_dft_tables(int n, int R, const std::vector<int>& drev, std::vector<unsigned char>& img,
                      std::vector<float2>& tw) {
    const int m = n / R;
    img.assign(2 * static_cast<size_t>(kSplitMatrixBytes), 0);
    auto put = [&](int row, int k, double v) {
        const float f = static_cast<float>(v);
        const uint16_t hi = bf16_rn(f);
        const uint16_t lo = bf16_rn(f - bf16_to_float(hi));
        const uint32_t off = umma_offset(row, k, kSplitK);
        std::memcpy(&img[off], &hi, 2);
        std::memcpy(&img[kSplitMatrixBytes + off], &lo, 2);
    };
    for (int sl = 0; sl < m; ++sl) {
        const int k1 = drev[static_cast<size_t>(R) * sl];
        for (int j = 0; j < m; ++j) {
            const double a = -2.0 * kPi * static_cast<double>((static_cast<long long>(j) * k1) % m) / m;
            const double fr = std::cos(a), fi = std::sin(a);
            put(2 * sl, 2 * j, fr);
            put(2 * sl, 2 * j + 1, -fi);
            put(2 * sl + 1, 2 * j, fi);
            put(2 * sl + 1, 2 * j + 1, fr);
        }
    }
    tw.assign(static_cast<size_t>(R) * m, make_float2(1.0f, 0.0f));
    for (int r = 0; r < R; ++r)
        for (int sl = 0; sl < m; ++sl) {
            const int k1 = drev[static_cast<size_t>(R) * sl];
            const double a = -2.0 * kPi * static_cast<double>((static_cast<long long>(r) * k1) % n) / n;
            tw[static_cast<size_t>(r) * m + sl] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
        }
}

void matched_filter_table(const std::complex<float>* chirp, int nc, const HostFft& fft, std::vector<float2>& mf) {
    // conj(DFT_L(replica)) / L in FP64, stored in the forward transform's digit-reversed order
    const int L = fft.plan.n;
    mf.assign(L, make_float2(0.0f, 0.0f));
    std::vector<std::complex<double>> w(L);
    for (int m = 0; m < L; ++m) w[m] = std::polar(1.0, -2.0 * kPi * m / L);
    for (int pos = 0; pos < L; ++pos) {
        const int k = fft.drev[pos];
        std::complex<double> acc(0.0, 0.0);
        for (int n = 0; n < nc; ++n) {
            const long long idx = (static_cast<long long>(n) * k) % L;
            acc += std::complex<double>(chirp[n].real(), chirp[n].imag()) * w[idx];
        }
        const std::complex<double> h = std::conj(acc) / static_cast<double>(L);
        mf[pos] = make_float2(static_cast<float>(h.real()), static_cast<float>(h.imag()));
    }
}

int32_t fft_size_above(int32_t v) {
    // smallest 2^a 3^b 5^c 7^d strictly greater than v, up to 131072 (cuda_util/cufft_plan.cc:147-181)
    for (int n = v + 1; n <= 131072; ++n)
        if (smooth(n)) return n;
    return -1;
}

bool build_fft(int n, HostFft& h) { return build_fft_radices(n, factorize(n), h); }

std::vector<int> strided_radices(int n) {
    // the default factors with each pair of 3s merged into a 9 (first, so that the short
    // radices run on the shortest spans)
    std::vector<int> rest, out;
    int threes = 0;
    for (int r : factorize(n)) {
        if (r == 3)
            ++threes;
        else
            rest.push_back(r);
    }
    for (int k = 0; k < threes / 2; ++k) out.push_back(9);
    out.insert(out.end(), rest.begin(), rest.end());
    if (threes & 1) out.push_back(3);
    return out;
}

bool build_fft_radices(int n, const std::vector<int>& f, HostFft& h) {
    long long prod = 1;
    for (int r : f) prod *= r;
    if (f.empty() || prod != n || static_cast<int>(f.size()) > kMaxStages) return false;
    h.plan.n = n;
    h.plan.nst = static_cast<int>(f.size());
    int M = n;
    std::vector<int> spans;
    for (size_t i = 0; i < f.size(); ++i) {
        h.plan.radix[i] = f[i];
        h.plan.span[i] = M / f[i];
        h.plan.sdiv[i] = make_fastdiv(static_cast<unsigned int>(M / f[i]));
        spans.push_back(M / f[i]);
        M /= f[i];
    }
    h.drev.assign(n, 0);
    for (int p = 0; p < n; ++p) {
        int rem = p, k = 0, mult = 1;
        for (size_t i = 0; i < f.size(); ++i) {
            const int q = rem / spans[i];
            rem %= spans[i];
            k += q * mult;
            mult *= f[i];
        }
        h.drev[p] = k;
    }
    h.tw.resize(n);
    for (int m = 0; m < n; ++m) {
        const double a = -2.0 * kPi * static_cast<double>(m) / n;
        h.tw[m] = make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a)));
    }
    return true;
}

int choose_rc_len(int nr) {
    // a compile-time-scheduled length when one is close above (within 1.5x)
    for (int L : kCtLengths)
        if (L >= nr && 2 * L <= 3 * nr) return L;
    int best = -1;
    double bc = 1e30;
    for (int n = nr; n <= 2 * nr + 64; ++n) {
        if (!smooth(n)) continue;
        const double c = fft_cost(n);
        if (c < bc) {
            bc = c;
            best = n;
        }
    }
    return best;
}

}  // namespace asarf

// ============================================================================ plan

using namespace asarf;


extern "C" {

const char* asarf_last_error(void) { return g_last_error.c_str(); }

const char* asarf_version(void) {
    static std::string v = std::string("asarf 0.1 (") + backend_name() + ")";
    return v.c_str();
}

void asarf_default_options(asarf_options* opt) {
    if (!opt) return;
    opt->rc_fft_len = 0;
    opt->ref_compat_stats = 1;
    opt->iq_padding_ref = 0;
    opt->dc_poly_given = 0;
    opt->dc_poly[0] = opt->dc_poly[1] = opt->dc_poly[2] = 0.0;
    opt->product = ASARF_PRODUCT_DETECTED;
    opt->record_header_bytes = 17;  // main.cc: 12 + 1 + 4
    opt->calibration = 1.0f;
    opt->sq_stats = 0;
    opt->precision = ASARF_PRECISION_FP32;
    opt->absolute_phase = 0;
    opt->az_n2 = 0;
    opt->az_tile_width = 0;
    opt->strided_tile_width = 0;
    opt->keep_slc = 1;
    opt->compiled_schedules = 1;
}

int32_t asarf_fft_size_above(int32_t v) { return fft_size_above(v); }

int asarf_interpolate_orbit(const asarf_osv* osv, int32_t n, int64_t time_us, asarf_osv* out) {
    if (!osv || n < 1 || !out) return set_error(ASARF_ERR_INVALID, "interpolate_orbit: bad arguments");
    *out = interpolate_orbit(osv, n, time_us);
    return ASARF_OK;
}

int asarf_geolocate(const double vel[3], const double pos[3], const double init_guess[3], double slant_range,
                    double out_xyz[3]) {
    if (!vel || !pos || !init_guess || !out_xyz) return set_error(ASARF_ERR_INVALID, "geolocate: null argument");
    if (!geolocate(vel, pos, init_guess, slant_range, out_xyz))
        return set_error(ASARF_ERR_NUMERIC, "Failed to converge for RangeDopplerGeoLocate");
    return ASARF_OK;
}

int asarf_polyfit(const double* x, const double* y, int32_t n, int32_t degree, double* coeffs) {
    if (!x || !y || !coeffs || degree < 0 || degree > 4 || n > 128 || n < degree + 1)
        return set_error(ASARF_ERR_INVALID, "polyfit: bad arguments");
    if (!polyfit_qr<128, 5>(x, y, n, degree, coeffs)) return set_error(ASARF_ERR_NUMERIC, "polyfit: rank deficient");
    return ASARF_OK;
}

int asarf_estimate_processing_velocity(const asarf_scene* scene, double vr_poly[3]) {
    if (!scene || !vr_poly) return set_error(ASARF_ERR_INVALID, "estimate_processing_velocity: null argument");
    return estimate_vr_poly(*scene, vr_poly);
}

int asarf_generate_chirp(double kr, double fs, int32_t n_samples, int32_t apply_window, int32_t padding,
                         float* out_interleaved) {
    if (n_samples <= 0 || padding < n_samples || !out_interleaved)
        return set_error(ASARF_ERR_INVALID, "generate_chirp: bad arguments");
    std::vector<std::complex<float>> c;
    generate_chirp(kr, fs, n_samples, apply_window != 0, padding, c);
    std::memcpy(out_interleaved, c.data(), sizeof(float) * 2 * padding);
    return ASARF_OK;
}

int asarf_srgr_polynomial(const asarf_scene* scene, double slant_first, int32_t range_size, int32_t azimuth_size,
                          double line_time_interval, double poly[5], int32_t* ground_samples) {
    if (!scene || !poly || !ground_samples) return set_error(ASARF_ERR_INVALID, "srgr_polynomial: null argument");
    int ng = 0;
    int rc = srgr_poly(*scene, slant_first, range_size, azimuth_size, line_time_interval, poly, &ng);
    *ground_samples = ng;
    return rc;
}

static int validate_scene(const asarf_scene* s) {
    if (!s) return set_error(ASARF_ERR_INVALID, "scene is NULL");
    if (s->range_size <= 0 || s->azimuth_size <= 1 || s->samples_per_line <= 0)
        return set_error(ASARF_ERR_INVALID, "scene sizes must be positive (range %d, azimuth %d)", s->range_size,
                         s->azimuth_size);
    if (s->samples_per_line > s->range_size)
        return set_error(ASARF_ERR_INVALID, "samples_per_line %d exceeds range_size %d", s->samples_per_line,
                         s->range_size);
    if (s->raw_format == ASARF_RAW_ASAR_FBAQ4) {
        // samples_per_line samples take 63 per 64-byte block plus one id byte for a partial block
        const int spl = s->samples_per_line;
        const long long need = 2 + 64ll * (spl / 63) + (spl % 63 ? spl % 63 + 1 : 0);
        if (s->raw_line_bytes < need)
            return set_error(ASARF_ERR_INVALID, "raw_line_bytes %d cannot hold %d FBAQ4 samples (%lld bytes)",
                             s->raw_line_bytes, spl, need);
        if (!s->fbaq_i_lut || !s->fbaq_q_lut)
            return set_error(ASARF_ERR_INVALID, "FBAQ4 records need the instrument reconstruction tables");
    } else if (s->raw_format == ASARF_RAW_ERS_BYTES) {
        if (s->raw_line_bytes < 2 * s->samples_per_line || (s->raw_line_bytes & 1))
            return set_error(ASARF_ERR_INVALID, "raw_line_bytes must be even and >= 2*samples_per_line");
    } else {
        return set_error(ASARF_ERR_INVALID, "unknown raw_format %d", s->raw_format);
    }
    if (s->chirp_samples <= 0 || s->chirp_samples >= s->range_size - 32)
        return set_error(ASARF_ERR_INVALID, "chirp_samples %d incompatible with range_size %d", s->chirp_samples,
                         s->range_size);
    if (!(s->prf > 0) || !(s->wavelength > 0) || !(s->range_spacing > 0) || !(s->azimuth_spacing > 0))
        return set_error(ASARF_ERR_INVALID, "prf, wavelength, range_spacing, azimuth_spacing must be positive");
    if (s->n_osv < 2 || !s->osv) return set_error(ASARF_ERR_INVALID, "at least two orbit state vectors are needed");
    return ASARF_OK;
}

int asarf_plan_create(const asarf_scene* scene, const asarf_options* opt_in, asarf_plan** out) {
    if (!out) return set_error(ASARF_ERR_INVALID, "plan output pointer is NULL");
    *out = nullptr;
    int rc = validate_scene(scene);
    if (rc) return rc;
    asarf_options opt;
    asarf_default_options(&opt);
    if (opt_in) opt = *opt_in;

    auto* p = new asarf_plan();
    p->scene = *scene;
    p->osv.assign(scene->osv, scene->osv + scene->n_osv);
    p->scene.osv = p->osv.data();
    if (scene->raw_format == ASARF_RAW_ASAR_FBAQ4) {
        p->fbaq_luts.assign(scene->fbaq_i_lut, scene->fbaq_i_lut + 4096);
        p->fbaq_luts.insert(p->fbaq_luts.end(), scene->fbaq_q_lut, scene->fbaq_q_lut + 4096);
        p->scene.fbaq_i_lut = p->fbaq_luts.data();
        p->scene.fbaq_q_lut = p->fbaq_luts.data() + 4096;
    } else {
        p->scene.fbaq_i_lut = p->scene.fbaq_q_lut = nullptr;
    }
    p->opt = opt;
    const asarf_scene& s = p->scene;
    p->nr = s.range_size;
    p->na = s.azimuth_size;
    p->nc = s.chirp_samples;
    p->nk = p->nr - p->nc;
    p->nx = p->nk - kRcmcTaps;
    if (p->nx < 4) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "range too short after compression");
    }
    p->rg_pad_ref = opt.iq_padding_ref > 0 ? opt.iq_padding_ref : fft_size_above(p->nr + p->nc);
    p->az_pad = fft_size_above(p->na);
    if (p->rg_pad_ref < 0 || p->az_pad < 0) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "sizes exceed the 131072 FFT size table");
    }
    p->rc_len = opt.rc_fft_len > 0 ? opt.rc_fft_len : choose_rc_len(p->nr);
    if (p->rc_len < p->nr || !smooth(p->rc_len)) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "range FFT length %d must be >= range_size and 2^a3^b5^c7^d", p->rc_len);
    }
    // azimuth split N = n1 * n2, n2 = largest divisor <= sqrt(N) unless the caller names one
    {
        const int N = p->az_pad;
        int best = 1;
        for (int d = 1; static_cast<long long>(d) * d <= N; ++d)
            if (N % d == 0) best = d;
        if (opt.az_n2 > 0) {
            if (N % opt.az_n2 != 0 || opt.az_n2 < 16 || opt.az_n2 > 256) {
                delete p;
                return set_error(ASARF_ERR_INVALID, "az_n2 %d must divide the azimuth FFT size %d and lie in [16, 256]",
                                 opt.az_n2, N);
            }
            best = opt.az_n2;
        }
        p->n2 = best;
        p->n1 = N / best;
        if (p->n2 < 2) {
            delete p;
            return set_error(ASARF_ERR_INVALID, "azimuth FFT size %d cannot be split", N);
        }
    }
    // compile-time lengths use their own three-pass radix sequence (and so its output order)
    int ctr[3];
    const int n_ctr = ct_radices(p->rc_len, ctr);
    const bool rc_ok = n_ctr ? build_fft_radices(p->rc_len, std::vector<int>(ctr, ctr + n_ctr), p->rc)
                             : build_fft(p->rc_len, p->rc);
    // the split-precision form takes the contiguous transform's last radix as its FP32 pass, so
    // that pass gets the largest radix (smallest tensor-core DFT)
    std::vector<int> f2_radices = factorize(p->n2);
    if (opt.precision == ASARF_PRECISION_SPLIT && !f2_radices.empty()) {
        auto big = std::max_element(f2_radices.begin(), f2_radices.end());
        std::rotate(big, big + 1, f2_radices.end());
    }
    if (!rc_ok || !build_fft_radices(p->n1, strided_radices(p->n1), p->f1) ||
        !build_fft_radices(p->n2, f2_radices, p->f2) || !build_fft(p->az_pad, p->fN)) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "FFT schedule failed");
    }
    // Vr polynomial
    if (s.vr_poly_given) {
        for (int k = 0; k < 3; ++k) p->vr_poly[k] = s.vr_poly[k];
    } else {
        rc = estimate_vr_poly(s, p->vr_poly);
        if (rc) {
            delete p;
            return rc;
        }
    }
    // RCMC halo from the largest walk at |f| <= PRF (Doppler centroid within +-PRF/2)
    {
        double vr_min = 1e30;
        for (int x = 0; x < p->nk; x += std::max(1, p->nk / 64))
            vr_min = std::min(vr_min, std::fabs(polyval_d(p->vr_poly, 3, x)));
        vr_min = std::min(vr_min, std::fabs(polyval_d(p->vr_poly, 3, p->nk - 1)));
        const double rmax = s.slant_range_first + p->nk * s.range_spacing;
        const double f = s.prf;
        const double walk = s.wavelength * s.wavelength * f * f * rmax / (8 * vr_min * vr_min) / s.range_spacing;
        p->hl = kRcmcTaps / 2;
        p->hr = rcmc_right_halo(walk);
        if ((p->hl + p->hr) & 1) ++p->hr;  // even tile width: TMA rows are whole 16-byte units
    }
    p->pitch = (p->nk + 31) / 32 * 32;
    p->xt1 = (p->n1 * 32 * 8 <= 160 * 1024) ? 32 : 16;
    if (opt.strided_tile_width == 16 || opt.strided_tile_width == 32) p->xt1 = opt.strided_tile_width;
    else if (opt.strided_tile_width != 0) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "strided_tile_width must be 16 or 32");
    }
    p->xt2 = az_rd_tile_width(p->n2, p->hl, p->hr);
    if (opt.az_tile_width != 0) {
        if (opt.az_tile_width < 16 || opt.az_tile_width > 64 || (opt.az_tile_width & 1)) {
            delete p;
            return set_error(ASARF_ERR_INVALID, "az_tile_width must be even and in [16, 64]");
        }
        p->xt2 = opt.az_tile_width;
    }
    if (opt.precision == ASARF_PRECISION_SPLIT && opt.az_tile_width == 0) {
        // the split block holds the DFT matrix (16 KB) besides the tile: the widest tile that
        // still leaves two blocks resident per SM
        while (p->xt2 > 16 && az_rd_smem(p->n2, p->xt2 + p->hl + p->hr, p->xt2) + 2 * kSplitMatrixBytes >
                                  kAzRdTwoBlockSmem)
            p->xt2 -= 2;
    }

    // chirp matched filter in the forward transform's output order, scaled by 1/L
    std::vector<std::complex<float>> chirp;
    generate_chirp(s.chirp_kr, s.range_sampling_rate, p->nc, s.apply_window != 0, p->rc_len, chirp);
    std::vector<float2> mf;
    matched_filter_table(chirp.data(), p->nc, p->rc, mf);
    std::vector<float2> ctw;
    if (n_ctr) {
        // transposed filter (position b*R + q at q*(L/R) + b) and the per-pass twiddle tables
        const int L = p->rc_len, R = ctr[n_ctr - 1], nb = L / R;
        std::vector<float2> t(mf.size());
        for (int b = 0; b < nb; ++b)
            for (int q = 0; q < R; ++q) t[static_cast<size_t>(q) * nb + b] = mf[static_cast<size_t>(b) * R + q];
        mf.swap(t);
        int m = L;
        for (int k = 0; k + 1 < n_ctr; ++k) {
            const int S = m / ctr[k], M = m;
            for (int q = 1; q < ctr[k]; ++q)
                for (int j = 0; j < S; ++j) {
                    const double a = -2.0 * kPi * static_cast<double>(static_cast<long long>(j) * q % M) / M;
                    ctw.push_back(make_float2(static_cast<float>(std::cos(a)), static_cast<float>(std::sin(a))));
                }
            m = S;
        }
    }

    // results-window variants (CalcResultsWindow, main_flow.cc:155-201) and their tails
    const int max_ap = max_aperture_pixels(s);
    int first_line[2], n_lines[2], out_az[2], ng[2];
    float grsr32[2][5];
    const float ratio = static_cast<float>(12.5f / s.azimuth_spacing);
    const double sub_first = s.slant_range_first + (kRcmcTaps / 2) * s.range_spacing;
    for (int v = 0; v < 2; ++v) {
        const bool dc_pos = (v == 0);
        int after_start = 0, before_stop = 0;
        if (dc_pos) {
            if (s.lines_before < max_ap) after_start = max_ap - s.lines_before;
        } else {
            if (s.lines_after < max_ap) before_stop = max_ap - s.lines_after;
        }
        first_line[v] = s.lines_before + after_start;
        n_lines[v] = p->na - first_line[v] - (before_stop + s.lines_after);
        if (n_lines[v] < 8) {
            delete p;
            return set_error(ASARF_ERR_INVALID, "results window leaves %d lines (aperture %d)", n_lines[v], max_ap);
        }
        out_az[v] = static_cast<int>(std::round(static_cast<float>(n_lines[v]) / ratio));
        double poly[5];
        const double lti_ml = (1.0 / s.prf) * static_cast<double>(ratio);
        rc = srgr_poly(s, sub_first, p->nx, out_az[v], lti_ml, poly, &ng[v]);
        if (rc) {
            delete p;
            return rc;
        }
        for (int k = 0; k < 5; ++k) grsr32[v][k] = static_cast<float>(poly[k]);
    }
    p->out_rows_max = std::max(out_az[0], out_az[1]);
    p->out_cols_max = std::max(ng[0], ng[1]);
    if (opt.product < ASARF_PRODUCT_DETECTED || opt.product > ASARF_PRODUCT_IMS_MDS || opt.record_header_bytes < 0) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "unknown product %d or negative record header", opt.product);
    }
    {
        const long long hdr = opt.record_header_bytes;
        long long bytes = 4ll * p->out_rows_max * p->out_cols_max;
        for (int v = 0; v < 2; ++v) {
            if (opt.product == ASARF_PRODUCT_IMP_MDS) bytes = std::max(bytes, out_az[v] * (hdr + 2ll * ng[v]));
            if (opt.product == ASARF_PRODUCT_IMS_MDS) bytes = std::max(bytes, n_lines[v] * (hdr + 4ll * p->nx));
        }
        p->out_bytes = bytes;
        p->ims_rows_max = std::max(n_lines[0], n_lines[1]);
    }
    std::vector<float> rsl(p->nx);
    for (int i = 0; i < p->nx; ++i) {
        const double R = sub_first + i * s.range_spacing;
        const double ratio_r = kReferenceRange / R;
        rsl[i] = static_cast<float>(1.0 / std::sqrt(std::pow(ratio_r, 3)));
    }

    // ---- device memory
    const size_t img = static_cast<size_t>(p->az_pad) * p->pitch;
    p->bufA = p->alloc<float2>(img);
    p->bufB = p->alloc<float2>(img);
    p->acc = p->alloc<StatAccum>(1);
    p->state = p->alloc<FocusState>(1);
    p->raw_dev = p->alloc<uint8_t>(static_cast<size_t>(p->na) * s.raw_line_bytes);
    p->swst_dev = p->alloc<uint16_t>(p->na);
    p->out_dev = p->alloc<float>(static_cast<size_t>(p->out_bytes + 3) / 4);
    float2* rc_tw = p->alloc<float2>(p->rc_len);
    p->rc_mf = p->alloc<float2>(p->rc_len);
    float2* ct_tw = ctw.empty() ? nullptr : p->alloc<float2>(ctw.size());
    float2* tw1 = p->alloc<float2>(p->n1);
    int* drev1 = p->alloc<int>(p->n1);
    float2* tw2 = p->alloc<float2>(p->n2);
    int* drev2 = p->alloc<int>(p->n2);
    float2* twN = p->alloc<float2>(p->az_pad);
    float* win = p->alloc<float>(16);
    float* rsl_dev = p->alloc<float>(p->nx);
    // FBAQ4 records: reconstruction tables permuted to [block id][raw code], and the
    // statistics partials of every 32-column x kFbaqStatsLines tile
    const bool fbaq = s.raw_format == ASARF_RAW_ASAR_FBAQ4;
    const int fb_tiles_x = (p->nr + 31) / 32;
    const int fb_tiles_y = (p->na + kFbaqStatsLines - 1) / kFbaqStatsLines;
    const int dc_step0 = p->nr / 32 > 0 ? p->nr / 32 : 1;
    int fb_span = 1;
    for (int bx = 0; bx < fb_tiles_x; ++bx) {
        const int x1 = std::min(bx * 32 + 31, p->nr - 1);
        fb_span = std::max(fb_span, x1 / dc_step0 - (bx * 32) / dc_step0 + 1);
    }
    const int fb_slots = 6 + 9 * fb_span;
    float* lut_dev = fbaq ? p->alloc<float>(2 * 4096) : nullptr;
    double* part_dev = fbaq ? p->alloc<double>(static_cast<size_t>(fb_tiles_y) * fb_tiles_x * fb_slots) : nullptr;
    FloatStatAccum* facc_dev = fbaq ? p->alloc<FloatStatAccum>(1) : nullptr;
    constexpr int kPstatBlocks = 4 * 148;
    double* pstat_dev = opt.sq_stats ? p->alloc<double>(5 * kPstatBlocks + 4) : nullptr;
    if (!p->bufA || !p->bufB || !p->acc || !p->state || !p->raw_dev || !p->swst_dev || !p->out_dev || !rc_tw ||
        !p->rc_mf || !tw1 || !drev1 || !tw2 || !drev2 || !twN || !win || !rsl_dev || (fbaq && (!lut_dev || !part_dev || !facc_dev)) ||
        (opt.sq_stats && !pstat_dev)) {
        const size_t need = p->bytes;
        delete p;
        return set_error(ASARF_ERR_NOMEM, "device allocation failed (plan needs about %zu MB)",
                         (need + 2 * img * sizeof(float2)) >> 20);
    }
    float w16[16];
    for (int n = 0; n < 16; ++n)  // numpy.blackman(16) (sar/range_doppler_algorithm.cu:49-52)
        w16[n] = static_cast<float>(0.42 - 0.5 * std::cos(2 * kPi * n / 15) + 0.08 * std::cos(4 * kPi * n / 15));
    rc = 0;
    rc |= mem_h2d(rc_tw, p->rc.tw.data(), sizeof(float2) * p->rc_len, nullptr);
    rc |= mem_h2d(p->rc_mf, mf.data(), sizeof(float2) * p->rc_len, nullptr);
    if (ct_tw) rc |= mem_h2d(ct_tw, ctw.data(), sizeof(float2) * ctw.size(), nullptr);
    rc |= mem_h2d(tw1, p->f1.tw.data(), sizeof(float2) * p->n1, nullptr);
    rc |= mem_h2d(drev1, p->f1.drev.data(), sizeof(int) * p->n1, nullptr);
    rc |= mem_h2d(tw2, p->f2.tw.data(), sizeof(float2) * p->n2, nullptr);
    rc |= mem_h2d(drev2, p->f2.drev.data(), sizeof(int) * p->n2, nullptr);
    rc |= mem_h2d(twN, p->fN.tw.data(), sizeof(float2) * p->az_pad, nullptr);
    rc |= mem_h2d(win, w16, sizeof(w16), nullptr);
    rc |= mem_h2d(rsl_dev, rsl.data(), sizeof(float) * p->nx, nullptr);
    if (fbaq) {
        std::vector<float> lut(2 * 4096);
        for (int id = 0; id < 256; ++id)
            for (int code = 0; code < 16; ++code) {
                lut[16 * id + code] = s.fbaq_i_lut[fbaq4_index(id, code)];
                lut[4096 + 16 * id + code] = s.fbaq_q_lut[fbaq4_index(id, code)];
            }
        rc |= mem_h2d(lut_dev, lut.data(), sizeof(float) * lut.size(), nullptr);
    }
    rc |= mem_zero(p->state, sizeof(FocusState), nullptr);
    rc |= stream_sync(nullptr);
    if (rc) {
        delete p;
        return ASARF_ERR_CUDA;
    }
    p->rc.plan.tw = rc_tw;
    p->f1.plan.tw = tw1;
    p->f2.plan.tw = tw2;

    // ---- launch argument blocks
    const int dc_step = p->nr / 32;
    const int nblk = (p->nr + dc_step - 1) / dc_step;
    if (dc_step < 1 || nblk > kMaxDcBlocks) {
        delete p;
        return set_error(ASARF_ERR_INVALID, "range size %d gives %d Doppler blocks", p->nr, nblk);
    }
    RawStatsArgs& st = p->a_stats;
    st.line_bytes = s.raw_line_bytes;
    st.spl = s.samples_per_line;
    st.na = p->na;
    st.nr = p->nr;
    st.dc_step = dc_step;
    st.nblk = nblk;
    st.acc = p->acc;
    {
        // block height for the grid of aligned raw buffers (the 4-column path, any address
        // that is a multiple of 8: a null pointer stands for one); an unaligned buffer runs
        // the one-column path over the same lines
        RawStatsArgs shape = st;
        const int gx = raw_stats_grid_x(shape, nullptr);
        st.lines_per_cta = stats_lines_per_block(p->na, gx, backend_sm_count() * kStatsBlocksPerSm);
    }
    p->stats_gy = (p->na + st.lines_per_cta - 1) / st.lines_per_cta;
    if (fbaq) {
        st.lut_i = lut_dev;
        st.lut_q = lut_dev + 4096;
        st.part = part_dev;
        st.facc = facc_dev;
        st.tiles_x = fb_tiles_x;
        st.span = fb_span;
        st.part_slots = fb_slots;
        p->stats_gy = fb_tiles_y;
    }


    FinalizeArgs& fin = p->a_fin;
    fin.acc = p->acc;
    fin.state = p->state;
    fin.n_total = s.total_raw_samples > 0 ? s.total_raw_samples
                                          : static_cast<long long>(s.samples_per_line) * p->na;
    fin.n_pad = opt.ref_compat_stats ? static_cast<long long>(p->rg_pad_ref - p->nr) * p->na : 0;
    fin.nr = p->nr;
    fin.na = p->na;
    fin.rg_stride = p->rg_pad_ref;
    fin.dc_step = dc_step;
    fin.nblk = nblk;
    fin.prf = s.prf;
    fin.lines_before = s.lines_before;
    fin.lines_after = s.lines_after;
    fin.max_aperture = max_ap;
    fin.facc = facc_dev;
    fin.dc_given = opt.dc_poly_given ? 1 : 0;
    for (int k = 0; k < 3; ++k) fin.dc_in[k] = opt.dc_poly[k];
    for (int v = 0; v < 2; ++v) {
        fin.first_line[v] = first_line[v];
        fin.n_lines[v] = n_lines[v];
    }

    RangeCompressArgs& r = p->a_rc;
    r.line_bytes = s.raw_line_bytes;
    r.spl = s.samples_per_line;
    r.na = p->na;
    r.nr = p->nr;
    r.state = p->state;
    r.plan = p->rc.plan;
    r.mf = p->rc_mf;
    r.ctw = ct_tw;
    r.nk = p->nk;
    r.out = p->bufA;
    r.out_pitch = p->pitch;
    r.format = s.raw_format;
    if (fbaq) {
        r.lut_i = lut_dev;
        r.lut_q = lut_dev + 4096;
    }
    const int rc_elems = n_ctr ? ct_smem_elems_of(p->rc_len) : p->rc_len;  // compile-time lengths: padded tile
    p->raw_smem_offset = static_cast<int>((sizeof(float2) * static_cast<size_t>(rc_elems) + 127) / 128 * 128);
    const size_t raw_area = fbaq ? static_cast<size_t>(s.raw_line_bytes) + 16
                                 : (2 * static_cast<size_t>(s.samples_per_line) + 15) / 16 * 16;
    p->sh_rc = {512, static_cast<size_t>(p->raw_smem_offset) + raw_area};

    AzStridedArgs& f = p->a_fwd;
    f.in = p->bufA;
    f.out = p->bufA;
    f.pitch = p->pitch;
    f.n1 = p->n1;
    f.n2 = p->n2;
    f.plan1 = p->f1.plan;
    f.drev1 = drev1;
    f.twn = twN;
    f.nk = p->nk;
    f.xt = p->xt1;
    f.valid_rows = p->na;
    f.state = p->state;
    f.scale = 1.0f;
    f.inverse = 0;
    p->a_inv = f;
    p->a_inv.in = p->bufB;
    p->a_inv.out = p->bufB;
    p->a_inv.valid_rows = p->az_pad;
    p->a_inv.state = p->state;
    p->a_inv.scale = 1.0f / static_cast<float>(p->az_pad);
    p->a_inv.inverse = 1;
    p->tiles1 = (p->nk + p->xt1 - 1) / p->xt1;
    p->sh_st = {256, az_strided_smem(p->n1, p->xt1)};

    AzRdArgs& d = p->a_rd;
    d.in = p->bufA;
    d.out = p->bufB;
    d.pitch = p->pitch;
    d.n1 = p->n1;
    d.n2 = p->n2;
    d.az_pad = p->az_pad;
    d.plan2 = p->f2.plan;
    d.drev2 = drev2;
    d.nk = p->nk;
    d.xt = p->xt2;
    d.hl = p->hl;
    d.hr = p->hr;
    d.wt = p->xt2 + p->hl + p->hr;
    d.chunk_rows = 0;
    d.prf = static_cast<float>(s.prf);
    d.bin_step = d.prf / static_cast<float>(p->az_pad);
    d.half_prf = d.prf * 0.5f;
    d.lambda = static_cast<float>(s.wavelength);
    d.frac = static_cast<float>(s.az_bw_frac);
    d.slant = s.slant_range_first;
    d.range_spacing = s.range_spacing;
    for (int k = 0; k < 3; ++k) d.vr_poly[k] = static_cast<float>(p->vr_poly[k]);
    d.state = p->state;
    d.win = win;
    d.absolute_phase = opt.absolute_phase ? 1 : 0;
    d.compiled = p->a_fwd.compiled = p->a_inv.compiled = opt.compiled_schedules ? 1 : 0;
    d.lambda_d = s.wavelength;
    p->tiles2 = (p->nk + p->xt2 - 1) / p->xt2;
    p->sh_rd = {512, az_rd_smem(p->n2, d.wt, d.xt)};

    // detected products without a kept SLC: the inverse azimuth pass writes |z|^2 rows into
    // bufA (free once the range-Doppler block has read it) and the tail reads those
    p->intensity_only = !opt.keep_slc &&
                        (opt.product == ASARF_PRODUCT_DETECTED || (opt.product == ASARF_PRODUCT_IMP_MDS && !opt.sq_stats));
    if (p->intensity_only) p->a_inv.out_intensity = reinterpret_cast<float*>(p->bufA);
    TailArgs& t = p->a_tail;
    t.slc = p->bufB;
    t.intensity = p->intensity_only ? reinterpret_cast<const float*>(p->bufA) : nullptr;
    t.pitch = p->pitch;
    t.state = p->state;
    t.col0 = kRcmcTaps / 2;
    t.nx = p->nx;
    for (int v = 0; v < 2; ++v) {
        t.tail[v].n_lines = n_lines[v];
        t.tail[v].out_az = out_az[v];
        t.tail[v].ratio = ratio;
        t.tail[v].ng = ng[v];
        for (int k = 0; k < 5; ++k) t.tail[v].grsr[k] = grsr32[v][k];
        t.tail[v].rsl = rsl_dev;
    }
    t.range_spacing = static_cast<float>(s.range_spacing);
    t.ground_spacing = kGroundSpacing;
    t.out_pitch = p->out_cols_max;
    t.mds_hdr = opt.record_header_bytes;
    t.mds_cal = opt.calibration;
    p->sh_tail = {256, sizeof(float) * static_cast<size_t>(p->nx)};
    if (opt.sq_stats) {
        ProductStatsArgs& ps = p->a_pstats;
        ps.imaged = opt.product == ASARF_PRODUCT_IMS_MDS ? 0 : 1;
        ps.slc = p->bufB + kRcmcTaps / 2;
        ps.slc_pitch = p->pitch;
        ps.nx = p->nx;
        ps.img_pitch = p->out_cols_max;
        for (int v = 0; v < 2; ++v) {
            ps.ng[v] = ng[v];
            ps.out_az[v] = out_az[v];
        }
        ps.state = p->state;
        ps.part = pstat_dev;
        ps.blocks = kPstatBlocks;
        ps.cal = opt.calibration;
        ps.out = pstat_dev + 5 * kPstatBlocks;
    }

    // ---- TMA tensor maps (all tiles come from this GPU's own buffers; loads only)
    {
        auto largest_divisor_le = [](int n, int cap) {
            for (int d = std::min(n, cap); d >= 1; --d)
                if (n % d == 0) return d;
            return 1;
        };
        const int n1_box = largest_divisor_le(p->n1, 256);
        const int n2_box = largest_divisor_le(p->n2, 256);
        const unsigned long long row_bytes = static_cast<unsigned long long>(p->pitch) * sizeof(float2);
        const unsigned long long d3[3] = {2ull * p->nk, static_cast<unsigned long long>(p->n2),
                                          static_cast<unsigned long long>(p->n1)};
        const unsigned long long s3[2] = {row_bytes, row_bytes * p->n2};
        const unsigned int b3[3] = {static_cast<unsigned int>(2 * p->xt1), 1u, static_cast<unsigned int>(n1_box)};
        const unsigned long long d2[2] = {2ull * p->nk, static_cast<unsigned long long>(p->az_pad)};
        const unsigned long long s2[1] = {row_bytes};
        const unsigned int b2[2] = {static_cast<unsigned int>(2 * d.wt), static_cast<unsigned int>(n2_box)};
        const bool shapes_ok = (d.wt % 2 == 0) && 2 * d.wt <= 256 && 2 * p->xt1 <= 256;
        p->use_tma = shapes_ok && backend_make_tmap(p->tmapA3, 3, p->bufA, d3, s3, b3) == ASARF_OK &&
                     backend_make_tmap(p->tmapB3, 3, p->bufB, d3, s3, b3) == ASARF_OK &&
                     backend_make_tmap(p->tmapA2, 2, p->bufA, d2, s2, b2) == ASARF_OK;
        p->a_fwd.use_tma = p->a_inv.use_tma = d.use_tma = p->use_tma ? 1 : 0;
        p->a_fwd.n1_box = p->a_inv.n1_box = n1_box;
        d.n2_box = n2_box;
    }

    // ---- split precision: n2 = R * m with R the FP32 plan's last radix (so that its digit
    // reversal puts frequency k1 + m k2 at position R s + k2) and m <= 32
    if (opt.precision == ASARF_PRECISION_SPLIT) {
        const int R = p->f2.plan.radix[p->f2.plan.nst - 1];
        const int m = p->n2 / R;
        const bool radix_ok = R == 2 || R == 3 || R == 4 || R == 5 || R == 7 || R == 8;
        const size_t smem_split = 2 * static_cast<size_t>(kSplitMatrixBytes) + p->sh_rd.smem;
        if (p->use_tma && radix_ok && m >= 2 && 2 * m <= kSplitK && smem_split <= smem_optin_limit()) {
            std::vector<unsigned char> img;
            std::vector<float2> tws;
            split_dft_tables(p->n2, R, p->f2.drev, img, tws);
            unsigned char* bmat = p->alloc<unsigned char>(img.size());
            float2* tw_dev = p->alloc<float2>(tws.size());
            if (!bmat || !tw_dev) {
                delete p;
                return set_error(ASARF_ERR_CUDA, "device allocation failed (split tables)");
            }
            rc = mem_h2d(bmat, img.data(), img.size(), nullptr);
            rc |= mem_h2d(tw_dev, tws.data(), sizeof(float2) * tws.size(), nullptr);
            if (rc) {
                delete p;
                return set_error(ASARF_ERR_CUDA, "split table upload failed");
            }
            p->split = true;
            p->a_split.bmat = bmat;
            p->a_split.tw = tw_dev;
            p->a_split.radix = R;
            p->a_split.m = m;
            p->sh_rd_split = {512, smem_split};
        }
    }

    const size_t lim = smem_optin_limit();
    if (p->sh_rc.smem > lim || p->sh_st.smem > lim || p->sh_rd.smem > lim || p->sh_tail.smem > lim) {
        const size_t a1 = p->sh_rc.smem, a2 = p->sh_st.smem, a3 = p->sh_rd.smem;
        delete p;
        return set_error(ASARF_ERR_INVALID, "shared memory need exceeds %zu (rc %zu, strided %zu, rd %zu)", lim, a1, a2,
                         a3);
    }

    asarf_dims& dm = p->dims;
    dm.nk = p->nk;
    dm.rg_pad_ref = p->rg_pad_ref;
    dm.az_pad = p->az_pad;
    dm.rc_fft_len = p->rc_len;
    dm.n1 = p->n1;
    dm.n2 = p->n2;
    dm.slc_cols = p->nx;
    for (int v = 0; v < 2; ++v) {
        dm.out_rows[v] = out_az[v];
        dm.out_cols[v] = ng[v];
    }
    dm.out_rows_max = p->out_rows_max;
    dm.out_cols_max = p->out_cols_max;
    dm.out_bytes_max = p->out_bytes;
    dm.max_aperture = max_ap;
    for (int k = 0; k < 3; ++k) dm.vr_poly[k] = p->vr_poly[k];
    dm.device_bytes = p->bytes;
    dm.precision = p->split ? ASARF_PRECISION_SPLIT : ASARF_PRECISION_FP32;
    dm.split_radix = p->split ? p->a_split.radix : 0;
    dm.split_m = p->split ? p->a_split.m : 0;
    dm.az_tile_width = p->xt2;
    dm.strided_tile_width = p->xt1;
    dm.compiled_schedules = (p->a_fwd.compiled && strided_schedule_compiled(p->a_fwd.plan1, p->a_fwd.xt) ? 1 : 0) |
                            (p->a_rd.compiled && block_schedule_compiled(p->a_rd.plan2) ? 2 : 0);
    *out = p;
    return ASARF_OK;
}

void asarf_plan_destroy(asarf_plan* plan) { delete plan; }

int asarf_plan_dims(const asarf_plan* plan, asarf_dims* dims) {
    if (!plan || !dims) return set_error(ASARF_ERR_INVALID, "plan_dims: null argument");
    *dims = plan->dims;
    return ASARF_OK;
}

static constexpr int kKernelsPerRun = 7;
static const char* const kKernelNames[kKernelsPerRun] = {"raw_stats", "finalize", "range_compress", "az_strided_fwd",
                                                          "az_rd", "az_strided_inv", "tail"};

int asarf_focus(asarf_plan* p, const uint8_t* d_raw, const uint16_t* d_swst, int32_t min_swst, float* d_out,
                void* stream) {
    if (!p || !d_raw || (!d_out && !p->skip_tail)) return set_error(ASARF_ERR_INVALID, "focus: null argument");
    const bool fbaq = p->scene.raw_format == ASARF_RAW_ASAR_FBAQ4;
    if (!fbaq && (reinterpret_cast<uintptr_t>(d_raw) & 1))
        return set_error(ASARF_ERR_INVALID, "raw buffer must be 2-byte aligned");
    void** ev = nullptr;
    if (p->timing_used < p->timing_slots) {
        ev = &p->events[static_cast<size_t>(p->timing_used) * (kKernelsPerRun + 1)];
        ++p->timing_used;
    }
    int k = 0;
    auto mark = [&]() {
        if (ev) event_record(ev[k], stream);
        ++k;
    };
    int rc = mem_zero(p->acc, sizeof(StatAccum), stream);
    if (rc) return rc;
    RawStatsArgs st = p->a_stats;
    st.raw = d_raw;
    st.swst = d_swst;
    st.min_swst = min_swst;
    mark();
    if (fbaq) {
        rc = backend_raw_stats_fbaq(st, st.tiles_x, p->stats_gy, stream);
        if (!rc) rc = backend_stats_fold(st, p->stats_gy, stream);
    } else {
        const int stats_gx = raw_stats_grid_x(st, d_raw);
        rc = backend_raw_stats(st, stats_gx, p->stats_gy, stream);
    }
    if (rc) return rc;
    mark();
    rc = backend_finalize(p->a_fin, stream);
    if (rc) return rc;
    RangeCompressArgs r = p->a_rc;
    r.raw = d_raw;
    r.swst = d_swst;
    r.min_swst = min_swst;
    const bool aligned = (reinterpret_cast<uintptr_t>(d_raw) % 16 == 0) && (p->scene.raw_line_bytes % 16 == 0);
    r.bulk_bytes = (p->use_tma && aligned && !fbaq) ? (2 * p->scene.samples_per_line) / 16 * 16 : 0;
    r.raw_smem_offset = p->raw_smem_offset;
    mark();
    rc = backend_range_compress(r, p->na, p->sh_rc, stream);
    if (rc) return rc;
    mark();
    rc = backend_az_strided(p->a_fwd, p->use_tma ? p->tmapA3 : nullptr, p->tiles1, p->n2, p->sh_st, stream);
    if (rc) return rc;
    mark();
    rc = p->split ? backend_az_rd_split(p->a_rd, p->a_split, p->tmapA2, p->tiles2, p->n1, p->sh_rd_split,
                                        &p->state->errors, stream)
                  : backend_az_rd(p->a_rd, p->use_tma ? p->tmapA2 : nullptr, p->tiles2, p->n1, p->sh_rd,
                                  &p->state->errors, stream);
    if (rc) return rc;
    mark();
    rc = backend_az_strided(p->a_inv, p->use_tma ? p->tmapB3 : nullptr, p->tiles1, p->n2, p->sh_st, stream);
    if (rc) return rc;
    mark();
    if (!p->skip_tail && p->opt.product == ASARF_PRODUCT_IMS_MDS) {
        ConditionArgs c{};
        c.product = 2;
        c.slc = p->bufB + kRcmcTaps / 2;
        c.stride = p->pitch;
        c.x_size = p->nx;
        c.hdr = p->opt.record_header_bytes;
        c.cal = p->opt.calibration;
        c.dest = reinterpret_cast<uint8_t*>(d_out);
        c.state = p->state;
        rc = backend_condition(c, p->ims_rows_max, stream);
        if (rc) return rc;
    } else if (!p->skip_tail) {
        TailArgs t = p->a_tail;
        t.out = d_out;
        if (p->opt.product == ASARF_PRODUCT_IMP_MDS) {
            t.mds = reinterpret_cast<uint8_t*>(d_out);
            // the statistics read the float image, which the records do not keep: bufA is
            // free once the inverse azimuth pass has run
            if (p->opt.sq_stats) t.out2 = reinterpret_cast<float*>(p->bufA);
        }
        rc = backend_tail(t, p->out_rows_max, p->sh_tail, &p->state->errors, stream);
        if (rc) return rc;
    }
    if (!p->skip_tail && p->opt.sq_stats) {
        ProductStatsArgs ps = p->a_pstats;
        ps.img = p->opt.product == ASARF_PRODUCT_DETECTED ? d_out : reinterpret_cast<float*>(p->bufA);
        rc = backend_product_stats(ps, stream);
        if (rc) return rc;
    }
    mark();
    return ASARF_OK;
}

int asarf_plan_enable_timing(asarf_plan* p, int32_t runs) {
    if (!p || runs < 0) return set_error(ASARF_ERR_INVALID, "enable_timing: bad arguments");
    for (void* e : p->events) event_destroy(e);
    p->events.clear();
    p->timing_slots = 0;
    p->timing_used = 0;
    for (int i = 0; i < runs * (kKernelsPerRun + 1); ++i) {
        void* e = event_create();
        if (!e) return set_error(ASARF_ERR_CUDA, "event creation failed");
        p->events.push_back(e);
    }
    p->timing_slots = runs;
    return ASARF_OK;
}

int asarf_plan_kernel_times(asarf_plan* p, float* total_ms, int32_t* runs, const char** names) {
    if (!p || !total_ms || !runs) return set_error(ASARF_ERR_INVALID, "kernel_times: null argument");
    for (int k = 0; k < kKernelsPerRun; ++k) {
        total_ms[k] = 0.0f;
        if (names) names[k] = kKernelNames[k];
    }
    for (int r = 0; r < p->timing_used; ++r) {
        void** ev = &p->events[static_cast<size_t>(r) * (kKernelsPerRun + 1)];
        for (int k = 0; k < kKernelsPerRun; ++k) {
            float ms = 0.0f;
            int rc = event_elapsed(ev[k], ev[k + 1], &ms);
            if (rc) return rc;
            total_ms[k] += ms;
        }
    }
    *runs = p->timing_used;
    p->timing_used = 0;
    return ASARF_OK;
}

}  // extern "C"

// Raw (and SWST) upload, focus run and image download, enqueued on `stream` in that order.
static int enqueue_host_run(asarf_plan* p, const uint8_t* h_raw, const uint16_t* h_swst, int32_t min_swst,
                            float* h_out, void* stream) {
    int rc = mem_h2d(p->raw_dev, h_raw, static_cast<size_t>(p->na) * p->scene.raw_line_bytes, stream);
    if (rc) return rc;
    if (h_swst) {
        rc = mem_h2d(p->swst_dev, h_swst, sizeof(uint16_t) * p->na, stream);
        if (rc) return rc;
    }
    rc = asarf_focus(p, p->raw_dev, h_swst ? p->swst_dev : nullptr, min_swst, p->out_dev, stream);
    if (rc) return rc;
    return mem_d2h(h_out, p->out_dev, static_cast<size_t>(p->out_bytes), stream);
}

extern "C" {

int asarf_focus_host(asarf_plan* p, const uint8_t* h_raw, const uint16_t* h_swst, int32_t min_swst, float* h_out,
                     void* stream) {
    if (!p || !h_raw || !h_out) return set_error(ASARF_ERR_INVALID, "focus_host: null argument");
    const int rc = enqueue_host_run(p, h_raw, h_swst, min_swst, h_out, stream);
    if (rc) return rc;
    return stream_sync(stream);
}

int asarf_focus_host_async(asarf_plan* p, const uint8_t* h_raw, const uint16_t* h_swst, int32_t min_swst,
                           float* h_out, void* stream) {
    if (!p || !h_raw || !h_out) return set_error(ASARF_ERR_INVALID, "focus_host_async: null argument");
    if (!stream) {
        if (!p->own_stream) p->own_stream = asarf::stream_create();
        if (!p->own_stream) return set_error(ASARF_ERR_CUDA, "focus_host_async: stream creation failed");
        stream = p->own_stream;
    }
    if (!p->done) p->done = asarf::event_create();
    if (!p->done) return set_error(ASARF_ERR_CUDA, "focus_host_async: event creation failed");
    const int rc = enqueue_host_run(p, h_raw, h_swst, min_swst, h_out, stream);
    if (rc) return rc;
    return asarf::event_record(p->done, stream);
}

int asarf_plan_wait(asarf_plan* p) {
    if (!p) return set_error(ASARF_ERR_INVALID, "plan_wait: null plan");
    return p->done ? asarf::event_sync(p->done) : ASARF_OK;
}

int asarf_plan_results(asarf_plan* p, asarf_results* res, void* stream) {
    if (!p || !res) return set_error(ASARF_ERR_INVALID, "plan_results: null argument");
    FocusState st;
    int rc = mem_d2h(&st, p->state, sizeof(st), stream);
    if (rc) return rc;
    rc = stream_sync(stream);
    if (rc) return rc;
    std::memset(res, 0, sizeof(*res));
    res->dc_i = st.dc_i_d;
    res->dc_q = st.dc_q_d;
    res->iq_gain = st.iq_gain;
    res->phase_error = st.phase_error;
    res->stddev_i = st.stddev_i;
    res->stddev_q = st.stddev_q;
    for (int k = 0; k < 3; ++k) {
        res->doppler_centroid_poly[k] = st.dc_poly[k];
        res->doppler_centroid_estimate[k] = st.dc_est[k];
        res->vr_poly[k] = p->vr_poly[k];
    }
    res->n_dc_blocks = st.nblk;
    for (int b = 0; b < st.nblk && b < 80; ++b) res->dc_block_hz[b] = st.dc_blk_hz[b];
    res->variant = st.variant;
    res->first_line = st.first_line;
    res->n_lines = st.n_lines;
    res->out_rows = p->dims.out_rows[st.variant & 1];
    res->out_cols = p->dims.out_cols[st.variant & 1];
    res->errors = st.errors;
    if (p->opt.sq_stats) {
        rc = mem_d2h(res->sq_stats, p->a_pstats.out, sizeof(res->sq_stats), stream);
        if (!rc) rc = stream_sync(stream);
        if (rc) return rc;
    }
    const int hdr = p->opt.record_header_bytes;
    if (p->opt.product == ASARF_PRODUCT_IMP_MDS) {
        res->records = res->out_rows;
        res->record_bytes = hdr + 2 * res->out_cols;
    } else if (p->opt.product == ASARF_PRODUCT_IMS_MDS) {
        res->records = st.n_lines;
        res->record_bytes = hdr + 4 * p->nx;
    } else {
        res->records = res->out_rows;
        res->record_bytes = 4 * p->out_cols_max;
    }
    return ASARF_OK;
}

int asarf_plan_slc(asarf_plan* p, void* d_slc, void* stream) {
    if (!p || !d_slc) return set_error(ASARF_ERR_INVALID, "plan_slc: null argument");
    if (p->intensity_only)
        return set_error(ASARF_ERR_INVALID, "plan_slc: the plan keeps no complex SLC (asarf_options.keep_slc = 0)");
    FocusState st;
    int rc = mem_d2h(&st, p->state, sizeof(st), stream);
    if (rc) return rc;
    rc = stream_sync(stream);
    if (rc) return rc;
    const float2* src = p->bufB + static_cast<long long>(st.first_line) * p->pitch + kRcmcTaps / 2;
    return mem_d2d_2d(d_slc, sizeof(float2) * p->nx, src, sizeof(float2) * p->pitch, sizeof(float2) * p->nx,
                      st.n_lines, stream);
}

}  // extern "C"
