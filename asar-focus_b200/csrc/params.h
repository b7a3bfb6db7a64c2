// Plain-data structures shared by the host planner and the kernels.
#pragma once

#include <cstdint>

#include "fft.cuh"

namespace asarf {

constexpr int kMaxDcBlocks = 80;   // CalculateDopplerCentroid uses XSize/32-wide blocks (32 or 33 of them)
constexpr int kRcmcTaps = 16;      // RCMC interpolator length (reference: RCMC_INTERPOLATOR_SIZE 16)
constexpr int kNumTailVariants = 2;

// Integer accumulators of the raw-statistics pass (zeroed before every run).
//   mom: filled-sample count, sum I, sum Q, sum I^2, sum Q^2, sum I*Q
//   lag[b]: over azimuth-adjacent sample pairs (y-1, y) that are both filled, in Doppler
//           block b: n, sum A, sum B, sum C, sum D, sum AC, sum BD, sum AD, sum BC with
//           (A, B) = raw (I, Q) of line y-1 and (C, D) = raw (I, Q) of line y.
struct StatAccum {
    unsigned long long mom[6];
    unsigned long long lag[kMaxDcBlocks][9];
};

// ASAR FBAQ4 records: the same sums over the decoded float samples, in FP64, written (not
// accumulated) by the fold of the per-tile partials in a fixed order, so reproducible.
struct FloatStatAccum {
    double mom[6];
    double lag[kMaxDcBlocks][9];
};

// Raw record formats of the fused path.
enum RawFormat : int {
    kRawErsBytes = 0,   // ERS byte I/Q pairs, SWST shift 4 samples per code step
    kRawAsarFbaq4 = 1,  // ENVISAT ASAR FBAQ4 blocks, SWST shift 1 sample per code step
};

// FBAQ4 statistics tiles: 32 columns (one per lane) x kFbaqStatsLines lines, split over the
// 8 warps of a block.
constexpr int kFbaqStatsLines = 2048;
constexpr int kFbaqStatsWarps = 8;

// Per-column-independent output of the statistics finalisation, read by later kernels.
struct FocusState {
    float dc_i, dc_q, gain, sin_c, cos_c;  // IQ correction as the reference applies it
    float rgain, rcos;                     // RN(1 / gain), RN(1 / cos_c): exact divisions by reciprocal
    float dc_poly32[3];                    // Doppler centroid polynomial (float, highest power first)
    double dc_poly[3];                     // polynomial in use (estimate or the caller's)
    double dc_est[3];                      // ACCC estimate
    double dc_i_d, dc_q_d, iq_gain, phase_error, stddev_i, stddev_q;
    int nblk;
    double dc_blk_hz[kMaxDcBlocks];
    int variant;     // tail variant: 0 when the DC constant term > 0, else 1
    int first_line;  // first azimuth line kept by the results window
    int n_lines;     // kept lines
    unsigned int errors;
};

enum ErrorBits : unsigned int {
    kErrRcmcHalo = 1u << 0,      // an RCMC tap fell outside the loaded range halo
    kErrSrgrIndex = 1u << 1,     // an SRGR index fell outside the slant row
    kErrStatsEmpty = 1u << 2,    // no filled samples
    kErrDcBlocks = 1u << 3,      // too many Doppler blocks
};

// Everything the statistics finalisation needs besides the accumulators.
struct FinalizeArgs {
    const StatAccum* acc;
    FocusState* state;
    long long n_total;       // CorrectionParams::n_total_samples
    long long n_pad;         // range-padding samples entering the gain / phase sums
    int nr;                  // range samples (XSize)
    int na;                  // azimuth lines (YSize)
    int rg_stride;           // reference XStride (for Doppler blocks that run into the padding)
    int dc_step;             // Doppler block width (XSize / 32)
    int nblk;
    double prf;
    // results window inputs (CalcResultsWindow)
    int lines_before, lines_after, max_aperture;
    const FloatStatAccum* facc;  // FBAQ4 records: read these FP64 sums instead of acc
    int dc_given;            // use dc_in instead of the estimate
    double dc_in[3];
    int first_line[kNumTailVariants];
    int n_lines[kNumTailVariants];
};

struct RawStatsArgs {
    const uint8_t* raw;
    long long line_bytes;
    int spl;              // I/Q sample pairs per raw record
    int na, nr;
    const uint16_t* swst; // nullable
    int min_swst;
    int dc_step, nblk;
    int lines_per_cta;    // at most kStatsMaxLines
    int quad;             // 4-column units (raw base and line stride 8-byte aligned)
    int gpb;              // 4-column groups per Doppler block: ceil(dc_step / 4)
    StatAccum* acc;
    // ASAR FBAQ4 records (k_raw_stats_fbaq): FP64 partial sums of each 32-column tile
    const float* lut_i;   // [256 block ids][16 raw codes]
    const float* lut_q;
    double* part;         // [tiles_y][tiles_x][part_slots]
    FloatStatAccum* facc; // folded sums
    int tiles_x;          // ceil(nr / 32)
    int span;             // Doppler blocks one 32-column tile can touch
    int part_slots;       // 6 moments + 9 lag sums per touched Doppler block
};

struct RangeCompressArgs {
    const uint8_t* raw;
    long long line_bytes;
    int spl;
    int na, nr;
    const uint16_t* swst;
    int min_swst;
    const FocusState* state;
    FftPlan plan;
    const float2* mf;     // matched filter in the forward transform's digit-reversed order, / L
                          // (compile-time lengths: transposed, see fft_ct.cuh)
    const float2* ctw;    // compile-time lengths: per-pass twiddle tables (fft_ct.cuh)
    int nk;
    float2* out;
    long long out_pitch;
    int bulk_bytes;       // raw bytes per line fetched by one bulk copy (multiple of 16; 0 = plain loads)
    int raw_smem_offset;  // byte offset of the raw-line buffer in shared memory
    int format;           // RawFormat of the records
    const float* lut_i;   // ASAR FBAQ4 records: [256 block ids][16 raw codes]
    const float* lut_q;
};

// Transform schedules with compile-time instantiations of the azimuth kernels (the strided
// lengths 225 = 9 x 5 x 5 and 180 = 9 x 4 x 5 at the 32-column tile, the block lengths
// 125 = 5 x 5 x 5 and 168 = 8 x 7 x 3 of the ERS-like and ASAR IM-like scenes); every other
// schedule runs the run-time loops, with the same arithmetic.
ASARF_HD inline bool plan_is(const FftPlan& p, int r0, int r1, int r2) {
    return p.nst == 3 && p.radix[0] == r0 && p.radix[1] == r1 && p.radix[2] == r2;
}
ASARF_HD inline bool strided_schedule_compiled(const FftPlan& p, int xt) {
    return xt == 32 && (plan_is(p, 9, 5, 5) || plan_is(p, 9, 4, 5));
}
ASARF_HD inline bool block_schedule_compiled(const FftPlan& p) { return plan_is(p, 5, 5, 5) || plan_is(p, 8, 7, 3); }

struct AzStridedArgs {
    const float2* in;
    float2* out;
    long long pitch;
    int n1, n2;
    FftPlan plan1;
    const int* drev1;
    const float2* twn;    // exp(-2 pi i m / N), N = n1 * n2
    int nk;
    int xt;               // columns per block
    int valid_rows;       // forward: rows at or beyond this are zero
    const FocusState* state;  // inverse: rows outside the results window are not stored
    float scale;          // inverse: 1 / N as the reference multiplies
    int inverse;
    int use_tma;          // tile loaded by TMA (device only)
    int n1_box;           // rows per TMA box (n1 split into n1 / n1_box boxes of <= 256 rows)
    int out_row0;         // inverse: row r is stored at out + (r - out_row0) * pitch
    float* out_intensity; // inverse: when set, |z|^2 of row r goes to out_intensity + (r - out_row0) * pitch
                          // (floats) and no complex row is stored
    int compiled;         // 1: launch a compile-time instantiation of plan1's schedule when one exists
};

// Per range column constants of the range-Doppler block.
struct ColParams {
    float dc, dc_off, ka, cut_lo, cut_hi, den, dc_off_ka;
    float rden, rka;      // RN(1 / den), RN(1 / ka) for the exact divisions
    float pad;
    double r0_dr;         // R0 / range spacing (range walk metres -> pixels)
};

struct AzRdArgs {
    const float2* in;
    float2* out;
    long long pitch;
    int n1, n2, az_pad;
    FftPlan plan2;
    const int* drev2;
    int nk;
    int xt, hl, hr, wt;
    int chunk_rows;
    float prf, lambda, frac;
    float bin_step;       // prf / az_pad (float, as the reference divides)
    float half_prf;       // prf * 0.5
    double slant, range_spacing;
    float vr_poly[3];
    const FocusState* state;
    const float* win;     // 16 RCMC window taps
    int use_tma;
    int n2_box;           // rows per TMA box
    int absolute_phase;   // 1: multiply column x by exp(j (4 pi R0 / lambda + pi dc_off^2 / Ka)) (FP64)
    double lambda_d;      // wavelength, FP64
    int compiled;         // 1: launch a compile-time instantiation of plan2's schedule when one exists
};

// Split-precision form of the range-Doppler block's forward transform: n2 = radix * m,
// m-point DFTs on the tensor cores, one FP32 radix pass (tc.cuh, k_az_rd_split).
constexpr int kSplitK = 64;          // K of the DFT tile: m <= 32 complex inputs as (re, im) pairs
constexpr int kSplitN = 64;          // N: m <= 32 complex outputs as (re, im) pairs
constexpr int kSplitRows = 128;      // M: range columns of the tile (wt <= 128)
constexpr int kSplitMatrixBytes = kSplitN * kSplitK * 2;       // one bf16 B part (8 KB)
constexpr int kSplitTmemCols = 128;  // accumulator (64 columns) + A hi (32) + A lo (32), power of 2
// Byte offset of element (row, k) of a 16-bit tensor-core operand with K elements per row in
// the canonical no-swizzle K-major layout (8 x 8 core matrices of 128 contiguous bytes; K-adjacent
// core matrices 128 bytes apart, row-adjacent groups 16 K bytes apart).
ASARF_HD ASARF_INLINE unsigned int umma_offset(int row, int k, int kdim) {
    return static_cast<unsigned int>((row >> 3) * (kdim * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}
struct AzRdSplit {
    const unsigned char* bmat;  // B hi then lo, canonical K-major images (2 x kSplitMatrixBytes)
    const float2* tw;           // [radix][m]: W_n2^(r * k1(s)) for output slot s
    int radix, m;
};

struct TailVariant {
    int n_lines;
    int out_az;
    float ratio;
    int ng;
    float grsr[5];
    const float* rsl;     // nx gains
};

struct TailArgs {
    const float2* slc;
    const float* intensity;  // when set: |z|^2 rows (floats, same pitch) instead of the complex SLC
    long long pitch;
    const FocusState* state;
    int col0, nx;
    TailVariant tail[kNumTailVariants];
    float range_spacing;
    float ground_spacing;
    float* out;
    int out_pitch;
    // IMP product records instead of the float image (mds != nullptr): record y at
    // mds + y * (mds_hdr + 2 * ng), ng of the chosen variant; with out2 the float image is
    // also stored there (pitch out_pitch) for the product statistics
    float* out2;
    uint8_t* mds;
    int mds_hdr;
    float mds_cal;
};

// Statistics of the level-1 product written into its SQ ADS (CalculateStatistics /
// CalculateStatisticsImaged, main_flow.cc:666-676, through DevicePaddedImage::CalcMean /
// CalcStdDev): FP64 sums over pairs (x, y), pairs holding a NaN skipped.
struct ProductStatsArgs {
    int imaged;             // 1: IMP form, 0: IMS form (pairs = complex SLC pixels)
    const float2* slc;      // SLC of the results window starts at row state->first_line
    long long slc_pitch;
    int nx;                 // SLC columns
    const float* img;       // IMP form: ground-range float image [out_az][img_pitch]
    int img_pitch;
    int ng[kNumTailVariants], out_az[kNumTailVariants];
    const FocusState* state;
    double* part;           // [blocks][5]: pairs counted, sum x, sum y, sum x^2, sum y^2
    int blocks;
    float cal;
    double* out;            // 4 statistics as main.cc hands them to the product header
};

// Level-1 product records (ConditionResultsSLC / ConditionResultsDetected).
struct ConditionArgs {
    int product;            // 1: IMP from img, 2: IMS from slc
    const float* img;       // IMP input [y][stride]
    const float2* slc;      // IMS input [y][stride]
    long long stride;       // elements per input row
    int x_size, y_size;
    int hdr;                // record header bytes (zeroed)
    float cal;              // calibration constant
    uint8_t* dest;
    const FocusState* state;  // fused IMS: rows first_line .. first_line + n_lines of slc
};

// ------------------------------------------------------------------ per-stage entry points
// (the reference's sar/ functions one by one, on its padded complex image layout)

struct DecodeArgs {
    const uint8_t* raw;
    long long line_bytes;
    int spl, lines, nr;
    const uint16_t* swst;
    int min_swst;
    float2* img;
    long long stride;   // complex elements per image row
};

// ERS IM level-0 measurement data set (ERS_SAR_0P MDSRs of 11498 bytes) -> raw lines
// (ParseErsLevel0ImPackets, envisat_format/src/ers_im_parse.cc:356-580)
constexpr int kErsMdsrBytes = 11498;         // ers::highrate::MDSR_SIZE_BYTES
constexpr int kErsMeasurementBytes = 11232;  // ers::highrate::MEASUREMENT_DATA_SIZE_BYTES (5616 I/Q pairs)
constexpr int kErsMeasurementOffset = 266;   // 12 sensing time + 20 FEP + 4 record no. + 10 IDHT + 220 auxiliary
constexpr unsigned kErrL0IspLength = 1u << 0;   // a packet's FEP ISP length is not 11465
constexpr unsigned kErrL0AuxMarker = 1u << 1;   // a packet's auxiliary section does not start with 0xAA
struct ErsUnpackArgs {
    const uint8_t* mdsr;      // packets, in file order
    const long long* offset;  // per line: byte offset of its packet in mdsr
    int lines;
    uint8_t* raw;             // [lines][kErsMeasurementBytes]
    uint16_t* swst;           // per line SWST code (nullable)
    uint16_t* pri;            // per line PRI code (nullable)
    unsigned int* errors;     // kErrL0* bits
};

// ENVISAT ASAR IM source packets (ASA_IM__0P measurement data set, variable length):
// 12 bytes ISP sensing time, 20 bytes FEP annotation (ISP length at 24), packet ID (32),
// sequence control (34), packet length (36), data field header length 29 (38), then the data
// field header (mode ID at 41, echo / noise / calibration flags at 52, PRI code at 54, SWST
// code at 56) and the FBAQ4 sample blocks from byte 68 (packet length - 29 bytes).  The next
// packet starts 39 + ISP length bytes after this one.
constexpr int kAsarPacketHeader = 68;
constexpr int kAsarNextPacketBase = 39;
constexpr unsigned kErrL0DataField = 1u << 0;   // a packet's data field header length is not 29
constexpr unsigned kErrL0Mode = 1u << 1;        // a packet's mode ID is not 0x54 (IM)
constexpr unsigned kErrL0Length = 1u << 2;      // a packet's sample blocks do not fit the record
struct AsarUnpackArgs {
    const uint8_t* mdsr;      // packets, in file order
    const long long* src;     // per line: byte offset of the echo packet whose sample blocks it holds
    int lines;
    int record_bytes;         // 2-byte length + the largest block-data length of the lines
    uint8_t* records;         // [lines][record_bytes]: FBAQ4 records
    uint16_t* swst;           // per line SWST code (nullable)
    uint16_t* pri;            // per line PRI code (nullable)
    unsigned int* errors;     // kErrL0DataField / kErrL0Mode / kErrL0Length bits
};

// ASAR FBAQ4 records -> complex rows, NaN where no sample (ConvertAsarImBlocksToComplex)
struct DecodeFbaqArgs {
    const uint8_t* raw;
    long long line_bytes;   // record stride: 2 length bytes + block data
    int lines, nr;
    const uint16_t* swst;
    int min_swst;
    const float* lut_i;     // 4096 entries, [level][block id] order of the instrument file
    const float* lut_q;
    float2* img;
    long long stride;
};

// NaN-aware moment partials of rows [row0, row0 + rows) per block: data region x < x_size
// and padding region x_size <= x < x_stride, 12 doubles per block:
// n, sI, sQ, sII, sQQ, sIQ (data) then the same six for the padding.
struct ImgMomentsArgs {
    const float2* img;
    int x_size, y_size, x_stride;
    int rows_per_block;
    double* partial;    // [blocks][12]
    float mean_i, mean_q;   // second pass: sums of (I - mean)^2, (Q - mean)^2 over the data region
    int centered;
};

struct IqApplyArgs {
    float2* img;
    int x_stride, y_size;
    float dc_i, dc_q, gain, sin_c, cos_c;
};

struct AcccArgs {
    const float2* img;
    int x_size, y_size, x_stride;
    int step, nblk, rows_per_block;
    double* partial;    // [blocks][nblk][2]
};

struct RcRowsArgs {
    float2* img;          // in place, rows y < y_size
    long long stride;
    int nr, nk, x_zero_end;  // inputs x < nr; keep x < nk; zero [nk, x_zero_end)
    FftPlan plan;
    const float2* mf;
};

struct MultilookArgs {
    const float2* slc;
    int x_size, in_y, out_y;
    float ratio;
    float* out;
};

struct RslArgs {
    float* img;
    int range_size, az_size;
    double slant_first, range_spacing, ref_range;
};

struct SrgrArgs {
    const float* in;
    int in_x, y_size, out_x;
    float grsr[5];
    float range_spacing, ground_spacing;
    float* out;
    int* start;           // optional index map
    float* frac;
    unsigned int* err;
};

}  // namespace asarf
