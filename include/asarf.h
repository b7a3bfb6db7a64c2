/*
 * asar-focus B200 — C ABI of the range-Doppler focusing path.
 *
 * Plain C: fixed-width integers, doubles, and raw pointers.  Device pointers are CUDA
 * global-memory addresses on the current device; `stream` is a cudaStream_t (NULL = the
 * legacy default stream).  Every function returns ASARF_OK (0) or a negative status and
 * never throws; asarf_last_error() gives the message of the last failure on the calling
 * thread.  Nothing here allocates inside asarf_focus*(): all device memory is taken at
 * plan creation, so a focus call can be captured into a CUDA graph.
 *
 * Each entry point names the reference interface it replaces (paths relative to the
 * cgi-estonia-space/asar-focus source tree, v0.3.2).
 */
#ifndef ASARF_H_
#define ASARF_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASARF_OK 0
#define ASARF_ERR_INVALID (-1)   /* bad argument; reference: std::logic_error / CHECK_BOOL */
#define ASARF_ERR_CUDA (-2)      /* CUDA runtime error; reference: alus::CudaErrorException */
#define ASARF_ERR_NOMEM (-3)     /* allocation failed */
#define ASARF_ERR_NUMERIC (-4)   /* non-convergence (geolocation) / degenerate fit */

/* One orbit state vector (sar/orbit_state_vector.h:24-32); time in microseconds. */
typedef struct asarf_osv {
    int64_t time_us;
    double pos[3];
    double vel[3];
} asarf_osv;

/* Raw record formats (asarf_scene.raw_format). */
#define ASARF_RAW_ERS_BYTES 0   /* ERS byte I/Q pairs (ConvertErsImSamplesToComplex) */
#define ASARF_RAW_ASAR_FBAQ4 1  /* ENVISAT ASAR FBAQ4 blocks (ConvertAsarImBlocksToComplex) */

/* Scene description: the fields of SARMetadata (sar/sar_metadata.h:57-88) that the
 * focusing path reads, plus the raw record layout of the decoder. */
typedef struct asarf_scene {
    int32_t range_size;        /* XSize of the decoded image: samples_per_line + k*(max_swst-min_swst),
                                  k = 4 (ERS) or 1 (ASAR) */
    int32_t azimuth_size;      /* YSize: number of echo lines */
    int32_t samples_per_line;  /* ERS: I/Q byte pairs per raw record; ASAR: the most samples of any record */
    int32_t raw_line_bytes;    /* byte stride of raw records; ERS: even, >= 2*samples_per_line;
                                  ASAR: 2 length bytes + block data (RawSampleMeasurements::single_entry_length + 2) */
    int64_t total_raw_samples; /* CorrectionParams::n_total_samples (sar/iq_correction.cuh:22-25) */
    /* ChirpInfo (sar/sar_metadata.h:34-44) */
    double range_sampling_rate;
    double chirp_kr;
    double pulse_duration;
    int32_t chirp_samples;     /* round(pulse_duration * fs) (main_flow.cc:391) */
    int32_t apply_window;      /* range Hamming window on the replica */
    /* radar / geometry */
    double prf;
    double wavelength;
    double carrier_frequency;
    double range_spacing;
    double slant_range_first;
    double azimuth_spacing;    /* AzimuthMultiLook ratio = 12.5 / azimuth_spacing */
    double az_bw_frac;         /* processed azimuth bandwidth / PRF */
    double vr_poly[3];         /* processing velocity polynomial (range pixel), highest power first */
    int32_t vr_poly_given;     /* 0: estimate it from the orbit (EstimateProcessingVelocity) */
    double vr_poly_init[3];    /* metadata Vr guess used for aperture lengths (main_flow.cc:465-473) */
    int32_t n_osv;
    const asarf_osv* osv;
    int64_t first_line_time_us;
    double line_time_interval;
    double center_point[3];    /* ECEF scene centre, initial guess of every geolocation */
    int32_t lines_before;      /* lines cached before sensing start (CalcResultsWindow) */
    int32_t lines_after;       /* lines cached after sensing stop */
    int32_t raw_format;        /* ASARF_RAW_ERS_BYTES (0) or ASARF_RAW_ASAR_FBAQ4 */
    /* ASAR FBAQ4: the instrument file's reconstruction tables (InstrumentFile fbp.i_LUT_fbaq4 /
     * q_LUT_fbaq4, envisat_format/include/envisat_aux_file.h:145-148), 4096 floats each at
     * index 256 * level + block id; read at plan creation only */
    const float* fbaq_i_lut;
    const float* fbaq_q_lut;
} asarf_scene;

/* What asarf_focus writes at d_out (asarf_options.product). */
#define ASARF_PRODUCT_DETECTED 0  /* float ground-range intensity [out_rows][out_cols_max] */
#define ASARF_PRODUCT_IMP_MDS 1   /* IMP level-1 MDS records: out_rows records of header + 2*out_cols bytes
                                     (FormatResultsDetected, main.cc:345-370) */
#define ASARF_PRODUCT_IMS_MDS 2   /* IMS level-1 MDS records of the complex SLC: n_lines records of
                                     header + 4*slc_cols bytes (FormatResultsSLC, main.cc:378-420) */

/* Options of the fused plan. */
typedef struct asarf_options {
    int32_t rc_fft_len;        /* range FFT length; 0 = auto (any >= range_size gives the same result) */
    int32_t ref_compat_stats;  /* 1 (default): gain/phase sums include the range padding as the reference does */
    int32_t iq_padding_ref;    /* range padding the reference would use for those sums; 0 = its own rule */
    int32_t dc_poly_given;     /* 1: use dc_poly instead of the ACCC estimate (the estimate is still reported) */
    double dc_poly[3];         /* Doppler centroid polynomial (range pixel), highest power first */
    int32_t product;           /* ASARF_PRODUCT_* (default ASARF_PRODUCT_DETECTED) */
    int32_t record_header_bytes; /* MDS record header, zero-filled (main.cc: 12 + 1 + 4 = 17, the default) */
    float calibration;         /* MDS calibration constant (main.cc: process gain / sqrt(scaling factor));
                                  default 1 */
    int32_t sq_stats;          /* 1: also compute the product statistics of the SQ ADS (asarf_results.sq_stats) */
    int32_t precision;         /* ASARF_PRECISION_* (default ASARF_PRECISION_FP32) */
    int32_t absolute_phase;    /* 1: zero-Doppler phase preserved: the azimuth matched filter also carries
                                  exp(j 4 pi R0 / lambda) (R0 = slant range of the column, FP64 on the GPU,
                                  reduced modulo 2 pi) and exp(j pi dc_off^2 / Ka); 0 (default): the
                                  reference's convention, whose SLC phase keeps -4 pi R0 / lambda
                                  (sar/range_doppler_algorithm.cu:265-290) */
    /* launch shapes (0 = the planner's choice; asarf.autotune times candidates and caches the best
     * per scene shape): */
    int32_t az_n2;             /* contiguous azimuth transform length n2 (az_pad = n1 * n2; a divisor of az_pad,
                                  16 <= n2 <= 256) */
    int32_t az_tile_width;     /* output range columns per range-Doppler block (even, 16..64) */
    int32_t strided_tile_width; /* range columns per strided-pass block (16 or 32) */
    int32_t keep_slc;          /* 1 (default): the complex SLC stays in device memory after a run
                                  (asarf_plan_slc, IMS records, the IMP product statistics);
                                  0: detected output only -- the inverse azimuth pass writes |z|^2 rows
                                  (half the bytes written, and read again by the multilook) */
    int32_t compiled_schedules; /* 1 (default): azimuth transforms whose radix schedule has a compile-time
                                  instantiation (strided 225 = 9*5*5 and 180 = 9*4*5 at 32 columns,
                                  blocks 125 = 5*5*5 and 168 = 8*7*3) run it; 0: run-time schedules only.
                                  Both give identical results */
} asarf_options;

/* Arithmetic of the azimuth transforms (asarf_options.precision).  The reference runs every
 * transform through cuFFT in FP32 (sar/range_doppler_algorithm.cu:319-323, 385-389). */
#define ASARF_PRECISION_FP32 0   /* FP32 mixed-radix transforms on the CUDA cores */
#define ASARF_PRECISION_SPLIT 1  /* forward contiguous azimuth transform of length n2 = R * m (m <= 32) as
                                    m-point DFT tiles on the tensor cores (tcgen05, bf16 hi + lo operands,
                                    three products, FP32 accumulation) and one FP32 radix-R pass; plans
                                    whose n2 has no such split keep FP32 (asarf_dims.precision) */

/* Output geometry of a plan (both tail variants: the Doppler-centroid sign picks one). */
typedef struct asarf_dims {
    int32_t nk;                /* range samples after range compression */
    int32_t rg_pad_ref, az_pad;
    int32_t rc_fft_len, n1, n2;
    int32_t slc_cols;          /* nk - 16 */
    int32_t out_rows[2];       /* multilooked lines, variant 0 (DC > 0) / 1 */
    int32_t out_cols[2];       /* ground-range samples */
    int32_t out_rows_max, out_cols_max;
    int32_t max_aperture;
    double vr_poly[3];
    size_t device_bytes;       /* device memory held by the plan */
    int64_t out_bytes_max;     /* bytes asarf_focus may write at d_out for the plan's product */
    int32_t precision;         /* ASARF_PRECISION_* the plan runs (SPLIT falls back to FP32 where n2 does not split) */
    int32_t split_radix, split_m; /* with SPLIT: n2 = split_radix * split_m */
    int32_t az_tile_width, strided_tile_width; /* launch shapes in use */
    int32_t compiled_schedules; /* bit 0: the strided passes, bit 1: the range-Doppler block run a
                                   compile-time schedule */
} asarf_dims;

/* Per-run results: SARResults (sar/sar_metadata.h:46-55) plus the chosen window. */
typedef struct asarf_results {
    double dc_i, dc_q, iq_gain, phase_error, stddev_i, stddev_q;
    double doppler_centroid_poly[3];     /* polynomial used (estimate unless overridden) */
    double doppler_centroid_estimate[3]; /* ACCC estimate (CalculateDopplerCentroid) */
    double vr_poly[3];
    int32_t n_dc_blocks;
    double dc_block_hz[80];
    int32_t variant, first_line, n_lines, out_rows, out_cols;
    uint32_t errors;
    int32_t records, record_bytes;  /* rows written at d_out and their byte stride (product layout) */
    /* with asarf_options.sq_stats: the statistics main.cc writes into the product header,
     * scaled by the calibration constant as there (main.cc:331-342 IMP, 380-390 IMS):
     * IMS (mean I, mean Q, std I, std Q) of the SLC (CalculateStatistics, main_flow.cc:666-670);
     * otherwise the IMP form ((mean I + mean Q) / 2, 0, (std I + std Q) / 2, 0) over the
     * ground-range buffer viewed as complex (CalculateStatisticsImaged, main_flow.cc:672-676) */
    double sq_stats[4];
} asarf_results;

typedef struct asarf_plan asarf_plan;

const char* asarf_last_error(void);
const char* asarf_version(void);

void asarf_default_options(asarf_options* opt);

/* Plan one scene shape: sizes, FFT schedules, chirp matched filter, Vr polynomial, SRGR
 * polynomials, device buffers.  Replaces the setup in main.cc:213-269 (FFT sizes, chirp,
 * Vr estimation, workspace allocation). */
int asarf_plan_create(const asarf_scene* scene, const asarf_options* opt, asarf_plan** out);
void asarf_plan_destroy(asarf_plan* plan);
int asarf_plan_dims(const asarf_plan* plan, asarf_dims* dims);

/* Focus one scene from device-resident raw bytes to the plan's product at d_out (default: the
 * detected ground-range image, float [out_rows][out_cols_max], row pitch out_cols_max; see
 * ASARF_PRODUCT_* for the level-1 record forms, asarf_dims.out_bytes_max for the size).  Replaces main.cc:233-327:
 * ConvertErsImSamplesToComplex (FBAQ4 records: ConvertAsarImBlocksToComplex) +
 * RawDataCorrection + ZeroNaNs + CalculateDopplerCentroid +
 * RangeCompression + RangeDopplerAlgorithm + SubsetResultsAndReassembleMeta +
 * AzimuthMultiLook + RangeSpreadingLossCorrection + SlantRangeToGroundRangeInterpolation.
 * swst may be NULL (all lines start at range sample 0). Asynchronous on `stream`. */
int asarf_focus(asarf_plan* plan, const uint8_t* d_raw, const uint16_t* d_swst, int32_t min_swst, float* d_out,
                void* stream);

/* Same from HOST buffers: copies raw bytes (and SWST codes) in, the image out, inside the
 * call, then synchronises `stream`.  Host buffers may be pageable or pinned. */
int asarf_focus_host(asarf_plan* plan, const uint8_t* h_raw, const uint16_t* h_swst, int32_t min_swst, float* h_out,
                     void* stream);

/* The work of asarf_focus_host (raw and SWST upload, focus run, image download), enqueued on
 * `stream` -- or, when stream is NULL, on the plan's own non-blocking stream -- and returned
 * from without waiting.  With page-locked host buffers the copies are asynchronous, so
 * scenes submitted to different plans overlap: one scene's upload and another's download
 * run on the copy engines while a third is focused.  Neither host buffer may be touched,
 * nor asarf_plan_results read, until asarf_plan_wait(plan) has returned.  Main.cc's
 * per-file flow (main.cc:233-327) runs one scene per process; this is its multi-scene form. */
int asarf_focus_host_async(asarf_plan* plan, const uint8_t* h_raw, const uint16_t* h_swst, int32_t min_swst,
                           float* h_out, void* stream);

/* Block until everything asarf_focus_host_async last enqueued on this plan has finished
 * (immediately when nothing was enqueued). */
int asarf_plan_wait(asarf_plan* plan);

/* Copy the complex subset SLC (IMS tail input) of the last run: complex float
 * [n_lines][slc_cols] into d_slc (row pitch slc_cols).  Asynchronous. */
int asarf_plan_slc(asarf_plan* plan, void* d_slc, void* stream);

/* Per-kernel timing: record CUDA events between the kernel launches of the next `runs`
 * asarf_focus calls (0 disables).  No counterpart in the reference (it has wall-clock
 * TimeStart/TimeStop logging only, main.cc:63-69). */
int asarf_plan_enable_timing(asarf_plan* plan, int32_t runs);
/* Sum of each kernel's event-timed duration over the recorded runs (7 kernels: raw_stats,
 * finalize, range_compress, az_strided_fwd, az_rd, az_strided_inv, tail); synchronises on
 * the events, then clears them.  `names` (optional) receives 7 static strings. */
int asarf_plan_kernel_times(asarf_plan* plan, float* total_ms, int32_t* runs, const char** names);

/* Results of the last run (synchronises `stream`). */
int asarf_plan_results(asarf_plan* plan, asarf_results* res, void* stream);

/* ---------------------------------------------------------------- allocation-free statistics */

/* Output of asarf_raw_statistics_noalloc (written to device memory). */
typedef struct asarf_raw_stats {
    double dc_i, dc_q, iq_gain, phase_error, stddev_i, stddev_q;
    double doppler_centroid_poly[3]; /* ACCC estimate, highest power first */
    int32_t n_dc_blocks;
    int32_t reserved;
    double dc_block_hz[80];
    float applied_dc_i, applied_dc_q, applied_gain, applied_sin, applied_cos;
    uint32_t errors;
} asarf_raw_stats;

/* IQ statistics and Doppler-centroid estimate of device-resident raw ERS byte-I/Q data,
 * taking no device memory at all.  This entry point has no counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc: a check that runs while a CUDA graph is
 * being captured, a host application whose own allocator owns all device memory, or a
 * real-time ingest loop that cannot afford cudaMalloc's implicit synchronisation.  It
 * computes what asarf_focus computes first (the statistics of RawDataCorrection and the
 * estimate of CalculateDopplerCentroid) and writes them to `d_out`, a device buffer the
 * caller owns.  Its only scratch is a fixed 8 KiB array in this library's static device
 * memory, held on every GPU that loads the library until exit; it bounds the number of
 * Doppler blocks to 80 and larger counts are rejected with ASARF_ERR_INVALID (blocks are
 * floor(range_size / 32) samples wide, so range_size 32..63 gives range_size blocks, at most
 * 63, and every larger size gives 32 to 63: the bound is never reached).  All calls on a
 * device share that array: calls whose work overlaps on the GPU race, so issue them in order
 * on one stream.  The first call in each CUDA context looks up the array's device address
 * (cudaGetSymbolAddress), keyed by the context's id: after cudaDeviceReset, or under a host
 * application's own driver context, the next call looks it up again.  Make that first call
 * in a context before any stream capture.  `stats_stride` is the padded width the reference
 * runs its gain / phase sums over (its range FFT size; 0 = data samples only). */
int asarf_raw_statistics_noalloc(const uint8_t* d_raw, int32_t raw_line_bytes, int32_t samples_per_line,
                                 int32_t range_size, int32_t azimuth_size, const uint16_t* d_swst, int32_t min_swst,
                                 int64_t total_raw_samples, int32_t stats_stride, double prf, asarf_raw_stats* d_out,
                                 void* stream);

/* ---------------------------------------------------------------- ERS level-0 packets */

/* ENVISAT-format time: days since 2000-01-01, seconds of the day, microseconds (mjd,
 * envisat_format/include/envisat_types.h:37-72). */
typedef struct asarf_mjd {
    int32_t days;
    uint32_t seconds;
    uint32_t micros;
} asarf_mjd;

/* FetchErsL0ImForecastMeta (envisat_format/src/ers_im_parse.cc:228-354) over the measurement
 * data set of an ERS_SAR_0P product held in host memory (`mdsr`, `blob_bytes` = num_dsr *
 * dsr_size): the packet of each line (byte offset into mdsr) and its sensing time.  A packet
 * whose data record number skips ahead is preceded by copies of the previous packet (at most
 * 900, else ASARF_ERR_INVALID with the reference's message); packets before `start` / after
 * `stop` are counted and trimmed to *packets_before_start / *packets_after_stop, which return
 * the counts kept, as in the reference.  offsets / times (nullable) receive *count entries,
 * `capacity` bounds them.  No PATC sensing-time correction is applied (the reference applies
 * one only when a PATC auxiliary file is registered). */
int asarf_ers_l0_forecast(const uint8_t* mdsr, int64_t blob_bytes, int64_t num_dsr, int64_t dsr_size,
                          const asarf_mjd* start, const asarf_mjd* stop, int64_t* packets_before_start,
                          int64_t* packets_after_stop, int64_t* offsets, asarf_mjd* times, int64_t capacity,
                          int64_t* count);
/* ParseErsLevel0ImPackets (envisat_format/src/ers_im_parse.cc:356-580) on the GPU: the packets
 * as they lie in the file (d_mdsr, device memory, 2-byte aligned), one kernel for all `lines`:
 * line y's 11232 measurement bytes -> d_raw + y * 11232 (the byte I/Q layout asarf_focus reads,
 * raw_line_bytes = 11232), its SWST and PRI codes -> d_swst[y], d_pri[y] (nullable).  A packet
 * whose FEP ISP length is not 11465 or whose auxiliary section does not start with 0xAA sets
 * bit 0 / bit 1 of *d_errors (device memory, not cleared here).  Asynchronous on `stream`. */
int asarf_ers_l0_unpack(const uint8_t* d_mdsr, const int64_t* d_offsets, int32_t lines, uint8_t* d_raw,
                        uint16_t* d_swst, uint16_t* d_pri, uint32_t* d_errors, void* stream);

/* FetchEnvisatL0ImForecastMeta (envisat_format/src/envisat_im_parse.cc:297-385) over the
 * measurement data set of an ASA_IM__0P product in host memory: `num_dsr` source packets of
 * variable length from `mdsr` (each 39 + its FEP ISP length bytes; `blob_bytes` bounds the walk).
 * Lines are the echo and calibration packets from the first echo packet on (noise packets
 * skipped); the sensing-time window, counts and trimming as asarf_ers_l0_forecast, and a
 * calibration packet left first after trimming is dropped (the reference accepts that only
 * when the walk's last packet was a calibration packet, else ASARF_ERR_INVALID with its
 * "Programming error" message).  A data field header length other than 29 is an error. */
int asarf_asar_l0_forecast(const uint8_t* mdsr, int64_t blob_bytes, int64_t num_dsr, const asarf_mjd* start,
                           const asarf_mjd* stop, int64_t* packets_before_start, int64_t* packets_after_stop,
                           int64_t* offsets, asarf_mjd* times, int64_t capacity, int64_t* count);
/* The host part of ParseEnvisatLevel0ImPackets (:387-676) for `count` forecast lines:
 * *record_bytes = 2 + the largest echo block-data length (packet length - 29) over `count`
 * consecutive packets from the first line's (ForecastMaxBlockDataLength, :159-197; fewer than
 * 10 echo packets is an error); src_offsets[k] = the packet whose sample blocks line k holds
 * (its own for an echo, the previous line's for a calibration packet), times[k] (nullable) its
 * sensing time (a calibration line: the previous line's plus uint32(1 / (range_sampling_rate /
 * PRI code) * 1e6) microseconds, in the reference's float arithmetic), *max_samples (nullable)
 * the most samples a line holds.  Mode IDs other than 0x54 (IM) and the reference's other
 * consistency failures are errors with its messages, and so is an echo packet whose sample
 * blocks end past blob_bytes (the unpack kernel reads them from the device copy). */
int asarf_asar_l0_lines(const uint8_t* mdsr, int64_t blob_bytes, const int64_t* offsets, int64_t count,
                        float range_sampling_rate, int64_t* src_offsets, asarf_mjd* times, int32_t* record_bytes,
                        int32_t* max_samples);
/* The record copy of ParseEnvisatLevel0ImPackets on the GPU, one kernel for all `lines`: line y
 * <- the sample blocks of the packet at d_mdsr + d_src_offsets[y] (device memory) as an FBAQ4
 * record of `record_bytes` at d_records + y * record_bytes (2-byte little-endian block-data
 * length, the blocks, zeros; the layout asarf_focus reads with raw_line_bytes = record_bytes),
 * its SWST and PRI codes -> d_swst[y], d_pri[y] (nullable).  Bits of *d_errors (device memory,
 * not cleared here): 0 data field header length not 29, 1 mode ID not 0x54, 2 block data longer
 * than the record (the record keeps what fits).  Asynchronous on `stream`. */
int asarf_asar_l0_unpack(const uint8_t* d_mdsr, const int64_t* d_src_offsets, int32_t lines, int32_t record_bytes,
                         uint8_t* d_records, uint16_t* d_swst, uint16_t* d_pri, uint32_t* d_errors, void* stream);

/* ---------------------------------------------------------------- host FP64 geometry */

/* InterpolateOrbit (sar/orbit_state_vector.cc:23-48). */
int asarf_interpolate_orbit(const asarf_osv* osv, int32_t n, int64_t time_us, asarf_osv* out);
/* RangeDopplerGeoLocate (util/src/geo_tools.cc:27-85). */
int asarf_geolocate(const double vel[3], const double pos[3], const double init_guess[3], double slant_range,
                    double out_xyz[3]);
/* Polyfit (util/src/math_utils.cc:23-44), highest power first, n <= 128, degree <= 4. */
int asarf_polyfit(const double* x, const double* y, int32_t n, int32_t degree, double* coeffs);
/* EstimateProcessingVelocity (sar/processing_velocity_estimation.cc:105-148). */
int asarf_estimate_processing_velocity(const asarf_scene* scene, double vr_poly[3]);
/* GenerateChirpData (sar/sar_chirp.cc:70-104): padded, windowed, power-normalised replica. */
int asarf_generate_chirp(double kr, double fs, int32_t n_samples, int32_t apply_window, int32_t padding,
                         float* out_interleaved);
/* SRGR polynomial of SlantRangeToGroundRangeInterpolation (sar/srgr.cu:73-121). */
int asarf_srgr_polynomial(const asarf_scene* scene, double slant_first, int32_t range_size, int32_t azimuth_size,
                          double line_time_interval, double poly[5], int32_t* ground_samples);
/* GetOptimalFFTSizes().upper_bound(v) (cuda_util/cufft_plan.cc:147-181, main.cc:217,223). */
int32_t asarf_fft_size_above(int32_t v);

/* ---------------------------------------------------------------------------------------
 * Batches of independent segments of uneven size.  No reference counterpart: the reference
 * focuses one scene per process run (main.cc:176-327).  Each segment gets its own plan;
 * asarf_batch_focus captures every segment's kernels once into a CUDA graph whose branches
 * (up to `branches` side streams, segments dealt largest first) run concurrently, and
 * replays it on later calls with the same buffers (new buffers: a new capture; the first
 * call with a set of buffers also runs the segments once directly, outside the capture).
 * ------------------------------------------------------------------------------------- */
typedef struct asarf_batch asarf_batch;

/* opts: NULL or one asarf_options per scene; branches <= 0 means 4. */
int asarf_batch_create(const asarf_scene* scenes, int32_t n, const asarf_options* opts, int32_t branches,
                       asarf_batch** out);
void asarf_batch_destroy(asarf_batch* batch);
/* The plan of segment i (owned by the batch): dims, results, SLC access. */
int asarf_batch_plan(asarf_batch* batch, int32_t i, asarf_plan** out);
/* Branch (side stream index) segment i runs on, -1 if i is out of range. */
int asarf_batch_branch(const asarf_batch* batch, int32_t i);
/* Segment i: raw bytes d_raw[i], SWST codes d_swst[i] (d_swst may be NULL, or hold NULLs),
 * min_swst[i] (NULL = 0), detected output d_out[i] (asarf_focus's layout). */
int asarf_batch_focus(asarf_batch* batch, const uint8_t* const* d_raw, const uint16_t* const* d_swst,
                      const int32_t* min_swst, float* const* d_out, void* stream);
/* Longest-processing-time assignment of n work items to `bins` bins (largest item first,
 * to the least-loaded bin): the rule that deals segments to graph branches and to GPUs. */
int asarf_lpt_assign(const int64_t* work, int32_t n, int32_t bins, int32_t* out_bin);

/* ---------------------------------------------------------------------------------------
 * Long strips as overlapped azimuth blocks.  No reference counterpart: the reference focuses
 * a scene as one padded image and does not support an azimuth-varying Doppler centroid.
 * Blocks of block_lines lines start (block_lines - overlap) apart (the last one ends at the
 * strip's last line); each is an ordinary plan with its own IQ statistics, Doppler estimate
 * and Vr (from the orbit at its own azimuth time unless the scene gives Vr), and writes the lines between the
 * midpoints of its overlaps (past one synthetic aperture at the strip ends) into one strip
 * SLC; one multilook + RSL + SRGR pass then runs over the whole strip.  overlap must be at
 * least the synthetic aperture in lines.
 * ------------------------------------------------------------------------------------- */
typedef struct asarf_strip asarf_strip;

typedef struct asarf_strip_dims {
    int32_t n_blocks, block_lines, overlap;
    int32_t first_line;        /* strip line of the first SLC row */
    int32_t slc_rows, slc_cols, slc_pitch;
    int32_t out_rows, out_cols; /* detected ground-range image, row pitch out_cols */
    int32_t max_aperture;
    size_t device_bytes;
} asarf_strip_dims;

int asarf_strip_create(const asarf_scene* scene, int32_t block_lines, int32_t overlap, const asarf_options* opt,
                       asarf_strip** out);
void asarf_strip_destroy(asarf_strip* strip);
int asarf_strip_get_dims(const asarf_strip* strip, asarf_strip_dims* dims);
/* Block k: first strip line, kept block-relative lines [keep_lo, keep_hi), its plan (owned by
 * the strip; asarf_plan_results gives the block's own statistics and Doppler estimate). */
int asarf_strip_block(const asarf_strip* strip, int32_t k, int32_t* start, int32_t* keep_lo, int32_t* keep_hi,
                      asarf_plan** plan);
/* Raw strip bytes [azimuth_size][raw_line_bytes] -> detected image [out_rows][out_cols].
 * Blocks run concurrently on the strip's side streams, forked from and joined into `stream`. */
int asarf_focus_strip(asarf_strip* strip, const uint8_t* d_raw, const uint16_t* d_swst, int32_t min_swst,
                      float* d_out, void* stream);
/* Copy the strip SLC, complex [slc_rows][slc_cols] (row pitch slc_cols), into d_slc. */
int asarf_strip_slc(asarf_strip* strip, void* d_slc, void* stream);
/* Error flags of the last run over every block and the strip tail (synchronises). */
int asarf_strip_errors(asarf_strip* strip, uint32_t* errors, void* stream);

/* ---------------------------------------------------------------------------------------
 * Per-stage entry points: the reference's sar/ functions one at a time, for a caller that
 * keeps the reference's own pipeline (main.cc) and swaps stages.  Images use the layout of
 * DevicePaddedImage (cuda_util/device_padded_image.cuh:13-27): complex float
 * [y_stride][x_stride] on the device, data block [0, y_size) x [0, x_size) at the top left.
 * Like the reference functions these allocate their own temporaries and synchronise
 * `stream` before returning; the planned asarf_focus path above is the fused, allocation-
 * free form of the same chain.
 * ------------------------------------------------------------------------------------- */

/* SARResults fields written by RawDataCorrection (sar/sar_metadata.h:46-55). */
typedef struct asarf_iq_results {
    double dc_i, dc_q;         /* CalcMean over the data block, float as the reference keeps it */
    double iq_gain;            /* sqrt(sum I^2 / sum Q^2) after the DC step */
    double phase_error;        /* degrees */
    double stddev_i, stddev_q; /* CalcStdDev over the data block */
} asarf_iq_results;

/* The SARMetadata fields RangeDopplerAlgorithm reads (sar/range_doppler_algorithm.cu:340-360). */
typedef struct asarf_rda_params {
    double prf;
    double wavelength;
    double range_spacing;
    double slant_range_first;
    double az_bw_frac;
    double vr_poly[3];         /* results.Vr_poly, highest power first */
    double dc_poly[3];         /* results.doppler_centroid_poly, highest power first */
} asarf_rda_params;

/* ConvertErsImSamplesToComplexKernel (envisat_format/src/envisat_format_kernels.cu:116-134)
 * with the NaN pre-fill of main_flow.cc:537-540: raw byte I/Q records -> complex rows of
 * `range_size` samples, shifted right by 4*(swst[y]-min_swst) (d_swst may be NULL), samples
 * outside the record NaN.  Writes columns [0, range_size) of `lines` rows of d_img. */
int asarf_convert_ers_samples(const uint8_t* d_raw, int32_t raw_line_bytes, int32_t samples_per_line, int32_t lines,
                              const uint16_t* d_swst, int32_t min_swst, void* d_img, int64_t img_stride,
                              int32_t range_size, void* stream);
/* ConvertAsarImBlocksToComplexKernel (envisat_format/src/envisat_format_kernels.cu:160-209) with
 * the NaN pre-fill of main_flow.cc:537-540, on device buffers: FBAQ4 records of `record_bytes`
 * bytes (2-byte little-endian block-data length, then 64-byte blocks of a block id and 63
 * codewords) -> complex rows of `range_size` samples, record y shifted right by
 * swst[y] - min_swst (d_swst may be NULL), samples the record does not hold NaN.  d_lut_i /
 * d_lut_q: the 4096-entry reconstruction tables on the device, instrument-file order. */
int asarf_convert_asar_blocks(const uint8_t* d_raw, int32_t record_bytes, int32_t records, const uint16_t* d_swst,
                              int32_t min_swst, const float* d_lut_i, const float* d_lut_q, void* d_img,
                              int64_t img_stride, int32_t range_size, void* stream);
/* ConditionResultsSLC (envisat_format/src/envisat_format_kernels.cu:28-61, 95-106): IMS MDS records
 * from a complex image (x_size x y_size, x_stride complex per row): per row `record_header_bytes`
 * zeros, then per pixel big-endian int16 I and Q of trunc(clamp(value * calibration)).
 * d_dest receives y_size * (record_header_bytes + 4 * x_size) bytes. */
int asarf_condition_slc(const void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride,
                        int32_t record_header_bytes, float calibration, void* d_dest, void* stream);
/* ConditionResultsDetected (:63-93, 108-114): IMP MDS records from a float image
 * [azimuth_size][range_size]: per row the zero header, then per pixel
 * uint16(min(10 log10(value * calibration), 65535)), least significant byte first. */
int asarf_condition_detected(const float* d_img, int32_t range_size, int32_t azimuth_size,
                             int32_t record_header_bytes, float calibration, void* d_dest, void* stream);
/* Fbaq4Index (envisat_format/include/envisat_parse_util.h:21): reconstruction-table index of
 * the 4-bit code `code` in a block with block id `block` (256 * level + block). */
int32_t asarf_fbaq4_index(int32_t block, int32_t code);
/* RawDataCorrection (sar/iq_correction.cu:188-274): means and deviations over the data
 * block (NaN samples skipped, divided by n_total_samples; <= 0 means x_size*y_size), then
 * DC, gain and phase correction applied over x < x_stride, y < y_size with the gain and
 * phase statistics taken over that same region, as the reference does. */
int asarf_raw_data_correction(void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, int32_t y_stride,
                              int64_t n_total_samples, asarf_iq_results* results, void* stream);
/* DevicePaddedImage::ZeroNaNs (cuda_util/device_padded_image.cu:69-85, 322-329). */
int asarf_zero_nans(void* d_img, int32_t x_stride, int32_t y_stride, void* stream);
/* CalculateDopplerCentroid (sar/fractional_doppler_centroid.cu:98-139): ACCC phase over
 * 32 range blocks of x_size/32 columns (the last one may reach into the padding, as in the
 * reference), quadratic fit of the block centroids; poly highest power first.  Pair sums
 * are FP64 in a fixed order (the reference sums float partials). */
int asarf_doppler_centroid(const void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, double prf,
                           double poly[3], void* stream);
/* RangeCompression (sar/range_compression.cu:57-111) in place: chirp_padded is
 * ChirpInfo::padded_windowed_data (interleaved re/im, chirp_len = x_stride complex samples,
 * else "Range padding and chirp size mismatch"); rows y < y_size keep x < x_size -
 * chirp_samples compressed samples and are zero from there to x_stride.  *new_x_size gets
 * the new XSize.  The range FFT length is chosen freely (>= x_size): the kept samples do
 * not depend on it. */
int asarf_range_compression(void* d_img, int32_t x_size, int32_t y_size, int32_t x_stride, const float* chirp_padded,
                            int32_t chirp_len, int32_t chirp_samples, int32_t* new_x_size, void* stream);
/* RangeDopplerAlgorithm (sar/range_doppler_algorithm.cu:312-407): azimuth FFT over all
 * y_stride rows of columns x < x_size (in place on d_src, which the reference also
 * consumes), 16-tap RCMC into d_out, azimuth matched filter, inverse FFT scaled by
 * 1/y_stride.  d_out (same shape) holds the focused block [0, y_size) x [0, x_size) and
 * zeros elsewhere (the reference leaves unscaled transform values in rows >= y_size).
 * y_stride must factor into 2, 3, 5 and 7. */
int asarf_range_doppler(const asarf_rda_params* prm, void* d_src, void* d_out, int32_t x_size, int32_t y_size,
                        int32_t x_stride, int32_t y_stride, void* stream);
/* AzimuthMultiLook / TimeDomainAzimuthLook (sar/az_multilook.cu:25-98) on a contiguous
 * complex [y_size][x_size] SLC: d_out float [out_y][x_size], out_y = round(y_size / ratio),
 * ratio = float(12.5 / azimuth_spacing).  d_out must hold that many rows. */
int asarf_azimuth_multilook(const void* d_slc, int32_t x_size, int32_t y_size, double azimuth_spacing, float* d_out,
                            int32_t* out_y, void* stream);
/* RangeSpreadingLossCorrection (sar/range_spreading_loss.cu:29-68) in place on a float
 * [azimuth_size][range_size] image. */
int asarf_range_spreading_loss(float* d_img, int32_t range_size, int32_t azimuth_size, double slant_range_first,
                               double range_spacing, double reference_range, void* stream);
/* SrGrInterpolation (sar/srgr.cu:49-71) with the polynomial of asarf_srgr_polynomial:
 * float [y_size][in_x] slant rows -> float [y_size][out_x] ground rows at 12.5 m.  An index
 * outside the slant row (the reference reads past it) is clamped to the last pair. */
int asarf_srgr(const float* d_in, int32_t in_x, int32_t y_size, const double grsr_poly[5], double range_spacing,
               int32_t out_x, float* d_out, void* stream);
/* The per-column (start index, fraction) map SrGrInterpolation computes, for inspection. */
int asarf_srgr_index(const double grsr_poly[5], double range_spacing, int32_t out_x, int32_t* d_start, float* d_frac,
                     void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ASARF_H_ */
