// Execution backend of the planner: the CUDA kernels (kernels.cu, the product) or the
// single-threaded host emulation of the same kernel bodies (emu.cpp, built only for the
// CPU test suite as a separate library).
#pragma once

#include <cstddef>

#include "params.h"

namespace asarf {

struct LaunchShape {
    int threads;
    size_t smem;
};

// grid (ceil(nr / kStatsCols), ceil(na / lines_per_cta)), kStatsCols threads
int backend_raw_stats(const RawStatsArgs& a, int gx, int gy, void* stream);
int backend_finalize(const FinalizeArgs& a, void* stream);
// ASAR FBAQ4 records: FP64 statistics tiles (gx = tiles_x, gy line tiles) and their fold
int backend_raw_stats_fbaq(const RawStatsArgs& a, int gx, int gy, void* stream);
int backend_stats_fold(const RawStatsArgs& a, int tiles_y, void* stream);
int backend_range_compress(const RangeCompressArgs& a, int lines, LaunchShape sh, void* stream);
int backend_az_strided(const AzStridedArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh, void* stream);
int backend_az_rd(const AzRdArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh, unsigned int* err,
                  void* stream);
// split-precision range-Doppler block (tensor-core forward transform); device build only
int backend_az_rd_split(const AzRdArgs& a, const AzRdSplit& sp, const void* tmap, int tiles, int nblocks,
                        LaunchShape sh, unsigned int* err, void* stream);
int backend_tail(const TailArgs& a, int rows, LaunchShape sh, unsigned int* err, void* stream);
int backend_condition(const ConditionArgs& a, int rows, void* stream);
int backend_product_stats(const ProductStatsArgs& a, void* stream);  // partials then fold

// per-stage kernels
int backend_decode(const DecodeArgs& a, long long n, void* stream);
int backend_decode_fbaq(const DecodeFbaqArgs& a, long long n, void* stream);
int backend_img_moments(const ImgMomentsArgs& a, int blocks, void* stream);
int backend_iq_apply(const IqApplyArgs& a, long long n, void* stream);
int backend_zero_nans(float2* img, long long n, void* stream);
int backend_accc(const AcccArgs& a, int blocks, void* stream);
int backend_rc_rows(const RcRowsArgs& a, int rows, LaunchShape sh, void* stream);
int backend_multilook(const MultilookArgs& a, void* stream);
int backend_ers_unpack(const ErsUnpackArgs& a, void* stream);
int backend_asar_unpack(const AsarUnpackArgs& a, void* stream);
int backend_rsl(const RslArgs& a, long long n, void* stream);
int backend_srgr(const SrgrArgs& a, long long n, void* stream);

void* mem_alloc(size_t bytes);
void mem_free(void* p);
int mem_h2d(void* dst, const void* src, size_t n, void* stream);
int mem_d2h(void* dst, const void* src, size_t n, void* stream);
int mem_d2d(void* dst, const void* src, size_t n, void* stream);
int mem_d2d_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows, void* stream);
int mem_zero(void* dst, size_t n, void* stream);
int stream_sync(void* stream);
void* event_create();
void event_destroy(void* e);
int event_record(void* e, void* stream);
int event_elapsed(void* a, void* b, float* ms);
int event_sync(void* e);
size_t smem_optin_limit();
int backend_sm_count();  // streaming multiprocessors of the current device
// Streams, cross-stream waits and CUDA graphs (device build).  The host emulation has no
// graphs: graphs_supported() is false there and callers run their sequence directly.
void* stream_create();
void stream_destroy(void* s);
int stream_wait_event(void* stream, void* event);
bool graphs_supported();
int graph_capture_begin(void* stream);
int graph_capture_end(void* stream, void** exec);
int graph_launch(void* exec, void* stream);
void graph_destroy(void* exec);
const char* backend_name();
// Encode a float32 tiled tensor map (128-byte blob) of `rank` dims: dims[rank] innermost
// first, strides[rank-1] in bytes, box[rank]; zero fill out of bounds.
int backend_make_tmap(void* out, int rank, void* base, const unsigned long long* dims,
                      const unsigned long long* strides, const unsigned int* box);

// Records a message for asarf_last_error(); returns `code`.
int set_error(int code, const char* fmt, ...);

}  // namespace asarf
