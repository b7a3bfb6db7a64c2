// Host emulation backend: runs the kernel bodies of bodies.cuh single-threaded on the CPU
// (tid = 0, nthr = 1, one block after another).  Built only into the test library
// libasarf_emu.so so the CPU test suite can check the exact kernel code against the
// oracle; the product library links kernels.cu instead and has no CPU path.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "context_cache.h"
#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"

namespace asarf {

namespace {
// Shared-memory stand-in with the device's 16-byte vector alignment.
struct TileBuf {
    std::vector<float4> v;
    explicit TileBuf(size_t bytes) : v(bytes / sizeof(float4) + 2) {}
    float2* data() { return reinterpret_cast<float2*>(v.data()); }
};
}  // namespace

int backend_raw_stats(const RawStatsArgs& a, int gx, int gy, void*) {
    RawStatsSmem sm;
    for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx) raw_stats_body(a, bx, by, 0, 1, &sm);
    return ASARF_OK;
}

int backend_raw_stats_fbaq(const RawStatsArgs& a, int gx, int gy, void*) {
    std::vector<FbaqStatsSmem> sm(1);
    for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx) raw_stats_fbaq_body(a, bx, by, 0, 1, sm.data());
    return ASARF_OK;
}

int backend_stats_fold(const RawStatsArgs& a, int tiles_y, void*) {
    std::vector<double> tree(6 * kFoldTree);
    stats_fold_body(a, tiles_y, 0, 1, tree.data());
    return ASARF_OK;
}

int backend_finalize(const FinalizeArgs& a, void*) {
    finalize_body(a);
    return ASARF_OK;
}

template <int L, int FMT>
static void emu_rc_ct(const RangeCompressArgs& a, int lines, float2* s) {
    for (int y = 0; y < lines; ++y) range_compress_ct_body<L, FMT>(a, y, 0, s, nullptr);
}

template <int FMT>
static void emu_rc(const RangeCompressArgs& a, int lines, LaunchShape sh) {
    std::vector<float2> s(sh.smem / sizeof(float2) + 1);
    switch (a.plan.n) {
        case 768: emu_rc_ct<768, FMT>(a, lines, s.data()); return;
        case 1024: emu_rc_ct<1024, FMT>(a, lines, s.data()); return;
        case 1536: emu_rc_ct<1536, FMT>(a, lines, s.data()); return;
        case 2048: emu_rc_ct<2048, FMT>(a, lines, s.data()); return;
        case 3072: emu_rc_ct<3072, FMT>(a, lines, s.data()); return;
        case 4096: emu_rc_ct<4096, FMT>(a, lines, s.data()); return;
        case 6144: emu_rc_ct<6144, FMT>(a, lines, s.data()); return;
        case 8192: emu_rc_ct<8192, FMT>(a, lines, s.data()); return;
        default: break;
    }
    for (int y = 0; y < lines; ++y) range_compress_body<FMT>(a, y, 0, 1, s.data(), nullptr);
}

int backend_range_compress(const RangeCompressArgs& a, int lines, LaunchShape sh, void*) {
    if (a.format == kRawAsarFbaq4)
        emu_rc<kRawAsarFbaq4>(a, lines, sh);
    else
        emu_rc<kRawErsBytes>(a, lines, sh);
    return ASARF_OK;
}

// The same instantiation choice as the device backend (strided_schedule_compiled).
template <int R0, int R1, int R2, int XT>
static void emu_az_strided(const AzStridedArgs& a, int tiles, int nblocks, LaunchShape sh) {
    TileBuf s(sh.smem);
    float2* tw = s.data() + static_cast<size_t>(a.n1) * a.xt;
    int* row = reinterpret_cast<int*>(tw + a.n1);
    for (int b = 0; b < nblocks; ++b) {
        az_strided_tables(a, b, 0, 1, tw, row);
        for (int t = 0; t < tiles; ++t) az_strided_body<R0, R1, R2, XT>(a, t, b, 0, 1, s.data(), tw, row, false);
    }
}

int backend_az_strided(const AzStridedArgs& a, const void*, int tiles, int nblocks, LaunchShape sh, void*) {
    if (a.compiled && strided_schedule_compiled(a.plan1, a.xt)) {
        if (plan_is(a.plan1, 9, 5, 5)) emu_az_strided<9, 5, 5, 32>(a, tiles, nblocks, sh);
        else emu_az_strided<9, 4, 5, 32>(a, tiles, nblocks, sh);
    } else {
        emu_az_strided<0, 0, 0, 0>(a, tiles, nblocks, sh);
    }
    return ASARF_OK;
}

template <int R0, int R1, int R2>
static void emu_az_rd(const AzRdArgs& a, int tiles, int nblocks, LaunchShape sh, unsigned int* err) {
    TileBuf buf(sh.smem + 128);
    float2* s = buf.data();
    ColParams* cps = reinterpret_cast<ColParams*>(s + static_cast<size_t>(a.n2) * a.wt);
    float* fbf = az_rd_freq_table(cps, a);
    for (int b = 0; b < nblocks; ++b)
        for (int t = 0; t < tiles; ++t) {
            az_rd_tables(a, t, b, 0, 1, cps, fbf);
            az_rd_body<true, R0, R1, R2>(a, t, b, 0, 1, s, cps, fbf, err, false);
        }
}

// The same instantiation choice as the device backend (block_schedule_compiled).
int backend_az_rd(const AzRdArgs& a, const void*, int tiles, int nblocks, LaunchShape sh, unsigned int* err, void*) {
    if (a.compiled && block_schedule_compiled(a.plan2)) {
        if (plan_is(a.plan2, 5, 5, 5)) emu_az_rd<5, 5, 5>(a, tiles, nblocks, sh, err);
        else emu_az_rd<8, 7, 3>(a, tiles, nblocks, sh, err);
    } else {
        emu_az_rd<0, 0, 0>(a, tiles, nblocks, sh, err);
    }
    return ASARF_OK;
}

int backend_tail(const TailArgs& a, int rows, LaunchShape sh, unsigned int* err, void*) {
    std::vector<float> s(sh.smem / sizeof(float) + 1);
    for (int y = 0; y < rows; ++y) tail_body(a, y, 0, 1, s.data(), err);
    return ASARF_OK;
}

int backend_ers_unpack(const ErsUnpackArgs& a, void*) {
    for (int y = 0; y < a.lines; ++y) ers_unpack_line(a, y, 0, 1);
    return ASARF_OK;
}

int backend_asar_unpack(const AsarUnpackArgs& a, void*) {
    for (int y = 0; y < a.lines; ++y) asar_unpack_line(a, y, 0, 1);
    return ASARF_OK;
}

int backend_decode(const DecodeArgs& a, long long n, void*) {
    for (long long i = 0; i < n; ++i) decode_item(a, i);
    return ASARF_OK;
}
int backend_product_stats(const ProductStatsArgs& a, void*) {
    std::vector<double> red(5 * 256), tree(5 * kStatsFoldLeaves);
    for (int b = 0; b < a.blocks; ++b) product_stats_body(a, b, 0, 1, red.data());
    product_stats_fold(a, 0, 1, tree.data());
    return ASARF_OK;
}

int backend_condition(const ConditionArgs& a, int rows, void*) {
    for (int y = 0; y < rows; ++y) condition_row(a, y, 0, 1);
    return ASARF_OK;
}

int backend_decode_fbaq(const DecodeFbaqArgs& a, long long n, void*) {
    for (long long i = 0; i < n; ++i) decode_fbaq_item(a, i);
    return ASARF_OK;
}

int backend_img_moments(const ImgMomentsArgs& a, int blocks, void*) {
    std::vector<double> red(12);
    for (int b = 0; b < blocks; ++b) img_moments_body(a, b, 0, 1, red.data());
    return ASARF_OK;
}
int backend_iq_apply(const IqApplyArgs& a, long long n, void*) {
    for (long long i = 0; i < n; ++i) iq_apply_item(a, i);
    return ASARF_OK;
}
int backend_zero_nans(float2* img, long long n, void*) {
    for (long long i = 0; i < n; ++i) {
        if (is_nan_f(img[i].x)) img[i].x = 0.0f;
        if (is_nan_f(img[i].y)) img[i].y = 0.0f;
    }
    return ASARF_OK;
}
int backend_accc(const AcccArgs& a, int blocks, void*) {
    for (int b = 0; b < blocks; ++b) accc_body(a, b, 0, 1);
    return ASARF_OK;
}
int backend_rc_rows(const RcRowsArgs& a, int rows, LaunchShape sh, void*) {
    std::vector<float2> s(sh.smem / sizeof(float2) + 1);
    for (int y = 0; y < rows; ++y) rc_rows_body(a, y, 0, 1, s.data());
    return ASARF_OK;
}
int backend_multilook(const MultilookArgs& a, void*) {
    for (int y = 0; y < a.out_y; ++y) multilook_row_body(a, y, 0, 1);
    return ASARF_OK;
}
int backend_rsl(const RslArgs& a, long long n, void*) {
    for (long long i = 0; i < n; ++i) rsl_item(a, i);
    return ASARF_OK;
}
int backend_srgr(const SrgrArgs& a, long long n, void*) {
    for (long long i = 0; i < n; ++i) srgr_item(a, i);
    return ASARF_OK;
}

void* mem_alloc(size_t bytes) { return std::calloc(1, bytes ? bytes : 1); }
void mem_free(void* p) { std::free(p); }
int mem_h2d(void* dst, const void* src, size_t n, void*) {
    std::memcpy(dst, src, n);
    return ASARF_OK;
}
int mem_d2h(void* dst, const void* src, size_t n, void*) {
    std::memcpy(dst, src, n);
    return ASARF_OK;
}
int mem_d2d(void* dst, const void* src, size_t n, void*) {
    std::memmove(dst, src, n);
    return ASARF_OK;
}
int mem_d2d_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows, void*) {
    for (size_t r = 0; r < rows; ++r)
        std::memcpy(static_cast<char*>(dst) + r * dpitch, static_cast<const char*>(src) + r * spitch, width);
    return ASARF_OK;
}
int mem_zero(void* dst, size_t n, void*) {
    std::memset(dst, 0, n);
    return ASARF_OK;
}
int stream_sync(void*) { return ASARF_OK; }
void* event_create() { return std::calloc(1, 8); }
void event_destroy(void* e) { std::free(e); }
int event_record(void*, void*) { return ASARF_OK; }
int event_elapsed(void*, void*, float* ms) {
    *ms = 0.0f;
    return ASARF_OK;
}
size_t smem_optin_limit() { return 227 * 1024; }
int backend_sm_count() { return 148; }  // the B200's, so plans take the device build's shapes

}  // namespace asarf

// Host-emulation counterpart of noalloc.cu: the same bodies over a static host array.
namespace {
struct EmuNoallocScratch {
    asarf::StatAccum acc;
    asarf::FocusState state;
};
EmuNoallocScratch g_emu_scratch;
}  // namespace

extern "C" int asarf_raw_statistics_noalloc(const uint8_t* d_raw, int32_t raw_line_bytes, int32_t samples_per_line,
                                            int32_t range_size, int32_t azimuth_size, const uint16_t* d_swst,
                                            int32_t min_swst, int64_t total_raw_samples, int32_t stats_stride,
                                            double prf, asarf_raw_stats* d_out, void*) {
    using namespace asarf;
    if (!d_raw || !d_out || range_size < 32 || azimuth_size < 2 || samples_per_line <= 0 ||
        samples_per_line > range_size || (stats_stride != 0 && stats_stride < range_size))
        return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: bad arguments");
    const int dc_step = range_size / 32;
    const int nblk = (range_size + dc_step - 1) / dc_step;
    if (nblk > kMaxDcBlocks) return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: too many Doppler blocks");
    std::memset(&g_emu_scratch.acc, 0, sizeof(StatAccum));
    RawStatsArgs st{};
    st.raw = d_raw;
    st.line_bytes = raw_line_bytes;
    st.spl = samples_per_line;
    st.na = azimuth_size;
    st.nr = range_size;
    st.swst = d_swst;
    st.min_swst = min_swst;
    st.dc_step = dc_step;
    st.nblk = nblk;
    st.lines_per_cta = kStatsLinesPerBlock;
    st.acc = &g_emu_scratch.acc;
    backend_raw_stats(st, raw_stats_grid_x(st, d_raw), (azimuth_size + st.lines_per_cta - 1) / st.lines_per_cta,
                      nullptr);
    FinalizeArgs fin{};
    fin.acc = &g_emu_scratch.acc;
    fin.state = &g_emu_scratch.state;
    fin.n_total = total_raw_samples > 0 ? total_raw_samples : static_cast<long long>(samples_per_line) * azimuth_size;
    const int stride = stats_stride > 0 ? stats_stride : range_size;
    fin.n_pad = static_cast<long long>(stride - range_size) * azimuth_size;
    fin.nr = range_size;
    fin.na = azimuth_size;
    fin.rg_stride = stride;
    fin.dc_step = dc_step;
    fin.nblk = nblk;
    fin.prf = prf;
    finalize_body(fin);
    const FocusState& s = g_emu_scratch.state;
    d_out->dc_i = s.dc_i_d;
    d_out->dc_q = s.dc_q_d;
    d_out->iq_gain = s.iq_gain;
    d_out->phase_error = s.phase_error;
    d_out->stddev_i = s.stddev_i;
    d_out->stddev_q = s.stddev_q;
    for (int k = 0; k < 3; ++k) d_out->doppler_centroid_poly[k] = s.dc_est[k];
    d_out->n_dc_blocks = s.nblk;
    for (int b = 0; b < kMaxDcBlocks; ++b) d_out->dc_block_hz[b] = b < s.nblk ? s.dc_blk_hz[b] : 0.0;
    d_out->applied_dc_i = s.dc_i;
    d_out->applied_dc_q = s.dc_q;
    d_out->applied_gain = s.gain;
    d_out->applied_sin = s.sin_c;
    d_out->applied_cos = s.cos_c;
    d_out->errors = s.errors;
    return ASARF_OK;
}

// Test hook of the host emulation only: drives the context-keyed address cache of the
// allocation-free entry point (context_cache.h) with made-up context ids and a resolver that
// hands out a fresh fake address on every call.  For each key i, addrs[i] receives the
// address returned and the function returns how many times the resolver ran.
extern "C" int asarf_emu_context_cache_probe(const unsigned long long* ids, int n, unsigned long long* addrs) {
    static asarf::ContextAddressCache<4> cache;
    static unsigned long long next_fake = 0x1000;
    int resolutions = 0;
    for (int i = 0; i < n; ++i) {
        void* p = nullptr;
        bool resolved = false;
        cache.get(ids[i], [](void** q) { *q = reinterpret_cast<void*>(next_fake); next_fake += 0x1000; return 0; },
                  &p, &resolved);
        resolutions += resolved ? 1 : 0;
        addrs[i] = reinterpret_cast<unsigned long long>(p);
    }
    return resolutions;
}

namespace asarf {
int backend_az_rd_split(const AzRdArgs&, const AzRdSplit&, const void*, int, int, LaunchShape, unsigned int*, void*) {
    return set_error(ASARF_ERR_INVALID, "split precision runs on the tensor cores only (no host emulation)");
}
int event_sync(void*) { return ASARF_OK; }
void* stream_create() { return std::calloc(1, 8); }
void stream_destroy(void* s) { std::free(s); }
int stream_wait_event(void*, void*) { return ASARF_OK; }
bool graphs_supported() { return false; }
int graph_capture_begin(void*) { return set_error(ASARF_ERR_INVALID, "no graphs in the host emulation"); }
int graph_capture_end(void*, void**) { return set_error(ASARF_ERR_INVALID, "no graphs in the host emulation"); }
int graph_launch(void*, void*) { return set_error(ASARF_ERR_INVALID, "no graphs in the host emulation"); }
void graph_destroy(void*) {}
const char* backend_name() { return "host-emulation"; }
int backend_make_tmap(void*, int, void*, const unsigned long long*, const unsigned long long*, const unsigned int*) {
    return set_error(ASARF_ERR_INVALID, "no tensor maps in host emulation");
}

}  // namespace asarf
