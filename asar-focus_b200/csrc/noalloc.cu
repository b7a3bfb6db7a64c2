// Raw-data statistics without any device allocation.
//
// asarf_raw_statistics_noalloc computes what the planned path's first two kernels compute
// (IQ bias / gain / quadrature statistics and the Doppler-centroid estimate of a raw
// ERS byte-I/Q scene) for callers that cannot take device memory from cudaMalloc: a
// screening step that runs inside someone else's CUDA graph capture or under a host
// application whose allocator owns the whole device, or a real-time ingest loop that must
// not hit cudaMalloc's implicit synchronisation.  Such a caller passes its raw bytes and a
// small output struct it already owns; the only other memory used is the fixed scratch
// array below.
//
// The scratch lives in this library's own device memory for as long as the library is
// loaded, on every GPU that loads it.  All calls on a device share it, so calls whose
// kernels overlap on the GPU (two streams, two host threads) race and corrupt each
// other's sums; serialise them.  Each call clears the accumulators before use.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"
#include "context_cache.h"

namespace asarf {
namespace {

// Accumulators + finalisation state: 5.8 KB + ~1 KB, inside a fixed 8 KiB array.
struct NoallocScratch {
    StatAccum acc;
    FocusState state;
};
constexpr size_t kNoallocScratchBytes = 8192;
static_assert(sizeof(NoallocScratch) <= kNoallocScratchBytes, "scratch layout exceeds the static array");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

ContextAddressCache<64> g_scratch_cache;

// Unique id of the calling thread's current CUDA context (0 when none is current yet),
// through the driver entry points the runtime exposes.
int current_context_id(unsigned long long* id) {
    static std::once_flag once;
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id)
        return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: cuCtxGetCurrent / cuCtxGetId unavailable");
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS)
        return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: cuCtxGetCurrent failed");
    *id = 0;
    if (ctx && get_id(ctx, id) != CUDA_SUCCESS)
        return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: cuCtxGetId failed");
    return ASARF_OK;
}

int resolve_scratch(void** p) {
    *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(p, g_noalloc_scratch);
    if (e != cudaSuccess || !*p)
        return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    return ASARF_OK;
}

// Device address of the scratch array in the current CUDA context, resolved once per
// context (a new context after cudaDeviceReset, or a host application's own context, gets
// its own lookup).  In host code the array's name is only a stand-in symbol, never a usable
// pointer.  With no context current yet, the lookup itself makes the runtime bind the
// device's primary context, whose id then keys the entry.
int scratch_address(NoallocScratch** out) {
    unsigned long long id = 0;
    int rc = current_context_id(&id);
    if (rc) return rc;
    void* p = nullptr;
    if (id == 0) {
        rc = resolve_scratch(&p);
        if (rc) return rc;
        rc = current_context_id(&id);
        if (rc) return rc;
        if (id == 0) return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: no CUDA context after set-up");
        rc = g_scratch_cache.get(id, [p](void** q) { *q = p; return 0; }, &p);
    } else {
        rc = g_scratch_cache.get(id, resolve_scratch, &p);
    }
    if (rc) return rc;
    *out = static_cast<NoallocScratch*>(p);
    return ASARF_OK;
}

__global__ void __launch_bounds__(kStatsCols) k_noalloc_raw_stats(RawStatsArgs a) {
    __shared__ RawStatsSmem sm;
    raw_stats_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, &sm);
}

__global__ void k_noalloc_finalize(FinalizeArgs a, asarf_raw_stats* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    finalize_body(a);
    const FocusState& st = *a.state;
    out->dc_i = st.dc_i_d;
    out->dc_q = st.dc_q_d;
    out->iq_gain = st.iq_gain;
    out->phase_error = st.phase_error;
    out->stddev_i = st.stddev_i;
    out->stddev_q = st.stddev_q;
    for (int k = 0; k < 3; ++k) out->doppler_centroid_poly[k] = st.dc_est[k];
    out->n_dc_blocks = st.nblk;
    for (int b = 0; b < kMaxDcBlocks; ++b) out->dc_block_hz[b] = b < st.nblk ? st.dc_blk_hz[b] : 0.0;
    out->applied_dc_i = st.dc_i;
    out->applied_dc_q = st.dc_q;
    out->applied_gain = st.gain;
    out->applied_sin = st.sin_c;
    out->applied_cos = st.cos_c;
    out->errors = st.errors;
}

}  // namespace
}  // namespace asarf

using namespace asarf;

extern "C" int asarf_raw_statistics_noalloc(const uint8_t* d_raw, int32_t raw_line_bytes, int32_t samples_per_line,
                                            int32_t range_size, int32_t azimuth_size, const uint16_t* d_swst,
                                            int32_t min_swst, int64_t total_raw_samples, int32_t stats_stride,
                                            double prf, asarf_raw_stats* d_out, void* stream) {
    if (!d_raw || !d_out) return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: null raw or output pointer");
    if (reinterpret_cast<uintptr_t>(d_raw) & 1)
        return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: raw buffer must be 2-byte aligned");
    if (range_size < 32 || azimuth_size < 2 || samples_per_line <= 0 || samples_per_line > range_size)
        return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: sizes out of range (range %d, lines %d, samples %d)",
                         range_size, azimuth_size, samples_per_line);
    if (raw_line_bytes < 2 * samples_per_line || (raw_line_bytes & 1))
        return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: raw_line_bytes must be even and >= 2*samples_per_line");
    if (stats_stride != 0 && stats_stride < range_size)
        return set_error(ASARF_ERR_INVALID, "raw_statistics_noalloc: stats_stride %d below range_size %d", stats_stride,
                         range_size);
    const int dc_step = range_size / 32;
    const int nblk = (range_size + dc_step - 1) / dc_step;
    if (nblk > kMaxDcBlocks)
        return set_error(ASARF_ERR_INVALID,
                         "raw_statistics_noalloc: %d Doppler blocks exceed the static scratch (at most %d)", nblk,
                         kMaxDcBlocks);
    NoallocScratch* scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the accumulators keep the previous call's sums: clear them first
    cudaError_t e = cudaMemsetAsync(&scratch->acc, 0, sizeof(StatAccum), s);
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: clear: %s", cudaGetErrorString(e));

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
    st.lines_per_cta = kStatsMaxLines / 4;
    st.acc = &scratch->acc;
    dim3 grid(raw_stats_grid_x(st, d_raw), (azimuth_size + st.lines_per_cta - 1) / st.lines_per_cta);
    k_noalloc_raw_stats<<<grid, kStatsCols, 0, s>>>(st);

    FinalizeArgs fin{};
    fin.acc = &scratch->acc;
    fin.state = &scratch->state;
    fin.n_total = total_raw_samples > 0 ? total_raw_samples : static_cast<long long>(samples_per_line) * azimuth_size;
    const int stride = stats_stride > 0 ? stats_stride : range_size;
    fin.n_pad = static_cast<long long>(stride - range_size) * azimuth_size;
    fin.nr = range_size;
    fin.na = azimuth_size;
    fin.rg_stride = stride;
    fin.dc_step = dc_step;
    fin.nblk = nblk;
    fin.prf = prf;
    k_noalloc_finalize<<<1, 32, 0, s>>>(fin, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "raw_statistics_noalloc: launch: %s", cudaGetErrorString(e));
    return ASARF_OK;
}
