// CUDA kernels of the focusing path (sm_100a) and their launchers.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"
#include "tc.cuh"
#include "tma.cuh"

namespace asarf {

namespace {

// Three blocks per SM (80 registers, no spills).  Four blocks at 64 registers spilled 176
// bytes per thread in the batched loads and measured slower on the ERS-like scene:
// 0.156 against 0.143 ms.
__global__ void __launch_bounds__(kStatsCols, kStatsBlocksPerSm) k_raw_stats(RawStatsArgs a) {
    __shared__ RawStatsSmem sm;
    raw_stats_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, &sm);
}

__global__ void __launch_bounds__(32 * kFbaqStatsWarps, 3) k_raw_stats_fbaq(RawStatsArgs a) {
    __shared__ FbaqStatsSmem sm;
    raw_stats_fbaq_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, &sm);
}

__global__ void __launch_bounds__(1024) k_stats_fold(RawStatsArgs a, int tiles_y) {
    __shared__ double tree[6 * kFoldTree];
    stats_fold_body(a, tiles_y, threadIdx.x, blockDim.x, tree);
}

__global__ void __launch_bounds__(256) k_product_stats(ProductStatsArgs a) {
    __shared__ double red[5 * 256];
    product_stats_body(a, blockIdx.x, threadIdx.x, blockDim.x, red);
}

__global__ void __launch_bounds__(1024) k_product_stats_fold(ProductStatsArgs a) {
    __shared__ double tree[5 * kStatsFoldLeaves];
    product_stats_fold(a, threadIdx.x, blockDim.x, tree);
}

__global__ void __launch_bounds__(256) k_condition(ConditionArgs a) {
    condition_row(a, blockIdx.x, threadIdx.x, blockDim.x);
}

// One warp: the Doppler blocks' angles (an FP64 atan2 each) lane-parallel, the fit on lane 0.
__global__ void k_finalize(FinalizeArgs a) {
    __shared__ double xs[kMaxDcBlocks], ys[kMaxDcBlocks];
    if (blockIdx.x != 0) return;
    FocusState& st = *a.state;
    const FinalizeMap m = finalize_stats(a, threadIdx.x == 0 ? &st : nullptr);
    const int nblk = a.nblk < kMaxDcBlocks ? a.nblk : kMaxDcBlocks;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) finalize_block(a, m, b, xs, ys, st);
    __syncthreads();
    if (threadIdx.x == 0) finalize_fit(a, st, xs, ys, m.err);
}

// FBAQ4 record into shared memory: its 16-byte-aligned interior with vector loads, the
// unaligned head and tail bytewise, so nothing outside the record is read (records are not
// 16-byte multiples).  The copy starts at buf + (address mod 16), which keeps the interior
// aligned in shared memory as well; buf itself is 16-byte aligned.
__device__ __forceinline__ const uint8_t* stage_record(uint8_t* buf, const uint8_t* rec, int n) {
    const int lead = static_cast<int>(reinterpret_cast<uintptr_t>(rec) & 15);
    const int head = min(n, (16 - lead) & 15);
    const int nv = (n - head) >> 4;
    uint8_t* dst = buf + lead;
    for (int i = threadIdx.x; i < head; i += blockDim.x) dst[i] = rec[i];
    const uint4* src4 = reinterpret_cast<const uint4*>(rec + head);
    uint4* dst4 = reinterpret_cast<uint4*>(dst + head);
    for (int i = threadIdx.x; i < nv; i += blockDim.x) dst4[i] = __ldg(src4 + i);
    for (int i = head + 16 * nv + threadIdx.x; i < n; i += blockDim.x) dst[i] = rec[i];
    __syncthreads();
    return dst;
}

// One raw line per block; with bulk_bytes > 0 thread 0 fetches the line with one bulk copy
// into shared memory (the sub-16-byte tail with plain loads) while the others wait.
template <int FMT>
__global__ void __launch_bounds__(512) k_range_compress(RangeCompressArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_rc_raw[];
    float2* s = reinterpret_cast<float2*>(smem_rc_raw);
    __shared__ uint64_t bar;
    const uint8_t* line = nullptr;
    if constexpr (FMT == kRawAsarFbaq4) {
        line = stage_record(smem_rc_raw + a.raw_smem_offset, a.raw + static_cast<long long>(blockIdx.x) * a.line_bytes,
                            static_cast<int>(a.line_bytes));
    } else if (a.bulk_bytes > 0) {
        uint8_t* buf = smem_rc_raw + a.raw_smem_offset;
        const uint8_t* src = a.raw + static_cast<long long>(blockIdx.x) * a.line_bytes;
        const int total = 2 * a.spl;
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, static_cast<uint32_t>(a.bulk_bytes));
            bulk_load(buf, src, static_cast<uint32_t>(a.bulk_bytes), &bar);
        }
        for (int i = a.bulk_bytes + threadIdx.x; i < total; i += blockDim.x) buf[i] = src[i];
        __syncthreads();
        mbar_wait(&bar, 0, &const_cast<FocusState*>(a.state)->errors);
        line = buf;
    }
    range_compress_body<FMT>(a, blockIdx.x, threadIdx.x, blockDim.x, s, line);
}

// Compile-time-scheduled variant (L in kCtLengths).
template <int L, int FMT>
__global__ void __launch_bounds__(CtSchedule<L>::nthr, 2) k_range_compress_ct(RangeCompressArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_rcc_raw[];
    float2* s = reinterpret_cast<float2*>(smem_rcc_raw);
    __shared__ uint64_t bar;
    const uint8_t* line = nullptr;
    if constexpr (FMT == kRawAsarFbaq4) {
        line = stage_record(smem_rcc_raw + a.raw_smem_offset, a.raw + static_cast<long long>(blockIdx.x) * a.line_bytes,
                            static_cast<int>(a.line_bytes));
    } else if (a.bulk_bytes > 0) {
        uint8_t* buf = smem_rcc_raw + a.raw_smem_offset;
        const uint8_t* src = a.raw + static_cast<long long>(blockIdx.x) * a.line_bytes;
        const int total = 2 * a.spl;
        if (threadIdx.x == 0) {
            mbar_init(&bar, 1);
            mbar_expect_tx(&bar, static_cast<uint32_t>(a.bulk_bytes));
            bulk_load(buf, src, static_cast<uint32_t>(a.bulk_bytes), &bar);
        }
        for (int i = a.bulk_bytes + threadIdx.x; i < total; i += blockDim.x) buf[i] = src[i];
        __syncthreads();
        mbar_wait(&bar, 0, &const_cast<FocusState*>(a.state)->errors);
        line = buf;
    }
    range_compress_ct_body<L, FMT>(a, blockIdx.x, threadIdx.x, s, line);
}

// Strided azimuth pass: the [n1][xt] tile (rows r*n2 + b) arrives by 3-D TMA boxes.
// R0..XT > 0: compile-time transform schedule and tile width (az_strided_body).
template <int R0 = 0, int R1 = 0, int R2 = 0, int XT = 0>
__global__ void __launch_bounds__(512) k_az_strided(AzStridedArgs a, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(1024) unsigned char smem_as_raw[];
    float2* s = reinterpret_cast<float2*>(smem_as_raw);
    float2* tw = s + static_cast<size_t>(a.n1) * a.xt;
    int* row = reinterpret_cast<int*>(tw + a.n1);
    __shared__ uint64_t bar;
    if (a.use_tma && threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, static_cast<uint32_t>(sizeof(float2) * a.n1 * a.xt));
        for (int r0 = 0; r0 < a.n1; r0 += a.n1_box)
            tma_load_3d(s + static_cast<size_t>(r0) * a.xt, &map, &bar, 2 * blockIdx.x * a.xt, blockIdx.y, r0);
    }
    // twiddle and row tables are gathered while the tile is in flight
    az_strided_tables(a, blockIdx.y, threadIdx.x, blockDim.x, tw, row);
    __syncthreads();
    if (a.use_tma) mbar_wait(&bar, 0, a.state ? &const_cast<FocusState*>(a.state)->errors : nullptr);
    az_strided_body<R0, R1, R2, XT>(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, s, tw, row, a.use_tma != 0);
}

// Range-Doppler block: the [n2][wt] tile (contiguous rows, range halo) arrives by 2-D TMA
// boxes; columns left of 0 and right of nk are filled with zeros by the TMA unit.
// R0..R2 > 0: compile-time radix schedule of the n2 transforms (az_rd_body).
template <int R0 = 0, int R1 = 0, int R2 = 0>
__global__ void __launch_bounds__(512) k_az_rd(AzRdArgs a, unsigned int* err, const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(1024) unsigned char smem_rd_raw[];
    const int wt = a.wt;
    float2* s = reinterpret_cast<float2*>(smem_rd_raw);
    ColParams* cps = reinterpret_cast<ColParams*>(s + static_cast<size_t>(a.n2) * wt);
    float* fbf = az_rd_freq_table(cps, a);
    __shared__ uint64_t bar;
    if (a.use_tma && threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, static_cast<uint32_t>(sizeof(float2) * a.n2 * wt));
        const int x = 2 * (static_cast<int>(blockIdx.x) * a.xt - a.hl);
        for (int r0 = 0; r0 < a.n2; r0 += a.n2_box)
            tma_load_2d(s + static_cast<size_t>(r0) * wt, &map, &bar, x, blockIdx.y * a.n2 + r0);
    }
    // column constants and row frequencies are computed while the tile is in flight
    az_rd_tables(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, cps, fbf);
    __syncthreads();
    if (a.use_tma) mbar_wait(&bar, 0, err);
    az_rd_body<true, R0, R1, R2>(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, s, cps, fbf, err,
                                 a.use_tma != 0);
}

// ----------------------------------------------------------------------------- split precision
// Forward transform of the range-Doppler tile on the tensor cores.  Tile s[l][c], l < n2 =
// R * m, c < wt.  Operand row rho = r * wt + c holds the sub-sequence x[r + R mm] (mm < m) of
// column c as bf16 hi + lo parts (K = (mm, re / im)); it multiplies the m-point DFT matrix B
// (hi + lo, output slot s = frequency k1(s)) as Ahi Bhi + Ahi Blo + Alo Bhi with FP32
// accumulation, and the result times W_n2^(r k1(s)) goes back to row r + R s of column c (a
// row of the same sub-sequence, already consumed).  The operands live in tensor memory
// beside the accumulator (TMEM columns [0, 64) accumulator, [64, 96) A hi, [96, 128) A lo),
// so shared memory holds only B and the tile and two blocks stay resident per SM, as in the
// FP32 kernel.  Rounds of 128 operand rows: warp w writes TMEM lanes 32 (w % 4) .., K chunk
// w / 4 (8 inputs), one thread issues the products, every thread reads back its lane.  A
// radix-R FP32 pass over rows R s .. R s + R - 1 then leaves frequency k1(s) + m k2 at row
// R s + k2: the digit-reversed order of the FP32 forward transform (k1(s) from that
// transform's order table).  Returns false (error bit set, products drained) if a product did
// not complete in time.
constexpr uint32_t kSplitColAcc = 0, kSplitColAHi = 64, kSplitColALo = 96;

__device__ bool split_forward(const AzRdArgs& a, const AzRdSplit& sp, float2* s, const unsigned char* b_hi,
                              const unsigned char* b_lo, uint32_t tmem, uint64_t* mbar, unsigned int* err) {
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int wt = a.wt, R = sp.radix, m = sp.m;
    const int rows = R * wt;
    const int q = warp & 3, jb = warp >> 2;  // TMEM lane quarter, K chunk / accumulator column block
    const uint32_t lane_base = static_cast<uint32_t>(32 * q) << 16;
    const FastDiv dwt = make_fastdiv(static_cast<unsigned int>(wt));
    constexpr uint32_t kIdesc = umma_idesc_bf16(kSplitRows, kSplitN);
    constexpr uint32_t kSbo = kSplitK * 16;  // 8 rows x K bf16
    (void)nthr;
    uint32_t phase = 0;
    for (int g0 = 0; g0 < rows; g0 += kSplitRows) {
        const int rho = g0 + 32 * q + lane;
        const bool live = rho < rows;
        int r = 0, c = 0;
        if (live) {
            r = static_cast<int>(fdiv_u(static_cast<unsigned int>(rho), dwt));
            c = rho - r * wt;
        }
        {
            uint32_t hi[8], lo[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int mm = 8 * jb + i;
                const float2 v = (live && mm < m) ? s[(r + R * mm) * wt + c] : make_float2(0.0f, 0.0f);
                split_bf16x2(v.x, v.y, hi[i], lo[i]);
            }
            tmem_st8(tmem + lane_base + kSplitColAHi + 8u * jb, hi);
            tmem_st8(tmem + lane_base + kSplitColALo + 8u * jb, lo);
            tmem_wait_st();
        }
        tc_fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after_sync();
            const uint32_t bh = smem_u32(b_hi), bl = smem_u32(b_lo);
#pragma unroll
            for (int ks = 0; ks < kSplitK / 16; ++ks) {
                const uint32_t o = 256u * ks;  // B: two 128-byte core-matrix columns per k-step
                const uint64_t dbh = umma_smem_desc(bh + o, 128, kSbo), dbl = umma_smem_desc(bl + o, 128, kSbo);
                const uint32_t ah = tmem + kSplitColAHi + 8u * ks, al = tmem + kSplitColALo + 8u * ks;
                umma_bf16_ts(tmem + kSplitColAcc, ah, dbh, kIdesc, ks > 0);
                umma_bf16_ts(tmem + kSplitColAcc, ah, dbl, kIdesc, true);
                umma_bf16_ts(tmem + kSplitColAcc, al, dbh, kIdesc, true);
            }
            umma_commit(mbar);
        }
        const bool done = mbar_wait(mbar, phase, nullptr);
        if (__syncthreads_or(!done)) {
            if (tid == 0) atomicOr(err, kErrMmaTimeout);
            mbar_wait(mbar, phase, nullptr);  // one more bounded wait for the products in flight
            return false;
        }
        phase ^= 1u;
        tc_fence_after_sync();
        // accumulator: this warp's lanes, columns 16 jb .. (output slots 8 jb ..)
        if (8 * jb < m) {  // warp-uniform
            float v[16];
            tmem_ld16(tmem + lane_base + kSplitColAcc + 16u * jb, v);
            if (live) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int slot = 8 * jb + i;
                    if (slot < m)
                        s[(r + R * slot) * wt + c] = cmul(make_float2(v[2 * i], v[2 * i + 1]), __ldg(sp.tw + r * m + slot));
                }
            }
        }
        tc_fence_before_sync();
        __syncthreads();
    }
    // radix-R DFT over r of every (slot, column pair): rows R * slot + r, no twiddles
    const int npair = wt >> 1;
    fft_stage_pair_dispatch<false, false>(R, s, a.n2, 1, make_fastdiv(1u), npair,
                                          make_fastdiv(static_cast<unsigned int>(npair)), wt, a.plan2.tw, tid,
                                          blockDim.x);
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(512, 2) k_az_rd_split(AzRdArgs a, AzRdSplit sp, unsigned int* err,
                                                        const __grid_constant__ CUtensorMap map) {
    extern __shared__ __align__(1024) unsigned char smem_rds_raw[];
    unsigned char* b_hi = smem_rds_raw;
    unsigned char* b_lo = b_hi + kSplitMatrixBytes;
    float2* s = reinterpret_cast<float2*>(b_lo + kSplitMatrixBytes);
    const int wt = a.wt;
    ColParams* cps = reinterpret_cast<ColParams*>(s + static_cast<size_t>(a.n2) * wt);
    float* fbf = az_rd_freq_table(cps, a);
    __shared__ uint64_t bar, mbar;
    __shared__ uint32_t tmem_base;
    if (threadIdx.x < 32) tmem_alloc(&tmem_base, kSplitTmemCols);
    if (threadIdx.x == 0) {
        mbar_init(&mbar, 1);
        mbar_init(&bar, 1);
        mbar_expect_tx(&bar, static_cast<uint32_t>(sizeof(float2) * a.n2 * wt));
        const int x = 2 * (static_cast<int>(blockIdx.x) * a.xt - a.hl);
        for (int r0 = 0; r0 < a.n2; r0 += a.n2_box)
            tma_load_2d(s + static_cast<size_t>(r0) * wt, &map, &bar, x, blockIdx.y * a.n2 + r0);
    }
    // the DFT matrix images and the column / row tables while the tile is in flight
    const uint4* bsrc = reinterpret_cast<const uint4*>(sp.bmat);
    for (int i = threadIdx.x; i < 2 * kSplitMatrixBytes / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(b_hi)[i] = __ldg(bsrc + i);
    az_rd_tables(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, cps, fbf);
    fence_async_smem();  // B is read by the tensor cores
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    const uint32_t tmem = tmem_base;
    mbar_wait(&bar, 0, err);
    if (split_forward(a, sp, s, b_hi, b_lo, tmem, &mbar, err))
        az_rd_body<false>(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, s, cps, fbf, err, true);
    tc_fence_before_sync();
    __syncthreads();
    tc_fence_after_sync();
    if (threadIdx.x < 32) tmem_dealloc(tmem, kSplitTmemCols);
}

__global__ void __launch_bounds__(512, 2) k_tail(TailArgs a, unsigned int* err) {
    extern __shared__ float smem_tail[];
    tail_body(a, blockIdx.x, threadIdx.x, blockDim.x, smem_tail, err);
}

template <class Args, void (*Item)(const Args&, long long)>
__global__ void __launch_bounds__(256) k_items(Args a, long long n) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        Item(a, i);
}

ASARF_HD ASARF_INLINE void zero_nan_item(float2* const& img, long long i) {
    float2 v = img[i];
    if (is_nan_f(v.x)) v.x = 0.0f;
    if (is_nan_f(v.y)) v.y = 0.0f;
    img[i] = v;
}

__global__ void __launch_bounds__(256) k_img_moments(ImgMomentsArgs a) {
    __shared__ double red[12 * 256];
    img_moments_body(a, blockIdx.x, threadIdx.x, blockDim.x, red);
}

__global__ void __launch_bounds__(256) k_accc(AcccArgs a) { accc_body(a, blockIdx.x, threadIdx.x, blockDim.x); }

__global__ void __launch_bounds__(512) k_rc_rows(RcRowsArgs a) {
    extern __shared__ float2 smem_rcr[];
    rc_rows_body(a, blockIdx.x, threadIdx.x, blockDim.x, smem_rcr);
}

__global__ void __launch_bounds__(256) k_ers_unpack(ErsUnpackArgs a) {
    ers_unpack_line(a, blockIdx.x, threadIdx.x, blockDim.x);
}

__global__ void __launch_bounds__(256) k_asar_unpack(AsarUnpackArgs a) {
    asar_unpack_line(a, blockIdx.x, threadIdx.x, blockDim.x);
}

__global__ void __launch_bounds__(256) k_multilook(MultilookArgs a) {
    multilook_row_body(a, blockIdx.x, threadIdx.x, blockDim.x);
}

int grid_for(long long n) {
    long long g = (n + 255) / 256;
    return static_cast<int>(g < 148 * 32 ? (g > 0 ? g : 1) : 148 * 32);
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
    return ASARF_OK;
}

// Raise a kernel's dynamic shared-memory limit to `bytes` (once per kernel, device and size:
// the default limit of 48 KiB counts the kernel's static shared memory too, so any dynamic
// size is checked, not only those above 48 KiB).
template <class K>
int ensure_smem(K kernel, size_t bytes, const char* what) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return ASARF_OK;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "%s smem %zu: %s", what, bytes, cudaGetErrorString(e));
    done[key] = bytes;
    return ASARF_OK;
}

cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

int backend_raw_stats(const RawStatsArgs& a, int gx, int gy, void* stream) {
    k_raw_stats<<<dim3(gx, gy), kStatsCols, 0, S(stream)>>>(a);
    return check_launch("raw_stats");
}

int backend_finalize(const FinalizeArgs& a, void* stream) {
    k_finalize<<<1, 32, 0, S(stream)>>>(a);
    return check_launch("finalize");
}

int backend_raw_stats_fbaq(const RawStatsArgs& a, int gx, int gy, void* stream) {
    k_raw_stats_fbaq<<<dim3(gx, gy), 32 * kFbaqStatsWarps, 0, S(stream)>>>(a);
    return check_launch("raw_stats_fbaq");
}

int backend_stats_fold(const RawStatsArgs& a, int tiles_y, void* stream) {
    k_stats_fold<<<1, 1024, 0, S(stream)>>>(a, tiles_y);
    return check_launch("stats_fold");
}

template <int L, int FMT>
static int launch_rc_ct(const RangeCompressArgs& a, int lines, size_t smem, void* stream) {
    int rc = ensure_smem(k_range_compress_ct<L, FMT>, smem, "range_compress");
    if (rc) return rc;
    k_range_compress_ct<L, FMT><<<lines, CtSchedule<L>::nthr, smem, S(stream)>>>(a);
    return check_launch("range_compress");
}

template <int FMT>
static int launch_rc(const RangeCompressArgs& a, int lines, LaunchShape sh, void* stream) {
    switch (a.plan.n) {
        case 768: return launch_rc_ct<768, FMT>(a, lines, sh.smem, stream);
        case 1024: return launch_rc_ct<1024, FMT>(a, lines, sh.smem, stream);
        case 1536: return launch_rc_ct<1536, FMT>(a, lines, sh.smem, stream);
        case 2048: return launch_rc_ct<2048, FMT>(a, lines, sh.smem, stream);
        case 3072: return launch_rc_ct<3072, FMT>(a, lines, sh.smem, stream);
        case 4096: return launch_rc_ct<4096, FMT>(a, lines, sh.smem, stream);
        case 6144: return launch_rc_ct<6144, FMT>(a, lines, sh.smem, stream);
        case 8192: return launch_rc_ct<8192, FMT>(a, lines, sh.smem, stream);
        default: break;
    }
    int rc = ensure_smem(k_range_compress<FMT>, sh.smem, "range_compress");
    if (rc) return rc;
    k_range_compress<FMT><<<lines, sh.threads, sh.smem, S(stream)>>>(a);
    return check_launch("range_compress");
}

int backend_range_compress(const RangeCompressArgs& a, int lines, LaunchShape sh, void* stream) {
    if (a.format == kRawAsarFbaq4) return launch_rc<kRawAsarFbaq4>(a, lines, sh, stream);
    return launch_rc<kRawErsBytes>(a, lines, sh, stream);
}

static CUtensorMap tmap_or_zero(const void* tmap) {
    CUtensorMap m;
    if (tmap)
        std::memcpy(&m, tmap, sizeof(m));
    else
        std::memset(&m, 0, sizeof(m));
    return m;
}

template <int R0, int R1, int R2, int XT>
static int launch_az_strided(const AzStridedArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh,
                             void* stream) {
    int rc = ensure_smem(k_az_strided<R0, R1, R2, XT>, sh.smem, "az_strided");
    if (rc) return rc;
    k_az_strided<R0, R1, R2, XT><<<dim3(tiles, nblocks), sh.threads, sh.smem, S(stream)>>>(a, tmap_or_zero(tmap));
    return check_launch("az_strided");
}

// The compiled schedules (strided_schedule_compiled) when the plan allows them.
int backend_az_strided(const AzStridedArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh, void* stream) {
    if (a.compiled && strided_schedule_compiled(a.plan1, a.xt)) {
        if (plan_is(a.plan1, 9, 5, 5)) return launch_az_strided<9, 5, 5, 32>(a, tmap, tiles, nblocks, sh, stream);
        return launch_az_strided<9, 4, 5, 32>(a, tmap, tiles, nblocks, sh, stream);
    }
    return launch_az_strided<0, 0, 0, 0>(a, tmap, tiles, nblocks, sh, stream);
}

template <int R0, int R1, int R2>
static int launch_az_rd(const AzRdArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh,
                        unsigned int* err, void* stream) {
    int rc = ensure_smem(k_az_rd<R0, R1, R2>, sh.smem, "az_rd");
    if (rc) return rc;
    k_az_rd<R0, R1, R2><<<dim3(tiles, nblocks), sh.threads, sh.smem, S(stream)>>>(a, err, tmap_or_zero(tmap));
    return check_launch("az_rd");
}

// The compiled schedules (block_schedule_compiled) when the plan allows them.
int backend_az_rd(const AzRdArgs& a, const void* tmap, int tiles, int nblocks, LaunchShape sh, unsigned int* err,
                  void* stream) {
    if (a.compiled && block_schedule_compiled(a.plan2)) {
        if (plan_is(a.plan2, 5, 5, 5)) return launch_az_rd<5, 5, 5>(a, tmap, tiles, nblocks, sh, err, stream);
        return launch_az_rd<8, 7, 3>(a, tmap, tiles, nblocks, sh, err, stream);
    }
    return launch_az_rd<0, 0, 0>(a, tmap, tiles, nblocks, sh, err, stream);
}

int backend_az_rd_split(const AzRdArgs& a, const AzRdSplit& sp, const void* tmap, int tiles, int nblocks,
                        LaunchShape sh, unsigned int* err, void* stream) {
    if (!tmap) return set_error(ASARF_ERR_INVALID, "az_rd_split: needs the TMA tile loads");
    int rc = ensure_smem(k_az_rd_split, sh.smem, "az_rd_split");
    if (rc) return rc;
    k_az_rd_split<<<dim3(tiles, nblocks), sh.threads, sh.smem, S(stream)>>>(a, sp, err, tmap_or_zero(tmap));
    return check_launch("az_rd_split");
}

int backend_make_tmap(void* out, int rank, void* base, const unsigned long long* dims,
                      const unsigned long long* strides, const unsigned int* box) {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn) {
            cudaGetLastError();
            return set_error(ASARF_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    cuuint64_t gdim[5], gstr[4];
    cuuint32_t bdim[5], estr[5];
    for (int i = 0; i < rank; ++i) {
        gdim[i] = dims[i];
        bdim[i] = box[i];
        estr[i] = 1;
    }
    for (int i = 0; i + 1 < rank; ++i) gstr[i] = strides[i];
    CUresult r = encode(static_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, base, gdim, gstr, bdim,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(ASARF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", static_cast<int>(r));
    return ASARF_OK;
}

int backend_tail(const TailArgs& a, int rows, LaunchShape sh, unsigned int* err, void* stream) {
    int rc = ensure_smem(k_tail, sh.smem, "tail");
    if (rc) return rc;
    k_tail<<<rows, sh.threads, sh.smem, S(stream)>>>(a, err);
    return check_launch("tail");
}

int backend_decode(const DecodeArgs& a, long long n, void* stream) {
    k_items<DecodeArgs, decode_item><<<grid_for(n), 256, 0, S(stream)>>>(a, n);
    return check_launch("decode");
}
int backend_product_stats(const ProductStatsArgs& a, void* stream) {
    k_product_stats<<<a.blocks, 256, 0, S(stream)>>>(a);
    int rc = check_launch("product_stats");
    if (rc) return rc;
    k_product_stats_fold<<<1, 1024, 0, S(stream)>>>(a);
    return check_launch("product_stats_fold");
}
int backend_condition(const ConditionArgs& a, int rows, void* stream) {
    if (rows <= 0) return ASARF_OK;
    k_condition<<<rows, 256, 0, S(stream)>>>(a);
    return check_launch("condition");
}
int backend_decode_fbaq(const DecodeFbaqArgs& a, long long n, void* stream) {
    k_items<DecodeFbaqArgs, decode_fbaq_item><<<grid_for(n), 256, 0, S(stream)>>>(a, n);
    return check_launch("decode_fbaq");
}
int backend_img_moments(const ImgMomentsArgs& a, int blocks, void* stream) {
    k_img_moments<<<blocks, 256, 0, S(stream)>>>(a);
    return check_launch("img_moments");
}
int backend_iq_apply(const IqApplyArgs& a, long long n, void* stream) {
    k_items<IqApplyArgs, iq_apply_item><<<grid_for(n), 256, 0, S(stream)>>>(a, n);
    return check_launch("iq_apply");
}
int backend_zero_nans(float2* img, long long n, void* stream) {
    k_items<float2*, zero_nan_item><<<grid_for(n), 256, 0, S(stream)>>>(img, n);
    return check_launch("zero_nans");
}
int backend_accc(const AcccArgs& a, int blocks, void* stream) {
    k_accc<<<blocks, 256, 0, S(stream)>>>(a);
    return check_launch("accc");
}
int backend_rc_rows(const RcRowsArgs& a, int rows, LaunchShape sh, void* stream) {
    int rc = ensure_smem(k_rc_rows, sh.smem, "rc_rows");
    if (rc) return rc;
    k_rc_rows<<<rows, sh.threads, sh.smem, S(stream)>>>(a);
    return check_launch("rc_rows");
}
int backend_ers_unpack(const ErsUnpackArgs& a, void* stream) {
    if (a.lines <= 0) return ASARF_OK;
    k_ers_unpack<<<a.lines, 256, 0, S(stream)>>>(a);
    return check_launch("ers_unpack");
}

int backend_asar_unpack(const AsarUnpackArgs& a, void* stream) {
    if (a.lines <= 0) return ASARF_OK;
    k_asar_unpack<<<a.lines, 256, 0, S(stream)>>>(a);
    return check_launch("asar_unpack");
}
int backend_multilook(const MultilookArgs& a, void* stream) {
    k_multilook<<<a.out_y, 256, 0, S(stream)>>>(a);
    return check_launch("multilook");
}
int backend_rsl(const RslArgs& a, long long n, void* stream) {
    k_items<RslArgs, rsl_item><<<grid_for(n), 256, 0, S(stream)>>>(a, n);
    return check_launch("rsl");
}
int backend_srgr(const SrgrArgs& a, long long n, void* stream) {
    k_items<SrgrArgs, srgr_item><<<grid_for(n), 256, 0, S(stream)>>>(a, n);
    return check_launch("srgr");
}

void* mem_alloc(size_t bytes) {
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return p;
}

void mem_free(void* p) {
    if (p) cudaFree(p);
}

static int cuda_rc(cudaError_t e, const char* what) {
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    return ASARF_OK;
}

int mem_h2d(void* dst, const void* src, size_t n, void* stream) {
    return cuda_rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, S(stream)), "H2D copy");
}
int mem_d2h(void* dst, const void* src, size_t n, void* stream) {
    return cuda_rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, S(stream)), "D2H copy");
}
int mem_d2d(void* dst, const void* src, size_t n, void* stream) {
    return cuda_rc(cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToDevice, S(stream)), "D2D copy");
}
int mem_d2d_2d(void* dst, size_t dpitch, const void* src, size_t spitch, size_t width, size_t rows, void* stream) {
    return cuda_rc(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, rows, cudaMemcpyDeviceToDevice, S(stream)),
                   "2D D2D copy");
}
int mem_zero(void* dst, size_t n, void* stream) {
    return cuda_rc(cudaMemsetAsync(dst, 0, n, S(stream)), "memset");
}
int stream_sync(void* stream) { return cuda_rc(cudaStreamSynchronize(S(stream)), "stream sync"); }

void* event_create() {
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return e;
}
void event_destroy(void* e) {
    if (e) cudaEventDestroy(static_cast<cudaEvent_t>(e));
}
int event_record(void* e, void* stream) {
    return cuda_rc(cudaEventRecord(static_cast<cudaEvent_t>(e), S(stream)), "event record");
}
int event_elapsed(void* a, void* b, float* ms) {
    cudaError_t e = cudaEventSynchronize(static_cast<cudaEvent_t>(b));
    if (e == cudaSuccess) e = cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(a), static_cast<cudaEvent_t>(b));
    return cuda_rc(e, "event elapsed");
}

int event_sync(void* e) { return cuda_rc(cudaEventSynchronize(static_cast<cudaEvent_t>(e)), "event sync"); }

void* stream_create() {
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return s;
}
void stream_destroy(void* s) {
    if (s) cudaStreamDestroy(static_cast<cudaStream_t>(s));
}
int stream_wait_event(void* stream, void* event) {
    return cuda_rc(cudaStreamWaitEvent(S(stream), static_cast<cudaEvent_t>(event), 0), "stream wait");
}
bool graphs_supported() { return true; }
int graph_capture_begin(void* stream) {
    return cuda_rc(cudaStreamBeginCapture(S(stream), cudaStreamCaptureModeRelaxed), "begin capture");
}
int graph_capture_end(void* stream, void** exec) {
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(S(stream), &g);
    if (e != cudaSuccess) return cuda_rc(e, "end capture");
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_rc(e, "graph instantiate");
    *exec = x;
    return ASARF_OK;
}
int graph_launch(void* exec, void* stream) {
    return cuda_rc(cudaGraphLaunch(static_cast<cudaGraphExec_t>(exec), S(stream)), "graph launch");
}
void graph_destroy(void* exec) {
    if (exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec));
}

size_t smem_optin_limit() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 227 * 1024;
    }
    return static_cast<size_t>(v);
}

int backend_sm_count() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
        cudaGetLastError();
        return 148;
    }
    return v;
}

const char* backend_name() { return "cuda-sm100a"; }

}  // namespace asarf
