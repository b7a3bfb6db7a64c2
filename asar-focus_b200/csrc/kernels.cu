// CUDA kernels of the focusing path (sm_100a) and their launchers.
#include <cuda_runtime.h>

#include <cstdio>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"

namespace asarf {

namespace {

__global__ void __launch_bounds__(256) k_raw_stats(RawStatsArgs a, int cols) {
    __shared__ RawStatsSmem sm;
    raw_stats_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, cols, &sm);
}

__global__ void k_finalize(FinalizeArgs a) {
    if (blockIdx.x == 0 && threadIdx.x == 0) finalize_body(a);
}

__global__ void __launch_bounds__(512) k_range_compress(RangeCompressArgs a) {
    extern __shared__ float2 smem_rc[];
    range_compress_body(a, blockIdx.x, threadIdx.x, blockDim.x, smem_rc);
}

__global__ void __launch_bounds__(512) k_az_strided(AzStridedArgs a) {
    extern __shared__ float2 smem_as[];
    az_strided_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, smem_as);
}

__global__ void __launch_bounds__(512) k_az_rd(AzRdArgs a, unsigned int* err) {
    extern __shared__ float2 smem_rd[];
    const int wt = a.wt;
    float2* s = smem_rd;
    float2* tmp = s + a.n2 * wt;
    ColParams* cps = reinterpret_cast<ColParams*>(tmp + a.chunk_rows * a.xt);
    az_rd_body(a, blockIdx.x, blockIdx.y, threadIdx.x, blockDim.x, s, tmp, cps, err);
}

__global__ void __launch_bounds__(512) k_tail(TailArgs a, unsigned int* err) {
    extern __shared__ float smem_tail[];
    tail_body(a, blockIdx.x, threadIdx.x, blockDim.x, smem_tail, err);
}

int check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "%s launch: %s", what, cudaGetErrorString(e));
    return ASARF_OK;
}

template <class K>
int ensure_smem(K kernel, size_t bytes, const char* what) {
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
        if (e != cudaSuccess) return set_error(ASARF_ERR_CUDA, "%s smem %zu: %s", what, bytes, cudaGetErrorString(e));
    }
    return ASARF_OK;
}

cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

}  // namespace

int backend_raw_stats(const RawStatsArgs& a, int gx, int gy, int threads, int cols, void* stream) {
    k_raw_stats<<<dim3(gx, gy), threads, 0, S(stream)>>>(a, cols);
    return check_launch("raw_stats");
}

int backend_finalize(const FinalizeArgs& a, void* stream) {
    k_finalize<<<1, 32, 0, S(stream)>>>(a);
    return check_launch("finalize");
}

int backend_range_compress(const RangeCompressArgs& a, int lines, LaunchShape sh, void* stream) {
    int rc = ensure_smem(k_range_compress, sh.smem, "range_compress");
    if (rc) return rc;
    k_range_compress<<<lines, sh.threads, sh.smem, S(stream)>>>(a);
    return check_launch("range_compress");
}

int backend_az_strided(const AzStridedArgs& a, int tiles, int nblocks, LaunchShape sh, void* stream) {
    int rc = ensure_smem(k_az_strided, sh.smem, "az_strided");
    if (rc) return rc;
    k_az_strided<<<dim3(tiles, nblocks), sh.threads, sh.smem, S(stream)>>>(a);
    return check_launch("az_strided");
}

int backend_az_rd(const AzRdArgs& a, int tiles, int nblocks, LaunchShape sh, unsigned int* err, void* stream) {
    int rc = ensure_smem(k_az_rd, sh.smem, "az_rd");
    if (rc) return rc;
    k_az_rd<<<dim3(tiles, nblocks), sh.threads, sh.smem, S(stream)>>>(a, err);
    return check_launch("az_rd");
}

int backend_tail(const TailArgs& a, int rows, LaunchShape sh, unsigned int* err, void* stream) {
    int rc = ensure_smem(k_tail, sh.smem, "tail");
    if (rc) return rc;
    k_tail<<<rows, sh.threads, sh.smem, S(stream)>>>(a, err);
    return check_launch("tail");
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

size_t smem_optin_limit() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) {
        cudaGetLastError();
        return 227 * 1024;
    }
    return static_cast<size_t>(v);
}

const char* backend_name() { return "cuda-sm100a"; }

}  // namespace asarf
