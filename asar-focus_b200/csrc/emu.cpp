// Host emulation backend: runs the kernel bodies of bodies.cuh single-threaded on the CPU
// (tid = 0, nthr = 1, one block after another).  Built only into the test library
// libasarf_emu.so so the CPU test suite can check the exact kernel code against the
// oracle; the product library links kernels.cu instead and has no CPU path.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "asarf.h"
#include "backend.h"
#include "bodies.cuh"

namespace asarf {

int backend_raw_stats(const RawStatsArgs& a, int gx, int gy, int threads, int cols, void*) {
    (void)threads;
    RawStatsSmem sm;
    for (int by = 0; by < gy; ++by)
        for (int bx = 0; bx < gx; ++bx) raw_stats_body(a, bx, by, 0, 1, cols, &sm);
    return ASARF_OK;
}

int backend_finalize(const FinalizeArgs& a, void*) {
    finalize_body(a);
    return ASARF_OK;
}

int backend_range_compress(const RangeCompressArgs& a, int lines, LaunchShape sh, void*) {
    std::vector<float2> s(sh.smem / sizeof(float2) + 1);
    for (int y = 0; y < lines; ++y) range_compress_body(a, y, 0, 1, s.data());
    return ASARF_OK;
}

int backend_az_strided(const AzStridedArgs& a, int tiles, int nblocks, LaunchShape sh, void*) {
    std::vector<float2> s(sh.smem / sizeof(float2) + 1);
    for (int b = 0; b < nblocks; ++b)
        for (int t = 0; t < tiles; ++t) az_strided_body(a, t, b, 0, 1, s.data());
    return ASARF_OK;
}

int backend_az_rd(const AzRdArgs& a, int tiles, int nblocks, LaunchShape sh, unsigned int* err, void*) {
    std::vector<float2> buf(sh.smem / sizeof(float2) + 16);
    float2* s = buf.data();
    float2* tmp = s + a.n2 * a.wt;
    ColParams* cps = reinterpret_cast<ColParams*>(tmp + a.chunk_rows * a.xt);
    for (int b = 0; b < nblocks; ++b)
        for (int t = 0; t < tiles; ++t) az_rd_body(a, t, b, 0, 1, s, tmp, cps, err);
    return ASARF_OK;
}

int backend_tail(const TailArgs& a, int rows, LaunchShape sh, unsigned int* err, void*) {
    std::vector<float> s(sh.smem / sizeof(float) + 1);
    for (int y = 0; y < rows; ++y) tail_body(a, y, 0, 1, s.data(), err);
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
const char* backend_name() { return "host-emulation"; }

}  // namespace asarf
