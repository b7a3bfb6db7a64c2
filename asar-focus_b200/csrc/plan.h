// The plan object behind asarf_plan, shared by the planner (host.cpp) and the strip driver
// (strip.cpp): scene, sizes, FFT schedules, device buffers and the launch argument blocks of
// the seven kernels of one focus run.
#pragma once

#include <vector>

#include "asarf.h"
#include "backend.h"
#include "internal.h"
#include "params.h"

using asarf::AzRdArgs;
using asarf::AzStridedArgs;
using asarf::FinalizeArgs;
using asarf::FocusState;
using asarf::HostFft;
using asarf::LaunchShape;
using asarf::RangeCompressArgs;
using asarf::RawStatsArgs;
using asarf::StatAccum;
using asarf::TailArgs;
using asarf::ProductStatsArgs;
using asarf::event_destroy;
using asarf::mem_alloc;
using asarf::mem_free;
using asarf::stream_destroy;

struct asarf_plan {
    asarf_scene scene{};
    std::vector<asarf_osv> osv;
    std::vector<float> fbaq_luts;  // the scene's FBAQ4 tables (I then Q), owned copy
    asarf_options opt{};
    asarf_dims dims{};
    int nr = 0, na = 0, nc = 0, nk = 0, nx = 0;
    int rg_pad_ref = 0, az_pad = 0, rc_len = 0, n1 = 0, n2 = 0;
    long long pitch = 0;
    int xt1 = 32, xt2 = 32, hl = 8, hr = 8;
    double vr_poly[3] = {0, 0, 0};
    // device memory
    std::vector<void*> allocs;
    size_t bytes = 0;
    float2* bufA = nullptr;
    float2* bufB = nullptr;
    StatAccum* acc = nullptr;
    FocusState* state = nullptr;
    uint8_t* raw_dev = nullptr;
    uint16_t* swst_dev = nullptr;
    float* out_dev = nullptr;
    HostFft rc, f1, f2, fN;
    float2* rc_mf = nullptr;
    // launch argument blocks
    RawStatsArgs a_stats{};
    FinalizeArgs a_fin{};
    RangeCompressArgs a_rc{};
    AzStridedArgs a_fwd{}, a_inv{};
    AzRdArgs a_rd{};
    TailArgs a_tail{};
    asarf::AzRdSplit a_split{};   // split-precision form of the range-Doppler block (opt.precision)
    bool split = false;
    LaunchShape sh_rd_split{};
    int stats_gy = 0;
    LaunchShape sh_rc{}, sh_st{}, sh_rd{}, sh_tail{};
    int tiles1 = 0, tiles2 = 0;
    int out_rows_max = 0, out_cols_max = 0;
    long long out_bytes = 0;      // bytes written at d_out for the product
    int ims_rows_max = 0;         // IMS records: most lines a results window keeps
    ProductStatsArgs a_pstats{};  // SQ ADS statistics (opt.sq_stats)
    // optional per-kernel timing (events recorded between the launches of each run)
    std::vector<void*> events;
    int timing_slots = 0, timing_used = 0;
    // TMA tensor maps (device build): strided views of A and B, contiguous view of A
    alignas(64) unsigned char tmapA3[128] = {};
    alignas(64) unsigned char tmapB3[128] = {};
    alignas(64) unsigned char tmapA2[128] = {};
    bool use_tma = false;
    bool skip_tail = false;       // strip blocks: the strip runs one tail over all blocks
    bool intensity_only = false;  // keep_slc = 0: |z|^2 rows instead of the complex SLC
    int raw_smem_offset = 0;
    // asynchronous host runs: the plan's own non-blocking stream (created on first use) and
    // the event recorded after the last enqueued image download
    void* own_stream = nullptr;
    void* done = nullptr;

    template <class T>
    T* alloc(size_t count) {
        void* p = mem_alloc(count * sizeof(T));
        if (p) {
            allocs.push_back(p);
            bytes += count * sizeof(T);
        }
        return static_cast<T*>(p);
    }
    ~asarf_plan() {
        if (done) event_destroy(done);
        if (own_stream) stream_destroy(own_stream);
        for (void* e : events) event_destroy(e);
        for (void* p : allocs) mem_free(p);
    }
};
