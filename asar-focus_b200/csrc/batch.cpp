// Batched focusing of independent segments of uneven size.
//
// Each segment keeps its own plan (its own FFT schedules, tile shapes and buffers), and the
// whole batch - every segment's kernels - is captured once into a CUDA graph whose
// branches run concurrently: segments are dealt to `branches` side streams largest first
// (LPT on Nr * Na), and the side streams fork from and join back into the batch's own
// capture stream.  The graph is launched onto the caller's stream, and later calls with the
// same buffers replay it with that single launch.  The graph bakes in the buffer addresses,
// so a call with different buffers captures a new one.
#include <algorithm>
#include <numeric>
#include <vector>

#include "asarf.h"
#include "backend.h"

using namespace asarf;

struct asarf_batch {
    std::vector<asarf_plan*> plans;
    std::vector<long long> work;          // Nr * Na per segment
    std::vector<int> branch_of;           // side stream of each segment
    int branches = 1;
    std::vector<void*> streams;           // side streams
    void* cap_stream = nullptr;           // origin stream of the capture (never the legacy stream)
    void* ev_fork = nullptr;
    std::vector<void*> ev_join;
    void* graph = nullptr;
    std::vector<const void*> key;         // buffers baked into the graph

    ~asarf_batch() {
        graph_destroy(graph);
        for (void* s : streams) stream_destroy(s);
        stream_destroy(cap_stream);
        if (ev_fork) event_destroy(ev_fork);
        for (void* e : ev_join) event_destroy(e);
        for (asarf_plan* p : plans) asarf_plan_destroy(p);
    }
};

namespace {

// Longest-processing-time assignment of segments to branches; returns the branch of each.
std::vector<int> lpt_assign(const std::vector<long long>& work, int branches) {
    std::vector<int> order(work.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
    std::vector<long long> load(static_cast<size_t>(branches), 0);
    std::vector<int> out(work.size(), 0);
    for (int i : order) {
        const int k = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
        out[static_cast<size_t>(i)] = k;
        load[static_cast<size_t>(k)] += work[static_cast<size_t>(i)];
    }
    return out;
}

}  // namespace

extern "C" {

int asarf_lpt_assign(const int64_t* work, int32_t n, int32_t bins, int32_t* out_bin) {
    if (!work || !out_bin || n < 0 || bins < 1) return set_error(ASARF_ERR_INVALID, "lpt_assign: bad arguments");
    std::vector<long long> w(work, work + n);
    const std::vector<int> b = lpt_assign(w, bins);
    for (int i = 0; i < n; ++i) out_bin[i] = b[static_cast<size_t>(i)];
    return ASARF_OK;
}

int asarf_batch_create(const asarf_scene* scenes, int32_t n, const asarf_options* opts, int32_t branches,
                       asarf_batch** out) {
    if (!scenes || !out || n < 1) return set_error(ASARF_ERR_INVALID, "batch_create: need at least one scene");
    *out = nullptr;
    auto* b = new asarf_batch();
    b->branches = std::max(1, std::min<int>(branches > 0 ? branches : 4, n));
    for (int i = 0; i < n; ++i) {
        asarf_plan* p = nullptr;
        const int rc = asarf_plan_create(&scenes[i], opts ? &opts[i] : nullptr, &p);
        if (rc) {
            delete b;
            return rc;
        }
        b->plans.push_back(p);
        b->work.push_back(static_cast<long long>(scenes[i].range_size) * scenes[i].azimuth_size);
    }
    b->branch_of = lpt_assign(b->work, b->branches);
    for (int k = 0; k < b->branches; ++k) {
        void* s = stream_create();
        void* e = event_create();
        if (!s || !e) {
            stream_destroy(s);
            if (e) event_destroy(e);
            delete b;
            return set_error(ASARF_ERR_CUDA, "batch_create: stream or event creation failed");
        }
        b->streams.push_back(s);
        b->ev_join.push_back(e);
    }
    b->ev_fork = event_create();
    b->cap_stream = stream_create();
    if (!b->ev_fork || !b->cap_stream) {
        delete b;
        return set_error(ASARF_ERR_CUDA, "batch_create: event creation failed");
    }
    *out = b;
    return ASARF_OK;
}

void asarf_batch_destroy(asarf_batch* b) { delete b; }

int asarf_batch_plan(asarf_batch* b, int32_t i, asarf_plan** out) {
    if (!b || !out || i < 0 || i >= static_cast<int>(b->plans.size()))
        return set_error(ASARF_ERR_INVALID, "batch_plan: index out of range");
    *out = b->plans[static_cast<size_t>(i)];
    return ASARF_OK;
}

int asarf_batch_branch(const asarf_batch* b, int32_t i) {
    if (!b || i < 0 || i >= static_cast<int>(b->plans.size())) return -1;
    return b->branch_of[static_cast<size_t>(i)];
}

int asarf_batch_focus(asarf_batch* b, const uint8_t* const* d_raw, const uint16_t* const* d_swst,
                      const int32_t* min_swst, float* const* d_out, void* stream) {
    if (!b || !d_raw || !d_out) return set_error(ASARF_ERR_INVALID, "batch_focus: null argument");
    const int n = static_cast<int>(b->plans.size());
    auto focus_all = [&](bool branched) -> int {
        for (int i = 0; i < n; ++i) {
            void* s = branched ? b->streams[static_cast<size_t>(b->branch_of[static_cast<size_t>(i)])] : stream;
            const int rc = asarf_focus(b->plans[static_cast<size_t>(i)], d_raw[i], d_swst ? d_swst[i] : nullptr,
                                       min_swst ? min_swst[i] : 0, d_out[i], s);
            if (rc) return rc;
        }
        return ASARF_OK;
    };
    if (!graphs_supported()) return focus_all(false);

    std::vector<const void*> key;
    for (int i = 0; i < n; ++i) {
        key.push_back(d_raw[i]);
        key.push_back(d_swst ? d_swst[i] : nullptr);
        key.push_back(reinterpret_cast<const void*>(static_cast<intptr_t>(min_swst ? min_swst[i] : 0)));
        key.push_back(d_out[i]);
    }
    if (!b->graph || key != b->key) {
        graph_destroy(b->graph);
        b->graph = nullptr;
        // one direct run first: sets the kernels' shared-memory attributes and surfaces
        // argument errors outside the capture
        int rc = focus_all(false);
        if (rc) return rc;
        // capture on the batch's own stream: the caller's may be the legacy default stream,
        // which cannot be captured; the graph is launched onto the caller's stream below
        rc = stream_sync(stream);
        if (rc) return rc;
        void* cs = b->cap_stream;
        rc = graph_capture_begin(cs);
        if (rc) return rc;
        rc = event_record(b->ev_fork, cs);
        for (int k = 0; !rc && k < b->branches; ++k) rc = stream_wait_event(b->streams[static_cast<size_t>(k)], b->ev_fork);
        if (!rc) rc = focus_all(true);
        for (int k = 0; !rc && k < b->branches; ++k) {
            rc = event_record(b->ev_join[static_cast<size_t>(k)], b->streams[static_cast<size_t>(k)]);
            if (!rc) rc = stream_wait_event(cs, b->ev_join[static_cast<size_t>(k)]);
        }
        void* exec = nullptr;
        const int rc_end = graph_capture_end(cs, &exec);
        if (rc) {
            graph_destroy(exec);
            return rc;
        }
        if (rc_end) return rc_end;
        b->graph = exec;
        b->key = key;
    }
    return graph_launch(b->graph, stream);
}

}  // extern "C"
