// Long strips focused as overlapped azimuth blocks.
//
// The reference focuses one scene as one padded image and does not support a Doppler
// centroid that drifts along azimuth.  A strip of Na lines is cut here into blocks of
// B lines whose starts are (B - overlap) apart (the last block ends at the strip's last
// line).  Every block is an ordinary plan - its own IQ statistics, its own Doppler
// estimate (so the centroid may vary from block to block), its own Vr (estimated from the
// orbit at its own azimuth time unless the scene gives one) - and its inverse azimuth pass writes only the block's share of the
// strip straight into one strip-wide SLC: the lines between the midpoints of its overlaps
// with the neighbouring blocks (and, at the two strip ends, the lines past a full synthetic
// aperture).  One multilook + range-spreading-loss + SRGR pass then runs over the whole
// strip SLC, so the detected image has no seams.  A block's share is bit-identical to what
// focusing that block alone gives for those lines.
#include <algorithm>
#include <cmath>
#include <vector>

#include "asarf.h"
#include "backend.h"
#include "internal.h"
#include "plan.h"

using namespace asarf;

struct asarf_strip {
    asarf_scene scene{};
    std::vector<asarf_osv> osv;
    int block_lines = 0, overlap = 0, n_blocks = 0;
    int start_margin = 0, end_margin = 0, max_ap = 0;
    std::vector<int> start, keep_lo, keep_hi;
    std::vector<asarf_plan*> plans;
    long long pitch = 0;
    int nx = 0, rows = 0, out_rows = 0, out_cols = 0;
    float2* slc = nullptr;
    FocusState* state = nullptr;
    float* rsl = nullptr;
    TailArgs tail{};
    LaunchShape sh_tail{};
    size_t bytes = 0;
    std::vector<void*> streams, ev_join;
    void* ev_fork = nullptr;

    ~asarf_strip() {
        for (void* s : streams) stream_destroy(s);
        for (void* e : ev_join) event_destroy(e);
        if (ev_fork) event_destroy(ev_fork);
        for (asarf_plan* p : plans) asarf_plan_destroy(p);
        mem_free(slc);
        mem_free(state);
        mem_free(rsl);
    }
};

extern "C" {

int asarf_strip_create(const asarf_scene* scene, int32_t block_lines, int32_t overlap, const asarf_options* opt,
                       asarf_strip** out) {
    if (!scene || !out) return set_error(ASARF_ERR_INVALID, "strip_create: null argument");
    *out = nullptr;
    const int na = scene->azimuth_size;
    if (block_lines < 64 || overlap < 0 || overlap >= block_lines)
        return set_error(ASARF_ERR_INVALID, "strip_create: need 64 <= block_lines and 0 <= overlap < block_lines");
    auto* st = new asarf_strip();
    st->scene = *scene;
    if (scene->n_osv > 0 && scene->osv) st->osv.assign(scene->osv, scene->osv + scene->n_osv);
    st->scene.osv = st->osv.data();
    const int B = std::min<int>(block_lines, na);
    st->block_lines = B;
    st->overlap = overlap;
    st->n_blocks = na <= B ? 1 : 1 + (na - B + (B - overlap) - 1) / (B - overlap);
    for (int k = 0; k < st->n_blocks; ++k) st->start.push_back(std::min(k * (B - overlap), na - B));
    st->max_ap = max_aperture_pixels(st->scene);
    if (st->n_blocks > 1 && overlap < st->max_ap) {
        const int ap = st->max_ap;
        delete st;
        return set_error(ASARF_ERR_INVALID, "strip_create: overlap %d is shorter than the synthetic aperture (%d lines)",
                         overlap, ap);
    }
    st->start_margin = std::max(scene->lines_before, st->max_ap);
    st->end_margin = std::max(scene->lines_after, st->max_ap);
    for (int k = 0; k < st->n_blocks; ++k) {
        const int s = st->start[static_cast<size_t>(k)];
        const int lo = k == 0 ? st->start_margin : (st->start[static_cast<size_t>(k - 1)] + B + s) / 2 - s;
        const int hi = k == st->n_blocks - 1 ? B - st->end_margin : (s + B + st->start[static_cast<size_t>(k + 1)]) / 2 - s;
        if (hi - lo < 8) {
            delete st;
            return set_error(ASARF_ERR_INVALID, "strip_create: block %d keeps %d lines", k, hi - lo);
        }
        st->keep_lo.push_back(lo);
        st->keep_hi.push_back(hi);
    }
    st->rows = na - st->start_margin - st->end_margin;

    // one plan per block, each at its own azimuth time
    for (int k = 0; k < st->n_blocks; ++k) {
        asarf_scene bs = st->scene;
        const int s = st->start[static_cast<size_t>(k)];
        bs.azimuth_size = B;
        bs.total_raw_samples = static_cast<int64_t>(bs.samples_per_line) * B;
        bs.first_line_time_us = scene->first_line_time_us +
                                static_cast<int64_t>(std::llround(s * scene->line_time_interval * 1e6));
        bs.lines_before = bs.lines_after = 0;
        asarf_plan* p = nullptr;
        const int rc = asarf_plan_create(&bs, opt, &p);
        if (rc) {
            delete st;
            return rc;
        }
        st->plans.push_back(p);
    }
    asarf_plan* p0 = st->plans[0];
    st->pitch = p0->pitch;
    st->nx = p0->nx;
    st->slc = static_cast<float2*>(mem_alloc(sizeof(float2) * static_cast<size_t>(st->rows) * st->pitch));
    st->state = static_cast<FocusState*>(mem_alloc(sizeof(FocusState)));
    st->rsl = static_cast<float*>(mem_alloc(sizeof(float) * st->nx));
    if (!st->slc || !st->state || !st->rsl) {
        delete st;
        return set_error(ASARF_ERR_NOMEM, "strip_create: device allocation failed");
    }
    st->bytes = sizeof(float2) * static_cast<size_t>(st->rows) * st->pitch;
    for (int k = 0; k < st->n_blocks; ++k) {
        asarf_plan* p = st->plans[static_cast<size_t>(k)];
        p->skip_tail = true;
        st->bytes += p->bytes;
        // the block's results window is its share of the strip, whatever its Doppler sign
        for (int v = 0; v < kNumTailVariants; ++v) {
            p->a_fin.first_line[v] = st->keep_lo[static_cast<size_t>(k)];
            p->a_fin.n_lines[v] = st->keep_hi[static_cast<size_t>(k)] - st->keep_lo[static_cast<size_t>(k)];
        }
        p->a_inv.out = st->slc;
        p->a_inv.out_row0 = st->start_margin - st->start[static_cast<size_t>(k)];
        p->a_inv.out_intensity = nullptr;  // blocks write their complex share into the strip SLC
        p->intensity_only = false;
    }

    // tail over the whole strip SLC (the planned path's tail with a strip-wide window)
    const asarf_scene& s = st->scene;
    const float ratio = static_cast<float>(12.5f / s.azimuth_spacing);
    st->out_rows = static_cast<int>(std::round(static_cast<float>(st->rows) / ratio));
    asarf_scene ts = s;
    ts.first_line_time_us = s.first_line_time_us +
                            static_cast<int64_t>(std::llround(st->start_margin * s.line_time_interval * 1e6));
    const double sub_first = s.slant_range_first + (kRcmcTaps / 2) * s.range_spacing;
    double poly[5];
    int rc = srgr_poly(ts, sub_first, st->nx, st->out_rows, (1.0 / s.prf) * static_cast<double>(ratio), poly,
                       &st->out_cols);
    if (rc) {
        delete st;
        return rc;
    }
    std::vector<float> rsl(static_cast<size_t>(st->nx));
    for (int i = 0; i < st->nx; ++i) {
        const double R = sub_first + i * s.range_spacing;
        const double ratio_r = 800000.0 / R;  // envisat_format/include/asar_constants.h:37
        rsl[static_cast<size_t>(i)] = static_cast<float>(1.0 / std::sqrt(std::pow(ratio_r, 3)));
    }
    FocusState hs{};
    hs.first_line = 0;
    hs.n_lines = st->rows;
    hs.variant = 0;
    rc = mem_h2d(st->rsl, rsl.data(), sizeof(float) * st->nx, nullptr);
    if (!rc) rc = mem_h2d(st->state, &hs, sizeof(hs), nullptr);
    if (!rc) rc = stream_sync(nullptr);
    if (rc) {
        delete st;
        return rc;
    }
    TailArgs& t = st->tail;
    t = p0->a_tail;
    t.slc = st->slc;
    t.pitch = st->pitch;
    t.state = st->state;
    t.col0 = p0->a_tail.col0;  // full compressed rows are stored; the tail skips the RCMC margin
    for (int v = 0; v < kNumTailVariants; ++v) {
        t.tail[v].n_lines = st->rows;
        t.tail[v].out_az = st->out_rows;
        t.tail[v].ratio = ratio;
        t.tail[v].ng = st->out_cols;
        for (int k = 0; k < 5; ++k) t.tail[v].grsr[k] = static_cast<float>(poly[k]);
        t.tail[v].rsl = st->rsl;
    }
    t.out_pitch = st->out_cols;
    st->sh_tail = p0->sh_tail;

    const int nb = std::min(st->n_blocks, 4);
    for (int k = 0; k < nb; ++k) {
        void* sk = stream_create();
        void* ek = event_create();
        if (!sk || !ek) {
            stream_destroy(sk);
            if (ek) event_destroy(ek);
            delete st;
            return set_error(ASARF_ERR_CUDA, "strip_create: stream creation failed");
        }
        st->streams.push_back(sk);
        st->ev_join.push_back(ek);
    }
    st->ev_fork = event_create();
    if (!st->ev_fork) {
        delete st;
        return set_error(ASARF_ERR_CUDA, "strip_create: event creation failed");
    }
    *out = st;
    return ASARF_OK;
}

void asarf_strip_destroy(asarf_strip* st) { delete st; }

int asarf_strip_get_dims(const asarf_strip* st, asarf_strip_dims* d) {
    if (!st || !d) return set_error(ASARF_ERR_INVALID, "strip_dims: null argument");
    d->n_blocks = st->n_blocks;
    d->block_lines = st->block_lines;
    d->overlap = st->overlap;
    d->first_line = st->start_margin;
    d->slc_rows = st->rows;
    d->slc_cols = st->nx;
    d->slc_pitch = static_cast<int32_t>(st->pitch);
    d->out_rows = st->out_rows;
    d->out_cols = st->out_cols;
    d->max_aperture = st->max_ap;
    d->device_bytes = st->bytes;
    return ASARF_OK;
}

int asarf_strip_block(const asarf_strip* st, int32_t k, int32_t* start, int32_t* keep_lo, int32_t* keep_hi,
                      asarf_plan** plan) {
    if (!st || k < 0 || k >= st->n_blocks) return set_error(ASARF_ERR_INVALID, "strip_block: index out of range");
    if (start) *start = st->start[static_cast<size_t>(k)];
    if (keep_lo) *keep_lo = st->keep_lo[static_cast<size_t>(k)];
    if (keep_hi) *keep_hi = st->keep_hi[static_cast<size_t>(k)];
    if (plan) *plan = st->plans[static_cast<size_t>(k)];
    return ASARF_OK;
}

int asarf_focus_strip(asarf_strip* st, const uint8_t* d_raw, const uint16_t* d_swst, int32_t min_swst, float* d_out,
                      void* stream) {
    if (!st || !d_raw || !d_out) return set_error(ASARF_ERR_INVALID, "focus_strip: null argument");
    const int nb = static_cast<int>(st->streams.size());
    int rc = event_record(st->ev_fork, stream);
    for (int k = 0; !rc && k < nb; ++k) rc = stream_wait_event(st->streams[static_cast<size_t>(k)], st->ev_fork);
    for (int k = 0; !rc && k < st->n_blocks; ++k) {
        const long long s = st->start[static_cast<size_t>(k)];
        rc = asarf_focus(st->plans[static_cast<size_t>(k)], d_raw + s * st->scene.raw_line_bytes,
                         d_swst ? d_swst + s : nullptr, min_swst, nullptr, st->streams[static_cast<size_t>(k % nb)]);
    }
    for (int k = 0; !rc && k < nb; ++k) {
        rc = event_record(st->ev_join[static_cast<size_t>(k)], st->streams[static_cast<size_t>(k)]);
        if (!rc) rc = stream_wait_event(stream, st->ev_join[static_cast<size_t>(k)]);
    }
    if (!rc) rc = mem_zero(&st->state->errors, sizeof(unsigned int), stream);
    if (rc) return rc;
    TailArgs t = st->tail;
    t.out = d_out;
    return backend_tail(t, st->out_rows, st->sh_tail, &st->state->errors, stream);
}

int asarf_strip_slc(asarf_strip* st, void* d_slc, void* stream) {
    if (!st || !d_slc) return set_error(ASARF_ERR_INVALID, "strip_slc: null argument");
    return mem_d2d_2d(d_slc, sizeof(float2) * st->nx, st->slc + st->tail.col0, sizeof(float2) * st->pitch,
                      sizeof(float2) * st->nx, st->rows, stream);
}

int asarf_strip_errors(asarf_strip* st, uint32_t* errors, void* stream) {
    if (!st || !errors) return set_error(ASARF_ERR_INVALID, "strip_errors: null argument");
    unsigned int e = 0, v = 0;
    int rc = mem_d2h(&v, &st->state->errors, sizeof(v), stream);
    if (!rc) rc = stream_sync(stream);
    if (rc) return rc;
    e |= v;
    for (asarf_plan* p : st->plans) {
        asarf_results r{};
        rc = asarf_plan_results(p, &r, stream);
        if (rc) return rc;
        e |= r.errors;
    }
    *errors = e;
    return ASARF_OK;
}

}  // extern "C"
