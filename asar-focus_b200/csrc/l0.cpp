// ERS IM level-0 packets -> device-resident raw lines.
//
// The reference reads an ERS_SAR_0P product's measurement data set (MDSRs of 11498 bytes) in
// two host passes: FetchErsL0ImForecastMeta (envisat_format/src/ers_im_parse.cc:228-354)
// walks the packets' data record numbers and sensing times to decide which packets make the
// lines (a packet whose record number skips ahead is preceded by copies of the previous
// packet, at most 900; a sensing-time window trims the ends), then ParseErsLevel0ImPackets
// (:356-580) copies each listed packet's 11232 measurement bytes into a host raw buffer that
// main.cc uploads.  Here the forecast stays on the host (it reads 18 bytes per packet), and
// the packets travel to the GPU as they lie in the file: asarf_ers_l0_unpack gathers the
// measurement bytes and the SWST / PRI codes of every line in one kernel, so the raw buffer
// the focusing kernels read is written on the device and the upload moves the packets once.
#include <cstdint>
#include <cstring>
#include <vector>

#include "asarf.h"
#include "backend.h"
#include "params.h"

namespace asarf {
namespace {

uint32_t be32(const uint8_t* p) {
    return (static_cast<uint32_t>(p[0]) << 24) | (static_cast<uint32_t>(p[1]) << 16) |
           (static_cast<uint32_t>(p[2]) << 8) | p[3];
}
uint16_t be16(const uint8_t* p) { return static_cast<uint16_t>((p[0] << 8) | p[1]); }

asarf_mjd packet_time(const uint8_t* pk) {
    asarf_mjd t;
    t.days = static_cast<int32_t>(be32(pk));
    t.seconds = be32(pk + 4);
    t.micros = be32(pk + 8);
    return t;
}

// mjd::operator< / operator> (envisat_format/include/envisat_types.h:50-72)
bool mjd_less(const asarf_mjd& a, const asarf_mjd& b) {
    if (a.days != b.days) return a.days < b.days;
    if (a.seconds != b.seconds) return a.seconds < b.seconds;
    return a.micros < b.micros;
}
bool mjd_greater(const asarf_mjd& a, const asarf_mjd& b) { return mjd_less(b, a); }

// parseutil::CounterGap<uint32_t, LIMIT> (envisat_format/include/parse_util.h:33-46)
uint32_t counter_gap(uint32_t last, uint32_t cur, uint32_t limit) {
    if (static_cast<uint32_t>(last + 1u) == cur) return 1;
    if (cur < last) return static_cast<uint32_t>(limit - last + cur + 1u);
    return cur - last;
}

// InitializeDataRecordNo (ers_im_parse.cc:93-103): the packet's record number minus one
uint32_t record_no_before(const uint8_t* pk) {
    const uint32_t v = be32(pk + 32);
    return v != 0 ? v - 1 : 0xFFFFFFFFu;
}

}  // namespace
}  // namespace asarf

using namespace asarf;

extern "C" int asarf_ers_l0_forecast(const uint8_t* mdsr, int64_t blob_bytes, int64_t num_dsr, int64_t dsr_size,
                                     const asarf_mjd* start, const asarf_mjd* stop, int64_t* packets_before_start,
                                     int64_t* packets_after_stop, int64_t* offsets, asarf_mjd* times,
                                     int64_t capacity, int64_t* count) {
    if (!mdsr || !start || !stop || !packets_before_start || !packets_after_stop || !count || num_dsr <= 0)
        return set_error(ASARF_ERR_INVALID, "ers_l0_forecast: null argument or no packets");
    if (dsr_size != kErsMdsrBytes)
        return set_error(ASARF_ERR_INVALID,
                         "Expected DSR to be %d bytes, actual - %lld. This is a failsafe abort, check the dataset.",
                         kErsMdsrBytes, static_cast<long long>(dsr_size));
    if (blob_bytes != num_dsr * dsr_size)
        return set_error(ASARF_ERR_INVALID,
                         "Actual packets BLOB array (%lld bytes) is not equal to dataset defined packets (%lld bytes).",
                         static_cast<long long>(blob_bytes), static_cast<long long>(num_dsr * dsr_size));
    struct Entry {
        int64_t offset;
        asarf_mjd time;
    };
    std::vector<Entry> fc;
    int64_t before = 0, after = 0;
    uint32_t last_dr = record_no_before(mdsr);
    for (int64_t i = 0; i < num_dsr; ++i) {
        const uint8_t* pk = mdsr + i * dsr_size;
        Entry cur{i * dsr_size, packet_time(pk)};
        const uint16_t isp_length = be16(pk + 24);
        if (isp_length != 11465)
            return set_error(ASARF_ERR_INVALID,
                             "FEP annotation's ISP length shall be 11465. Check the dataset, current one has %u",
                             static_cast<unsigned>(isp_length));
        // sensing times are adjusted by a PATC auxiliary correction only when one is registered
        // (ers::AdjustIspSensingTime, envisat_format/src/ers_sbt.cc:56-84); none is used here
        const uint32_t dr = record_no_before(pk);
        const uint32_t gap = counter_gap(last_dr, dr, 0xFFFFFFFFu);
        if (gap > 1) {
            if (fc.empty())
                return set_error(ASARF_ERR_INVALID,
                                 "Implementation error detected - data record no. discontinuity detected, but no "
                                 "packets have been fetched yet in order to fill packets");
            const int64_t fill = static_cast<int64_t>(gap) - 1;
            if (fill > 900)
                return set_error(ASARF_ERR_INVALID,
                                 "There are %lld packets missing, which is more than threshold 900 in order to "
                                 "continue. It was detected between %lldth and %lldth packets.",
                                 static_cast<long long>(fill), static_cast<long long>(i - 1),
                                 static_cast<long long>(i));
            const Entry prev = fc.back();
            for (int64_t k = 0; k < fill; ++k) fc.push_back(prev);
            if (mjd_less(prev.time, *start)) before += fill;
            if (mjd_greater(prev.time, *stop)) after += fill;
        } else {
            if (mjd_less(cur.time, *start)) ++before;
            if (mjd_greater(cur.time, *stop)) ++after;
        }
        if (after > *packets_after_stop) {
            --after;
            break;
        }
        last_dr = dr;
        fc.push_back(cur);
    }
    if (before > *packets_before_start) {
        const int64_t drop = before - *packets_before_start;
        fc.erase(fc.begin(), fc.begin() + drop);
        before -= drop;
        if (*packets_before_start == 0)
            while (!fc.empty() && mjd_less(fc.front().time, *start)) fc.erase(fc.begin());
    }
    *packets_before_start = before;
    *packets_after_stop = after;
    *count = static_cast<int64_t>(fc.size());
    if (offsets || times) {
        if (capacity < *count)
            return set_error(ASARF_ERR_INVALID, "ers_l0_forecast: %lld lines, capacity %lld",
                             static_cast<long long>(*count), static_cast<long long>(capacity));
        for (size_t k = 0; k < fc.size(); ++k) {
            if (offsets) offsets[k] = fc[k].offset;
            if (times) times[k] = fc[k].time;
        }
    }
    return ASARF_OK;
}

extern "C" int asarf_ers_l0_unpack(const uint8_t* d_mdsr, const int64_t* d_offsets, int32_t lines, uint8_t* d_raw,
                                   uint16_t* d_swst, uint16_t* d_pri, uint32_t* d_errors, void* stream) {
    if (!d_mdsr || !d_offsets || !d_raw || !d_errors || lines <= 0)
        return set_error(ASARF_ERR_INVALID, "ers_l0_unpack: null argument or no lines");
    if (reinterpret_cast<uintptr_t>(d_mdsr) & 1)
        return set_error(ASARF_ERR_INVALID, "ers_l0_unpack: the packet buffer must be 2-byte aligned");
    ErsUnpackArgs a{};
    a.mdsr = d_mdsr;
    a.offset = reinterpret_cast<const long long*>(d_offsets);
    a.lines = lines;
    a.raw = d_raw;
    a.swst = d_swst;
    a.pri = d_pri;
    a.errors = d_errors;
    return backend_ers_unpack(a, stream);
}
