// ERS IM and ENVISAT ASAR IM level-0 packets -> device-resident raw lines / FBAQ4 records.
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
//
// ASA_IM__0P packets have variable length (FBAQ4 sample blocks), so the walk follows each
// packet's ISP length: FetchEnvisatL0ImForecastMeta (envisat_format/src/envisat_im_parse.cc:
// 297-385) keeps echo and calibration packets from the first echo on under the same window
// rule; ParseEnvisatLevel0ImPackets (:387-676) sizes the records by the largest echo block
// length (ForecastMaxBlockDataLength, :159-197) and copies each echo's blocks behind a 2-byte
// length, a calibration packet repeating the previous line.  Here asarf_asar_l0_lines does the
// host bookkeeping (which echo packet each line holds, sensing times) and asarf_asar_l0_unpack
// writes the FBAQ4 records the focusing path reads, on the device.
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

// ---- ENVISAT ASAR IM packets (variable length)
struct AsarHeader {
    asarf_mjd time;
    uint16_t isp_length, packet_length, datafield_length, pri;
    uint8_t mode, flags;
    bool echo() const { return (flags & 0x80) != 0; }
    bool cal() const { return (flags & 0x20) != 0; }
};

// The header of the packet at byte `off`; false when it does not lie inside the data set.
bool asar_header(const uint8_t* mdsr, int64_t blob_bytes, int64_t off, AsarHeader& h) {
    if (off < 0 || off + kAsarPacketHeader > blob_bytes) return false;
    const uint8_t* pk = mdsr + off;
    h.time = packet_time(pk);
    h.isp_length = be16(pk + 24);
    h.packet_length = be16(pk + 36);
    h.datafield_length = be16(pk + 38);
    h.mode = pk[41];
    h.flags = pk[52];
    h.pri = be16(pk + 54);
    return true;
}

int64_t asar_next(int64_t off, const AsarHeader& h) { return off + kAsarNextPacketBase + h.isp_length; }

// MjdAddMicros (envisat_format/include/envisat_utils.h:74-78): the time plus whole microseconds,
// carried into seconds and days.
asarf_mjd mjd_add_micros(asarf_mjd t, uint64_t add) {
    const uint64_t us = static_cast<uint64_t>(t.micros) + add;
    const uint64_t sec = static_cast<uint64_t>(t.seconds) + us / 1000000u;
    t.micros = static_cast<uint32_t>(us % 1000000u);
    t.days += static_cast<int32_t>(sec / 86400u);
    t.seconds = static_cast<uint32_t>(sec % 86400u);
    return t;
}

// Samples held by `bytes` of FBAQ4 block data: 63 per 64-byte block, the last block partial
// (envisat_format/src/envisat_im_parse.cc:589-592).
int64_t fbaq_block_samples(int64_t bytes) { return (bytes / 64) * 63 + bytes % 64 - (bytes % 64 > 0 ? 1 : 0); }

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

extern "C" int asarf_asar_l0_forecast(const uint8_t* mdsr, int64_t blob_bytes, int64_t num_dsr, const asarf_mjd* start,
                                      const asarf_mjd* stop, int64_t* packets_before_start,
                                      int64_t* packets_after_stop, int64_t* offsets, asarf_mjd* times,
                                      int64_t capacity, int64_t* count) {
    if (!mdsr || !start || !stop || !packets_before_start || !packets_after_stop || !count || num_dsr <= 0)
        return set_error(ASARF_ERR_INVALID, "asar_l0_forecast: null argument or no packets");
    struct Entry {
        int64_t offset;
        asarf_mjd time;
    };
    std::vector<Entry> fc;
    int64_t before = 0, after = 0;
    bool last_cal = false;  // the calibration flag of the last packet read by the walk
    int64_t off = 0;
    for (int64_t i = 0; i < num_dsr; ++i) {
        AsarHeader h;
        if (!asar_header(mdsr, blob_bytes, off, h))
            return set_error(ASARF_ERR_INVALID, "asar_l0_forecast: packet %lld at byte %lld lies outside the %lld bytes",
                             static_cast<long long>(i), static_cast<long long>(off),
                             static_cast<long long>(blob_bytes));
        if (h.datafield_length != 29)
            return set_error(ASARF_ERR_INVALID,
                             "Fetching metadat for ENVISAT IM parse error. Date Field Header Length should be 29 - "
                             "is %u",
                             static_cast<unsigned>(h.datafield_length));
        const Entry cur{off, h.time};
        off = asar_next(off, h);
        last_cal = h.cal();
        if (fc.empty() && !h.echo()) continue;  // the list starts at an echo packet
        if (!h.echo() && !h.cal()) continue;    // noise packets are not lines
        if (mjd_less(cur.time, *start)) ++before;
        if (mjd_greater(cur.time, *stop)) ++after;
        if (after > *packets_after_stop) {
            --after;
            break;
        }
        fc.push_back(cur);
    }
    if (before > *packets_before_start) {
        const int64_t drop = before - *packets_before_start;
        fc.erase(fc.begin(), fc.begin() + drop);
        before -= drop;
        // a calibration packet left in front is removed, which the reference allows only when the
        // walk's last packet was a calibration packet (it tests that packet's flag,
        // envisat_im_parse.cc:359-378); the count goes down with it (below zero it wraps there)
        while (!fc.empty()) {
            AsarHeader h;
            asar_header(mdsr, blob_bytes, fc.front().offset, h);
            if (h.echo()) break;
            if (!last_cal)
                return set_error(ASARF_ERR_INVALID,
                                 "Programming error detected - only echo and calibration packets should have been "
                                 "fetched.");
            fc.erase(fc.begin());
            --before;
        }
    }
    *packets_before_start = before;
    *packets_after_stop = after;
    *count = static_cast<int64_t>(fc.size());
    if (offsets || times) {
        if (capacity < *count)
            return set_error(ASARF_ERR_INVALID, "asar_l0_forecast: %lld lines, capacity %lld",
                             static_cast<long long>(*count), static_cast<long long>(capacity));
        for (size_t k = 0; k < fc.size(); ++k) {
            if (offsets) offsets[k] = fc[k].offset;
            if (times) times[k] = fc[k].time;
        }
    }
    return ASARF_OK;
}

extern "C" int asarf_asar_l0_lines(const uint8_t* mdsr, int64_t blob_bytes, const int64_t* offsets, int64_t count,
                                   float range_sampling_rate, int64_t* src_offsets, asarf_mjd* times,
                                   int32_t* record_bytes, int32_t* max_samples) {
    if (!mdsr || !offsets || !src_offsets || !record_bytes || count <= 0)
        return set_error(ASARF_ERR_INVALID, "asar_l0_lines: null argument or no lines");
    // ForecastMaxBlockDataLength (envisat_im_parse.cc:159-197): `count` consecutive packets from
    // the first line's packet, the largest echo block-data length
    uint16_t max_block = 0;
    int64_t echoes = 0;
    int64_t off = offsets[0];
    for (int64_t k = 0; k < count; ++k) {
        AsarHeader h;
        if (!asar_header(mdsr, blob_bytes, off, h))
            return set_error(ASARF_ERR_INVALID, "asar_l0_lines: packet at byte %lld lies outside the %lld bytes",
                             static_cast<long long>(off), static_cast<long long>(blob_bytes));
        if (h.datafield_length != 29)
            return set_error(ASARF_ERR_INVALID,
                             "DSR sequence = %lld parsing error. Date Field Header Length should be 29 - is %u",
                             static_cast<long long>(k + 1), static_cast<unsigned>(h.datafield_length));
        if (h.echo()) {
            const uint16_t len = static_cast<uint16_t>(h.packet_length - 29);
            if (len > max_block) max_block = len;
            ++echoes;
        }
        off = asar_next(off, h);
    }
    if (echoes < 10)
        return set_error(ASARF_ERR_INVALID,
                         "Could not gather atleast 10 echo packets in order to forecast data block lengths - invalid "
                         "dataset?");
    // ParseEnvisatLevel0ImPackets (envisat_im_parse.cc:387-676), the host part: which packet's
    // blocks each line holds and its sensing time
    int64_t most = 0;
    uint16_t last_pri = 0;
    for (int64_t k = 0; k < count; ++k) {
        AsarHeader h;
        if (!asar_header(mdsr, blob_bytes, offsets[k], h))
            return set_error(ASARF_ERR_INVALID, "asar_l0_lines: line %lld's packet lies outside the data set",
                             static_cast<long long>(k));
        if (h.datafield_length != 29)
            return set_error(ASARF_ERR_INVALID,
                             "DSR index = %lld parsing error. Date Field Header Length should be 29 - is %u",
                             static_cast<long long>(k), static_cast<unsigned>(h.datafield_length));
        if (h.mode != 0x54)
            return set_error(ASARF_ERR_INVALID, "Expected only IM mode packets, but encountered mode ID %#x",
                             static_cast<unsigned>(h.mode));
        if (h.echo()) {
            // the unpack kernel reads the packet's blocks from the device copy of this data set
            const int64_t blocks = static_cast<uint16_t>(h.packet_length - 29);
            if (offsets[k] + kAsarPacketHeader + blocks > blob_bytes)
                return set_error(ASARF_ERR_INVALID, "asar_l0_lines: line %lld's sample blocks end past the data set",
                                 static_cast<long long>(k));
            src_offsets[k] = offsets[k];
            if (times) times[k] = h.time;
            last_pri = h.pri;
            const int64_t n = fbaq_block_samples(blocks);
            if (n > most) most = n;
        } else if (h.cal()) {
            // the previous line repeated, its sensing time advanced by one PRI in whole
            // microseconds (float PRF = sampling rate / PRI code, as the reference computes it)
            if (k == 0)
                return set_error(ASARF_ERR_INVALID, "asar_l0_lines: the first line is a calibration packet");
            src_offsets[k] = src_offsets[k - 1];
            if (times) {
                const float prf = range_sampling_rate / static_cast<float>(last_pri);
                const float pri_s = 1.0f / prf;
                const uint32_t add = static_cast<uint32_t>(static_cast<double>(pri_s) * 10e5);
                times[k] = mjd_add_micros(times[k - 1], add);
            }
        } else {
            return set_error(ASARF_ERR_INVALID,
                             "Programming error detected - only echo and calibration packets should have been "
                             "fetched.");
        }
    }
    const int64_t forecast_most = fbaq_block_samples(max_block);
    if (most != forecast_most)
        return set_error(ASARF_ERR_INVALID, "Post-parse max samples %lld do not equal with forecast %lld",
                         static_cast<long long>(most), static_cast<long long>(forecast_most));
    *record_bytes = static_cast<int32_t>(max_block) + 2;
    if (max_samples) *max_samples = static_cast<int32_t>(most);
    return ASARF_OK;
}

extern "C" int asarf_asar_l0_unpack(const uint8_t* d_mdsr, const int64_t* d_src_offsets, int32_t lines,
                                    int32_t record_bytes, uint8_t* d_records, uint16_t* d_swst, uint16_t* d_pri,
                                    uint32_t* d_errors, void* stream) {
    if (!d_mdsr || !d_src_offsets || !d_records || !d_errors || lines <= 0 || record_bytes < 2)
        return set_error(ASARF_ERR_INVALID, "asar_l0_unpack: null argument, no lines or record_bytes < 2");
    AsarUnpackArgs a{};
    a.mdsr = d_mdsr;
    a.src = reinterpret_cast<const long long*>(d_src_offsets);
    a.lines = lines;
    a.record_bytes = record_bytes;
    a.records = d_records;
    a.swst = d_swst;
    a.pri = d_pri;
    a.errors = d_errors;
    return backend_asar_unpack(a, stream);
}
