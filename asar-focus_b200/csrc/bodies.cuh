// Kernel bodies of the focusing path, written once for the device and the host emulation.
//
// A body is a function of (block coordinates, tid, nthr, shared-memory pointer) made of
// phases separated by ASARF_SYNC(); inside a phase every work item is independent.
// Reference behaviour each body reproduces is cited in its comment
// (paths relative to the asar-focus source tree).
#pragma once

#include <cmath>
#include <cstdint>

#include "fft.cuh"
#include "fft_ct.cuh"
#include "hd.cuh"
#include "params.h"

namespace asarf {

ASARF_HD ASARF_INLINE void atomic_or_u32(unsigned int* p, unsigned int v) {
#if defined(__CUDA_ARCH__)
    atomicOr(p, v);
#else
    *p |= v;
#endif
}

// numpy.blackman(16) in float32, the RCMC tap window (sar/range_doppler_algorithm.cu:46-52):
// 0.42 - 0.5 cos(2 pi n / 15) + 0.08 cos(4 pi n / 15) rounded to float.
#define ASARF_BLACKMAN16                                                                                      \
    {-1.3877787807814457e-17f, 0.016757719218730927f, 0.07707241922616959f, 0.20077013969421387f,             \
     0.3940124213695526f,      0.6299999952316284f,   0.8492298722267151f,  0.9821574091911316f,              \
     0.9821574091911316f,      0.8492298722267151f,   0.6299999952316284f,  0.3940124213695526f,              \
     0.20077013969421387f,     0.07707241922616959f,  0.016757719218730927f, -1.3877787807814457e-17f}

// Device Polyval<N> of the reference (float Horner; nvcc contracts r*x + e into one fma).
template <int N>
ASARF_HD ASARF_INLINE float polyval_f32(const float (&p)[N], float x) {
    float r = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) r = fma_rn(r, x, p[i]);
    return r;
}

// ----------------------------------------------------------------------------- least squares
// Householder-QR least-squares polynomial fit, coefficients highest power first
// (Polyfit, util/src/math_utils.cc:23-44).  m <= 128 points, degree <= 4.
template <int kM, int kN>
ASARF_HD inline bool polyfit_qr(const double* x, const double* y, int m, int deg, double* out) {
    const int n = deg + 1;
    if (m > kM || n > kN || m < n) return false;
    double A[kN][kM];  // column-major: A[col][row]
    double b[kM];
    for (int r = 0; r < m; ++r) {
        double v = 1.0;
        for (int c = 0; c < n; ++c) {
            A[c][r] = v;
            v *= x[r];
        }
        b[r] = y[r];
    }
    for (int k = 0; k < n; ++k) {
        double nrm = 0.0;
        for (int r = k; r < m; ++r) nrm += A[k][r] * A[k][r];
        nrm = sqrt(nrm);
        if (nrm == 0.0) return false;
        const double alpha = A[k][k] > 0 ? -nrm : nrm;
        // Householder vector v = A[k][k:] - alpha e_k kept in column k (its head in vk)
        const double vk = A[k][k] - alpha;
        double vn = vk * vk;
        for (int r = k + 1; r < m; ++r) vn += A[k][r] * A[k][r];
        if (vn == 0.0) return false;
        for (int c = k + 1; c < n; ++c) {
            double d = vk * A[c][k];
            for (int r = k + 1; r < m; ++r) d += A[k][r] * A[c][r];
            const double f = 2.0 * d / vn;
            A[c][k] -= f * vk;
            for (int r = k + 1; r < m; ++r) A[c][r] -= f * A[k][r];
        }
        double d = vk * b[k];
        for (int r = k + 1; r < m; ++r) d += A[k][r] * b[r];
        const double f = 2.0 * d / vn;
        b[k] -= f * vk;
        for (int r = k + 1; r < m; ++r) b[r] -= f * A[k][r];
        A[k][k] = alpha;  // R diagonal
    }
    double c[kN];
    for (int k = n - 1; k >= 0; --k) {
        double s = b[k];
        for (int j = k + 1; j < n; ++j) s -= A[j][k] * c[j];
        c[k] = s / A[k][k];
    }
    for (int k = 0; k < n; ++k) out[k] = c[n - 1 - k];
    return true;
}

// ----------------------------------------------------------------------------- raw statistics
// One pass over the raw I/Q bytes.  Replaces, exactly and in integers, the reductions of
// RawDataCorrection (sar/iq_correction.cu:188-274: mean, std-dev, gain and phase sums)
// and of CalculateDopplerCentroid (sar/fractional_doppler_centroid.cu:33-69: lag-1
// azimuth correlation per range block): the IQ correction is affine in the raw bytes,
// so every sum the reference takes over corrected floats is a closed form of these.
// Block (bx, by) covers kStatsCols work units and lines [by*L, (by+1)*L).  A unit is either
// one column (general path) or, when the raw base and line stride are 8-byte aligned, the
// columns of one Doppler block inside an aligned group of 4 (quad path: columns 4g .. 4g + 3,
// one aligned 8-byte load per line, byte-lane dot products for all sums; a group that straddles
// a Doppler block boundary is two units, one per block, each masking the other's columns).
// Either way every sum a thread keeps belongs to a single Doppler block, and kStatsBatch lines
// are loaded before any is consumed.
constexpr int kStatsCols = 256;
constexpr int kStatsBatch = 8;
constexpr int kStatsMaxLines = 256;
// lines per block of the statistics kernel (measured on the 28000- and 30000-line scenes:
// 64 -> 0.203, 128 -> 0.170, 192 -> 0.155, 256 -> 0.171 ms)
constexpr int kStatsLinesPerBlock = 192;
constexpr int kStatsBlocksPerSm = 3;  // resident blocks of k_raw_stats (its launch bounds)

// Lines per statistics block for a grid of gx block columns over na lines: kStatsLinesPerBlock,
// raised in whole batches (at most kStatsMaxLines) when that fits the grid into one wave fewer
// of the `slots` resident blocks, since the last wave of a grid of equal blocks runs mostly
// empty (ASAR IM-like 30000 lines, 6 columns, 444 slots: 942 blocks of 192 lines take three
// waves, 870 of 208 lines two).
inline int stats_lines_per_block(int na, int gx, int slots) {
    const long long rows = (na + kStatsLinesPerBlock - 1) / kStatsLinesPerBlock;
    const long long waves = (rows * gx + slots - 1) / slots;
    if (waves > 1 && gx > 0) {
        const long long fit_rows = (waves - 1) * slots / gx;
        if (fit_rows > 0) {
            long long l = (na + fit_rows - 1) / fit_rows;
            l = (l + kStatsBatch - 1) / kStatsBatch * kStatsBatch;
            if (l <= kStatsMaxLines) return static_cast<int>(l);
        }
    }
    return kStatsLinesPerBlock;
}

struct RawStatsSmem {
    unsigned long long mom[6];
    unsigned long long lag[kMaxDcBlocks][9];
    int off[kStatsMaxLines + 1];  // SWST shift of the block's lines (and the line before)
};

// Host side: work units and grid width of the statistics kernel for this raw buffer.
inline int raw_stats_grid_x(RawStatsArgs& a, const void* raw) {
    a.gpb = (a.dc_step + 3) / 4 + 1;  // aligned groups a block's columns touch
    a.quad = (reinterpret_cast<uintptr_t>(raw) % 8 == 0 && a.line_bytes % 8 == 0) ? 1 : 0;
    const int units = a.quad ? a.nblk * a.gpb : a.nr;
    return (units + kStatsCols - 1) / kStatsCols;
}

// sum over the four byte lanes of a * b, plus c
ASARF_HD ASARF_INLINE unsigned int dp4(unsigned int a, unsigned int b, unsigned int c) {
#if defined(__CUDA_ARCH__)
    return __dp4a(a, b, c);
#else
    for (int k = 0; k < 32; k += 8) c += ((a >> k) & 0xffu) * ((b >> k) & 0xffu);
    return c;
#endif
}

ASARF_HD ASARF_INLINE unsigned int funnel_r(unsigned int lo, unsigned int hi, unsigned int sh) {
#if defined(__CUDA_ARCH__)
    return __funnelshift_r(lo, hi, sh);
#else
    return sh == 0 ? lo : static_cast<unsigned int>(((static_cast<unsigned long long>(hi) << 32) | lo) >> sh);
#endif
}

// bytes of (x, y) = b0..b7 picked by the low 3 bits of each selector nibble (PRMT default mode)
ASARF_HD ASARF_INLINE unsigned int byte_perm(unsigned int x, unsigned int y, unsigned int s) {
#if defined(__CUDA_ARCH__)
    return __byte_perm(x, y, s);
#else
    const unsigned long long xy = (static_cast<unsigned long long>(y) << 32) | x;
    unsigned int r = 0;
    for (int n = 0; n < 4; ++n) r |= static_cast<unsigned int>((xy >> (8 * ((s >> (4 * n)) & 7u))) & 0xffu) << (8 * n);
    return r;
#endif
}

ASARF_HD ASARF_INLINE int popc_u32(unsigned int v) {
#if defined(__CUDA_ARCH__)
    return __popc(v);
#else
    return __builtin_popcount(v);
#endif
}

// Reduce this thread's sums into the block's shared accumulators (lag sums of Doppler block blk).
ASARF_HD ASARF_INLINE void raw_stats_reduce(RawStatsSmem* sm, bool valid, int blk, unsigned long long mv[6],
                                            unsigned int lv[9]) {
#if defined(__CUDA_ARCH__)
    // every lane of the block runs exactly one unit (kStatsCols == blockDim.x): warp sums first
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        unsigned long long v = mv[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        mv[k] = v;
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int k = 0; k < 6; ++k) atomic_add_u64(&sm->mom[k], mv[k]);
    }
    const int bmin = __reduce_min_sync(0xffffffffu, valid ? blk : 0x7fffffff);
    const int bmax = __reduce_max_sync(0xffffffffu, valid ? blk : -1);
    if (bmin == bmax) {
#pragma unroll
        for (int q = 0; q < 9; ++q) lv[q] = __reduce_add_sync(0xffffffffu, valid ? lv[q] : 0u);
        if ((threadIdx.x & 31) == 0)
            for (int q = 0; q < 9; ++q) atomic_add_u64(&sm->lag[bmin][q], lv[q]);
    } else if (valid) {
        for (int q = 0; q < 9; ++q) atomic_add_u64(&sm->lag[blk][q], lv[q]);
    }
#else
    for (int k = 0; k < 6; ++k) atomic_add_u64(&sm->mom[k], mv[k]);
    if (valid)
        for (int q = 0; q < 9; ++q) atomic_add_u64(&sm->lag[blk][q], lv[q]);
#endif
}

// General path: one column per unit, one 2-byte load per line.
ASARF_HD ASARF_INLINE void raw_stats_column(const RawStatsArgs& a, const RawStatsSmem* sm, int x, int y0, int y1,
                                            int ys, unsigned long long mv[6], unsigned int lv[9]) {
    unsigned int cnt = 0, si = 0, sq = 0, sii = 0, sqq = 0, siq = 0;
    unsigned int l0 = 0, l1 = 0, l2 = 0, l3 = 0, l4 = 0, l5 = 0, l6 = 0, l7 = 0, l8 = 0;
    unsigned int pi = 0, pq = 0;
    bool pf = false;
    const uint8_t* col = a.raw + 2ll * x;
    for (int yg = ys; yg < y1; yg += kStatsBatch) {
        unsigned int w[kStatsBatch];
        bool f[kStatsBatch];
#pragma unroll
        for (int u = 0; u < kStatsBatch; ++u) {
            const int y = yg + u;
            f[u] = false;
            w[u] = 0u;
            if (y < y1) {
                const int off = sm->off[y - ys];
                const int i = x - off;
                if (i >= 0 && i < a.spl) {
                    f[u] = true;
                    w[u] = *reinterpret_cast<const uint16_t*>(col + static_cast<long long>(y) * a.line_bytes - 2ll * off);
                }
            }
        }
#pragma unroll
        for (int u = 0; u < kStatsBatch; ++u) {
            const int y = yg + u;
            if (y >= y1) break;
            const unsigned int iv = w[u] & 0xffu, qv = w[u] >> 8;
            if (y >= y0 && f[u]) {
                cnt += 1;
                si += iv;
                sq += qv;
                sii += iv * iv;
                sqq += qv * qv;
                siq += iv * qv;
                if (y > 0 && pf) {
                    l0 += 1;
                    l1 += pi;
                    l2 += pq;
                    l3 += iv;
                    l4 += qv;
                    l5 += pi * iv;
                    l6 += pq * qv;
                    l7 += pi * qv;
                    l8 += pq * iv;
                }
            }
            pi = iv;
            pq = qv;
            pf = f[u];
        }
    }
    mv[0] = cnt, mv[1] = si, mv[2] = sq, mv[3] = sii, mv[4] = sqq, mv[5] = siq;
    lv[0] = l0, lv[1] = l1, lv[2] = l2, lv[3] = l3, lv[4] = l4, lv[5] = l5, lv[6] = l6, lv[7] = l7, lv[8] = l8;
}

// Quad path: the columns of `colmask` (bit k: column x0 + k) of the aligned group at x0
// (x0 % 4 == 0), all in one Doppler block.  A line's four samples are the aligned 8 bytes
// (I0 Q0 I1 Q1 | I2 Q2 I3 Q3) at raw + y*line_bytes + 2*(x0 - off) (the SWST shift is a
// multiple of 4 samples, so the window stays aligned on every line).  Samples outside the
// record or the mask are zero bytes, which drop out of every sum.
ASARF_HD ASARF_INLINE void raw_stats_quad(const RawStatsArgs& a, const RawStatsSmem* sm, int x0, unsigned int colmask,
                                          int y0, int y1, int ys, unsigned long long mv[6], unsigned int lv[9]) {
    constexpr unsigned int kLo = 0x00ff00ffu, kOnes = 0x01010101u;
    const unsigned int colbits = colmask;
    const int ncol = popc_u32(colmask);
    unsigned int cnt = 0, si = 0, sq = 0, sii = 0, sqq = 0, siq = 0;
    unsigned int l0 = 0, l1 = 0, l2 = 0, l3 = 0, l4 = 0, l5 = 0, l6 = 0, l7 = 0, l8 = 0;
    unsigned int pI0 = 0, pI1 = 0, pQ0 = 0, pQ1 = 0, pfb = 0;
    const uint8_t* base = a.raw + 2ll * x0;
    // byte masks of the group's columns: in the packed I (or Q) word byte k is column k; in the
    // two raw words column k is the 16-bit lane k % 2 of word k / 2
    const unsigned int cm = ((colmask & 1u) ? 0x000000ffu : 0u) | ((colmask & 2u) ? 0x0000ff00u : 0u) |
                            ((colmask & 4u) ? 0x00ff0000u : 0u) | ((colmask & 8u) ? 0xff000000u : 0u);
    // the line before the block's first (its lag-sum partner) is a batch of its own, so every
    // following batch holds kStatsBatch counted lines
    for (int yg = ys, ye = (ys < y0 ? y0 : (ys + kStatsBatch < y1 ? ys + kStatsBatch : y1)); yg < y1;
         yg = ye, ye = (ye + kStatsBatch < y1 ? ye + kStatsBatch : y1)) {
        // loads only in this loop (nothing consumes them), so all kStatsBatch lines are in flight
        uint2 w[kStatsBatch];
        unsigned int fbv[kStatsBatch];
        bool vec[kStatsBatch];
#pragma unroll
        for (int u = 0; u < kStatsBatch; ++u) {
            const int y = yg + u;
            w[u] = make_uint2(0u, 0u);
            fbv[u] = 0u;
            vec[u] = false;
            if (y < ye) {
                const int off = sm->off[y - ys];
                const int i = x0 - off;
                if (i >= 0 && i + 4 <= a.spl) {
                    // the whole 8-byte window is inside the record
                    w[u] = *reinterpret_cast<const uint2*>(base + static_cast<long long>(y) * a.line_bytes - 2ll * off);
                    fbv[u] = colbits;
                    vec[u] = true;
                } else {
                    // record edge: sample by sample
                    const uint8_t* row = a.raw + static_cast<long long>(y) * a.line_bytes;
                    for (int k = 0; k < 4; ++k) {
                        if (!((colbits >> k) & 1u) || i + k < 0 || i + k >= a.spl) continue;
                        const unsigned int v = *reinterpret_cast<const uint16_t*>(row + 2ll * (i + k));
                        if (k < 2) w[u].x |= v << (16 * k);
                        else w[u].y |= v << (16 * (k - 2));
                        fbv[u] |= 1u << k;
                    }
                }
            }
        }
        // Interior batch: every line and the one before it counted, filled and read through a
        // whole window.  The group's I and Q bytes are packed into one word each, so every sum
        // is one byte-lane dot product and nothing is masked per line.
        bool interior = ye - yg == kStatsBatch && pfb == colbits;
#pragma unroll
        for (int u = 0; u < kStatsBatch; ++u) interior = interior && vec[u];
        if (interior) {
            unsigned int pI = byte_perm(pI0, pI1, 0x6420u), pQ = byte_perm(pQ0, pQ1, 0x6420u);
            unsigned int psI = dp4(pI, kOnes, 0u), psQ = dp4(pQ, kOnes, 0u);
#pragma unroll
            for (int u = 0; u < kStatsBatch; ++u) {
                const unsigned int I = byte_perm(w[u].x, w[u].y, 0x6420u) & cm;
                const unsigned int Q = byte_perm(w[u].x, w[u].y, 0x7531u) & cm;
                const unsigned int sI = dp4(I, kOnes, 0u), sQ = dp4(Q, kOnes, 0u);
                si += sI;
                sq += sQ;
                sii = dp4(I, I, sii);
                sqq = dp4(Q, Q, sqq);
                siq = dp4(I, Q, siq);
                l1 += psI;
                l2 += psQ;
                l3 += sI;
                l4 += sQ;
                l5 = dp4(pI, I, l5);
                l6 = dp4(pQ, Q, l6);
                l7 = dp4(pI, Q, l7);
                l8 = dp4(pQ, I, l8);
                pI = I, pQ = Q, psI = sI, psQ = sQ;
            }
            cnt += static_cast<unsigned int>(kStatsBatch * ncol);
            l0 += static_cast<unsigned int>(kStatsBatch * ncol);
            // back to the two-word form the general loop carries (I or Q bytes in lanes 0 and 2)
            pI0 = byte_perm(pI, 0u, 0x4140u), pI1 = byte_perm(pI, 0u, 0x4342u);
            pQ0 = byte_perm(pQ, 0u, 0x4140u), pQ1 = byte_perm(pQ, 0u, 0x4342u);
            continue;
        }
#pragma unroll
        for (int u = 0; u < kStatsBatch; ++u) {
            const int y = yg + u;
            if (y >= ye) break;
            const unsigned int fb = fbv[u];
            const unsigned int m0 = ((fb & 1u) ? 0x0000ffffu : 0u) | ((fb & 2u) ? 0xffff0000u : 0u);
            const unsigned int m1 = ((fb & 4u) ? 0x0000ffffu : 0u) | ((fb & 8u) ? 0xffff0000u : 0u);
            const unsigned int c0 = w[u].x & m0, c1 = w[u].y & m1;
            const unsigned int I0 = c0 & kLo, I1 = c1 & kLo;
            const unsigned int Q0 = (c0 >> 8) & kLo, Q1 = (c1 >> 8) & kLo;
            if (y >= y0) {
                cnt += static_cast<unsigned int>(popc_u32(fb));
                si = dp4(I0, kOnes, dp4(I1, kOnes, si));
                sq = dp4(Q0, kOnes, dp4(Q1, kOnes, sq));
                sii = dp4(I0, I0, dp4(I1, I1, sii));
                sqq = dp4(Q0, Q0, dp4(Q1, Q1, sqq));
                siq = dp4(I0, Q0, dp4(I1, Q1, siq));
                if (y > 0) {
                    // pairs (y-1, y) with both samples filled
                    const unsigned int pb = fb & pfb;
                    if (pb == fb && pb == pfb) {
                        l1 = dp4(pI0, kOnes, dp4(pI1, kOnes, l1));
                        l2 = dp4(pQ0, kOnes, dp4(pQ1, kOnes, l2));
                        l3 = dp4(I0, kOnes, dp4(I1, kOnes, l3));
                        l4 = dp4(Q0, kOnes, dp4(Q1, kOnes, l4));
                    } else {
                        const unsigned int n0 = ((pb & 1u) ? 0x000000ffu : 0u) | ((pb & 2u) ? 0x00ff0000u : 0u);
                        const unsigned int n1 = ((pb & 4u) ? 0x000000ffu : 0u) | ((pb & 8u) ? 0x00ff0000u : 0u);
                        l1 = dp4(pI0 & n0, kOnes, dp4(pI1 & n1, kOnes, l1));
                        l2 = dp4(pQ0 & n0, kOnes, dp4(pQ1 & n1, kOnes, l2));
                        l3 = dp4(I0 & n0, kOnes, dp4(I1 & n1, kOnes, l3));
                        l4 = dp4(Q0 & n0, kOnes, dp4(Q1 & n1, kOnes, l4));
                    }
                    l0 += static_cast<unsigned int>(popc_u32(pb));
                    // products vanish wherever either sample is unfilled (its bytes are zero)
                    l5 = dp4(pI0, I0, dp4(pI1, I1, l5));
                    l6 = dp4(pQ0, Q0, dp4(pQ1, Q1, l6));
                    l7 = dp4(pI0, Q0, dp4(pI1, Q1, l7));
                    l8 = dp4(pQ0, I0, dp4(pQ1, I1, l8));
                }
            }
            pI0 = I0, pI1 = I1, pQ0 = Q0, pQ1 = Q1, pfb = fb;
        }
    }
    mv[0] = cnt, mv[1] = si, mv[2] = sq, mv[3] = sii, mv[4] = sqq, mv[5] = siq;
    lv[0] = l0, lv[1] = l1, lv[2] = l2, lv[3] = l3, lv[4] = l4, lv[5] = l5, lv[6] = l6, lv[7] = l7, lv[8] = l8;
}

ASARF_HD ASARF_INLINE void raw_stats_body(const RawStatsArgs& a, int bx, int by, int tid, int nthr,
                                          RawStatsSmem* sm) {
    unsigned long long* flat = &sm->mom[0];
    const int nflat = 6 + a.nblk * 9;
    for (int i = tid; i < 6 + kMaxDcBlocks * 9; i += nthr) flat[i] = 0ull;
    const int y0 = by * a.lines_per_cta;
    const int y1 = (y0 + a.lines_per_cta < a.na) ? y0 + a.lines_per_cta : a.na;
    const int ys = y0 > 0 ? y0 - 1 : 0;
    for (int y = ys + tid; y < y1; y += nthr) sm->off[y - ys] = a.swst ? 4 * (static_cast<int>(a.swst[y]) - a.min_swst) : 0;
    ASARF_SYNC();
    const FastDiv dstep = make_fastdiv(static_cast<unsigned int>(a.dc_step));
    const FastDiv dgpb = make_fastdiv(static_cast<unsigned int>(a.gpb));
    for (int c = tid; c < kStatsCols; c += nthr) {
        const int unit = bx * kStatsCols + c;
        unsigned long long mv[6] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
        unsigned int lv[9] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
        bool valid;
        int blk;
        if (a.quad) {
            // group k of Doppler block blk: the aligned group at (block start & ~3) + 4k, the
            // block's columns [xs, xe) in it
            blk = static_cast<int>(fdiv_u(static_cast<unsigned int>(unit), dgpb));
            const int xs = blk * a.dc_step;
            const int xe = (blk + 1) * a.dc_step < a.nr ? (blk + 1) * a.dc_step : a.nr;
            const int x0 = (xs & ~3) + 4 * (unit - blk * a.gpb);
            const int c_lo = xs > x0 ? xs - x0 : 0;
            const int c_hi = xe - x0 < 4 ? xe - x0 : 4;
            valid = blk < a.nblk && c_hi > c_lo;
            const unsigned int colmask = valid ? ((1u << c_hi) - 1u) & ~((1u << c_lo) - 1u) : 0u;
            if (valid) raw_stats_quad(a, sm, x0, colmask, y0, y1, ys, mv, lv);
        } else {
            valid = unit < a.nr;
            blk = valid ? static_cast<int>(fdiv_u(static_cast<unsigned int>(unit), dstep)) : 0;
            if (valid) raw_stats_column(a, sm, unit, y0, y1, ys, mv, lv);
        }
        raw_stats_reduce(sm, valid, blk, mv, lv);
    }
    ASARF_SYNC();
    unsigned long long* gflat = &a.acc->mom[0];
    for (int i = tid; i < nflat; i += nthr) {
        const unsigned long long v = flat[i];
        if (v) atomic_add_u64(gflat + i, v);
    }
}

// ----------------------------------------------------------------------------- FBAQ4 records
// ENVISAT ASAR raw records (ConvertAsarImBlocksToComplexKernel,
// envisat_format/src/envisat_format_kernels.cu:160-209): a 2-byte little-endian length L of
// the block data, then 64-byte blocks of one block-id byte and 63 codeword bytes (I code in
// the high nibble, Q code in the low one).  Sample r of a record is codeword byte
// j = r + r / 63 + 1 of the block data and exists when j < L (and j lies inside the record).

// Instrument-file table index of a 4-bit code of block `block`: sign-magnitude codes 0..7 are
// levels 8..15, codes 8..15 levels 7..0 (Fbaq4IndexCalc, envisat_format/include/envisat_parse_util.cuh:75-84).
ASARF_HD ASARF_INLINE int fbaq4_index(int block, int code) { return 256 * (code > 7 ? 15 - code : 8 + code) + block; }

// Usable block-data bytes of a record: its length field, bounded by the record stride.
ASARF_HD ASARF_INLINE int fbaq_len(const uint8_t* rec, long long line_bytes) {
    const int len = rec[0] | (rec[1] << 8);
    const long long room = line_bytes - 2;
    return len < room ? len : static_cast<int>(room);
}

// Sample r >= 0 of a record through the permuted tables lut[16 * block id + code].
ASARF_HD ASARF_INLINE bool fbaq_sample(const uint8_t* rec, int len, int r, const FastDiv& d63,
                                       const float* __restrict__ lut_i, const float* __restrict__ lut_q, float* iv,
                                       float* qv) {
    const int b = static_cast<int>(fdiv_u(static_cast<unsigned int>(r), d63));
    const int j = r + b + 1;
    if (j >= len) return false;
    const int id = rec[2 + 64 * b];
    const int cw = rec[2 + j];
    *iv = ASARF_LDG(lut_i + 16 * id + (cw >> 4));
    *qv = ASARF_LDG(lut_q + 16 * id + (cw & 15));
    return true;
}

// Statistics of FBAQ4 records: the sums of k_raw_stats over the decoded float samples, in
// FP64.  Tile (bx, by) = 32 columns x kFbaqStatsLines lines; warp w of the block takes lines
// [y0 + w * sub, y0 + (w + 1) * sub) of the tile, lane = column.  Per-lane sums are combined
// over the warps, then over the lanes (moments: fixed pairwise tree; lag sums: per Doppler
// block in lane order), and the tile's partials are written, not accumulated: the fold sums
// them in a fixed order, so the statistics do not depend on scheduling.
constexpr int kFbaqSums = 15;  // 6 moments + 9 lag sums
constexpr int kFoldTree = 256; // leaves of the moment tree of the fold (column tiles wrap onto them)
struct FbaqStatsSmem {
    int off[kFbaqStatsLines + 1];  // SWST shift of the tile's lines (and the line before)
    int len[kFbaqStatsLines + 1];  // usable block-data bytes of those records
    double red[kFbaqStatsWarps][kFbaqSums][32];
};

ASARF_HD ASARF_INLINE void raw_stats_fbaq_body(const RawStatsArgs& a, int bx, int by, int tid, int nthr,
                                               FbaqStatsSmem* sm) {
    const int y0 = by * kFbaqStatsLines;
    const int y1 = (y0 + kFbaqStatsLines < a.na) ? y0 + kFbaqStatsLines : a.na;
    const int ys = y0 > 0 ? y0 - 1 : 0;
    for (int y = ys + tid; y < y1; y += nthr) {
        sm->off[y - ys] = a.swst ? static_cast<int>(a.swst[y]) - a.min_swst : 0;
        sm->len[y - ys] = fbaq_len(a.raw + static_cast<long long>(y) * a.line_bytes, a.line_bytes);
    }
    ASARF_SYNC();
    const FastDiv d63 = make_fastdiv(63u);
    constexpr int sub = kFbaqStatsLines / kFbaqStatsWarps;
    for (int t = tid; t < 32 * kFbaqStatsWarps; t += nthr) {
        const int lane = t & 31, w = t >> 5;
        const int x = bx * 32 + lane;
        const int wy0 = y0 + w * sub;
        const int wy1 = (wy0 + sub < y1) ? wy0 + sub : y1;
        double v[kFbaqSums];
#pragma unroll
        for (int k = 0; k < kFbaqSums; ++k) v[k] = 0.0;
        float pi = 0.0f, pq = 0.0f;
        bool pf = false;
        const int start = wy0 > 0 ? wy0 - 1 : 0;
        if (x < a.nr && wy0 < wy1) {
            for (int yb = start; yb < wy1; yb += kStatsBatch) {
                float iv[kStatsBatch], qv[kStatsBatch];
                bool f[kStatsBatch];
                // branch-free batch: an absent sample reads byte 0 of its record's block data
                // (inside the record: every record holds at least one block byte) and is masked
#pragma unroll
                for (int u = 0; u < kStatsBatch; ++u) {
                    const int y = yb + u < wy1 ? yb + u : wy1 - 1;
                    const int r = x - sm->off[y - ys];
                    const int rr = r > 0 ? r : 0;
                    const int b = static_cast<int>(fdiv_u(static_cast<unsigned int>(rr), d63));
                    const int j = rr + b + 1;
                    f[u] = (yb + u < wy1) && r >= 0 && j < sm->len[y - ys];
                    const uint8_t* rec = a.raw + static_cast<long long>(y) * a.line_bytes + 2;
                    const int id = rec[f[u] ? 64 * b : 0];
                    const int cw = rec[f[u] ? j : 0];
                    iv[u] = ASARF_LDG(a.lut_i + 16 * id + (cw >> 4));
                    qv[u] = ASARF_LDG(a.lut_q + 16 * id + (cw & 15));
                }
#pragma unroll
                for (int u = 0; u < kStatsBatch; ++u) {
                    const int y = yb + u;
                    if (y >= wy1) break;
                    const double ci = f[u] ? iv[u] : 0.0, cq = f[u] ? qv[u] : 0.0;
                    if (y >= wy0 && f[u]) {
                        v[0] += 1.0;
                        v[1] += ci;
                        v[2] += cq;
                        v[3] += ci * ci;
                        v[4] += cq * cq;
                        v[5] += ci * cq;
                        if (y > 0 && pf) {
                            const double ai = pi, aq = pq;
                            v[6] += 1.0;
                            v[7] += ai;
                            v[8] += aq;
                            v[9] += ci;
                            v[10] += cq;
                            v[11] += ai * ci;
                            v[12] += aq * cq;
                            v[13] += ai * cq;
                            v[14] += aq * ci;
                        }
                    }
                    pi = f[u] ? iv[u] : 0.0f;
                    pq = f[u] ? qv[u] : 0.0f;
                    pf = f[u];
                }
            }
        }
#pragma unroll
        for (int k = 0; k < kFbaqSums; ++k) sm->red[w][k][lane] = v[k];
    }
    ASARF_SYNC();
    // over the warps, in warp order (into warp 0's row)
    for (int t = tid; t < kFbaqSums * 32; t += nthr) {
        const int k = t >> 5, lane = t & 31;
        double acc = sm->red[0][k][lane];
        for (int w = 1; w < kFbaqStatsWarps; ++w) acc += sm->red[w][k][lane];
        sm->red[0][k][lane] = acc;
    }
    ASARF_SYNC();
    double* out = a.part + (static_cast<long long>(by) * a.tiles_x + bx) * a.part_slots;
    const int b0 = static_cast<int>((bx * 32) / a.dc_step);
    // lag sums: per Doppler block, lanes in order (before the moment tree reuses the row)
    for (int t = tid; t < 9 * a.span; t += nthr) {
        const int bl = t / 9, q = t - bl * 9;
        double acc = 0.0;
        for (int lane = 0; lane < 32; ++lane) {
            const int x = bx * 32 + lane;
            if (x < a.nr && x / a.dc_step == b0 + bl) acc += sm->red[0][6 + q][lane];
        }
        out[6 + t] = acc;
    }
    ASARF_SYNC();
    // moments: pairwise tree over the 32 lanes
    for (int h = 16; h > 0; h >>= 1) {
        for (int t = tid; t < 6 * h; t += nthr) {
            const int k = t / h, lane = t - k * h;
            sm->red[0][k][lane] += sm->red[0][k][lane + h];
        }
        ASARF_SYNC();
    }
    for (int k = tid; k < 6; k += nthr) out[k] = sm->red[0][k][0];
}

// Fold of the FBAQ4 partials into FloatStatAccum: over the line tiles of every
// column tile, then over the column tiles touching each sum, both in index order.
ASARF_HD ASARF_INLINE void stats_fold_body(const RawStatsArgs& a, int tiles_y, int tid, int nthr, double* tree) {
    const int slots = a.part_slots;
    for (int t = tid; t < a.tiles_x * slots; t += nthr) {
        double acc = a.part[t];
        for (int by = 1; by < tiles_y; ++by) acc += a.part[static_cast<long long>(by) * a.tiles_x * slots + t];
        a.part[t] = acc;
    }
    ASARF_SYNC();
    // moments: pairwise tree over the column tiles (tree holds 6 x kFoldTree doubles)
    for (int t = tid; t < 6 * kFoldTree; t += nthr) {
        const int m = t / kFoldTree, bx = t - m * kFoldTree;
        double acc = 0.0;
        for (int k = bx; k < a.tiles_x; k += kFoldTree) acc += a.part[k * slots + m];
        tree[t] = acc;
    }
    ASARF_SYNC();
    for (int h = kFoldTree / 2; h > 0; h >>= 1) {
        for (int t = tid; t < 6 * h; t += nthr) {
            const int m = t / h, i = t - m * h;
            tree[m * kFoldTree + i] += tree[m * kFoldTree + i + h];
        }
        ASARF_SYNC();
    }
    for (int t = tid; t < 6; t += nthr) a.facc->mom[t] = tree[t * kFoldTree];
    // lag sums: the few column tiles touching each Doppler block, in order
    for (int t = tid; t < 9 * a.nblk; t += nthr) {
        const int b = t / 9, q = t - 9 * b;
        const int lo = (b * a.dc_step) / 32;
        int hi = ((b + 1) * a.dc_step - 1) / 32;
        if (hi > a.tiles_x - 1) hi = a.tiles_x - 1;
        double acc = 0.0;
        for (int bx = lo; bx <= hi; ++bx) {
            const int bl = b - (bx * 32) / a.dc_step;
            if (bl >= 0 && bl < a.span) acc += a.part[bx * slots + 6 + 9 * bl + q];
        }
        a.facc->lag[b][q] = acc;
    }
}

// ----------------------------------------------------------------------------- finalisation
// Single-threaded: IQ statistics and correction constants exactly as RawDataCorrection
// derives them (sar/iq_correction.cu:200-273, CalcMean/CalcStdDev of
// cuda_util/device_padded_image.cu:331-414), the Doppler centroid per range block and its
// quadratic fit (sar/fractional_doppler_centroid.cu:98-139), and the results-window choice
// that depends on the sign of the fitted constant term (main_flow.cc:155-178).
// Constants of the corrected-sample map z = (p*I + p0, u*Q + v*I + w) and the statistics
// error bits, shared by the IQ part and the per-block Doppler part of the finalisation.
struct FinalizeMap {
    double p, p0, u, v, w, pad_mag2;
    unsigned int err;
};

// IQ statistics and the correction constants; the FocusState fields are written when st is set.
ASARF_HD inline FinalizeMap finalize_stats(const FinalizeArgs& a, FocusState* st) {
    const StatAccum& s = *a.acc;
    const FloatStatAccum* fs = a.facc;
    auto mom = [&](int k) { return fs ? fs->mom[k] : static_cast<double>(s.mom[k]); };
    const double n = mom(0);
    const double SI = mom(1), SQ = mom(2);
    const double SII = mom(3), SQQ = mom(4);
    const double SIQ = mom(5);
    FinalizeMap m;
    m.err = 0;
    if (n == 0.0) m.err |= kErrStatsEmpty;
    const float total = static_cast<float>(a.n_total);
    // mean: float(sum) / float(total)
    const float dc_i = static_cast<float>(SI) / total;
    const float dc_q = static_cast<float>(SQ) / total;
    const double di = dc_i, dq = dc_q;
    const double cii = SII - 2.0 * di * SI + n * di * di;  // sum over filled of (I - dc_i)^2
    const double cqq = SQQ - 2.0 * dq * SQ + n * dq * dq;
    const double ciq = SIQ - dq * SI - di * SQ + n * di * dq;
    // padding samples hold 0 - dc after the DC step and enter the gain / phase sums
    const double npad = static_cast<double>(a.n_pad);
    const double i1sq = cii + npad * di * di;
    const double q1sq = cqq + npad * dq * dq;
    const double i1q1 = ciq + npad * di * dq;
    const double gain = sqrt(i1sq / q1sq);
    const float gain_f = static_cast<float>(gain);
    const double gf = gain_f;
    const double delta = (i1q1 / gf) / (i1sq / (gf * gf));
    const float sin_c = static_cast<float>(delta);
    const float cos_c = static_cast<float>(1.0 - delta * delta);
    if (st) {
        st->dc_i = dc_i;
        st->dc_q = dc_q;
        st->gain = gain_f;
        st->sin_c = sin_c;
        st->cos_c = cos_c;
        st->rgain = fdiv_rn(1.0f, gain_f);
        st->rcos = fdiv_rn(1.0f, cos_c);
        st->dc_i_d = dc_i;
        st->dc_q_d = dc_q;
        st->iq_gain = gain;
        st->phase_error = 360.0 * asin(delta) / (2.0 * 3.14159265358979323846);
        st->stddev_i = sqrtf(static_cast<float>(cii) / total);
        st->stddev_q = sqrtf(static_cast<float>(cqq) / total);
    }
    // corrected sample z = (p*I + p0, u*Q + v*I + w)
    m.p = 1.0 / gf;
    m.p0 = -di / gf;
    const double sc = sin_c, cc = cos_c;
    m.u = 1.0 / cc;
    m.v = -sc * m.p / cc;
    m.w = (-dq - sc * m.p0) / cc;
    m.pad_mag2 = m.p0 * m.p0 + m.w * m.w;  // |corrected zero padding sample|^2
    return m;
}

// Doppler centroid of range block b from its lag-1 sums through the correction map.
ASARF_HD inline void finalize_block(const FinalizeArgs& a, const FinalizeMap& m, int b, double* xs, double* ys,
                                    FocusState& st) {
    const StatAccum& s = *a.acc;
    const FloatStatAccum* fs = a.facc;
    auto lag = [&](int q) { return fs ? fs->lag[b][q] : static_cast<double>(s.lag[b][q]); };
    const double p = m.p, p0 = m.p0, u = m.u, v = m.v, w = m.w;
    const double np = lag(0);
    const double sA = lag(1), sB = lag(2);
    const double sC = lag(3), sD = lag(4);
    const double sAC = lag(5), sBD = lag(6);
    const double sAD = lag(7), sBC = lag(8);
    double re = p * p * sAC + p * p0 * (sA + sC) + p0 * p0 * np + u * u * sBD + u * v * (sBC + sAD) +
                u * w * (sB + sD) + v * v * sAC + v * w * (sA + sC) + w * w * np;
    const double im = p * u * (sAD - sBC) + p * w * (sA - sC) + p0 * u * (sD - sB) + p0 * v * (sC - sA);
    const int xb = b * a.dc_step;
    const int xe = xb + a.dc_step;
    // columns of this block beyond the data lie in the range padding (constant rows)
    int pad_lo = xb > a.nr ? xb : a.nr;
    int pad_hi = xe < a.rg_stride ? xe : a.rg_stride;
    // (only when the padding went through the correction, i.e. reference statistics)
    if (a.n_pad > 0 && pad_hi > pad_lo) re += static_cast<double>(pad_hi - pad_lo) * (a.na - 1) * m.pad_mag2;
    const double ang = atan2(im, re);
    const double hz = a.prf * (ang / (2.0 * 3.14159265358979323846));
    xs[b] = static_cast<double>((xb + xe) / 2);
    ys[b] = hz;
    st.dc_blk_hz[b] = hz;
}

// Doppler polynomial fit over the blocks, the DC-sign variant and the error bits.
ASARF_HD inline void finalize_fit(const FinalizeArgs& a, FocusState& st, const double* xs, const double* ys,
                                  unsigned int err) {
    const int nblk = a.nblk < kMaxDcBlocks ? a.nblk : kMaxDcBlocks;
    if (a.nblk > kMaxDcBlocks) err |= kErrDcBlocks;
    st.nblk = nblk;
    double poly[3] = {0.0, 0.0, 0.0};
    polyfit_qr<kMaxDcBlocks, 3>(xs, ys, nblk, 2, poly);
    st.dc_est[0] = poly[0];
    st.dc_est[1] = poly[1];
    st.dc_est[2] = poly[2];
    if (a.dc_given)
        for (int k = 0; k < 3; ++k) poly[k] = a.dc_in[k];
    for (int k = 0; k < 3; ++k) {
        st.dc_poly[k] = poly[k];
        st.dc_poly32[k] = static_cast<float>(poly[k]);
    }
    st.variant = poly[2] > 0 ? 0 : 1;
    st.first_line = a.first_line[st.variant];
    st.n_lines = a.n_lines[st.variant];
    st.errors = err;
}

// The whole finalisation on one thread.
ASARF_HD inline void finalize_body(const FinalizeArgs& a) {
    FocusState& st = *a.state;
    const FinalizeMap m = finalize_stats(a, &st);
    double xs[kMaxDcBlocks], ys[kMaxDcBlocks];
    const int nblk = a.nblk < kMaxDcBlocks ? a.nblk : kMaxDcBlocks;
    for (int b = 0; b < nblk; ++b) finalize_block(a, m, b, xs, ys, st);
    finalize_fit(a, st, xs, ys, m.err);
}

// ----------------------------------------------------------------------------- range compression
// One azimuth line per block: ERS byte decode (envisat_format/src/envisat_format_kernels.cu:116-134),
// IQ correction with the reference's float operation order (sar/iq_correction.cu:140-178),
// forward FFT, chirp matched filter and inverse FFT (sar/range_compression.cu:25-107), keeping
// x < XSize - chirp_samples.  Samples the decoder leaves empty are 0 (ZeroNaNs after the
// correction, main.cc:245).  The FFT length is any L >= XSize: outputs x < Nk only correlate
// data samples [x, x + Nc) so they do not depend on L.
// The IQ correction constants of a run, copied out of the FocusState into registers before a
// line's decode loop (read through the state's pointer, they were reloaded for every sample:
// range compression 1.066 -> 0.996 ms on the ERS scene).
struct IqCorr {
    float dc_i, dc_q, gain, rgain, sin_c, cos_c, rcos;
    ASARF_HD ASARF_INLINE explicit IqCorr(const FocusState& s)
        : dc_i(s.dc_i), dc_q(s.dc_q), gain(s.gain), rgain(s.rgain), sin_c(s.sin_c), cos_c(s.cos_c), rcos(s.rcos) {}
};

ASARF_HD ASARF_INLINE float2 correct_sample_f(float iv, float qv, const IqCorr& st) {
    const float i1 = fsub_rn(iv, st.dc_i);
    const float q1 = fsub_rn(qv, st.dc_q);
    // the reference's two IEEE divisions, correctly rounded through the reciprocals
    const float i2 = div_by_recip_rn(i1, st.gain, st.rgain);
    const float q2 = div_by_recip_rn(fma_rn(-i2, st.sin_c, q1), st.cos_c, st.rcos);
    return make_float2(i2, q2);
}

ASARF_HD ASARF_INLINE float2 correct_sample(int iv, int qv, const IqCorr& st) {
    return correct_sample_f(static_cast<float>(iv), static_cast<float>(qv), st);
}

// Corrected sample at range position l of line y (FMT: RawFormat; row: the line's record).
template <int FMT>
struct LineDecoder {
    int off, len;
    FastDiv d63;
    const uint8_t* row;
    ASARF_HD ASARF_INLINE LineDecoder(const RangeCompressArgs& a, int y, const uint8_t* raw_line) {
        row = raw_line ? raw_line : a.raw + static_cast<long long>(y) * a.line_bytes;
        if constexpr (FMT == kRawAsarFbaq4) {
            off = a.swst ? static_cast<int>(a.swst[y]) - a.min_swst : 0;
            len = fbaq_len(row, a.line_bytes);
            d63 = make_fastdiv(63u);
        } else {
            off = a.swst ? 4 * (static_cast<int>(a.swst[y]) - a.min_swst) : 0;
            len = 0;
        }
    }
    ASARF_HD ASARF_INLINE float2 operator()(const RangeCompressArgs& a, const IqCorr& st, int l) const {
        float2 z = make_float2(0.0f, 0.0f);
        const int i = l - off;
        if constexpr (FMT == kRawAsarFbaq4) {
            float iv, qv;
            if (l < a.nr && i >= 0 && fbaq_sample(row, len, i, d63, a.lut_i, a.lut_q, &iv, &qv))
                z = correct_sample_f(iv, qv, st);
        } else {
            if (l < a.nr && i >= 0 && i < a.spl) {
                const uint16_t wv = *reinterpret_cast<const uint16_t*>(row + 2ll * i);
                z = correct_sample(wv & 0xff, wv >> 8, st);
            }
        }
        return z;
    }
};

template <int FMT = kRawErsBytes>
ASARF_HD ASARF_INLINE void range_compress_body(const RangeCompressArgs& a, int y, int tid, int nthr, float2* s,
                                               const uint8_t* raw_line) {
    const IqCorr st(*a.state);
    const int L = a.plan.n;
    const LineDecoder<FMT> dec(a, y, raw_line);
    for (int l = tid; l < L; l += nthr) s[l] = dec(a, st, l);
    ASARF_SYNC();
    fft_forward(a.plan, s, 1, 1, tid, nthr);
    for (int l = tid; l < L; l += nthr) s[l] = cmul(s[l], ASARF_LDG(a.mf + l));
    ASARF_SYNC();
    fft_inverse(a.plan, s, 1, 1, tid, nthr);
    float2* orow = a.out + static_cast<long long>(y) * a.out_pitch;
    for (int l = tid; l < a.nk; l += nthr) orow[l] = s[l];
}

// Compressed line store of the compile-time transform: sample x < nk to orow[x].
struct RcOut {
    static constexpr bool kActive = true;
    float2* orow;
    int nk;
    ASARF_HD ASARF_INLINE void operator()(int x, float2 v) const {
        if (x < nk) orow[x] = v;
    }
};

// Same transform with a compile-time schedule (lengths in kCtLengths): all loops unrolled,
// all index arithmetic constant.
template <int L, int FMT = kRawErsBytes>
ASARF_HD ASARF_INLINE void range_compress_ct_body(const RangeCompressArgs& a, int y, int tid, float2* s,
                                                  const uint8_t* raw_line) {
    constexpr int NTHR = CtSchedule<L>::nthr;
    constexpr int PER = (L + NTHR - 1) / NTHR;
    const IqCorr st(*a.state);
    const LineDecoder<FMT> dec(a, y, raw_line);
    ct_phase<NTHR>(
        [&](int t) {
#pragma unroll
            for (int k = 0; k < PER; ++k) {
                const int l = t + k * NTHR;
                if (L % NTHR != 0 && l >= L) break;
                s[ct_pad<L>(l)] = dec(a, st, l);
            }
        },
        tid);
    // the last inverse pass stores the kept samples x < Nk of the line directly
    ct_fft_mf_ifft<L>(s, a.ctw, a.mf, tid, RcOut{a.out + static_cast<long long>(y) * a.out_pitch, a.nk});
}

// ----------------------------------------------------------------------------- azimuth strided pass
// Four-step azimuth FFT of length N = n1 * n2 along the rows of a [N][pitch] block, columns
// [x0, x0 + xt).  Time index n = a*n2 + b, frequency k = k1 + n1*k2.
//  forward (block b): Y[k1][b] = W_N^{b k1} * FFT_n1(x[a*n2 + b])[k1], stored at row k1*n2 + b.
//  inverse (block b): x[a*n2 + b] = IFFT_n1(conj(W_N^{b k1}) * Z[k1][b])[a] * scale.
// Both read their rows in natural order (one strided tile, TMA-loaded on the device) and
// write the digit-reversed transform output straight to its destination rows.
// Together with the contiguous pass this is the transpose-free equivalent of the reference's
// transpose + batched row FFT + transpose (sar/range_doppler_algorithm.cu:314-326, 381-391).
// Per-block tables of the strided pass, staged in shared memory while the tile is in flight:
// tw[p] = W_N^{b * k1} and row[p] = destination row, for transform position p (forward:
// k1 = drev1(p), digit-reversed output; inverse: tw indexed by the natural input row k1 = p,
// row by the digit-reversed output position).  b * k1 < N, so no reduction is needed.
ASARF_HD ASARF_INLINE void az_strided_tables(const AzStridedArgs& a, int b, int tid, int nthr, float2* tw, int* row) {
    for (int p = tid; p < a.n1; p += nthr) {
        const int kd = ASARF_LDG(a.drev1 + p);
        tw[p] = ASARF_LDG(a.twn + b * (a.inverse ? p : kd));
        row[p] = kd * a.n2 + b;
    }
}

// Store of a column pair (u at column x, v at x + 1) of one output row: one 16-byte store when
// both columns exist and the address allows it.
ASARF_HD ASARF_INLINE void store_pair(float2* dst, int x, int nk, float2 u, float2 v) {
    if (x + 1 < nk && (reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
        *reinterpret_cast<float4*>(dst) = make_float4(u.x, u.y, v.x, v.y);
    } else {
        dst[0] = u;
        if (x + 1 < nk) dst[1] = v;
    }
}

// R0, R1, R2, XT > 0: the transform's radix schedule and tile width as compile-time constants
// (they must be the plan's: the planner picks this instantiation only when they are).
template <int R0 = 0, int R1 = 0, int R2 = 0, int XT = 0>
ASARF_HD ASARF_INLINE void az_strided_body(const AzStridedArgs& a, int tile, int b, int tid, int nthr, float2* s,
                                           const float2* tw, const int* rowmap, bool preloaded) {
    constexpr bool kCt = R0 > 0;
    const int n1 = kCt ? R0 * R1 * R2 : a.n1, xt = kCt ? XT : a.xt;
    const int x0 = tile * xt;
    const FastDiv dxt = make_fastdiv(static_cast<unsigned int>(xt));
    // position t of the tile -> row (t / xt), by a constant when the schedule is compiled
    auto row_of = [&](int t) { return kCt ? t / XT : static_cast<int>(fdiv_u(t, dxt)); };
    // tile [r][c] = row r*n2 + b, column x0 + c (natural order; columns >= nk read as 0)
    if (!preloaded) {
        for (int t = tid; t < n1 * xt; t += nthr) {
            const int r = row_of(t), c = t - r * xt;
            const int row = r * a.n2 + b;
            const int x = x0 + c;
            float2 v = make_float2(0.0f, 0.0f);
            if (row < a.valid_rows && x < a.nk) v = a.in[static_cast<long long>(row) * a.pitch + x];
            s[t] = v;
        }
    } else if (a.valid_rows < n1 * a.n2) {
        // rows past the data hold stale values in memory: they are zero by definition
        const int r0 = (a.valid_rows - b + a.n2 - 1) / a.n2;
        for (int t = r0 * xt + tid; t < n1 * xt; t += nthr) s[t] = make_float2(0.0f, 0.0f);
    }
    ASARF_SYNC();
    if (!a.inverse) {
        // (writing the last stage straight to HBM, as the range-Doppler block does, measured
        // slower here: its rows scatter through the digit-reversed row map)
        if constexpr (R0 > 0)
            fft_forward_pairs_ct3<R0, R1, R2, XT / 2, XT, true>(s, a.plan1.tw, tid, nthr);
        else
            fft_forward_pairs<true, true>(a.plan1, s, xt, xt, tid, nthr);
        for (int t = tid; t < n1 * xt; t += nthr) {
            const int p = row_of(t), c = t - p * xt;
            const int x = x0 + c;
            if (x < a.nk) a.out[static_cast<long long>(rowmap[p]) * a.pitch + x] = cmul(s[t], tw[p]);
        }
    } else {
        // conj(twiddle) of row k1 applied as the first stage loads the row
        if constexpr (R0 > 0)
            fft_inverse_dif_pairs_ct3<R0, R1, R2, XT / 2, XT, true>(s, a.plan1.tw, tid, nthr, tw);
        else
            fft_inverse_dif_pairs<true, true>(a.plan1, s, xt, xt, tid, nthr, tw);
        const int lo = a.state ? a.state->first_line : 0;
        const int hi = a.state ? lo + a.state->n_lines : n1 * a.n2;
        for (int t = tid; t < n1 * xt; t += nthr) {
            const int p = row_of(t), c = t - p * xt;
            const int row = rowmap[p];
            const int x = x0 + c;
            if (x < a.nk && row >= lo && row < hi) {
                const float2 v = s[t];
                const float2 u = make_float2(fmul_rn(v.x, a.scale), fmul_rn(v.y, a.scale));
                const long long o = static_cast<long long>(row - a.out_row0) * a.pitch + x;
                if (a.out_intensity)
                    a.out_intensity[o] = fma_rn(u.x, u.x, fmul_rn(u.y, u.y));  // the tail's |z|^2, same rounding
                else
                    a.out[o] = u;
            }
        }
    }
}

// Shared-memory bytes of the strided pass: tile, twiddle table, row table.
inline size_t az_strided_smem(int n1, int xt) {
    return sizeof(float2) * static_cast<size_t>(n1) * xt + sizeof(float2) * n1 + sizeof(int) * n1;
}

// ----------------------------------------------------------------------------- range-Doppler block
// Block (tile, k1): rows k1*n2 .. k1*n2 + n2 - 1 of the strided-pass output, output columns
// [x0, x0 + xt) plus a range halo (hl left, hr right) for the interpolator.
//   1. contiguous forward FFT_n2 -> range-Doppler rows, frequency bin k1 + n1*drev2(p);
//   2. RCMC: 16-tap Blackman-windowed sinc at the parabolic range walk
//      (RangeCellMigrationCorrection, sar/range_doppler_algorithm.cu:107-195);
//   3. azimuth matched filter with Doppler-centroid band cut and linear phase ramp
//      (AzimuthReferenceMultiply, sar/range_doppler_algorithm.cu:197-309);
//   4. contiguous inverse FFT_n2 of the xt output columns.
// Both use the reference's float32 operation order for every branch-deciding quantity.
ASARF_HD ASARF_INLINE ColParams az_col_params(const AzRdArgs& a, int x) {
    ColParams cp;
    const float xf = static_cast<float>(x);
    float dcp[3] = {a.state->dc_poly32[0], a.state->dc_poly32[1], a.state->dc_poly32[2]};
    float vrp[3] = {a.vr_poly[0], a.vr_poly[1], a.vr_poly[2]};
    cp.dc = polyval_f32(dcp, xf);
    const float vr = polyval_f32(vrp, xf);
    const float step = a.bin_step;
    const float dc_steps = roundf(fdiv_rn(cp.dc, step));
    cp.dc_off = fmul_rn(dc_steps, step);
    const double r0 = a.slant + static_cast<double>(x) * a.range_spacing;
    cp.r0_dr = r0 / a.range_spacing;
    const float kav = fmul_rn(fmul_rn(2.0f, vr), vr);
    cp.ka = static_cast<float>(static_cast<double>(kav) / (static_cast<double>(a.lambda) * r0));
    const float half = fmul_rn(a.prf, 0.5f);
    cp.cut_hi = fma_rn(half, a.frac, cp.dc_off);
    cp.cut_lo = fma_rn(-half, a.frac, cp.dc_off);
    cp.den = fmul_rn(fmul_rn(8.0f, vr), vr);
    cp.dc_off_ka = fdiv_rn(cp.dc_off, cp.ka);
    cp.rden = fdiv_rn(1.0f, cp.den);
    cp.rka = fdiv_rn(1.0f, cp.ka);
    cp.pad = 0.0f;
    return cp;
}

ASARF_HD ASARF_INLINE float bin_frequency(int f, int az_pad, float step) {
    const int k = (f < az_pad / 2) ? f : f - az_pad;
    return fmul_rn(static_cast<float>(k), step);
}

// bf: the row's Doppler bin frequency (bin_frequency of its bin, from the block's row table).
ASARF_HD ASARF_INLINE float2 rcmc_mf_sample(const AzRdArgs& a, const ColParams& cp, int x, float bf, const float2* srow,
                                            int cs, unsigned int* err_flag) {
    const float prf = a.prf;
    const float half = a.half_prf;
    // --- aliased frequency (the same test decides the matched-filter band and the RCMC walk)
    float fn = bf;
    if (cp.dc < 0.0f) {
        if (bf > fadd_rn(half, cp.dc)) fn = fsub_rn(fn, prf);
    } else if (cp.dc > 0.0f) {
        if (fn < fadd_rn(-half, cp.dc)) fn = fadd_rn(fn, prf);
    }
    // outside the processed band the reference writes zero whatever RCMC gave
    if (fn < cp.cut_lo || fn > cp.cut_hi) return make_float2(0.0f, 0.0f);
    // --- RCMC: walk = lambda^2 fn^2 / (8 Vr^2) [float, IEEE divide] * R0 [double] / range spacing
    const float num = fmul_rn(fmul_rn(fmul_rn(a.lambda, a.lambda), fn), fn);
    const float shift = static_cast<float>(static_cast<double>(div_by_recip_rn(num, cp.den, cp.rden)) * cp.r0_dr);
    const int walk = static_cast<int>(roundf(shift));
    const int calc_x = x + walk;
    float2 out = make_float2(0.0f, 0.0f);
    if (!(calc_x - kRcmcTaps / 2 < 0 || calc_x + kRcmcTaps / 2 >= a.nk)) {
        const int first = cs + walk - kRcmcTaps / 2;  // smem column of tap 0
        if (first + 1 < 0 || first + kRcmcTaps - 1 > a.wt) {
            atomic_or_u32(err_flag, kErrRcmcHalo);
        } else {
            // Windowed sinc at off - i, off = shift - walk + 8 in [7.5, 8.5]:
            // sin(pi (off - i)) = (-1)^i sin(pi off), and the common factor sin(pi off) / pi
            // cancels in the normalised sum, leaving weights (-1)^i W_i / (off - i).  The two end
            // taps are skipped: their window values W_0 = W_15 = -1.4e-17 (a numpy.blackman
            // rounding residue of an exact zero) give terms below half an ulp of every sum.
            // With dl = off - 8 (exact) a weight is 1 / fma(dl, c_i, (8 - i) c_i), c_i = (-1)^i / W_i
            // (constants): one FMA and one reciprocal per tap, within 2 ulp of the quotient since
            // |8 - i| >= 1 wherever the constant term is not zero.  The normaliser sums in pairs.
            const float off = fadd_rn(fsub_rn(shift, static_cast<float>(walk)), static_cast<float>(kRcmcTaps / 2));
            const float dl = fsub_rn(off, static_cast<float>(kRcmcTaps / 2));
            if (dl == 0.0f) {
                out = srow[first + kRcmcTaps / 2];  // integer shift: sinc is a unit impulse
            } else {
                constexpr float kWin[kRcmcTaps] = ASARF_BLACKMAN16;
                float2 acc = make_float2(0.0f, 0.0f);
                float2 nrm2 = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int i = 1; i < kRcmcTaps - 1; i += 2) {
                    const float ca = -1.0f / kWin[i];  // i odd
                    const float cb = 1.0f / kWin[i + 1];
                    const float wa = rcp_approx(fma_rn(dl, ca, static_cast<float>(kRcmcTaps / 2 - i) * ca));
                    const float wb = rcp_approx(fma_rn(dl, cb, static_cast<float>(kRcmcTaps / 2 - i - 1) * cb));
                    acc = pfma(srow[first + i], wa, acc);
                    acc = pfma(srow[first + i + 1], wb, acc);
                    nrm2 = padd(nrm2, make_float2(wa, wb));
                }
                const float nrm = fadd_rn(nrm2.x, nrm2.y);
                if (nrm != 0.0f) {
                    const float inv = rcp_approx(nrm);
                    out = make_float2(fmul_rn(acc.x, inv), fmul_rn(acc.y, inv));
                }
            }
        }
    }
    // --- matched filter exp(-j pi fc^2 / Ka) * exp(-j 2 pi (dc_off / Ka) f), both phases
    // rounded as the reference rounds them, combined into one reduced exponential
    float fc = fsub_rn(bf, cp.dc_off);
    if (fc > half) fc = fsub_rn(fc, prf);
    else if (fc < -half) fc = fadd_rn(fc, prf);
    const float pi = 3.14159265358979323846f;
    const float mf_phase = div_by_recip_rn(fmul_rn(fmul_rn(pi, fc), fc), cp.ka, cp.rka);
    const float sh_phase = fmul_rn(fmul_rn(fmul_rn(2.0f, pi), cp.dc_off_ka), bf);
    return cmul(out, expj_neg_sum(mf_phase, sh_phase));
}

// Absolute-phase factor of column x: exp(j phi), phi = 4 pi R0 / lambda + pi dc_off^2 / Ka, in
// FP64 (4 pi R0 / lambda is about 1.9e8 rad at 850 km; it is reduced modulo 2 pi before the
// cast).  With it the matched filter is exp(-j pi f^2 / Ka) in the unaliased Doppler
// frequency times the removal of the carrier phase -4 pi R0 / lambda, so a point target keeps
// its own phase.  The reference has neither term (sar/range_doppler_algorithm.cu:265-290).
ASARF_HD ASARF_INLINE float2 az_abs_phase(const AzRdArgs& a, const ColParams& cp, int x) {
    const double kTwoPi = 6.283185307179586476925286766559;
    const double r0 = a.slant + static_cast<double>(x) * a.range_spacing;
    const double d = static_cast<double>(cp.dc_off);
    const double ph = fmod(fmod(2.0 * kTwoPi * r0 / a.lambda_d, kTwoPi) +
                           fmod(0.5 * kTwoPi * d * d / static_cast<double>(cp.ka), kTwoPi), kTwoPi);
    return make_float2(static_cast<float>(cos(ph)), static_cast<float>(sin(ph)));
}

// Shared-memory tables after the tile: column constants (xt), absolute-phase factors (xt),
// row bin frequencies (n2).
ASARF_HD ASARF_INLINE float2* az_rd_phase_table(ColParams* cps, const AzRdArgs& a) {
    return reinterpret_cast<float2*>(cps + a.xt);
}
ASARF_HD ASARF_INLINE float* az_rd_freq_table(ColParams* cps, const AzRdArgs& a) {
    return reinterpret_cast<float*>(az_rd_phase_table(cps, a) + a.xt);
}

// Per-block tables of the range-Doppler block, built while the tile is in flight: column
// constants of the xt output columns (and their absolute-phase factors when asked for) and
// the Doppler bin frequency of each of the n2 rows (bin k1 + n1 drev2(p)).
ASARF_HD ASARF_INLINE void az_rd_tables(const AzRdArgs& a, int tile, int k1, int tid, int nthr, ColParams* cps,
                                        float* fbf) {
    const int x0 = tile * a.xt;
    float2* phs = az_rd_phase_table(cps, a);
    for (int c = tid; c < a.xt; c += nthr) {
        cps[c] = az_col_params(a, x0 + c);
        if (a.absolute_phase) phs[c] = az_abs_phase(a, cps[c], x0 + c);
    }
    for (int p = tid; p < a.n2; p += nthr)
        fbf[p] = bin_frequency(k1 + a.n1 * ASARF_LDG(a.drev2 + p), a.az_pad, a.bin_step);
}

// Shared-memory bytes of the range-Doppler block: tile, column constants, phase factors, row frequencies.
inline size_t az_rd_smem(int n2, int wt, int xt) {
    return sizeof(float2) * static_cast<size_t>(n2) * wt + sizeof(ColParams) * static_cast<size_t>(xt) +
           sizeof(float2) * static_cast<size_t>(xt) + sizeof(float) * static_cast<size_t>(n2) + 16;
}

// Right range halo of the range-Doppler block: the taps used (1 .. 14 of 16) reach 6 columns
// right of the integer walk, which is at most ceil of the largest walk (the left halo is the
// 8 columns of tap 0, kept whole so that the tile's TMA start stays 16-byte aligned).
inline int rcmc_right_halo(double max_walk) { return kRcmcTaps / 2 - 1 + static_cast<int>(std::ceil(max_walk)); }

// Range-tile width of the range-Doppler block: the widest even width <= 64 whose block leaves
// room for two resident blocks per SM (2 x 512 threads at 64 registers fill the register file;
// 228 KB of shared memory per SM, 1 KB reserved per block).  With one block per SM the
// block-wide barriers of the FFT stages leave the SM idle (measured 2.63 -> 1.92 ms at n2 = 168).
constexpr size_t kAzRdTwoBlockSmem = 228 * 1024 / 2 - 1024 - 256;
inline int az_rd_tile_width(int n2, int hl, int hr) {
    int xt = 64;
    while (xt > 16 && az_rd_smem(n2, xt + hl + hr, xt) > kAzRdTwoBlockSmem) xt -= 2;
    return xt;
}

// Epilogue of the range-Doppler block: row r of the inverse transform, column pair cp.
struct AzRdOut {
    static constexpr bool kActive = true;
    const AzRdArgs* a;
    int x0, k1;
    ASARF_HD ASARF_INLINE void operator()(int r, int cp, float2 u, float2 v) const {
        const int x = x0 + 2 * cp;
        if (x >= a->nk) return;
        store_pair(a->out + static_cast<long long>(k1 * a->n2 + r) * a->pitch + x, x, a->nk, u, v);
    }
};

// Packed twiddle products in the range-Doppler block's n2 transforms: for schedules of radices
// <= 5 only (ERS 5 x 5 x 5: 1.483 -> 1.460 ms; ASAR IM 8 x 7 x 3 measured slower with them,
// 1.604 -> 1.683 ms).  The compiled and run-time schedules apply the same rule, so they give
// identical results.
ASARF_HD ASARF_INLINE bool az_rd_packed_twiddles(const FftPlan& p) {
    bool small = true;
    for (int i = 0; i < p.nst; ++i) small = small && p.radix[i] <= 5;
    return small;
}

// FWD = false: the caller has already put the tile through the forward transform (the
// split-precision kernel's tensor-core DFT) and synchronised.  R0, R1, R2 > 0: the n2
// transforms' radix schedule as compile-time constants (it must be the plan's).
template <bool FWD = true, int R0 = 0, int R1 = 0, int R2 = 0>
ASARF_HD ASARF_INLINE void az_rd_body(const AzRdArgs& a, int tile, int k1, int tid, int nthr, float2* s,
                                      const ColParams* cps, const float* fbf, unsigned int* err_flag, bool preloaded) {
    const int x0 = tile * a.xt;
    const int n2 = a.n2, wt = a.wt;
    const FastDiv dwt = make_fastdiv(static_cast<unsigned int>(wt));
    if (!preloaded) {
        for (int t = tid; t < n2 * wt; t += nthr) {
            const int r = static_cast<int>(fdiv_u(t, dwt)), c = t - r * wt;
            const int x = x0 - a.hl + c;
            float2 v = make_float2(0.0f, 0.0f);
            if (x >= 0 && x < a.nk) v = a.in[static_cast<long long>(k1 * n2 + r) * a.pitch + x];
            s[t] = v;
        }
    }
    if constexpr (FWD) {
        ASARF_SYNC();
        if constexpr (R0 > 0)
            fft_forward_pairs_cs3<R0, R1, R2, (R0 <= 5 && R1 <= 5 && R2 <= 5)>(s, wt, wt, a.plan2.tw, tid, nthr);
        else if (az_rd_packed_twiddles(a.plan2))
            fft_forward_pairs<false, true>(a.plan2, s, wt, wt, tid, nthr);
        else
            fft_forward_pairs<false, false>(a.plan2, s, wt, wt, tid, nthr);
    }
    // RCMC + matched filter.  Every output (row p, column c) reads taps of row p only, so a
    // row is computed into registers by one warp (lane = column, xt <= 64), the warp
    // synchronises, and writes it back in place: no block-wide barrier per row.
#if defined(__CUDA_ARCH__)
    {
        const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
        // a lane's two column records stay in registers for all rows (read from shared memory
        // per sample, the 48-byte records cost 4-way bank conflicts on every field)
        const ColParams cp0 = cps[lane < a.xt ? lane : 0], cp1 = cps[lane + 32 < a.xt ? lane + 32 : 0];
        for (int p = warp; p < n2; p += nwarps) {
            const float f = fbf[p];
            const float2* srow = s + p * wt;
            float2 v0 = make_float2(0.0f, 0.0f), v1 = make_float2(0.0f, 0.0f);
            const int c0 = lane, c1 = lane + 32;
            if (c0 < a.xt && x0 + c0 < a.nk) v0 = rcmc_mf_sample(a, cp0, x0 + c0, f, srow, a.hl + c0, err_flag);
            if (c1 < a.xt && x0 + c1 < a.nk) v1 = rcmc_mf_sample(a, cp1, x0 + c1, f, srow, a.hl + c1, err_flag);
            if (a.absolute_phase) {
                const float2* phs = az_rd_phase_table(const_cast<ColParams*>(cps), a);
                if (c0 < a.xt) v0 = cmul(v0, phs[c0]);
                if (c1 < a.xt) v1 = cmul(v1, phs[c1]);
            }
            __syncwarp();
            if (c0 < a.xt) s[p * wt + a.hl + c0] = v0;
            if (c1 < a.xt) s[p * wt + a.hl + c1] = v1;
            __syncwarp();
        }
    }
    ASARF_SYNC();
#else
    {
        float2 rowbuf[64];
        for (int p = 0; p < n2; ++p) {
            const float f = fbf[p];
            for (int c = 0; c < a.xt; ++c) {
                rowbuf[c] = (x0 + c < a.nk) ? rcmc_mf_sample(a, cps[c], x0 + c, f, s + p * wt, a.hl + c, err_flag)
                                            : make_float2(0.0f, 0.0f);
                if (a.absolute_phase) rowbuf[c] = cmul(rowbuf[c], az_rd_phase_table(const_cast<ColParams*>(cps), a)[c]);
            }
            for (int c = 0; c < a.xt; ++c) s[p * wt + a.hl + c] = rowbuf[c];
        }
    }
#endif
    // the inverse transform's last stage stores the block's rows k1 * n2 + r directly
    if constexpr (R0 > 0)
        fft_inverse_pairs_cs3<R0, R1, R2, AzRdOut, (R0 <= 5 && R1 <= 5 && R2 <= 5)>(s + a.hl, a.xt, wt, a.plan2.tw,
                                                                                   tid, nthr, AzRdOut{&a, x0, k1});
    else if (az_rd_packed_twiddles(a.plan2))
        fft_inverse_pairs<AzRdOut, true>(a.plan2, s + a.hl, a.xt, wt, tid, nthr, AzRdOut{&a, x0, k1});
    else
        fft_inverse_pairs<AzRdOut, false>(a.plan2, s + a.hl, a.xt, wt, tid, nthr, AzRdOut{&a, x0, k1});
}

// ----------------------------------------------------------------------------- ERS level-0 packets
// Line y of an ERS IM measurement data set: its packet's 11232 measurement bytes go to raw
// line y, its SWST and PRI codes (big-endian, ISP bytes 38-39 and 40-41 after the 32 bytes of
// sensing time and FEP annotation) to swst[y] / pri[y]; the FEP ISP length (11465) and the
// auxiliary section's 0xAA marker are checked as ParseErsLevel0ImPackets checks them
// (envisat_format/src/ers_im_parse.cc:423-453).  Block y, threads over 2-byte words
// (packet offsets are even: whole MDSRs of 11498 bytes).
ASARF_HD ASARF_INLINE void ers_unpack_line(const ErsUnpackArgs& a, int y, int tid, int nthr) {
    const uint8_t* pk = a.mdsr + ASARF_LDG(a.offset + y);
    const uint16_t* src = reinterpret_cast<const uint16_t*>(pk + kErsMeasurementOffset);
    uint16_t* dst = reinterpret_cast<uint16_t*>(a.raw + static_cast<long long>(y) * kErsMeasurementBytes);
    for (int i = tid; i < kErsMeasurementBytes / 2; i += nthr) dst[i] = src[i];
    if (tid == 0) {
        const int isp_len = (pk[24] << 8) | pk[25];
        unsigned e = 0;
        if (isp_len != 11465) e |= kErrL0IspLength;
        if (pk[32 + 4 + 10] != 0xAA) e |= kErrL0AuxMarker;
        if (e) atomic_or_u32(a.errors, e);
        const uint8_t* aux = pk + 32 + 4 + 10;  // 0xAA, OBRC/orbit, 4-byte OBT, activity, flags, 4-byte IF counter
        if (a.swst) a.swst[y] = static_cast<uint16_t>((aux[12] << 8) | aux[13]);
        if (a.pri) a.pri[y] = static_cast<uint16_t>((aux[14] << 8) | aux[15]);
    }
}

// Line y of an ASAR IM level-0 list: the sample blocks of its source packet (an echo packet;
// a calibration line repeats the previous line's echo, as ParseEnvisatLevel0ImPackets copies
// the previous record, envisat_format/src/envisat_im_parse.cc:599-615) become FBAQ4 record y:
// the block-data length as a little-endian uint16 (the reference's memcpy of a uint16 on a
// little-endian host), the blocks, zeros up to record_bytes.  SWST and PRI codes are the source
// packet's.  The packet's data field header length (29) and mode ID (0x54) are checked as the
// reference checks them (:470-484); a block length beyond the record sets kErrL0Length and the
// record keeps only what fits.  Block y, threads over the record's bytes.
ASARF_HD ASARF_INLINE void asar_unpack_line(const AsarUnpackArgs& a, int y, int tid, int nthr) {
    const uint8_t* pk = a.mdsr + ASARF_LDG(a.src + y);
    const int packet_length = (pk[36] << 8) | pk[37];
    int len = packet_length - 29;
    const int cap = a.record_bytes - 2;
    unsigned e = 0;
    if (((pk[38] << 8) | pk[39]) != 29) e |= kErrL0DataField;
    if (pk[41] != 0x54) e |= kErrL0Mode;
    if (len < 0 || len > cap) {
        e |= kErrL0Length;
        len = len < 0 ? 0 : cap;
    }
    uint8_t* rec = a.records + static_cast<long long>(y) * a.record_bytes;
    const uint8_t* blocks = pk + kAsarPacketHeader;
    for (int i = tid; i < a.record_bytes; i += nthr) {
        uint8_t v;
        if (i == 0) v = static_cast<uint8_t>(len & 0xFF);
        else if (i == 1) v = static_cast<uint8_t>(len >> 8);
        else v = (i - 2 < len) ? blocks[i - 2] : static_cast<uint8_t>(0);
        rec[i] = v;
    }
    if (tid == 0) {
        if (e) atomic_or_u32(a.errors, e);
        if (a.pri) a.pri[y] = static_cast<uint16_t>((pk[54] << 8) | pk[55]);
        if (a.swst) a.swst[y] = static_cast<uint16_t>((pk[56] << 8) | pk[57]);
    }
}

// ----------------------------------------------------------------------------- L1 product records
// Envisat MDS records of the level-1 products (ConditionResultsSLC / ConditionResultsDetected,
// envisat_format/src/envisat_format_kernels.cu:28-114): `hdr` zero bytes of record header, then
// the pixels.  IMS: I and Q of a complex pixel times the calibration constant, clamped to the
// int16 range and truncated toward zero (NaN gives 0), big-endian.  IMP: 10 log10 of the
// intensity times the constant, capped at 65535 and truncated to uint16 (negative, -inf and NaN
// give 0), least significant byte first as the reference kernel stores it.
ASARF_HD ASARF_INLINE int f2i_rz(float v) {
#if defined(__CUDA_ARCH__)
    return __float2int_rz(v);  // NaN -> 0
#else
    return v != v ? 0 : static_cast<int>(v);
#endif
}

ASARF_HD ASARF_INLINE unsigned int f2u_rz(float v) {
#if defined(__CUDA_ARCH__)
    return __float2uint_rz(v);  // negative, NaN -> 0
#else
    return (v != v || v <= 0.0f) ? 0u : static_cast<unsigned int>(v);
#endif
}

ASARF_HD ASARF_INLINE float log10_f32(float x) {
#if defined(__CUDA_ARCH__)
    return log10f(x);
#else
    return static_cast<float>(__builtin_log10(static_cast<double>(x)));
#endif
}

ASARF_HD ASARF_INLINE int ims_value(float v, float cal) {
    const float s = fmul_rn(v, cal);
    const float c = s > 32767.0f ? 32767.0f : (s < -32768.0f ? -32768.0f : s);
    return f2i_rz(c);
}

ASARF_HD ASARF_INLINE unsigned int imp_value(float v, float cal) {
    const float db = fmul_rn(10.0f, log10_f32(fmul_rn(v, cal)));
    return f2u_rz(65535.0f < db ? 65535.0f : db);
}

// One IMS record: row of x_size complex pixels -> dest (header + 4 bytes per pixel).
ASARF_HD ASARF_INLINE void ims_record(const float2* row, int x_size, float cal, int hdr, uint8_t* dest, int tid,
                                      int nthr) {
    for (int i = tid; i < hdr; i += nthr) dest[i] = 0;
    uint8_t* d = dest + hdr;
    for (int x = tid; x < x_size; x += nthr) {
        const float2 v = row[x];
        const int i = ims_value(v.x, cal), q = ims_value(v.y, cal);
        d[4 * x + 0] = static_cast<uint8_t>((i >> 8) & 0xff);
        d[4 * x + 1] = static_cast<uint8_t>(i & 0xff);
        d[4 * x + 2] = static_cast<uint8_t>((q >> 8) & 0xff);
        d[4 * x + 3] = static_cast<uint8_t>(q & 0xff);
    }
}

// IMP pixel x of a record payload.
ASARF_HD ASARF_INLINE void imp_store(uint8_t* payload, int x, float v, float cal) {
    const unsigned int u = imp_value(v, cal);
    payload[2 * x] = static_cast<uint8_t>(u & 0xff);
    payload[2 * x + 1] = static_cast<uint8_t>((u >> 8) & 0xff);
}

// ----------------------------------------------------------------------------- detected tail
// One output line per block: results-window subset (main_flow.cc:585-627), time-domain
// azimuth multilook (TimeDomainAzimuthLook, sar/az_multilook.cu:25-80), range spreading loss
// gain (sar/range_spreading_loss.cu:29-52) and slant-to-ground resampling with the
// reference's float Horner / IEEE division / truncation index (SrGrInterpolation,
// sar/srgr.cu:49-71).  ml holds one multilooked slant row (nx floats).
ASARF_HD ASARF_INLINE void tail_body(const TailArgs& a, int y, int tid, int nthr, float* ml, unsigned int* err_flag) {
    const FocusState& st = *a.state;
    const TailVariant& tv = a.tail[st.variant];
    if (y >= tv.out_az) return;
    const int in_y = st.n_lines;
    const float in_idx = fmul_rn(static_cast<float>(y), tv.ratio);
    const float mu = fsub_rn(in_idx, static_cast<float>(static_cast<int>(in_idx)));
    int s0 = static_cast<int>(fsub_rn(in_idx, 2.0f)), e0 = static_cast<int>(fadd_rn(in_idx, 2.0f));
    int s1 = static_cast<int>(fsub_rn(in_idx, 1.0f)), e1 = static_cast<int>(fadd_rn(in_idx, 3.0f));
    s0 = s0 > 0 ? s0 : 0;
    s1 = s1 > 0 ? s1 : 0;
    e0 = e0 < in_y ? e0 : in_y;
    e1 = e1 < in_y ? e1 : in_y;
    const int c0 = e0 > s0 ? e0 - s0 : 0;
    const int c1 = e1 > s1 ? e1 - s1 : 0;
    const float2* base = a.slc + static_cast<long long>(st.first_line) * a.pitch + a.col0;
    const float* ibase = a.intensity ? a.intensity + static_cast<long long>(st.first_line) * a.pitch + a.col0 : nullptr;
    const int r_lo = s0 < s1 ? s0 : s1;
    const int r_hi = e0 > e1 ? e0 : e1;
    // each input row is read once and added to whichever box mean(s) contain it, in row
    // order, so both sums accumulate exactly as the reference's two loops do
    // the window spans at most kTailRows rows (5, or 6 where x + 3 rounds up across a power
    // of two); all of a column's rows are loaded before any is summed, two columns at a time
    constexpr int kTailRows = 6;
    const int nr = r_hi - r_lo;
    // the box divisions and the resampling index divide by block constants: correctly rounded
    // quotients from their correctly rounded reciprocals (div_by_recip_rn)
    const float fc0 = c0 ? static_cast<float>(c0) : 1.0f, fc1 = c1 ? static_cast<float>(c1) : 1.0f;
    const float rc0 = fdiv_rn(1.0f, fc0), rc1 = fdiv_rn(1.0f, fc1);
    // |z|^2 of row r, column c: from the complex SLC, or read directly from the intensity rows
    // the inverse azimuth pass wrote for detected products (half the bytes, same rounding)
    auto power = [&](int r, int c) -> float {
        const long long o = static_cast<long long>(r) * a.pitch + c;
        if (ibase) return ibase[o];
        const float2 w = base[o];
        return fma_rn(w.x, w.x, fmul_rn(w.y, w.y));
    };
    // column c from its window rows v[0 .. kTailRows) (rows r_lo + k; later rows, when the window
    // is longer, read here): both box means, their interpolation and the range spreading loss
    auto finish = [&](int c, const float* v) {
        float sum0 = 0.0f, sum1 = 0.0f;
#pragma unroll
        for (int k = 0; k < kTailRows; ++k) {
            const int r = r_lo + k;
            if (k >= nr) break;
            if (r >= s0 && r < e0) sum0 = fadd_rn(sum0, v[k]);
            if (r >= s1 && r < e1) sum1 = fadd_rn(sum1, v[k]);
        }
        for (int r = r_lo + kTailRows; r < r_hi; ++r) {
            const float p2 = power(r, c);
            if (r >= s0 && r < e0) sum0 = fadd_rn(sum0, p2);
            if (r >= s1 && r < e1) sum1 = fadd_rn(sum1, p2);
        }
        if (c0) sum0 = div_by_recip_rn(sum0, fc0, rc0);
        if (c1) sum1 = div_by_recip_rn(sum1, fc1, rc1);
        float val = 0.0f;
        if (c0 && c1) val = fma_rn(fsub_rn(sum1, sum0), mu, sum0);
        ml[c] = fmul_rn(val, ASARF_LDG(tv.rsl + c));
    };
    // 16-byte aligned rows: four adjacent columns per thread, one 16-byte load per row of |z|^2
    // floats, or two of complex samples (|z|^2 formed with the same rounding as power())
    // (columns past the last whole group of four, when nx is not a multiple of 4, one per thread)
    const bool quad = (a.pitch & 3) == 0 && (ibase ? (reinterpret_cast<uintptr_t>(ibase) & 15) == 0
                                                   : (reinterpret_cast<uintptr_t>(base) & 15) == 0);
    if (quad) {
        for (int q = tid; q < a.nx / 4; q += nthr) {
            float4 w[kTailRows];
            if (ibase) {
#pragma unroll
                for (int k = 0; k < kTailRows; ++k) {
                    w[k] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                    if (k < nr)
                        w[k] = *reinterpret_cast<const float4*>(ibase + static_cast<long long>(r_lo + k) * a.pitch + 4 * q);
                }
            } else {
#pragma unroll
                for (int k = 0; k < kTailRows; ++k) {
                    float4 z0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), z1 = z0;
                    if (k < nr) {
                        const float4* p =
                            reinterpret_cast<const float4*>(base + static_cast<long long>(r_lo + k) * a.pitch + 4 * q);
                        z0 = p[0];
                        z1 = p[1];
                    }
                    w[k] = make_float4(fma_rn(z0.x, z0.x, fmul_rn(z0.y, z0.y)), fma_rn(z0.z, z0.z, fmul_rn(z0.w, z0.w)),
                                       fma_rn(z1.x, z1.x, fmul_rn(z1.y, z1.y)), fma_rn(z1.z, z1.z, fmul_rn(z1.w, z1.w)));
                }
            }
            float v[kTailRows];
#pragma unroll
            for (int k = 0; k < kTailRows; ++k) v[k] = w[k].x;
            finish(4 * q, v);
#pragma unroll
            for (int k = 0; k < kTailRows; ++k) v[k] = w[k].y;
            finish(4 * q + 1, v);
#pragma unroll
            for (int k = 0; k < kTailRows; ++k) v[k] = w[k].z;
            finish(4 * q + 2, v);
#pragma unroll
            for (int k = 0; k < kTailRows; ++k) v[k] = w[k].w;
            finish(4 * q + 3, v);
        }
        for (int c = (a.nx & ~3) + tid; c < a.nx; c += nthr) {
            float v[kTailRows];
#pragma unroll
            for (int k = 0; k < kTailRows; ++k) v[k] = k < nr ? power(r_lo + k, c) : 0.0f;
            finish(c, v);
        }
    } else {
        for (int cb = tid; cb < a.nx; cb += 2 * nthr) {
            float v[2][kTailRows];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = cb + h * nthr;
#pragma unroll
                for (int k = 0; k < kTailRows; ++k) {
                    v[h][k] = 0.0f;
                    if (k < nr && c < a.nx) v[h][k] = power(r_lo + k, c);
                }
            }
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int c = cb + h * nthr;
                if (c >= a.nx) break;
                finish(c, v[h]);
            }
        }
    }
    ASARF_SYNC();
    float* orow = a.mds ? nullptr : a.out + static_cast<long long>(y) * a.out_pitch;
    uint8_t* rec = a.mds ? a.mds + static_cast<long long>(y) * (a.mds_hdr + 2 * tv.ng) : nullptr;
    if (rec)
        for (int i = tid; i < a.mds_hdr; i += nthr) rec[i] = 0;
    const float rsp = fdiv_rn(1.0f, a.range_spacing);
    for (int xg = tid; xg < tv.ng; xg += nthr) {
        const float gd = fmul_rn(static_cast<float>(xg), a.ground_spacing);
        const float rd = polyval_f32(tv.grsr, gd);
        const float idx = div_by_recip_rn(rd, a.range_spacing, rsp);
        int i0 = static_cast<int>(idx);
        const float dx = fsub_rn(idx, static_cast<float>(i0));
        if (i0 < 0 || i0 + 1 >= a.nx) {
            atomic_or_u32(err_flag, kErrSrgrIndex);
            i0 = i0 < 0 ? 0 : a.nx - 2;
        }
        const float v0 = ml[i0], v1 = ml[i0 + 1];
        const float v = fma_rn(dx, fsub_rn(v1, v0), v0);
        if (rec)
            imp_store(rec + a.mds_hdr, xg, v, a.mds_cal);
        else
            orow[xg] = v;
        if (a.out2) a.out2[static_cast<long long>(y) * a.out_pitch + xg] = v;
    }
}

// One record of a level-1 product (row y of the input).
ASARF_HD ASARF_INLINE void condition_row(const ConditionArgs& a, int y, int tid, int nthr) {
    if (a.product == 2) {
        const float2* base = a.slc;
        int rows = a.y_size;
        if (a.state) {
            base += static_cast<long long>(a.state->first_line) * a.stride;
            rows = a.state->n_lines;
        }
        if (y >= rows) return;
        ims_record(base + static_cast<long long>(y) * a.stride, a.x_size, a.cal, a.hdr,
                   a.dest + static_cast<long long>(y) * (a.hdr + 4ll * a.x_size), tid, nthr);
    } else {
        if (y >= a.y_size) return;
        uint8_t* rec = a.dest + static_cast<long long>(y) * (a.hdr + 2ll * a.x_size);
        for (int i = tid; i < a.hdr; i += nthr) rec[i] = 0;
        const float* row = a.img + static_cast<long long>(y) * a.stride;
        for (int x = tid; x < a.x_size; x += nthr) imp_store(rec + a.hdr, x, row[x], a.cal);
    }
}

// ----------------------------------------------------------------------------- product statistics
// Pair p of the product statistics.  IMS form: SLC pixel p of the results window.  IMP form: the
// reference reuses the subset SLC's buffer for the ground-range floats and views it as a
// complex image of the ground-range size (main.cc:327-331), so pair p is floats 2p, 2p+1 of
// that buffer: ground-range pixels below N = ng * out_az, beyond it the SLC floats the
// resampling did not overwrite (SLC stored contiguously [lines][nx], as the subset copy leaves it).
ASARF_HD ASARF_INLINE float stats_float(const ProductStatsArgs& a, long long f, long long n_img, int ng) {
    if (f < n_img) {
        const long long r = f / ng;
        return a.img[r * a.img_pitch + (f - r * ng)];
    }
    const long long k = f >> 1;
    const long long r = k / a.nx;
    const float2 z = a.slc[(a.state->first_line + r) * a.slc_pitch + (k - r * a.nx)];
    return (f & 1) ? z.y : z.x;
}

ASARF_HD ASARF_INLINE long long stats_pairs(const ProductStatsArgs& a) {
    const FocusState& st = *a.state;
    return a.imaged ? static_cast<long long>(a.ng[st.variant]) * a.out_az[st.variant]
                    : static_cast<long long>(st.n_lines) * a.nx;
}

// Block `blk` of `a.blocks`: pairs blk * 256 + t, stepping by blocks * 256, into part[blk]
// (pairwise tree over the 256 lanes).
ASARF_HD ASARF_INLINE void product_stats_body(const ProductStatsArgs& a, int blk, int tid, int nthr, double* red) {
    const FocusState& st = *a.state;
    const long long n = stats_pairs(a);
    const int ng = a.ng[st.variant];
    const long long n_img = static_cast<long long>(ng) * a.out_az[st.variant];
    for (int t = tid; t < 256; t += nthr) {
        double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
        for (long long p = static_cast<long long>(blk) * 256 + t; p < n; p += static_cast<long long>(a.blocks) * 256) {
            float x, y;
            if (a.imaged) {
                x = stats_float(a, 2 * p, n_img, ng);
                y = stats_float(a, 2 * p + 1, n_img, ng);
            } else {
                const long long r = p / a.nx;
                const float2 z = a.slc[(st.first_line + r) * a.slc_pitch + (p - r * a.nx)];
                x = z.x;
                y = z.y;
            }
            if (x != x || y != y) continue;
            v[0] += 1.0;
            v[1] += x;
            v[2] += y;
            v[3] += static_cast<double>(x) * x;
            v[4] += static_cast<double>(y) * y;
        }
        for (int k = 0; k < 5; ++k) red[k * 256 + t] = v[k];
    }
    ASARF_SYNC();
    for (int h = 128; h > 0; h >>= 1) {
        for (int t = tid; t < 5 * h; t += nthr) {
            const int k = t / h, i = t - k * h;
            red[k * 256 + i] += red[k * 256 + i + h];
        }
        ASARF_SYNC();
    }
    for (int k = tid; k < 5; k += nthr) a.part[static_cast<long long>(blk) * 5 + k] = red[k * 256];
}

// Fold of the block partials (pairwise tree over kStatsFoldLeaves leaves) and the statistics in
// the reference's arithmetic: mean = float(float(sum) / float(N)), deviation = sqrt(float(
// float(sum of squared differences) / float(N))) with N all pairs, as CalcMean / CalcStdDev
// divide by the image size; IMS: (mean I, mean Q, dev I, dev Q), IMP: ((mean I + mean Q) / 2, 0,
// (dev I + dev Q) / 2, 0); then scaled by the calibration constant as main.cc:336-342, 384-390.
constexpr int kStatsFoldLeaves = 1024;
ASARF_HD ASARF_INLINE void product_stats_fold(const ProductStatsArgs& a, int tid, int nthr, double* tree) {
    for (int t = tid; t < 5 * kStatsFoldLeaves; t += nthr) {
        const int k = t / kStatsFoldLeaves, i = t - k * kStatsFoldLeaves;
        tree[t] = i < a.blocks ? a.part[static_cast<long long>(i) * 5 + k] : 0.0;
    }
    ASARF_SYNC();
    for (int h = kStatsFoldLeaves / 2; h > 0; h >>= 1) {
        for (int t = tid; t < 5 * h; t += nthr) {
            const int k = t / h, i = t - k * h;
            tree[k * kStatsFoldLeaves + i] += tree[k * kStatsFoldLeaves + i + h];
        }
        ASARF_SYNC();
    }
    if (tid != 0) return;
    const double cnt = tree[0], sx = tree[kStatsFoldLeaves], sy = tree[2 * kStatsFoldLeaves];
    const double sxx = tree[3 * kStatsFoldLeaves], syy = tree[4 * kStatsFoldLeaves];
    const float nf = static_cast<float>(stats_pairs(a));
    const float mx = static_cast<float>(sx) / nf, my = static_cast<float>(sy) / nf;
    const double dx = sxx - 2.0 * mx * sx + cnt * static_cast<double>(mx) * mx;
    const double dy = syy - 2.0 * my * sy + cnt * static_cast<double>(my) * my;
    const float vx = static_cast<float>(dx) / nf, vy = static_cast<float>(dy) / nf;
    const float ex = sqrtf(vx), ey = sqrtf(vy);
    const double c = a.cal;
    if (a.imaged) {
        a.out[0] = static_cast<double>((mx + my) / 2) * c;
        a.out[1] = 0.0;
        a.out[2] = static_cast<double>((ex + ey) / 2) * c;
        a.out[3] = 0.0;
    } else {
        a.out[0] = mx * c;
        a.out[1] = my * c;
        a.out[2] = ex * c;
        a.out[3] = ey * c;
    }
}

// ============================================================================= per-stage bodies

// ConvertErsImSamplesToComplexKernel (envisat_format/src/envisat_format_kernels.cu:116-134)
// after the NaN pre-fill of ConvertRawSampleSetsToComplex (main_flow.cc:537-540): one item
// per (line, range sample).
ASARF_HD ASARF_INLINE void decode_item(const DecodeArgs& a, long long idx) {
    const int y = static_cast<int>(idx / a.nr);
    const int x = static_cast<int>(idx - static_cast<long long>(y) * a.nr);
    const int off = a.swst ? 4 * (static_cast<int>(a.swst[y]) - a.min_swst) : 0;
    const int i = x - off;
    float2 v = make_float2(qnan_f(), qnan_f());
    if (i >= 0 && i < a.spl) {
        const uint8_t* p = a.raw + static_cast<long long>(y) * a.line_bytes + 2ll * i;
        v = make_float2(static_cast<float>(p[0]), static_cast<float>(p[1]));
    }
    a.img[static_cast<long long>(y) * a.stride + x] = v;
}

// ConvertAsarImBlocksToComplexKernel (envisat_format/src/envisat_format_kernels.cu:160-209) as
// a gather over output pixels: sample r = x - (swst[y] - min_swst) of record y through the
// instrument-file tables, NaN where the record holds no sample.
ASARF_HD ASARF_INLINE void decode_fbaq_item(const DecodeFbaqArgs& a, long long idx) {
    const int y = static_cast<int>(idx / a.nr);
    const int x = static_cast<int>(idx - static_cast<long long>(y) * a.nr);
    const int r = x - (a.swst ? static_cast<int>(a.swst[y]) - a.min_swst : 0);
    float2 v = make_float2(qnan_f(), qnan_f());
    if (r >= 0) {
        const uint8_t* rec = a.raw + static_cast<long long>(y) * a.line_bytes;
        const int len = fbaq_len(rec, a.line_bytes);
        const int b = r / 63;
        const int j = r + b + 1;
        if (j < len) {
            const int id = rec[2 + 64 * b];
            const int cw = rec[2 + j];
            v = make_float2(ASARF_LDG(a.lut_i + fbaq4_index(id, cw >> 4)), ASARF_LDG(a.lut_q + fbaq4_index(id, cw & 15)));
        }
    }
    a.img[static_cast<long long>(y) * a.stride + x] = v;
}

ASARF_HD ASARF_INLINE bool is_nan_f(float v) { return v != v; }

// Moment partials for RawDataCorrection / CalcMean / CalcStdDev
// (sar/iq_correction.cu:40-138, cuda_util/device_padded_image.cu:156-257): block `blk` sums
// rows [blk*rpb, ...) in double, NaN samples skipped; deterministic in-block tree.
ASARF_HD ASARF_INLINE void img_moments_body(const ImgMomentsArgs& a, int blk, int tid, int nthr, double* red) {
    double acc[12];
    for (int k = 0; k < 12; ++k) acc[k] = 0.0;
    const int y0 = blk * a.rows_per_block;
    const int y1 = (y0 + a.rows_per_block < a.y_size) ? y0 + a.rows_per_block : a.y_size;
    for (int y = y0; y < y1; ++y) {
        const float2* row = a.img + static_cast<long long>(y) * a.x_stride;
        for (int x = tid; x < a.x_stride; x += nthr) {
            const float2 v = row[x];
            if (is_nan_f(v.x) || is_nan_f(v.y)) continue;
            const int o = x < a.x_size ? 0 : 6;
            if (a.centered) {
                if (o) continue;
                const float di = fsub_rn(v.x, a.mean_i), dq = fsub_rn(v.y, a.mean_q);
                acc[3] += static_cast<double>(fmul_rn(di, di));
                acc[4] += static_cast<double>(fmul_rn(dq, dq));
                acc[0] += 1.0;
                continue;
            }
            const double i = v.x, q = v.y;
            acc[o + 0] += 1.0;
            acc[o + 1] += i;
            acc[o + 2] += q;
            acc[o + 3] += i * i;
            acc[o + 4] += q * q;
            acc[o + 5] += i * q;
        }
    }
    for (int k = 0; k < 12; ++k) red[k * nthr + tid] = acc[k];
    ASARF_SYNC();
#if defined(__CUDA_ARCH__)
    for (int w = nthr / 2; w > 0; w >>= 1) {
        if (tid < w)
            for (int k = 0; k < 12; ++k) red[k * nthr + tid] += red[k * nthr + tid + w];
        ASARF_SYNC();
    }
    if (tid == 0)
        for (int k = 0; k < 12; ++k) a.partial[blk * 12 + k] = red[k * nthr];
#else
    for (int k = 0; k < 12; ++k) a.partial[blk * 12 + k] = red[k * nthr];
#endif
}

// CorrectDCBias + ApplyGainCorrection + ApplyPhaseCorrection (sar/iq_correction.cu:140-178)
// over x < XStride, y < YSize; NaN stays NaN.
ASARF_HD ASARF_INLINE void iq_apply_item(const IqApplyArgs& a, long long idx) {
    float2 v = a.img[idx];
    const float i1 = fsub_rn(v.x, a.dc_i);
    const float q1 = fsub_rn(v.y, a.dc_q);
    const float i2 = fdiv_rn(i1, a.gain);
    const float q2 = fdiv_rn(fma_rn(-i2, a.sin_c, q1), a.cos_c);
    a.img[idx] = make_float2(i2, q2);
}

// PhaseDifference partials of CalculateDopplerCentroid (sar/fractional_doppler_centroid.cu:33-69):
// per block of rows and per column x (columns up to nblk*step, which may reach into the
// padding as the reference's last block does), the FP64 sum over pairs (y-1, y), y >= 1,
// of conj(z[y-1]) z[y]; the host adds columns into range blocks in a fixed order.
ASARF_HD ASARF_INLINE void accc_body(const AcccArgs& a, int blk, int tid, int nthr) {
    const int y0 = blk * a.rows_per_block;
    const int y1 = (y0 + a.rows_per_block < a.y_size) ? y0 + a.rows_per_block : a.y_size;
    const int xend = a.nblk * a.step < a.x_stride ? a.nblk * a.step : a.x_stride;
    for (int x = tid; x < xend; x += nthr) {
        double re = 0.0, im = 0.0;
        for (int y = (y0 > 1 ? y0 : 1); y < y1; ++y) {
            const float2 p = a.img[static_cast<long long>(y - 1) * a.x_stride + x];
            const float2 c = a.img[static_cast<long long>(y) * a.x_stride + x];
            re += static_cast<double>(p.x) * c.x + static_cast<double>(p.y) * c.y;
            im += static_cast<double>(p.x) * c.y - static_cast<double>(p.y) * c.x;
        }
        a.partial[(static_cast<long long>(blk) * xend + x) * 2] = re;
        a.partial[(static_cast<long long>(blk) * xend + x) * 2 + 1] = im;
    }
}

// RangeCompression on complex rows in place (sar/range_compression.cu:57-111): inputs
// x < nr, outputs x < nk scaled, [nk, x_zero_end) zeroed (FinishRangeCompression).
ASARF_HD ASARF_INLINE void rc_rows_body(const RcRowsArgs& a, int y, int tid, int nthr, float2* s) {
    const int L = a.plan.n;
    float2* row = a.img + static_cast<long long>(y) * a.stride;
    for (int l = tid; l < L; l += nthr) s[l] = l < a.nr ? row[l] : make_float2(0.0f, 0.0f);
    ASARF_SYNC();
    fft_forward(a.plan, s, 1, 1, tid, nthr);
    for (int l = tid; l < L; l += nthr) s[l] = cmul(s[l], ASARF_LDG(a.mf + l));
    ASARF_SYNC();
    fft_inverse(a.plan, s, 1, 1, tid, nthr);
    for (int l = tid; l < a.x_zero_end; l += nthr) row[l] = l < a.nk ? s[l] : make_float2(0.0f, 0.0f);
}

// TimeDomainAzimuthLook (sar/az_multilook.cu:25-80): one output line per block.
ASARF_HD ASARF_INLINE void multilook_row_body(const MultilookArgs& a, int y, int tid, int nthr) {
    const float in_idx = fmul_rn(static_cast<float>(y), a.ratio);
    const float mu = fsub_rn(in_idx, static_cast<float>(static_cast<int>(in_idx)));
    int s0 = static_cast<int>(fsub_rn(in_idx, 2.0f)), e0 = static_cast<int>(fadd_rn(in_idx, 2.0f));
    int s1 = static_cast<int>(fsub_rn(in_idx, 1.0f)), e1 = static_cast<int>(fadd_rn(in_idx, 3.0f));
    s0 = s0 > 0 ? s0 : 0;
    s1 = s1 > 0 ? s1 : 0;
    e0 = e0 < a.in_y ? e0 : a.in_y;
    e1 = e1 < a.in_y ? e1 : a.in_y;
    const int c0 = e0 > s0 ? e0 - s0 : 0;
    const int c1 = e1 > s1 ? e1 - s1 : 0;
    const int r_lo = s0 < s1 ? s0 : s1;
    const int r_hi = e0 > e1 ? e0 : e1;
    for (int c = tid; c < a.x_size; c += nthr) {
        float sum0 = 0.0f, sum1 = 0.0f;
        for (int r = r_lo; r < r_hi; ++r) {
            const float2 v = a.slc[static_cast<long long>(r) * a.x_size + c];
            const float p2 = fma_rn(v.x, v.x, fmul_rn(v.y, v.y));
            if (r >= s0 && r < e0) sum0 = fadd_rn(sum0, p2);
            if (r >= s1 && r < e1) sum1 = fadd_rn(sum1, p2);
        }
        if (c0) sum0 = fdiv_rn(sum0, static_cast<float>(c0));
        if (c1) sum1 = fdiv_rn(sum1, static_cast<float>(c1));
        float val = 0.0f;
        if (c0 && c1) val = fma_rn(fsub_rn(sum1, sum0), mu, sum0);
        a.out[static_cast<long long>(y) * a.x_size + c] = val;
    }
}

// CorrectionKernel of RangeSpreadingLossCorrection (sar/range_spreading_loss.cu:29-52).
ASARF_HD ASARF_INLINE void rsl_item(const RslArgs& a, long long idx) {
    const int x = static_cast<int>(idx % a.range_size);
    const double r = a.slant_first + x * a.range_spacing;
    const double ratio = a.ref_range / r;
    const float g = static_cast<float>(1.0 / sqrt(pow(ratio, 3.0)));
    a.img[idx] = fmul_rn(a.img[idx], g);
}

// SrGrInterpolation (sar/srgr.cu:49-71) with the float Horner / IEEE divide / truncation index.
ASARF_HD ASARF_INLINE void srgr_item(const SrgrArgs& a, long long idx) {
    const int y = static_cast<int>(idx / a.out_x);
    const int xg = static_cast<int>(idx - static_cast<long long>(y) * a.out_x);
    const float gd = fmul_rn(static_cast<float>(xg), a.ground_spacing);
    const float rd = polyval_f32(a.grsr, gd);
    const float ridx = fdiv_rn(rd, a.range_spacing);
    int i0 = static_cast<int>(ridx);
    const float dx = fsub_rn(ridx, static_cast<float>(i0));
    if (a.start && y == 0) {
        a.start[xg] = i0;
        a.frac[xg] = dx;
    }
    if (!a.in) return;
    if (i0 < 0 || i0 + 1 >= a.in_x) {
        if (a.err) atomic_or_u32(a.err, kErrSrgrIndex);
        i0 = i0 < 0 ? 0 : a.in_x - 2;
    }
    const float* row = a.in + static_cast<long long>(y) * a.in_x;
    const float v0 = row[i0], v1 = row[i0 + 1];
    a.out[idx] = fma_rn(dx, fsub_rn(v1, v0), v0);
}

}  // namespace asarf
