/* flac_decode.c -- FLAC stream decoder (host, C99), the C ABI of include/eemd_flac.h.
 *
 * The reference reads its audio through soundfile / libsndfile
 * (audio_eemd/audio_io.py:71-103); FLAC is its primary input format.  This
 * is a decoder of the FLAC format as published in RFC 9639 ("Free Lossless
 * Audio Codec"), written from that specification:
 *   - stream: "fLaC" marker, metadata blocks (STREAMINFO first; the others
 *     are skipped), then frames;
 *   - frame header: 14-bit sync code 0x3FFE, blocking strategy, block size,
 *     sample rate, channel assignment and sample size codes, the coded
 *     frame / sample number, optional explicit block size and rate, CRC-8
 *     (polynomial x^8 + x^2 + x + 1);
 *   - subframes: CONSTANT, VERBATIM, FIXED (orders 0-4) and LPC (orders
 *     1-32) with wasted bits; residuals in partitioned Rice coding with 4- or
 *     5-bit parameters and the escape to raw binary;
 *   - channel decorrelation: left/side, side/right and mid/side;
 *   - frame footer: byte alignment and CRC-16 (x^16 + x^15 + x^2 + 1).
 * Every header, reserved value and CRC is checked; a malformed stream ends the
 * decode with a status instead of reading past the buffer.
 */
#include "../../include/eemd_flac.h"

#include <stdlib.h>
#include <string.h>

typedef struct {
    const uint8_t* p;
    size_t n;      /* bytes */
    size_t bit;    /* bit position from the start */
    int err;       /* read past the end */
} Bits;

static uint32_t bits_u(Bits* b, int k) { /* k <= 32 */
    uint64_t v = 0;
    if (k == 0) return 0;
    if (b->bit + (size_t)k > b->n * 8) {
        b->err = 1;
        b->bit = b->n * 8;
        return 0;
    }
    for (int i = 0; i < k;) {
        const size_t byte = b->bit >> 3;
        const int off = (int)(b->bit & 7);
        const int take = (8 - off) < (k - i) ? (8 - off) : (k - i);
        const uint32_t chunk = ((uint32_t)b->p[byte] >> (8 - off - take)) & ((1u << take) - 1u);
        v = (v << take) | chunk;
        b->bit += (size_t)take;
        i += take;
    }
    return (uint32_t)v;
}

static uint64_t bits_u64(Bits* b, int k) { /* k <= 64 */
    if (k <= 32) return bits_u(b, k);
    const uint64_t hi = bits_u(b, k - 32);
    return (hi << 32) | bits_u(b, 32);
}

static int32_t bits_s(Bits* b, int k) { /* two's complement, k <= 32 */
    if (k == 0) return 0;
    const uint32_t v = bits_u(b, k);
    if (k == 32) return (int32_t)v;
    const uint32_t sign = 1u << (k - 1);
    return (int32_t)((v ^ sign) - sign);
}

/* number of 0 bits before the next 1 bit (the 1 is consumed) */
static uint32_t bits_unary(Bits* b) {
    uint32_t q = 0;
    for (;;) {
        if (b->bit >= b->n * 8) {
            b->err = 1;
            return q;
        }
        const size_t byte = b->bit >> 3;
        const int off = (int)(b->bit & 7);
        const uint32_t rest = ((uint32_t)b->p[byte] << off) & 0xFFu;
        if (rest == 0) {
            q += (uint32_t)(8 - off);
            b->bit += (size_t)(8 - off);
            continue;
        }
        int lead = 0;
        while (!(rest & (0x80u >> lead))) ++lead;
        q += (uint32_t)lead;
        b->bit += (size_t)lead + 1;
        return q;
    }
}

static uint8_t crc8(const uint8_t* p, size_t n) {
    uint8_t c = 0;
    for (size_t i = 0; i < n; ++i) {
        c ^= p[i];
        for (int k = 0; k < 8; ++k) c = (uint8_t)((c & 0x80) ? ((c << 1) ^ 0x07) : (c << 1));
    }
    return c;
}

static uint16_t crc16(const uint8_t* p, size_t n) {
    uint16_t c = 0;
    for (size_t i = 0; i < n; ++i) {
        c ^= (uint16_t)((uint16_t)p[i] << 8);
        for (int k = 0; k < 8; ++k) c = (uint16_t)((c & 0x8000) ? ((c << 1) ^ 0x8005) : (c << 1));
    }
    return c;
}

int32_t eemd_flac_info(const uint8_t* data, size_t n, eemd_flac_stream_info* info) {
    if (!data || !info) return EEMD_FLAC_E_BADARG;
    memset(info, 0, sizeof(*info));
    if (n < 4 || memcmp(data, "fLaC", 4) != 0) return EEMD_FLAC_E_FORMAT;
    size_t pos = 4;
    int have_info = 0, last = 0;
    while (!last) {
        if (pos + 4 > n) return EEMD_FLAC_E_TRUNCATED;
        last = data[pos] >> 7;
        const int type = data[pos] & 0x7F;
        const size_t len = ((size_t)data[pos + 1] << 16) | ((size_t)data[pos + 2] << 8) | data[pos + 3];
        pos += 4;
        if (pos + len > n) return EEMD_FLAC_E_TRUNCATED;
        if (type == 127) return EEMD_FLAC_E_FORMAT; /* forbidden block type */
        if (type == 0) {
            if (have_info || len != 34) return EEMD_FLAC_E_FORMAT;
            Bits b = {data + pos, len, 0, 0};
            info->min_block = (int32_t)bits_u(&b, 16);
            info->max_block = (int32_t)bits_u(&b, 16);
            (void)bits_u(&b, 24); /* min frame size */
            (void)bits_u(&b, 24); /* max frame size */
            info->sample_rate = (int32_t)bits_u(&b, 20);
            info->channels = (int32_t)bits_u(&b, 3) + 1;
            info->bits_per_sample = (int32_t)bits_u(&b, 5) + 1;
            info->total_frames = (int64_t)bits_u64(&b, 36);
            for (int i = 0; i < 16; ++i) info->md5[i] = (uint8_t)bits_u(&b, 8);
            have_info = 1;
        } else if (!have_info) {
            return EEMD_FLAC_E_FORMAT; /* STREAMINFO must come first */
        }
        pos += len;
    }
    if (!have_info || info->sample_rate == 0 || info->bits_per_sample < 4 || info->min_block < 16 ||
        info->max_block < info->min_block)
        return EEMD_FLAC_E_FORMAT;
    info->first_frame_offset = (int64_t)pos;
    return EEMD_FLAC_OK;
}

/* residual of one subframe: out[order..bs) receives the decoded residuals */
static int read_residual(Bits* b, int32_t* out, int bs, int order) {
    const uint32_t method = bits_u(b, 2);
    if (method > 1) return EEMD_FLAC_E_FORMAT;
    const int pbits = method == 0 ? 4 : 5;
    const uint32_t escape = method == 0 ? 15u : 31u;
    const int porder = (int)bits_u(b, 4);
    const int parts = 1 << porder;
    if ((bs >> porder) << porder != bs || (bs >> porder) < order) return EEMD_FLAC_E_FORMAT;
    int i = order;
    for (int part = 0; part < parts; ++part) {
        const int cnt = (bs >> porder) - (part == 0 ? order : 0);
        const uint32_t k = bits_u(b, pbits);
        if (k == escape) {
            const int raw = (int)bits_u(b, 5);
            for (int j = 0; j < cnt; ++j) out[i++] = bits_s(b, raw);
        } else {
            for (int j = 0; j < cnt; ++j) {
                const uint32_t q = bits_unary(b);
                if (q > 0xFFFFFu) return EEMD_FLAC_E_FORMAT; /* no sample value needs that many */
                const uint64_t u = ((uint64_t)q << k) | bits_u(b, (int)k);
                out[i++] = (int32_t)((int64_t)(u >> 1) ^ -(int64_t)(u & 1u));
            }
        }
        if (b->err) return EEMD_FLAC_E_TRUNCATED;
    }
    return EEMD_FLAC_OK;
}

/* one subframe of bs samples at sample size bps into s[0..bs) */
static int read_subframe(Bits* b, int32_t* s, int bs, int bps) {
    if (bits_u(b, 1) != 0) return EEMD_FLAC_E_FORMAT;
    const uint32_t type = bits_u(b, 6);
    int wasted = 0;
    if (bits_u(b, 1)) wasted = (int)bits_unary(b) + 1;
    if (wasted >= bps) return EEMD_FLAC_E_FORMAT;
    const int ebps = bps - wasted;
    int rc = EEMD_FLAC_OK;
    if (type == 0) { /* CONSTANT */
        const int32_t v = bits_s(b, ebps);
        for (int i = 0; i < bs; ++i) s[i] = v;
    } else if (type == 1) { /* VERBATIM */
        for (int i = 0; i < bs; ++i) s[i] = bits_s(b, ebps);
    } else if (type >= 8 && type <= 12) { /* FIXED, order 0..4 */
        const int order = (int)type - 8;
        if (order > bs) return EEMD_FLAC_E_FORMAT;
        for (int i = 0; i < order; ++i) s[i] = bits_s(b, ebps);
        rc = read_residual(b, s, bs, order);
        if (rc) return rc;
        for (int i = order; i < bs; ++i) {
            int64_t pred = 0;
            switch (order) {
                case 1: pred = s[i - 1]; break;
                case 2: pred = 2 * (int64_t)s[i - 1] - s[i - 2]; break;
                case 3: pred = 3 * (int64_t)s[i - 1] - 3 * (int64_t)s[i - 2] + s[i - 3]; break;
                case 4:
                    pred = 4 * (int64_t)s[i - 1] - 6 * (int64_t)s[i - 2] + 4 * (int64_t)s[i - 3] - s[i - 4];
                    break;
                default: break;
            }
            s[i] = (int32_t)(pred + s[i]);
        }
    } else if (type >= 32) { /* LPC, order 1..32 */
        const int order = (int)(type & 31u) + 1;
        if (order > bs) return EEMD_FLAC_E_FORMAT;
        for (int i = 0; i < order; ++i) s[i] = bits_s(b, ebps);
        const int prec = (int)bits_u(b, 4) + 1;
        if (prec == 16) return EEMD_FLAC_E_FORMAT;
        const int shift = bits_s(b, 5);
        if (shift < 0) return EEMD_FLAC_E_FORMAT;
        int32_t coef[32];
        for (int j = 0; j < order; ++j) coef[j] = bits_s(b, prec);
        rc = read_residual(b, s, bs, order);
        if (rc) return rc;
        for (int i = order; i < bs; ++i) {
            int64_t acc = 0;
            for (int j = 0; j < order; ++j) acc += (int64_t)coef[j] * s[i - 1 - j];
            s[i] = (int32_t)((acc >> shift) + s[i]);
        }
    } else {
        return EEMD_FLAC_E_FORMAT; /* reserved subframe type */
    }
    if (b->err) return EEMD_FLAC_E_TRUNCATED;
    if (wasted)
        for (int i = 0; i < bs; ++i) s[i] = (int32_t)((uint32_t)s[i] << wasted);
    return EEMD_FLAC_OK;
}

int32_t eemd_flac_decode(const uint8_t* data, size_t n, int32_t* out, int64_t out_frames,
                         int64_t* frames_decoded) {
    if (!data || !out || out_frames < 0 || !frames_decoded) return EEMD_FLAC_E_BADARG;
    *frames_decoded = 0;
    eemd_flac_stream_info info;
    int32_t rc = eemd_flac_info(data, n, &info);
    if (rc) return rc;
    const int C = info.channels;
    int32_t* ch[8] = {0};
    int32_t* tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)65536 * (size_t)C);
    if (!tmp) return EEMD_FLAC_E_NOMEM;
    for (int c = 0; c < C; ++c) ch[c] = tmp + (size_t)c * 65536;
    size_t pos = (size_t)info.first_frame_offset;
    int64_t done = 0;
    rc = EEMD_FLAC_OK;
    while (pos < n && (info.total_frames == 0 || done < info.total_frames)) {
        const size_t start = pos;
        Bits b = {data, n, pos * 8, 0};
        if (bits_u(&b, 14) != 0x3FFE || bits_u(&b, 1) != 0) { rc = EEMD_FLAC_E_FORMAT; break; }
        (void)bits_u(&b, 1); /* blocking strategy: the frame header carries the block size either way */
        const uint32_t bsc = bits_u(&b, 4), src = bits_u(&b, 4), chc = bits_u(&b, 4), ssc = bits_u(&b, 3);
        if (bits_u(&b, 1) != 0 || bsc == 0 || src == 15 || chc > 10 || ssc == 3) { rc = EEMD_FLAC_E_FORMAT; break; }
        /* coded frame / sample number (UTF-8 style, up to 7 bytes) */
        const uint32_t first = bits_u(&b, 8);
        int more = 0;
        if (first >= 0x80) {
            if ((first & 0xE0) == 0xC0) more = 1;
            else if ((first & 0xF0) == 0xE0) more = 2;
            else if ((first & 0xF8) == 0xF0) more = 3;
            else if ((first & 0xFC) == 0xF8) more = 4;
            else if ((first & 0xFE) == 0xFC) more = 5;
            else if (first == 0xFE) more = 6;
            else { rc = EEMD_FLAC_E_FORMAT; break; }
        }
        for (int i = 0; i < more; ++i)
            if ((bits_u(&b, 8) & 0xC0) != 0x80) { rc = EEMD_FLAC_E_FORMAT; break; }
        if (rc) break;
        int bs;
        if (bsc == 1) bs = 192;
        else if (bsc <= 5) bs = 576 << (bsc - 2);
        else if (bsc == 6) bs = (int)bits_u(&b, 8) + 1;
        else if (bsc == 7) bs = (int)bits_u(&b, 16) + 1;
        else bs = 256 << (bsc - 8);
        if (src == 12) (void)bits_u(&b, 8);
        else if (src == 13 || src == 14) (void)bits_u(&b, 16);
        if (b.err) { rc = EEMD_FLAC_E_TRUNCATED; break; }
        const size_t hdr_end = b.bit >> 3;
        const uint32_t hcrc = bits_u(&b, 8);
        if (b.err) { rc = EEMD_FLAC_E_TRUNCATED; break; }
        if (crc8(data + start, hdr_end - start) != hcrc) { rc = EEMD_FLAC_E_CRC; break; }
        static const int sizes[8] = {0, 8, 12, 0, 16, 20, 24, 32};
        const int bps = ssc == 0 ? info.bits_per_sample : sizes[ssc];
        const int nch = chc < 8 ? (int)chc + 1 : 2;
        if (nch != C || bs > 65536) { rc = EEMD_FLAC_E_FORMAT; break; }
        for (int c = 0; c < nch; ++c) {
            /* the side channel carries one more bit */
            const int extra = (chc == 8 && c == 1) || (chc == 9 && c == 0) || (chc == 10 && c == 1);
            rc = read_subframe(&b, ch[c], bs, bps + extra);
            if (rc) break;
        }
        if (rc) break;
        if (b.bit & 7) {
            if (bits_u(&b, 8 - (int)(b.bit & 7)) != 0) { rc = EEMD_FLAC_E_FORMAT; break; }
        }
        const size_t body_end = b.bit >> 3;
        const uint32_t fcrc = bits_u(&b, 16);
        if (b.err) { rc = EEMD_FLAC_E_TRUNCATED; break; }
        if (crc16(data + start, body_end - start) != fcrc) { rc = EEMD_FLAC_E_CRC; break; }
        pos = b.bit >> 3;
        if (chc == 8) { /* left, side */
            for (int i = 0; i < bs; ++i) ch[1][i] = ch[0][i] - ch[1][i];
        } else if (chc == 9) { /* side, right */
            for (int i = 0; i < bs; ++i) ch[0][i] = ch[0][i] + ch[1][i];
        } else if (chc == 10) { /* mid, side */
            for (int i = 0; i < bs; ++i) {
                const int64_t side = ch[1][i];
                const int64_t mid = ((int64_t)ch[0][i] * 2) | (side & 1);
                ch[0][i] = (int32_t)((mid + side) >> 1);
                ch[1][i] = (int32_t)((mid - side) >> 1);
            }
        }
        const int64_t take = (done + bs <= out_frames) ? bs : out_frames - done;
        if (take < bs) { rc = EEMD_FLAC_E_BADARG; break; } /* output buffer too small */
        for (int64_t i = 0; i < bs; ++i)
            for (int c = 0; c < C; ++c) out[(done + i) * C + c] = ch[c][i];
        done += bs;
    }
    free(tmp);
    *frames_decoded = done;
    if (rc == EEMD_FLAC_OK && info.total_frames != 0 && done != info.total_frames) rc = EEMD_FLAC_E_TRUNCATED;
    return rc;
}

const char* eemd_flac_strerror(int32_t status) {
    switch (status) {
        case EEMD_FLAC_OK: return "ok";
        case EEMD_FLAC_E_BADARG: return "invalid argument or output buffer too small";
        case EEMD_FLAC_E_FORMAT: return "not a FLAC stream, or a malformed or reserved field";
        case EEMD_FLAC_E_TRUNCATED: return "stream ends inside a block or frame";
        case EEMD_FLAC_E_CRC: return "frame CRC mismatch";
        case EEMD_FLAC_E_NOMEM: return "out of host memory";
        default: return "unknown status";
    }
}
