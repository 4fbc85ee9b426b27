/*
 * eemd_flac.h -- C ABI of the FLAC decoder (libeemd_flac.so, host code).
 *
 * Replaces the FLAC read of the reference's audio input
 * (audio_eemd/audio_io.py:71-103, soundfile.read(path, dtype="float64",
 * always_2d=True) on libsndfile), the step before the EEMD path.  The decoder
 * follows the FLAC format of RFC 9639.  All pointers are host pointers; the
 * library keeps no state between calls.  eemd4cuda_b200/audio.py binds it with
 * ctypes and scales the integer samples by 2^-(bits_per_sample-1), the float
 * convention soundfile uses.
 */
#ifndef EEMD_FLAC_H
#define EEMD_FLAC_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EEMD_FLAC_OK           0
#define EEMD_FLAC_E_BADARG    -1  /* null pointer, or the output buffer is too small */
#define EEMD_FLAC_E_FORMAT    -2  /* not a FLAC stream, or a malformed or reserved field */
#define EEMD_FLAC_E_TRUNCATED -3  /* the stream ends inside a metadata block or a frame */
#define EEMD_FLAC_E_CRC       -4  /* a frame header's CRC-8 or a frame's CRC-16 does not match */
#define EEMD_FLAC_E_NOMEM     -5  /* host allocation of the per-frame channel buffers failed */

typedef struct eemd_flac_stream_info {
    int32_t sample_rate;         /* Hz */
    int32_t channels;            /* 1..8 */
    int32_t bits_per_sample;     /* 4..32 */
    int32_t min_block;           /* samples per channel in a frame (STREAMINFO) */
    int32_t max_block;
    int32_t pad;
    int64_t total_frames;        /* samples per channel in the stream (0 = unknown) */
    int64_t first_frame_offset;  /* byte offset of the first audio frame */
    uint8_t md5[16];             /* MD5 of the decoded samples (all zero = not computed) */
} eemd_flac_stream_info;

/* Parse the "fLaC" marker and the metadata blocks (STREAMINFO first) of the
 * n bytes at data. */
int32_t eemd_flac_info(const uint8_t* data, size_t n, eemd_flac_stream_info* info);

/* Decode every audio frame into out[frame][channel] (int32, interleaved;
 * out_frames frames of room).  *frames_decoded receives the frames written.
 * Every frame header's CRC-8 and frame's CRC-16 is checked. */
int32_t eemd_flac_decode(const uint8_t* data, size_t n, int32_t* out, int64_t out_frames,
                         int64_t* frames_decoded);

/* Human-readable text for a status code. */
const char* eemd_flac_strerror(int32_t status);

#ifdef __cplusplus
}
#endif
#endif /* EEMD_FLAC_H */
