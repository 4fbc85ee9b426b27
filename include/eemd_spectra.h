/* eemd_spectra.h -- C ABI of the IMF spectra stage (libeemd_spectra.so, sm_100a).
 *
 * The consumer of the IMFs in the reference, audio_eemd/spectra.py, computed
 * on the device while the IMFs are resident:
 *
 *   eemd_sp_hilbert_if  replaces spectra.py:32-45 hilbert_if: analytic
 *       signal z = x + i H(x) (scipy.signal.hilbert: FFT, weights 1 / 2 / 0 on
 *       DC / positive / negative frequencies, inverse FFT), instantaneous
 *       frequency = gradient of the unwrapped phase (np.unwrap, np.gradient
 *       with spacing 1/sr) / 2 pi, instantaneous amplitude = |z|.
 *   eemd_sp_stft        replaces spectra.py:18-29 stft_block:
 *       scipy.signal.stft(window='hann', boundary='zeros', padded=False),
 *       one-sided, divided by the window's sum.
 *   eemd_sp_fft         the complex FFT both use (numpy.fft.fft's convention
 *       for sign -1, unnormalised), this library's own: Stockham passes of
 *       radix 4, 2, 3, 5 and odd primes up to 31, Bluestein's chirp-z for a
 *       length with a larger prime factor.
 *
 * Rows are batched: M signals of N samples each, float64, row-major.  All
 * pointers are device pointers owned by the caller, including the workspace
 * (size from the *_workspace queries); the library allocates no memory and
 * keeps no state.  Calls are asynchronous on `stream`; calls that share a
 * workspace must not overlap.
 */
#ifndef EEMD_SPECTRA_H
#define EEMD_SPECTRA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EEMD_SP_ABI_VERSION 1

#define EEMD_SP_OK 0
#define EEMD_SP_E_BADARG -1
#define EEMD_SP_E_NOMEM -2   /* the workspace is smaller than the query returned */
#define EEMD_SP_E_CUDA -5

int32_t eemd_sp_version(void);

/* Workspace bytes for eemd_sp_fft on M rows of N points. */
int32_t eemd_sp_fft_workspace(int32_t M, int64_t N, size_t* bytes);

/* out[m][k] = sum_n in[m][n] exp(sign 2 pi i n k / N) for every row (complex,
 * interleaved re/im float64; sign -1 or +1; N >= 1; out may equal in). */
int32_t eemd_sp_fft(const double* in, double* out, int32_t M, int64_t N, int32_t sign, void* ws, size_t ws_bytes,
                    void* stream);

/* Workspace bytes for eemd_sp_hilbert_if on M rows of N samples. */
int32_t eemd_sp_hilbert_workspace(int32_t M, int64_t N, size_t* bytes);

/* inst_freq[m][n] (Hz) and inst_amp[m][n] of every row x[m][:] (N >= 2). */
int32_t eemd_sp_hilbert_if(const double* x, int32_t M, int64_t N, double sr, double* inst_freq, double* inst_amp,
                           void* ws, size_t ws_bytes, void* stream);

/* Frequencies F = nperseg/2 + 1 and frames T = (N + 2*(nperseg/2) - noverlap) / (nperseg - noverlap)
 * of the STFT (2 <= nperseg, 0 <= noverlap < nperseg). */
int32_t eemd_sp_stft_shape(int64_t N, int32_t nperseg, int32_t noverlap, int32_t* F, int32_t* T);

/* Workspace bytes for eemd_sp_stft. */
int32_t eemd_sp_stft_workspace(int32_t M, int64_t N, int32_t nperseg, int32_t noverlap, size_t* bytes);

/* Z[m][f][t] (complex, interleaved re/im float64) of every row x[m][:]. */
int32_t eemd_sp_stft(const double* x, int32_t M, int64_t N, int32_t nperseg, int32_t noverlap, double* Z, void* ws,
                     size_t ws_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* EEMD_SPECTRA_H */
