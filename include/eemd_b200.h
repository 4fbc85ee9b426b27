/*
 * eemd_b200.h -- C ABI of the B200-native EEMD engine (libeemd_b200.so).
 *
 * The engine runs Ensemble Empirical Mode Decomposition of many signals x
 * many noise trials on one sm_100a GPU.  Every pointer argument marked
 * "device" is a CUDA device pointer owned by the caller; "host" pointers are
 * read during the call only.  The library allocates no device memory: the
 * scratch of eemd_run() lives in the caller's workspace (size from
 * eemd_workspace_size()); calls on different workspaces may overlap, calls on
 * the same workspace must not.  The one piece of library-owned device memory
 * and global state is the fixed-size static scratch array of eemd_run_static()
 * (EEMD_STATIC_SCRATCH_BYTES on every GPU that loads the library, plus a
 * per-device cache of its address); nothing else is kept between calls.
 *
 * Reference interface this replaces (misureaudio/EEMD4CUDA, Python):
 *   - emd_gpu.py:301-334 gpu_eemd_full(x[E,N], E, tau, max_sifts, max_imf)
 *       -> (imfs[E,m,N], nsift[E], nmode[E])          => eemd_run(imfs=...)
 *   - emd_par.py:198-254 _gpu_decompose: noise draw, batch loop, per-mode
 *       masked mean over trials                        => eemd_run(imf_sum=...)
 *                                                         + eemd_finalize()
 *   - emd_gpu.py:120-285 / emd_gpu_v5_dsbt.py:141-338 the numba kernels
 *       (extrema scan, spline system, Thomas / seam-window Thomas, spline
 *       evaluation, SD stop rule, IMF store)           => internal kernels
 * Python binds these through ctypes (eemd4cuda_b200/_lib.py); the same
 * declarations are what a cffi / ctypes stub in the reference would bind.
 */
#ifndef EEMD_B200_H
#define EEMD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EEMD_ABI_VERSION 2

/* status codes (0 = success, negative = error) */
#define EEMD_OK                 0
#define EEMD_E_BADARG          -1  /* invalid argument (maps to ValueError) */
#define EEMD_E_NOMEM           -2  /* workspace smaller than eemd_workspace_size() */
#define EEMD_E_KNOT_OVERFLOW   -3  /* knot buffer capacity exceeded (internal bound violated) */
#define EEMD_E_TIMEOUT         -4  /* a task exceeded its step bound, or the watchdog test
                                         mode's bounded wait gave up */
#define EEMD_E_CUDA            -5  /* CUDA runtime error */
#define EEMD_E_NOTSUP          -6  /* unsupported combination (e.g. exact mode with float32) */
#define EEMD_E_STATIC_CAPACITY -7  /* eemd_run_static(): the problem needs more scratch than
                                      EEMD_STATIC_SCRATCH_BYTES */

/* storage type of signals, IMFs and working arrays; the spline solve is
 * always float64 */
#define EEMD_F64 0
#define EEMD_F32 1

/* end handling of the envelopes (emd_ref.py:77-103 envelope(end=...)) */
#define EEMD_END_NATURAL 0
#define EEMD_END_MIRROR  1

/* stop-rule family
 *  EEMD_RULES_REF   : emd_ref.py:108-156 emd_1d -- IMF loop stops when
 *                     nmax+nmin < min_extrema or max_imf reached; a sift is
 *                     skipped when nmax<1 or nmin<1; SD = sum((h-h_new)^2)/sum(h^2)
 *  EEMD_RULES_NUMBA : emd_gpu.py:152-274 numba kernel -- additionally stops
 *                     the IMF loop when nmax<2 or nmin<2, skips a sift when
 *                     nmax<2 or nmin<2; SD = sum(m^2)/sum(h^2) */
#define EEMD_RULES_REF   0
#define EEMD_RULES_NUMBA 1

/* noise source for the trials */
#define EEMD_NOISE_NONE         0  /* trial input = x (plain EMD) */
#define EEMD_NOISE_PHILOX       1  /* x + eps*std(x)*N(0,1), Philox4x32-10 keyed by (seed, signal, trial) */
#define EEMD_NOISE_INJECTED     2  /* x + noise[task][n] (noise already scaled) */
#define EEMD_NOISE_PREPERTURBED 3  /* x holds one perturbed signal per task: x[task][n] */
#define EEMD_NOISE_SCALED       4  /* x + eps * noise[task][n] (eps absolute; product and sum each
                                      rounded): the CEEMDAN stage input, emd_ref.py:247-248 */

typedef struct eemd_params {
    int32_t  dtype;           /* EEMD_F64 or EEMD_F32 */
    int32_t  noise_mode;      /* EEMD_NOISE_* */
    double   eps;             /* noise std as a fraction of std(x) (PHILOX) */
    uint64_t seed;            /* PHILOX key */
    double   tau;             /* SD threshold; sift loop stops when sd < tau (from the 2nd sift) */
    int32_t  max_sifts;       /* sift cap per IMF (>= 1) */
    int32_t  max_imf;         /* IMF slots per trial (>= 1) */
    int32_t  min_extrema;     /* IMF loop stops below this many extrema */
    int32_t  end_mode;        /* EEMD_END_* */
    int32_t  rules;           /* EEMD_RULES_* */
    int32_t  exact;           /* 1: reference operation order, IEEE division, no FMA (float64 only) */
    int32_t  tile;            /* samples per warp tile of the fused sift pass: 0, or the only
                                 supported value (256 for float32, 128 for float64) */
    int32_t  knots_per_block; /* owned rows per exact-mode seam window (0 = 16; the fast
                                 solve owns 3 rows per window) */
    int32_t  halo;            /* seam halo rows on each side of a window (0 = 32 exact,
                                 24 fast float64, 16 fast float32; at most 64 in fast mode) */
    int64_t  watchdog;        /* >= 0: no effect (the engine has no device waits on its data
                                 path; every loop is bounded by the sift and IMF caps);
                                 a negative value -k is the watchdog test mode: every task
                                 first waits on a flag nothing sets, gives up after k polls
                                 and the run returns EEMD_E_TIMEOUT */
    int32_t  cluster_size;    /* CTAs (thread-block cluster) per task, 1..16 (0 = autotune; 9..16 are
                                 non-portable cluster sizes the device must support) */
    int32_t  reserved;        /* 0.  Test hook honoured only by the bounds-checked build
                                 (libeemd_b200_checked.so): a value k > 0 caps the knot
                                 lists at k knots of one kind per warp segment, so that
                                 the EEMD_E_KNOT_OVERFLOW path can be exercised; the
                                 release build ignores it */
    int32_t  cta_warps;       /* warps per CTA of the persistent kernel: 0 = 4, 4 or 5 (5: three
                                 CTAs per SM instead of four; float64 exact mode runs 4) */
    int32_t  reserved2;       /* 0 */
} eemd_params;

/* Fill p with the defaults of emd_par.decompose (emd_par.py:260-262):
 * float64, tau 0.25, max_sifts 50, min_extrema 4, natural ends, REF rules. */
void eemd_default_params(eemd_params* p);

/* ABI version (EEMD_ABI_VERSION). */
int32_t eemd_version(void);

/* Human-readable text for a status code. */
const char* eemd_strerror(int32_t status);

/* out[e][t] (device, float64 [trial_count][n]) = the standard normal that
 * EEMD_NOISE_PHILOX adds, scaled by eps*std(x), to trial trial_begin + e of
 * signal `signal` at sample t.  The device counterpart of a host noise draw
 * such as emd_ref.py:166-168 _gen_noise (a different stream: Philox4x32-10
 * with Box-Muller, not numpy's PCG64 ziggurat). */
int32_t eemd_philox_normals(uint64_t seed, int32_t signal, int32_t trial_begin, int32_t trial_count, int64_t n,
                            double* out, void* stream);

/* Device bytes of workspace one eemd_run() needs for n_signals signals of the
 * given lengths (host array) with trial_count trials each.  imfs_external != 0
 * means the caller passes its own per-trial IMF buffer to eemd_run(). */
int32_t eemd_workspace_size(const eemd_params* p, const int64_t* lengths,
                            int32_t n_signals, int32_t trial_count,
                            int32_t imfs_external, size_t* ws_bytes);

/* Run the full EMD of every (signal, trial) task of one batch.
 *   x          device  signals back to back (dtype); with PREPERTURBED one
 *                      signal per task, task = s*trial_count + e
 *   lengths    host    n_signals lengths (>= 8 each)
 *   trial_begin        absolute index of the first trial in this batch
 *                      (Philox counter; emd_par.py:230-246 batch loop)
 *   noise      device  INJECTED: scaled noise per task back to back, else NULL
 *   imfs       device  per-trial IMFs [task][max_imf][n_s] (dtype) or NULL
 *                      (then kept in the workspace);  emd_gpu.py:325 `out`
 *   resid_out  device  final per-trial residual [task][n_s] (dtype) or NULL
 *   imf_sum    device  [s][max_imf][n_s] float64, += trial-ordered sum of the
 *                      batch's IMFs of the trials that produced that mode, or
 *                      NULL                         (emd_par.py:241-245)
 *   mode_count device  [s][max_imf] int32, += number of contributing trials
 *   nsift      device  [task] total sifts           (emd_gpu.py:283-285)
 *   nmode      device  [task] number of IMFs
 *   mode_sifts device  [task][max_imf] sifts per IMF or NULL
 *   knot_log   device  [task][max_imf][max_sifts][2] (maxima, minima) knot
 *                      counts of every sift, -1 where no sift ran, or NULL
 *   flags      device  [task] bit0: max_imf slots exhausted while extrema
 *                      remained, or NULL
 * Synchronises `stream` before returning and reports device-side errors. */
int32_t eemd_run(const eemd_params* p, const void* x, const int64_t* lengths,
                 int32_t n_signals, int32_t trial_begin, int32_t trial_count,
                 const void* noise, void* imfs, void* resid_out,
                 double* imf_sum, int32_t* mode_count,
                 int32_t* nsift, int32_t* nmode, int32_t* mode_sifts,
                 int32_t* knot_log, int32_t* flags,
                 void* ws, size_t ws_bytes, void* stream);

/* Kernel kinds of eemd_run_traced() */
#define EEMD_K_SIGMA   0  /* per-signal eps*std(x) */
#define EEMD_K_EMD     1  /* persistent cluster kernel: every IMF and sift of every task */
#define EEMD_K_REDUCE  2  /* trial-ordered ensemble sum */
#define EEMD_K_OUTPUTS 3  /* per-task counters */
#define EEMD_KERNEL_KINDS 8

typedef struct eemd_kernel_times {
    double  ms[EEMD_KERNEL_KINDS];        /* summed CUDA-event time per kind */
    int64_t launches[EEMD_KERNEL_KINDS];  /* launches per kind */
} eemd_kernel_times;

/* eemd_run() that also brackets every kernel launch with a CUDA event pair on
 * `stream` and returns per-kind launch counts and summed durations in *times
 * (host struct).  No counterpart in the reference (its timing is host
 * perf_counter around the call, test_emd_gpu.py:154-183). */
int32_t eemd_run_traced(const eemd_params* p, const void* x, const int64_t* lengths,
                        int32_t n_signals, int32_t trial_begin, int32_t trial_count,
                        const void* noise, void* imfs, void* resid_out,
                        double* imf_sum, int32_t* mode_count,
                        int32_t* nsift, int32_t* nmode, int32_t* mode_sifts,
                        int32_t* knot_log, int32_t* flags,
                        void* ws, size_t ws_bytes, void* stream,
                        eemd_kernel_times* times);

/* Size of the device scratch eemd_run_static() owns: a file-scope array in the
 * library, present on every GPU that loads the library until the process exits. */
#define EEMD_STATIC_SCRATCH_BYTES (64u * 1024u * 1024u)

/* eemd_run() without a workspace argument, for callers that cannot allocate
 * device memory themselves: host applications whose device memory is owned by
 * another allocator or framework (a memory pool that hands out no raw
 * buffers, a plugin host that forbids device allocations from plugins), or
 * code that has no allocator at hand at all.  The engine's scratch is the
 * library's own static device array of EEMD_STATIC_SCRATCH_BYTES; problems
 * whose eemd_workspace_size() exceeds it are rejected with
 * EEMD_E_STATIC_CAPACITY before any GPU work.  The caller still passes x and
 * the outputs.  The first call on each device looks the array up
 * (cudaGetSymbolAddress with that device current) and caches the address for
 * the life of the process, so make that first call before any stream capture,
 * and do not reset the device (cudaDeviceReset) between calls: the cached
 * address would then be stale.  The call is synchronous like eemd_run(): it
 * copies the task descriptors from host memory, waits for the stream and reads
 * the device status back.  All calls share the one array and it keeps the
 * previous call's contents (the engine re-initialises what it reads), so calls
 * that overlap on the GPU -- on different streams or host threads -- race and
 * must be serialised by the caller.  No cudaMalloc, cudaFree or allocating
 * library routine is called.  No counterpart in the reference. */
int32_t eemd_run_static(const eemd_params* p, const void* x, const int64_t* lengths,
                        int32_t n_signals, int32_t trial_begin, int32_t trial_count,
                        const void* noise, void* imfs, void* resid_out,
                        double* imf_sum, int32_t* mode_count,
                        int32_t* nsift, int32_t* nmode, int32_t* mode_sifts,
                        int32_t* knot_log, int32_t* flags, void* stream);

/* Ensemble mean and residual from the accumulated sums (emd_par.py:248-250):
 *   imf_mean[s][m][n] = imf_sum[s][m][n] / max(mode_count[s][m], 1)
 *   residual[s][n]    = x[s][n] - (sum over m < n_modes[s] of imf_mean)
 * n_modes[s] (device int32, out) = number of modes with mode_count > 0.
 * x is the original signal (dtype); imf_mean and residual are float64.
 * Synchronises `stream` before returning (the outputs are complete). */
int32_t eemd_finalize(const eemd_params* p, const void* x,
                      const int64_t* lengths, int32_t n_signals,
                      const double* imf_sum, const int32_t* mode_count,
                      double* imf_mean, double* residual, int32_t* n_modes,
                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EEMD_B200_H */
