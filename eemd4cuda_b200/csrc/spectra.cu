// spectra.cu -- the IMF spectra stage on the device (sm_100a): Hilbert
// instantaneous frequency / amplitude and the STFT of batched float64 rows.
//
// Hilbert:  x -> k_promote (complex rows) -> FFT -> k_analytic (weights
//           1 / 2 / 0 on DC (and Nyquist) / positive / negative frequencies,
//           1/N) -> inverse FFT -> k_if_amp (phase differences wrapped as
//           np.unwrap does, centred differences as np.gradient does, |z|).
//           The frequency needs only neighbouring phase differences, so no
//           scan over the unwrapped phase is formed.
// STFT:     x -> k_frames (zero-extended by nperseg/2 at both ends, periodic
//           Hann window, complex rows) -> FFT batched over rows x frames ->
//           k_stft_out (one-sided half, transposed to [F][T], divided by the
//           window sum).
// The FFTs are this file's own (below): no FFT library is linked.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "../../include/eemd_spectra.h"

namespace sp {

constexpr double PI = 3.141592653589793238462643383279502884;

// analytic spectrum from the full one: z[k] = w_k X[k] / N with w = 1 at DC
// (and at N/2 for even N), 2 on 1 <= k < N/2 (k < (N+1)/2 for odd N), 0 above
__global__ void k_analytic(const double2* __restrict__ spec, double2* out, int M, int64_t N) {
    const int64_t total = (int64_t)M * N;
    const double inv = 1.0 / (double)N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t k = i % N;
        double w;
        if (k == 0) w = 1.0;
        else if ((N & 1) == 0 && k == N / 2) w = 1.0;
        else if (2 * k < N) w = 2.0;
        else w = 0.0;
        double2 z = make_double2(0.0, 0.0);
        if (w != 0.0) {
            const double2 X = spec[i];
            z = make_double2(X.x * w * inv, X.y * w * inv);
        }
        out[i] = z;
    }
}

// complex rows from real ones
__global__ void k_promote(const double* __restrict__ x, double2* z, int64_t total) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        z[i] = make_double2(x[i], 0.0);
}

// the unwrapped difference of two wrapped phases (np.unwrap, period 2 pi,
// discont pi): dd itself when |dd| < pi, else dd taken into [-pi, pi) with
// -pi mapped to pi when dd > 0
__device__ __forceinline__ double unwrap_diff(double dd) {
    if (fabs(dd) < PI) return dd;
    const double a = dd + PI, b = 2.0 * PI;
    double r = fmod(a, b);
    if (r != 0.0 && r < 0.0) r += b;  // floor-mod as numpy's mod
    double d = r - PI;
    if (d == -PI && dd > 0.0) d = PI;
    return d;
}

__global__ void k_if_amp(const double2* __restrict__ z, double* inst_freq, double* inst_amp, int M, int64_t N,
                         double sr) {
    const int64_t total = (int64_t)M * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t n = i % N;
        const double2 c = z[i];
        const double p = atan2(c.y, c.x);
        double f;
        if (n == 0) {
            const double2 r = z[i + 1];
            f = unwrap_diff(atan2(r.y, r.x) - p) * sr;
        } else if (n == N - 1) {
            const double2 l = z[i - 1];
            f = unwrap_diff(p - atan2(l.y, l.x)) * sr;
        } else {
            const double2 l = z[i - 1], r = z[i + 1];
            f = (unwrap_diff(p - atan2(l.y, l.x)) + unwrap_diff(atan2(r.y, r.x) - p)) * sr * 0.5;
        }
        inst_freq[i] = f / (2.0 * PI);
        inst_amp[i] = hypot(c.x, c.y);
    }
}

// frames[m][j][n] = w[n] * x[m][j*step + n - half] (zero outside the row), complex
__global__ void k_frames(const double* __restrict__ x, double2* frames, int M, int64_t N, int nperseg, int step,
                         int T) {
    const int half = nperseg / 2;
    const int64_t total = (int64_t)M * T * nperseg;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int n = (int)(i % nperseg);
        const int64_t mj = i / nperseg;
        const int j = (int)(mj % T);
        const int64_t m = mj / T;
        const int64_t s = (int64_t)j * step + n - half;
        const double w = 0.5 - 0.5 * cos(2.0 * PI * (double)n / (double)nperseg);
        frames[i] = make_double2((s >= 0 && s < N) ? x[m * N + s] * w : 0.0, 0.0);
    }
}

// Z[m][f][t] = spec[m][t][f] / wsum (f < F of each frame's nperseg bins)
__global__ void k_stft_out(const double2* __restrict__ spec, double2* Z, int M, int F, int T, int nperseg,
                           double inv_wsum) {
    const int64_t total = (int64_t)M * F * T;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(i % T);
        const int64_t mf = i / T;
        const int f = (int)(mf % F);
        const int64_t m = mf / F;
        const double2 v = spec[(m * T + t) * nperseg + f];
        Z[i] = make_double2(v.x * inv_wsum, v.y * inv_wsum);
    }
}

size_t al(size_t b) { return (b + 255) / 256 * 256; }

unsigned grid_for(int64_t total) {
    const int64_t b = (total + 255) / 256;
    return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

// ---------------------------------------------------------------------------
// Complex FFT of batched rows, this library's own (no FFT library):
// Stockham autosort passes of radix 4, 2, 3, 5 and of the odd primes up to 31
// (the formulation of Govindaraju et al., "High performance discrete Fourier
// transforms on graphics processors", SC'08: pass s reads x[j + q N/R],
// multiplies by the twiddle w^(q k) of the current sub-transform length
// Ns R (k = j mod Ns), takes a radix-R DFT and writes the results sorted, so
// no bit reversal is needed); a length with a prime factor above 31 goes
// through Bluestein's chirp-z identity, n k = (n^2 + k^2 - (k-n)^2) / 2, as a
// circular convolution of power-of-two length.  Unnormalised; sign -1 is the
// forward transform X[k] = sum_n x[n] exp(-2 pi i n k / N) (numpy's and
// scipy's), +1 the inverse.  Twiddles and chirps are formed on the fly with
// sincospi of an exactly reduced argument.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
// i * sign * z
__device__ __forceinline__ double2 cisg(double2 z, int sign) {
    return sign < 0 ? make_double2(z.y, -z.x) : make_double2(-z.y, z.x);
}
// exp(sign 2 pi i num / den), num reduced exactly into [0, den)
__device__ __forceinline__ double2 twiddle(int64_t num, int64_t den, int sign) {
    int64_t r = num % den;
    if (r < 0) r += den;
    double s, c;
    sincospi(2.0 * ((double)r / (double)den), &s, &c);
    return make_double2(c, sign < 0 ? -s : s);
}

template <int R>
__device__ __forceinline__ void dft_small(double2 (&a)[R], int sign) {
    if constexpr (R == 2) {
        const double2 t = a[1];
        a[1] = csub(a[0], t);
        a[0] = cadd(a[0], t);
    } else if constexpr (R == 3) {
        // w = exp(sign 2 pi i / 3) = -1/2 + sign i sqrt(3)/2
        const double h = 0.86602540378443864676;  // sqrt(3) / 2
        const double2 t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
        const double2 m = make_double2(fma(-0.5, t1.x, a[0].x), fma(-0.5, t1.y, a[0].y));
        const double2 r = cisg(make_double2(h * t2.x, h * t2.y), sign);
        a[0] = cadd(a[0], t1);
        a[1] = cadd(m, r);
        a[2] = csub(m, r);
    } else if constexpr (R == 4) {
        const double2 t0 = cadd(a[0], a[2]), t1 = csub(a[0], a[2]);
        const double2 t2 = cadd(a[1], a[3]), t3 = cisg(csub(a[1], a[3]), sign);
        a[0] = cadd(t0, t2);
        a[2] = csub(t0, t2);
        a[1] = cadd(t1, t3);
        a[3] = csub(t1, t3);
    } else if constexpr (R == 5) {
        // cos and sin of 2 pi / 5 and 4 pi / 5 from their closed forms
        const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        const double2 t1 = cadd(a[1], a[4]), t2 = cadd(a[2], a[3]);
        const double2 t3 = csub(a[1], a[4]), t4 = csub(a[2], a[3]);
        const double2 m1 = make_double2(a[0].x + c1 * t1.x + c2 * t2.x, a[0].y + c1 * t1.y + c2 * t2.y);
        const double2 m2 = make_double2(a[0].x + c2 * t1.x + c1 * t2.x, a[0].y + c2 * t1.y + c1 * t2.y);
        const double2 r1 = cisg(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), sign);
        const double2 r2 = cisg(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), sign);
        a[0] = cadd(a[0], cadd(t1, t2));
        a[1] = cadd(m1, r1);
        a[4] = csub(m1, r1);
        a[2] = cadd(m2, r2);
        a[3] = csub(m2, r2);
    }
}

// butterfly j of a Stockham pass of radix R over one row of N (nb = N / R):
// reads x[j + q nb], twiddles by w^(q k) of the sub-transform length Ns R
// (k = j mod Ns), takes the radix-R DFT and writes y[(j / Ns) Ns R + k + q Ns]
// twiddles formed on the fly
struct TwDirect {
    __device__ __forceinline__ double2 operator()(int64_t num, int64_t den, int sign) const {
        return twiddle(num, den, sign);
    }
};

// twiddles looked up in a table of exp(2 pi i m / n), m < n, made with the
// same sincospi arguments (m / n and r / den are the same correctly rounded
// quotient when r = m den / n), so the values are twiddle()'s bit for bit
struct TwTable {
    const double2* tab;
    int64_t n;
    __device__ __forceinline__ double2 operator()(int64_t num, int64_t den, int sign) const {
        int64_t r = num % den;
        if (r < 0) r += den;
        const double2 v = tab[r * (n / den)];
        return make_double2(v.x, sign < 0 ? -v.y : v.y);
    }
};

template <int R, typename TW = TwDirect>
__device__ __forceinline__ void bfly(const double2* x, double2* y, int64_t j, int64_t nb, int64_t Ns, int sign,
                                     const TW& tw = TW()) {
    const int64_t k = j % Ns;
    double2 a[R];
#pragma unroll
    for (int q = 0; q < R; ++q) a[q] = x[j + q * nb];
    if (Ns > 1) {
#pragma unroll
        for (int q = 1; q < R; ++q) a[q] = cmul(a[q], tw((int64_t)q * k, Ns * R, sign));
    }
    dft_small<R>(a, sign);
    const int64_t base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) y[base + q * Ns] = a[q];
}

// the same butterfly for an odd prime radix r <= 31 (a direct DFT of the r points)
__device__ __forceinline__ void bfly_prime(const double2* x, double2* y, int64_t j, int64_t nb, int64_t Ns, int r,
                                           int sign) {
    const int64_t k = j % Ns;
    double2 a[31];
    for (int q = 0; q < r; ++q) {
        a[q] = x[j + q * nb];
        if (q > 0 && Ns > 1) a[q] = cmul(a[q], twiddle((int64_t)q * k, Ns * r, sign));
    }
    const int64_t base = (j / Ns) * Ns * r + k;
    for (int q = 0; q < r; ++q) {
        double2 s = a[0];
        for (int p = 1; p < r; ++p) s = cadd(s, cmul(a[p], twiddle((int64_t)p * q, r, sign)));
        y[base + q * Ns] = s;
    }
}

template <typename TW>
__device__ __forceinline__ void bfly_any(const double2* x, double2* y, int64_t j, int64_t nb, int64_t Ns, int r,
                                         int sign, const TW& tw) {
    switch (r) {
        case 2: bfly<2>(x, y, j, nb, Ns, sign, tw); break;
        case 3: bfly<3>(x, y, j, nb, Ns, sign, tw); break;
        case 4: bfly<4>(x, y, j, nb, Ns, sign, tw); break;
        case 5: bfly<5>(x, y, j, nb, Ns, sign, tw); break;
        default: bfly_prime(x, y, j, nb, Ns, r, sign); break;
    }
}

// one Stockham pass of radix R over M rows of N: in -> out (distinct buffers)
template <int R>
__global__ void k_fft_pass(const double2* __restrict__ in, double2* __restrict__ out, int M, int64_t N, int64_t Ns,
                           int sign) {
    const int64_t nb = N / R;
    const int64_t total = (int64_t)M * nb;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / nb, j = i % nb;
        bfly<R>(in + m * N, out + m * N, j, nb, Ns, sign);
    }
}

__global__ void k_fft_pass_prime(const double2* __restrict__ in, double2* __restrict__ out, int M, int64_t N,
                                 int64_t Ns, int r, int sign) {
    const int64_t nb = N / r;
    const int64_t total = (int64_t)M * nb;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / nb, j = i % nb;
        bfly_prime(in + m * N, out + m * N, j, nb, Ns, r, sign);
    }
}

// ---------------------------------------------------------------------------
// One row per CTA in shared memory: every pass of a direct plan (no
// Bluestein) of length n <= SMEM_FFT_MAX in one launch, the two ping-pong
// buffers and a table of the n twiddles exp(2 pi i m / n) in shared memory
// (made once per CTA: n sincospi instead of (R - 1) n / R per pass).  The
// butterflies are the global passes' own (bfly, bfly_prime) and the table
// holds twiddle()'s values, so the results are the same bit for bit.
// ---------------------------------------------------------------------------
constexpr int SMEM_FFT_MAX = 4096;   // three arrays of n complex doubles: 192 KB
// one butterfly per thread in a radix-4 pass of 4096 (0.153 against 0.160 ms
// for the 48 kHz spectra step with 512 threads)
constexpr int SMEM_FFT_THREADS = 1024;
constexpr int SMEM_FFT_MAXRAD = 16;  // factors of n <= 4096 (at most 12)

struct SmemPlan {
    int n, nrad;
    int rad[SMEM_FFT_MAXRAD];
};

// tab[m] = exp(2 pi i m / n), m < n (twiddle()'s arithmetic)
__device__ void smem_twiddles(double2* tab, int n) {
    for (int m = threadIdx.x; m < n; m += blockDim.x) {
        double sv, cv;
        sincospi(2.0 * ((double)m / (double)n), &sv, &cv);
        tab[m] = make_double2(cv, sv);
    }
}

// the passes over `rows` rows of n at a stride of ld elements in a (b: the
// other buffer, tab: the twiddle table); returns the buffer holding the result
__device__ double2* smem_stockham(double2* a, double2* b, const double2* tab, const SmemPlan& P, int sign,
                                  int rows = 1, int ld = 0) {
    double2* cur = a;
    double2* dst = b;
    const TwTable tw{tab, P.n};
    int Ns = 1;
    for (int s = 0; s < P.nrad; ++s) {
        const int r = P.rad[s], nb = P.n / r;
        for (int j = threadIdx.x; j < rows * nb; j += blockDim.x) {
            const int row = j / nb, jj = j - row * nb;
            bfly_any(cur + row * ld, dst + row * ld, jj, nb, Ns, r, sign, tw);
        }
        __syncthreads();
        Ns *= r;
        double2* t = cur;
        cur = dst;
        dst = t;
    }
    return cur;
}

__global__ void __launch_bounds__(SMEM_FFT_THREADS) k_fft_smem(const double2* __restrict__ in, double2* out, int M,
                                                               const __grid_constant__ SmemPlan P, int sign) {
    extern __shared__ double2 sfft[];
    double2* a = sfft;
    double2* b = sfft + P.n;
    double2* tab = sfft + 2 * P.n;
    smem_twiddles(tab, P.n);
    for (int m = blockIdx.x; m < M; m += gridDim.x) {
        const double2* x = in + (int64_t)m * P.n;
        for (int i = threadIdx.x; i < P.n; i += blockDim.x) a[i] = x[i];
        __syncthreads();
        const double2* r = smem_stockham(a, b, tab, P, sign);
        double2* y = out + (int64_t)m * P.n;
        for (int i = threadIdx.x; i < P.n; i += blockDim.x) y[i] = r[i];
        __syncthreads();
    }
}

// The whole STFT of one frame per CTA iteration: frame (m, j) windowed into
// shared memory (k_frames' arithmetic), its transform, and bins f < F scaled
// into Z[m][f][j] (k_stft_out's arithmetic).
__global__ void __launch_bounds__(SMEM_FFT_THREADS) k_stft_smem(const double* __restrict__ x, double2* Z, int M,
                                                                int64_t N, int step, int T, int F, double inv_wsum,
                                                                const __grid_constant__ SmemPlan P) {
    extern __shared__ double2 sfft[];
    double2* a = sfft;
    double2* b = sfft + P.n;
    double2* tab = sfft + 2 * P.n;
    smem_twiddles(tab, P.n);
    const int nperseg = P.n, half = nperseg / 2;
    for (int64_t mj = blockIdx.x; mj < (int64_t)M * T; mj += gridDim.x) {
        const int j = (int)(mj % T);
        const int64_t m = mj / T;
        for (int n = threadIdx.x; n < nperseg; n += blockDim.x) {
            const int64_t s = (int64_t)j * step + n - half;
            const double w = 0.5 - 0.5 * cos(2.0 * PI * (double)n / (double)nperseg);
            a[n] = make_double2((s >= 0 && s < N) ? x[m * N + s] * w : 0.0, 0.0);
        }
        __syncthreads();
        const double2* r = smem_stockham(a, b, tab, P, -1);
        for (int f = threadIdx.x; f < F; f += blockDim.x) {
            const double2 v = r[f];
            Z[(m * F + f) * T + j] = make_double2(v.x * inv_wsum, v.y * inv_wsum);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Rows longer than SMEM_FFT_MAX whose length splits as N = N1 N2 with both
// factors direct shared-memory lengths: the four-step transform (Bailey),
//     X[k1 + N1 k2] = sum_n2 W_N2^(n2 k2) W_N^(n2 k1) sum_n1 x[n1 N2 + n2] W_N1^(n1 k1),
// in two launches with the transposes folded into their loads and stores:
// k_fft4_cols transforms CB columns n2 of x (viewed as N1 x N2) per CTA
// iteration, multiplies by the twiddles W_N^(n2 k1) and writes Y[k1][n2];
// k_fft4_rows transforms KB rows k1 of Y and writes X[k1 + N1 k2].  Shared-
// memory rows are padded by one element (ld = n + 1) so that column-wise
// accesses spread over the banks.  The column kernel's load can promote real
// rows (the Hilbert transform's input) or apply the analytic-signal weights
// to a spectrum (its inverse transform), so those need no pass of their own.
// ---------------------------------------------------------------------------
// small CTAs with a few rows each, so that 8 rows of 48 000 give several
// hundred CTAs (with 96 KB per CTA they were 128 and 136: SMs stayed idle)
constexpr int FFT4_THREADS = 128;
constexpr size_t FFT4_SMEM = 24 * 1024;  // two padded buffers of the CTA's rows

struct Fft4Plan {
    SmemPlan p1, p2;  // column (N1) and row (N2) transforms
    int64_t n;        // N1 N2
    int cb, kb;       // columns / rows per CTA iteration
};

enum { LOAD_COMPLEX = 0, LOAD_REAL = 1, LOAD_ANALYTIC = 2 };

// element idx of row m of the column kernel's input
template <int LOAD>
__device__ __forceinline__ double2 fft4_load(const void* in, int64_t m, int64_t N, int64_t idx) {
    if constexpr (LOAD == LOAD_REAL) {
        return make_double2(static_cast<const double*>(in)[m * N + idx], 0.0);
    } else if constexpr (LOAD == LOAD_ANALYTIC) {
        // k_analytic's weights and scaling
        const int64_t k = idx;
        double w;
        if (k == 0) w = 1.0;
        else if ((N & 1) == 0 && k == N / 2) w = 1.0;
        else if (2 * k < N) w = 2.0;
        else w = 0.0;
        if (w == 0.0) return make_double2(0.0, 0.0);
        const double inv = 1.0 / (double)N;
        const double2 X = static_cast<const double2*>(in)[m * N + idx];
        return make_double2(X.x * w * inv, X.y * w * inv);
    } else {
        return static_cast<const double2*>(in)[m * N + idx];
    }
}

template <int LOAD>
__global__ void __launch_bounds__(FFT4_THREADS) k_fft4_cols(const void* __restrict__ in, double2* Y, int M,
                                                            const __grid_constant__ Fft4Plan F, int sign) {
    extern __shared__ double2 s4[];
    const int N1 = F.p1.n, N2 = F.p2.n, CB = F.cb, ld = N1 + 1;
    const int64_t N = F.n;
    double2* a = s4;
    double2* b = s4 + CB * ld;
    double2* tab = s4 + 2 * CB * ld;
    smem_twiddles(tab, N1);
    const int nblk = (N2 + CB - 1) / CB;
    for (int64_t blk = blockIdx.x; blk < (int64_t)M * nblk; blk += gridDim.x) {
        const int64_t m = blk / nblk;
        const int c0 = (int)(blk % nblk) * CB;
        const int cb = min(CB, N2 - c0);
        for (int i = threadIdx.x; i < N1 * CB; i += blockDim.x) {
            const int n1 = i / CB, c = i - n1 * CB;
            a[c * ld + n1] = c < cb ? fft4_load<LOAD>(in, m, N, (int64_t)n1 * N2 + c0 + c) : make_double2(0.0, 0.0);
        }
        __syncthreads();
        const double2* r = smem_stockham(a, b, tab, F.p1, sign, CB, ld);
        for (int i = threadIdx.x; i < N1 * CB; i += blockDim.x) {
            const int k1 = i / CB, c = i - k1 * CB;
            if (c < cb) {
                const int64_t n2 = c0 + c;
                Y[m * N + (int64_t)k1 * N2 + n2] = cmul(r[c * ld + k1], twiddle(n2 * k1, N, sign));
            }
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(FFT4_THREADS) k_fft4_rows(const double2* __restrict__ Y, double2* X, int M,
                                                            const __grid_constant__ Fft4Plan F, int sign) {
    extern __shared__ double2 s4[];
    const int N1 = F.p1.n, N2 = F.p2.n, KB = F.kb, ld = N2 + 1;
    const int64_t N = F.n;
    double2* a = s4;
    double2* b = s4 + KB * ld;
    double2* tab = s4 + 2 * KB * ld;
    smem_twiddles(tab, N2);
    const int nblk = (N1 + KB - 1) / KB;
    for (int64_t blk = blockIdx.x; blk < (int64_t)M * nblk; blk += gridDim.x) {
        const int64_t m = blk / nblk;
        const int k0 = (int)(blk % nblk) * KB;
        const int kb = min(KB, N1 - k0);
        for (int i = threadIdx.x; i < KB * N2; i += blockDim.x) {
            const int kk = i / N2, n2 = i - kk * N2;
            a[kk * ld + n2] = kk < kb ? Y[m * N + (int64_t)(k0 + kk) * N2 + n2] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        const double2* r = smem_stockham(a, b, tab, F.p2, sign, KB, ld);
        for (int i = threadIdx.x; i < KB * N2; i += blockDim.x) {
            const int k2 = i / KB, kk = i - k2 * KB;
            if (kk < kb) X[m * N + k0 + kk + (int64_t)N1 * k2] = r[kk * ld + k2];
        }
        __syncthreads();
    }
}


// Bluestein: chirp c_n = exp(sign pi i n^2 / N) (n^2 reduced mod 2N exactly)
__device__ __forceinline__ double2 chirp(int64_t n, int64_t N, int sign) {
    const int64_t r = (int64_t)(((unsigned long long)n * (unsigned long long)n) % (unsigned long long)(2 * N));
    double s, c;
    sincospi((double)r / (double)N, &s, &c);
    return make_double2(c, sign < 0 ? -s : s);
}

// a[m][n] = x[m][n] c_n for n < N, 0 up to L
__global__ void k_blue_pre(const double2* __restrict__ x, double2* a, int M, int64_t N, int64_t L, int sign) {
    const int64_t total = (int64_t)M * L;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / L, n = i % L;
        a[i] = n < N ? cmul(x[m * N + n], chirp(n, N, sign)) : make_double2(0.0, 0.0);
    }
}

// b[n] = conj(c_n) for n < N, b[L-n] = conj(c_n) for 0 < n < N, 0 elsewhere
__global__ void k_blue_kernel(double2* b, int64_t N, int64_t L, int sign) {
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < L; n += (int64_t)gridDim.x * blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (n < N) v = chirp(n, N, -sign);
        else if (L - n < N) v = chirp(L - n, N, -sign);
        b[n] = v;
    }
}

// A[m][n] *= B[n] / L
__global__ void k_blue_mul(double2* A, const double2* __restrict__ B, int M, int64_t L) {
    const int64_t total = (int64_t)M * L;
    const double inv = 1.0 / (double)L;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = cmul(A[i], B[i % L]);
        A[i] = make_double2(v.x * inv, v.y * inv);
    }
}

// y[m][k] = c_k C[m][k] for k < N
__global__ void k_blue_post(const double2* __restrict__ Cv, double2* y, int M, int64_t N, int64_t L, int sign) {
    const int64_t total = (int64_t)M * N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / N, k = i % N;
        y[i] = cmul(Cv[m * L + k], chirp(k, N, sign));
    }
}

struct FftPlan {
    int64_t n = 0, L = 0;        // length; Bluestein's power-of-two length (0 = direct)
    std::vector<int> radices;    // of n (direct) or of L (Bluestein)
};

bool factor(int64_t n, std::vector<int>& rad) {
    rad.clear();
    while (n % 4 == 0) { rad.push_back(4); n /= 4; }
    while (n % 2 == 0) { rad.push_back(2); n /= 2; }
    for (int p = 3; p <= 31; p += 2) {
        while (n % p == 0) { rad.push_back(p); n /= p; }
    }
    return n == 1;
}

FftPlan make_fft_plan(int64_t n) {
    FftPlan P;
    P.n = n;
    if (!factor(n, P.radices)) {
        int64_t L = 1;
        while (L < 2 * n - 1) L <<= 1;
        P.L = L;
        factor(L, P.radices);
    }
    return P;
}

// complex elements of scratch an FFT of M rows needs beyond its two ping-pong buffers
int64_t fft_extra(const FftPlan& P, int M) { return P.L ? 2 * (int64_t)M * P.L + 2 * P.L : 0; }

// the shared-memory plan of a length, or false when it runs as global passes
bool smem_plan(int64_t len, const std::vector<int>& rad, SmemPlan& sp) {
    if (len > SMEM_FFT_MAX || rad.empty() || rad.size() > (size_t)SMEM_FFT_MAXRAD) return false;
    sp.n = (int)len;
    sp.nrad = (int)rad.size();
    for (size_t i = 0; i < rad.size(); ++i) sp.rad[i] = rad[i];
    return true;
}

// shared memory of the one-row-per-CTA kernels (set once per kernel)
bool smem_ready(const void* fn) {
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(3 * SMEM_FFT_MAX * sizeof(double2))) == cudaSuccess;
}

unsigned smem_grid(int64_t rows) { return (unsigned)(rows < 65535 ? rows : 65535); }

// the Hann window's sum, added in index order (as the reference's window sum
// is formed); the last length's sum is kept per thread, since the host loop
// of nperseg cosines costs more than the STFT's launch
double window_sum(int nperseg) {
    thread_local int last_n = 0;
    thread_local double last_sum = 0.0;
    if (nperseg != last_n) {
        double wsum = 0.0;
        for (int n = 0; n < nperseg; ++n) wsum += 0.5 - 0.5 * cos(2.0 * PI * (double)n / (double)nperseg);
        last_n = nperseg;
        last_sum = wsum;
    }
    return last_sum;
}

// the four-step split of a length: N1 the divisor nearest below sqrt(n) with
// both N1 and n / N1 direct shared-memory lengths; false when there is none
bool fft4_plan(int64_t n, Fft4Plan& F) {
    if (n <= SMEM_FFT_MAX || n > (int64_t)SMEM_FFT_MAX * SMEM_FFT_MAX) return false;
    int64_t n1 = 1;
    while ((n1 + 1) * (n1 + 1) <= n) ++n1;
    for (; n1 >= 2; --n1) {
        if (n % n1) continue;
        const int64_t n2 = n / n1;
        if (n2 > SMEM_FFT_MAX) break;  // n2 only grows as n1 shrinks
        std::vector<int> r1, r2;
        if (!factor(n1, r1) || !factor(n2, r2) || !smem_plan(n1, r1, F.p1) || !smem_plan(n2, r2, F.p2)) continue;
        F.n = n;
        F.cb = (int)std::max<size_t>(1, FFT4_SMEM / (2 * (size_t)(n1 + 1) * sizeof(double2)));
        F.kb = (int)std::max<size_t>(1, FFT4_SMEM / (2 * (size_t)(n2 + 1) * sizeof(double2)));
        F.cb = (int)std::min<int64_t>(F.cb, n2);
        F.kb = (int)std::min<int64_t>(F.kb, n1);
        return true;
    }
    return false;
}

size_t fft4_cols_smem(const Fft4Plan& F) { return (2 * (size_t)F.cb * (F.p1.n + 1) + F.p1.n) * sizeof(double2); }
size_t fft4_rows_smem(const Fft4Plan& F) { return (2 * (size_t)F.kb * (F.p2.n + 1) + F.p2.n) * sizeof(double2); }

// largest shared memory a four-step launch asks for: one padded row of 4096
// in each buffer and its table
constexpr int FFT4_SMEM_MAX = (2 * (SMEM_FFT_MAX + 1) + SMEM_FFT_MAX) * (int)sizeof(double2);

bool fft4_ready() {
    const void* fns[] = {reinterpret_cast<const void*>(k_fft4_cols<LOAD_COMPLEX>),
                         reinterpret_cast<const void*>(k_fft4_cols<LOAD_REAL>),
                         reinterpret_cast<const void*>(k_fft4_cols<LOAD_ANALYTIC>),
                         reinterpret_cast<const void*>(k_fft4_rows)};
    for (const void* fn : fns)
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, FFT4_SMEM_MAX) != cudaSuccess)
            return false;
    return true;
}

// the two launches of a four-step transform of M rows: in -> y (columns), y -> out (rows)
template <int LOAD>
void fft4(const void* in, double2* y, double2* out, int M, const Fft4Plan& F, int sign, cudaStream_t st) {
    const int64_t nc = (int64_t)M * ((F.p2.n + F.cb - 1) / F.cb), nr = (int64_t)M * ((F.p1.n + F.kb - 1) / F.kb);
    k_fft4_cols<LOAD><<<smem_grid(nc), FFT4_THREADS, fft4_cols_smem(F), st>>>(in, y, M, F, sign);
    k_fft4_rows<<<smem_grid(nr), FFT4_THREADS, fft4_rows_smem(F), st>>>(y, out, M, F, sign);
}

// Stockham passes of length len over M rows: src -> (b1, b2 alternately); returns the result buffer
double2* stockham(const double2* src, double2* b1, double2* b2, int M, int64_t len, const std::vector<int>& rad,
                  int sign, cudaStream_t st) {
    const double2* cur = src;
    double2* dst = b1;
    int64_t Ns = 1;
    if (rad.empty()) {  // length 1: the transform is the identity
        cudaMemcpyAsync(b1, src, sizeof(double2) * (size_t)M * (size_t)len, cudaMemcpyDeviceToDevice, st);
        return b1;
    }
    SmemPlan sp;
    static const bool smem_ok = smem_ready(reinterpret_cast<const void*>(k_fft_smem));
    if (smem_ok && smem_plan(len, rad, sp)) {
        k_fft_smem<<<smem_grid(M), SMEM_FFT_THREADS, 3 * sp.n * sizeof(double2), st>>>(src, b1, M, sp, sign);
        return b1;
    }
    Fft4Plan f4;
    static const bool f4_ok = fft4_ready();
    if (f4_ok && fft4_plan(len, f4)) {
        // src -> b1 (columns), b1 -> b2 (rows): b2 may be src, which only the first launch reads
        fft4<LOAD_COMPLEX>(src, b1, b2, M, f4, sign, st);
        return b2;
    }
    for (int r : rad) {
        const unsigned g = grid_for((int64_t)M * (len / r));
        switch (r) {
            case 2: k_fft_pass<2><<<g, 256, 0, st>>>(cur, dst, M, len, Ns, sign); break;
            case 3: k_fft_pass<3><<<g, 256, 0, st>>>(cur, dst, M, len, Ns, sign); break;
            case 4: k_fft_pass<4><<<g, 256, 0, st>>>(cur, dst, M, len, Ns, sign); break;
            case 5: k_fft_pass<5><<<g, 256, 0, st>>>(cur, dst, M, len, Ns, sign); break;
            default: k_fft_pass_prime<<<g, 256, 0, st>>>(cur, dst, M, len, Ns, r, sign); break;
        }
        Ns *= r;
        cur = dst;
        dst = (dst == b1) ? b2 : b1;
    }
    return const_cast<double2*>(cur);
}

// FFT of M rows of length P.n: `in` is read only; b1, b2 hold M*n each and
// `extra` fft_extra(P, M) elements; returns the buffer (b1 or b2) with the result
double2* fft_rows(const double2* in, double2* b1, double2* b2, double2* extra, int M, const FftPlan& P, int sign,
                  cudaStream_t st) {
    if (!P.L) return stockham(in, b1, b2, M, P.n, P.radices, sign, st);
    const int64_t N = P.n, L = P.L;
    double2* A = extra;                 // M * L
    double2* T = extra + (int64_t)M * L;  // M * L
    double2* Bk = T + (int64_t)M * L;   // L
    double2* Bt = Bk + L;               // L
    k_blue_pre<<<grid_for((int64_t)M * L), 256, 0, st>>>(in, A, M, N, L, sign);
    k_blue_kernel<<<grid_for(L), 256, 0, st>>>(Bk, N, L, sign);
    double2* Af = stockham(A, T, A, M, L, P.radices, -1, st);
    double2* Bf = stockham(Bk, Bt, Bk, 1, L, P.radices, -1, st);
    k_blue_mul<<<grid_for((int64_t)M * L), 256, 0, st>>>(Af, Bf, M, L);
    double2* other = (Af == A) ? T : A;
    double2* Cv = stockham(Af, other, Af, M, L, P.radices, +1, st);
    k_blue_post<<<grid_for((int64_t)M * N), 256, 0, st>>>(Cv, b1, M, N, L, sign);
    return b1;
}

// three complex buffers of `rows` x `len` plus the FFT's extra scratch
struct FftLayout {
    FftPlan P;
    int64_t rows = 0;
    size_t buf = 0, extra = 0, total = 0;
};

int fft_layout(int64_t rows, int64_t len, FftLayout& L) {
    if (rows < 1 || len < 1 || rows > (1LL << 31)) return EEMD_SP_E_BADARG;
    L.P = make_fft_plan(len);
    L.rows = rows;
    L.buf = al((size_t)rows * (size_t)len * sizeof(double2));
    L.extra = al((size_t)fft_extra(L.P, (int)rows) * sizeof(double2));
    L.total = 3 * L.buf + L.extra;
    return EEMD_SP_OK;
}

struct Bufs {
    double2 *x, *y, *z, *extra;
};

Bufs carve(void* ws, const FftLayout& L) {
    char* base = static_cast<char*>(ws);
    Bufs b;
    b.x = reinterpret_cast<double2*>(base);
    b.y = reinterpret_cast<double2*>(base + L.buf);
    b.z = reinterpret_cast<double2*>(base + 2 * L.buf);
    b.extra = reinterpret_cast<double2*>(base + 3 * L.buf);
    return b;
}

int stft_shape(int64_t N, int nperseg, int noverlap, int& F, int& T) {
    if (N < 1 || nperseg < 2 || noverlap < 0 || noverlap >= nperseg) return EEMD_SP_E_BADARG;
    const int64_t ext = N + 2 * (int64_t)(nperseg / 2);
    if (ext < nperseg) return EEMD_SP_E_BADARG;
    const int64_t t = (ext - noverlap) / (nperseg - noverlap);
    if (t < 1 || t > (1LL << 30)) return EEMD_SP_E_BADARG;
    F = nperseg / 2 + 1;
    T = (int)t;
    return EEMD_SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" {

int32_t eemd_sp_version(void) { return EEMD_SP_ABI_VERSION; }

int32_t eemd_sp_fft_workspace(int32_t M, int64_t N, size_t* bytes) {
    if (!bytes) return EEMD_SP_E_BADARG;
    FftLayout L;
    const int rc = fft_layout(M, N, L);
    if (rc) return rc;
    *bytes = L.total;
    return EEMD_SP_OK;
}

int32_t eemd_sp_fft(const double* in, double* out, int32_t M, int64_t N, int32_t sign, void* ws, size_t ws_bytes,
                    void* stream) {
    if (!in || !out || !ws || (sign != -1 && sign != 1)) return EEMD_SP_E_BADARG;
    FftLayout L;
    int rc = fft_layout(M, N, L);
    if (rc) return rc;
    if (ws_bytes < L.total) return EEMD_SP_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Bufs b = carve(ws, L);
    const size_t nb = sizeof(double2) * (size_t)M * (size_t)N;
    if (cudaMemcpyAsync(b.x, in, nb, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return EEMD_SP_E_CUDA;
    double2* r = fft_rows(b.x, b.y, b.z, b.extra, M, L.P, sign, st);
    if (cudaMemcpyAsync(out, r, nb, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return EEMD_SP_E_CUDA;
    return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
}

int32_t eemd_sp_hilbert_workspace(int32_t M, int64_t N, size_t* bytes) {
    if (!bytes || N < 2) return EEMD_SP_E_BADARG;
    return eemd_sp_fft_workspace(M, N, bytes);
}

int32_t eemd_sp_hilbert_if(const double* x, int32_t M, int64_t N, double sr, double* inst_freq, double* inst_amp,
                           void* ws, size_t ws_bytes, void* stream) {
    if (!x || !inst_freq || !inst_amp || !ws || !(sr > 0.0) || N < 2) return EEMD_SP_E_BADARG;
    FftLayout L;
    int rc = fft_layout(M, N, L);
    if (rc) return rc;
    if (ws_bytes < L.total) return EEMD_SP_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Bufs b = carve(ws, L);
    const int64_t total = (int64_t)M * N;
    Fft4Plan f4;
    static const bool f4_ok = fft4_ready();
    if (f4_ok && !L.P.L && fft4_plan(N, f4)) {
        // four-step transforms with the real input and the analytic weights folded into their loads
        fft4<LOAD_REAL>(x, b.y, b.x, M, f4, -1, st);
        fft4<LOAD_ANALYTIC>(b.x, b.y, b.z, M, f4, +1, st);
        k_if_amp<<<grid_for(total), 256, 0, st>>>(b.z, inst_freq, inst_amp, M, N, sr);
        return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
    }
    // the caller's rows stay untouched: the transform runs on complex copies
    k_promote<<<grid_for(total), 256, 0, st>>>(x, b.x, total);
    double2* spec = fft_rows(b.x, b.y, b.z, b.extra, M, L.P, -1, st);
    k_analytic<<<grid_for(total), 256, 0, st>>>(spec, b.x, M, N);
    double2* z = fft_rows(b.x, b.y, b.z, b.extra, M, L.P, +1, st);
    k_if_amp<<<grid_for(total), 256, 0, st>>>(z, inst_freq, inst_amp, M, N, sr);
    return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
}

int32_t eemd_sp_stft_shape(int64_t N, int32_t nperseg, int32_t noverlap, int32_t* F, int32_t* T) {
    if (!F || !T) return EEMD_SP_E_BADARG;
    int f = 0, t = 0;
    const int rc = stft_shape(N, nperseg, noverlap, f, t);
    if (rc) return rc;
    *F = f;
    *T = t;
    return EEMD_SP_OK;
}

int32_t eemd_sp_stft_workspace(int32_t M, int64_t N, int32_t nperseg, int32_t noverlap, size_t* bytes) {
    if (!bytes || M < 1) return EEMD_SP_E_BADARG;
    int F = 0, T = 0;
    int rc = stft_shape(N, nperseg, noverlap, F, T);
    if (rc) return rc;
    FftLayout L;
    rc = fft_layout((int64_t)M * T, nperseg, L);
    if (rc) return rc;
    *bytes = L.total;
    return EEMD_SP_OK;
}

int32_t eemd_sp_stft(const double* x, int32_t M, int64_t N, int32_t nperseg, int32_t noverlap, double* Z, void* ws,
                     size_t ws_bytes, void* stream) {
    if (!x || !Z || !ws || M < 1) return EEMD_SP_E_BADARG;
    int F = 0, T = 0;
    int rc = stft_shape(N, nperseg, noverlap, F, T);
    if (rc) return rc;
    FftLayout L;
    rc = fft_layout((int64_t)M * T, nperseg, L);
    if (rc) return rc;
    if (ws_bytes < L.total) return EEMD_SP_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const Bufs b = carve(ws, L);
    const double wsum = window_sum(nperseg);
    SmemPlan sp;
    static const bool smem_ok = smem_ready(reinterpret_cast<const void*>(k_stft_smem));
    if (smem_ok && !L.P.L && smem_plan(nperseg, L.P.radices, sp)) {
        // one launch: frames, their transforms and the scaled bins
        k_stft_smem<<<smem_grid((int64_t)M * T), SMEM_FFT_THREADS, 3 * sp.n * sizeof(double2), st>>>(
            x, reinterpret_cast<double2*>(Z), M, N, nperseg - noverlap, T, F, 1.0 / wsum, sp);
        return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
    }
    k_frames<<<grid_for((int64_t)M * T * nperseg), 256, 0, st>>>(x, b.x, M, N, nperseg, nperseg - noverlap, T);
    double2* spec = fft_rows(b.x, b.y, b.z, b.extra, M * T, L.P, -1, st);
    k_stft_out<<<grid_for((int64_t)M * F * T), 256, 0, st>>>(spec, reinterpret_cast<double2*>(Z), M, F, T, nperseg,
                                                             1.0 / wsum);
    return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
}

}  // extern "C"
