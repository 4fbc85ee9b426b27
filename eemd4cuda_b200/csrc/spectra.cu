// spectra.cu -- the IMF spectra stage on the device (sm_100a): Hilbert
// instantaneous frequency / amplitude and the STFT of batched float64 rows.
//
// Hilbert:  x -> (copy) -> cuFFT D2Z -> k_analytic (one-sided spectrum to the
//           full analytic spectrum, weights 1 / 2 / 0, 1/N) -> cuFFT Z2Z
//           inverse in place -> k_if_amp (phase differences wrapped as
//           np.unwrap does, centred differences as np.gradient does, |z|).
//           The frequency needs only neighbouring phase differences, so no
//           scan over the unwrapped phase is formed.
// STFT:     x -> k_frames (zero-extended by nperseg/2 at both ends, periodic
//           Hann window) -> cuFFT D2Z batched over rows x frames ->
//           k_stft_out (transpose to [F][T], divide by the window sum).
// The FFTs are library calls; everything between them is one pass per step.
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <tuple>

#include "../../include/eemd_spectra.h"

namespace sp {

constexpr double PI = 3.141592653589793238462643383279502884;

// full analytic spectrum from the one-sided one: z[k] = w_k X[k] / N with
// w = 1 at DC (and at N/2 for even N), 2 on 1 <= k < N/2 (k < (N+1)/2 for
// odd N), 0 above
__global__ void k_analytic(const double2* __restrict__ half, double2* full, int M, int64_t N) {
    const int64_t H = N / 2 + 1;
    const int64_t total = (int64_t)M * N;
    const double inv = 1.0 / (double)N;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = i / N, k = i % N;
        double w;
        if (k == 0) w = 1.0;
        else if ((N & 1) == 0 && k == N / 2) w = 1.0;
        else if (2 * k < N) w = 2.0;
        else w = 0.0;
        double2 z = make_double2(0.0, 0.0);
        if (w != 0.0) {
            const double2 X = half[m * H + k];
            z = make_double2(X.x * w * inv, X.y * w * inv);
        }
        full[i] = z;
    }
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

// frames[m][j][n] = w[n] * x[m][j*step + n - half] (zero outside the row)
__global__ void k_frames(const double* __restrict__ x, double* frames, int M, int64_t N, int nperseg, int step,
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
        frames[i] = (s >= 0 && s < N) ? x[m * N + s] * w : 0.0;
    }
}

// Z[m][f][t] = spec[m][t][f] / wsum
__global__ void k_stft_out(const double2* __restrict__ spec, double2* Z, int M, int F, int T, double inv_wsum) {
    const int64_t total = (int64_t)M * F * T;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int t = (int)(i % T);
        const int64_t mf = i / T;
        const int f = (int)(mf % F);
        const int64_t m = mf / F;
        const double2 v = spec[(m * T + t) * F + f];
        Z[i] = make_double2(v.x * inv_wsum, v.y * inv_wsum);
    }
}

// ---------------------------------------------------------------------------
// cuFFT plans, cached per (device, type, n, batch); no automatic work area
// ---------------------------------------------------------------------------
struct Plan {
    cufftHandle h = 0;
    size_t work = 0;
};

std::mutex g_mu;
std::map<std::tuple<int, int, long long, long long>, Plan> g_plans;

int get_plan(cufftType type, long long n, long long batch, Plan& out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return EEMD_SP_E_CUDA;
    const auto key = std::make_tuple(dev, (int)type, n, batch);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
        out = it->second;
        return EEMD_SP_OK;
    }
    Plan p;
    if (cufftCreate(&p.h) != CUFFT_SUCCESS) return EEMD_SP_E_CUFFT;
    if (cufftSetAutoAllocation(p.h, 0) != CUFFT_SUCCESS) {
        cufftDestroy(p.h);
        return EEMD_SP_E_CUFFT;
    }
    long long nn = n;
    if (cufftMakePlanMany64(p.h, 1, &nn, nullptr, 1, 0, nullptr, 1, 0, type, batch, &p.work) != CUFFT_SUCCESS) {
        cufftDestroy(p.h);
        return EEMD_SP_E_CUFFT;
    }
    g_plans[key] = p;
    out = p;
    return EEMD_SP_OK;
}

// runs one transform with the plan's work area at `work` (under the cache lock:
// the stream and the work area are plan state)
int exec_plan(const Plan& p, cufftType type, void* in, void* out, int dir, void* work, cudaStream_t st) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (cufftSetStream(p.h, st) != CUFFT_SUCCESS) return EEMD_SP_E_CUFFT;
    if (cufftSetWorkArea(p.h, work) != CUFFT_SUCCESS) return EEMD_SP_E_CUFFT;
    cufftResult r;
    if (type == CUFFT_D2Z)
        r = cufftExecD2Z(p.h, static_cast<cufftDoubleReal*>(in), static_cast<cufftDoubleComplex*>(out));
    else
        r = cufftExecZ2Z(p.h, static_cast<cufftDoubleComplex*>(in), static_cast<cufftDoubleComplex*>(out), dir);
    return r == CUFFT_SUCCESS ? EEMD_SP_OK : EEMD_SP_E_CUFFT;
}

size_t al(size_t b) { return (b + 255) / 256 * 256; }

unsigned grid_for(int64_t total) {
    const int64_t b = (total + 255) / 256;
    return (unsigned)(b < 148 * 32 ? (b > 0 ? b : 1) : 148 * 32);
}

struct HilbertLayout {
    size_t copy, half, full, work, total;
    Plan fwd, inv;
};

int hilbert_layout(int M, int64_t N, HilbertLayout& L) {
    if (M < 1 || N < 2) return EEMD_SP_E_BADARG;
    int rc = get_plan(CUFFT_D2Z, N, M, L.fwd);
    if (rc) return rc;
    rc = get_plan(CUFFT_Z2Z, N, M, L.inv);
    if (rc) return rc;
    L.copy = al((size_t)M * N * sizeof(double));
    L.half = al((size_t)M * (N / 2 + 1) * sizeof(double2));
    L.full = al((size_t)M * N * sizeof(double2));
    L.work = al(L.fwd.work > L.inv.work ? L.fwd.work : L.inv.work);
    L.total = L.copy + L.half + L.full + L.work;
    return EEMD_SP_OK;
}

struct StftLayout {
    int F, T, step;
    size_t frames, spec, work, total;
    Plan fwd;
};

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

int stft_layout(int M, int64_t N, int nperseg, int noverlap, StftLayout& L) {
    if (M < 1) return EEMD_SP_E_BADARG;
    int rc = stft_shape(N, nperseg, noverlap, L.F, L.T);
    if (rc) return rc;
    L.step = nperseg - noverlap;
    rc = get_plan(CUFFT_D2Z, nperseg, (long long)M * L.T, L.fwd);
    if (rc) return rc;
    L.frames = al((size_t)M * L.T * nperseg * sizeof(double));
    L.spec = al((size_t)M * L.T * L.F * sizeof(double2));
    L.work = al(L.fwd.work);
    L.total = L.frames + L.spec + L.work;
    return EEMD_SP_OK;
}

}  // namespace sp

using namespace sp;

extern "C" {

int32_t eemd_sp_version(void) { return EEMD_SP_ABI_VERSION; }

int32_t eemd_sp_hilbert_workspace(int32_t M, int64_t N, size_t* bytes) {
    if (!bytes) return EEMD_SP_E_BADARG;
    HilbertLayout L;
    const int rc = hilbert_layout(M, N, L);
    if (rc) return rc;
    *bytes = L.total;
    return EEMD_SP_OK;
}

int32_t eemd_sp_hilbert_if(const double* x, int32_t M, int64_t N, double sr, double* inst_freq, double* inst_amp,
                           void* ws, size_t ws_bytes, void* stream) {
    if (!x || !inst_freq || !inst_amp || !ws || !(sr > 0.0)) return EEMD_SP_E_BADARG;
    HilbertLayout L;
    int rc = hilbert_layout(M, N, L);
    if (rc) return rc;
    if (ws_bytes < L.total) return EEMD_SP_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(ws);
    double* copy = reinterpret_cast<double*>(base);
    double2* half = reinterpret_cast<double2*>(base + L.copy);
    double2* full = reinterpret_cast<double2*>(base + L.copy + L.half);
    void* work = base + L.copy + L.half + L.full;
    // the transform's input is a scratch copy: the caller's rows stay untouched
    if (cudaMemcpyAsync(copy, x, (size_t)M * N * sizeof(double), cudaMemcpyDeviceToDevice, st) != cudaSuccess)
        return EEMD_SP_E_CUDA;
    rc = exec_plan(L.fwd, CUFFT_D2Z, copy, half, 0, work, st);
    if (rc) return rc;
    k_analytic<<<grid_for((int64_t)M * N), 256, 0, st>>>(half, full, M, N);
    if (cudaGetLastError() != cudaSuccess) return EEMD_SP_E_CUDA;
    rc = exec_plan(L.inv, CUFFT_Z2Z, full, full, CUFFT_INVERSE, work, st);
    if (rc) return rc;
    k_if_amp<<<grid_for((int64_t)M * N), 256, 0, st>>>(full, inst_freq, inst_amp, M, N, sr);
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
    if (!bytes) return EEMD_SP_E_BADARG;
    StftLayout L;
    const int rc = stft_layout(M, N, nperseg, noverlap, L);
    if (rc) return rc;
    *bytes = L.total;
    return EEMD_SP_OK;
}

int32_t eemd_sp_stft(const double* x, int32_t M, int64_t N, int32_t nperseg, int32_t noverlap, double* Z, void* ws,
                     size_t ws_bytes, void* stream) {
    if (!x || !Z || !ws) return EEMD_SP_E_BADARG;
    StftLayout L;
    int rc = stft_layout(M, N, nperseg, noverlap, L);
    if (rc) return rc;
    if (ws_bytes < L.total) return EEMD_SP_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(ws);
    double* frames = reinterpret_cast<double*>(base);
    double2* spec = reinterpret_cast<double2*>(base + L.frames);
    void* work = base + L.frames + L.spec;
    // the window's sum, added in index order (as the reference's window sum is formed)
    double wsum = 0.0;
    for (int n = 0; n < nperseg; ++n) wsum += 0.5 - 0.5 * cos(2.0 * PI * (double)n / (double)nperseg);
    k_frames<<<grid_for((int64_t)M * L.T * nperseg), 256, 0, st>>>(x, frames, M, N, nperseg, L.step, L.T);
    if (cudaGetLastError() != cudaSuccess) return EEMD_SP_E_CUDA;
    rc = exec_plan(L.fwd, CUFFT_D2Z, frames, spec, 0, work, st);
    if (rc) return rc;
    k_stft_out<<<grid_for((int64_t)M * L.F * L.T), 256, 0, st>>>(spec, reinterpret_cast<double2*>(Z), M, L.F, L.T,
                                                                  1.0 / wsum);
    return cudaGetLastError() == cudaSuccess ? EEMD_SP_OK : EEMD_SP_E_CUDA;
}

}  // extern "C"
