// eemd_engine.cu -- sm_100a EEMD engine: kernels and the C ABI (include/eemd_b200.h).
//
// Reference algorithm (misureaudio/EEMD4CUDA):
//   emd_ref.py:31-48    interior tridiagonal system of the natural cubic spline
//   emd_ref.py:50-65    no-pivot Thomas solve
//   emd_ref.py:67-75    spline evaluation (searchsorted interval, cubic in a, b)
//   emd_ref.py:77-103   envelope through strict maxima / minima, mirror ends
//   emd_ref.py:108-156  emd_1d: IMF loop, sift loop, SD stop rule
//   emd_gpu.py:120-285  numba kernel: same loop, one block per trial
//   emd_gpu_v5_dsbt.py:51-74, 77-115  seam-window Thomas and tile extrema scan
//   emd_par.py:198-254  ensemble noise and per-mode masked mean
//
// Numerics.  exact=1 reproduces the reference's float64 operation order
// (separately rounded products, IEEE divisions, serial-Thomas recurrences;
// the file is compiled with --fmad=false so the compiler never contracts
// a*b+c).  exact=0 uses explicit fma(), a Newton-refined reciprocal per row,
// a twisted (two-sided) seam-window factorisation held in registers, and the
// monomial form of each spline interval.
#include "../../include/eemd_b200.h"
#include "eemd_internal.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <climits>
#include <mutex>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

namespace cg = cooperative_groups;

namespace eemd {

// ---------------------------------------------------------------------------
// small device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ void raise_error(Header* h, int code, int info) {
    if (atomicCAS(&h->error, 0, code) == 0) h->error_info = info;
}

template <typename T>
__device__ __forceinline__ double ldv(const void* p, int64_t i) {
    return (double)(static_cast<const T*>(p)[i]);
}

// value rounded to the storage type, held in double
template <typename T>
__device__ __forceinline__ double rnd(double v) { return (double)(T)v; }

// fused multiply-add in the storage type
__device__ __forceinline__ float fmat(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return __fma_rn(a, b, c); }

// knot sample index kept in a storage-type record plane as an integer bit pattern
template <typename T>
__device__ __forceinline__ T tbits(int t) {
    if constexpr (sizeof(T) == 4) return __int_as_float(t);
    else return __longlong_as_double((long long)t);
}
template <typename T>
__device__ __forceinline__ int tint(T v) {
    if constexpr (sizeof(T) == 4) return __float_as_int(v);
    else return (int)__double_as_longlong(v);
}

// 1/x: hardware approximation refined by one Newton step on f(y) = 1/y - x,
// y <- y + y(1 - xy); relative error about 2^-50 or better.
__device__ __forceinline__ double fast_rcp(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double e = fma(-x, y, 1.0);
    return fma(y, e, y);
}

// Asynchronous global->shared copies (sm_80+ cp.async): a thread issues its
// copies, commits them as a group and later waits for the group.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_el(T* smem, const T* gmem) {
    if (sizeof(T) == 8) cp_async8(smem, gmem);
    else cp_async4(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// emd_ref.py:67-75 (and emd_gpu.py:96-100), reference operation order
__device__ __forceinline__ double spline_exact(double t, double tl, double tr, double yl, double yr,
                                               double Ml, double Mr) {
    double h = tr - tl;
    double a = (tr - t) / h;
    double b = (t - tl) / h;
    double a3 = a * a * a;
    double b3 = b * b * b;
    return (a * yl + b * yr) + (((a3 - a) * Ml + (b3 - b) * Mr) * (h * h)) / 6.0;
}

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and Box-Muller normals
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// standard normal number for sample t of (signal, trial)
__device__ __forceinline__ double philox_normal(uint64_t seed, int signal, int trial, int64_t t) {
    uint4 ctr = make_uint4((uint32_t)(t >> 1), (uint32_t)trial, (uint32_t)signal, 0x45454D44u);
    uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    uint4 r = philox4x32_10(ctr, key);
    uint64_t a = (((uint64_t)r.x << 32) | r.y) >> 11;
    uint64_t b = (((uint64_t)r.z << 32) | r.w) >> 11;
    double u1 = ((double)a + 1.0) * 0x1.0p-53;  // (0, 1]
    double u2 = (double)b * 0x1.0p-53;          // [0, 1)
    double rad = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    return (t & 1) ? rad * s : rad * c;
}

// ---------------------------------------------------------------------------
// block reductions (fixed order => deterministic)
// ---------------------------------------------------------------------------
template <int NT>
__device__ __forceinline__ double2 block_sum2(double2 v, double2* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_down_sync(0xffffffffu, v.x, o);
        v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    if (wid == 0) {
        v = (lane < NT / 32) ? sh[lane] : make_double2(0.0, 0.0);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            v.x += __shfl_down_sync(0xffffffffu, v.x, o);
            v.y += __shfl_down_sync(0xffffffffu, v.y, o);
        }
    }
    __syncthreads();
    return v;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// k_sigma: per-signal eps*std(x) (population std, emd_par.py:117, 225)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(1024) k_sigma(const SignalDesc* sdesc, const void* xv, double eps,
                                                double* sigma_out) {
    __shared__ double2 sh[32];
    __shared__ double mean_s;
    const int s = blockIdx.x;
    const SignalDesc d = sdesc[s];
    const T* x = static_cast<const T*>(xv) + d.x_off;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < d.n; i += 1024) acc += (double)x[i];
    double2 r = block_sum2<1024>(make_double2(acc, 0.0), sh);
    if (threadIdx.x == 0) mean_s = r.x / (double)d.n;
    __syncthreads();
    const double mean = mean_s;
    acc = 0.0;
    for (int64_t i = threadIdx.x; i < d.n; i += 1024) {
        const double dv = (double)x[i] - mean;
        acc += dv * dv;
    }
    r = block_sum2<1024>(make_double2(acc, 0.0), sh);
    if (threadIdx.x == 0) sigma_out[s] = eps * sqrt(r.x / (double)d.n);
}

// ---------------------------------------------------------------------------
// per-CTA task context (shared memory)
// ---------------------------------------------------------------------------
struct Xchg {              // one CTA's published segment results (DSMEM-visible)
    double hf[2], hl[2];   // h after the step: first two / last two samples of the segment
    double rf[2], rl[2];   // residual after the step: same positions
    double num, den;       // SD partial sums of the segment
    int cnt[2];            // new knots (maxima, minima) found in the segment
};

struct TaskSm {
    int task, n, s0, s1, rank, csize;
    int phase, imf, sift, kpar, src_resid, imf_from_resid;
    int nsift_total, nmode, mode_sifts_cur, flags, step, mode;
    int P[2];                  // current knot totals
    int pref[2][MAXC + 1];     // current knots before each segment
    int mir[2], p2[2], tfirst[2], tlast[2];
    double yfirst[2], ylast[2];  // values of the virtual mirror knots
    double cval[2];            // constant envelope when P == 1
    // sweep scalars
    int left_knot[2];
    int run_cur[2], run_new[2];
    double hold_m1, hold_m2, rold_m1, rold_p, hold_p, f_m1, g_m1;
    double hf0, hf1, rf0, rf1;
    double fl, gl, fr, gr;     // new value / new residual at the tile's halo samples
    double f_last2, g_last2;   // new value / residual at the tile's second-to-last sample
};

struct Smem {
    void* hT[2];     // [TILE+8] old h, storage type (double buffer; the tile's sample 0 sits at
                     //          index TOFF + (16-byte phase of its global address), so that
                     //          16-byte copies line up; left halo just before, right halo after)
    void* rT[2];     // [TILE+8] residual, storage type (double buffer, same placement)
    void* kt;        // [2][cap] staged interval records, storage type: knot index bit pattern
    void* c[4];      // [2][cap] fast: monomial c0..c3 of the interval; exact: c[0] = y, c[1] = M
    int* skt;        // solve staging (padded): knot sample index
    void* sky;       // solve staging (padded): knot value, storage type
    double* ssl;     // solve staging (padded): slope of the interval starting at the knot
    int cap;
};

constexpr int RUN_MAX = 4;            // consecutive samples per thread in a tile
constexpr int NWARP = THREADS / 32;
constexpr int TOFF = 4;               // tile buffer index of the first 16-byte boundary used

__host__ __device__ inline int stage_pad(int k) { return k + (k >> 4); }

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

__host__ __device__ inline size_t smem_bytes(int TILE, int bt) {
    const size_t cap = (size_t)(TILE >> 1) + 8;
    const size_t tile = align16((size_t)(TILE + 8) * bt);
    const size_t sweep = 4 * tile + 10 * align16(cap * bt);
    const size_t sp = (size_t)stage_pad(SOLVE_CAP);
    const size_t solve = align16(sp * 8) + align16(sp * 4) + align16(sp * bt);
    return sweep > solve ? sweep : solve;
}

template <typename T>
__device__ __forceinline__ Smem carve(unsigned char* base, int TILE) {
    Smem m;
    const size_t cap = (size_t)(TILE >> 1) + 8;
    m.cap = (int)cap;
    const size_t tile = align16((size_t)(TILE + 8) * sizeof(T));
    const size_t plane = 2 * align16(cap * sizeof(T));
    unsigned char* p = base;
    m.hT[0] = p; p += tile;
    m.hT[1] = p; p += tile;
    m.rT[0] = p; p += tile;
    m.rT[1] = p; p += tile;
    m.kt = p; p += plane;
    for (int i = 0; i < 4; ++i) { m.c[i] = p; p += plane; }
    // solve staging overlays the sweep buffers (used in a different phase)
    const size_t sp = (size_t)stage_pad(SOLVE_CAP);
    m.ssl = reinterpret_cast<double*>(base);
    m.skt = reinterpret_cast<int*>(base + align16(sp * 8));
    m.sky = base + align16(sp * 8) + align16(sp * 4);
    return m;
}

// ---------------------------------------------------------------------------
// segmented knot lists: real knot i lives in segment r = seg_of(i) at
// position i - pref[r] of that segment's list
// ---------------------------------------------------------------------------
struct Slot {
    int32_t* kt;   // knot lists (segmented)
    void* ky;
    void* M;       // interval records, mirror space: [2 env][5][kcap] storage type
};

__device__ __forceinline__ int64_t knot_index(const Ctx& C, int par, int env, int seg, int i) {
    return ((int64_t)((par * 2 + env) * C.csize + seg)) * C.segcap + i;
}

// segment holding real knot i: largest r with pref[r] <= i
__device__ __forceinline__ int seg_of(const int* pref, int csize, int i) {
    int lo = 0, hi = csize;  // pref[lo] <= i < pref[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// element offset of real knot i in the current knot plane
__device__ __forceinline__ int64_t real_off(const Ctx& C, const TaskSm& S, int env, int i) {
    const int* pr = S.pref[env];
    int r = S.rank;  // most lookups fall in the CTA's own segment
    if (i < pr[r] || i >= pr[r + 1]) r = seg_of(pr, S.csize, i);
    return knot_index(C, S.kpar, env, r, i - pr[r]);
}

template <typename T>
__device__ __forceinline__ void real_knot(const Ctx& C, const Slot& sl, const TaskSm& S, int env, int i,
                                          int& t, double& y) {
    const int64_t o = real_off(C, S, env, i);
    t = __ldcg(sl.kt + o);
    y = (double)__ldcg(static_cast<const T*>(sl.ky) + o);
}

// Stage mirror-space knot i2 into shared memory: an asynchronous copy for a
// real knot, a direct store for a virtual mirror knot.
template <typename T>
__device__ __forceinline__ void stage_knot(const Ctx& C, const Slot& sl, const TaskSm& S, int env, int i2,
                                           int* kt_s, T* ky_s) {
    if (S.mir[env]) {
        if (i2 == 0) {
            *kt_s = S.tfirst[env];
            *ky_s = (T)S.yfirst[env];
            return;
        }
        if (i2 == S.P[env] + 1) {
            *kt_s = S.tlast[env];
            *ky_s = (T)S.ylast[env];
            return;
        }
        i2 -= 1;
    }
    const int64_t o = real_off(C, S, env, i2);
    cp_async4(kt_s, sl.kt + o);
    cp_async_el<T>(ky_s, static_cast<const T*>(sl.ky) + o);
}

// Knot i2 in "mirror space" (emd_ref.py:92-96): with mir=1 the list is
// [2t0-t1, t0..t_{P-1}, 2t_{P-1}-t_{P-2}] with values [y1, y.., y_{P-2}].
template <typename T>
__device__ __forceinline__ void knot2(const Ctx& C, const Slot& sl, const TaskSm& S, int env, int i2,
                                      int& t, double& y) {
    const int P = S.P[env];
    if (S.mir[env]) {
        if (i2 == 0) {
            int t0, t1;
            double y0, y1;
            real_knot<T>(C, sl, S, env, 0, t0, y0);
            real_knot<T>(C, sl, S, env, 1, t1, y1);
            t = 2 * t0 - t1;
            y = y1;
            return;
        }
        if (i2 == P + 1) {
            int ta, tb;
            double ya, yb;
            real_knot<T>(C, sl, S, env, P - 1, ta, ya);
            real_knot<T>(C, sl, S, env, P - 2, tb, yb);
            t = 2 * ta - tb;
            y = yb;
            return;
        }
        i2 -= 1;
    }
    real_knot<T>(C, sl, S, env, i2, t, y);
}

// ---------------------------------------------------------------------------
// solve: decay-seamed block Thomas over the cluster
// ---------------------------------------------------------------------------
// Row i (mirror space, i = 0..n-1 for M2[i+1]) from staged knots k = i - base:
//   H0 = t_{i+1}-t_i, H1 = t_{i+2}-t_{i+1}, d = 2(H0+H1), l = H0 (i>=1),
//   u = H1 (i<=n-2), r = 6(slope_{i+1} - slope_i)          (emd_ref.py:31-48)
// The sweeps slide along the rows: each row loads one new knot and one slope.
struct Row {
    double dg, l, u, r;
};

__device__ __forceinline__ Row row_of(int ta, int tb, int tc, double sa, double sb, int i, int n) {
    const double H0 = (double)(tb - ta), H1 = (double)(tc - tb);
    Row w;
    w.dg = 2.0 * (H0 + H1);
    w.l = (i >= 1) ? H0 : 0.0;
    w.u = (i <= n - 2) ? H1 : 0.0;
    w.r = 6.0 * (sb - sa);
    return w;
}

#define SKT(k) skt[stage_pad(k)]
#define SSL(k) ssl[stage_pad(k)]

// Interval records of one envelope in mirror space, five storage-type planes
// of stride kcap: t_k (integer bit pattern), then four coefficient planes.
template <typename T>
struct Rec {  // plane 0: t_k; planes 1..4: c0..c3 (fast) or y_k, M_k (exact)
    T* rc;
    int64_t stride;
    __device__ __forceinline__ T& c(int plane, int k) const { return rc[(plane + 1) * stride + k]; }
    __device__ __forceinline__ T& t(int k) const { return rc[k]; }
};

// exact: forward elimination from w0 (outer coupling dropped), back
// substitution from w1; identical recurrences to serial Thomas (emd_ref.py:50-65).
// Writes (t_k, y_k, M_k) of the owned knots k = o0+1 .. o1+1 (+ both end knots).
template <typename T>
__device__ void window_exact(const Ctx& C, const int* skt, const T* sky, const double* ssl, int base,
                             int n, int w, const Rec<T>& R, int p2) {
    const int B = C.B, S = C.S;
    const int o0 = w * B;
    const int o1 = min(n, o0 + B) - 1;
    const int w0 = max(0, o0 - S);
    const int w1 = min(n - 1, o1 + S);
    const int64_t gthreads = (int64_t)gridDim.x * blockDim.x;
    double2* sc = C.scr + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    double cp = 0.0, dp = 0.0;
    int ta = SKT(w0 - base), tb = SKT(w0 + 1 - base);
    double sa = SSL(w0 - base);
    for (int i = w0; i <= w1; ++i) {
        const int tc = SKT(i + 2 - base);
        const double sb = SSL(i + 1 - base);
        const Row rw = row_of(ta, tb, tc, sa, sb, i, n);
        const double c = (i == w1) ? 0.0 : rw.u / (rw.dg - rw.l * cp);
        const double dv = (rw.r - rw.l * dp) / (rw.dg - rw.l * cp);
        if (i >= o0) sc[(int64_t)(i - o0) * gthreads] = make_double2(c, dv);
        cp = c;
        dp = dv;
        ta = tb;
        tb = tc;
        sa = sb;
    }
    auto put = [&](int k, double Mk) {
        R.t(k) = tbits<T>(SKT(k - base));
        R.c(0, k) = sky[stage_pad(k - base)];
        R.c(1, k) = (T)Mk;
    };
    double xv = dp;
    if (w1 <= o1) put(w1 + 1, xv);
    for (int i = w1 - 1; i >= o0; --i) {
        const double2 cd = sc[(int64_t)(i - o0) * gthreads];
        xv = cd.y - cd.x * xv;
        if (i <= o1) put(i + 1, xv);
    }
    if (o0 == 0) put(0, 0.0);
    if (o1 == n - 1) put(p2 - 1, 0.0);
}

// fast: twisted factorisation of the window.  A left sweep (LU, coupling
// dropped at w0) keeps its (c, d) for the owned rows in registers; a right
// sweep (UL, coupling dropped at w1) meets it, and each owned unknown is
//   x_i = (r_i - l_i d_{i-1} - u_i g_{i+1}) / (dg_i - l_i c_{i-1} - u_i e_{i+1}).
template <typename T>
__device__ void window_fast(const Ctx& C, const int* skt, const T* sky, const double* ssl, int base, int n,
                            int w, const Rec<T>& R, int p2) {
    const int S = C.S;
    const int o0 = w * FAST_B;
    const int cnt = min(FAST_B, n - o0);
    const int o1 = o0 + cnt - 1;
    const int w0 = max(0, o0 - S);
    const int w1 = min(n - 1, o1 + S);
    double fc[FAST_B], fd[FAST_B];
    double cp = 0.0, dp = 0.0, cq = 0.0, dq = 0.0;  // (cq, dq): forward state after row o0-2
    int ta = SKT(w0 - base), tb = SKT(w0 + 1 - base);
    double sa = SSL(w0 - base);
    for (int i = w0; i <= o0 - 2; ++i) {
        const int tc = SKT(i + 2 - base);
        const double sb = SSL(i + 1 - base);
        const Row rw = row_of(ta, tb, tc, sa, sb, i, n);
        const double inv = fast_rcp(fma(-rw.l, cp, rw.dg));
        cp = rw.u * inv;
        dp = fma(-rw.l, dp, rw.r) * inv;
        ta = tb;
        tb = tc;
        sa = sb;
    }
    cq = cp;
    dq = dp;
    // forward state after rows o0-1 .. o1-1 (row -1 does not exist: zero state)
#pragma unroll
    for (int k = 0; k < FAST_B; ++k) {
        const int i = o0 - 1 + k;
        if (k < cnt) {
            if (i >= 0) {
                const int tc = SKT(i + 2 - base);
                const double sb = SSL(i + 1 - base);
                const Row rw = row_of(ta, tb, tc, sa, sb, i, n);
                const double inv = fast_rcp(fma(-rw.l, cp, rw.dg));
                cp = rw.u * inv;
                dp = fma(-rw.l, dp, rw.r) * inv;
                ta = tb;
                tb = tc;
                sa = sb;
            }
            fc[k] = cp;
            fd[k] = dp;
        }
    }
    // right sweep from w1 down to o1+1, then combine over the owned rows
    double e = 0.0, g = 0.0;
    int ub = SKT(w1 + 1 - base), uc = SKT(w1 + 2 - base);
    double vb = SSL(w1 + 1 - base);
    for (int i = w1; i > o1; --i) {
        const int ua = SKT(i - base);
        const double va = SSL(i - base);
        const Row rw = row_of(ua, ub, uc, va, vb, i, n);
        const double inv = fast_rcp(fma(-rw.u, e, rw.dg));
        e = rw.l * inv;
        g = fma(-rw.u, g, rw.r) * inv;
        uc = ub;
        ub = ua;
        vb = va;
    }
    // monomial record of interval k (knots k, k+1; M_k = Ma, M_{k+1} = Mb):
    // y_k + s(c1 + s(c2 + s c3)), s = t - t_k, c1 = slope - h(2Ma + Mb)/6,
    // c2 = Ma/2, c3 = (Mb - Ma)/(6h)
    auto put = [&](int k, double Ma, double Mb) {
        const int t0 = SKT(k - base), t1 = SKT(k + 1 - base);
        const double h = (double)(t1 - t0);
        R.t(k) = tbits<T>(t0);
        R.c(0, k) = sky[stage_pad(k - base)];
        R.c(1, k) = (T)fma(-h * (1.0 / 6.0), fma(2.0, Ma, Mb), SSL(k - base));
        R.c(2, k) = (T)(0.5 * Ma);
        R.c(3, k) = (T)((Mb - Ma) * fast_rcp(h) * (1.0 / 6.0));
    };
    double xnext = 0.0;  // x_{i+1} of the previous iteration
#pragma unroll
    for (int k = FAST_B - 1; k >= 0; --k) {
        if (k < cnt) {
            const int i = o0 + k;
            const int ua = SKT(i - base);
            const double va = SSL(i - base);
            const Row rw = row_of(ua, ub, uc, va, vb, i, n);
            const double num = fma(-rw.u, g, fma(-rw.l, fd[k], rw.r));
            const double den = fma(-rw.u, e, fma(-rw.l, fc[k], rw.dg));
            const double xi = num * fast_rcp(den);  // M at mirror knot i+1
            if (i < o1) put(i + 1, xi, xnext);
            else if (i == n - 1) put(n, xi, 0.0);   // last interval ends at the M = 0 knot
            xnext = xi;
            const double inv = fast_rcp(fma(-rw.u, e, rw.dg));
            e = rw.l * inv;
            g = fma(-rw.u, g, rw.r) * inv;
            uc = ub;
            ub = ua;
            vb = va;
        }
    }
    // M at knot o0 (x_{o0-1}) closes interval o0; zero at the natural end
    double xm = 0.0;
    if (o0 >= 1) {
        const int i = o0 - 1;
        const int ua = SKT(i - base);
        const double va = SSL(i - base);
        const Row rw = row_of(ua, ub, uc, va, vb, i, n);
        const double num = fma(-rw.u, g, fma(-rw.l, dq, rw.r));
        const double den = fma(-rw.u, e, fma(-rw.l, cq, rw.dg));
        xm = num * fast_rcp(den);
    }
    put(o0, xm, xnext);
}

#undef SKT
#undef SSL

template <typename T, bool EXACT>
__device__ void solve_task(const Ctx& C, const Slot& sl, TaskSm& S, const Smem& sm) {
    const int tid = threadIdx.x;
    for (int env = 0; env < 2; ++env) {
        const int p2 = S.p2[env];
        const int n = p2 - 2;
        Rec<T> R;
        R.rc = static_cast<T*>(sl.M) + (int64_t)env * 5 * C.kcap;
        R.stride = C.kcap;
        if (n <= 0) {
            // one or two knots: a constant or the straight line through them (M = 0)
            if (S.rank == 0 && tid < p2) {
                int tk, t1;
                double yk, y1;
                knot2<T>(C, sl, S, env, tid, tk, yk);
                R.t(tid) = tbits<T>(tk);
                R.c(0, tid) = (T)yk;
                R.c(1, tid) = (T)0;
                R.c(2, tid) = (T)0;
                R.c(3, tid) = (T)0;
                if (!EXACT && tid + 1 < p2) {
                    knot2<T>(C, sl, S, env, tid + 1, t1, y1);
                    R.c(1, tid) = (T)((y1 - yk) / (double)(t1 - tk));
                }
            }
            continue;
        }
        const int Bw = EXACT ? C.B : FAST_B;
        const int nwin = (n + Bw - 1) / Bw;
        const int wa = (int)((int64_t)S.rank * nwin / S.csize);
        const int wb = (int)((int64_t)(S.rank + 1) * nwin / S.csize);
        int wpp = (SOLVE_CAP - 2 * C.S - 8) / Bw;
        wpp = max(1, min(wpp, THREADS));
        for (int wbase = wa; wbase < wb; wbase += wpp) {
            const int wend = min(wb, wbase + wpp);
            const int rlo = max(0, wbase * Bw - C.S);
            const int rhi = min(n - 1, min(n, wend * Bw) - 1 + C.S);
            const int kcount = rhi + 3 - rlo;  // knots rlo .. rhi+2
            T* sky = static_cast<T*>(sm.sky);
            __syncthreads();
            for (int k = tid; k < kcount; k += THREADS)
                stage_knot<T>(C, sl, S, env, rlo + k, &sm.skt[stage_pad(k)], &sky[stage_pad(k)]);
            cp_async_commit();
            cp_async_wait<0>();
            __syncthreads();
            for (int k = tid; k + 1 < kcount; k += THREADS) {
                const int ta = sm.skt[stage_pad(k)], tb = sm.skt[stage_pad(k + 1)];
                const double ya = (double)sky[stage_pad(k)], yb = (double)sky[stage_pad(k + 1)];
                // emd_ref.py:47: (y_{q+1}-y_q)/H_q, the same IEEE division
                sm.ssl[stage_pad(k)] = (yb - ya) / (double)(tb - ta);
            }
            __syncthreads();
            const int w = wbase + tid;
            if (w < wend) {
                if (EXACT) window_exact<T>(C, sm.skt, sky, sm.ssl, rlo, n, w, R, p2);
                else window_fast<T>(C, sm.skt, sky, sm.ssl, rlo, n, w, R, p2);
            }
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// sweep: the fused per-segment pass
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ double trial_input(const Ctx& C, const TaskDesc& d, int64_t t) {
    const double xv = ldv<T>(C.x, d.x_off + t);
    switch (C.noise_mode) {
        case EEMD_NOISE_INJECTED: return rnd<T>(xv + ldv<T>(C.noise, d.noise_off + t));
        case EEMD_NOISE_PHILOX:
            return rnd<T>(xv + C.sigma[d.signal] * philox_normal(C.seed, d.signal, d.trial, t));
        default: return xv;  // NONE, PREPERTURBED
    }
}

// Block-wide exclusive scan of two per-thread counts (one __syncthreads).
// wtot: shared [2*NWARP], not reused before the next __syncthreads.
__device__ __forceinline__ void block_scan2(int a, int b, int& ea, int& eb, int& ta, int& tb, int* wtot) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int ia = a, ib = b;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int xa = __shfl_up_sync(0xffffffffu, ia, o);
        const int xb = __shfl_up_sync(0xffffffffu, ib, o);
        if (lane >= o) { ia += xa; ib += xb; }
    }
    if (lane == 31) { wtot[wid] = ia; wtot[NWARP + wid] = ib; }
    __syncthreads();
    int ba = 0, bb = 0;
    ta = 0;
    tb = 0;
#pragma unroll
    for (int w = 0; w < NWARP; ++w) {
        const int va = wtot[w], vb = wtot[NWARP + w];
        if (w < wid) { ba += va; bb += vb; }
        ta += va;
        tb += vb;
    }
    ea = ba + ia - a;
    eb = bb + ib - b;
}

// Interval cache of one envelope for a thread's run of consecutive samples:
// the staged record of interval k is loaded only when k changes.
template <typename T>
struct IvCache {
    int k, t0, t1;
    T y0, c1, c2, c3, y1, m1;  // fast: monomial c0..c3 of interval k; exact: y0, M0, y1, M1
};

template <typename T, bool EXACT>
__device__ __forceinline__ T iv_value(IvCache<T>& cc, const Smem& sm, int env, int idx2, int lo2, int t) {
    if (idx2 != cc.k) {
        const T* kt = static_cast<const T*>(sm.kt);
        const T* c0 = static_cast<const T*>(sm.c[0]);
        const T* c1 = static_cast<const T*>(sm.c[1]);
        const int o = env * sm.cap + (idx2 - lo2);
        cc.k = idx2;
        cc.t0 = tint<T>(kt[o]);
        cc.y0 = c0[o];
        cc.c1 = c1[o];
        if (EXACT) {
            cc.t1 = tint<T>(kt[o + 1]);
            cc.y1 = c0[o + 1];
            cc.m1 = c1[o + 1];
        } else {
            cc.c2 = static_cast<const T*>(sm.c[2])[o];
            cc.c3 = static_cast<const T*>(sm.c[3])[o];
        }
    }
    if (EXACT)
        return (T)spline_exact((double)t, (double)cc.t0, (double)cc.t1, (double)cc.y0, (double)cc.y1,
                               (double)cc.c1, (double)cc.m1);
    const T s = (T)(t - cc.t0);
    return fmat(s, fmat(s, fmat(s, cc.c3, cc.c2), cc.c1), cc.y0);
}

// envelope value at t with `cless` knots strictly before t (mirror space),
// interval = searchsorted - 1 clipped (emd_ref.py:70)
template <typename T, bool EXACT>
__device__ __forceinline__ T env_value(const TaskSm& S, IvCache<T>& cc, const Smem& sm, int env, int cless,
                                       int t, int lo2) {
    if (S.P[env] < 2) return (T)S.cval[env];
    const int idx2 = max(0, min(cless - 1, S.p2[env] - 2));
    return iv_value<T, EXACT>(cc, sm, env, idx2, lo2, t);
}

__device__ __forceinline__ int mirror_adj(const TaskSm& S, int env, int t) {
    return S.mir[env] ? (S.tfirst[env] < t ? 1 : 0) + (S.tlast[env] < t ? 1 : 0) : 0;
}

// element phase of an address within its 16-byte block
template <typename T>
__device__ __forceinline__ int phase16(const T* p) {
    return (int)((reinterpret_cast<uintptr_t>(p) / sizeof(T)) & (16 / sizeof(T) - 1));
}

// stores a thread's run of samples: one 16-byte-vector pass when the run is
// full and aligned, element stores otherwise
template <typename T>
__device__ __forceinline__ void store_run(T* p, const T (&v)[RUN_MAX], int nv) {
    if (nv == RUN_MAX && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        if constexpr (sizeof(T) == 4) {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        } else {
            reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
            reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < RUN_MAX; ++i)
        if (i < nv) p[i] = v[i];
}

// The sweep streams the CTA's segment in tiles of TILE samples; thread u owns
// the run of TILE/THREADS consecutive samples starting at u*TILE/THREADS and
// keeps its samples in registers.  The next tile is copied to shared memory
// (cp.async, 16-byte copies where the addresses allow) while the current one
// is processed; the interval records a tile needs are staged with one batch
// of asynchronous copies.  Arithmetic runs in the storage type T: the spline
// solve that produced the records ran in double, and the exact mode (double
// only) keeps the reference operation order.
template <typename T, bool EXACT>
__device__ void sweep(const Ctx& C, const Slot& sl, TaskSm& S, Xchg* X, const Smem& sm,
                      cg::cluster_group& cl) {
    constexpr int VEC = 16 / (int)sizeof(T);
    __shared__ double2 s_red[NWARP];
    __shared__ int s_w1[2 * NWARP], s_w2[2 * NWARP];
    __shared__ T s_gfirst[NWARP], s_glast[NWARP];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int TILE = C.tile, run = TILE / THREADS, cap = sm.cap;
    const int mode = S.mode, n = S.n, s0 = S.s0, s1 = S.s1, rank = S.rank;
    const bool sifting = (mode == TM_SIFT || mode == TM_LAST);
    const bool uses_r = (mode == TM_LAST || mode == TM_TRANS);
    const bool needs_h = sifting || (mode == TM_TRANS && !S.imf_from_resid);
    const int q = S.step & 1;
    const TaskDesc d = C.td[S.task];
    T* resid = static_cast<T*>(C.resid) + d.s_off;
    T* imf_m = static_cast<T*>(C.imfs) + d.imf_off + (int64_t)min(S.imf, C.max_imf - 1) * n;
    const T* src = (sifting && S.src_resid) ? resid : imf_m;
    const int np = S.kpar ^ 1;
    double num = 0.0, den = 0.0;
#ifdef EEMD_TRACE
    unsigned long long scyc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long smark = clock64();
#define SUB(k)                                          \
    do {                                                \
        const long long now_ = clock64();               \
        scyc[k] += (unsigned long long)(now_ - smark);  \
        smark = now_;                                   \
    } while (0)
#else
#define SUB(k) \
    do {       \
    } while (0)
#endif

    if (tid == 0) {
        S.run_cur[0] = S.run_cur[1] = 0;
        S.run_new[0] = S.run_new[1] = 0;
        S.hold_m1 = S.hold_m2 = S.rold_m1 = S.hold_p = S.rold_p = 0.0;
        if (mode != TM_INIT) {
            // neighbours' edge samples from their previous step (distributed shared memory)
            const bool hres = sifting && S.src_resid;
            if (s0 > 0) {
                const Xchg* xl = cl.map_shared_rank(&X[q ^ 1], rank - 1);
                S.hold_m1 = hres ? xl->rl[1] : xl->hl[1];
                S.hold_m2 = hres ? xl->rl[0] : xl->hl[0];
                S.rold_m1 = xl->rl[1];
            }
            if (s1 < n) {
                const Xchg* xr = cl.map_shared_rank(&X[q ^ 1], rank + 1);
                S.hold_p = hres ? xr->rf[0] : xr->hf[0];
                S.rold_p = xr->rf[0];
            }
        }
    }
    __syncthreads();

    // copies g[0 .. cnt) to dst[0 .. cnt); dst + j and g + j share their
    // 16-byte phase, so the body moves in 16-byte copies
    auto copy_stream = [&](T* dst, const T* g, int cnt) {
        const int head = min(cnt, (VEC - phase16(g)) & (VEC - 1));
        const int nvec = (cnt - head) / VEC;
        const int tail0 = head + nvec * VEC;
        for (int v = tid; v < nvec; v += THREADS) cp_async16(dst + head + v * VEC, g + head + v * VEC);
        const int ns = head + (cnt - tail0);
        for (int k = tid; k < ns; k += THREADS) {
            const int j = (k < head) ? k : tail0 + (k - head);
            cp_async_el<T>(dst + j, g + j);
        }
    };
    // tile buffer b positioned for the tile starting at t0p of stream g
    auto tile_h = [&](int b, int t0p) { return static_cast<T*>(sm.hT[b]) + TOFF + phase16(src + t0p); };
    auto tile_r = [&](int b, int t0p) { return static_cast<T*>(sm.rT[b]) + TOFF + phase16(resid + t0p); };
    // copies samples [t0p, t0p+tl] (the extra one when it is still this segment's) to buffer b
    auto prefetch = [&](int t0p, int b) {
        const int tlp = min(TILE, s1 - t0p);
        const int cnt = (t0p + tlp < s1) ? tlp + 1 : tlp;
        if (needs_h) copy_stream(tile_h(b, t0p), src + t0p, cnt);
        if (uses_r) copy_stream(tile_r(b, t0p), resid + t0p, cnt);
        cp_async_commit();
    };
    const bool streams = needs_h || uses_r;
    if (streams) prefetch(s0, 0);

    int buf = 0;
    for (int t0 = s0; t0 < s1; t0 += TILE, buf ^= 1) {
        const int tl = min(TILE, s1 - t0);
        const bool first = (t0 == s0), last = (t0 + tl == s1);
        const int j0 = tid * run;
        const int nv = max(0, min(run, tl - j0));  // valid samples of this thread's run
        T* hb = tile_h(buf, t0);  // hb[j] = sample t0+j, hb[-1] / hb[tl] halos
        T* rb = tile_r(buf, t0);
        // ---------------- (a) this tile's samples (prefetched), next tile's prefetch ----------------
        if (streams) {
            if (!last) {
                prefetch(t0 + TILE, buf ^ 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
        }
        if (tid == 0) {
            if (sifting) {
                hb[-1] = (T)S.hold_m1;
                if (last) hb[tl] = (T)((t0 + tl < n) ? S.hold_p : 0.0);
            } else if (needs_h) {  // TM_TRANS: the closed IMF at the halo samples
                hb[-1] = (first && t0 > 0) ? __ldcg(imf_m + t0 - 1) : (T)0;
                if (last) hb[tl] = (t0 + tl < n) ? __ldcg(imf_m + t0 + tl) : (T)0;
            }
            if (uses_r) {
                if (first) rb[-1] = (T)S.rold_m1;
                if (last) rb[tl] = (T)((t0 + tl < n) ? S.rold_p : 0.0);
            }
        }
        __syncthreads();
        SUB(0);
        T hv[RUN_MAX], rv[RUN_MAX], fv[RUN_MAX], gv[RUN_MAX];
#pragma unroll
        for (int i = 0; i < RUN_MAX; ++i) {
            const bool ok = i < nv;
            hv[i] = (ok && needs_h) ? hb[j0 + i] : (T)0;
            rv[i] = (ok && uses_r) ? rb[j0 + i] : (T)0;
            fv[i] = gv[i] = (T)0;
        }

        // ---------------- (b) current knots: strict extrema of h in the run ----------------
        unsigned kmx = 0u, kmn = 0u;
        int kb0 = 0, kb1 = 0, kc0 = 0, kc1 = 0, lo0 = 0, lo1 = 0, hi0 = -1, hi1 = -1;
        int cl0 = 0, cl1 = 0;
        if (sifting) {
            if (nv > 0) {
                const T hl0 = hb[j0 - 1], hr0 = hb[j0 + nv];
#pragma unroll
                for (int i = 0; i < RUN_MAX; ++i) {
                    const int t = t0 + j0 + i;
                    if (i < nv && t >= 1 && t <= n - 2) {
                        const T a = (i == 0) ? hl0 : hv[(i + RUN_MAX - 1) % RUN_MAX];
                        const T c = (i + 1 == nv) ? hr0 : hv[(i + 1) % RUN_MAX];
                        const T v = hv[i];
                        if (v > a && v > c) kmx |= 1u << i;
                        if (v < a && v < c) kmn |= 1u << i;
                    }
                }
            }
            int ex, en, tx, tn;
            block_scan2(__popc(kmx), __popc(kmn), ex, en, tx, tn, s_w1);
            kc0 = tx;
            kc1 = tn;
            kb0 = S.pref[0][rank] + S.run_cur[0];
            kb1 = S.pref[1][rank] + S.run_cur[1];
            if (S.P[0] >= 2) {
                lo0 = max(0, S.mir[0] + kb0 - 2);
                hi0 = min(S.p2[0] - 1, S.mir[0] + kb0 + kc0 + 1);
            }
            if (S.P[1] >= 2) {
                lo1 = max(0, S.mir[1] + kb1 - 2);
                hi1 = min(S.p2[1] - 1, S.mir[1] + kb1 + kc1 + 1);
            }
            const bool bad0 = hi0 - lo0 + 1 > cap || kb0 + kc0 > S.P[0];
            const bool bad1 = hi1 - lo1 + 1 > cap || kb1 + kc1 > S.P[1];
            if ((bad0 || bad1) && tid == 0) raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, S.task);
            if (bad0) hi0 = lo0 - 1;
            if (bad1) hi1 = lo1 - 1;
            cl0 = kb0 + ex;
            cl1 = kb1 + en;
            SUB(1);
            // ---------------- (c) stage the interval records the tile uses ----------------
            const int n0 = hi0 - lo0 + 1, n1 = hi1 - lo1 + 1;
            for (int k = tid; k < n0 + n1; k += THREADS) {
                const int env = (k >= n0) ? 1 : 0;
                const int kk = k - env * n0;
                const int i2 = (env ? lo1 : lo0) + kk;
                const int o = env * cap + kk;
                const T* rc = static_cast<const T*>(sl.M) + (int64_t)env * 5 * C.kcap + i2;
                cp_async_el<T>(static_cast<T*>(sm.kt) + o, rc);
                cp_async_el<T>(static_cast<T*>(sm.c[0]) + o, rc + C.kcap);
                cp_async_el<T>(static_cast<T*>(sm.c[1]) + o, rc + 2 * (int64_t)C.kcap);
                if (!EXACT) {
                    cp_async_el<T>(static_cast<T*>(sm.c[2]) + o, rc + 3 * (int64_t)C.kcap);
                    cp_async_el<T>(static_cast<T*>(sm.c[3]) + o, rc + 4 * (int64_t)C.kcap);
                }
            }
            cp_async_commit();
            if (tid == 0) {
                // is t0-1 a knot of each kind? (only the segment's first tile evaluates t0-1)
                S.left_knot[0] = S.left_knot[1] = 0;
                if (first && t0 - 1 >= 1 && t0 - 1 <= n - 2) {
                    const T a = (T)S.hold_m2, b = hb[-1], c = hb[0];
                    S.left_knot[0] = (b > a) && (b > c);
                    S.left_knot[1] = (b < a) && (b < c);
                }
            }
            cp_async_wait<0>();
            __syncthreads();
            SUB(2);
        }

        // ---------------- (d) new values ----------------
        IvCache<T> cc0, cc1;
        cc0.k = cc1.k = -1;
        cc0.t0 = cc0.t1 = 0;
        cc0.y0 = cc0.c1 = cc0.c2 = cc0.c3 = cc0.y1 = cc0.m1 = (T)0;
        cc1 = cc0;
        T tnum = (T)0, tden = (T)0;  // fast mode: this tile's SD partial sums
#pragma unroll
        for (int i = 0; i < RUN_MAX; ++i) {
            const int t = t0 + j0 + i;
            if (i < nv) {
                if (sifting) {
                    const T h = hv[i];
                    const T eu = env_value<T, EXACT>(S, cc0, sm, 0, cl0 + mirror_adj(S, 0, t), t, lo0);
                    const T el = env_value<T, EXACT>(S, cc1, sm, 1, cl1 + mirror_adj(S, 1, t), t, lo1);
                    cl0 += (kmx >> i) & 1u;
                    cl1 += (kmn >> i) & 1u;
                    const T m = (T)0.5 * (eu + el);
                    const T hn = h - m;
                    fv[i] = hn;
                    if (EXACT) {
                        const double dd = (C.rules == EEMD_RULES_NUMBA) ? (double)m : (double)(h - hn);
                        num = num + dd * dd;
                        den = den + (double)h * (double)h;
                    } else {
                        const T dd = (C.rules == EEMD_RULES_NUMBA) ? m : h - hn;
                        tnum = fmat(dd, dd, tnum);
                        tden = fmat(h, h, tden);
                    }
                    gv[i] = (mode == TM_LAST) ? rv[i] - hn : hn;
                } else if (mode == TM_TRANS) {
                    fv[i] = rv[i] - (S.imf_from_resid ? rv[i] : hv[i]);
                    gv[i] = fv[i];
                } else {  // TM_INIT
                    fv[i] = (T)trial_input<T>(C, d, t);
                    gv[i] = fv[i];
                }
            }
        }
        if (!EXACT) {
            num += (double)tnum;
            den += (double)tden;
        }
        // halo samples: t0-1 (first tile of the segment, thread 0) and t0+tl (last owner)
        const int u_last = (tl - 1) / run;
        for (int side = 0; side < 2; ++side) {
            int t, hj;
            if (side == 0) {
                if (!(tid == 0 && first && t0 > 0)) continue;
                t = t0 - 1;
                hj = -1;
            } else {
                if (!(tid == u_last && t0 + tl < n)) continue;
                t = t0 + tl;
                hj = tl;
            }
            T fn, gn;
            if (sifting) {
                IvCache<T> h0, h1;
                h0.k = h1.k = -1;
                const int c0v = (side == 0 ? kb0 - S.left_knot[0] : kb0 + kc0) + mirror_adj(S, 0, t);
                const int c1v = (side == 0 ? kb1 - S.left_knot[1] : kb1 + kc1) + mirror_adj(S, 1, t);
                const T eu = env_value<T, EXACT>(S, h0, sm, 0, c0v, t, lo0);
                const T el = env_value<T, EXACT>(S, h1, sm, 1, c1v, t, lo1);
                const T m = (T)0.5 * (eu + el);
                fn = hb[hj] - m;
                gn = (mode == TM_LAST) ? rb[hj] - fn : fn;
            } else if (mode == TM_TRANS) {
                const T ro = rb[hj];
                fn = ro - (S.imf_from_resid ? ro : hb[hj]);
                gn = fn;
            } else {
                fn = (T)trial_input<T>(C, d, t);
                gn = fn;
            }
            if (side == 0) {
                S.fl = fn;
                S.gl = gn;
            } else {
                S.fr = fn;
                S.gr = gn;
            }
        }
        SUB(3);
        // run edges for the neighbours' flags
        const T glast_mine = (run == 1) ? gv[0] : (run == 2) ? gv[1] : gv[RUN_MAX - 1];
        if (lane == 0) s_gfirst[wid] = gv[0];
        if (lane == 31) s_glast[wid] = glast_mine;
        __syncthreads();
        SUB(4);

        // ---------------- (e) next knots: strict extrema of the new values ----------------
        const T up = __shfl_up_sync(0xffffffffu, glast_mine, 1);
        const T dn = __shfl_down_sync(0xffffffffu, gv[0], 1);
        T gprev, gnext;
        if (j0 == 0) gprev = first ? (t0 > 0 ? (T)S.gl : (T)0) : (T)S.g_m1;
        else gprev = (lane > 0) ? up : s_glast[wid - 1];
        if (j0 + nv == tl) gnext = (t0 + tl < n) ? (T)S.gr : (T)0;
        else gnext = (lane < 31) ? dn : s_gfirst[wid + 1];
        unsigned nmx = 0u, nmn = 0u;
#pragma unroll
        for (int i = 0; i < RUN_MAX; ++i) {
            const int t = t0 + j0 + i;
            if (i < nv && t >= 1 && t <= n - 2) {
                const T a = (i == 0) ? gprev : gv[(i + RUN_MAX - 1) % RUN_MAX];
                const T c = (i + 1 == nv) ? gnext : gv[(i + 1) % RUN_MAX];
                const T v = gv[i];
                if (v > a && v > c) nmx |= 1u << i;
                if (v < a && v < c) nmn |= 1u << i;
            }
        }
        int ex2, en2, tx2, tn2;
        block_scan2(__popc(nmx), __popc(nmn), ex2, en2, tx2, tn2, s_w2);
        SUB(5);

        // ---------------- (f) writes ----------------
        {
            const int64_t pmx = knot_index(C, np, 0, rank, 0);
            const int64_t pmn = knot_index(C, np, 1, rank, 0);
            int px = S.run_new[0] + ex2, pn = S.run_new[1] + en2;
#pragma unroll
            for (int i = 0; i < RUN_MAX; ++i) {
                const int t = t0 + j0 + i;
                if (i < nv) {
                    if ((nmx >> i) & 1u) {
                        if (px < C.segcap) {
                            sl.kt[pmx + px] = t;
                            static_cast<T*>(sl.ky)[pmx + px] = gv[i];
                        } else {
                            raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, S.task);
                        }
                        ++px;
                    }
                    if ((nmn >> i) & 1u) {
                        if (pn < C.segcap) {
                            sl.kt[pmn + pn] = t;
                            static_cast<T*>(sl.ky)[pmn + pn] = gv[i];
                        } else {
                            raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, S.task);
                        }
                        ++pn;
                    }
                }
            }
            const int tj = t0 + j0;
            switch (mode) {
                case TM_SIFT: store_run<T>(imf_m + tj, fv, nv); break;
                case TM_LAST:
                    store_run<T>(imf_m + tj, fv, nv);
                    store_run<T>(resid + tj, gv, nv);
                    break;
                case TM_TRANS:
                    store_run<T>(resid + tj, fv, nv);
                    if (S.imf_from_resid) store_run<T>(imf_m + tj, rv, nv);
                    break;
                default: store_run<T>(resid + tj, fv, nv); break;
            }
            // edge and carry values of the tile, written by the threads that hold them
#pragma unroll
            for (int i = 0; i < RUN_MAX; ++i) {
                if (i >= nv) continue;
                const int j = j0 + i;
                if (first && j == 0) { S.hf0 = fv[i]; S.rf0 = gv[i]; }
                if (first && j == 1) { S.hf1 = fv[i]; S.rf1 = gv[i]; }
                if (j == tl - 2) { S.f_last2 = fv[i]; S.g_last2 = gv[i]; }
                if (j == tl - 1) {
                    if (last) {
                        Xchg& xo = X[q];
                        xo.hl[0] = (tl >= 2) ? 0.0 : S.f_m1;  // completed below for tl >= 2
                        xo.hl[1] = fv[i];
                        xo.rl[0] = (tl >= 2) ? 0.0 : S.g_m1;
                        xo.rl[1] = gv[i];
                    }
                    S.f_m1 = fv[i];
                    S.g_m1 = gv[i];
                    if (sifting) {
                        S.hold_m1 = hv[i];
                        S.hold_m2 = (tl >= 2) ? (double)hb[tl - 2] : (double)hb[-1];
                    }
                }
            }
        }
        __syncthreads();
        if (tid == 0) {
            if (last && tl >= 2) {
                X[q].hl[0] = S.f_last2;
                X[q].rl[0] = S.g_last2;
            }
            S.run_cur[0] += kc0;
            S.run_cur[1] += kc1;
            S.run_new[0] += tx2;
            S.run_new[1] += tn2;
        }
        __syncthreads();
        SUB(6);
    }
#ifdef EEMD_TRACE
    if (tid == 0) {
        for (int k = 0; k < 7; ++k) atomicAdd(&C.hdr->sweep_cycles[k], scyc[k]);
    }
#endif
#undef SUB
    // ---------------- publish the segment's results ----------------
    const double2 rs = block_sum2<THREADS>(make_double2(num, den), s_red);
    if (tid == 0) {
        Xchg& xo = X[q];
        xo.hf[0] = S.hf0;
        xo.hf[1] = S.hf1;
        if (mode == TM_SIFT) {
            // the residual is unchanged by a plain sift: carry the previous edges
            const Xchg& xp = X[q ^ 1];
            xo.rf[0] = xp.rf[0];
            xo.rf[1] = xp.rf[1];
            xo.rl[0] = xp.rl[0];
            xo.rl[1] = xp.rl[1];
        } else {
            xo.rf[0] = S.rf0;
            xo.rf[1] = S.rf1;
        }
        xo.num = rs.x;
        xo.den = rs.y;
        xo.cnt[0] = S.run_new[0];
        xo.cnt[1] = S.run_new[1];
    }
}

// ---------------------------------------------------------------------------
// decisions (emd_ref.py:120-153; emd_gpu.py:152-274)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void log_sift(const Ctx& C, const TaskSm& S) {
    if (C.knot_log && S.rank == 0) {
        int32_t* p = C.knot_log + (((int64_t)S.task * C.max_imf + S.imf) * C.max_sifts + S.sift) * 2;
        p[0] = S.P[0];
        p[1] = S.P[1];
    }
}

__device__ __forceinline__ void close_imf(const Ctx& C, TaskSm& S) {
    if (C.mode_sifts && S.rank == 0) C.mode_sifts[(int64_t)S.task * C.max_imf + S.imf] = S.mode_sifts_cur;
    S.nmode = S.imf + 1;
    S.imf += 1;
    S.mode_sifts_cur = 0;
}

// adopt the knots the last sweep produced (segment counts nc[env][r])
__device__ __forceinline__ void adopt(TaskSm& S, const int nc[2][MAXC], int cmax, int cmin) {
    S.kpar ^= 1;
    S.P[0] = cmax;
    S.P[1] = cmin;
    for (int env = 0; env < 2; ++env) {
        int acc = 0;
        for (int r = 0; r < S.csize; ++r) {
            S.pref[env][r] = acc;
            acc += nc[env][r];
        }
        S.pref[env][S.csize] = acc;
    }
}

__device__ __forceinline__ void imf_level(const Ctx& C, TaskSm& S, const int nc[2][MAXC], int cmax,
                                          int cmin) {
    bool stop = (cmax + cmin < C.min_extrema);
    if (C.rules == EEMD_RULES_NUMBA) stop = stop || cmax < 2 || cmin < 2;
    if (stop) { S.phase = PH_DONE; return; }
    if (S.imf >= C.max_imf) { S.phase = PH_DONE; S.flags |= 1; return; }
    S.mode_sifts_cur = 0;
    if (C.rules == EEMD_RULES_REF && (cmax < 1 || cmin < 1)) {
        // emd_ref.py:132-133: the sift loop breaks before its first sift; the IMF is the residual
        S.phase = PH_TRANS;
        S.imf_from_resid = 1;
        return;
    }
    S.phase = PH_SIFT;
    S.sift = 0;
    S.src_resid = 1;
    S.imf_from_resid = 0;
    adopt(S, nc, cmax, cmin);
}

__device__ void decide(const Ctx& C, TaskSm& S, Xchg* X, cg::cluster_group& cl) {
    if (threadIdx.x == 0) {
        const int q = S.step & 1;
        double num = 0.0, den = 0.0;
        int nc[2][MAXC];
        int cmax = 0, cmin = 0;
        for (int r = 0; r < S.csize; ++r) {
            const Xchg* xr = cl.map_shared_rank(&X[q], r);
            num += xr->num;
            den += xr->den;
            nc[0][r] = xr->cnt[0];
            nc[1][r] = xr->cnt[1];
            cmax += nc[0][r];
            cmin += nc[1][r];
        }
        const int mode = S.mode;
        if (mode == TM_SIFT) {
            log_sift(C, S);
            S.mode_sifts_cur += 1;
            S.nsift_total += 1;
            const double sdv = den > 0.0 ? num / den : 0.0;
            bool stop = (S.sift >= 1) && (sdv < C.tau);
            if (!stop) stop = (C.rules == EEMD_RULES_NUMBA) ? (cmax < 2 || cmin < 2) : (cmax < 1 || cmin < 1);
            if (stop) {
                S.phase = PH_TRANS;
                S.imf_from_resid = 0;
            } else {
                S.sift += 1;
                S.src_resid = 0;
                adopt(S, nc, cmax, cmin);
            }
        } else if (mode == TM_LAST) {
            log_sift(C, S);
            S.mode_sifts_cur += 1;
            S.nsift_total += 1;
            close_imf(C, S);
            imf_level(C, S, nc, cmax, cmin);
        } else if (mode == TM_TRANS) {
            close_imf(C, S);
            imf_level(C, S, nc, cmax, cmin);
        } else {
            S.imf = 0;
            S.nmode = 0;
            imf_level(C, S, nc, cmax, cmin);
        }
        S.step += 1;
        // every IMF ends after at most max_sifts sifts plus one closing step
        if (S.phase != PH_DONE && S.step > 2 + C.max_imf * (C.max_sifts + 1)) {
            raise_error(C.hdr, EEMD_E_TIMEOUT, S.task);
            S.phase = PH_DONE;
        }
    }
    __syncthreads();
}

// per-step constants of the envelopes (mirror knots, constant envelope)
template <typename T>
__device__ void step_setup(const Ctx& C, const Slot& sl, TaskSm& S) {
    if (threadIdx.x < 2) {
        const int env = threadIdx.x;
        const int P = S.P[env];
        const int mir = (C.end_mode == EEMD_END_MIRROR && P >= 3) ? 1 : 0;
        S.mir[env] = mir;
        S.p2[env] = P + 2 * mir;
        S.cval[env] = 0.0;
        S.tfirst[env] = S.tlast[env] = 0;
        if (P >= 1) {
            int t0;
            double y0;
            real_knot<T>(C, sl, S, env, 0, t0, y0);
            if (P == 1) S.cval[env] = y0;
            if (mir) {
                int t1, ta, tb;
                double y1, ya, yb;
                real_knot<T>(C, sl, S, env, 1, t1, y1);
                real_knot<T>(C, sl, S, env, P - 1, ta, ya);
                real_knot<T>(C, sl, S, env, P - 2, tb, yb);
                S.tfirst[env] = 2 * t0 - t1;
                S.tlast[env] = 2 * ta - tb;
                S.yfirst[env] = y1;
                S.ylast[env] = yb;
            }
        }
        if (S.p2[env] > C.kcap) raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, S.task);
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// k_emd: the persistent cluster kernel
// ---------------------------------------------------------------------------
#ifndef EEMD_MIN_CTAS_PER_SM
#define EEMD_MIN_CTAS_PER_SM 2
#endif

template <typename T, bool EXACT>
__global__ void __launch_bounds__(THREADS, EEMD_MIN_CTAS_PER_SM) k_emd(const __grid_constant__ Ctx C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TaskSm S;
    __shared__ Xchg X[2];
    __shared__ int s_claim;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int csize = (int)cl.num_blocks();
    const int slot = blockIdx.x / csize;
    const int tid = threadIdx.x;
    const Smem sm = carve<T>(smem_raw, C.tile);
    Slot sl;
    sl.kt = C.kt + (int64_t)slot * C.slot_knots;
    sl.ky = static_cast<T*>(C.ky) + (int64_t)slot * C.slot_knots;
    sl.M = static_cast<T*>(C.M) + (int64_t)slot * C.slot_M;

#ifdef EEMD_TRACE
    unsigned long long cyc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long tmark = clock64();
#define EEMD_PHASE(k)                                   \
    do {                                                \
        const long long now_ = clock64();               \
        cyc[k] += (unsigned long long)(now_ - tmark);   \
        tmark = now_;                                   \
    } while (0)
#else
#define EEMD_PHASE(k) \
    do {              \
    } while (0)
#endif
    for (;;) {
        if (rank == 0 && tid == 0) s_claim = atomicAdd(&C.hdr->next_task, 1);
        cl.sync();
        const int q = *cl.map_shared_rank(&s_claim, 0);
        cl.sync();
        EEMD_PHASE(6);
        if (q >= C.n_tasks) break;
        if (tid == 0) {
            const int task = C.order[q];
            const TaskDesc d = C.td[task];
            S.task = task;
            S.n = d.n;
            S.rank = rank;
            S.csize = csize;
            S.s0 = min(d.n, rank * d.seg);
            S.s1 = min(d.n, S.s0 + d.seg);
            S.phase = PH_INIT;
            S.imf = S.sift = S.kpar = S.src_resid = S.imf_from_resid = 0;
            S.nsift_total = S.nmode = S.mode_sifts_cur = S.flags = S.step = 0;
            S.P[0] = S.P[1] = 0;
            for (int r = 0; r <= MAXC; ++r) S.pref[0][r] = S.pref[1][r] = 0;
            S.mir[0] = S.mir[1] = 0;
            S.f_m1 = S.g_m1 = 0.0;
            if (C.watchdog < 0 && rank == 0) {
                // watchdog test mode: a bounded wait on a flag nothing sets
                long long spins = 0;
                while (*((volatile int32_t*)&C.hdr->wd_flag) == 0) {
                    if (++spins > -C.watchdog) {
                        raise_error(C.hdr, EEMD_E_TIMEOUT, task);
                        break;
                    }
                    __nanosleep(32);
                }
            }
        }
        __syncthreads();
        while (S.phase != PH_DONE) {
            if (tid == 0) {
                if (S.phase == PH_INIT) S.mode = TM_INIT;
                else if (S.phase == PH_TRANS) S.mode = TM_TRANS;
                else S.mode = (S.sift + 1 >= C.max_sifts) ? TM_LAST : TM_SIFT;
            }
            __syncthreads();
            if (S.mode == TM_SIFT || S.mode == TM_LAST) {
                step_setup<T>(C, sl, S);
                EEMD_PHASE(0);
                solve_task<T, EXACT>(C, sl, S, sm);
                EEMD_PHASE(1);
                cl.sync();  // second derivatives of every segment visible
                EEMD_PHASE(2);
            }
            sweep<T, EXACT>(C, sl, S, X, sm, cl);
            EEMD_PHASE(3);
            cl.sync();  // segment results published
            EEMD_PHASE(4);
            decide(C, S, X, cl);
            EEMD_PHASE(5);
        }
        if (rank == 0 && tid == 0) {
            TaskOut o;
            o.nsift = S.nsift_total;
            o.nmode = S.nmode;
            o.flags = S.flags;
            o.pad = 0;
            C.tout[S.task] = o;
            atomicAdd(&C.hdr->n_done, 1);
        }
        __syncthreads();
    }
#ifdef EEMD_TRACE
    if (tid == 0) {
        for (int k = 0; k < 8; ++k) atomicAdd(&C.hdr->phase_cycles[k], cyc[k]);
    }
#endif
#undef EEMD_PHASE
}

// ---------------------------------------------------------------------------
// k_reduce: imf_sum[s][m][t] += trial-ordered sum over the batch (emd_par.py:241-245)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_reduce(const SignalDesc* sdesc, const TaskDesc* td, const TaskOut* tout, const void* imfs,
                         int trial_count, int max_imf, double* imf_sum, int32_t* mode_count) {
    const int s = blockIdx.z, m = blockIdx.y;
    const SignalDesc sd = sdesc[s];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (mode_count && blockIdx.x == 0 && threadIdx.x == 0) {
        int cnt = 0;
        for (int e = 0; e < trial_count; ++e) cnt += (tout[sd.first_task + e].nmode > m) ? 1 : 0;
        mode_count[(int64_t)s * max_imf + m] += cnt;
    }
    if (!imf_sum || t >= sd.n) return;
    double acc = 0.0;
    bool any = false;
    for (int e = 0; e < trial_count; ++e) {
        const int task = sd.first_task + e;
        if (tout[task].nmode > m) {
            const double v = ldv<T>(imfs, td[task].imf_off + (int64_t)m * sd.n + t);
            acc = any ? acc + v : v;
            any = true;
        }
    }
    if (any) {
        double* p = imf_sum + sd.sum_off + (int64_t)m * sd.n + t;
        *p = *p + acc;
    }
}

__global__ void k_outputs(const TaskOut* tout, int n_tasks, int32_t* nsift, int32_t* nmode, int32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tasks) return;
    const TaskOut o = tout[i];
    if (nsift) nsift[i] = o.nsift;
    if (nmode) nmode[i] = o.nmode;
    if (flags) flags[i] = o.flags;
}

// ---------------------------------------------------------------------------
// k_finalize: mean + residual (emd_par.py:248-250)
// ---------------------------------------------------------------------------
constexpr int FIN_BATCH = 256;  // signal descriptors per launch, passed by value
struct FinBatch {
    SignalDesc sd[FIN_BATCH];
};

template <typename T>
__global__ void k_finalize(FinBatch fb, int s_base, int max_imf, const void* x, const double* imf_sum,
                           const int32_t* mode_count, double* imf_mean, double* residual,
                           int32_t* n_modes) {
    const int sl = blockIdx.y;
    const int s = s_base + sl;
    const SignalDesc sd = fb.sd[sl];
    const int32_t* cnt = mode_count + (int64_t)s * max_imf;
    int nm = 0;
    while (nm < max_imf && cnt[nm] > 0) ++nm;
    if (n_modes && blockIdx.x == 0 && threadIdx.x == 0) n_modes[s] = nm;
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= sd.n) return;
    double acc = 0.0;
    for (int m = 0; m < nm; ++m) {
        const int64_t o = sd.sum_off + (int64_t)m * sd.n + t;
        const double v = imf_sum[o] / (double)cnt[m];
        if (imf_mean) imf_mean[o] = v;
        acc = (m == 0) ? v : acc + v;
    }
    if (residual) residual[sd.r_off + t] = ldv<T>(x, sd.x_off + t) - acc;
}

}  // namespace eemd

// ===========================================================================
// host side
// ===========================================================================
using namespace eemd;

namespace {

constexpr int ASSUMED_SMS = 148;        // B200
constexpr int ASSUMED_CTAS_PER_SM = 2;  // resident k_emd CTAs per SM the grid is sized for

struct Layout {
    std::vector<TaskDesc> td;
    std::vector<SignalDesc> sd;
    std::vector<int32_t> order;
    int64_t NS = 0, NIMF = 0, slot_knots = 0, slot_M = 0;
    int tile = 0, B = 0, S = 0, csize = 1, slots = 1, segcap = 0, kcap = 0, scr_rows = 0;
    size_t o_hdr, o_td, o_order, o_tout, o_sd, o_sigma, o_resid, o_imfs, o_kt, o_ky, o_M, o_scr;
    size_t total = 0;
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Launch shapes by length bucket.  The cluster spreads one task over several
// SMs when there are fewer tasks than CTA slots; tiles live inside a segment.
int autotune_tile(int64_t seg) { return seg <= 4096 ? 512 : 1024; }

int autotune_csize(int64_t n_tasks, int64_t nmin) {
    const int64_t budget = (int64_t)ASSUMED_SMS * ASSUMED_CTAS_PER_SM;
    int c = (int)std::max<int64_t>(1, std::min<int64_t>(8, budget / std::max<int64_t>(n_tasks, 1)));
    while (c > 1 && nmin / c < 2048) --c;
    return c;
}

int check_params(const eemd_params* p) {
    if (!p) return EEMD_E_BADARG;
    if (p->dtype != EEMD_F64 && p->dtype != EEMD_F32) return EEMD_E_BADARG;
    if (p->exact && p->dtype != EEMD_F64) return EEMD_E_NOTSUP;
    if (p->max_sifts < 1 || p->max_imf < 1 || p->max_imf > 4096) return EEMD_E_BADARG;
    if (p->end_mode != EEMD_END_NATURAL && p->end_mode != EEMD_END_MIRROR) return EEMD_E_BADARG;
    if (p->rules != EEMD_RULES_REF && p->rules != EEMD_RULES_NUMBA) return EEMD_E_BADARG;
    if (p->noise_mode < EEMD_NOISE_NONE || p->noise_mode > EEMD_NOISE_PREPERTURBED) return EEMD_E_BADARG;
    if (p->tile != 0 && p->tile != 256 && p->tile != 512 && p->tile != 1024) return EEMD_E_BADARG;
    if (p->knots_per_block < 0 || p->knots_per_block > 4096 || p->halo < 0 || p->halo > 256)
        return EEMD_E_BADARG;
    if (p->cluster_size < 0 || p->cluster_size > 8) return EEMD_E_BADARG;
    return EEMD_OK;
}

int make_layout(const eemd_params* p, const int64_t* lengths, int n_signals, int trial_count,
                int trial_begin, bool imfs_external, Layout& L) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!lengths || n_signals < 1 || trial_count < 1) return EEMD_E_BADARG;
    const int64_t n_tasks = (int64_t)n_signals * trial_count;
    if (n_tasks > (1 << 24)) return EEMD_E_BADARG;
    int64_t nmax = 0, nmin = INT64_MAX;
    for (int s = 0; s < n_signals; ++s) {
        if (lengths[s] < 3 || lengths[s] > (1LL << 30)) return EEMD_E_BADARG;
        nmax = std::max(nmax, lengths[s]);
        nmin = std::min(nmin, lengths[s]);
    }
    L.csize = p->cluster_size ? p->cluster_size : autotune_csize(n_tasks, nmin);
    L.S = p->halo ? p->halo : (p->exact ? 32 : 24);
    L.B = p->knots_per_block ? p->knots_per_block : 64;
    if (p->exact && (2 * L.S + L.B + 8 > SOLVE_CAP)) return EEMD_E_BADARG;
    if (!p->exact && 2 * L.S + FAST_B + 8 > SOLVE_CAP) return EEMD_E_BADARG;
    int64_t segmax = 0;
    L.td.resize(n_tasks);
    L.sd.resize(n_signals);
    int64_t xo = 0, so = 0, imo = 0, sumo = 0;
    for (int s = 0; s < n_signals; ++s) {
        const int64_t n = lengths[s];
        SignalDesc& sd = L.sd[s];
        sd.x_off = xo;
        sd.sum_off = sumo;
        sd.r_off = xo;
        sd.n = (int32_t)n;
        sd.first_task = s * trial_count;
        sumo += (int64_t)p->max_imf * n;
        int64_t seg = (n + L.csize - 1) / L.csize;
        seg = (seg + 31) / 32 * 32;
        if ((L.csize - 1) * seg + 2 > n) return EEMD_E_BADARG;  // every segment keeps >= 2 samples
        segmax = std::max(segmax, seg);
        for (int e = 0; e < trial_count; ++e) {
            TaskDesc& d = L.td[(int64_t)s * trial_count + e];
            d.x_off = (p->noise_mode == EEMD_NOISE_PREPERTURBED) ? so : xo;
            d.s_off = so;
            d.imf_off = imo;
            d.noise_off = so;
            d.n = (int32_t)n;
            d.signal = s;
            d.trial = trial_begin + e;
            d.seg = (int32_t)seg;
            so += n;
            imo += (int64_t)p->max_imf * n;
        }
        xo += n;
    }
    // longest tasks first: the work queue hands them out in this order
    L.order.resize(n_tasks);
    std::iota(L.order.begin(), L.order.end(), 0);
    std::stable_sort(L.order.begin(), L.order.end(), [&](int a, int b) { return L.td[a].n > L.td[b].n; });
    L.tile = p->tile ? p->tile : autotune_tile(segmax);
    L.segcap = (int)(segmax / 2 + 2);
    L.kcap = (int)(nmax / 2 + 4);
    L.slots = (int)std::max<int64_t>(
        1, std::min<int64_t>(n_tasks, (int64_t)ASSUMED_SMS * ASSUMED_CTAS_PER_SM / L.csize));
    L.slot_knots = (int64_t)2 * 2 * L.csize * L.segcap;
    L.slot_M = (int64_t)2 * 5 * L.kcap;
    L.scr_rows = p->exact ? (L.B + L.S) : 0;
    L.NS = so;
    L.NIMF = imo;
    const size_t bt = (p->dtype == EEMD_F64) ? 8 : 4;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    L.o_hdr = take(sizeof(Header));
    L.o_td = take(sizeof(TaskDesc) * n_tasks);
    L.o_order = take(sizeof(int32_t) * n_tasks);
    L.o_tout = take(sizeof(TaskOut) * n_tasks);
    L.o_sd = take(sizeof(SignalDesc) * n_signals);
    L.o_sigma = take(sizeof(double) * n_signals);
    L.o_resid = take(bt * L.NS);
    L.o_imfs = imfs_external ? 0 : take(bt * L.NIMF);
    L.o_kt = take(sizeof(int32_t) * L.slot_knots * L.slots);
    L.o_ky = take(bt * L.slot_knots * L.slots);
    L.o_M = take(bt * L.slot_M * L.slots);
    L.o_scr = take(sizeof(double2) * (size_t)L.scr_rows * L.slots * L.csize * THREADS);
    L.total = off;
    return EEMD_OK;
}

// Optional per-launch CUDA-event timing (eemd_run_traced): one event pair
// per kernel launch, summed per kernel kind after the final synchronise.
struct Tracer {
    eemd_kernel_times* out = nullptr;
    std::vector<cudaEvent_t> ev;
    std::vector<int> kind;
    cudaStream_t st = nullptr;
    int64_t counts[EEMD_KERNEL_KINDS] = {0};
    void begin(int k) {
        counts[k] += 1;
        if (!out) return;
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, st);
        ev.push_back(a);
        ev.push_back(b);
        kind.push_back(k);
    }
    void end() {
        if (!out) return;
        cudaEventRecord(ev.back(), st);
    }
    void finish() {
        if (!out) return;
        for (int k = 0; k < EEMD_KERNEL_KINDS; ++k) {
            out->ms[k] = 0.0;
            out->launches[k] = counts[k];
        }
        for (size_t i = 0; i < kind.size(); ++i) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]) == cudaSuccess) out->ms[kind[i]] += ms;
        }
        for (auto e : ev) cudaEventDestroy(e);
        ev.clear();
        kind.clear();
    }
};

template <typename T, bool EXACT>
int launch_emd(const Ctx& C, const Layout& L, cudaStream_t st, Tracer& tr) {
    const size_t smem = smem_bytes(L.tile, (int)sizeof(T));
    if (cudaFuncSetAttribute(k_emd<T, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return EEMD_E_CUDA;
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(L.slots * L.csize), 1, 1);
    cfg.blockDim = dim3(THREADS, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)L.csize;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    tr.begin(EEMD_K_EMD);
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_emd<T, EXACT>, C);
    tr.end();
    return e == cudaSuccess ? EEMD_OK : EEMD_E_CUDA;
}

template <typename T>
int run_typed(const eemd_params* p, const Layout& L, Ctx& C, double* imf_sum, int32_t* mode_count,
              int32_t* nsift, int32_t* nmode, int32_t* flags, void* resid_out, cudaStream_t st,
              Tracer& tr) {
    const int64_t n_tasks = (int64_t)L.td.size();
    if (p->noise_mode == EEMD_NOISE_PHILOX) {
        tr.begin(EEMD_K_SIGMA);
        k_sigma<T><<<(int)L.sd.size(), 1024, 0, st>>>(C.sd, C.x, p->eps, const_cast<double*>(C.sigma));
        tr.end();
    }
    int rc = p->exact ? launch_emd<T, true>(C, L, st, tr) : launch_emd<T, false>(C, L, st, tr);
    if (rc) return rc;
    if (imf_sum || mode_count) {
        int64_t nmax = 0;
        for (auto& s : L.sd) nmax = std::max<int64_t>(nmax, s.n);
        dim3 g((unsigned)((nmax + 255) / 256), (unsigned)p->max_imf, (unsigned)L.sd.size());
        tr.begin(EEMD_K_REDUCE);
        k_reduce<T><<<g, 256, 0, st>>>(C.sd, C.td, C.tout, C.imfs, C.trial_count, C.max_imf, imf_sum,
                                        mode_count);
        tr.end();
    }
    if (nsift || nmode || flags) {
        tr.begin(EEMD_K_OUTPUTS);
        k_outputs<<<(int)((n_tasks + 255) / 256), 256, 0, st>>>(C.tout, (int)n_tasks, nsift, nmode, flags);
        tr.end();
    }
    if (resid_out) {
        cudaMemcpyAsync(resid_out, C.resid, (size_t)L.NS * sizeof(T), cudaMemcpyDeviceToDevice, st);
    }
    return cudaGetLastError() == cudaSuccess ? EEMD_OK : EEMD_E_CUDA;
}

}  // namespace

extern "C" {

void eemd_default_params(eemd_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->dtype = EEMD_F64;
    p->noise_mode = EEMD_NOISE_NONE;
    p->eps = 0.2;
    p->seed = 0;
    p->tau = 0.25;
    p->max_sifts = 50;
    p->max_imf = 16;
    p->min_extrema = 4;
    p->end_mode = EEMD_END_NATURAL;
    p->rules = EEMD_RULES_REF;
    p->exact = 0;
}

int32_t eemd_version(void) { return EEMD_ABI_VERSION; }

const char* eemd_strerror(int32_t status) {
    switch (status) {
        case EEMD_OK: return "ok";
        case EEMD_E_BADARG: return "invalid argument";
        case EEMD_E_NOMEM: return "workspace too small";
        case EEMD_E_KNOT_OVERFLOW: return "knot buffer capacity exceeded";
        case EEMD_E_TIMEOUT: return "device wait gave up (watchdog)";
        case EEMD_E_CUDA: return "CUDA runtime error";
        case EEMD_E_NOTSUP: return "unsupported parameter combination";
        case EEMD_E_STATIC_CAPACITY:
            return "problem needs more scratch than the static scratch of eemd_run_static "
                   "(EEMD_STATIC_SCRATCH_BYTES); use eemd_run with a workspace";
        default: return "unknown status";
    }
}

int32_t eemd_workspace_size(const eemd_params* p, const int64_t* lengths, int32_t n_signals,
                            int32_t trial_count, int32_t imfs_external, size_t* ws_bytes) {
    if (!ws_bytes) return EEMD_E_BADARG;
    Layout L;
    int rc = make_layout(p, lengths, n_signals, trial_count, 0, imfs_external != 0, L);
    if (rc) return rc;
    *ws_bytes = L.total;
    return EEMD_OK;
}

int32_t eemd_run(const eemd_params* p, const void* x, const int64_t* lengths, int32_t n_signals,
                 int32_t trial_begin, int32_t trial_count, const void* noise, void* imfs,
                 void* resid_out, double* imf_sum, int32_t* mode_count, int32_t* nsift,
                 int32_t* nmode, int32_t* mode_sifts, int32_t* knot_log, int32_t* flags, void* ws,
                 size_t ws_bytes, void* stream) {
    return eemd_run_traced(p, x, lengths, n_signals, trial_begin, trial_count, noise, imfs, resid_out,
                           imf_sum, mode_count, nsift, nmode, mode_sifts, knot_log, flags, ws, ws_bytes,
                           stream, nullptr);
}

int32_t eemd_run_traced(const eemd_params* p, const void* x, const int64_t* lengths, int32_t n_signals,
                        int32_t trial_begin, int32_t trial_count, const void* noise, void* imfs,
                        void* resid_out, double* imf_sum, int32_t* mode_count, int32_t* nsift,
                        int32_t* nmode, int32_t* mode_sifts, int32_t* knot_log, int32_t* flags,
                        void* ws, size_t ws_bytes, void* stream, eemd_kernel_times* times) {
    Layout L;
    int rc = make_layout(p, lengths, n_signals, trial_count, trial_begin, imfs != nullptr, L);
    if (rc) return rc;
    if (!x || !ws) return EEMD_E_BADARG;
    if (p->noise_mode == EEMD_NOISE_INJECTED && !noise) return EEMD_E_BADARG;
    if (ws_bytes < L.total) return EEMD_E_NOMEM;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(ws);
    Ctx C;
    memset(&C, 0, sizeof(C));
    C.hdr = reinterpret_cast<Header*>(base + L.o_hdr);
    C.td = reinterpret_cast<const TaskDesc*>(base + L.o_td);
    C.order = reinterpret_cast<const int32_t*>(base + L.o_order);
    C.tout = reinterpret_cast<TaskOut*>(base + L.o_tout);
    C.sd = reinterpret_cast<const SignalDesc*>(base + L.o_sd);
    C.sigma = reinterpret_cast<const double*>(base + L.o_sigma);
    C.resid = base + L.o_resid;
    C.imfs = imfs ? imfs : (void*)(base + L.o_imfs);
    C.kt = reinterpret_cast<int32_t*>(base + L.o_kt);
    C.ky = base + L.o_ky;
    C.M = base + L.o_M;
    C.scr = reinterpret_cast<double2*>(base + L.o_scr);
    C.x = x;
    C.noise = noise;
    C.knot_log = knot_log;
    C.mode_sifts = mode_sifts;
    C.slot_knots = L.slot_knots;
    C.slot_M = L.slot_M;
    C.segcap = L.segcap;
    C.kcap = L.kcap;
    C.n_tasks = (int32_t)L.td.size();
    C.n_signals = n_signals;
    C.trial_count = trial_count;
    C.csize = L.csize;
    C.max_sifts = p->max_sifts;
    C.max_imf = p->max_imf;
    C.min_extrema = p->min_extrema;
    C.end_mode = p->end_mode;
    C.rules = p->rules;
    C.noise_mode = p->noise_mode;
    C.tile = L.tile;
    C.B = L.B;
    C.S = L.S;
    C.scr_rows = L.scr_rows;
    C.tau = p->tau;
    C.seed = p->seed;
    C.watchdog = p->watchdog != 0 ? p->watchdog : (1LL << 24);

    if (cudaMemsetAsync(base + L.o_hdr, 0, sizeof(Header), st) != cudaSuccess) return EEMD_E_CUDA;
    if (cudaMemcpyAsync(base + L.o_td, L.td.data(), sizeof(TaskDesc) * L.td.size(), cudaMemcpyHostToDevice,
                        st) != cudaSuccess)
        return EEMD_E_CUDA;
    if (cudaMemcpyAsync(base + L.o_order, L.order.data(), sizeof(int32_t) * L.order.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return EEMD_E_CUDA;
    if (cudaMemcpyAsync(base + L.o_sd, L.sd.data(), sizeof(SignalDesc) * L.sd.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return EEMD_E_CUDA;
    if (knot_log) {
        const size_t nb = sizeof(int32_t) * 2 * L.td.size() * (size_t)p->max_imf * p->max_sifts;
        if (cudaMemsetAsync(knot_log, 0xff, nb, st) != cudaSuccess) return EEMD_E_CUDA;
    }
    if (mode_sifts) {
        if (cudaMemsetAsync(mode_sifts, 0, sizeof(int32_t) * L.td.size() * p->max_imf, st) != cudaSuccess)
            return EEMD_E_CUDA;
    }
    Tracer tr;
    tr.out = times;
    tr.st = st;
    rc = (p->dtype == EEMD_F64)
             ? run_typed<double>(p, L, C, imf_sum, mode_count, nsift, nmode, flags, resid_out, st, tr)
             : run_typed<float>(p, L, C, imf_sum, mode_count, nsift, nmode, flags, resid_out, st, tr);
    if (cudaStreamSynchronize(st) != cudaSuccess) return EEMD_E_CUDA;
    tr.finish();
    if (rc) return rc;
    Header h;
    if (cudaMemcpy(&h, C.hdr, sizeof(Header), cudaMemcpyDeviceToHost) != cudaSuccess) return EEMD_E_CUDA;
    if (h.error) return h.error;
    if (h.n_done != C.n_tasks) return EEMD_E_CUDA;
    return EEMD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point: the engine's scratch is this file-scope device
// array.  In host code `g_static_scratch` only names the symbol; its device
// address is looked up once per device with cudaGetSymbolAddress.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_static_scratch[EEMD_STATIC_SCRATCH_BYTES];

namespace {
constexpr int MAX_DEVICES = 64;
std::mutex g_static_mu;
void* g_static_addr[MAX_DEVICES] = {nullptr};
}  // namespace

extern "C" {

int32_t eemd_run_static(const eemd_params* p, const void* x, const int64_t* lengths, int32_t n_signals,
                        int32_t trial_begin, int32_t trial_count, const void* noise, void* imfs,
                        void* resid_out, double* imf_sum, int32_t* mode_count, int32_t* nsift,
                        int32_t* nmode, int32_t* mode_sifts, int32_t* knot_log, int32_t* flags,
                        void* stream) {
    size_t need = 0;
    int32_t rc = eemd_workspace_size(p, lengths, n_signals, trial_count, imfs != nullptr ? 1 : 0, &need);
    if (rc) return rc;
    if (need > (size_t)EEMD_STATIC_SCRATCH_BYTES) return EEMD_E_STATIC_CAPACITY;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return EEMD_E_CUDA;
    if (dev < 0 || dev >= MAX_DEVICES) return EEMD_E_NOTSUP;
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_static_mu);
        if (g_static_addr[dev] == nullptr) {
            void* addr = nullptr;
            if (cudaGetSymbolAddress(&addr, g_static_scratch) != cudaSuccess || addr == nullptr)
                return EEMD_E_CUDA;
            g_static_addr[dev] = addr;
        }
        base = g_static_addr[dev];
    }
    return eemd_run(p, x, lengths, n_signals, trial_begin, trial_count, noise, imfs, resid_out, imf_sum,
                    mode_count, nsift, nmode, mode_sifts, knot_log, flags, base,
                    (size_t)EEMD_STATIC_SCRATCH_BYTES, stream);
}

int32_t eemd_finalize(const eemd_params* p, const void* x, const int64_t* lengths, int32_t n_signals,
                      const double* imf_sum, const int32_t* mode_count, double* imf_mean, double* residual,
                      int32_t* n_modes, void* stream) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!x || !lengths || n_signals < 1 || !imf_sum || !mode_count) return EEMD_E_BADARG;
    std::vector<SignalDesc> sd(n_signals);
    int64_t xo = 0, sumo = 0;
    for (int s = 0; s < n_signals; ++s) {
        if (lengths[s] < 1) return EEMD_E_BADARG;
        sd[s].x_off = xo;
        sd[s].r_off = xo;
        sd[s].sum_off = sumo;
        sd[s].n = (int32_t)lengths[s];
        sd[s].first_task = 0;
        xo += lengths[s];
        sumo += (int64_t)p->max_imf * lengths[s];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    for (int s0 = 0; s0 < n_signals; s0 += FIN_BATCH) {
        const int ns = std::min(FIN_BATCH, n_signals - s0);
        FinBatch fb;
        memset(&fb, 0, sizeof(fb));
        int64_t bmax = 1;
        for (int i = 0; i < ns; ++i) {
            fb.sd[i] = sd[s0 + i];
            bmax = std::max<int64_t>(bmax, sd[s0 + i].n);
        }
        dim3 g((unsigned)((bmax + 255) / 256), (unsigned)ns);
        if (p->dtype == EEMD_F64)
            k_finalize<double><<<g, 256, 0, st>>>(fb, s0, p->max_imf, x, imf_sum, mode_count, imf_mean,
                                                  residual, n_modes);
        else
            k_finalize<float><<<g, 256, 0, st>>>(fb, s0, p->max_imf, x, imf_sum, mode_count, imf_mean,
                                                 residual, n_modes);
    }
    if (cudaStreamSynchronize(st) != cudaSuccess) return EEMD_E_CUDA;
    return cudaGetLastError() == cudaSuccess ? EEMD_OK : EEMD_E_CUDA;
}

}  // extern "C"
