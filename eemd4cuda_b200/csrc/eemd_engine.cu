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

// out[e][t] = the standard normal the Philox noise mode adds to trial
// trial_begin + e of signal `signal` at sample t (before the eps*std(x) scale)
__global__ void k_philox_fill(uint64_t seed, int signal, int trial_begin, int trials, int64_t n, double* out) {
    const int64_t total = (int64_t)trials * n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = philox_normal(seed, signal, trial_begin + (int)(i / n), i % n);
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
constexpr int MAXSEG = MAXC * MAXNW;  // knot segments per task: one per warp of up to MAXC CTAs

struct Xchg {              // one CTA's published segment results (DSMEM-visible)
    double num, den;       // SD partial sums of the segment
    int cnt[2][MAXNW];     // new knots (maxima, minima) found by each warp
    int err;               // this CTA raised an error during the step: the task stops
};

struct TaskSm {
    int task, n, s0, s1, rank, csize;
    int phase, imf, sift, kpar, src_resid, imf_from_resid;
    int nsift_total, nmode, mode_sifts_cur, flags, step, mode;
    int P[2];                  // current knot totals
    int pref[2][2][MAXSEG + 1];  // [list parity][env]: knots before each (CTA, warp) segment
    int mir[2], p2[2], tfirst[2], tlast[2];
    double yfirst[2], ylast[2];  // values of the virtual mirror knots
    double cval[2];            // constant envelope when P == 1
    int rcur;                  // current residual: 0 = the task's residual array, 1 = slot scratch
    int err;                   // this CTA raised an error during the current step
    int setup_fail;            // step_setup found a capacity exceeded (identical in every CTA)
};

// An error of the running task: recorded in the header (first error wins) and
// in the CTA's step flag, which decide() ORs over the cluster so that every
// CTA stops the task at the same step (no further step reads what the failed
// step left behind).
__device__ __forceinline__ void task_error(const Ctx& C, TaskSm& S, int code) {
    raise_error(C.hdr, code, S.task);
    S.err = 1;
}

#ifdef EEMD_CHECKED
// checked build: an interval record index outside [0, hi] is reported and
// clamped instead of read out of bounds
#define EEMD_CHECK_IV(k, hi)                                     \
    do {                                                         \
        if ((k) < 0 || (k) > (hi)) {                             \
            task_error(C, S, EEMD_E_KNOT_OVERFLOW);              \
            (k) = max(0, min((k), (hi)));                        \
        }                                                        \
    } while (0)
#else
#define EEMD_CHECK_IV(k, hi) \
    do {                     \
    } while (0)
#endif

// Per-warp sweep geometry for storage type T.  A warp tile is WT = 32*RUN
// samples; each warp owns, in dynamic shared memory, two tile buffers per
// stream (h, residual) and two sets of run records.  Interval records are
// RS storage-type elements (32 or 48 bytes).
template <typename T>
struct Geo {
    static constexpr int RUN = sizeof(T) == 4 ? 8 : 4;  // consecutive samples per lane
    static constexpr int WT = 32 * RUN;                 // samples per warp tile
    static constexpr int TB = WT + 4;                   // tile buffer elements (16-byte phase)
    static constexpr int RS = sizeof(T) == 4 ? 8 : 6;   // interval record stride
    static constexpr int NBUF = TILE_BUFS;               // tiles in flight per warp (ring)
    static constexpr size_t TB_BYTES = (size_t)NBUF * 2 * TB * sizeof(T);  // [buf][stream][TB]
    static constexpr size_t RI_BYTES = (size_t)NBUF * 32 * 16;          // [buf][lane]
    static constexpr int KCAP = WT / 2 + 4;                              // knots of one kind in a tile
    static constexpr size_t KN_BYTES = (size_t)2 * KCAP * (4 + sizeof(T));  // [kind][KCAP] index, value
    static constexpr size_t WARP_BYTES = TB_BYTES + RI_BYTES + KN_BYTES;
    static_assert(TB_BYTES % 16 == 0 && (RS * sizeof(T)) % 16 == 0 && KN_BYTES % 16 == 0,
                  "16-byte aligned layouts");
};


__host__ __device__ inline int stage_pad(int k) { return k + (k >> 4); }

// Staging slot of knot k.  The lanes of a solve pass read knots one window
// width apart: exact windows (16 knots) pad one slot every 16 so that the
// lanes spread over the banks; fast windows of an odd width already hit 32
// distinct banks unpadded (stride 3 is a permutation of the 32 banks, and of
// the 16 bank pairs of a half-warp's doubles), and padding would collide them.
template <bool EXACT>
__host__ __device__ inline int stage_slot(int k) {
    return (EXACT || FAST_B % 2 == 0) ? stage_pad(k) : k;
}

__host__ __device__ inline size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

// rows of one fast-solve pass: 32 lanes of FAST_B rows
constexpr int FAST_ROWS = 32 * FAST_B;
// largest seam halo of the fast solve, and the knots one fast pass stages:
// its rows, the left halo and the two knots past the last row
constexpr int FAST_SMAX = 64;
constexpr int WSCAP_FAST = FAST_ROWS + FAST_SMAX + 3;

// knots a solve pass stages per warp: exact windows carry both halos (up to
// WSCAP knots); the fast solve's lanes need WSCAP_FAST
__host__ __device__ constexpr int stage_cap(bool exact) { return exact ? WSCAP : WSCAP_FAST; }

// per-warp solve area: slopes (double), knot times (int), knot values
// (storage type), and in fast mode the forward (c, d) of a pass's rows.  It
// overlays the sweep's area; keeping it no larger leaves the L1 share of the
// SM's on-chip memory (used by the sweep's record loads) unchanged.
__host__ __device__ inline size_t wsolve_bytes(size_t bt, bool exact) {
    const size_t sp = (size_t)stage_pad(stage_cap(exact));
    return align16(sp * 8) + align16(sp * 4) + align16(sp * bt) + (exact ? 0 : (size_t)FAST_ROWS * 16);
}

// dynamic shared memory of k_emd: the sweep's and the solve's per-warp areas overlay
__host__ __device__ inline size_t smem_bytes(int bt, bool exact, int nw) {
    const size_t sweep = nw * (bt == 8 ? Geo<double>::WARP_BYTES : Geo<float>::WARP_BYTES);
    const size_t solve = nw * wsolve_bytes((size_t)bt, exact);
    return sweep > solve ? sweep : solve;
}

// ---------------------------------------------------------------------------
// segmented knot lists: real knot i lives in segment r = seg_of(i) at
// position i - pref[r] of that segment's list
// ---------------------------------------------------------------------------
struct Slot {
    int32_t* kt;   // knot lists (segmented)
    void* ky;
    void* M;       // interval records, mirror space: [2 env][5][kcap] storage type
    void* w1;      // scratch h buffer of the running task (storage type)
    void* r1;      // second residual buffer of the running task (storage type)
    int4* ri;      // run records [2 parity][runs]: first knot of each kind, knot masks
};

__device__ __forceinline__ int64_t knot_index(const Ctx& C, int par, int env, int seg, int i) {
    return ((int64_t)((par * 2 + env) * C.csize * C.nw + seg)) * C.segcap + i;
}

// segment holding real knot i: largest r in [lo, hi) with pref[r] <= i
__device__ __forceinline__ int seg_of(const int* pref, int lo, int hi, int i) {
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pref[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// element offset of real knot i in the current knot lists
__device__ __forceinline__ int64_t real_off(const Ctx& C, const TaskSm& S, int env, int i) {
    const int* pr = S.pref[S.kpar][env];
    const int a = S.rank * C.nw, b = a + C.nw;  // most lookups fall in the CTA's own segments
    const int r = (i >= pr[a] && i < pr[b]) ? seg_of(pr, a, b, i) : seg_of(pr, 0, S.csize * C.nw, i);
    return knot_index(C, S.kpar, env, r, i - pr[r]);
}

template <typename T>
__device__ __forceinline__ void real_knot(const Ctx& C, const Slot& sl, const TaskSm& S, int env, int i,
                                          int& t, double& y) {
    const int64_t o = real_off(C, S, env, i);
    t = __ldcg(sl.kt + o);
    y = (double)__ldcg(static_cast<const T*>(sl.ky) + o);
}

// Stage the mirror-space knots rlo .. rlo+kcount-1 (lane-strided); each lane
// finds the segment of its first real knot by binary search and then walks
// forward, since its later knots follow in the same or later segments.
template <typename T, bool EXACT>
__device__ __forceinline__ void stage_range(const Ctx& C, const Slot& sl, TaskSm& S, int env, int rlo,
                                            int kcount, int* skt, T* sky, int lane) {
    const int* pr = S.pref[S.kpar][env];
    const int nseg = S.csize * C.nw;
    const int mir = S.mir[env], P = S.P[env];
    int r = -1;
    for (int k = lane; k < kcount; k += 32) {
        int i2 = rlo + k;
        int* kt_s = &skt[stage_slot<EXACT>(k)];
        T* ky_s = &sky[stage_slot<EXACT>(k)];
        if (mir) {
            if (i2 == 0) {
                *kt_s = S.tfirst[env];
                *ky_s = (T)S.yfirst[env];
                continue;
            }
            if (i2 == P + 1) {
                *kt_s = S.tlast[env];
                *ky_s = (T)S.ylast[env];
                continue;
            }
            i2 -= 1;
        }
        if (r < 0) r = seg_of(pr, 0, nseg, i2);
        while (r + 1 < nseg && i2 >= pr[r + 1]) ++r;
#ifdef EEMD_CHECKED
        if (i2 < 0 || i2 >= P || i2 - pr[r] >= C.segcap) {
            task_error(C, S, EEMD_E_KNOT_OVERFLOW);
            continue;
        }
#endif
        const int64_t o = knot_index(C, S.kpar, env, r, i2 - pr[r]);
        cp_async4(kt_s, sl.kt + o);
        cp_async_el<T>(ky_s, static_cast<const T*>(sl.ky) + o);
    }
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

#define SKT(k) skt[stage_slot<kExact>(k)]
#define SSL(k) ssl[stage_slot<kExact>(k)]

// Interval records of one envelope in mirror space: RS storage-type elements
// per record: [0] t_k (integer bit pattern), [1] y_k, [2] fast: c1 / exact:
// M_k, [3] c2, [4] c3.
template <typename T>
struct Rec {
    T* rc;
    __device__ __forceinline__ T& at(int k, int e) const { return rc[(int64_t)k * Geo<T>::RS + e]; }
};

// exact: forward elimination from w0 (outer coupling dropped), back
// substitution from w1; identical recurrences to serial Thomas (emd_ref.py:50-65).
// Writes (t_k, y_k, M_k) of the owned knots k = o0+1 .. o1+1 (+ both end knots).
template <typename T>
__device__ void window_exact(const Ctx& C, const int* skt, const T* sky, const double* ssl, int base,
                             int n, int w, const Rec<T>& R, int p2) {
    constexpr bool kExact = true;
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
        R.at(k, 0) = tbits<T>(SKT(k - base));
        R.at(k, 1) = sky[stage_slot<kExact>(k - base)];
        R.at(k, 2) = (T)Mk;
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

// fast: each lane owns FAST_B consecutive rows of a pass.  The forward
// elimination (coupling dropped S rows before the lane's first row, where the
// influence of the neglected rows has decayed like prod c_i) stores (c_i, d_i)
// of the owned rows in the warp's shared memory; after __syncwarp each
// committing lane back-substitutes from S rows past its last row (x there
// truncated to d, the neglected term decaying the same way) down to its first
// row and writes the monomial interval records of its rows.  The lanes of a
// pass's last H = ceil(S / FAST_B) windows only provide that right halo
// (unless the pass reaches the envelope's last row) and are solved for good
// by the next pass.  Per owned row: (S + FAST_B) / FAST_B eliminated rows and
// as many back-substitution steps (one fused multiply-add each).
template <typename T>
__device__ __forceinline__ void window_fast_fwd(const int* skt, const double* ssl, int base, int n, int w, int S,
                                                double2* cd, int cdbase) {
    constexpr bool kExact = false;
    const int o0 = w * FAST_B;
    const int o1 = min(n, o0 + FAST_B) - 1;
    const int r0 = max(0, o0 - S);
    double cp = 0.0, dp = 0.0;
    int ta = SKT(r0 - base), tb = SKT(r0 + 1 - base);
    double sa = SSL(r0 - base);
    for (int i = r0; i <= o1; ++i) {
        const int tc = SKT(i + 2 - base);
        const double sb = SSL(i + 1 - base);
        const Row rw = row_of(ta, tb, tc, sa, sb, i, n);
        const double inv = fast_rcp(fma(-rw.l, cp, rw.dg));
        cp = rw.u * inv;
        dp = fma(-rw.l, dp, rw.r) * inv;
        if (i >= o0) cd[i - cdbase] = make_double2(cp, dp);
        ta = tb;
        tb = tc;
        sa = sb;
    }
}

// Back substitution of window w (rows o0..o1; x_i = M at mirror knot i+1) and
// its interval records: interval i+1 for every owned row i (knots i+1, i+2),
// and interval 0 (M_0 = 0 at the natural end) for the first window.
template <typename T>
__device__ __forceinline__ void window_fast_back(const int* skt, const T* sky, const double* ssl, int base, int n,
                                                 int w, int S, const double2* cd, int cdbase, const Rec<T>& R) {
    constexpr bool kExact = false;
    const int o0 = w * FAST_B;
    const int o1 = min(n, o0 + FAST_B) - 1;
    const int rh = min(n - 1, o1 + S);
    // monomial record of interval k (knots k, k+1; M_k = Ma, M_{k+1} = Mb):
    // y_k + s(c1 + s(c2 + s c3)), s = t - t_k, c1 = slope - h(2Ma + Mb)/6,
    // c2 = Ma/2, c3 = (Mb - Ma)/(6h)
    auto put = [&](int k, double Ma, double Mb) {
        const int t0 = SKT(k - base), t1 = SKT(k + 1 - base);
        const double h = (double)(t1 - t0);
        R.at(k, 0) = tbits<T>(t0);
        R.at(k, 1) = sky[stage_slot<kExact>(k - base)];
        R.at(k, 2) = (T)fma(-h * (1.0 / 6.0), fma(2.0, Ma, Mb), SSL(k - base));
        R.at(k, 3) = (T)(0.5 * Ma);
        R.at(k, 4) = (T)((Mb - Ma) * fast_rcp(h) * (1.0 / 6.0));
    };
    double xn = 0.0;  // x_{i+1}: zero past the natural end (M = 0) or at the truncation
    for (int i = rh; i >= o0; --i) {
        const double2 c = cd[i - cdbase];
        const double xi = fma(-c.x, xn, c.y);
        if (i <= o1) put(i + 1, xi, xn);
        xn = xi;
    }
    if (o0 == 0) put(0, 0.0, xn);
}

#undef SKT
#undef SSL

template <typename T, bool EXACT, int NW>
__device__ void solve_task(const Ctx& C, const Slot& sl, TaskSm& S, unsigned char* smem) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
#ifdef EEMD_TRACE
    unsigned long long scyc[3] = {0, 0, 0};
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
    // one or two knots: a constant or the straight line through them (M = 0)
    for (int env = 0; env < 2; ++env) {
        const int p2 = S.p2[env];
        if (p2 - 2 > 0 || S.rank != 0 || tid >= p2) continue;
        Rec<T> R;
        R.rc = static_cast<T*>(sl.M) + (int64_t)env * C.kcap * Geo<T>::RS;
        int tk, t1;
        double yk, y1;
        knot2<T>(C, sl, S, env, tid, tk, yk);
        R.at(tid, 0) = tbits<T>(tk);
        R.at(tid, 1) = (T)yk;
        R.at(tid, 2) = (T)0;
        R.at(tid, 3) = (T)0;
        R.at(tid, 4) = (T)0;
        if (!EXACT && tid + 1 < p2) {
            knot2<T>(C, sl, S, env, tid + 1, t1, y1);
            R.at(tid, 2) = (T)((y1 - yk) / (double)(t1 - tk));
        }
    }
    // The windows of both envelopes form one list (envelope 0 first); CTA r
    // takes an even share of it and each warp a contiguous part of the CTA's
    // share, solved 32 windows (one per lane) at a time from the warp's own
    // knot staging area: no block-wide barriers.
    const int Bw = EXACT ? C.B : FAST_B;
    const int n0 = max(0, S.p2[0] - 2), n1 = max(0, S.p2[1] - 2);
    const int nw0 = (n0 + Bw - 1) / Bw, nw1 = (n1 + Bw - 1) / Bw;
    const int nwt = nw0 + nw1;
    const int ca = (int)((int64_t)S.rank * nwt / S.csize), cb = (int)((int64_t)(S.rank + 1) * nwt / S.csize);
    const int wa = ca + (int)((int64_t)wid * (cb - ca) / NW);
    const int wb = ca + (int)((int64_t)(wid + 1) * (cb - ca) / NW);
    constexpr int CAP = stage_cap(EXACT);
    unsigned char* ws = smem + (size_t)wid * wsolve_bytes(sizeof(T), EXACT);
    double* ssl = reinterpret_cast<double*>(ws);
    int* skt = reinterpret_cast<int*>(ws + align16(stage_pad(CAP) * 8));
    T* sky = reinterpret_cast<T*>(ws + align16(stage_pad(CAP) * 8) + align16(stage_pad(CAP) * 4));
    double2* cd = reinterpret_cast<double2*>(ws + align16(stage_pad(CAP) * 8) + align16(stage_pad(CAP) * 4) +
                                             align16(stage_pad(CAP) * sizeof(T)));
    // exact: windows of B rows with halos on both sides, one per lane;
    // fast: lanes of FAST_B rows, the last H lanes of a pass as right halo
    const int H = (C.S + FAST_B - 1) / FAST_B;
    const int nlmax = min(32, (WSCAP_FAST - C.S - 3) / FAST_B);
    const int per = min(32, (WSCAP - 2 * C.S - 8) / Bw);  // exact windows per pass
    for (int g = wa; g < wb;) {
        const int env = (g < nw0) ? 0 : 1;
        const int w0 = env ? g - nw0 : g;  // first window of the pass (within its envelope)
        const int nwe = env ? nw1 : nw0;
        const int n = env ? n1 : n0;
        const int p2 = S.p2[env];
        int ncommit, nl, rlo, rhi;
        if (EXACT) {
            ncommit = nl = min(w0 + per, min(nwe, w0 + (wb - g))) - w0;
            rlo = max(0, w0 * Bw - C.S);
            rhi = min(n - 1, min(n, (w0 + nl) * Bw) - 1 + C.S);
        } else {
            const int rem = min(wb - g, nwe - w0);  // this warp's windows left in the envelope
            if (w0 + rem == nwe && rem <= nlmax) {
                ncommit = nl = rem;  // the pass reaches the envelope's last row
            } else {
                ncommit = min(rem, nlmax - H);
                nl = min(nlmax, min(ncommit + H, nwe - w0));
            }
            rlo = max(0, w0 * FAST_B - C.S);
            rhi = min(n - 1, (w0 + nl) * FAST_B - 1);
        }
        const int kcount = rhi + 3 - rlo;  // knots rlo .. rhi+2
        stage_range<T, EXACT>(C, sl, S, env, rlo, kcount, skt, sky, lane);
        cp_async_commit();
        cp_async_wait<0>();
        __syncwarp();
        SUB(0);
        for (int k = lane; k + 1 < kcount; k += 32) {
            const int ta = skt[stage_slot<EXACT>(k)], tb = skt[stage_slot<EXACT>(k + 1)];
            const double ya = (double)sky[stage_slot<EXACT>(k)], yb = (double)sky[stage_slot<EXACT>(k + 1)];
            // emd_ref.py:47: (y_{q+1}-y_q)/H_q (the same IEEE division in exact mode)
            ssl[stage_slot<EXACT>(k)] = EXACT ? (yb - ya) / (double)(tb - ta) : (yb - ya) * fast_rcp((double)(tb - ta));
        }
        __syncwarp();
        SUB(1);
        Rec<T> R;
        R.rc = static_cast<T*>(sl.M) + (int64_t)env * C.kcap * Geo<T>::RS;
        const int w = w0 + lane;
        if (EXACT) {
            if (lane < nl) window_exact<T>(C, skt, sky, ssl, rlo, n, w, R, p2);
        } else {
            if (lane < nl) window_fast_fwd<T>(skt, ssl, rlo, n, w, C.S, cd, w0 * FAST_B);
            __syncwarp();
            if (lane < ncommit) window_fast_back<T>(skt, sky, ssl, rlo, n, w, C.S, cd, w0 * FAST_B, R);
        }
        __syncwarp();
        SUB(2);
        g += ncommit;
    }
    __syncthreads();
#ifdef EEMD_TRACE
    if (lane == 0) {
        for (int k = 0; k < 3; ++k) atomicAdd(&C.hdr->sweep_cycles[4 + k], scyc[k]);
    }
#endif
#undef SUB
}

// ---------------------------------------------------------------------------
// sweep: the fused per-segment pass
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ double trial_input(const Ctx& C, const TaskDesc& d, int64_t t) {
    const double xv = ldv<T>(C.x, d.x_off + t);
    switch (C.noise_mode) {
        case EEMD_NOISE_INJECTED: return rnd<T>(xv + ldv<T>(C.noise, d.noise_off + t));
        case EEMD_NOISE_SCALED:
            // the product, then the sum, each rounded (the reference forms beta * w, then x + that)
            return rnd<T>(__dadd_rn(xv, __dmul_rn(C.noise_scale, ldv<T>(C.noise, d.noise_off + t))));
        case EEMD_NOISE_PHILOX:
            return rnd<T>(xv + C.sigma[d.signal] * philox_normal(C.seed, d.signal, d.trial, t));
        default: return xv;  // NONE, PREPERTURBED
    }
}

// One interval of an envelope (fast: monomial; exact: the two end knots).
template <typename T>
struct Iv {
    int k, t0, t1;
    T y0, c1, c2, c3, y1, m1;  // fast: y0 + s(c1 + s(c2 + s c3)); exact: y0, M0 = c1, y1, M1
};

// loads interval record k (and k+1 in exact mode) of an envelope's record array
template <typename T, bool EXACT>
__device__ __forceinline__ void load_iv(Iv<T>& v, const T* R, int k) {
    constexpr int RS = Geo<T>::RS;
    v.k = k;
    const T* p = R + (int64_t)k * RS;
    if constexpr (sizeof(T) == 4) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v.t0 = __float_as_int(a.x);
        v.y0 = a.y;
        v.c1 = a.z;
        v.c2 = a.w;
        v.c3 = p[4];
        if (EXACT) {
            const float4 c = *reinterpret_cast<const float4*>(p + RS);
            v.t1 = __float_as_int(c.x);
            v.y1 = c.y;
            v.m1 = c.z;
        }
    } else {
        const double2 a = *reinterpret_cast<const double2*>(p);
        const double2 b = *reinterpret_cast<const double2*>(p + 2);
        v.t0 = (int)__double_as_longlong(a.x);
        v.y0 = a.y;
        v.c1 = b.x;
        v.c2 = b.y;
        v.c3 = p[4];
        if (EXACT) {
            const double2 c = *reinterpret_cast<const double2*>(p + RS);
            const double2 e = *reinterpret_cast<const double2*>(p + RS + 2);
            v.t1 = (int)__double_as_longlong(c.x);
            v.y1 = c.y;
            v.m1 = e.x;
        }
    }
}

template <typename T, bool EXACT>
__device__ __forceinline__ T iv_eval(const Iv<T>& v, int t) {
    if (EXACT)
        return (T)spline_exact((double)t, (double)v.t0, (double)v.t1, (double)v.y0, (double)v.y1, (double)v.c1,
                               (double)v.m1);
    const T s = (T)(t - v.t0);
    return fmat(s, fmat(s, fmat(s, v.c3, v.c2), v.c1), v.y0);
}

__device__ __forceinline__ int mirror_adj(const TaskSm& S, int env, int t) {
    return S.mir[env] ? (S.tfirst[env] < t ? 1 : 0) + (S.tlast[env] < t ? 1 : 0) : 0;
}

// envelope value at t with `cless` real knots strictly before t: mirror-space
// interval = searchsorted - 1 clipped (emd_ref.py:70); reloads the interval
// record only when the interval changes
template <typename T, bool EXACT>
__device__ __forceinline__ T env_at(const Ctx& C, const TaskSm& S, Iv<T>& v, const T* R, int env, int cless, int t) {
    if (S.P[env] < 2) return (T)S.cval[env];
    const int idx2 = max(0, min(cless + mirror_adj(S, env, t) - 1, S.p2[env] - 2));
    if (idx2 != v.k) load_iv<T, EXACT>(v, R, idx2);
    return iv_eval<T, EXACT>(v, t);
}

// element phase of an address within its 16-byte block
template <typename T>
__device__ __forceinline__ int phase16(const T* p) {
    return (int)((reinterpret_cast<uintptr_t>(p) / sizeof(T)) & (16 / sizeof(T) - 1));
}

// One warp copies g[0 .. cnt) to the 16-byte aligned shared dst[0 .. cnt):
// 16-byte copies when g is 16-byte aligned too, element copies otherwise.
template <typename T>
__device__ __forceinline__ void tile_copy(T* dst, const T* g, int cnt, int lane) {
    constexpr int VEC = 16 / (int)sizeof(T);
    if (phase16(g) == 0) {
        const int nvec = cnt / VEC;
        for (int v = lane; v < nvec; v += 32) cp_async16(dst + v * VEC, g + v * VEC);
        for (int j = nvec * VEC + lane; j < cnt; j += 32) cp_async_el<T>(dst + j, g + j);
    } else {
        for (int j = lane; j < cnt; j += 32) cp_async_el<T>(dst + j, g + j);
    }
}

// a lane's run of RUN samples from a 16-byte aligned shared tile position
template <typename T, int RUN>
__device__ __forceinline__ void load_run(const T* p, T (&v)[RUN]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < RUN; i += 4) {
            const float4 a = *reinterpret_cast<const float4*>(p + i);
            v[i] = a.x;
            v[i + 1] = a.y;
            v[i + 2] = a.z;
            v[i + 3] = a.w;
        }
    } else {
#pragma unroll
        for (int i = 0; i < RUN; i += 2) {
            const double2 a = *reinterpret_cast<const double2*>(p + i);
            v[i] = a.x;
            v[i + 1] = a.y;
        }
    }
}

// stores a thread's run of samples: 16-byte vectors when the run is full and
// aligned, element stores otherwise
template <typename T, int RUN>
__device__ __forceinline__ void store_run(T* p, const T (&v)[RUN], int nv) {
    if (nv == RUN && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        if constexpr (sizeof(T) == 4) {
#pragma unroll
            for (int i = 0; i < RUN; i += 4)
                *reinterpret_cast<float4*>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        } else {
#pragma unroll
            for (int i = 0; i < RUN; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(v[i], v[i + 1]);
        }
        return;
    }
#pragma unroll
    for (int i = 0; i < RUN; ++i)
        if (i < nv) p[i] = v[i];
}

// a lane's run of RUN values into a 16-byte aligned shared position
template <typename T, int RUN>
__device__ __forceinline__ void store_run_smem(T* p, const T (&v)[RUN]) {
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int i = 0; i < RUN; i += 4)
            *reinterpret_cast<float4*>(p + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    } else {
#pragma unroll
        for (int i = 0; i < RUN; i += 2) *reinterpret_cast<double2*>(p + i) = make_double2(v[i], v[i + 1]);
    }
}

// value at tile position pos (lane pos/RUN, element pos%RUN), to every lane
template <typename T, int RUN>
__device__ __forceinline__ T tile_at(const T (&v)[RUN], int pos) {
    const int e = pos % RUN;
    T x = v[0];
#pragma unroll
    for (int i = 1; i < RUN; ++i)
        if (e == i) x = v[i];
    return __shfl_sync(0xffffffffu, x, pos / RUN);
}

// Pointers and flags of one sweep step.
template <typename T>
struct StepIo {
    const T* hsrc;   // h read by the step (sifting, TRANS from a sift)
    const T* rcur;   // current residual
    T* rnxt;         // residual written by LAST / TRANS / INIT
    T* hdst;         // h written by SIFT
    T* imf_m;        // the IMF slot (written by LAST, and by TRANS when the IMF is elsewhere)
    bool trans_imf;  // TRANS copies the IMF into its slot
};

// new value f and next-knot value g of sample t from h / r (not the envelopes)
template <typename T, int MODE>
__device__ __forceinline__ void plain_value(const Ctx& C, const TaskSm& S, const TaskDesc& d, int t, T h, T r,
                                            T& f, T& g) {
    if (MODE == TM_TRANS) {
        f = r - (S.imf_from_resid ? r : h);
        g = f;
    } else {  // TM_INIT
        f = (T)trial_input<T>(C, d, t);
        g = f;
    }
}

// next-knot value of a sample outside the warp range (t = range start - 1 or
// range end), evaluated by one lane from global memory
template <typename T, bool EXACT, int MODE>
__device__ T outside_g(const Ctx& C, const TaskSm& S, const TaskDesc& d, const StepIo<T>& io, const T* R0,
                       const T* R1, int t, int cl0, int cl1) {
    constexpr bool SIFTING = (MODE == TM_SIFT || MODE == TM_LAST);
    const T h = (SIFTING || (MODE == TM_TRANS && !S.imf_from_resid)) ? __ldcg(io.hsrc + t) : (T)0;
    const T r = (MODE == TM_LAST || MODE == TM_TRANS) ? __ldcg(io.rcur + t) : (T)0;
    if (SIFTING) {
        Iv<T> v0, v1;
        v0.k = v1.k = -1;
        const T eu = env_at<T, EXACT>(C, S, v0, R0, 0, cl0, t);
        const T el = env_at<T, EXACT>(C, S, v1, R1, 1, cl1, t);
        const T fn = h - (T)0.5 * (eu + el);
        return (MODE == TM_LAST) ? r - fn : fn;
    }
    T f, g;
    plain_value<T, MODE>(C, S, d, t, h, r, f, g);
    return g;
}

// The sweep.  The CTA's segment [s0, s1) is cut into warp tiles of WT = 32*RUN
// samples and warp w owns the contiguous tiles [w*NT/8, (w+1)*NT/8); lane u
// of a tile owns the run of RUN samples at u*RUN.  Each warp works through
// its range without block-wide barriers and keeps its own knot lists (one
// knot segment per warp, so no cross-warp prefix is needed).  Per tile:
//   - the tile's samples of each stream it reads and its run records from
//     the previous step (per run: position of the run's first current knot
//     of each kind in the warp's knot lists, and the run's knot masks) are
//     already in shared memory: cp.async, issued during the previous tile;
//   - each lane knows the interval of every sample from its run record, and
//     loads an interval record (32 or 48 bytes) only when the interval
//     changes; interior tiles take a path without end handling;
//   - new values and SD partials; strict extrema of the new values with lane
//     neighbours by shuffle; the tile's last sample is decided with the next
//     tile (its right neighbour), so only the two samples just outside the
//     warp's range are ever evaluated twice;
//   - a warp-shuffle scan places the knots in the warp's lists, and the
//     samples, knots and this step's run records are written.
// Every step reads one set of buffers and writes another (ping-pong), so the
// warps of a step never see each other's writes.
template <typename T, bool EXACT, int MODE, int NW>
__device__ void sweep(const Ctx& C, const Slot& sl, TaskSm& S, Xchg* X, unsigned char* smem) {
    using G = Geo<T>;
    constexpr int RUN = G::RUN, WT = G::WT, RS = G::RS;
    constexpr unsigned FULL = 0xffffffffu;
    constexpr bool SIFTING = (MODE == TM_SIFT || MODE == TM_LAST);
    constexpr bool USES_R = (MODE == TM_LAST || MODE == TM_TRANS);
    __shared__ double2 s_red[NW];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int n = S.n, s0 = S.s0, s1 = S.s1, rank = S.rank;
    const bool needs_h = SIFTING || (MODE == TM_TRANS && !S.imf_from_resid);
    const int q = S.step & 1;
    const TaskDesc d = C.td[S.task];
    StepIo<T> io;
    {
        T* const r0 = static_cast<T*>(C.resid) + d.s_off;
        T* const r1 = static_cast<T*>(sl.r1);
        T* const w1 = static_cast<T*>(sl.w1);
        io.imf_m = static_cast<T*>(C.imfs) + d.imf_off + (int64_t)min(S.imf, C.max_imf - 1) * n;
        io.rcur = S.rcur ? r1 : r0;
        io.rnxt = S.rcur ? r0 : r1;
        // h buffers W0 = the IMF slot, W1 = slot scratch: sift k writes W[(max_sifts-1-k) & 1], so
        // the last sift writes the IMF slot; sift k > 0 reads what sift k-1 wrote
        const int wd = (C.max_sifts - 1 - S.sift) & 1;
        io.hdst = wd ? w1 : io.imf_m;
        io.hsrc = io.rcur;
        if (SIFTING && !S.src_resid) io.hsrc = wd ? io.imf_m : w1;
        if (MODE == TM_TRANS && !S.imf_from_resid) io.hsrc = io.hdst;  // the sift that stopped wrote it
        io.trans_imf = (MODE == TM_TRANS) && (S.imf_from_resid || wd == 1);
    }
    const int4* ri_cur = sl.ri + (int64_t)S.kpar * C.slot_runs;
    int4* ri_nxt = sl.ri + (int64_t)(S.kpar ^ 1) * C.slot_runs;
    const int np = S.kpar ^ 1;
    const int seg = rank * NW + wid;
    const int64_t pmx = knot_index(C, np, 0, seg, 0);
    const int64_t pmn = knot_index(C, np, 1, seg, 0);
    const T* R0 = static_cast<const T*>(sl.M);
    const T* R1 = R0 + (int64_t)C.kcap * RS;
    const int kbase0 = S.pref[S.kpar][0][seg], kbase1 = S.pref[S.kpar][1][seg];
    // the warp's range [r0, r1): an equal share of the segment in whole runs
    // (shares in whole tiles left the last tiles' warps up to a tile behind),
    // cut into tiles of WT samples from r0 (the last one partial)
    const int nrun = (s1 - s0 + RUN - 1) / RUN;
    const int r0 = min(s1, s0 + (int)((int64_t)wid * nrun / NW) * RUN);
    const int r1 = min(s1, s0 + (int)((int64_t)(wid + 1) * nrun / NW) * RUN);
    const int ta = 0, tb = (r1 - r0 + WT - 1) / WT;

    unsigned char* wb = smem + (size_t)wid * G::WARP_BYTES;
    T* const tbuf = reinterpret_cast<T*>(wb);                      // [2 buf][2 stream][TB]
    int4* const rib = reinterpret_cast<int4*>(wb + G::TB_BYTES);  // [2 buf][32]
    // the tile's new knots, compacted in time order before one coalesced copy out
    int* const kts = reinterpret_cast<int*>(wb + G::TB_BYTES + G::RI_BYTES);  // [kind][KCAP]
    T* const kvs = reinterpret_cast<T*>(wb + G::TB_BYTES + G::RI_BYTES + 2 * G::KCAP * 4);
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

    // tile j's samples [t0, t1) and run records into buffer b
    // tile j's samples and run records live in ring buffer (j - ta) mod NBUF;
    // NBUF - 1 tiles are in flight while one is processed
    auto bufi = [&](int j) { return (j - ta) % G::NBUF; };
    auto prefetch = [&](int j) {
        const int t0 = r0 + j * WT, t1 = min(r1, t0 + WT), bi = bufi(j);
        if (needs_h) tile_copy<T>(tbuf + (bi * 2) * G::TB, io.hsrc + t0, t1 - t0, lane);
        if (USES_R) tile_copy<T>(tbuf + (bi * 2 + 1) * G::TB, io.rcur + t0, t1 - t0, lane);
        if (SIFTING && lane * RUN < t1 - t0) cp_async16(rib + bi * 32 + lane, ri_cur + t0 / RUN + lane);
        cp_async_commit();
    };

    int wcx = 0, wcy = 0;  // knots of each kind written to the warp's lists so far
    T gm1 = (T)0, gm2 = (T)0;  // next-knot values at t0-1 and t0-2 of the current tile
    int cpx = 0, cpn = 0, cmask = 0, crun = 0, cbit = 0;  // run record awaiting its last sample
    if (ta < tb) {
        for (int q = 0; q < G::NBUF - 1 && ta + q < tb; ++q) prefetch(ta + q);
        if (r0 > 0) {
            // the sample before the range: its value is the left neighbour of the range's first sample
            int c0 = 0, c1 = 0;
            if (SIFTING && lane == 0) {
                const unsigned pm = (unsigned)__ldcg(&ri_cur[r0 / RUN - 1].z);
                c0 = kbase0 - (int)((pm >> (RUN - 1)) & 1u);
                c1 = kbase1 - (int)((pm >> (16 + RUN - 1)) & 1u);
            }
            if (lane == 0) gm1 = outside_g<T, EXACT, MODE>(C, S, d, io, R0, R1, r0 - 1, c0, c1);
            gm1 = __shfl_sync(FULL, gm1, 0);
        }
    }

    for (int j = ta; j < tb; ++j) {
        const int t0 = r0 + j * WT, t1 = min(r1, t0 + WT), tl = t1 - t0;
        const int j0 = lane * RUN;
        const int nv = max(0, min(RUN, tl - j0));  // valid samples of this lane's run
        const int last_lane = (tl - 1) / RUN;
        const int b = bufi(j);
        // tile j's copies are complete when at most the later tiles' groups
        // (up to NBUF - 2 of them) are still pending
        const int later = min(G::NBUF - 2, tb - 1 - j);
        if (later >= 2) cp_async_wait<2>();
        else if (later == 1) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncwarp();
        if (j + G::NBUF - 1 < tb) prefetch(j + G::NBUF - 1);
        SUB(0);
        const T* hb = tbuf + (b * 2) * G::TB;
        const T* rb = tbuf + (b * 2 + 1) * G::TB;
        // (samples past the run's end are read but never used)
        T hv[RUN], rv[RUN], fv[RUN], gv[RUN];
#pragma unroll
        for (int i = 0; i < RUN; ++i) hv[i] = rv[i] = fv[i] = gv[i] = (T)0;
        if (nv > 0) {
            if (needs_h) load_run<T, RUN>(hb + j0, hv);
            if (USES_R) load_run<T, RUN>(rb + j0, rv);
        }

        // ---------------- new values ----------------
        if (SIFTING) {
            unsigned kmx = 0u, kmn = 0u;
            int kb0 = 0, kb1 = 0;
            if (nv > 0) {
                const int4 ri = rib[b * 32 + lane];
                kmx = (unsigned)ri.z & 0xffffu;
                kmn = (unsigned)ri.z >> 16;
                kb0 = kbase0 + ri.x;
                kb1 = kbase1 + ri.y;
            }
            // interior tile: every sample's interval is (knots before it) + mir - 1, no clipping
            const int ta0 = t0 + j0, ta1 = t0 + j0 + nv - 1;
            bool ok = S.P[0] >= 2 && S.P[1] >= 2;
#pragma unroll
            for (int env = 0; env < 2; ++env) {
                const int kb = env ? kb1 : kb0;
                const int kc = __popc(env ? kmn : kmx);
                const int mir = S.mir[env];
                ok = ok && (!mir || (S.tfirst[env] < ta0 && S.tlast[env] >= ta1));
                ok = ok && (kb + mir >= 1) && (kb + kc + mir <= S.p2[env] - 1);
            }
            const bool fast = __all_sync(FULL, ok || nv == 0);
            T tnum = (T)0, tden = (T)0;  // fast mode: this tile's SD partial sums
            // sample i of the run from its envelope mean m: new h, SD terms, next-knot value
            auto finish = [&](int i, T m) {
                const T h = hv[i];
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
                gv[i] = (MODE == TM_LAST) ? rv[i] - hn : hn;
            };
            if (fast) {
                // current and next interval of each envelope; the next record is
                // loaded as soon as the current one is entered
                Iv<T> c0, n0, c1, n1;
                c0.t0 = c0.t1 = 0;
                c0.y0 = c0.c1 = c0.c2 = c0.c3 = c0.y1 = c0.m1 = (T)0;
                n0 = c1 = n1 = c0;
                int k0 = kb0 + S.mir[0] - 1, k1 = kb1 + S.mir[1] - 1;
                if (nv > 0) {
                    // the interior test above keeps every index of the run in [0, p2 - 2]
                    EEMD_CHECK_IV(k0, S.p2[0] - 2 - (int)__popc(kmx));
                    EEMD_CHECK_IV(k1, S.p2[1] - 2 - (int)__popc(kmn));
                    load_iv<T, EXACT>(c0, R0, k0);
                    load_iv<T, EXACT>(c1, R1, k1);
                    if (kmx) load_iv<T, EXACT>(n0, R0, k0 + 1);
                    if (kmn) load_iv<T, EXACT>(n1, R1, k1 + 1);
                }
#pragma unroll
                for (int i = 0; i < RUN; ++i) {
                    if (i > 0 && ((kmx >> (i - 1)) & 1u)) {
                        c0 = n0;
                        ++k0;
                        if (kmx >> i) load_iv<T, EXACT>(n0, R0, k0 + 1);
                    }
                    if (i > 0 && ((kmn >> (i - 1)) & 1u)) {
                        c1 = n1;
                        ++k1;
                        if (kmn >> i) load_iv<T, EXACT>(n1, R1, k1 + 1);
                    }
                    const int t = t0 + j0 + i;
                    if (i < nv) finish(i, (T)0.5 * (iv_eval<T, EXACT>(c0, t) + iv_eval<T, EXACT>(c1, t)));
                }
            } else {
                Iv<T> v0, v1;
                v0.k = v1.k = -1;
                int cl0 = kb0, cl1 = kb1;
#pragma unroll
                for (int i = 0; i < RUN; ++i) {
                    const int t = t0 + j0 + i;
                    if (i < nv) {
                        const T eu = env_at<T, EXACT>(C, S, v0, R0, 0, cl0, t);
                        const T el = env_at<T, EXACT>(C, S, v1, R1, 1, cl1, t);
                        finish(i, (T)0.5 * (eu + el));
                    }
                    cl0 += (kmx >> i) & 1u;
                    cl1 += (kmn >> i) & 1u;
                }
            }
            if (!EXACT) {
                num += (double)tnum;
                den += (double)tden;
            }
        } else {
#pragma unroll
            for (int i = 0; i < RUN; ++i)
                if (i < nv) plain_value<T, MODE>(C, S, d, t0 + j0 + i, hv[i], rv[i], fv[i], gv[i]);
        }
        SUB(1);

        // ---------------- strict extrema of the new values ----------------
        // lanes decide their own samples except the tile's last one (its right
        // neighbour is the next tile's first sample); lane 0 decides the
        // previous tile's last sample
        const T up = __shfl_up_sync(FULL, gv[RUN - 1], 1);
        const T dn = __shfl_down_sync(FULL, gv[0], 1);
        const T gprev = (lane == 0) ? gm1 : up;
        // samples of the run that may be knots: inside the run, not the tile's
        // last sample, and 1 <= t <= n-2
        unsigned valid = (1u << nv) - 1u;
        if (j0 + nv == tl && nv > 0) valid &= ~(1u << (nv - 1));
        if (t0 + j0 == 0) valid &= ~1u;
        {
            const int lim = n - 2 - (t0 + j0);  // largest run index with t <= n-2
            if (lim < RUN - 1) valid &= (lim < 0) ? 0u : ((2u << lim) - 1u);
        }
        unsigned nmx = 0u, nmn = 0u;
#pragma unroll
        for (int i = 0; i < RUN; ++i) {
            const T a = (i == 0) ? gprev : gv[(i + RUN - 1) % RUN];
            const T c = (i + 1 < RUN) ? gv[(i + 1) % RUN] : dn;
            const T v = gv[i];
            nmx |= (unsigned)((v > a) & (v > c)) << i;
            nmn |= (unsigned)((v < a) & (v < c)) << i;
        }
        nmx &= valid;
        nmn &= valid;
        unsigned dmx = 0u, dmn = 0u;  // the previous tile's last sample (lane 0)
        if (lane == 0 && j > ta && t0 - 1 >= 1 && t0 - 1 <= n - 2) {
            dmx = (gm1 > gm2 && gm1 > gv[0]) ? 1u : 0u;
            dmn = (gm1 < gm2 && gm1 < gv[0]) ? 1u : 0u;
        }
        const int cnt = (int)(__popc(nmx) + dmx) | ((int)(__popc(nmn) + dmn) << 16);
        int inc = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int x = __shfl_up_sync(FULL, inc, o);
            if (lane >= o) inc += x;
        }
        const int tot = __shfl_sync(FULL, inc, 31);
        const int exc = inc - cnt;
        SUB(2);

        // ---------------- writes ----------------
        // knots go to shared memory at their tile position, then to the warp's
        // lists with one coalesced copy per kind
        int px = exc & 0xffff, pn = exc >> 16;  // tile positions
        if (lane == 0 && j > ta) {
            // the previous tile's last sample and the run record that waited for it
            if (dmx) {
                kts[px] = t0 - 1;
                kvs[px] = gm1;
            }
            if (dmn) {
                kts[G::KCAP + pn] = t0 - 1;
                kvs[G::KCAP + pn] = gm1;
            }
            ri_nxt[crun] = make_int4(cpx, cpn, cmask | (int)(dmx << cbit) | (int)(dmn << (16 + cbit)), 0);
            px += (int)dmx;
            pn += (int)dmn;
        }
        const int rpx = wcx + px, rpn = wcy + pn, rmask = (int)(nmx | (nmn << 16));
        if (nv > 0 && lane != last_lane) ri_nxt[t0 / RUN + lane] = make_int4(rpx, rpn, rmask, 0);
        {
            // the run's new values go to the (already consumed) h tile buffer, so a
            // knot's value is read by index; only the set bits are visited
            T* const gsm = tbuf + (b * 2) * G::TB + j0;
            store_run_smem<T, RUN>(gsm, gv);
            for (unsigned m = nmx; m; m &= m - 1u) {
                const int i = __ffs(m) - 1;
                kts[px] = t0 + j0 + i;
                kvs[px] = gsm[i];
                ++px;
            }
            for (unsigned m = nmn; m; m &= m - 1u) {
                const int i = __ffs(m) - 1;
                kts[G::KCAP + pn] = t0 + j0 + i;
                kvs[G::KCAP + pn] = gsm[i];
                ++pn;
            }
        }
        __syncwarp();
        {
            const int nx = tot & 0xffff, nn = tot >> 16;
            if (wcx + nx > C.segcap || wcy + nn > C.segcap || nx > G::KCAP || nn > G::KCAP) {
                if (lane == 0) task_error(C, S, EEMD_E_KNOT_OVERFLOW);
            } else {
                T* const ky = static_cast<T*>(sl.ky);
                for (int k = lane; k < nx; k += 32) {
                    sl.kt[pmx + wcx + k] = kts[k];
                    ky[pmx + wcx + k] = kvs[k];
                }
                for (int k = lane; k < nn; k += 32) {
                    sl.kt[pmn + wcy + k] = kts[G::KCAP + k];
                    ky[pmn + wcy + k] = kvs[G::KCAP + k];
                }
            }
        }
        const int tj = t0 + j0;
        if (MODE == TM_SIFT) {
            store_run<T, RUN>(io.hdst + tj, fv, nv);
        } else if (MODE == TM_LAST) {
            store_run<T, RUN>(io.imf_m + tj, fv, nv);
            store_run<T, RUN>(io.rnxt + tj, gv, nv);
        } else if (MODE == TM_TRANS) {
            store_run<T, RUN>(io.rnxt + tj, fv, nv);
            if (io.trans_imf) {
                if (S.imf_from_resid) store_run<T, RUN>(io.imf_m + tj, rv, nv);
                else store_run<T, RUN>(io.imf_m + tj, hv, nv);
            }
        } else {
            store_run<T, RUN>(io.rnxt + tj, fv, nv);
        }
        // carry to the next tile: the last sample's neighbours and its run record
        cpx = __shfl_sync(FULL, rpx, last_lane);
        cpn = __shfl_sync(FULL, rpn, last_lane);
        cmask = __shfl_sync(FULL, rmask, last_lane);
        crun = t0 / RUN + last_lane;
        cbit = tl - 1 - last_lane * RUN;
        gm2 = (tl >= 2) ? tile_at<T, RUN>(gv, tl - 2) : gm1;
        gm1 = tile_at<T, RUN>(gv, tl - 1);
        wcx += tot & 0xffff;
        wcy += tot >> 16;
        SUB(3);
    }
    if (ta < tb) {
        // the range's last sample r1-1: its right neighbour lies outside the range
        unsigned dmx = 0u, dmn = 0u;
        if (lane == 0 && r1 < n && r1 - 1 >= 1) {
            const T gr = outside_g<T, EXACT, MODE>(C, S, d, io, R0, R1, r1, S.pref[S.kpar][0][seg + 1],
                                                  S.pref[S.kpar][1][seg + 1]);
            dmx = (gm1 > gm2 && gm1 > gr) ? 1u : 0u;
            dmn = (gm1 < gm2 && gm1 < gr) ? 1u : 0u;
        }
        if (lane == 0) {
            if (dmx) {
                if (wcx < C.segcap) {
                    sl.kt[pmx + wcx] = r1 - 1;
                    static_cast<T*>(sl.ky)[pmx + wcx] = gm1;
                } else {
                    task_error(C, S, EEMD_E_KNOT_OVERFLOW);
                }
            }
            if (dmn) {
                if (wcy < C.segcap) {
                    sl.kt[pmn + wcy] = r1 - 1;
                    static_cast<T*>(sl.ky)[pmn + wcy] = gm1;
                } else {
                    task_error(C, S, EEMD_E_KNOT_OVERFLOW);
                }
            }
            ri_nxt[crun] = make_int4(cpx, cpn, cmask | (int)(dmx << cbit) | (int)(dmn << (16 + cbit)), 0);
        }
        wcx += (int)__shfl_sync(FULL, dmx, 0);
        wcy += (int)__shfl_sync(FULL, dmn, 0);
    }
    if (lane == 0) {
        X[q].cnt[0][wid] = wcx;
        X[q].cnt[1][wid] = wcy;
    }
#ifdef EEMD_TRACE
    if (lane == 0) {
        for (int k = 0; k < 4; ++k) atomicAdd(&C.hdr->sweep_cycles[k], scyc[k]);
    }
#endif
#undef SUB
    // ---------------- publish the segment's SD partials ----------------
    const double2 rs = block_sum2<32 * NW>(make_double2(num, den), s_red);
    if (tid == 0) {
        X[q].num = rs.x;
        X[q].den = rs.y;
        X[q].err = S.err;
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

// adopt the knots the last sweep produced (their segment prefixes are in pref[kpar ^ 1])
__device__ __forceinline__ void adopt(TaskSm& S, int cmax, int cmin) {
    S.kpar ^= 1;
    S.P[0] = cmax;
    S.P[1] = cmin;
}

__device__ __forceinline__ void imf_level(const Ctx& C, TaskSm& S, int cmax, int cmin) {
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
    adopt(S, cmax, cmin);
}

// Warp 0 gathers the knot counts of every (CTA, warp) segment through
// distributed shared memory and writes their prefixes for the new lists;
// thread 0 then takes the step decision, identical in every CTA.
template <int NW>
__device__ void decide(const Ctx& C, TaskSm& S, Xchg* X, cg::cluster_group& cl) {
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const int q = S.step & 1;
        const int nseg = S.csize * NW;
        // segments SPL*lane .. SPL*lane + SPL-1 per lane (SPL = 3 covers the
        // 16 x 5 = 80 segments of the largest cluster of 5-warp CTAs)
        constexpr int SPL = (MAXSEG + 31) / 32;
        static_assert(SPL * 32 >= MAXSEG, "segments per lane");
        int c[2][SPL];  // [env][segment SPL*lane + k]
#pragma unroll
        for (int k = 0; k < SPL; ++k) {
            const int sg = SPL * lane + k;
            c[0][k] = c[1][k] = 0;
            if (sg < nseg) {
                const Xchg* xr = cl.map_shared_rank(&X[q], sg / NW);
                c[0][k] = xr->cnt[0][sg % NW];
                c[1][k] = xr->cnt[1][sg % NW];
            }
        }
        int tot[2];
#pragma unroll
        for (int env = 0; env < 2; ++env) {
            int v = 0;
#pragma unroll
            for (int k = 0; k < SPL; ++k) v += c[env][k];
            int inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int x = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += x;
            }
            tot[env] = __shfl_sync(0xffffffffu, inc, 31);
            int* pr = S.pref[S.kpar ^ 1][env];
            int e = inc - v;
#pragma unroll
            for (int k = 0; k < SPL; ++k) {
                if (SPL * lane + k < nseg) pr[SPL * lane + k] = e;
                e += c[env][k];
            }
            if (lane == 0) pr[nseg] = tot[env];
        }
        if (lane == 0) {
            double num = 0.0, den = 0.0;
            int err = 0;
            for (int r = 0; r < S.csize; ++r) {
                const Xchg* xr = cl.map_shared_rank(&X[q], r);
                num += xr->num;
                den += xr->den;
                err |= xr->err;
            }
            const int cmax = tot[0], cmin = tot[1];
            const int mode = S.mode;
            if (err) {
                // an error of this task (recorded in the header): stop it here
                S.phase = PH_DONE;
                S.flags |= 2;
            } else if (mode == TM_SIFT) {
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
                    adopt(S, cmax, cmin);
                }
            } else if (mode == TM_LAST) {
                log_sift(C, S);
                S.mode_sifts_cur += 1;
                S.nsift_total += 1;
                S.rcur ^= 1;
                close_imf(C, S);
                imf_level(C, S, cmax, cmin);
            } else if (mode == TM_TRANS) {
                S.rcur ^= 1;
                close_imf(C, S);
                imf_level(C, S, cmax, cmin);
            } else {
                S.rcur ^= 1;
                S.imf = 0;
                S.nmode = 0;
                imf_level(C, S, cmax, cmin);
            }
            S.step += 1;
            // every IMF ends after at most max_sifts sifts plus one closing step
            if (S.phase != PH_DONE && S.step > 2 + C.max_imf * (C.max_sifts + 1)) {
                raise_error(C.hdr, EEMD_E_TIMEOUT, S.task);
                S.phase = PH_DONE;
            }
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
        if (S.p2[env] > C.kcap) {
            raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, S.task);
            S.setup_fail = 1;  // computed from the same counts in every CTA of the cluster
        }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// k_emd: the persistent cluster kernel
// ---------------------------------------------------------------------------
template <typename T, bool EXACT, int NW>
__global__ void __launch_bounds__(32 * NW, ctas_per_sm(NW, (int)sizeof(T))) k_emd(const __grid_constant__ Ctx C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ TaskSm S;
    __shared__ Xchg X[2];
    __shared__ int s_claim;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    const int csize = (int)cl.num_blocks();
    const int slot = blockIdx.x / csize;
    const int tid = threadIdx.x;
    Slot sl;
    sl.kt = C.kt + (int64_t)slot * C.slot_knots;
    sl.ky = static_cast<T*>(C.ky) + (int64_t)slot * C.slot_knots;
    sl.M = static_cast<T*>(C.M) + (int64_t)slot * C.slot_M;
    sl.w1 = static_cast<T*>(C.w1) + (int64_t)slot * C.slot_n;
    sl.r1 = static_cast<T*>(C.r1) + (int64_t)slot * C.slot_n;
    sl.ri = C.ri + (int64_t)slot * 2 * C.slot_runs;

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
            for (int r = 0; r <= MAXSEG; ++r)
                S.pref[0][0][r] = S.pref[0][1][r] = S.pref[1][0][r] = S.pref[1][1][r] = 0;
            S.mir[0] = S.mir[1] = 0;
            S.rcur = 1;  // the first step writes the residual array
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
                S.err = 0;
                S.setup_fail = 0;
            }
            __syncthreads();
            if (S.mode == TM_SIFT || S.mode == TM_LAST) {
                step_setup<T>(C, sl, S);
                if (S.setup_fail) {
                    // every CTA of the cluster sees the same counts and leaves together
                    if (tid == 0) {
                        S.phase = PH_DONE;
                        S.flags |= 2;
                    }
                    __syncthreads();
                    break;
                }
                EEMD_PHASE(0);
                solve_task<T, EXACT, NW>(C, sl, S, smem_raw);
                EEMD_PHASE(1);
                cl.sync();  // second derivatives of every segment visible
                EEMD_PHASE(2);
            }
            switch (S.mode) {
                case TM_SIFT: sweep<T, EXACT, TM_SIFT, NW>(C, sl, S, X, smem_raw); break;
                case TM_LAST: sweep<T, EXACT, TM_LAST, NW>(C, sl, S, X, smem_raw); break;
                case TM_TRANS: sweep<T, EXACT, TM_TRANS, NW>(C, sl, S, X, smem_raw); break;
                default: sweep<T, EXACT, TM_INIT, NW>(C, sl, S, X, smem_raw); break;
            }
            EEMD_PHASE(3);
            cl.sync();  // segment results published
            EEMD_PHASE(4);
            decide<NW>(C, S, X, cl);
            EEMD_PHASE(5);
        }
        if (S.rcur) {
            // the final residual sits in the slot scratch: move this segment to the task's array
            const TaskDesc d = C.td[S.task];
            T* r0 = static_cast<T*>(C.resid) + d.s_off;
            const T* r1 = static_cast<const T*>(sl.r1);
            for (int t = S.s0 + tid; t < S.s1; t += 32 * NW) r0[t] = r1[t];
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

struct Layout {
    std::vector<TaskDesc> td;
    std::vector<SignalDesc> sd;
    std::vector<int32_t> order;
    int64_t NS = 0, NIMF = 0, slot_knots = 0, slot_M = 0, slot_n = 0, slot_runs = 0;
    int B = 0, S = 0, csize = 1, slots = 1, segcap = 0, kcap = 0, scr_rows = 0, nw = NW_DEFAULT;
    size_t o_hdr, o_td, o_order, o_tout, o_sd, o_sigma, o_resid, o_imfs, o_kt, o_ky, o_M, o_w1, o_r1, o_ri,
        o_scr;
    size_t total = 0;
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Clusters of c CTAs of the k_emd instance for (dtype, exact) that the
// current device can hold at once (0 if the query fails, e.g. no device).
// the k_emd instance of (storage type, exact, warps per CTA)
const void* emd_fn(int dtype, bool exact, int nw) {
    if (dtype == EEMD_F32) return nw == 5 ? (const void*)k_emd<float, false, 5> : (const void*)k_emd<float, false, 4>;
    if (exact) return (const void*)k_emd<double, true, 4>;
    return nw == 5 ? (const void*)k_emd<double, false, 5> : (const void*)k_emd<double, false, 4>;
}

int active_clusters(int dtype, bool exact, int c, int nw) {
    const void* fn = emd_fn(dtype, exact, nw);
    const size_t smem = smem_bytes(dtype == EEMD_F32 ? 4 : 8, exact, nw);
    int n = 0;
    bool ok = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) == cudaSuccess;
    if (ok && c > 8) ok = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
    if (ok) {
        cudaLaunchConfig_t cfg;
        memset(&cfg, 0, sizeof(cfg));
        cfg.gridDim = dim3((unsigned)c, 1, 1);
        cfg.blockDim = dim3((unsigned)(32 * nw), 1, 1);
        cfg.dynamicSmemBytes = smem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)c;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        ok = cudaOccupancyMaxActiveClusters(&n, fn, &cfg) == cudaSuccess;
    }
    if (!ok) {
        (void)cudaGetLastError();  // a failed query leaves no sticky state for the launch checks
        n = 0;
    }
    return n;
}

// The cluster spreads one task over several SMs when there are fewer tasks
// than CTA slots.
int autotune_csize(int64_t n_tasks, int64_t nmin, int dtype, bool exact, int nw) {
    // leave a fifth of the CTA slots free: clusters must fit inside a GPC,
    // and the last clusters to be placed would otherwise wait for a second
    // wave.  Signals of a million samples or more take every slot: each CTA
    // then sweeps long ranges, and measured on 64 trials of 2^22 samples 8
    // CTAs per signal (512 CTAs) run 10 % faster than 7.
    const int64_t slots = (int64_t)ASSUMED_SMS * ctas_per_sm(nw, dtype == EEMD_F64 ? 8 : 4);
    const int64_t budget = nmin >= (1 << 20) ? slots : slots * 4 / 5;
    int c = (int)std::max<int64_t>(1, std::min<int64_t>(8, budget / std::max<int64_t>(n_tasks, 1)));
    // more tasks than slots: pairs of CTAs halve each task's time and with it
    // the last round's idle tail (1024 tasks of 65536 samples: 94.6 ms at 2
    // against 97.0 at 1)
    if (c == 1 && nmin >= (1 << 16)) c = 2;
    // signals of a million samples or more with slots to spare at 8 CTAs per
    // task (64 tasks use 512 of 592): a larger, non-portable cluster when the
    // device holds every task's cluster at once (a task waiting for a second
    // wave would double the launch)
    if (c == 8 && nmin >= (1 << 20)) {
        for (int c2 = (int)std::min<int64_t>(MAXC, slots / std::max<int64_t>(n_tasks, 1)); c2 > 8; --c2) {
            if (active_clusters(dtype, exact, c2, nw) >= n_tasks) {
                c = c2;
                break;
            }
        }
    }
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
    if (p->noise_mode < EEMD_NOISE_NONE || p->noise_mode > EEMD_NOISE_SCALED) return EEMD_E_BADARG;
    // warp tile: 32 lanes x 8 float32 samples or x 4 float64 samples
    const int wt = (p->dtype == EEMD_F64) ? Geo<double>::WT : Geo<float>::WT;
    if (p->tile != 0 && p->tile != wt) return EEMD_E_BADARG;
    if (p->knots_per_block < 0 || p->knots_per_block > 4096 || p->halo < 0 || p->halo > 256)
        return EEMD_E_BADARG;
    if (p->cluster_size < 0 || p->cluster_size > MAXC) return EEMD_E_BADARG;
    if (p->cta_warps != 0 && p->cta_warps != 4 && p->cta_warps != 5) return EEMD_E_BADARG;
    if (p->exact && p->cta_warps == 5) return EEMD_E_NOTSUP;  // exact mode runs 4-warp CTAs
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
    L.nw = p->cta_warps ? p->cta_warps : NW_DEFAULT;
    L.csize = p->cluster_size ? p->cluster_size : autotune_csize(n_tasks, nmin, p->dtype, p->exact != 0, L.nw);
    // decay halo of the seam windows: the truncation error falls like
    // (2 - sqrt 3)^S; 16 rows put it far below float32 rounding
    L.S = p->halo ? p->halo : (p->exact ? 32 : (p->dtype == EEMD_F32 ? 16 : 24));
    L.B = p->knots_per_block ? p->knots_per_block : 16;
    // a solve pass stages its windows' knots plus the halos in the warp's area:
    // exact windows carry both halos; a fast pass needs room for at least one
    // committing lane besides its ceil(S / FAST_B) right-halo lanes
    if (p->exact && 2 * L.S + L.B + 8 > WSCAP) return EEMD_E_BADARG;
    if (!p->exact && (L.S > FAST_SMAX || (L.S + FAST_B - 1) / FAST_B + 1 > std::min(32, (WSCAP_FAST - L.S - 3) / FAST_B)))
        return EEMD_E_BADARG;
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
    const int run = (p->dtype == EEMD_F64) ? Geo<double>::RUN : Geo<float>::RUN;
    const int wt = 32 * run;
    // knots of one kind in one warp's range: at most half its samples (+ends)
    const int64_t tiles_per_warp = ((segmax + wt - 1) / wt + L.nw - 1) / L.nw;
    L.segcap = (int)(tiles_per_warp * wt / 2 + 2);
#ifdef EEMD_CHECKED
    // test hook of the checked build only: params.reserved > 0 shrinks the knot
    // lists' capacity so that the overflow path can be exercised
    if (p->reserved > 0 && p->reserved < L.segcap) L.segcap = p->reserved;
#endif
    L.kcap = (int)(nmax / 2 + 4);
    const int rs = (p->dtype == EEMD_F64) ? Geo<double>::RS : Geo<float>::RS;
    L.slot_n = (nmax + 3) / 4 * 4;
    L.slot_runs = (nmax + run - 1) / run + 1;
    L.slots = (int)std::max<int64_t>(
        1, std::min<int64_t>(n_tasks, (int64_t)ASSUMED_SMS * ctas_per_sm(L.nw, p->dtype == EEMD_F64 ? 8 : 4) /
                                     L.csize));
    L.slot_knots = (int64_t)2 * 2 * L.csize * L.nw * L.segcap;
    L.slot_M = (int64_t)2 * L.kcap * rs;
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
    L.o_w1 = take(bt * L.slot_n * L.slots);
    L.o_r1 = take(bt * L.slot_n * L.slots);
    L.o_ri = take(16 * 2 * L.slot_runs * L.slots);
    L.o_scr = take(sizeof(double2) * (size_t)L.scr_rows * L.slots * L.csize * 32 * L.nw);
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

template <typename T, bool EXACT, int NW>
int launch_emd(const Ctx& C, const Layout& L, cudaStream_t st, Tracer& tr) {
    const size_t smem = smem_bytes((int)sizeof(T), EXACT, NW);
    if (cudaFuncSetAttribute(k_emd<T, EXACT, NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return EEMD_E_CUDA;
    if (L.csize > 8 &&
        cudaFuncSetAttribute(k_emd<T, EXACT, NW>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
        return EEMD_E_CUDA;
    cudaLaunchConfig_t cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.gridDim = dim3((unsigned)(L.slots * L.csize), 1, 1);
    cfg.blockDim = dim3(32 * NW, 1, 1);
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
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_emd<T, EXACT, NW>, C);
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
    int rc;
    if constexpr (sizeof(T) == 8) {
        if (p->exact)
            rc = launch_emd<T, true, 4>(C, L, st, tr);  // exact mode: float64, 4-warp CTAs
        else
            rc = L.nw == 5 ? launch_emd<T, false, 5>(C, L, st, tr) : launch_emd<T, false, 4>(C, L, st, tr);
    } else {
        rc = L.nw == 5 ? launch_emd<T, false, 5>(C, L, st, tr) : launch_emd<T, false, 4>(C, L, st, tr);
    }
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

int32_t eemd_philox_normals(uint64_t seed, int32_t signal, int32_t trial_begin, int32_t trial_count, int64_t n,
                            double* out, void* stream) {
    if (!out || signal < 0 || trial_begin < 0 || trial_count < 1 || n < 1) return EEMD_E_BADARG;
    const int64_t total = (int64_t)trial_count * n;
    const int64_t blocks = (total + 255) / 256;
    k_philox_fill<<<(unsigned)(blocks < 148 * 32 ? blocks : 148 * 32), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        seed, signal, trial_begin, trial_count, n, out);
    return cudaGetLastError() == cudaSuccess ? EEMD_OK : EEMD_E_CUDA;
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
    if ((p->noise_mode == EEMD_NOISE_INJECTED || p->noise_mode == EEMD_NOISE_SCALED) && !noise)
        return EEMD_E_BADARG;
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
    C.w1 = base + L.o_w1;
    C.r1 = base + L.o_r1;
    C.ri = reinterpret_cast<int4*>(base + L.o_ri);
    C.scr = reinterpret_cast<double2*>(base + L.o_scr);
    C.x = x;
    C.noise = noise;
    C.knot_log = knot_log;
    C.mode_sifts = mode_sifts;
    C.slot_knots = L.slot_knots;
    C.slot_M = L.slot_M;
    C.slot_n = L.slot_n;
    C.slot_runs = L.slot_runs;
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
    C.B = L.B;
    C.S = L.S;
    C.scr_rows = L.scr_rows;
    C.nw = L.nw;
    C.tau = p->tau;
    C.noise_scale = p->eps;
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
