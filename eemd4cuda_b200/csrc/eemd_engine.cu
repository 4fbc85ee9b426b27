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
// (separately rounded products, IEEE divisions; the file is compiled with
// --fmad=false so the compiler never contracts a*b+c).  exact=0 uses explicit
// fma() and one reciprocal per row / interval.
#include "../../include/eemd_b200.h"
#include "eemd_internal.cuh"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

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
template <typename T>
__device__ __forceinline__ void stv(void* p, int64_t i, double v) {
    static_cast<T*>(p)[i] = (T)v;
}
// value rounded to the storage type, held in double
template <typename T>
__device__ __forceinline__ double rnd(double v) { return (double)(T)v; }

__device__ __forceinline__ unsigned long long lb_pack(uint64_t flag, uint32_t a, uint32_t b) {
    return (flag << 62) | ((uint64_t)(a & 0x7fffffffu) << 31) | (uint64_t)(b & 0x7fffffffu);
}
__device__ __forceinline__ uint32_t lb_max(unsigned long long v) { return (uint32_t)((v >> 31) & 0x7fffffffu); }
__device__ __forceinline__ uint32_t lb_min(unsigned long long v) { return (uint32_t)(v & 0x7fffffffu); }
__device__ __forceinline__ uint32_t lb_flag(unsigned long long v) { return (uint32_t)(v >> 62); }

// largest pos in [0, count) with pref[pos] <= key (pref non-decreasing, pref[0] = 0)
__device__ __forceinline__ int find_item(const int32_t* pref, int count, int key) {
    int lo = 0, hi = count;  // invariant pref[lo] <= key < pref[hi] (pref[count] = total)
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (pref[mid] <= key) lo = mid; else hi = mid;
    }
    return lo;
}

// Knot i2 of the envelope in "mirror space" (emd_ref.py:92-96): with mir=1 the
// list is [2t0-t1, t0..t_{P-1}, 2t_{P-1}-t_{P-2}] with values [y1, y.., y_{P-2}].
template <typename T>
__device__ __forceinline__ void knot2(const int32_t* kt, const T* ky, int P, int mir, int i2,
                                      int& t, double& y) {
    if (mir) {
        if (i2 == 0) { t = 2 * kt[0] - kt[1]; y = (double)ky[1]; return; }
        if (i2 == P + 1) { t = 2 * kt[P - 1] - kt[P - 2]; y = (double)ky[P - 2]; return; }
        i2 -= 1;
    }
    t = kt[i2];
    y = (double)ky[i2];
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

// same cubic with the interval's reciprocal and h^2/6 precomputed
__device__ __forceinline__ double spline_fast(double t, double tl, double tr, double yl, double yr,
                                              double Ml, double Mr, double inv_h, double h26) {
    double a = (tr - t) * inv_h;
    double b = (t - tl) * inv_h;
    double ca = a * fma(a, a, -1.0);
    double cb = b * fma(b, b, -1.0);
    return fma(a, yl, b * yr) + fma(ca, Ml, cb * Mr) * h26;
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
__global__ void __launch_bounds__(1024) k_sigma(Ctx C, double eps, double* sigma_out) {
    __shared__ double2 sh[32];
    const int s = blockIdx.x;
    const SignalDesc d = C.sd[s];
    const T* x = static_cast<const T*>(C.x) + d.x_off;
    double acc = 0.0;
    for (int64_t i = threadIdx.x; i < d.n; i += 1024) acc += (double)x[i];
    double2 r = block_sum2<1024>(make_double2(acc, 0.0), sh);
    __shared__ double mean_s;
    if (threadIdx.x == 0) mean_s = r.x / (double)d.n;
    __syncthreads();
    const double mean = mean_s;
    acc = 0.0;
    for (int64_t i = threadIdx.x; i < d.n; i += 1024) {
        double dv = (double)x[i] - mean;
        acc += dv * dv;
    }
    r = block_sum2<1024>(make_double2(acc, 0.0), sh);
    if (threadIdx.x == 0) sigma_out[s] = eps * sqrt(r.x / (double)d.n);
}

// ---------------------------------------------------------------------------
// k_init: task states
// ---------------------------------------------------------------------------
__global__ void k_init(Ctx C) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.n_tasks) return;
    TaskState s;
    memset(&s, 0, sizeof(s));
    s.phase = PH_INIT;
    C.ts[i] = s;
}

// ---------------------------------------------------------------------------
// k_plan: compact the live tasks into the eval list (tiles) and the solve list
// (window chunks) of this step.  One CTA.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int solve_chunks(const Ctx& C, int P) {
    int mir = (C.end_mode == EEMD_END_MIRROR && P >= 3) ? 1 : 0;
    int n = P + 2 * mir - 2;
    int nwin = n > 0 ? (n + C.B - 1) / C.B : 1;
    return (nwin + SOLVE_THREADS - 1) / SOLVE_THREADS;
}

__global__ void __launch_bounds__(PLAN_THREADS) k_plan(Ctx C) {
    __shared__ int4 wsum[PLAN_THREADS / 32];
    __shared__ int4 carry;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) carry = make_int4(0, 0, 0, 0);
    __syncthreads();
    for (int base = 0; base < C.n_tasks; base += PLAN_THREADS) {
        const int task = base + tid;
        int ph = PH_DONE;
        if (task < C.n_tasks) ph = C.ts[task].phase;
        int4 v = make_int4(0, 0, 0, 0);  // (eval items, eval tiles, solve items, solve chunks)
        int c0 = 0, c1 = 0;
        if (ph != PH_DONE) {
            v.x = 1;
            v.y = C.td[task].ntiles;
            if (ph == PH_SIFT) {
                const TaskState s = C.ts[task];
                c0 = solve_chunks(C, s.pmax);
                c1 = solve_chunks(C, s.pmin);
                v.z = 2;
                v.w = c0 + c1;
            }
        }
        // block exclusive scan of v
        int4 inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int4 t;
            t.x = __shfl_up_sync(0xffffffffu, inc.x, o);
            t.y = __shfl_up_sync(0xffffffffu, inc.y, o);
            t.z = __shfl_up_sync(0xffffffffu, inc.z, o);
            t.w = __shfl_up_sync(0xffffffffu, inc.w, o);
            if (lane >= o) { inc.x += t.x; inc.y += t.y; inc.z += t.z; inc.w += t.w; }
        }
        if (lane == 31) wsum[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            int4 w = wsum[lane];
            int4 wi = w;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int4 t;
                t.x = __shfl_up_sync(0xffffffffu, wi.x, o);
                t.y = __shfl_up_sync(0xffffffffu, wi.y, o);
                t.z = __shfl_up_sync(0xffffffffu, wi.z, o);
                t.w = __shfl_up_sync(0xffffffffu, wi.w, o);
                if (lane >= o) { wi.x += t.x; wi.y += t.y; wi.z += t.z; wi.w += t.w; }
            }
            wsum[lane] = make_int4(wi.x - w.x, wi.y - w.y, wi.z - w.z, wi.w - w.w);
        }
        __syncthreads();
        const int4 wb = wsum[wid];
        const int4 cb = carry;
        int4 ex;
        ex.x = cb.x + wb.x + inc.x - v.x;
        ex.y = cb.y + wb.y + inc.y - v.y;
        ex.z = cb.z + wb.z + inc.z - v.z;
        ex.w = cb.w + wb.w + inc.w - v.w;
        if (v.x) {
            C.el_task[ex.x] = task;
            C.el_pref[ex.x] = ex.y;
        }
        if (v.z) {
            C.sl_item[ex.z] = task * 2;
            C.sl_pref[ex.z] = ex.w;
            C.sl_item[ex.z + 1] = task * 2 + 1;
            C.sl_pref[ex.z + 1] = ex.w + c0;
        }
        __syncthreads();
        if (tid == PLAN_THREADS - 1) {
            carry = make_int4(ex.x + v.x, ex.y + v.y, ex.z + v.z, ex.w + v.w);
        }
        __syncthreads();
    }
    if (tid == 0) {
        const int4 c = carry;
        C.el_pref[c.x] = c.y;
        C.sl_pref[c.z] = c.w;
        Header* h = C.hdr;
        h->n_elist = c.x;
        h->eval_total = c.y;
        h->n_slist = c.z;
        h->solve_total = c.w;
        h->eval_ticket = 0u;
        h->solve_ticket = 0u;
        h->active = c.x;
        h->step = h->step + 1;
    }
}

// ---------------------------------------------------------------------------
// k_solve: decay-seamed block Thomas (emd_gpu_v5_dsbt.py:51-74 window solve,
// emd_ref.py:31-65 system + Thomas).  One thread per window of B owned rows,
// halo S rows on each side with the outer couplings dropped; only owned rows
// are written (the seam error decays as (2-sqrt(3))^S).  The rows are built
// on the fly from the knots (no materialised d/l/u/r slabs).
// ---------------------------------------------------------------------------
template <typename T, bool EXACT>
__device__ __forceinline__ void solve_window(const Ctx& C, int task, int env, int chunk, int w) {
    const TaskDesc d = C.td[task];
    const TaskState s = C.ts[task];
    const int P = env ? s.pmin : s.pmax;
    const int64_t plane = (int64_t)(s.kpar * 2 + env) * C.KC + d.k_off;
    const int32_t* kt = C.kt + plane;
    const T* ky = static_cast<const T*>(C.ky) + plane;
    double* M2 = C.M + (int64_t)env * C.KC + d.k_off;
    const int mir = (C.end_mode == EEMD_END_MIRROR && P >= 3) ? 1 : 0;
    const int p2 = P + 2 * mir;
    const int n = p2 - 2;
    const int B = C.B, S = C.S;
    const int nwin = n > 0 ? (n + B - 1) / B : 1;
    if (w >= nwin) return;
    if (n <= 0) {
        for (int i = 0; i < p2; ++i) M2[i] = 0.0;
        return;
    }
    if (p2 > d.kcap) { raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, task); return; }
    const int o0 = w * B;
    const int o1 = min(n, o0 + B) - 1;
    const int w0 = max(0, o0 - S);
    const int w1 = min(n - 1, o1 + S);
    double2* sc = C.scr + d.scr_off + (int64_t)env * d.scr_env +
                  (int64_t)chunk * (B + S) * SOLVE_THREADS + threadIdx.x;

    int ta, tb, tc;
    double ya, yb, yc;
    knot2<T>(kt, ky, P, mir, w0, ta, ya);
    knot2<T>(kt, ky, P, mir, w0 + 1, tb, yb);
    double cp = 0.0, dp = 0.0;
    for (int i = w0; i <= w1; ++i) {
        knot2<T>(kt, ky, P, mir, i + 2, tc, yc);
        const double H0 = (double)(tb - ta);
        const double H1 = (double)(tc - tb);
        const double dg = 2.0 * (H0 + H1);
        const double l = (i >= 1) ? H0 : 0.0;
        const double u = (i <= n - 2) ? H1 : 0.0;
        const double r = 6.0 * ((yc - yb) / H1 - (yb - ya) / H0);
        double c, dv;
        if (EXACT) {
            c = (i == w1) ? 0.0 : u / (dg - l * cp);
            dv = (r - l * dp) / (dg - l * cp);
        } else {
            const double inv = 1.0 / fma(-l, cp, dg);
            c = (i == w1) ? 0.0 : u * inv;
            dv = fma(-l, dp, r) * inv;
        }
        if (i >= o0) sc[(int64_t)(i - o0) * SOLVE_THREADS] = make_double2(c, dv);
        cp = c;
        dp = dv;
        ta = tb; ya = yb;
        tb = tc; yb = yc;
    }
    double xv = dp;
    if (w1 <= o1) M2[w1 + 1] = xv;
    for (int i = w1 - 1; i >= o0; --i) {
        const double2 cd = sc[(int64_t)(i - o0) * SOLVE_THREADS];
        xv = EXACT ? (cd.y - cd.x * xv) : fma(-cd.x, xv, cd.y);
        if (i <= o1) M2[i + 1] = xv;
    }
    if (o0 == 0) M2[0] = 0.0;
    if (o1 == n - 1) M2[p2 - 1] = 0.0;
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(SOLVE_THREADS) k_solve(Ctx C) {
    __shared__ int sh_ticket, sh_pos;
    for (;;) {
        if (threadIdx.x == 0) {
            const int total = C.hdr->solve_total;
            const int t = (int)atomicAdd(&C.hdr->solve_ticket, 1u);
            sh_ticket = t;
            sh_pos = (t < total) ? find_item(C.sl_pref, C.hdr->n_slist, t) : -1;
        }
        __syncthreads();
        const int ticket = sh_ticket, pos = sh_pos;
        __syncthreads();
        if (pos < 0) break;
        const int item = C.sl_item[pos];
        const int chunk = ticket - C.sl_pref[pos];
        solve_window<T, EXACT>(C, item >> 1, item & 1, chunk, chunk * SOLVE_THREADS + threadIdx.x);
    }
}

// ---------------------------------------------------------------------------
// k_eval: the fused per-tile pass
// ---------------------------------------------------------------------------
enum TileMode : int { TM_INIT = 0, TM_SIFT = 1, TM_LAST = 2, TM_TRANS = 3 };

struct TileInfo {
    int task, tile, mode, n, t0, tl, ntiles, tile_off, is_last, q;
    int imf, sift, kpar, src_resid, imf_from_resid;
    int P[2], kb[2], kcnt[2], mir[2], p2[2], lo2[2], hi2[2];
    int tfirst[2], tlast[2];  // virtual mirror knot positions
    double cval[2];
    int excl[2], agg[2];
};

__device__ __forceinline__ size_t eval_smem_bytes_dev(int TILE) {
    const int W = TILE >> 5, cap = (TILE >> 1) + 8;
    return (size_t)3 * (TILE + 2) * 8 + (size_t)2 * cap * 8 * 3 + (size_t)2 * cap * 4 + (size_t)4 * 2 * W * 4;
}

// knots strictly before sample t (t in the tile, or t0-1 / t0+tl) in mirror space
__device__ __forceinline__ int count_less(const TileInfo& I, const unsigned* mask, const int* wb,
                                          const int* skt, int env, int t) {
    const int j = t - I.t0;
    int c;
    if (j < 0) {
        const int kb = I.kb[env];
        c = kb;
        if (kb >= 1) {
            const int loc = (kb - 1 + I.mir[env]) - I.lo2[env];
            if (skt[loc] == t) c -= 1;
        }
    } else if (j >= I.tl) {
        c = I.kb[env] + I.kcnt[env];
    } else {
        const int w = j >> 5, b = j & 31;
        c = I.kb[env] + wb[w] + __popc(mask[w] & ((1u << b) - 1u));
    }
    if (I.mir[env]) c += (I.tfirst[env] < t ? 1 : 0) + (I.tlast[env] < t ? 1 : 0);
    return c;
}

template <bool EXACT>
__device__ __forceinline__ double env_value(const TileInfo& I, int env, int t, const unsigned* mask,
                                            const int* wb, const int* skt, const double* sky,
                                            const double* sM, const double* saux, const Ctx& C) {
    const int P = I.P[env];
    if (P < 2) return I.cval[env];
    int idx2 = count_less(I, mask, wb, skt, env, t) - 1;
    idx2 = max(0, min(idx2, I.p2[env] - 2));
    const int loc = idx2 - I.lo2[env];
#ifdef EEMD_CHECKED
    if (loc < 0 || loc + 1 > I.hi2[env] - I.lo2[env]) {
        raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, 1000000 + loc);
        return 0.0;
    }
#endif
    const double tl = (double)skt[loc], tr = (double)skt[loc + 1];
    if (EXACT) return spline_exact((double)t, tl, tr, sky[loc], sky[loc + 1], sM[loc], sM[loc + 1]);
    const double h = tr - tl;
    return spline_fast((double)t, tl, tr, sky[loc], sky[loc + 1], sM[loc], sM[loc + 1], saux[loc],
                       h * h * (1.0 / 6.0));
}

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

// IMF-level decision for the IMF about to start (emd_ref.py:120-127; emd_gpu.py:155-168)
__device__ __forceinline__ void imf_level(const Ctx& C, TaskState& s, int cmax, int cmin) {
    bool stop = (cmax + cmin < C.min_extrema);
    if (C.rules == EEMD_RULES_NUMBA) stop = stop || cmax < 2 || cmin < 2;
    if (stop) { s.phase = PH_DONE; return; }
    if (s.imf >= C.max_imf) { s.phase = PH_DONE; s.flags |= 1; return; }
    s.mode_sifts_cur = 0;
    if (C.rules == EEMD_RULES_REF && (cmax < 1 || cmin < 1)) {
        // emd_ref.py:132-133: the sift loop breaks before its first sift; the IMF is the residual
        s.phase = PH_TRANS;
        s.imf_from_resid = 1;
        return;
    }
    s.phase = PH_SIFT;
    s.sift = 0;
    s.src_resid = 1;
    s.imf_from_resid = 0;
    s.kpar ^= 1;
    s.pmax = cmax;
    s.pmin = cmin;
}

__device__ __forceinline__ void close_imf(const Ctx& C, TaskState& s, int task) {
    if (C.mode_sifts) C.mode_sifts[(int64_t)task * C.max_imf + s.imf] = s.mode_sifts_cur;
    s.nmode = s.imf + 1;
    s.imf += 1;
    s.mode_sifts_cur = 0;
}

__device__ __forceinline__ void log_sift(const Ctx& C, int task, const TaskState& s) {
    if (C.knot_log) {
        int32_t* p = C.knot_log + (((int64_t)task * C.max_imf + s.imf) * C.max_sifts + s.sift) * 2;
        p[0] = s.pmax;
        p[1] = s.pmin;
    }
}

template <typename T, bool EXACT>
__global__ void __launch_bounds__(EVAL_THREADS) k_eval(Ctx C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int TILE = C.tile;
    const int W = TILE >> 5;
    const int cap = (TILE >> 1) + 8;
    double* s_h = reinterpret_cast<double*>(smem_raw);  // old h      [TILE+2]
    double* s_f = s_h + (TILE + 2);                      // new values [TILE+2]
    double* s_r = s_f + (TILE + 2);                      // residual   [TILE+2]
    double* s_ky = s_r + (TILE + 2);                     // [2][cap]
    double* s_M = s_ky + 2 * cap;                        // [2][cap]
    double* s_aux = s_M + 2 * cap;                       // [2][cap] 1/h of interval
    int* s_kt = reinterpret_cast<int*>(s_aux + 2 * cap); // [2][cap]
    unsigned* s_mask = reinterpret_cast<unsigned*>(s_kt + 2 * cap);  // [2][W]
    int* s_wb = reinterpret_cast<int*>(s_mask + 2 * W);               // [2][W]
    unsigned* s_nm = reinterpret_cast<unsigned*>(s_wb + 2 * W);       // [2][W]
    int* s_nb = reinterpret_cast<int*>(s_nm + 2 * W);                 // [2][W]

    __shared__ TileInfo I;
    __shared__ double2 s_red[EVAL_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;

    for (;;) {
        // ---------------- 0. claim a tile ----------------
        if (tid == 0) {
            const int total = C.hdr->eval_total;
            const int ticket = (int)atomicAdd(&C.hdr->eval_ticket, 1u);
            if (ticket >= total) {
                I.task = -1;
            } else {
                const int pos = find_item(C.el_pref, C.hdr->n_elist, ticket);
                const int task = C.el_task[pos];
                const TaskDesc d = C.td[task];
                const TaskState s = C.ts[task];
                I.task = task;
                I.tile = ticket - C.el_pref[pos];
                I.n = d.n;
                I.t0 = I.tile * TILE;
                I.tl = min(TILE, d.n - I.t0);
                I.ntiles = d.ntiles;
                I.tile_off = d.tile_off;
                I.q = C.hdr->step & 1;
                I.imf = s.imf;
                I.sift = s.sift;
                I.kpar = s.kpar;
                I.src_resid = s.src_resid;
                I.imf_from_resid = s.imf_from_resid;
                I.P[0] = s.pmax;
                I.P[1] = s.pmin;
                if (s.phase == PH_INIT) I.mode = TM_INIT;
                else if (s.phase == PH_TRANS) I.mode = TM_TRANS;
                else I.mode = (s.sift + 1 >= C.max_sifts) ? TM_LAST : TM_SIFT;
            }
        }
        __syncthreads();
        if (I.task < 0) break;

        const int task = I.task, tile = I.tile, n = I.n, t0 = I.t0, tl = I.tl, mode = I.mode;
        const TaskDesc d = C.td[task];
        const int64_t gt = (int64_t)d.tile_off + tile;
        const bool sifting = (mode == TM_SIFT || mode == TM_LAST);
        T* resid = static_cast<T*>(C.resid) + d.s_off;
        T* imf_m = static_cast<T*>(C.imfs) + d.imf_off + (int64_t)min(I.imf, C.max_imf - 1) * n;

        // ---------------- 1. load the tile ----------------
        if (sifting) {
            const T* src = I.src_resid ? resid : imf_m;
            for (int j = tid; j < tl; j += EVAL_THREADS) s_h[1 + j] = (double)src[t0 + j];
            if (tid == 0 && t0 > 0) {
                s_h[0] = I.src_resid ? C.redge[(int64_t)(I.imf & 1) * C.TT + gt - 1].y
                                     : C.hedge[(int64_t)(I.sift & 1) * C.TT + gt - 1].y;
            }
            if (tid == 1 && t0 + tl < n) {
                s_h[tl + 1] = I.src_resid ? C.redge[(int64_t)(I.imf & 1) * C.TT + gt + 1].x
                                          : C.hedge[(int64_t)(I.sift & 1) * C.TT + gt + 1].x;
            }
        }
        if (mode == TM_LAST || mode == TM_TRANS) {
            for (int j = tid; j < tl; j += EVAL_THREADS) s_r[1 + j] = (double)resid[t0 + j];
            if (tid == 0 && t0 > 0) s_r[0] = C.redge[(int64_t)(I.imf & 1) * C.TT + gt - 1].y;
            if (tid == 1 && t0 + tl < n) s_r[tl + 1] = C.redge[(int64_t)(I.imf & 1) * C.TT + gt + 1].x;
        }

        // ---------------- 2. stage the current knots ----------------
        if (sifting) {
            if (tid < 2) {
                const int env = tid;
                const int P = I.P[env];
                const int64_t plane = (int64_t)(I.kpar * 2 + env) * C.KC + d.k_off;
                const int32_t* kt = C.kt + plane;
                const T* ky = static_cast<const T*>(C.ky) + plane;
                const int2 tp = C.tpref[(int64_t)I.kpar * C.TT + gt];
                const int kb = env ? tp.y : tp.x;
                int kend = P;
                if (tile + 1 < I.ntiles) {
                    const int2 tn = C.tpref[(int64_t)I.kpar * C.TT + gt + 1];
                    kend = env ? tn.y : tn.x;
                }
                const int mir = (C.end_mode == EEMD_END_MIRROR && P >= 3) ? 1 : 0;
                I.kb[env] = kb;
                I.kcnt[env] = kend - kb;
                I.mir[env] = mir;
                I.p2[env] = P + 2 * mir;
                I.cval[env] = (P == 1) ? (double)ky[0] : 0.0;
                if (P >= 2) {
                    I.lo2[env] = max(0, mir + kb - 2);
                    I.hi2[env] = min(P + 2 * mir - 1, mir + kb + (kend - kb) + 1);
                } else {
                    I.lo2[env] = 0;
                    I.hi2[env] = -1;
                }
                if (mir) {
                    I.tfirst[env] = 2 * kt[0] - kt[1];
                    I.tlast[env] = 2 * kt[P - 1] - kt[P - 2];
                } else {
                    I.tfirst[env] = 0;
                    I.tlast[env] = 0;
                }
                if (I.hi2[env] - I.lo2[env] + 1 > cap || I.kcnt[env] < 0 || I.kcnt[env] > (TILE >> 1) + 1) {
                    raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, task);
                    I.hi2[env] = I.lo2[env] - 1;
                    I.kcnt[env] = 0;
                }
            }
            for (int w = tid; w < 2 * W; w += EVAL_THREADS) s_mask[w] = 0u;
            __syncthreads();
#pragma unroll
            for (int env = 0; env < 2; ++env) {
                const int P = I.P[env];
                const int64_t plane = (int64_t)(I.kpar * 2 + env) * C.KC + d.k_off;
                const int32_t* kt = C.kt + plane;
                const T* ky = static_cast<const T*>(C.ky) + plane;
                const double* M2 = C.M + (int64_t)env * C.KC + d.k_off;
                const int lo2 = I.lo2[env], cnt = I.hi2[env] - lo2 + 1;
                for (int k = tid; k < cnt; k += EVAL_THREADS) {
                    int tt;
                    double yy;
                    knot2<T>(kt, ky, P, I.mir[env], lo2 + k, tt, yy);
                    s_kt[env * cap + k] = tt;
                    s_ky[env * cap + k] = yy;
                    s_M[env * cap + k] = M2[lo2 + k];
                }
                const int kb = I.kb[env], kc = I.kcnt[env];
                for (int k = tid; k < kc; k += EVAL_THREADS) {
                    const int j = kt[kb + k] - t0;
                    if (j >= 0 && j < tl) atomicOr(&s_mask[env * W + (j >> 5)], 1u << (j & 31));
                    else raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, 2000000 + task);
                }
            }
            __syncthreads();
            if (!EXACT) {
                for (int k = tid; k < 2 * cap; k += EVAL_THREADS) {
                    const int env = k >= cap ? 1 : 0, kk = k - env * cap;
                    if (kk < I.hi2[env] - I.lo2[env]) {
                        s_aux[k] = 1.0 / (double)(s_kt[k + 1] - s_kt[k]);
                    }
                }
            }
            if (wid < 2) {  // exclusive prefix of the word popcounts
                const int env = wid;
                int carry = 0;
                for (int w0 = 0; w0 < W; w0 += 32) {
                    const int w = w0 + lane;
                    const int c = (w < W) ? __popc(s_mask[env * W + w]) : 0;
                    int inc = c;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int t = __shfl_up_sync(0xffffffffu, inc, o);
                        if (lane >= o) inc += t;
                    }
                    if (w < W) s_wb[env * W + w] = carry + inc - c;
                    carry += __shfl_sync(0xffffffffu, inc, 31);
                }
            }
        }
        __syncthreads();

        // ---------------- 3. compute the new values (tile + 1-sample halo) ----------------
        double num = 0.0, den = 0.0;
        for (int jj = tid; jj < tl + 2; jj += EVAL_THREADS) {
            const int j = jj - 1;
            const int t = t0 + j;
            if (t < 0 || t >= n) continue;
            if (sifting) {
                const double h = s_h[jj];
                const double eu = env_value<EXACT>(I, 0, t, s_mask, s_wb, s_kt, s_ky, s_M, s_aux, C);
                const double el = env_value<EXACT>(I, 1, t, s_mask + W, s_wb + W, s_kt + cap, s_ky + cap,
                                                   s_M + cap, s_aux + cap, C);
                const double m = 0.5 * (eu + el);
                const double hn = rnd<T>(h - m);
                s_f[jj] = hn;
                if (j >= 0 && j < tl) {
                    if (C.rules == EEMD_RULES_NUMBA) {
                        num += m * m;
                    } else {
                        const double dd = h - hn;
                        num += dd * dd;
                    }
                    den += h * h;
                }
                if (mode == TM_LAST) s_r[jj] = rnd<T>(s_r[jj] - hn);
            } else if (mode == TM_TRANS) {
                const double ro = s_r[jj];
                const double hv = I.imf_from_resid ? ro : (double)imf_m[t];
                s_f[jj] = rnd<T>(ro - hv);
            } else {  // TM_INIT
                s_f[jj] = trial_input<T>(C, d, t);
            }
        }
        __syncthreads();
        const double* G = (mode == TM_LAST) ? s_r : s_f;  // signal whose extrema are the next knots

        // ---------------- 4. next knots: flags, counts ----------------
        for (int j0 = 0; j0 < TILE; j0 += EVAL_THREADS) {
            const int j = j0 + tid;
            const int t = t0 + j;
            bool fmx = false, fmn = false;
            if (j < tl && t >= 1 && t <= n - 2) {
                const double g = G[j + 1], gl = G[j], gr = G[j + 2];
                fmx = (g > gl) && (g > gr);
                fmn = (g < gl) && (g < gr);
            }
            const unsigned bm = __ballot_sync(0xffffffffu, fmx);
            const unsigned bn = __ballot_sync(0xffffffffu, fmn);
            if (lane == 0 && j < TILE) {
                s_nm[j >> 5] = bm;
                s_nm[W + (j >> 5)] = bn;
            }
        }
        __syncthreads();
        if (wid < 2) {
            const int env = wid;
            int carry = 0;
            for (int w0 = 0; w0 < W; w0 += 32) {
                const int w = w0 + lane;
                const int c = (w < W) ? __popc(s_nm[env * W + w]) : 0;
                int inc = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, inc, o);
                    if (lane >= o) inc += t;
                }
                if (w < W) s_nb[env * W + w] = carry + inc - c;
                carry += __shfl_sync(0xffffffffu, inc, 31);
            }
            if (lane == 0) I.agg[env] = carry;
        }
        __syncthreads();

        // ---------------- 5. decoupled look-back over the task's tiles ----------------
        if (tid == 0) {
            unsigned long long* st = C.status + (int64_t)I.q * C.TT + d.tile_off;
            const uint32_t amax = (uint32_t)I.agg[0], amin = (uint32_t)I.agg[1];
            uint32_t emax = 0, emin = 0;
            if (tile == 0) {
                atomicExch(&st[0], lb_pack(LB_INC, amax, amin));
            } else {
                atomicExch(&st[tile], lb_pack(LB_AGG, amax, amin));
                const long long limit = C.watchdog > 0 ? C.watchdog : -C.watchdog;
                if (C.watchdog < 0) {
                    // watchdog test mode: wait on a flag nothing sets, give up after `limit` polls
                    long long spins = 0;
                    while (*((volatile int32_t*)&C.hdr->pad[0]) == 0) {
                        if (++spins > limit) {
                            raise_error(C.hdr, EEMD_E_TIMEOUT, task);
                            break;
                        }
                        __nanosleep(32);
                    }
                }
                int k = tile - 1;
                long long spins = 0;
                while (k >= 0) {
                    const unsigned long long v = *((volatile unsigned long long*)&st[k]);
                    const uint32_t fl = lb_flag(v);
                    if (fl == LB_EMPTY) {
                        if (++spins > limit) {
                            raise_error(C.hdr, EEMD_E_TIMEOUT, task);
                            break;
                        }
                        __nanosleep(64);
                        continue;
                    }
                    emax += lb_max(v);
                    emin += lb_min(v);
                    if (fl == LB_INC) break;
                    --k;
                }
                atomicExch(&st[tile], lb_pack(LB_INC, emax + amax, emin + amin));
            }
            // clear this tile's word of the other plane for the next step
            C.status[(int64_t)(I.q ^ 1) * C.TT + gt] = 0ull;
            I.excl[0] = (int)emax;
            I.excl[1] = (int)emin;
            C.tpref[(int64_t)(I.kpar ^ 1) * C.TT + gt] = make_int2((int)emax, (int)emin);
        }
        __syncthreads();

        // ---------------- 6. write knots, samples, edges ----------------
        {
            const int np = I.kpar ^ 1;
            const int64_t pmx = (int64_t)(np * 2 + 0) * C.KC + d.k_off;
            const int64_t pmn = (int64_t)(np * 2 + 1) * C.KC + d.k_off;
            int32_t* ktx = C.kt + pmx;
            int32_t* ktn = C.kt + pmn;
            T* kyx = static_cast<T*>(C.ky) + pmx;
            T* kyn = static_cast<T*>(C.ky) + pmn;
            const int kcap_real = d.kcap - 2;
            for (int j = tid; j < tl; j += EVAL_THREADS) {
                const int t = t0 + j;
                const int w = j >> 5, b = j & 31;
                const unsigned lt = (1u << b) - 1u;
                const unsigned mx = s_nm[w], mn = s_nm[W + w];
                const double g = G[j + 1];
                if ((mx >> b) & 1u) {
                    const int pos = I.excl[0] + s_nb[w] + __popc(mx & lt);
                    if (pos < kcap_real) { ktx[pos] = t; kyx[pos] = (T)g; }
                    else raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, task);
                }
                if ((mn >> b) & 1u) {
                    const int pos = I.excl[1] + s_nb[W + w] + __popc(mn & lt);
                    if (pos < kcap_real) { ktn[pos] = t; kyn[pos] = (T)g; }
                    else raise_error(C.hdr, EEMD_E_KNOT_OVERFLOW, task);
                }
                switch (mode) {
                    case TM_SIFT: imf_m[t] = (T)s_f[j + 1]; break;
                    case TM_LAST: imf_m[t] = (T)s_f[j + 1]; resid[t] = (T)s_r[j + 1]; break;
                    case TM_TRANS:
                        resid[t] = (T)s_f[j + 1];
                        if (I.imf_from_resid) imf_m[t] = (T)s_r[j + 1];
                        break;
                    default: resid[t] = (T)s_f[j + 1]; break;
                }
            }
            if (tid == 0) {
                const double2 e = make_double2(G[1], G[tl]);
                if (mode == TM_SIFT) C.hedge[(int64_t)((I.sift + 1) & 1) * C.TT + gt] = e;
                else if (mode == TM_INIT) C.redge[gt] = e;
                else C.redge[(int64_t)((I.imf + 1) & 1) * C.TT + gt] = e;
            }
        }

        // ---------------- 7. SD partial sums, completion ----------------
        {
            const double2 r = block_sum2<EVAL_THREADS>(make_double2(num, den), s_red);
            if (tid == 0) {
                C.partial[gt] = r;
                __threadfence();
                const unsigned old = atomicAdd(&C.ts[task].done_count, 1u);
                I.is_last = (old + 1 == (unsigned)I.ntiles) ? 1 : 0;
            }
            __syncthreads();
        }

        // ---------------- 8. per-task decision (last tile to finish) ----------------
        if (I.is_last) {
            __threadfence();
            double2 acc = make_double2(0.0, 0.0);
            if (sifting) {
                for (int i = tid; i < I.ntiles; i += EVAL_THREADS) {
                    const double2 p = __ldcg(&C.partial[(int64_t)d.tile_off + i]);
                    acc.x += p.x;
                    acc.y += p.y;
                }
            }
            acc = block_sum2<EVAL_THREADS>(acc, s_red);
            if (tid == 0) {
                const unsigned long long v =
                    __ldcg(&C.status[(int64_t)I.q * C.TT + d.tile_off + I.ntiles - 1]);
                const int cmax = (int)lb_max(v), cmin = (int)lb_min(v);
                TaskState s = C.ts[task];
                if (mode == TM_SIFT) {
                    log_sift(C, task, s);
                    s.mode_sifts_cur += 1;
                    s.nsift_total += 1;
                    const double sdv = acc.y > 0.0 ? acc.x / acc.y : 0.0;
                    bool stop = (s.sift >= 1) && (sdv < C.tau);
                    if (!stop) {
                        stop = (C.rules == EEMD_RULES_NUMBA) ? (cmax < 2 || cmin < 2) : (cmax < 1 || cmin < 1);
                    }
                    if (stop) {
                        s.phase = PH_TRANS;
                        s.imf_from_resid = 0;
                    } else {
                        s.sift += 1;
                        s.kpar ^= 1;
                        s.pmax = cmax;
                        s.pmin = cmin;
                        s.src_resid = 0;
                    }
                } else if (mode == TM_LAST) {
                    log_sift(C, task, s);
                    s.mode_sifts_cur += 1;
                    s.nsift_total += 1;
                    close_imf(C, s, task);
                    imf_level(C, s, cmax, cmin);
                } else if (mode == TM_TRANS) {
                    close_imf(C, s, task);
                    imf_level(C, s, cmax, cmin);
                } else {
                    s.imf = 0;
                    s.nmode = 0;
                    imf_level(C, s, cmax, cmin);
                }
                s.done_count = 0u;
                C.ts[task] = s;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// k_reduce: imf_sum[s][m][t] += trial-ordered sum over the batch (emd_par.py:241-245)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_reduce(Ctx C, double* imf_sum, int32_t* mode_count) {
    const int s = blockIdx.z, m = blockIdx.y;
    const SignalDesc sd = C.sd[s];
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (mode_count && blockIdx.x == 0 && threadIdx.x == 0) {
        int cnt = 0;
        for (int e = 0; e < C.trial_count; ++e) cnt += (C.ts[sd.first_task + e].nmode > m) ? 1 : 0;
        mode_count[(int64_t)s * C.max_imf + m] += cnt;
    }
    if (!imf_sum || t >= sd.n) return;
    double acc = 0.0;
    bool any = false;
    for (int e = 0; e < C.trial_count; ++e) {
        const int task = sd.first_task + e;
        if (C.ts[task].nmode > m) {
            const double v = ldv<T>(C.imfs, C.td[task].imf_off + (int64_t)m * sd.n + t);
            acc = any ? acc + v : v;
            any = true;
        }
    }
    if (any) {
        double* p = imf_sum + sd.sum_off + (int64_t)m * sd.n + t;
        *p = *p + acc;
    }
}

__global__ void k_outputs(Ctx C, int32_t* nsift, int32_t* nmode, int32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.n_tasks) return;
    const TaskState s = C.ts[i];
    if (nsift) nsift[i] = s.nsift_total;
    if (nmode) nmode[i] = s.nmode;
    if (flags) flags[i] = s.flags;
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

struct Layout {
    std::vector<TaskDesc> td;
    std::vector<SignalDesc> sd;
    int64_t TT = 0, NS = 0, KC = 0, NIMF = 0, SCR = 0;
    int tile = 0, B = 0, S = 0;
    int max_chunks = 0;
    size_t o_hdr, o_td, o_ts, o_sd, o_sigma, o_el_task, o_el_pref, o_sl_item, o_sl_pref;
    size_t o_status, o_partial, o_tpref, o_hedge, o_redge, o_resid, o_imfs, o_kt, o_ky, o_M, o_scr;
    size_t total = 0;
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int autotune_tile(int64_t nmax) {
    // length buckets: short signals use small tiles so that a task spans
    // several CTAs; long ones amortise the tile's halo and look-back.
    if (nmax <= 8192) return 512;
    if (nmax <= 262144) return 1024;
    return 2048;
}

int autotune_block(int64_t nmax) { return nmax <= 262144 ? 64 : 256; }

size_t eval_smem_bytes(int TILE) {
    const int W = TILE >> 5, cap = (TILE >> 1) + 8;
    return (size_t)3 * (TILE + 2) * 8 + (size_t)2 * cap * 8 * 3 + (size_t)2 * cap * 4 + (size_t)4 * 2 * W * 4;
}

int check_params(const eemd_params* p) {
    if (!p) return EEMD_E_BADARG;
    if (p->dtype != EEMD_F64 && p->dtype != EEMD_F32) return EEMD_E_BADARG;
    if (p->exact && p->dtype != EEMD_F64) return EEMD_E_NOTSUP;
    if (p->max_sifts < 1 || p->max_imf < 1 || p->max_imf > 4096) return EEMD_E_BADARG;
    if (p->end_mode != EEMD_END_NATURAL && p->end_mode != EEMD_END_MIRROR) return EEMD_E_BADARG;
    if (p->rules != EEMD_RULES_REF && p->rules != EEMD_RULES_NUMBA) return EEMD_E_BADARG;
    if (p->noise_mode < EEMD_NOISE_NONE || p->noise_mode > EEMD_NOISE_PREPERTURBED) return EEMD_E_BADARG;
    if (p->tile != 0 && (p->tile < 256 || p->tile > 4096 || p->tile % 256 != 0)) return EEMD_E_BADARG;
    if (p->knots_per_block < 0 || p->halo < 0) return EEMD_E_BADARG;
    return EEMD_OK;
}

int make_layout(const eemd_params* p, const int64_t* lengths, int n_signals, int trial_count,
                int trial_begin, bool imfs_external, Layout& L) {
    int rc = check_params(p);
    if (rc) return rc;
    if (!lengths || n_signals < 1 || trial_count < 1) return EEMD_E_BADARG;
    const int64_t n_tasks = (int64_t)n_signals * trial_count;
    if (n_tasks > (1 << 24)) return EEMD_E_BADARG;
    int64_t nmax = 0;
    for (int s = 0; s < n_signals; ++s) {
        if (lengths[s] < 3 || lengths[s] > (1LL << 30)) return EEMD_E_BADARG;
        nmax = std::max(nmax, lengths[s]);
    }
    L.tile = p->tile ? p->tile : autotune_tile(nmax);
    L.B = p->knots_per_block ? p->knots_per_block : autotune_block(nmax);
    L.S = p->halo ? p->halo : 32;
    L.td.resize(n_tasks);
    L.sd.resize(n_signals);
    int64_t xo = 0, so = 0, imo = 0, ko = 0, scro = 0, sumo = 0;
    int64_t to = 0;
    int64_t chunks = 0;
    for (int s = 0; s < n_signals; ++s) {
        const int64_t n = lengths[s];
        SignalDesc& sd = L.sd[s];
        sd.x_off = xo;
        sd.sum_off = sumo;
        sd.r_off = xo;
        sd.n = (int32_t)n;
        sd.first_task = s * trial_count;
        sumo += (int64_t)p->max_imf * n;
        const int kcap = (int)(n / 2 + 4);
        const int nwin_max = (kcap + L.B - 1) / L.B;
        const int nch = (nwin_max + SOLVE_THREADS - 1) / SOLVE_THREADS;
        const int64_t scr_env = (int64_t)nch * (L.B + L.S) * SOLVE_THREADS;
        for (int e = 0; e < trial_count; ++e) {
            TaskDesc& d = L.td[(int64_t)s * trial_count + e];
            d.x_off = (p->noise_mode == EEMD_NOISE_PREPERTURBED) ? so : xo;
            d.s_off = so;
            d.imf_off = imo;
            d.k_off = ko;
            d.scr_off = scro;
            d.scr_env = scr_env;
            d.noise_off = so;
            d.n = (int32_t)n;
            d.kcap = kcap;
            d.tile_off = (int32_t)to;
            d.ntiles = (int32_t)((n + L.tile - 1) / L.tile);
            d.signal = s;
            d.trial = trial_begin + e;
            so += n;
            imo += (int64_t)p->max_imf * n;
            ko += kcap;
            scro += 2 * scr_env;
            to += d.ntiles;
            chunks += 2 * nch;
        }
        xo += n;
    }
    if (to > (1LL << 30)) return EEMD_E_BADARG;
    L.TT = to;
    L.NS = so;
    L.KC = ko;
    L.NIMF = imo;
    L.SCR = scro;
    L.max_chunks = (int)std::min<int64_t>(chunks, 1 << 30);
    const size_t bt = (p->dtype == EEMD_F64) ? 8 : 4;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
    L.o_hdr = take(sizeof(Header));
    L.o_td = take(sizeof(TaskDesc) * n_tasks);
    L.o_ts = take(sizeof(TaskState) * n_tasks);
    L.o_sd = take(sizeof(SignalDesc) * n_signals);
    L.o_sigma = take(sizeof(double) * n_signals);
    L.o_el_task = take(sizeof(int32_t) * (n_tasks + 1));
    L.o_el_pref = take(sizeof(int32_t) * (n_tasks + 1));
    L.o_sl_item = take(sizeof(int32_t) * (2 * n_tasks + 1));
    L.o_sl_pref = take(sizeof(int32_t) * (2 * n_tasks + 1));
    L.o_status = take(sizeof(unsigned long long) * 2 * L.TT);
    L.o_partial = take(sizeof(double2) * L.TT);
    L.o_tpref = take(sizeof(int2) * 2 * L.TT);
    L.o_hedge = take(sizeof(double2) * 2 * L.TT);
    L.o_redge = take(sizeof(double2) * 2 * L.TT);
    L.o_resid = take(bt * L.NS);
    L.o_imfs = imfs_external ? 0 : take(bt * L.NIMF);
    L.o_kt = take(sizeof(int32_t) * 4 * L.KC);
    L.o_ky = take(bt * 4 * L.KC);
    L.o_M = take(sizeof(double) * 2 * L.KC);
    L.o_scr = take(sizeof(double2) * L.SCR);
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

template <typename K>
int grid_for(K kernel, int threads, size_t smem, int64_t work_items) {
    int dev = 0, nsm = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem);
    if (occ < 1) occ = 1;
    int64_t g = (int64_t)nsm * occ;
    if (work_items < g) g = work_items;
    return (int)std::max<int64_t>(g, 1);
}

template <typename T, bool EXACT>
int launch_steps(const Ctx& C, const Layout& L, int nsteps, cudaStream_t st, Tracer& tr) {
    const size_t smem = eval_smem_bytes(L.tile);
    cudaFuncSetAttribute(k_eval<T, EXACT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const int ge = grid_for(k_eval<T, EXACT>, EVAL_THREADS, smem, L.TT);
    const int gs = grid_for(k_solve<T, EXACT>, SOLVE_THREADS, 0, L.max_chunks);
    for (int i = 0; i < nsteps; ++i) {
        tr.begin(EEMD_K_PLAN);
        k_plan<<<1, PLAN_THREADS, 0, st>>>(C);
        tr.end();
        tr.begin(EEMD_K_SOLVE);
        k_solve<T, EXACT><<<gs, SOLVE_THREADS, 0, st>>>(C);
        tr.end();
        tr.begin(EEMD_K_EVAL);
        k_eval<T, EXACT><<<ge, EVAL_THREADS, smem, st>>>(C);
        tr.end();
    }
    return cudaGetLastError() == cudaSuccess ? EEMD_OK : EEMD_E_CUDA;
}

template <typename T>
int run_typed(const eemd_params* p, const Layout& L, Ctx& C, double* imf_sum, int32_t* mode_count,
              int32_t* nsift, int32_t* nmode, int32_t* flags, void* resid_out, cudaStream_t st,
              Tracer& tr) {
    const int64_t n_tasks = (int64_t)L.td.size();
    if (p->noise_mode == EEMD_NOISE_PHILOX) {
        tr.begin(EEMD_K_SIGMA);
        k_sigma<T><<<(int)L.sd.size(), 1024, 0, st>>>(C, p->eps, const_cast<double*>(C.sigma));
        tr.end();
    }
    tr.begin(EEMD_K_INIT);
    k_init<<<(int)((n_tasks + 255) / 256), 256, 0, st>>>(C);
    tr.end();
    const int64_t bound = 1 + (int64_t)p->max_imf * (p->max_sifts + 1);
    const int chunk = (p->tau > 0.0) ? 8 : (int)std::min<int64_t>(bound, 1 << 30);
    int64_t done = 0;
    while (done < bound) {
        const int k = (int)std::min<int64_t>(chunk, bound - done);
        int rc = p->exact ? launch_steps<T, true>(C, L, k, st, tr) : launch_steps<T, false>(C, L, k, st, tr);
        if (rc) return rc;
        done += k;
        if (done < bound) {
            // a cheap plan tells how many tasks are still alive
            tr.begin(EEMD_K_PLAN);
            k_plan<<<1, PLAN_THREADS, 0, st>>>(C);
            tr.end();
            Header h;
            if (cudaMemcpyAsync(&h, C.hdr, sizeof(Header), cudaMemcpyDeviceToHost, st) != cudaSuccess)
                return EEMD_E_CUDA;
            if (cudaStreamSynchronize(st) != cudaSuccess) return EEMD_E_CUDA;
            if (h.error) break;
            if (h.active == 0) break;
        }
    }
    if (imf_sum || mode_count) {
        int64_t nmax = 0;
        for (auto& s : L.sd) nmax = std::max<int64_t>(nmax, s.n);
        dim3 g((unsigned)((nmax + 255) / 256), (unsigned)p->max_imf, (unsigned)L.sd.size());
        tr.begin(EEMD_K_REDUCE);
        k_reduce<T><<<g, 256, 0, st>>>(C, imf_sum, mode_count);
        tr.end();
    }
    if (nsift || nmode || flags) {
        tr.begin(EEMD_K_OUTPUTS);
        k_outputs<<<(int)((n_tasks + 255) / 256), 256, 0, st>>>(C, nsift, nmode, flags);
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
    C.ts = reinterpret_cast<TaskState*>(base + L.o_ts);
    C.sd = reinterpret_cast<const SignalDesc*>(base + L.o_sd);
    C.sigma = reinterpret_cast<const double*>(base + L.o_sigma);
    C.el_task = reinterpret_cast<int32_t*>(base + L.o_el_task);
    C.el_pref = reinterpret_cast<int32_t*>(base + L.o_el_pref);
    C.sl_item = reinterpret_cast<int32_t*>(base + L.o_sl_item);
    C.sl_pref = reinterpret_cast<int32_t*>(base + L.o_sl_pref);
    C.status = reinterpret_cast<unsigned long long*>(base + L.o_status);
    C.partial = reinterpret_cast<double2*>(base + L.o_partial);
    C.tpref = reinterpret_cast<int2*>(base + L.o_tpref);
    C.hedge = reinterpret_cast<double2*>(base + L.o_hedge);
    C.redge = reinterpret_cast<double2*>(base + L.o_redge);
    C.resid = base + L.o_resid;
    C.imfs = imfs ? imfs : (void*)(base + L.o_imfs);
    C.kt = reinterpret_cast<int32_t*>(base + L.o_kt);
    C.ky = base + L.o_ky;
    C.M = reinterpret_cast<double*>(base + L.o_M);
    C.scr = reinterpret_cast<double2*>(base + L.o_scr);
    C.x = x;
    C.noise = noise;
    C.knot_log = knot_log;
    C.mode_sifts = mode_sifts;
    C.TT = L.TT;
    C.KC = L.KC;
    C.n_tasks = (int32_t)L.td.size();
    C.n_signals = n_signals;
    C.trial_count = trial_count;
    C.max_sifts = p->max_sifts;
    C.max_imf = p->max_imf;
    C.min_extrema = p->min_extrema;
    C.end_mode = p->end_mode;
    C.rules = p->rules;
    C.noise_mode = p->noise_mode;
    C.tile = L.tile;
    C.B = L.B;
    C.S = L.S;
    C.tau = p->tau;
    C.seed = p->seed;
    C.watchdog = p->watchdog != 0 ? p->watchdog : (1LL << 24);

    // tables and zeroed control state
    if (cudaMemsetAsync(base + L.o_hdr, 0, sizeof(Header), st) != cudaSuccess) return EEMD_E_CUDA;
    if (cudaMemsetAsync(base + L.o_status, 0, sizeof(unsigned long long) * 2 * L.TT, st) != cudaSuccess)
        return EEMD_E_CUDA;
    if (cudaMemcpyAsync(base + L.o_td, L.td.data(), sizeof(TaskDesc) * L.td.size(), cudaMemcpyHostToDevice,
                        st) != cudaSuccess)
        return EEMD_E_CUDA;
    if (cudaMemcpyAsync(base + L.o_sd, L.sd.data(), sizeof(SignalDesc) * L.sd.size(),
                        cudaMemcpyHostToDevice, st) != cudaSuccess)
        return EEMD_E_CUDA;
    // pageable-host copies above are staged before returning; keep L alive to the sync below anyway
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
    return EEMD_OK;
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
