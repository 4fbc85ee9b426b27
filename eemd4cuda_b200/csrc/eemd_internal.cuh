// eemd_internal.cuh -- device-side structures of the EEMD engine.
//
// Work model.  A *task* is one (signal, trial) pair: the full EMD of one
// perturbed signal (emd_ref.py:108-156 emd_1d; emd_gpu.py:120-285 runs the
// same loop with one CUDA block per trial).  Tasks are independent, so the
// whole ensemble runs as ONE persistent kernel (k_emd): a thread-block cluster
// of C CTAs takes a task from a queue and carries it through every IMF and
// every sift before taking the next one.  CTA r of the cluster owns the
// contiguous sample segment [r*seg, (r+1)*seg).  Per sift:
//
//   solve   both envelope systems, decay-seamed block Thomas: the windows of
//           each envelope are split over the cluster's CTAs; knots are staged
//           in shared memory; second derivatives go to global memory
//           (emd_ref.py:31-65, emd_gpu_v5_dsbt.py:51-74)
//   barrier.cluster (release/acquire)
//   sweep   each CTA streams its segment tile by tile: spline evaluation of
//           both envelopes, mean subtraction, SD partial sums, strict extrema
//           of the new values compacted in time order into the segment's own
//           knot list (no cross-CTA prefix is needed: a knot index is the
//           segment prefix plus the position in the segment list), IMF store,
//           residual update
//   publish segment results (counts, SD partials, edge samples) in shared
//           memory; barrier.cluster; every CTA reads all C entries through
//           distributed shared memory and takes the same stop decision
//
// Knot lists, second derivatives and solve scratch live in per-cluster-slot
// regions of the workspace; residuals and IMFs live per task.
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace eemd {

// warps per CTA of k_emd: 4 (the default) or 5, chosen per launch (the
// autotune table's choice per length bucket).  CTAs per SM (the launch
// bound, and with it the registers per thread): float32 storage 4 CTAs of 4
// warps or 3 of 5 (128 registers); float64 storage 3 CTAs of either (168
// registers for 4 warps: at 4 CTAs the float64 build spilled 200 bytes per
// thread)
constexpr int NW_DEFAULT = 4;
constexpr int MAXNW = 5;
__host__ __device__ constexpr int ctas_per_sm(int nw, int bt) { return bt == 8 ? 3 : 16 / nw; }
// largest cluster: portable clusters reach 8 CTAs; 9 to 16 are non-portable
// and are taken only when the device reports that all of them fit at once
constexpr int MAXC = 16;
// owned rows per lane of the fast solve: the forward (c, d) of a pass's rows
// live in shared memory, so the width costs no registers; odd widths keep the
// lanes' strided shared-memory accesses free of bank conflicts
#ifndef EEMD_FAST_B
#define EEMD_FAST_B 5
#endif
constexpr int FAST_B = EEMD_FAST_B;
// warp tiles of samples in flight per sweep warp (a ring of buffers: the
// copies of the next TILE_BUFS - 1 tiles run while one tile is processed)
#ifndef EEMD_TILE_BUFS
#define EEMD_TILE_BUFS 2
#endif
constexpr int TILE_BUFS = EEMD_TILE_BUFS;
static_assert(TILE_BUFS >= 2 && TILE_BUFS <= 4, "two to four tile buffers");
#ifndef EEMD_WSCAP
#define EEMD_WSCAP 352
#endif
constexpr int WSCAP = EEMD_WSCAP;  // knots staged in shared memory per warp and solve pass

enum Phase : int32_t { PH_DONE = 0, PH_INIT = 1, PH_SIFT = 2, PH_TRANS = 3 };
enum TileMode : int32_t { TM_INIT = 0, TM_SIFT = 1, TM_LAST = 2, TM_TRANS = 3 };

struct Header {
    int32_t error;        // first EEMD_E_* raised on the device (0 = none)
    int32_t error_info;   // task index / detail of the first error
    int32_t next_task;    // work queue head (index into the task order)
    int32_t n_done;       // tasks finished
    int32_t wd_flag;      // the watchdog test mode waits on this word; nothing sets it
    int32_t pad[11];
    // -DEEMD_TRACE builds: SM cycles spent per phase, summed over CTAs
    // (0 setup, 1 solve, 2 barrier after solve, 3 sweep, 4 barrier after sweep, 5 decide, 6 claim)
    unsigned long long phase_cycles[8];
    // sweep sub-phases (lane 0 of each warp): 0 tile wait, 1 values, 2 extrema +
    // warp scan, 3 writes; solve sub-phases (lane 0 of each warp): 4 knot
    // staging, 5 slopes, 6 windows
    unsigned long long sweep_cycles[8];
};

struct TaskDesc {
    int64_t x_off;      // element offset of the task's source signal in x
    int64_t s_off;      // element offset in the residual array (and resid_out)
    int64_t imf_off;    // element offset of IMF slot 0 (slot m at + m*n)
    int64_t noise_off;  // element offset in the injected noise array
    int32_t n;          // samples
    int32_t signal;
    int32_t trial;      // absolute trial index (Philox counter)
    int32_t seg;        // samples per segment (multiple of 32)
};

struct TaskOut {
    int32_t nsift, nmode, flags, pad;
};

struct SignalDesc {
    int64_t x_off;     // element offset in x
    int64_t sum_off;   // element offset in imf_sum / imf_mean ([max_imf][n])
    int64_t r_off;     // element offset in the residual output
    int32_t n;
    int32_t first_task;
};

// Everything a kernel needs, passed by value.
struct Ctx {
    Header* hdr;
    const TaskDesc* td;
    const int32_t* order;         // task processing order (longest first)
    TaskOut* tout;
    const SignalDesc* sd;
    const double* sigma;          // per signal: eps*std(x) (Philox noise scale)
    void* resid;                  // residual per task (dtype)
    void* imfs;                   // IMF slots per task (dtype)
    int32_t* kt;                  // per slot: [2 parity][2 env][C seg][segcap] knot sample index
    void* ky;                     // per slot: same layout, knot value (dtype)
    void* M;                      // per slot: [2 env][5][kcap] interval records (mirror space,
                                  //   storage type): plane 0 = t_k; fast: monomial c0..c3 of
                                  //   interval [k, k+1]; exact: y_k, M_k
    void* w1;                     // per slot: scratch h buffer [slot_n] (storage type)
    void* r1;                     // per slot: second residual buffer [slot_n] (storage type)
    int4* ri;                     // per slot: run records [2 parity][slot_runs]
    double2* scr;                 // exact-mode solve scratch: [rows][grid threads]
    const void* x;
    const void* noise;
    int32_t* knot_log;            // optional [task][max_imf][max_sifts][2]
    int32_t* mode_sifts;          // optional [task][max_imf]
    int64_t slot_knots;           // kt/ky elements per slot
    int64_t slot_M;               // record elements per slot
    int64_t slot_n;               // w1 / r1 elements per slot
    int64_t slot_runs;            // run records per slot and parity
    int32_t segcap;               // knots of one kind per segment list
    int32_t kcap;                 // knots per envelope in mirror space (M plane size)
    int32_t n_tasks, n_signals, trial_count, csize;
    int32_t max_sifts, max_imf, min_extrema, end_mode, rules, noise_mode;
    int32_t B, S, scr_rows;
    int32_t nw;                   // warps per CTA of this launch
    double tau;
    double noise_scale;           // EEMD_NOISE_SCALED: the factor on noise[task][n]
    uint64_t seed;
    long long watchdog;
};

}  // namespace eemd
