// eemd_internal.cuh -- device-side structures of the EEMD engine.
//
// Work model.  A *task* is one (signal, trial) pair: the full EMD of one
// perturbed signal (emd_ref.py:108-156 emd_1d; emd_gpu.py:120-285 runs the
// same loop with one CUDA block per trial).  Here every task advances by one
// *step* per round of three launches:
//
//   k_plan   one CTA: list the live tasks, their tiles and their solve chunks
//   k_solve  decay-seamed block-Thomas solve of both envelope systems of
//            every task that is sifting (emd_ref.py:31-65, emd_gpu_v5_dsbt.py:51-74)
//   k_eval   fused pass over the task's samples, one tile per CTA: spline
//            evaluation of both envelopes, mean subtraction, SD partial sums,
//            extrema detection + compaction of the *next* sift's knots
//            (decoupled look-back across the tiles of the task), IMF store,
//            residual update and the per-task stop decision (last tile done)
//
// A task's step is one of: INIT (noise injection + first extrema scan),
// SIFT (one sift; the last allowed sift of an IMF also closes the IMF),
// TRANS (close an IMF that stopped on the SD rule or on missing extrema).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace eemd {

enum Phase : int32_t { PH_DONE = 0, PH_INIT = 1, PH_SIFT = 2, PH_TRANS = 3 };

// status word of the decoupled look-back: [63:62] flag, [61:31] maxima, [30:0] minima
enum : uint64_t { LB_EMPTY = 0, LB_AGG = 1, LB_INC = 2 };

constexpr int EVAL_THREADS = 256;
constexpr int SOLVE_THREADS = 128;
constexpr int PLAN_THREADS = 1024;

struct Header {
    int32_t error;        // first EEMD_E_* raised on the device (0 = none)
    int32_t error_info;   // task index / detail of the first error
    int32_t active;       // tasks not DONE after the last plan
    int32_t step;         // plan counter (parity selects the look-back plane)
    uint32_t eval_ticket;
    uint32_t solve_ticket;
    int32_t eval_total;   // tiles to process this step
    int32_t solve_total;  // solve chunks this step
    int32_t n_elist;
    int32_t n_slist;
    int32_t pad[6];
};

struct TaskDesc {
    int64_t x_off;      // element offset of the task's source signal in x
    int64_t s_off;      // element offset in the residual array (and resid_out)
    int64_t imf_off;    // element offset of IMF slot 0 (slot m at + m*n)
    int64_t k_off;      // offset in each knot plane (capacity kcap)
    int64_t scr_off;    // double2 offset of the solve scratch, env 0
    int64_t scr_env;    // double2 size of one env's scratch
    int64_t noise_off;  // element offset in the injected noise array
    int32_t n;          // samples
    int32_t kcap;       // knot capacity per envelope (incl. 2 mirror knots)
    int32_t tile_off;   // offset in the per-tile arrays
    int32_t ntiles;
    int32_t signal;
    int32_t trial;      // absolute trial index (Philox counter)
};

struct TaskState {
    int32_t phase;
    int32_t imf;            // index of the IMF being built
    int32_t sift;           // index of the next sift of that IMF
    int32_t kpar;           // knot/prefix plane holding the current knots
    int32_t pmax, pmin;     // current knot counts (knots of the pending sift)
    int32_t src_resid;      // the pending sift reads h from the residual
    int32_t imf_from_resid; // pending TRANS: the IMF is the residual itself (0 sifts)
    int32_t nsift_total;
    int32_t nmode;
    int32_t mode_sifts_cur;
    int32_t flags;          // bit0: IMF slots exhausted while extrema remained
    uint32_t done_count;    // tiles of this step finished (last one finalises)
    int32_t pad[3];
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
    TaskState* ts;
    const SignalDesc* sd;
    const double* sigma;          // per signal: eps*std(x) (Philox noise scale)
    int32_t* el_task;             // eval list: task
    int32_t* el_pref;             // eval list: tile prefix (n_elist+1)
    int32_t* sl_item;             // solve list: task*2+env
    int32_t* sl_pref;             // solve list: chunk prefix
    unsigned long long* status;   // [2][TT] look-back words
    double2* partial;             // [TT] (num, den)
    int2* tpref;                  // [2][TT] knots before the tile (max, min)
    double2* hedge;               // [2][TT] h at the tile's first/last sample
    double2* redge;               // [2][TT] residual at the tile's first/last sample
    void* resid;                  // residual per task (dtype)
    void* imfs;                   // IMF slots per task (dtype)
    int32_t* kt;                  // [2 parity][2 env][KC] knot sample index
    void* ky;                     // [2 parity][2 env][KC] knot value (dtype)
    double* M;                    // [2 env][KC] spline second derivatives (mirror space)
    double2* scr;                 // solve scratch (c, d') per window row
    const void* x;
    const void* noise;
    int32_t* knot_log;            // optional [task][max_imf][max_sifts][2]
    int32_t* mode_sifts;          // optional [task][max_imf]
    int64_t TT;                   // total tiles
    int64_t KC;                   // knot plane size
    int32_t n_tasks, n_signals, trial_count;
    int32_t max_sifts, max_imf, min_extrema, end_mode, rules, noise_mode;
    int32_t tile, B, S;
    double tau;
    uint64_t seed;
    long long watchdog;
};

}  // namespace eemd
