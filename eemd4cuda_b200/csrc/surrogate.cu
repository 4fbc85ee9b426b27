// surrogate.cu -- kernels of the learned ensemble surrogate (sm_100a).
//
// The surrogate maps the 8-trial ensemble-mean IMFs of a signal to its
// 256-trial ensemble mean with a dilated 1-D convolution network (8 layers,
// 64 channels, kernel 3, dilations 1..128; bfloat16 weights and activations,
// float32 accumulation).  Activations are channels-last, [batch][time][C]
// with C = 16 (10 IMF channels, zero padded) or 64.
//
// Every convolution is an implicit GEMM on the 5th-generation tensor cores
// (four forms: k_conv_tc, single-buffered with cp.async staging; k_conv_tc2,
// double-buffered; k_conv_tma, double-buffered with bulk-tensor loads;
// k_conv_ws, warp-specialised with swizzled operands and bulk-tensor loads
// and stores):
//     D[t][n] = sum_{tap, c} X[t + dir*(tap-1)*dil][c] * W[n][tap*Cin + c]
// with M = 128 time samples per tile, N = the output channels and
// K = 3*Cin.  The CTA stages the three shifted copies of its input tile
// (zero-filled outside [0, T)) and the packed weights in shared memory in the
// canonical K-major core-matrix layout (8 rows x 16 bytes per core matrix, no
// swizzle), one elected thread issues tcgen05.mma (kind::f16, bf16 inputs,
// f32 accumulator in tensor memory), tcgen05.commit signals an mbarrier, and
// the four warps read the accumulator back with tcgen05.ld (warp w owns TMEM
// lanes 32w..32w+31, i.e. 32 time samples) for the epilogue (bias, ReLU or a
// ReLU-derivative mask, bf16 store).  dir = +1 is the forward convolution;
// dir = -1 with transposed weights is the gradient with respect to the input.
//
// The weight gradient is an implicit GEMM over time on tcgen05 too
// (k_wgrad_tc; k_wgrad is its CUDA-core form); the loss, Adam and the packing
// kernels run on CUDA cores.  A plain CUDA-core convolution with the same
// arguments is kept for checking the tensor-core path on the GPU.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/eemd_surrogate.h"

namespace sg {

constexpr int TM = 128;   // time samples per tile (MMA M)
constexpr int NT = 128;   // threads per CTA (4 warps)

__device__ __forceinline__ void raise(int* err, int code) {
    if (err) atomicCAS(err, 0, code);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// 16-byte asynchronous copy; src_bytes = 0 fills the destination with zeros
__device__ __forceinline__ void cp16(void* dst, const void* src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// shared-memory matrix descriptor, K-major, no swizzle (canonical layout
// ((8,n),2):((1,SBO),LBO) in 16-byte units), Blackwell version field = 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: bf16 x bf16 -> f32, both K-major, M x N
__host__ __device__ constexpr uint32_t instr_desc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// element offset of (row, k) in a K-major no-swizzle tile with `rows` rows:
// core matrices of 8 rows x 8 k; k-chunks of 8 at stride rows*8 elements
__host__ __device__ __forceinline__ int kmaj_off(int row, int k, int rows) {
    return (k >> 3) * (rows * 8) + (row >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[N]);

template <>
__device__ __forceinline__ void tmem_ld<16>(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void tmem_ld<64>(uint32_t taddr, float (&v)[64]) {
    // four 16-column loads keep the asm operand lists short
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t r[16];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
            "[%16];\n"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
              "=r"(r[15])
            : "r"(taddr + 16u * q));
#pragma unroll
        for (int i = 0; i < 16; ++i) v[16 * q + i] = __uint_as_float(r[i]);
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// Tensor-core convolution (see the file header).  One CTA keeps the packed
// weights in shared memory and walks tiles of 128 time samples.
template <int CIN, int COUT>
__global__ void __launch_bounds__(NT) k_conv_tc(const __nv_bfloat16* __restrict__ in,
                                                const __nv_bfloat16* __restrict__ wpk,
                                                const float* __restrict__ bias, __nv_bfloat16* out, int B,
                                                int T, int dil, int dir, int relu,
                                                const __nv_bfloat16* __restrict__ mask, int* err,
                                                long long spin_limit) {
    constexpr int K = 3 * CIN;
    constexpr int KSTEPS = K / 16;
    constexpr int A_BYTES = K * TM * 2;
    constexpr int B_BYTES = K * COUT * 2;
    constexpr int TCOLS = COUT < 32 ? 32 : COUT;
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && COUT <= 256, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sB = reinterpret_cast<__nv_bfloat16*>(smem + A_BYTES);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ float sbias[COUT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < COUT; i += NT) sbias[i] = bias ? bias[i] : 0.f;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // packed weights: a flat copy of the K-major B-tile image
    for (int i = tid; i < B_BYTES / 16; i += NT) cp16(reinterpret_cast<char*>(sB) + 16 * i, wpk + 8 * i, 16);
    cp_commit();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
    constexpr uint32_t IDESC = instr_desc(TM, COUT);
    const int tiles_per_b = (T + TM - 1) / TM;
    const int n_tiles = B * tiles_per_b;
    uint32_t phase = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * TM;
        const __nv_bfloat16* inb = in + (size_t)b * T * CIN;
        // im2col of the tile: row r, k = tap*CIN + c <- in[t0 + r + dir*(tap-1)*dil][c]
        for (int i = tid; i < 3 * TM * (CIN / 8); i += NT) {
            const int chunk = i % (CIN / 8);
            const int r = (i / (CIN / 8)) % TM;
            const int tap = i / ((CIN / 8) * TM);
            const int ts = t0 + r + dir * (tap - 1) * dil;
            const bool ok = (ts >= 0 && ts < T);
            const int k = tap * CIN + chunk * 8;
            cp16(sA + kmaj_off(r, k, TM), ok ? (const void*)(inb + (size_t)ts * CIN + chunk * 8) : (const void*)inb,
                 ok ? 16 : 0);
        }
        cp_commit();
        cp_wait_all();
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
            for (int s = 0; s < KSTEPS; ++s) {
                const uint64_t da = smem_desc(a_base + s * 2 * (TM * 16), TM * 16, 128);
                const uint64_t db = smem_desc(b_base + s * 2 * (COUT * 16), COUT * 16, 128);
                const uint32_t acc = s > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(IDESC), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        // wait for the accumulator (bounded)
        {
            long long spins = 0;
            uint32_t done = 0;
            while (!done) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.u32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_u32(&mbar)), "r"(phase)
                    : "memory");
                if (!done && ++spins > spin_limit) {
                    raise(err, EEMD_SG_E_TIMEOUT);
                    failed = true;
                    break;
                }
            }
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (__syncthreads_or(failed ? 1 : 0)) break;
        float v[COUT];
        tmem_ld<COUT>(tmem + ((uint32_t)(32 * warp) << 16), v);
        const int t = t0 + 32 * warp + lane;
        if (t < T) {
            __nv_bfloat16* o = out + ((size_t)b * T + t) * COUT;
            const __nv_bfloat16* mk = mask ? mask + ((size_t)b * T + t) * COUT : nullptr;
#pragma unroll
            for (int c0 = 0; c0 < COUT; c0 += 8) {
                __align__(16) __nv_bfloat16 h[8];
                uint4 mv = make_uint4(0, 0, 0, 0);
                if (mk) mv = *reinterpret_cast<const uint4*>(mk + c0);
                const __nv_bfloat16* mh = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float x = v[c0 + i] + sbias[c0 + i];
                    if (relu) x = fmaxf(x, 0.f);
                    if (mk && !(__bfloat162float(mh[i]) > 0.f)) x = 0.f;
                    h[i] = __float2bfloat16(x);
                }
                *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(h);
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
}

// ---------------------------------------------------------------------------
// Double-buffered variant: two input-tile buffers and two accumulators in
// tensor memory.  Per tile k of this CTA: wait until MMA(k-1) is done (its
// accumulator is complete and its input buffer free), start the copies of
// tile k+1 into that buffer, wait for tile k's copies, issue MMA(k), then run
// the epilogue of tile k-1 while MMA(k) and the copies of tile k+1 proceed.
// ---------------------------------------------------------------------------
template <int CIN>
__device__ __forceinline__ void stage_tile(__nv_bfloat16* sA, const __nv_bfloat16* in, int tile, int tiles_per_b,
                                           int T, int dil, int dir, int tid) {
    const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * TM;
    const __nv_bfloat16* inb = in + (size_t)b * T * CIN;
    for (int i = tid; i < 3 * TM * (CIN / 8); i += NT) {
        const int chunk = i % (CIN / 8);
        const int r = (i / (CIN / 8)) % TM;
        const int tap = i / ((CIN / 8) * TM);
        const int ts = t0 + r + dir * (tap - 1) * dil;
        const bool ok = (ts >= 0 && ts < T);
        cp16(sA + kmaj_off(r, tap * CIN + chunk * 8, TM),
             ok ? (const void*)(inb + (size_t)ts * CIN + chunk * 8) : (const void*)inb, ok ? 16 : 0);
    }
}

// bounded wait for an mbarrier phase; false when it gave up
__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t phase, long long limit) {
    long long spins = 0;
    uint32_t done = 0;
    while (!done) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (!done && ++spins > limit) return false;
    }
    return true;
}

// columns [c0, c0 + NC) of this warp's 32 accumulator lanes (NC a multiple of 8)
template <int NC>
__device__ __forceinline__ void tmem_ld_cols(uint32_t taddr, float (&v)[NC]) {
    static_assert(NC % 8 == 0, "columns");
#pragma unroll
    for (int q = 0; q < NC / 8; ++q) {
        uint32_t r[8];
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];\n"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                       "=r"(r[7])
                     : "r"(taddr + 8u * q));
#pragma unroll
        for (int i = 0; i < 8; ++i) v[8 * q + i] = __uint_as_float(r[i]);
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// epilogue of a column slice: warp `warp` reads lane quadrant warp % 4 and
// columns [(warp / 4) * NC, +NC) of the accumulator at taddr
template <int COUT, int NC>
__device__ __forceinline__ void epilogue_cols(uint32_t taddr, const float* sbias, __nv_bfloat16* out,
                                              const __nv_bfloat16* __restrict__ mask, int tile, int tiles_per_b,
                                              int T, int relu, int warp, int lane) {
    const int quad = warp & 3, c_base = (warp >> 2) * NC;
    float v[NC];
    tmem_ld_cols<NC>(taddr + ((uint32_t)(32 * quad) << 16) + (uint32_t)c_base, v);
    const int b = tile / tiles_per_b, t = (tile % tiles_per_b) * TM + 32 * quad + lane;
    if (t >= T) return;
    __nv_bfloat16* o = out + ((size_t)b * T + t) * COUT + c_base;
    const __nv_bfloat16* mk = mask ? mask + ((size_t)b * T + t) * COUT + c_base : nullptr;
#pragma unroll
    for (int c0 = 0; c0 < NC; c0 += 8) {
        __align__(16) __nv_bfloat16 h[8];
        uint4 mv = make_uint4(0, 0, 0, 0);
        if (mk) mv = *reinterpret_cast<const uint4*>(mk + c0);
        const __nv_bfloat16* mh = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float x = v[c0 + i] + sbias[c_base + c0 + i];
            if (relu) x = fmaxf(x, 0.f);
            if (mk && !(__bfloat162float(mh[i]) > 0.f)) x = 0.f;
            h[i] = __float2bfloat16(x);
        }
        *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(h);
    }
}

template <int COUT>
__device__ __forceinline__ void epilogue(uint32_t taddr, const float* sbias, __nv_bfloat16* out,
                                         const __nv_bfloat16* __restrict__ mask, int tile, int tiles_per_b, int T,
                                         int relu, int warp, int lane) {
    float v[COUT];
    tmem_ld<COUT>(taddr + ((uint32_t)(32 * warp) << 16), v);
    const int b = tile / tiles_per_b, t = (tile % tiles_per_b) * TM + 32 * warp + lane;
    if (t >= T) return;
    __nv_bfloat16* o = out + ((size_t)b * T + t) * COUT;
    const __nv_bfloat16* mk = mask ? mask + ((size_t)b * T + t) * COUT : nullptr;
#pragma unroll
    for (int c0 = 0; c0 < COUT; c0 += 8) {
        __align__(16) __nv_bfloat16 h[8];
        uint4 mv = make_uint4(0, 0, 0, 0);
        if (mk) mv = *reinterpret_cast<const uint4*>(mk + c0);
        const __nv_bfloat16* mh = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float x = v[c0 + i] + sbias[c0 + i];
            if (relu) x = fmaxf(x, 0.f);
            if (mk && !(__bfloat162float(mh[i]) > 0.f)) x = 0.f;
            h[i] = __float2bfloat16(x);
        }
        *reinterpret_cast<uint4*>(o + c0) = *reinterpret_cast<const uint4*>(h);
    }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(NT) k_conv_tc2(const __nv_bfloat16* __restrict__ in,
                                                 const __nv_bfloat16* __restrict__ wpk,
                                                 const float* __restrict__ bias, __nv_bfloat16* out, int B, int T,
                                                 int dil, int dir, int relu, const __nv_bfloat16* __restrict__ mask,
                                                 int* err, long long spin_limit) {
    constexpr int K = 3 * CIN;
    constexpr int KSTEPS = K / 16;
    constexpr int A_BYTES = K * TM * 2;
    constexpr int B_BYTES = K * COUT * 2;
    constexpr int ACOLS = COUT < 32 ? 32 : COUT;  // columns of one accumulator
    constexpr int TCOLS = 2 * ACOLS;
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && TCOLS <= 512, "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sA0 = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sB = reinterpret_cast<__nv_bfloat16*>(smem + 2 * A_BYTES);
    __shared__ __align__(8) uint64_t mbar[2];
    __shared__ uint32_t tmem_slot;
    __shared__ float sbias[COUT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < COUT; i += NT) sbias[i] = bias ? bias[i] : 0.f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[0])));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar[1])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    const int tiles_per_b = (T + TM - 1) / TM;
    const int n_tiles = B * tiles_per_b;
    const int nk = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    // weights and the first tile: one copy group
    for (int i = tid; i < B_BYTES / 16; i += NT) cp16(reinterpret_cast<char*>(sB) + 16 * i, wpk + 8 * i, 16);
    if (nk > 0) stage_tile<CIN>(sA0, in, blockIdx.x, tiles_per_b, T, dil, dir, tid);
    cp_commit();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t a_base = smem_u32(sA0), b_base = smem_u32(sB);
    constexpr uint32_t IDESC = instr_desc(TM, COUT);
    uint32_t phase[2] = {0u, 0u};
    bool failed = false;
    for (int k = 0; k < nk; ++k) {
        const int buf = k & 1;
        if (k >= 1) {
            // MMA(k-1): its accumulator complete, its input buffer free
            if (!wait_parity(&mbar[buf ^ 1], phase[buf ^ 1], spin_limit)) failed = true;
            phase[buf ^ 1] ^= 1u;
        }
        if (__syncthreads_or(failed ? 1 : 0)) {
            if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
            break;
        }
        if (k + 1 < nk)
            stage_tile<CIN>(reinterpret_cast<__nv_bfloat16*>(smem + (buf ^ 1) * A_BYTES), in,
                            blockIdx.x + (k + 1) * gridDim.x, tiles_per_b, T, dil, dir, tid);
        cp_commit();
        asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // tile k's copies (and the weights) landed
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t a_buf = a_base + buf * A_BYTES;
#pragma unroll
            for (int s2 = 0; s2 < KSTEPS; ++s2) {
                const uint64_t da = smem_desc(a_buf + s2 * 2 * (TM * 16), TM * 16, 128);
                const uint64_t db = smem_desc(b_base + s2 * 2 * (COUT * 16), COUT * 16, 128);
                const uint32_t acc = s2 > 0 ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + buf * ACOLS),
                    "l"(da), "l"(db), "r"(IDESC), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar[buf]))
                         : "memory");
        }
        if (k >= 1) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue<COUT>(tmem + (buf ^ 1) * ACOLS, sbias, out, mask, blockIdx.x + (k - 1) * gridDim.x,
                           tiles_per_b, T, relu, warp, lane);
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    }
    if (nk > 0 && !failed) {
        const int last = (nk - 1) & 1;
        const bool ok = wait_parity(&mbar[last], phase[last], spin_limit);
        if (__syncthreads_or(ok ? 0 : 1)) {
            if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue<COUT>(tmem + last * ACOLS, sbias, out, mask, blockIdx.x + (nk - 1) * gridDim.x, tiles_per_b, T,
                           relu, warp, lane);
        }
    }
    cp_wait_all();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
}

// ---------------------------------------------------------------------------
// TMA-fed variant.  The input is a 3-D tensor map [B][T][CIN] (bf16, box
// {8 channels, 128 samples, 1}); one tile's A operand is 3*CIN/8 boxes, each
// exactly one K-chunk column of the K-major no-swizzle layout (128 rows x
// 16 bytes), issued by one thread with cp.async.bulk.tensor and counted on a
// transaction mbarrier.  Rows outside [0, T) of the signal are zero-filled by
// the tensor map's bounds (the channel coordinate is a multiple of 8, so every
// box starts on a 16-byte boundary).  Pipeline: TMA_STAGES input buffers
// (tiles k+1 .. k+TMA_STAGES-1 in flight while tile k is multiplied), two
// tensor-memory accumulators, the epilogue of tile k-1 overlapping MMA k.
// No multicast.
// ---------------------------------------------------------------------------
// input-tile buffers of k_conv_tma (tiles in flight while one is multiplied);
// 3 measured no faster than 2 (1.364 vs 1.349 ms for the 8-layer pass over
// 16 x 65536 samples): the copies are not what each tile waits for
#ifndef EEMD_SG_TMA_STAGES
#define EEMD_SG_TMA_STAGES 2
#endif
constexpr int TMA_STAGES = EEMD_SG_TMA_STAGES;
// warps of k_conv_tma: 4 (one per accumulator lane quadrant) or 8 (two per
// quadrant, each reading half the columns in the epilogue)
#ifndef EEMD_SG_TMA_EPI_WARPS
#define EEMD_SG_TMA_EPI_WARPS 8
#endif
constexpr int TMA_EPI_WARPS = EEMD_SG_TMA_EPI_WARPS;

template <int CIN>
__device__ __forceinline__ void tma_tile(const CUtensorMap* tmap, uint32_t dst, uint64_t* full, int tile,
                                         int tiles_per_b, int dil, int dir) {
    constexpr uint32_t BYTES = 3u * CIN * TM * 2u;
    const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * TM;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(full)), "r"(BYTES)
                 : "memory");
#pragma unroll
    for (int tap = 0; tap < 3; ++tap) {
        const int ts = t0 + dir * (tap - 1) * dil;
#pragma unroll
        for (int kc = 0; kc < CIN / 8; ++kc) {
            const uint32_t d = dst + (uint32_t)((tap * (CIN / 8) + kc) * TM * 16);
            asm volatile(
                "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                "[%5];\n" ::"r"(d),
                "l"(reinterpret_cast<uint64_t>(tmap)), "r"(kc * 8), "r"(ts), "r"(b), "r"(smem_u32(full))
                : "memory");
        }
    }
}

template <int CIN, int COUT, int EW>
__global__ void __launch_bounds__(32 * EW) k_conv_tma(const __grid_constant__ CUtensorMap tmap,
                                                 const __nv_bfloat16* __restrict__ wpk,
                                                 const float* __restrict__ bias, __nv_bfloat16* out, int B, int T,
                                                 int dil, int dir, int relu, const __nv_bfloat16* __restrict__ mask,
                                                 int* err, long long spin_limit) {
    constexpr int K = 3 * CIN;
    constexpr int KSTEPS = K / 16;
    constexpr int A_BYTES = K * TM * 2;
    constexpr int B_BYTES = K * COUT * 2;
    constexpr int NBUF = TMA_STAGES;              // input tiles in flight + the one being multiplied
    constexpr int ACOLS = COUT < 32 ? 32 : COUT;
    constexpr int TCOLS = 2 * ACOLS;
    constexpr int THR = 32 * EW;                  // EW = 4: one warp per lane quadrant; 8: two, each half the columns
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && TCOLS <= 512 && (EW == 4 || EW == 8), "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t full[NBUF];
    __shared__ __align__(8) uint64_t mmad[2];
    __shared__ uint32_t tmem_slot;
    __shared__ float sbias[COUT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    for (int i = tid; i < COUT; i += THR) sbias[i] = bias ? bias[i] : 0.f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int i = 0; i < NBUF; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[i])));
        for (int i = 0; i < 2; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mmad[i])));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    const int tiles_per_b = (T + TM - 1) / TM;
    const int n_tiles = B * tiles_per_b;
    const uint32_t a_base = smem_u32(smem), b_base = a_base + NBUF * A_BYTES;
    // the bulk-tensor copies need 128-byte aligned destinations: refuse to run otherwise
    const bool aligned = (a_base & 127u) == 0;
    if (!aligned && tid == 0) raise(err, EEMD_SG_E_BADARG);
    const int nk = (aligned && blockIdx.x < n_tiles) ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    // the packed weights once (ordinary copies, then made visible to the async proxy)
    for (int i = tid; i < B_BYTES / 16; i += THR) cp16(smem + NBUF * A_BYTES + 16 * i, wpk + 8 * i, 16);
    cp_commit();
    cp_wait_all();
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    constexpr uint32_t IDESC = instr_desc(TM, COUT);
    // tiles 0 .. NBUF-2 in flight before the loop
    if (tid == 0)
        for (int j = 0; j < NBUF - 1 && j < nk; ++j)
            tma_tile<CIN>(&tmap, a_base + j * A_BYTES, &full[j], blockIdx.x + j * gridDim.x, tiles_per_b, dil, dir);
    uint32_t fph[NBUF], mph[2] = {0u, 0u};
#pragma unroll
    for (int i = 0; i < NBUF; ++i) fph[i] = 0u;
    bool failed = false;
    int ib = 0;  // input buffer of tile k (k mod NBUF)
    for (int k = 0; k < nk; ++k) {
        const int acc_b = k & 1;
        if (k >= 1) {
            // MMA(k-1): its accumulator complete, its input buffer free
            if (!wait_parity(&mmad[acc_b ^ 1], mph[acc_b ^ 1], spin_limit)) failed = true;
            mph[acc_b ^ 1] ^= 1u;
        }
        if (__syncthreads_or(failed ? 1 : 0)) {
            if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
            break;
        }
        if (tid == 0) {
            // tile k+NBUF-1 into the buffer MMA(k-1) used (the last free one)
            const int kn = k + NBUF - 1;
            if (kn < nk) {
                const int nb = ib == 0 ? NBUF - 1 : ib - 1;
                tma_tile<CIN>(&tmap, a_base + nb * A_BYTES, &full[nb], blockIdx.x + kn * gridDim.x, tiles_per_b,
                              dil, dir);
            }
            uint32_t ph = 0;
#pragma unroll
            for (int i = 0; i < NBUF; ++i)
                if (i == ib) ph = fph[i];
            if (!wait_parity(&full[ib], ph, spin_limit)) {
                failed = true;
            } else {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t a_buf = a_base + ib * A_BYTES;
#pragma unroll
                for (int s2 = 0; s2 < KSTEPS; ++s2) {
                    const uint64_t da = smem_desc(a_buf + s2 * 2 * (TM * 16), TM * 16, 128);
                    const uint64_t db = smem_desc(b_base + s2 * 2 * (COUT * 16), COUT * 16, 128);
                    const uint32_t acc = s2 > 0 ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + acc_b * ACOLS),
                        "l"(da), "l"(db), "r"(IDESC), "r"(acc));
                }
                asm volatile(
                    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                        smem_u32(&mmad[acc_b]))
                    : "memory");
            }
#pragma unroll
            for (int i = 0; i < NBUF; ++i)
                if (i == ib) fph[i] ^= 1u;
        }
        __syncwarp();
        if (k >= 1) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue_cols<COUT, COUT * 4 / EW>(tmem + (acc_b ^ 1) * ACOLS, sbias, out, mask, blockIdx.x + (k - 1) * gridDim.x,
                           tiles_per_b, T, relu, warp, lane);
        }
        asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
        ib = ib + 1 == NBUF ? 0 : ib + 1;
    }
    if (__syncthreads_or(failed ? 1 : 0)) {
        if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
    } else if (nk > 0) {
        const int last = (nk - 1) & 1;
        const bool ok = wait_parity(&mmad[last], mph[last], spin_limit);
        if (__syncthreads_or(ok ? 0 : 1)) {
            if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
        } else {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            epilogue_cols<COUT, COUT * 4 / EW>(tmem + last * ACOLS, sbias, out, mask, blockIdx.x + (nk - 1) * gridDim.x, tiles_per_b, T,
                           relu, warp, lane);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
}

// ---------------------------------------------------------------------------
// Warp-specialised variant (tensor_cores = 4).  Every operand is in a
// swizzled K-major layout whose rows are one tap's CIN channels: 64 channels
// in the 128-byte swizzle (rows of 128 bytes, the 16-byte chunks of row r
// permuted by XOR with r mod 8, 8-row groups 1024 bytes apart), 16 channels
// in the 32-byte swizzle (rows of 32 bytes, chunk XOR (r / 4) mod 2, 8-row
// groups 256 bytes apart).  A tap of the input tile is ONE bulk-tensor box
// {CIN channels, 128 samples} written in that layout by the copy engine, so
// a tile takes 3 copies instead of 3 * CIN / 8 narrow ones, and the weights
// are re-laid into the same form in shared memory once per CTA.  The roles
// run concurrently on their own mbarriers:
//   copy warp  (lane 0): tile k into input stage k mod WS_STAGES once MMA
//                        k - WS_STAGES has released it (empty[s]);
//   MMA warp   (lane 0): waits full[s] and the accumulator's release
//                        (acce[k & 1]), issues the 3 * CIN / 16 MMAs of tile k into
//                        accumulator k & 1, commits to empty[s] and accf[k & 1];
//   8 epilogue warps   : read their lane quadrant x half the columns of the
//                        accumulator, release it, add bias / ReLU / mask,
//                        write the bf16 tile into a swizzled staging buffer,
//                        and one thread stores it with a bulk-tensor store
//                        (rows past T are clipped by the tensor map).
// The MMA's K order (tap-major, 16 channels per instruction) is the same as
// the other forms', so the results are bit-identical to theirs.  Every wait
// is bounded; a wait that gives up sets *err and every role leaves its loop.
// No multicast.
// ---------------------------------------------------------------------------
constexpr int WS_STAGES = 3;                    // input tiles in flight
constexpr int WS_EPI = 8;                       // epilogue warps
constexpr int WS_THREADS = 32 * (WS_EPI + 2);   // + the copy warp and the MMA warp

template <int CIN, int COUT>
struct WsGeo {
    static constexpr int ROWB = CIN * 2;                     // bytes of one operand row (one tap)
    static constexpr int SBO = 8 * ROWB;                     // 8-row group stride
    static constexpr uint64_t LAYOUT = CIN == 64 ? 2 : 6;    // descriptor swizzle: 128-byte / 32-byte
    static constexpr int TAP_BYTES = TM * ROWB;              // 128 rows of one tap
    static constexpr int A_BYTES = 3 * TAP_BYTES;            // one input stage
    static constexpr int B_TAP = COUT * ROWB;                // one tap of the weights
    static constexpr int B_BYTES = 3 * B_TAP;
    static constexpr int O_BYTES = TM * COUT * 2;            // one output tile
    static constexpr int SMEM = WS_STAGES * A_BYTES + B_BYTES + 2 * O_BYTES + 1024;  // + alignment slack
    // 16-byte chunk c of operand row r in the swizzled layout
    static __device__ __forceinline__ int chunk(int c, int r) { return CIN == 64 ? c ^ (r & 7) : c ^ ((r >> 2) & 1); }
};

// shared-memory descriptor of a K-major swizzled operand: 8-row groups sbo
// bytes apart; the leading offset is unused for these layouts
__device__ __forceinline__ uint64_t sw_desc(uint32_t addr, uint32_t sbo, uint64_t layout) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46) | (layout << 61);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// named barrier 1 over the epilogue warps, OR of v over their threads
__device__ __forceinline__ bool epi_bar_or(bool v) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\tbar.red.or.pred q, 1, %2, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "n"(32 * WS_EPI)
        : "memory");
    return r != 0;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(WS_THREADS, 1) k_conv_ws(const __grid_constant__ CUtensorMap tin,
                                                            const __grid_constant__ CUtensorMap tout,
                                                            const __nv_bfloat16* __restrict__ wpk,
                                                            const float* __restrict__ bias, int B, int T, int dil,
                                                            int dir, int relu,
                                                            const __nv_bfloat16* __restrict__ mask, int* err,
                                                            long long spin_limit) {
    using G = WsGeo<CIN, COUT>;
    constexpr int NS = WS_STAGES;
    constexpr int KC = CIN / 8;            // 16-byte chunks per operand row
    constexpr int ACOLS = COUT < 32 ? 32 : COUT;
    constexpr int TCOLS = 2 * ACOLS;
    constexpr int NC = COUT * 4 / WS_EPI;  // accumulator columns per epilogue warp
    constexpr uint32_t IDESC = instr_desc(TM, COUT);
    static_assert((CIN == 64 || CIN == 16) && (COUT == 64 || COUT == 16), "shape");
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[NS], empty[NS], accf[2], acce[2];
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ float sbias[COUT];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t a_base = (raw + 1023u) & ~1023u;  // swizzled operands need 1024-byte alignment
    unsigned char* const sm = smem_raw + (a_base - raw);
    const uint32_t b_base = a_base + NS * G::A_BYTES;
    const uint32_t o_base = b_base + G::B_BYTES;
    unsigned char* const so = sm + NS * G::A_BYTES + G::B_BYTES;
    for (int i = tid; i < COUT; i += WS_THREADS) sbias[i] = bias ? bias[i] : 0.f;
    // weights: the packed K-major image (8-element chunks (n, k8) at k8*COUT*8 + (n/8)*64 + (n%8)*8)
    // into swizzled rows: tap k8 / KC, row n, chunk k8 % KC
    for (int i = tid; i < COUT * 3 * KC; i += WS_THREADS) {
        const int n = i % COUT, k8 = i / COUT;
        const int tap = k8 / KC, c8 = k8 % KC;
        const uint4 v = *reinterpret_cast<const uint4*>(wpk + (size_t)k8 * COUT * 8 + (n >> 3) * 64 + (n & 7) * 8);
        *reinterpret_cast<uint4*>(sm + NS * G::A_BYTES + tap * G::B_TAP + (n >> 3) * G::SBO + (n & 7) * G::ROWB +
                                  (G::chunk(c8, n) << 4)) = v;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        for (int i = 0; i < NS; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&full[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&empty[i])));
        }
        for (int i = 0; i < 2; ++i) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&accf[i])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(&acce[i])), "n"(WS_EPI));
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // the weights, for the MMA
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const int tiles_per_b = (T + TM - 1) / TM;
    const int n_tiles = B * tiles_per_b;
    const int nk = blockIdx.x < n_tiles ? (n_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == WS_EPI) {
        // ---------------- copy warp ----------------
        if (lane == 0) {
            int k = 0;
            for (; k < nk && !abort_flag; ++k) {
                const int s = k % NS;
                if (k >= NS && !wait_parity(&empty[s], (uint32_t)((k / NS) - 1) & 1u, spin_limit)) {
                    raise(err, EEMD_SG_E_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                const int tile = blockIdx.x + k * gridDim.x;
                const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * TM;
                const uint32_t dst = a_base + s * G::A_BYTES;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(&full[s])),
                             "n"(G::A_BYTES)
                             : "memory");
#pragma unroll
                for (int tap = 0; tap < 3; ++tap)
                    asm volatile(
                        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], "
                        "[%1, {%2, %3, %4}], [%5];\n" ::"r"(dst + tap * G::TAP_BYTES),
                        "l"(reinterpret_cast<uint64_t>(&tin)), "r"(0), "r"(t0 + dir * (tap - 1) * dil), "r"(b),
                        "r"(smem_u32(&full[s]))
                        : "memory");
            }
            // copies still in flight (only when a role gave up) land before the CTA leaves
            for (int j = k - 1; j >= 0 && j >= k - NS; --j) wait_parity(&full[j % NS], (uint32_t)(j / NS) & 1u, spin_limit);
        }
    } else if (warp == WS_EPI + 1) {
        // ---------------- MMA warp ----------------
        if (lane == 0) {
            int k = 0;
            for (; k < nk && !abort_flag; ++k) {
                const int s = k % NS, a = k & 1;
                if (!wait_parity(&full[s], (uint32_t)(k / NS) & 1u, spin_limit) ||
                    (k >= 2 && !wait_parity(&acce[a], (uint32_t)((k >> 1) - 1) & 1u, spin_limit))) {
                    raise(err, EEMD_SG_E_TIMEOUT);
                    abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                const uint32_t a_buf = a_base + s * G::A_BYTES;
#pragma unroll
                for (int s2 = 0; s2 < 3 * CIN / 16; ++s2) {
                    const int tap = s2 / (CIN / 16), kk = s2 % (CIN / 16);
                    const uint64_t da = sw_desc(a_buf + tap * G::TAP_BYTES + kk * 32, G::SBO, G::LAYOUT);
                    const uint64_t db = sw_desc(b_base + tap * G::B_TAP + kk * 32, G::SBO, G::LAYOUT);
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + a * ACOLS),
                        "l"(da), "l"(db), "r"(IDESC), "r"(s2 > 0 ? 1u : 0u));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 smem_u32(&empty[s]))
                             : "memory");
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 smem_u32(&accf[a]))
                             : "memory");
            }
            // the issued MMAs are complete before the tensor memory is freed
            if (k > 0) wait_parity(&accf[(k - 1) & 1], (uint32_t)((k - 1) >> 1) & 1u, spin_limit);
        }
    } else {
        // ---------------- epilogue warps ----------------
        const int quad = warp & 3, cb = (warp >> 2) * NC;
        const int r = 32 * quad + lane;  // tile row of this lane
        for (int k = 0; k < nk; ++k) {
            const int a = k & 1;
            const int tile = blockIdx.x + k * gridDim.x;
            const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * TM;
            const bool ok = __all_sync(0xffffffffu, wait_parity(&accf[a], (uint32_t)(k >> 1) & 1u, spin_limit));
            if (ok) {
                asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
                float v[NC];
                tmem_ld_cols<NC>(tmem + a * ACOLS + ((uint32_t)(32 * quad) << 16) + (uint32_t)cb, v);
                asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&acce[a]);
                const int t = t0 + r;
                const __nv_bfloat16* mk = (mask && t < T) ? mask + ((size_t)b * T + t) * COUT + cb : nullptr;
                unsigned char* const ob = so + (k & 1) * G::O_BYTES;
#pragma unroll
                for (int j = 0; j < NC / 8; ++j) {
                    __align__(16) __nv_bfloat16 h[8];
                    uint4 mv = make_uint4(0, 0, 0, 0);
                    if (mk) mv = *reinterpret_cast<const uint4*>(mk + 8 * j);
                    const __nv_bfloat16* mh = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
                    for (int i = 0; i < 8; ++i) {
                        float x = v[8 * j + i] + sbias[cb + 8 * j + i];
                        if (relu) x = fmaxf(x, 0.f);
                        if (mask && !(__bfloat162float(mh[i]) > 0.f)) x = 0.f;
                        h[i] = __float2bfloat16(x);
                    }
                    const int c = (cb >> 3) + j;  // 16-byte chunk of the output row
                    const int off = COUT == 64 ? r * 128 + ((c ^ (r & 7)) << 4) : r * (COUT * 2) + (c << 4);
                    *reinterpret_cast<uint4*>(ob + off) = *reinterpret_cast<const uint4*>(h);
                }
                asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
            }
            // the stores issued so far (tile k-1's) have read their staging buffer
            // before tile k+1 overwrites it
            if (tid == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
            __syncwarp();
            if (epi_bar_or(!ok)) {
                if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
                abort_flag = 1;
                break;
            }
            if (tid == 0) {
                asm volatile(
                    "cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(
                        reinterpret_cast<uint64_t>(&tout)),
                    "r"(0), "r"(t0), "r"(b), "r"(o_base + (k & 1) * G::O_BYTES)
                    : "memory");
                asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
            }
        }
        if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    }
    __syncwarp();
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
}

// CUDA-core convolution with the same arguments (reference for the tensor-core path)
__global__ void k_conv_ref(const __nv_bfloat16* __restrict__ in, const __nv_bfloat16* __restrict__ wpk,
                           const float* __restrict__ bias, __nv_bfloat16* out, int B, int T, int cin, int cout,
                           int dil, int dir, int relu, const __nv_bfloat16* __restrict__ mask) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)B * T * cout) return;
    const int n = (int)(i % cout);
    const int t = (int)((i / cout) % T);
    const int b = (int)(i / ((long long)cout * T));
    float acc = 0.f;
    for (int tap = 0; tap < 3; ++tap) {
        const int ts = t + dir * (tap - 1) * dil;
        if (ts < 0 || ts >= T) continue;
        for (int c = 0; c < cin; ++c)
            acc += __bfloat162float(in[((size_t)b * T + ts) * cin + c]) *
                   __bfloat162float(wpk[kmaj_off(n, tap * cin + c, cout)]);
    }
    float x = acc + (bias ? bias[n] : 0.f);
    if (relu) x = fmaxf(x, 0.f);
    if (mask && !(__bfloat162float(mask[i]) > 0.f)) x = 0.f;
    out[i] = __float2bfloat16(x);
}

// Packs f32 weights into the bf16 K-major B-tile image of an (N rows) x (3*C)
// operand.  transpose = 0: w is [nv][3][cv] and row n, column tap*C + c holds
// w[n][tap][c]; transpose = 1: w is [cv][3][nv] and the same position holds
// w[c][tap][n] (the input-gradient operand).  Zero beyond nv, cv.  project = 1
// subtracts from every weight the mean over the output channels of the
// forward layer (n for transpose = 0, c for transpose = 1): the layer's
// outputs then sum to zero over those channels.
__global__ void k_pack(const float* __restrict__ w, __nv_bfloat16* wpk, int N, int C, int nv, int cv,
                       int transpose, int project) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * 3 * C) return;
    const int n = i / (3 * C), k = i % (3 * C);
    const int tap = k / C, c = k % C;
    const int o = transpose ? c : n, ii = transpose ? n : c;      // forward output / input channel
    const int ov = transpose ? cv : nv, iv = transpose ? nv : cv;
    float x = 0.f;
    if (n < nv && c < cv) {
        x = w[((size_t)o * 3 + tap) * iv + ii];
        if (project) {
            float s = 0.f;
            for (int q = 0; q < ov; ++q) s += w[((size_t)q * 3 + tap) * iv + ii];
            x -= s / (float)ov;
        }
    }
    wpk[kmaj_off(n, k, N)] = __float2bfloat16(x);
}

// bias[n] = b[n] (n < nv, minus the mean over nv when project), 0 up to N
__global__ void k_bias(const float* __restrict__ b, float* bias, int N, int nv, int project) {
    const int n = threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    if (project)
        for (int q = 0; q < nv; ++q) s += b[q];
    bias[n] = n < nv ? b[n] - s / (float)nv : 0.f;
}

// Weight and bias gradients of y[t][n] = b[n] + sum w[n][tap][c] x[t+(tap-1)d][c]
// from dy (bf16, [B][T][N]) and x (bf16, [B][T][C]); accumulates into f32
// dw[n][tap][c] (n < nv, c < cv) and db[n].  A CTA owns 64 time samples of one
// batch item and one tap, keeps the dy and x rows in shared memory and gives
// each thread an 8 x 4 block of (n, c).
__global__ void __launch_bounds__(NT) k_wgrad(const __nv_bfloat16* __restrict__ dy,
                                             const __nv_bfloat16* __restrict__ x, float* dw, float* db, int B,
                                             int T, int N, int C, int nv, int cv, int dil) {
    constexpr int R = 64;
    __shared__ float sdy[R][64 + 1];
    __shared__ float sx[R][64 + 1];
    const int tiles = (T + R - 1) / R;
    const int tap = blockIdx.y;
    const int b = blockIdx.x / tiles, t0 = (blockIdx.x % tiles) * R;
    const int tid = threadIdx.x;
    for (int i = tid; i < R * 64; i += NT) {
        const int r = i / 64, c = i % 64;
        const int t = t0 + r, ts = t + (tap - 1) * dil;
        sdy[r][c] = (t < T && c < N) ? __bfloat162float(dy[((size_t)b * T + t) * N + c]) : 0.f;
        sx[r][c] = (t < T && ts >= 0 && ts < T && c < C) ? __bfloat162float(x[((size_t)b * T + ts) * C + c]) : 0.f;
    }
    __syncthreads();
    // 64 x 64 (n, c) outputs: thread -> n block (8) x c block (4)
    const int nb = (tid / 16) * 8, cb = (tid % 16) * 4;
    float acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.f;
    for (int r = 0; r < R; ++r) {
        float a[8], xx[4];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = sdy[r][nb + i];
#pragma unroll
        for (int j = 0; j < 4; ++j) xx[j] = sx[r][cb + j];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], xx[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = nb + i, c = cb + j;
            if (n < nv && c < cv) atomicAdd(&dw[((size_t)n * 3 + tap) * cv + c], acc[i][j]);
        }
    if (tap == 1 && tid < 64 && tid < nv) {
        float s = 0.f;
        for (int r = 0; r < R; ++r) s += sdy[r][tid];
        atomicAdd(&db[tid], s);
    }
}

// Weight gradient on the tensor cores.  A GEMM with K = time: per tile of 128
// time samples of one batch row the CTA stages, in the K-major core-matrix
// layout of the forward kernel (8 rows x 16 bytes, no swizzle),
//   A_j[r][k] = x[b][t0 + k + (tap - 1) dil][c]   for row m = 128 j + r = tap C + c
//               (rows past 3C, and times outside [0, T), zero)
//   Bm[n][k]  = dy[b][t0 + k][n]
// with plain loads (the time-major image is a transpose of the channels-last
// tensors), and one thread issues tcgen05.mma kind::f16 (bf16 x bf16 -> f32,
// M = 128, N = NP, K = 16 per instruction) into NB accumulators D_j[m][n] in
// tensor memory that stay resident over all the CTA's tiles.  The epilogue
// reads them with tcgen05.ld and adds them to dw[n][tap][c] with atomics; db
// is summed from the staged dy on the CUDA cores.  Same operand shapes and
// descriptors as k_conv_tc (M = 128 rows, N = output channels).
template <int NB, int NP>
__global__ void __launch_bounds__(NT) k_wgrad_tc(const __nv_bfloat16* __restrict__ dy,
                                                 const __nv_bfloat16* __restrict__ x, float* dw, float* db,
                                                 int B, int T, int N, int C, int nv, int cv, int dil, int* err,
                                                 long long spin_limit) {
    constexpr int KT = 128;                  // time samples per tile (the GEMM's K)
    constexpr int A_BYTES = 128 * KT * 2;    // one M block
    constexpr int TCOLS = (NB * NP) <= 32 ? 32 : ((NB * NP) <= 64 ? 64 : 128);
    static_assert(NB >= 1 && NB <= 2 && (NP == 16 || NP == 64), "shape");
    extern __shared__ __align__(1024) unsigned char smem[];
    __nv_bfloat16* sA = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sB = reinterpret_cast<__nv_bfloat16*>(smem + NB * A_BYTES);
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ float sdb[NP];
    const int tid = threadIdx.x, warp = tid >> 5;
    if (tid < NP) sdb[tid] = 0.f;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const uint32_t tmem = tmem_slot;
    const uint32_t a_base = smem_u32(sA), b_base = smem_u32(sB);
    constexpr uint32_t IDESC = instr_desc(128, NP);
    const int tiles_per_b = (T + KT - 1) / KT;
    const int n_tiles = B * tiles_per_b;
    uint32_t phase = 0;
    bool failed = false;
    int issued = 0;
    float dbacc = 0.f;  // this thread's share of db (rows n = tid when tid < NP)
    for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const int b = tile / tiles_per_b, t0 = (tile % tiles_per_b) * KT;
        const __nv_bfloat16* xb = x + (size_t)b * T * C;
        const __nv_bfloat16* dyb = dy + (size_t)b * T * N;
        // A: thread r fills row r of every block, 8 times at a time
        for (int j = 0; j < NB; ++j) {
            const int m = 128 * j + tid;
            const bool row_ok = m < 3 * C;
            const int tap = row_ok ? m / C : 0, c = row_ok ? m % C : 0;
            for (int kc = 0; kc < KT / 8; ++kc) {
                __align__(16) __nv_bfloat16 h[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int t = t0 + kc * 8 + i, ts = t + (tap - 1) * dil;
                    h[i] = (row_ok && t < T && ts >= 0 && ts < T) ? xb[(size_t)ts * C + c] : __float2bfloat16(0.f);
                }
                *reinterpret_cast<uint4*>(sA + j * (A_BYTES / 2) + kmaj_off(tid, kc * 8, 128)) =
                    *reinterpret_cast<const uint4*>(h);
            }
        }
        // B (and the bias gradient): item (n, kc), n fastest
        for (int it = tid; it < NP * (KT / 8); it += NT) {
            const int n = it % NP, kc = it / NP;
            __align__(16) __nv_bfloat16 h[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int t = t0 + kc * 8 + i;
                h[i] = (n < N && t < T) ? dyb[(size_t)t * N + n] : __float2bfloat16(0.f);
                if (n < nv) dbacc += __bfloat162float(h[i]);
            }
            *reinterpret_cast<uint4*>(sB + kmaj_off(n, kc * 8, NP)) = *reinterpret_cast<const uint4*>(h);
        }
        // generic-proxy shared-memory writes become visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
#pragma unroll
            for (int j = 0; j < NB; ++j) {
#pragma unroll
                for (int s = 0; s < KT / 16; ++s) {
                    const uint64_t da = smem_desc(a_base + j * A_BYTES + s * 2 * (128 * 16), 128 * 16, 128);
                    const uint64_t dd = smem_desc(b_base + s * 2 * (NP * 16), NP * 16, 128);
                    const uint32_t acc = (issued > 0 || s > 0) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem + (uint32_t)(j * NP)),
                        "l"(da), "l"(dd), "r"(IDESC), "r"(acc));
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(&mbar))
                         : "memory");
        }
        ++issued;
        // the next tile's staging overwrites the operands: wait for the MMAs (bounded)
        if (!wait_parity(&mbar, phase, spin_limit)) failed = true;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        if (__syncthreads_or(failed ? 1 : 0)) {
            if (tid == 0) raise(err, EEMD_SG_E_TIMEOUT);
            break;
        }
    }
    if (!failed && issued > 0) {
        // epilogue: warp w holds accumulator lanes 32w..32w+31 (rows m of each block)
        for (int j = 0; j < NB; ++j) {
            float v[NP];
            tmem_ld<NP>(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(j * NP), v);
            const int m = 128 * j + 32 * warp + (tid & 31);
            if (m < 3 * C) {
                const int tap = m / C, c = m % C;
                if (c < cv) {
#pragma unroll
                    for (int n = 0; n < NP; ++n)
                        if (n < nv) atomicAdd(&dw[((size_t)n * 3 + tap) * cv + c], v[n]);
                }
            }
        }
    }
    // bias gradient: the per-thread partial sums of the staged dy rows
    if (NP * (KT / 8) % NT == 0) {
        // every thread always handled the same row n = tid % NP
        atomicAdd(&sdb[tid % NP], dbacc);
    }
    __syncthreads();
    if (tid < nv && tid < NP && !failed) atomicAdd(&db[tid], sdb[tid]);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS));
    }
}

// prediction = base + out (residual form; base may be null) over the first
// `cv` of `C` channels; loss partial sums over the interior [margin, T - margin)
// and the gradient d loss / d out as bf16.  The loss per element is d^2 for
// d = pred - target, or with delta > 0 the Huber loss (d^2 for |d| <= delta,
// 2 delta |d| - delta^2 beyond), each over the element count and times the
// channel's weight wch[c] when wch is not null.
// project = 1 (C = 16) removes the mean over the cv channels from the
// gradient of every sample: the gradient with respect to the raw output of a
// layer whose outputs are projected onto zero channel sum.
__global__ void k_loss(const __nv_bfloat16* __restrict__ out, const __nv_bfloat16* __restrict__ base,
                       const __nv_bfloat16* __restrict__ target, __nv_bfloat16* dout, float* loss, int B, int T,
                       int C, int cv, int margin, float inv_count, int project, float delta,
                       const float* __restrict__ wch) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in_range = i < (long long)B * T * C;
    float l = 0.f, g = 0.f;
    int c = 0;
    if (in_range) {
        c = (int)(i % C);
        const int t = (int)((i / C) % T);
        if (c < cv && t >= margin && t < T - margin) {
            const float d = (base ? __bfloat162float(base[i]) : 0.f) + __bfloat162float(out[i]) -
                            __bfloat162float(target[i]);
            const float wc = wch ? wch[c] : 1.f;
            if (delta > 0.f && fabsf(d) > delta) {
                l = wc * (2.f * delta * fabsf(d) - delta * delta);
                g = 2.f * wc * copysignf(delta, d) * inv_count;
            } else {
                l = wc * d * d;
                g = 2.f * wc * d * inv_count;
            }
        }
    }
    if (project) {
        // the 16 channels of one sample are 16 consecutive lanes
        float s = g;
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, 16);
        if (c < cv) g -= s / (float)cv;
    }
    if (in_range) dout[i] = __float2bfloat16(g);
    // warp sum, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l * inv_count);
}

// Adam (Kingma & Ba 2015) on f32 parameters
// (with gnorm2, the gradient is scaled to norm at most max_norm; a step
// whose gradient norm is not finite is skipped)
__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2, const float* gnorm2, float max_norm) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float sc = 1.f;
    if (gnorm2) {
        const float nrm = sqrtf(*gnorm2);
        if (!isfinite(nrm)) return;
        if (nrm > max_norm) sc = max_norm / nrm;
    }
    const float gi = g[i] * sc;
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// out[0] = sum of g[i]^2 (one CTA, fixed order)
__global__ void __launch_bounds__(1024) k_sumsq(const float* __restrict__ g, int n, float* out) {
    __shared__ float part[32];
    float a = 0.f;
    for (int i = threadIdx.x; i < n; i += 1024) a = fmaf(g[i], g[i], a);
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < 32; ++w) s += part[w];
        out[0] = s;
    }
}

// ---------------------------------------------------------------------------
// surrogate input and output stages.  A batch holds S signals of N samples;
// the engine's ensemble sums are imf_sum[s][m][t] (float64) with trial counts
// count[s][m] for m < K; the network sees K IMF channels and the residual
// channel (K + 1 <= C), all divided by the signal's RMS.
// ---------------------------------------------------------------------------
constexpr int GK = 10;                        // IMF channels of the network
constexpr int PMAX = 6;                       // corrected modes at most
constexpr int NGRAM = (GK + 1) * (GK + 2) / 2;  // Gram entries over IMFs + residual
constexpr int NREF = PMAX * (PMAX - 1) / 2;   // cross terms of the small-ensemble modes < PMAX
constexpr int NSTAT = 2 + NGRAM + NREF;       // sum x^2, sum reconstruction error^2, Gram, reference cross terms

// scale[s] = sqrt(mean x[s]^2) (1 for a zero signal); one CTA per signal
__global__ void __launch_bounds__(256) k_scale(const float* __restrict__ x, float* scale, int N) {
    __shared__ double part[8];
    const float* xs = x + (size_t)blockIdx.x * N;
    double a = 0.0;
    for (int t = threadIdx.x; t < N; t += 256) a += (double)xs[t] * (double)xs[t];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += part[w];
        const double r = sqrt(s / N);
        scale[blockIdx.x] = r > 0.0 ? (float)r : 1.f;
    }
}

// per-mode means and the residual x - sum(means) (the order of the engine's
// finalisation), divided by scale[s], as bf16 channels [s][t][C].  With
// imf_sum2 / count2, the difference of the two decompositions (a training
// target: large-ensemble minus small-ensemble channels), formed in float64.
__global__ void k_prepare(const double* __restrict__ imf_sum, const int* __restrict__ count,
                          const double* __restrict__ imf_sum2, const int* __restrict__ count2,
                          const float* __restrict__ x, const float* __restrict__ scale, __nv_bfloat16* out, int S,
                          int N, int K, int C) {
    const long long total = (long long)S * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int s = (int)(i / N), t = (int)(i % N);
        const double inv = 1.0 / (double)scale[s];
        __align__(16) __nv_bfloat16 h[32];
        for (int m = 0; m < C; ++m) h[m] = __float2bfloat16(0.f);
        double acc = 0.0, acc2 = 0.0;
        for (int m = 0; m < K; ++m) {
            const size_t e = ((size_t)s * K + m) * N + t;
            const int cnt = count[(size_t)s * K + m];
            const double mean = imf_sum[e] / (double)(cnt > 0 ? cnt : 1);
            acc += mean;
            double v = mean;
            if (imf_sum2) {
                const int cnt2 = count2[(size_t)s * K + m];
                const double mean2 = imf_sum2[e] / (double)(cnt2 > 0 ? cnt2 : 1);
                acc2 += mean2;
                v -= mean2;
            }
            h[m] = __float2bfloat16((float)(v * inv));
        }
        const double r = (double)x[i] - acc;
        const double r2 = imf_sum2 ? (double)x[i] - acc2 : 0.0;
        h[K] = __float2bfloat16((float)((r - r2) * inv));
        uint4* o = reinterpret_cast<uint4*>(out + (size_t)i * C);
        for (int q = 0; q < C / 8; ++q) o[q] = reinterpret_cast<const uint4*>(h)[q];
    }
}

// served decomposition from the network's corrections of the first P modes:
// imf[m] = mean_m + scale * net[m] (m < P), imf[m] = mean_m (P <= m < K),
// resid = (x - sum mean) - scale * sum_{m<P} net[m] (the corrections move
// content between the modes and the residual, the sum stays x); per-CTA
// partial sums of x^2, of the reconstruction error (x - sum imf - resid)^2 and
// of the Gram matrix of (imf_0..imf_{K-1}, resid).  grid (chunks, S), 128
// threads.
__global__ void __launch_bounds__(128) k_combine(const double* __restrict__ imf_sum, const int* __restrict__ count,
                                                 const float* __restrict__ x, const float* __restrict__ scale,
                                                 const __nv_bfloat16* __restrict__ net, double* imfs_out,
                                                 double* resid_out, double* partial, int N, int C, int P) {
    constexpr int K = GK;
    __shared__ double red[4][NSTAT];
    const int s = blockIdx.y, chunk = blockIdx.x, chunks = gridDim.x;
    const int per = (N + chunks - 1) / chunks;
    const int lo = chunk * per, hi = min(N, lo + per);
    const double sc = (double)scale[s];
    double cnt_d[K];
#pragma unroll
    for (int m = 0; m < K; ++m) {
        const int cnt = count[(size_t)s * K + m];
        cnt_d[m] = (double)(cnt > 0 ? cnt : 1);
    }
    double st[NSTAT];
#pragma unroll
    for (int j = 0; j < NSTAT; ++j) st[j] = 0.0;
    for (int t = lo + (int)threadIdx.x; t < hi; t += 128) {
        const size_t it = (size_t)s * N + t;
        const __nv_bfloat16* o = net + it * C;
        double c[K + 1], mr[PMAX];
        double acc = 0.0, moved = 0.0, sum_c = 0.0;
#pragma unroll
        for (int m = 0; m < K; ++m) {
            const double mean = imf_sum[((size_t)s * K + m) * N + t] / cnt_d[m];
            if (m < PMAX) mr[m] = mean;
            acc += mean;
            const double d = m < P ? sc * (double)__bfloat162float(o[m]) : 0.0;
            moved += d;
            c[m] = mean + d;
            imfs_out[((size_t)s * K + m) * N + t] = c[m];
            sum_c += c[m];
        }
        const double xv = (double)x[it];
        c[K] = (xv - acc) - moved;
        resid_out[it] = c[K];
        const double e = xv - (sum_c + c[K]);
        st[0] += xv * xv;
        st[1] += e * e;
        int q = 2;
#pragma unroll
        for (int a = 0; a <= K; ++a)
#pragma unroll
            for (int b = a; b <= K; ++b) st[q++] += c[a] * c[b];
#pragma unroll
        for (int a = 0; a < PMAX; ++a)
#pragma unroll
            for (int b = a + 1; b < PMAX; ++b) st[q++] += mr[a] * mr[b];
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 0; j < NSTAT; ++j) {
        double v = st[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][j] = v;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < NSTAT; j += 128)
        partial[((size_t)s * chunks + chunk) * NSTAT + j] = ((red[0][j] + red[1][j]) + red[2][j]) + red[3][j];
}

// per signal: the chunk partials added in chunk order; metrics[s] =
// {relative reconstruction error, orthogonality index of the P modes the
// network corrects, orthogonality index of all IMFs and the residual,
// orthogonality index of the same P modes of the small-ensemble means};
// fallback[s] = 1 when the error exceeds recon_bound or the corrected modes'
// index exceeds io_bound: in magnitude, or with io_relative by its magnitude
// less that of the small-ensemble modes (or any of these is not finite).
// Orthogonality index (Huang et al. 1998): sum over pairs j != k of
// <c_j, c_k> over ||x||^2.
__global__ void k_gate(const double* __restrict__ partial, int S, int chunks, int P, double recon_bound,
                       double io_bound, int io_relative, double* metrics, int* fallback) {
    constexpr int K = GK;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    double tot[NSTAT];
    for (int j = 0; j < NSTAT; ++j) tot[j] = 0.0;
    for (int ch = 0; ch < chunks; ++ch)
        for (int j = 0; j < NSTAT; ++j) tot[j] += partial[((size_t)s * chunks + ch) * NSTAT + j];
    double cross = 0.0, cross_p = 0.0, cross_ref = 0.0;
    int q = 2;
    for (int a = 0; a <= K; ++a)
        for (int b = a; b <= K; ++b, ++q)
            if (b != a) {
                cross += tot[q];
                if (b < P) cross_p += tot[q];
            }
    for (int a = 0; a < PMAX; ++a)
        for (int b = a + 1; b < PMAX; ++b, ++q)
            if (b < P) cross_ref += tot[q];
    const double xx = tot[0] > 0.0 ? tot[0] : 1.0;
    const double recon = sqrt(tot[1] / xx), io_p = 2.0 * cross_p / xx, io = 2.0 * cross / xx,
                 io_ref = 2.0 * cross_ref / xx;
    metrics[4 * s] = recon;
    metrics[4 * s + 1] = io_p;
    metrics[4 * s + 2] = io;
    metrics[4 * s + 3] = io_ref;
    const double check = io_relative ? fabs(io_p) - fabs(io_ref) : fabs(io_p);
    fallback[s] = !(recon <= recon_bound) || !(check <= io_bound) ? 1 : 0;
}

}  // namespace sg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace sg;

namespace {
// 3-D tensor map of the input [B][T][CIN] bf16 with the box {8, 128, 1}
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// 3-D tensor map of a bf16 [B][T][C] array with the box {box_c, 128, 1}
int tensor_map3(CUtensorMap* m, const void* p, int B, int T, int C, int box_c, CUtensorMapSwizzle swz) {
    static EncodeTiled encode = nullptr;
    if (!encode) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess || !fn)
            return EEMD_SG_E_CUDA;
        encode = reinterpret_cast<EncodeTiled>(fn);
    }
    if ((reinterpret_cast<uintptr_t>(p) & 15) != 0) return EEMD_SG_E_BADARG;  // a tensor map needs 16-byte alignment
    const cuuint64_t dims[3] = {(cuuint64_t)C, (cuuint64_t)T, (cuuint64_t)B};
    const cuuint64_t strides[2] = {(cuuint64_t)C * 2, (cuuint64_t)T * C * 2};
    const cuuint32_t box[3] = {(cuuint32_t)box_c, (cuuint32_t)TM, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<void*>(p), dims, strides, box, estr,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

// the input of k_conv_tma: boxes of 8 channels (one K-major no-swizzle chunk column)
int input_map(CUtensorMap* m, const void* in, int B, int T, int CIN) {
    return tensor_map3(m, in, B, T, CIN, 8, CU_TENSOR_MAP_SWIZZLE_NONE);
}

template <int CIN, int COUT>
int launch_tma(const void* in, const void* wpk, const float* bias, void* out, int B, int T, int dil, int dir,
               int relu, const void* mask, int* err, long long spin, cudaStream_t st) {
    const size_t smem = (size_t)TMA_STAGES * 3 * CIN * TM * 2 + (size_t)3 * CIN * COUT * 2;
    constexpr int EW = TMA_EPI_WARPS;
    if (cudaFuncSetAttribute(k_conv_tma<CIN, COUT, EW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_conv_tma<CIN, COUT, EW>, cudaFuncAttributePreferredSharedMemoryCarveout, 100) !=
            cudaSuccess)
        return EEMD_SG_E_CUDA;
    CUtensorMap m;
    const int rc = input_map(&m, in, B, T, CIN);
    if (rc) return rc;
    static int resident = 0;
    if (resident == 0) {
        int dev = 0, sms = 0, smem_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
            return EEMD_SG_E_CUDA;
        int per_sm = smem_sm / ((int)smem + 2048);
        const int tcols = 2 * (COUT < 32 ? 32 : COUT);
        if (per_sm > 512 / tcols) per_sm = 512 / tcols;
        if (per_sm > 2048 / (32 * EW)) per_sm = 2048 / (32 * EW);
        resident = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int tiles = B * ((T + TM - 1) / TM);
    const int grid = tiles < resident ? tiles : resident;
    k_conv_tma<CIN, COUT, EW><<<grid, 32 * EW, smem, st>>>(m, static_cast<const __nv_bfloat16*>(wpk), bias,
                                                   static_cast<__nv_bfloat16*>(out), B, T, dil, dir, relu,
                                                   static_cast<const __nv_bfloat16*>(mask), err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

// the warp-specialised kernel: one CTA per SM, the input through a swizzled
// tensor map (128-byte for 64 channels, 32-byte for 16), the output through a
// 128-byte-swizzled one (no swizzle for 16 output channels, rows of 32 bytes)
template <int CIN, int COUT>
int launch_ws(const void* in, const void* wpk, const float* bias, void* out, int B, int T, int dil, int dir,
              int relu, const void* mask, int* err, long long spin, cudaStream_t st) {
    using G = WsGeo<CIN, COUT>;
    const auto misaligned = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) != 0; };
    if (misaligned(wpk) || misaligned(out) || (mask && misaligned(mask))) return EEMD_SG_E_BADARG;
    if (cudaFuncSetAttribute(k_conv_ws<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, G::SMEM) !=
        cudaSuccess)
        return EEMD_SG_E_CUDA;
    CUtensorMap mi, mo;
    int rc = tensor_map3(&mi, in, B, T, CIN, CIN, CIN == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_32B);
    if (rc) return rc;
    rc = tensor_map3(&mo, out, B, T, COUT, COUT, COUT == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE);
    if (rc) return rc;
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return EEMD_SG_E_CUDA;
    }
    const int tiles = B * ((T + TM - 1) / TM);
    const int grid = tiles < sms ? tiles : sms;
    k_conv_ws<CIN, COUT><<<grid, WS_THREADS, G::SMEM, st>>>(mi, mo, static_cast<const __nv_bfloat16*>(wpk), bias,
                                                           B, T, dil, dir, relu,
                                                           static_cast<const __nv_bfloat16*>(mask), err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

// the double-buffered kernel: CTAs per SM from shared memory (the carveout
// at its maximum), tensor-memory columns and threads
template <int CIN, int COUT>
int launch_tc2(const void* in, const void* wpk, const float* bias, void* out, int B, int T, int dil, int dir,
               int relu, const void* mask, int* err, long long spin, cudaStream_t st) {
    const size_t smem = (size_t)2 * 3 * CIN * TM * 2 + (size_t)3 * CIN * COUT * 2;
    if (cudaFuncSetAttribute(k_conv_tc2<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
            cudaSuccess ||
        cudaFuncSetAttribute(k_conv_tc2<CIN, COUT>, cudaFuncAttributePreferredSharedMemoryCarveout, 100) !=
            cudaSuccess)
        return EEMD_SG_E_CUDA;
    static int resident = 0;
    if (resident == 0) {
        int dev = 0, sms = 0, smem_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
            return EEMD_SG_E_CUDA;
        const int per_block = (int)smem + 1024 + 1024;  // dynamic + static + the per-block reservation
        int per_sm = smem_sm / per_block;
        const int tcols = 2 * (COUT < 32 ? 32 : COUT);
        if (per_sm > 512 / tcols) per_sm = 512 / tcols;
        if (per_sm > 2048 / NT) per_sm = 2048 / NT;
        resident = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int tiles = B * ((T + TM - 1) / TM);
    const int grid = tiles < resident ? tiles : resident;
    k_conv_tc2<CIN, COUT><<<grid, NT, smem, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                   static_cast<const __nv_bfloat16*>(wpk), bias,
                                                   static_cast<__nv_bfloat16*>(out), B, T, dil, dir, relu,
                                                   static_cast<const __nv_bfloat16*>(mask), err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

template <int CIN, int COUT>
int launch_tc(const void* in, const void* wpk, const float* bias, void* out, int B, int T, int dil, int dir,
              int relu, const void* mask, int* err, long long spin, cudaStream_t st) {
    const size_t smem = (size_t)3 * CIN * TM * 2 + (size_t)3 * CIN * COUT * 2;
    if (cudaFuncSetAttribute(k_conv_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return EEMD_SG_E_CUDA;
    // persistent CTAs: as many as fit on the device at once (shared memory bounds them)
    static int resident = 0;
    if (resident == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_conv_tc<CIN, COUT>, NT, smem) != cudaSuccess)
            return EEMD_SG_E_CUDA;
        // tensor memory: 512 columns per SM, TCOLS per CTA (an allocation that
        // does not fit would wait for another CTA's release)
        const int tcols = COUT < 32 ? 32 : COUT;
        if (per_sm > 512 / tcols) per_sm = 512 / tcols;
        resident = sms * (per_sm > 0 ? per_sm : 1);
    }
    const int tiles = B * ((T + TM - 1) / TM);
    const int grid = tiles < resident ? tiles : resident;
    k_conv_tc<CIN, COUT><<<grid, NT, smem, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                  static_cast<const __nv_bfloat16*>(wpk), bias,
                                                  static_cast<__nv_bfloat16*>(out), B, T, dil, dir, relu,
                                                  static_cast<const __nv_bfloat16*>(mask), err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}
}  // namespace

template <int NB, int NP>
int32_t launch_wgrad_tc(const __nv_bfloat16* dy, const __nv_bfloat16* x, float* dw, float* db, int B, int T, int N,
                        int C, int nv, int cv, int dil, int* err, long long spin, cudaStream_t st) {
    const size_t smem = (size_t)NB * 128 * 128 * 2 + (size_t)NP * 128 * 2;
    if (cudaFuncSetAttribute(k_wgrad_tc<NB, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return EEMD_SG_E_CUDA;
    const long long tiles = (long long)B * ((T + 127) / 128);
    const int grid = (int)(tiles < 296 ? tiles : 296);  // two CTAs per SM (shared memory and tensor memory allow it)
    if (grid < 1) return EEMD_SG_OK;
    k_wgrad_tc<NB, NP><<<grid, NT, smem, st>>>(dy, x, dw, db, B, T, N, C, nv, cv, dil, err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

extern "C" {

int32_t eemd_sg_version(void) { return EEMD_SG_ABI_VERSION; }

int32_t eemd_sg_conv(const void* in, const void* wpk, const float* bias, void* out, int32_t B, int32_t T,
                     int32_t cin, int32_t cout, int32_t dil, int32_t dir, int32_t relu, const void* mask,
                     int32_t tensor_cores, int32_t* err, int64_t spin_limit, void* stream) {
    if (!in || !wpk || !out || B < 1 || T < 1 || dil < 1 || (dir != 1 && dir != -1)) return EEMD_SG_E_BADARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!tensor_cores) {
        const long long n = (long long)B * T * cout;
        k_conv_ref<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
            static_cast<const __nv_bfloat16*>(in), static_cast<const __nv_bfloat16*>(wpk), bias,
            static_cast<__nv_bfloat16*>(out), B, T, cin, cout, dil, dir, relu,
            static_cast<const __nv_bfloat16*>(mask));
        return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
    }
    const long long spin = spin_limit > 0 ? spin_limit : (1LL << 24);
    if (tensor_cores == 4) {
        if (cin == 64 && cout == 64) return launch_ws<64, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 16 && cout == 64) return launch_ws<16, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 64 && cout == 16) return launch_ws<64, 16>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        return EEMD_SG_E_BADARG;
    }
    if (tensor_cores >= 3) {
        if (cin == 64 && cout == 64)
            return launch_tma<64, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 16 && cout == 64)
            return launch_tma<16, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 64 && cout == 16)
            return launch_tma<64, 16>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        return EEMD_SG_E_BADARG;
    }
    if (tensor_cores == 2) {
        if (cin == 64 && cout == 64)
            return launch_tc2<64, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 16 && cout == 64)
            return launch_tc2<16, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        if (cin == 64 && cout == 16)
            return launch_tc2<64, 16>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
        return EEMD_SG_E_BADARG;
    }
    if (cin == 64 && cout == 64) return launch_tc<64, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    if (cin == 16 && cout == 64) return launch_tc<16, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    if (cin == 64 && cout == 16) return launch_tc<64, 16>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    return EEMD_SG_E_BADARG;
}

int32_t eemd_sg_pack(const float* w, void* wpk, int32_t n_rows, int32_t c, int32_t nv, int32_t cv,
                     int32_t transpose, int32_t project, void* stream) {
    if (!w || !wpk || n_rows % 16 || c % 16 || nv > n_rows || cv > c) return EEMD_SG_E_BADARG;
    const int n = n_rows * 3 * c;
    k_pack<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(w, static_cast<__nv_bfloat16*>(wpk),
                                                                           n_rows, c, nv, cv, transpose, project);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_wgrad(const void* dy, const void* x, float* dw, float* db, int32_t B, int32_t T, int32_t n_rows,
                      int32_t c, int32_t nv, int32_t cv, int32_t dil, int32_t tensor_cores, int32_t* err,
                      int64_t spin_limit, void* stream) {
    if (!dy || !x || !dw || !db || n_rows > 64 || c > 64 || nv > n_rows || cv > c) return EEMD_SG_E_BADARG;
    if (tensor_cores && (n_rows == 64 || n_rows == 16) && c >= 1) {
        const long long spin = spin_limit > 0 ? spin_limit : (1LL << 24);
        const cudaStream_t st = static_cast<cudaStream_t>(stream);
        const auto* pdy = static_cast<const __nv_bfloat16*>(dy);
        const auto* px = static_cast<const __nv_bfloat16*>(x);
        if (3 * c <= 128)
            return n_rows == 64 ? launch_wgrad_tc<1, 64>(pdy, px, dw, db, B, T, n_rows, c, nv, cv, dil, err, spin, st)
                                : launch_wgrad_tc<1, 16>(pdy, px, dw, db, B, T, n_rows, c, nv, cv, dil, err, spin, st);
        return n_rows == 64 ? launch_wgrad_tc<2, 64>(pdy, px, dw, db, B, T, n_rows, c, nv, cv, dil, err, spin, st)
                            : launch_wgrad_tc<2, 16>(pdy, px, dw, db, B, T, n_rows, c, nv, cv, dil, err, spin, st);
    }
    dim3 grid((unsigned)(B * ((T + 63) / 64)), 3);
    k_wgrad<<<grid, NT, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(dy),
                                                                 static_cast<const __nv_bfloat16*>(x), dw, db, B, T,
                                                                 n_rows, c, nv, cv, dil);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_loss(const void* out, const void* base, const void* target, void* dout, float* loss, int32_t B,
                     int32_t T, int32_t c, int32_t cv, int32_t margin, int32_t project, float delta,
                     const float* channel_weight, void* stream) {
    if (!out || !target || !dout || !loss || 2 * margin >= T || cv < 1 || cv > c || (project && c != 16))
        return EEMD_SG_E_BADARG;
    const long long n = (long long)B * T * c;
    const float inv = 1.f / (float)((long long)B * (T - 2 * margin) * cv);
    k_loss<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(out), static_cast<const __nv_bfloat16*>(base),
        static_cast<const __nv_bfloat16*>(target), static_cast<__nv_bfloat16*>(dout), loss, B, T, c, cv, margin,
        inv, project, delta, channel_weight);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float b1, float b2,
                     float eps, int32_t step, float max_norm, float* work, void* stream) {
    if (!p || !g || !m || !v || n < 0 || step < 1 || (max_norm > 0.f && !work)) return EEMD_SG_E_BADARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    if (max_norm > 0.f) k_sumsq<<<1, 1024, 0, st>>>(g, n, work);
    k_adam<<<(n + 255) / 256, 256, 0, st>>>(p, g, m, v, n, lr, b1, b2, eps, bc1, bc2,
                                            max_norm > 0.f ? work : nullptr, max_norm);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_bias(const float* b, float* bias, int32_t n_rows, int32_t nv, int32_t project, void* stream) {
    if (!b || !bias || n_rows < 1 || n_rows > 1024 || nv < 1 || nv > n_rows) return EEMD_SG_E_BADARG;
    k_bias<<<1, n_rows, 0, static_cast<cudaStream_t>(stream)>>>(b, bias, n_rows, nv, project);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_scale(const float* x, float* scale, int32_t S, int32_t N, void* stream) {
    if (!x || !scale || S < 1 || N < 1) return EEMD_SG_E_BADARG;
    k_scale<<<S, 256, 0, static_cast<cudaStream_t>(stream)>>>(x, scale, N);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_prepare(const double* imf_sum, const int32_t* mode_count, const double* imf_sum2,
                        const int32_t* mode_count2, const float* x, const float* scale, void* out, int32_t S,
                        int32_t N, int32_t K, int32_t C, void* stream) {
    if (!imf_sum || !mode_count || !x || !scale || !out || S < 1 || N < 1 || K < 1 || C % 8 || C > 32 ||
        K + 1 > C || (imf_sum2 && !mode_count2))
        return EEMD_SG_E_BADARG;
    const long long total = (long long)S * N;
    const long long blocks = (total + 255) / 256;
    k_prepare<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        imf_sum, mode_count, imf_sum2, mode_count2, x, scale, static_cast<__nv_bfloat16*>(out), S, N, K, C);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_combine(const double* imf_sum, const int32_t* mode_count, const float* x, const float* scale,
                        const void* net_out, double* imfs_out, double* resid_out, double* partial, int32_t chunks,
                        int32_t S, int32_t N, int32_t K, int32_t C, int32_t P, double recon_bound,
                        double io_bound, int32_t io_relative, double* metrics, int32_t* fallback,
                        void* stream) {
    if (!imf_sum || !mode_count || !x || !scale || !net_out || !imfs_out || !resid_out || !partial || !metrics ||
        !fallback || S < 1 || N < 1 || K != GK || C % 8 || C > 32 || P < 0 || P > PMAX || P > C || chunks < 1 ||
        chunks > 65535)
        return EEMD_SG_E_BADARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_combine<<<dim3(chunks, S), 128, 0, st>>>(imf_sum, mode_count, x, scale,
                                                static_cast<const __nv_bfloat16*>(net_out), imfs_out, resid_out,
                                                partial, N, C, P);
    k_gate<<<(S + 127) / 128, 128, 0, st>>>(partial, S, chunks, P, recon_bound, io_bound, io_relative, metrics,
                                            fallback);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_stat_count(void) { return NSTAT; }

}  // extern "C"
