// surrogate.cu -- kernels of the learned ensemble surrogate (sm_100a).
//
// The surrogate maps the 8-trial ensemble-mean IMFs of a signal to its
// 256-trial ensemble mean with a dilated 1-D convolution network (8 layers,
// 64 channels, kernel 3, dilations 1..128; bfloat16 weights and activations,
// float32 accumulation).  Activations are channels-last, [batch][time][C]
// with C = 16 (10 IMF channels, zero padded) or 64.
//
// Every convolution is an implicit GEMM on the 5th-generation tensor cores:
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
// The weight gradient, the loss, Adam and the packing kernels run on CUDA
// cores.  A plain CUDA-core convolution with the same arguments is kept for
// checking the tensor-core path on the GPU.
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
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

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
                    float x = v[c0 + i] + (bias ? bias[c0 + i] : 0.f);
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

// Packs f32 weights w[n][tap][c] (n < nv, c < cv, zero elsewhere) into the
// bf16 K-major B-tile image of an (N rows) x (3*C) operand.  transpose = 1
// packs w[c][tap][n] instead (the input-gradient operand).
__global__ void k_pack(const float* __restrict__ w, __nv_bfloat16* wpk, int N, int C, int nv, int cv,
                       int transpose) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N * 3 * C) return;
    const int n = i / (3 * C), k = i % (3 * C);
    const int tap = k / C, c = k % C;
    float x = 0.f;
    if (n < nv && c < cv) x = transpose ? w[((size_t)c * 3 + tap) * nv + n] : w[((size_t)n * 3 + tap) * cv + c];
    wpk[kmaj_off(n, k, N)] = __float2bfloat16(x);
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

// prediction = base + out (residual form) over the first `cv` of `C` channels;
// loss partial sums over the interior [margin, T - margin) and the gradient
// d loss / d out = 2 (pred - target) / count as bf16
__global__ void k_loss(const __nv_bfloat16* __restrict__ out, const __nv_bfloat16* __restrict__ base,
                       const __nv_bfloat16* __restrict__ target, __nv_bfloat16* dout, float* loss, int B, int T,
                       int C, int cv, int margin, float inv_count) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (i < (long long)B * T * C) {
        const int c = (int)(i % C);
        const int t = (int)((i / C) % T);
        float g = 0.f;
        if (c < cv && t >= margin && t < T - margin) {
            const float d = __bfloat162float(base[i]) + __bfloat162float(out[i]) - __bfloat162float(target[i]);
            l = d * d;
            g = 2.f * d * inv_count;
        }
        dout[i] = __float2bfloat16(g);
    }
    // warp sum, one atomic per warp
    for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l * inv_count);
}

// Adam (Kingma & Ba 2015) on f32 parameters
__global__ void k_adam(float* p, const float* g, float* m, float* v, int n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

}  // namespace sg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace sg;

namespace {
template <int CIN, int COUT>
int launch_tc(const void* in, const void* wpk, const float* bias, void* out, int B, int T, int dil, int dir,
              int relu, const void* mask, int* err, long long spin, cudaStream_t st) {
    const size_t smem = (size_t)3 * CIN * TM * 2 + (size_t)3 * CIN * COUT * 2;
    if (cudaFuncSetAttribute(k_conv_tc<CIN, COUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return EEMD_SG_E_CUDA;
    const int tiles = B * ((T + TM - 1) / TM);
    const int grid = tiles < 2 * 148 ? tiles : 2 * 148;
    k_conv_tc<CIN, COUT><<<grid, NT, smem, st>>>(static_cast<const __nv_bfloat16*>(in),
                                                  static_cast<const __nv_bfloat16*>(wpk), bias,
                                                  static_cast<__nv_bfloat16*>(out), B, T, dil, dir, relu,
                                                  static_cast<const __nv_bfloat16*>(mask), err, spin);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}
}  // namespace

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
    if (cin == 64 && cout == 64) return launch_tc<64, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    if (cin == 16 && cout == 64) return launch_tc<16, 64>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    if (cin == 64 && cout == 16) return launch_tc<64, 16>(in, wpk, bias, out, B, T, dil, dir, relu, mask, err, spin, st);
    return EEMD_SG_E_BADARG;
}

int32_t eemd_sg_pack(const float* w, void* wpk, int32_t n_rows, int32_t c, int32_t nv, int32_t cv,
                     int32_t transpose, void* stream) {
    if (!w || !wpk || n_rows % 16 || c % 16 || nv > n_rows || cv > c) return EEMD_SG_E_BADARG;
    const int n = n_rows * 3 * c;
    k_pack<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(w, static_cast<__nv_bfloat16*>(wpk),
                                                                           n_rows, c, nv, cv, transpose);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_wgrad(const void* dy, const void* x, float* dw, float* db, int32_t B, int32_t T, int32_t n_rows,
                      int32_t c, int32_t nv, int32_t cv, int32_t dil, void* stream) {
    if (!dy || !x || !dw || !db || n_rows > 64 || c > 64 || nv > n_rows || cv > c) return EEMD_SG_E_BADARG;
    dim3 grid((unsigned)(B * ((T + 63) / 64)), 3);
    k_wgrad<<<grid, NT, 0, static_cast<cudaStream_t>(stream)>>>(static_cast<const __nv_bfloat16*>(dy),
                                                                 static_cast<const __nv_bfloat16*>(x), dw, db, B, T,
                                                                 n_rows, c, nv, cv, dil);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_loss(const void* out, const void* base, const void* target, void* dout, float* loss, int32_t B,
                     int32_t T, int32_t c, int32_t cv, int32_t margin, void* stream) {
    if (!out || !base || !target || !dout || !loss || 2 * margin >= T) return EEMD_SG_E_BADARG;
    const long long n = (long long)B * T * c;
    const float inv = 1.f / (float)((long long)B * (T - 2 * margin) * cv);
    k_loss<<<(unsigned)((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const __nv_bfloat16*>(out), static_cast<const __nv_bfloat16*>(base),
        static_cast<const __nv_bfloat16*>(target), static_cast<__nv_bfloat16*>(dout), loss, B, T, c, cv, margin,
        inv);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

int32_t eemd_sg_adam(float* p, const float* g, float* m, float* v, int32_t n, float lr, float b1, float b2,
                     float eps, int32_t step, void* stream) {
    if (!p || !g || !m || !v || n < 0 || step < 1) return EEMD_SG_E_BADARG;
    const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
    k_adam<<<(n + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(p, g, m, v, n, lr, b1, b2, eps, bc1,
                                                                          bc2);
    return cudaGetLastError() == cudaSuccess ? EEMD_SG_OK : EEMD_SG_E_CUDA;
}

}  // extern "C"
