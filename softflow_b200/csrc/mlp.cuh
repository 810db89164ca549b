// mlp.cuh -- the per-marker network of learned multi-direct forcing:
// 8 -> 64 -> 64 -> 2 with ReLU, BF16 operands on the 5th-generation tensor
// cores (tcgen05.mma, accumulators in tensor memory, FP32 accumulation).
//
// One CTA of 128 threads owns a tile of 128 rows (markers or samples); row r
// is thread r and tensor-memory lane r.  Operands live in shared memory in
// the K-major, no-swizzle canonical layout: 8-row x 16-byte core matrices of
// 128 contiguous bytes, ordered K-chunk-fastest inside each 8-row group, so
// the leading-byte offset (next core matrix along K) is 128 B and the
// stride-byte offset (next 8-row group) is K/8 * 128 B.  One elected thread
// issues the MMAs; their completion arrives on an mbarrier through
// tcgen05.commit, and every wait is bounded.
//
// Shape and conventions follow the reference surrogate network
// (src/ml/simple_nn.cpp:45-79): h1 = relu(W1 x + b1), h2 = relu(W2 h1 + b2),
// y = W3 h2 + b3, inputs and outputs normalised by mean and standard deviation
// (:156-165).  Layer 1 carries b1 as a ninth input fixed at 1.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace sfg {
namespace mlp {

constexpr int N_IN = 8, N_H = 64, N_OUT = 2;
constexpr int K1 = 16;           // padded layer-1 width (8 features, 1, zeros)
constexpr int ROWS = 128;        // rows per tile = threads per CTA
constexpr int N3 = 16;           // padded layer-3 width (MMA N >= 16 at M = 128)
constexpr int N_PARAMS = N_H * N_IN + N_H + N_H * N_H + N_H + N_OUT * N_H + N_OUT;  // 4866
// parameter vector offsets (W1 [64x8], b1, W2 [64x64], b2, W3 [2x64], b3)
constexpr int P_W1 = 0, P_B1 = P_W1 + N_H * N_IN, P_W2 = P_B1 + N_H, P_B2 = P_W2 + N_H * N_H,
              P_W3 = P_B2 + N_H, P_B3 = P_W3 + N_OUT * N_H;
constexpr uint32_t WAIT_LIMIT = 1u << 22;  // try_wait rounds before giving up

// Normalisation and BF16 weights in the shared-memory operand layouts, as
// the inference kernels copy them (built once from the FP32 parameters).
struct ModelDev {
    __nv_bfloat16 W1[N_H * K1];     // [64 x 16] K-major, column 8 = b1
    __nv_bfloat16 W2[N_H * N_H];    // [64 x 64] K-major
    __nv_bfloat16 W3[N3 * N_H];     // [16 x 64] K-major, rows 2..15 zero
    float b2[N_H];
    float b3[N_OUT];
    float in_mean[N_IN], in_inv_std[N_IN];
    float out_mean[N_OUT], out_std[N_OUT];
};

// element offset of (r, k) in a K-major no-swizzle operand with K columns
__host__ __device__ __forceinline__ int kmaj(int r, int k, int K) {
    return ((((r >> 3) * (K >> 3)) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), version 1, no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Descriptor of the K-step kk (16 columns) of a K-major operand with K columns.
__device__ __forceinline__ uint64_t opdesc(const __nv_bfloat16* base, int K, int kk) {
    return sdesc(smem_u32(base) + (uint32_t)kk * 256u, 128u, (uint32_t)(K >> 3) * 128u);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 :
                 : "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" : : : "memory");
}

// Waits for the phase with the given parity to complete; false after
// WAIT_LIMIT rounds (each try_wait suspends for a bounded time).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (uint32_t i = 0; i < WAIT_LIMIT; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" : : : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" : : : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" : : : "memory");
}

// Allocation by one whole warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" : : : "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(taddr), "r"(ncols)
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's lane (warp w reads lanes
// 32w..32w+31); the wait sits in the same asm block as the load.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// lane-row address of column `col` for the calling thread's warp
__device__ __forceinline__ uint32_t tmem_row(uint32_t tbase, int col) {
    const uint32_t warp = threadIdx.x >> 5;
    return tbase + ((warp * 32u) << 16) + (uint32_t)col;
}

// Shared-memory image of the forward pass of one tile.
struct __align__(1024) FwdSmem {
    __nv_bfloat16 X[ROWS * K1];     // 4 KB
    __nv_bfloat16 W1[N_H * K1];     // 2 KB
    __nv_bfloat16 W3[N3 * N_H];     // 2 KB
    __nv_bfloat16 W2[N_H * N_H];    // 8 KB
    __nv_bfloat16 H1[ROWS * N_H];   // 16 KB
    __nv_bfloat16 H2[ROWS * N_H];   // 16 KB
    float b2[N_H], b3[N_OUT];
    float in_mean[N_IN], in_inv_std[N_IN], out_mean[N_OUT], out_std[N_OUT];
    uint64_t bar;
    uint32_t taddr;
    int error;
};

// Copies the model (already in operand layout) into shared memory.
template <typename SM>
__device__ __forceinline__ void load_model(SM& s, const ModelDev* __restrict__ md) {
    const int t = threadIdx.x;
    const uint4* w1 = reinterpret_cast<const uint4*>(md->W1);
    const uint4* w2 = reinterpret_cast<const uint4*>(md->W2);
    const uint4* w3 = reinterpret_cast<const uint4*>(md->W3);
    uint4* s1 = reinterpret_cast<uint4*>(s.W1);
    uint4* s2 = reinterpret_cast<uint4*>(s.W2);
    uint4* s3 = reinterpret_cast<uint4*>(s.W3);
    for (int i = t; i < N_H * K1 / 8; i += ROWS) s1[i] = w1[i];
    for (int i = t; i < N_H * N_H / 8; i += ROWS) s2[i] = w2[i];
    for (int i = t; i < N3 * N_H / 8; i += ROWS) s3[i] = w3[i];
    if (t < N_H) s.b2[t] = md->b2[t];
    if (t < N_OUT) {
        s.b3[t] = md->b3[t];
        s.out_mean[t] = md->out_mean[t];
        s.out_std[t] = md->out_std[t];
    }
    if (t < N_IN) {
        s.in_mean[t] = md->in_mean[t];
        s.in_inv_std[t] = md->in_inv_std[t];
    }
}

// Writes this thread's row of X: normalised features, 1 (bias), zeros.
template <typename SM>
__device__ __forceinline__ void put_input_row(SM& s, const float* feat, bool valid) {
    const int r = threadIdx.x;
#pragma unroll
    for (int k = 0; k < K1; ++k) {
        float v = 0.0f;
        if (valid && k < N_IN) v = (feat[k] - s.in_mean[k]) * s.in_inv_std[k];
        if (valid && k == N_IN) v = 1.0f;
        s.X[kmaj(r, k, K1)] = __float2bfloat16_rn(v);
    }
}

// One layer: makes the operands written by the threads visible to the tensor
// cores, issues the K/16 MMAs from thread 0 and waits for their commit.
// After a timed-out wait the CTA issues nothing more (s.error, read after
// the next barrier) and finish_tile waits once more before freeing.
template <int K, typename SM>
__device__ __forceinline__ bool layer(SM& s, uint32_t tmem_d, const __nv_bfloat16* A,
                                      const __nv_bfloat16* B, uint32_t idesc,
                                      uint32_t& phase) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (s.error) return false;  // uniform: read after the barrier
    if (threadIdx.x == 0) {
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk)
            mma(tmem_d, opdesc(A, K, kk), opdesc(B, K, kk), idesc, kk > 0 ? 1u : 0u);
        mma_commit(&s.bar);
    }
    if (!mbar_wait(&s.bar, phase)) s.error = 1;
    phase ^= 1u;
    tc_fence_after();
    return true;
}

// Forward pass of a tile whose X rows are written.  Tensor-memory columns:
// layer 1 [0, 64), layer 2 [64, 128), layer 3 [0, 16) of tbase.  Leaves the
// normalised outputs of this thread's row in y[2] and the BF16 activations in
// s.H1 / s.H2; false when a wait timed out.
__device__ __forceinline__ bool forward_tile(FwdSmem& s, uint32_t tbase, uint32_t& phase,
                                             float* y) {
    const int r = threadIdx.x;
    if (!layer<K1>(s, tbase, s.X, s.W1, idesc_bf16(ROWS, N_H), phase)) return false;
    {
        // relu, BF16 (b1 came in through the constant input)
        float v[16];
#pragma unroll
        for (int c = 0; c < N_H; c += 16) {
            tmem_ld16(tmem_row(tbase, c), v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                s.H1[kmaj(r, c + i, N_H)] = __float2bfloat16_rn(fmaxf(v[i], 0.0f));
        }
    }
    if (!layer<N_H>(s, tbase + 64, s.H1, s.W2, idesc_bf16(ROWS, N_H), phase)) return false;
    {
        float v[16];
#pragma unroll
        for (int c = 0; c < N_H; c += 16) {
            tmem_ld16(tmem_row(tbase, 64 + c), v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                s.H2[kmaj(r, c + i, N_H)] = __float2bfloat16_rn(fmaxf(v[i] + s.b2[c + i], 0.0f));
        }
    }
    if (!layer<N_H>(s, tbase, s.H2, s.W3, idesc_bf16(ROWS, N3), phase)) return false;
    {
        float v[16];
        tmem_ld16(tmem_row(tbase, 0), v);
        y[0] = v[0] + s.b3[0];
        y[1] = v[1] + s.b3[1];
    }
    return true;
}

// The network seed's image: the two inputs of the odd part (x and Px) go
// through the layers together, 2 x 128 rows a tile, so each layer is one
// round of MMAs, commit and wait for both instead of two.  Per input, one
// activation buffer reused by both hidden layers (layer 2's MMAs have
// completed before its outputs are written back) and 64 tensor-memory
// columns reused by all three layers (x's in [0, 64), Px's in [64, 128)).
// Each input's MMAs are those of forward_tile, so the outputs do not depend
// on the pairing.  About 53 KB: four CTAs per SM, whose 4 x 128 columns fill
// the tensor memory exactly (more resident CTAs would wait in the
// allocation; shared memory rules them out).
struct __align__(1024) FwdSmemDual {
    __nv_bfloat16 X[2][ROWS * K1];    // 8 KB
    __nv_bfloat16 W1[N_H * K1];       // 2 KB
    __nv_bfloat16 W3[N3 * N_H];       // 2 KB
    __nv_bfloat16 W2[N_H * N_H];      // 8 KB
    __nv_bfloat16 H1[2][ROWS * N_H];  // 32 KB
    float b2[N_H], b3[N_OUT];
    float in_mean[N_IN], in_inv_std[N_IN], out_mean[N_OUT], out_std[N_OUT];
    uint64_t bar;
    uint32_t taddr;
    int error;
};
constexpr uint32_t DUAL_TMEM_COLS = 128;

// put_input_row into input buffer `b` of the dual image.
__device__ __forceinline__ void put_input_row_dual(FwdSmemDual& s, int b, const float* feat,
                                                   bool valid) {
    const int r = threadIdx.x;
#pragma unroll
    for (int k = 0; k < K1; ++k) {
        float v = 0.0f;
        if (valid && k < N_IN) v = (feat[k] - s.in_mean[k]) * s.in_inv_std[k];
        if (valid && k == N_IN) v = 1.0f;
        s.X[b][kmaj(r, k, K1)] = __float2bfloat16_rn(v);
    }
}

// layer() for both inputs of the dual image: the MMAs of A0 into d0 and of
// A1 into d1 (same weights B), one commit and one wait.
template <int K>
__device__ __forceinline__ bool layer_dual(FwdSmemDual& s, uint32_t d0, uint32_t d1,
                                           const __nv_bfloat16* A0, const __nv_bfloat16* A1,
                                           const __nv_bfloat16* B, uint32_t idesc,
                                           uint32_t& phase) {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (s.error) return false;  // uniform: read after the barrier
    if (threadIdx.x == 0) {
        tc_fence_after();
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk)
            mma(d0, opdesc(A0, K, kk), opdesc(B, K, kk), idesc, kk > 0 ? 1u : 0u);
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk)
            mma(d1, opdesc(A1, K, kk), opdesc(B, K, kk), idesc, kk > 0 ? 1u : 0u);
        mma_commit(&s.bar);
    }
    if (!mbar_wait(&s.bar, phase)) s.error = 1;
    phase ^= 1u;
    tc_fence_after();
    return true;
}

// The forward pass of both inputs: outputs of this thread's row in y
// (input 0) and ym (input 1).
__device__ __forceinline__ bool forward_tile_dual(FwdSmemDual& s, uint32_t tbase,
                                                  uint32_t& phase, float* y, float* ym) {
    const int r = threadIdx.x;
    const uint32_t t1 = tbase + 64;
    if (!layer_dual<K1>(s, tbase, t1, s.X[0], s.X[1], s.W1, idesc_bf16(ROWS, N_H), phase))
        return false;
    {
        float v[16];
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < N_H; c += 16) {
                tmem_ld16(tmem_row(b ? t1 : tbase, c), v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    s.H1[b][kmaj(r, c + i, N_H)] = __float2bfloat16_rn(fmaxf(v[i], 0.0f));
            }
    }
    if (!layer_dual<N_H>(s, tbase, t1, s.H1[0], s.H1[1], s.W2, idesc_bf16(ROWS, N_H), phase))
        return false;
    {
        // layer 2's MMAs have completed (their commit was waited for), so
        // its operands H1 can take its outputs; each thread rewrites its row
        float v[16];
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < N_H; c += 16) {
                tmem_ld16(tmem_row(b ? t1 : tbase, c), v);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    s.H1[b][kmaj(r, c + i, N_H)] =
                        __float2bfloat16_rn(fmaxf(v[i] + s.b2[c + i], 0.0f));
            }
    }
    if (!layer_dual<N_H>(s, tbase, t1, s.H1[0], s.H1[1], s.W3, idesc_bf16(ROWS, N3), phase))
        return false;
    {
        float v[16];
        tmem_ld16(tmem_row(tbase, 0), v);
        y[0] = v[0] + s.b3[0];
        y[1] = v[1] + s.b3[1];
        tmem_ld16(tmem_row(t1, 0), v);
        ym[0] = v[0] + s.b3[0];
        ym[1] = v[1] + s.b3[1];
    }
    return true;
}

// Start of a kernel: barrier init and the tensor-memory allocation (warp 0).
template <typename SM>
__device__ __forceinline__ void start_tiles(SM& s, uint32_t ncols) {
    if (threadIdx.x == 0) {
        s.error = 0;
        mbar_init(&s.bar, 1);
        fence_mbar_init();
    }
    if (threadIdx.x < 32) tmem_alloc(&s.taddr, ncols);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

// End of a kernel: after a timed-out wait, one more bounded wait for the
// MMAs in flight; then warp 0 frees the tensor memory.  Returns the error.
template <typename SM>
__device__ __forceinline__ int finish_tiles(SM& s, uint32_t phase, uint32_t ncols) {
    tc_fence_before();
    __syncthreads();
    const int err = s.error;
    if (err && threadIdx.x == 0) mbar_wait(&s.bar, phase);
    __syncthreads();
    if (threadIdx.x < 32) tmem_free(s.taddr, ncols);
    return err;
}

// Builds the operand-layout model from FP32 parameters (one thread per
// element of the largest operand).
__device__ __forceinline__ void build_model_elem(ModelDev* md, const float* __restrict__ p,
                                                 const float* norm, int i) {
    if (i < N_H * K1) {
        const int o = i / K1, k = i % K1;
        float v = 0.0f;
        if (k < N_IN) v = p[P_W1 + o * N_IN + k];
        else if (k == N_IN) v = p[P_B1 + o];
        md->W1[kmaj(o, k, K1)] = __float2bfloat16_rn(v);
    }
    if (i < N_H * N_H) {
        const int o = i / N_H, k = i % N_H;
        md->W2[kmaj(o, k, N_H)] = __float2bfloat16_rn(p[P_W2 + i]);
    }
    if (i < N3 * N_H) {
        const int o = i / N_H, k = i % N_H;
        md->W3[kmaj(o, k, N_H)] = __float2bfloat16_rn(o < N_OUT ? p[P_W3 + o * N_H + k] : 0.0f);
    }
    if (i < N_H) md->b2[i] = p[P_B2 + i];
    if (i < N_OUT) {
        md->b3[i] = p[P_B3 + i];
        md->out_mean[i] = norm[16 + i];
        md->out_std[i] = norm[18 + i];
    }
    if (i < N_IN) {
        md->in_mean[i] = norm[i];
        md->in_inv_std[i] = norm[8 + i];
    }
}

}  // namespace mlp
}  // namespace sfg
