// mlp.cu -- training and stand-alone inference of the learned-MDF network on
// the tensor cores (tcgen05), plus the C ABI of the trainer object.
//
// A training step over a batch of n samples runs k_mlp_train_tile (one CTA
// per 128 samples: forward, backward and the CTA's partial weight gradients,
// all GEMMs as tcgen05.mma with BF16 operands and FP32 accumulators in tensor
// memory) and k_mlp_adam (sums the partials in a fixed order, so training is
// deterministic, and applies Adam to the FP32 master weights).
//
// Loss: mean over samples and outputs of (y - t)^2 on normalised targets; the
// per-sample output gradient 2 (y - t) / 2 and the batch mean follow the
// reference surrogate network (src/ml/simple_nn.cpp:195-198, :236).
#include <cstring>
#include <string>
#include <vector>

#include "../../include/softflow_gpu.h"
#include "mlp.cuh"

namespace sfg_host {
void set_error(const std::string& msg);
}

namespace sfg {
namespace mlp {

constexpr int NB = 96;  // width of the weight-gradient GEMM (H1^T, X^T, ones, zeros)

struct __align__(1024) BwdSmem {
    __nv_bfloat16 dY[ROWS * K1];     // [128 x 16] A of dH2 (columns 0, 1)
    __nv_bfloat16 W3T[N_H * K1];     // [64 x 16]  B of dH2: (n, k) = W3[k][n]
    __nv_bfloat16 W2T[N_H * N_H];    // [64 x 64]  B of dH1: (n, k) = W2[k][n]
    __nv_bfloat16 dZ2[ROWS * N_H];   // [128 x 64] A of dH1
    __nv_bfloat16 AT[ROWS * ROWS];   // [128 x 128] rows 0..63 dZ2^T, 64..127 dZ1^T
    __nv_bfloat16 BT[NB * ROWS];     // [96 x 128] rows 0..63 H1^T, 64..79 X^T, 80 ones
    float dYf[ROWS * N_OUT];
    float red[ROWS / 32];
};

constexpr size_t TRAIN_SMEM = sizeof(FwdSmem) + sizeof(BwdSmem);

// norm layout: in_mean[8], in_inv_std[8], out_mean[2], out_std[2]
__global__ void k_build_model(const float* __restrict__ p, const float* __restrict__ norm,
                              ModelDev* __restrict__ md) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N_H * N_H) build_model_elem(md, p, norm, i);
}

__global__ void __launch_bounds__(ROWS)
k_mlp_forward(const ModelDev* __restrict__ md, const float* __restrict__ x, int n,
              float* __restrict__ y, unsigned* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FwdSmem& s = *reinterpret_cast<FwdSmem*>(smem_raw);
    load_model(s, md);
    start_tiles(s, 128);
    uint32_t phase = 0;
    const int ntiles = (n + ROWS - 1) / ROWS;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int i = tile * ROWS + threadIdx.x;
        const bool valid = i < n;
        float f[N_IN];
#pragma unroll
        for (int k = 0; k < N_IN; ++k) f[k] = valid ? x[(size_t)i * N_IN + k] : 0.0f;
        put_input_row(s, f, valid);
        float out[2];
        if (!forward_tile(s, s.taddr, phase, out)) break;
        if (valid) {
            y[(size_t)i * 2 + 0] = out[0] * s.out_std[0] + s.out_mean[0];
            y[(size_t)i * 2 + 1] = out[1] * s.out_std[1] + s.out_mean[1];
        }
    }
    if (finish_tiles(s, phase, 128) && threadIdx.x == 0) atomicOr(status, 1u);
}

// One CTA: samples [128 b, 128 b + 128) of the batch.  Writes the CTA's
// partial gradient (N_PARAMS floats) and partial squared error.
__global__ void __launch_bounds__(ROWS)
k_mlp_train_tile(const float* __restrict__ p, const float* __restrict__ norm,
                 const float* __restrict__ x, const float* __restrict__ t, int n, float inv_n,
                 float* __restrict__ part, float* __restrict__ part_loss,
                 unsigned* __restrict__ status) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FwdSmem& s = *reinterpret_cast<FwdSmem*>(smem_raw);
    BwdSmem& b = *reinterpret_cast<BwdSmem*>(smem_raw + sizeof(FwdSmem));
    const int r = threadIdx.x;
    // weights in operand layouts, straight from the FP32 master copy
    for (int i = r; i < N_H * N_H; i += ROWS) {
        const int o = i / N_H, k = i % N_H;
        const float w = p[P_W2 + i];
        s.W2[kmaj(o, k, N_H)] = __float2bfloat16_rn(w);
        b.W2T[kmaj(k, o, N_H)] = __float2bfloat16_rn(w);
    }
    for (int i = r; i < N_H * K1; i += ROWS) {
        const int o = i / K1, k = i % K1;
        float v = 0.0f;
        if (k < N_IN) v = p[P_W1 + o * N_IN + k];
        else if (k == N_IN) v = p[P_B1 + o];
        s.W1[kmaj(o, k, K1)] = __float2bfloat16_rn(v);
        // W3T: (n = o, k) = W3[k][o] for k < 2
        b.W3T[kmaj(o, k, K1)] = __float2bfloat16_rn(k < N_OUT ? p[P_W3 + k * N_H + o] : 0.0f);
    }
    for (int i = r; i < N3 * N_H; i += ROWS) {
        const int o = i / N_H, k = i % N_H;
        s.W3[kmaj(o, k, N_H)] = __float2bfloat16_rn(o < N_OUT ? p[P_W3 + o * N_H + k] : 0.0f);
    }
    if (r < N_H) s.b2[r] = p[P_B2 + r];
    if (r < N_OUT) {
        s.b3[r] = p[P_B3 + r];
        s.out_mean[r] = norm[16 + r];
        s.out_std[r] = norm[18 + r];
    }
    if (r < N_IN) {
        s.in_mean[r] = norm[r];
        s.in_inv_std[r] = norm[8 + r];
    }
    // rows 80..95 of BT: ones (bias gradient of layer 2), then zeros
    for (int k = 80; k < NB; ++k) b.BT[kmaj(k, r, ROWS)] = __float2bfloat16_rn(k == 80 ? 1.0f : 0.0f);
    __syncthreads();
    start_tiles(s, 256);
    uint32_t phase = 0;
    const int i = blockIdx.x * ROWS + r;
    const bool valid = i < n;
    float f[N_IN];
#pragma unroll
    for (int k = 0; k < N_IN; ++k) f[k] = valid ? x[(size_t)i * N_IN + k] : 0.0f;
    put_input_row(s, f, valid);
    float y[2];
    bool ok = forward_tile(s, s.taddr, phase, y);
    float dy0 = 0.0f, dy1 = 0.0f, se = 0.0f;
    if (valid) {
        const float t0 = (t[(size_t)i * 2 + 0] - s.out_mean[0]) / s.out_std[0];
        const float t1 = (t[(size_t)i * 2 + 1] - s.out_mean[1]) / s.out_std[1];
        const float e0 = y[0] - t0, e1 = y[1] - t1;
        se = e0 * e0 + e1 * e1;
        dy0 = e0 * inv_n;
        dy1 = e1 * inv_n;
    }
    b.dYf[r * 2 + 0] = dy0;
    b.dYf[r * 2 + 1] = dy1;
#pragma unroll
    for (int k = 0; k < K1; ++k)
        b.dY[kmaj(r, k, K1)] = __float2bfloat16_rn(k == 0 ? dy0 : (k == 1 ? dy1 : 0.0f));
    // transposed copies of this row's H1 and X for the weight-gradient GEMM
#pragma unroll 8
    for (int c = 0; c < N_H; ++c) b.BT[kmaj(c, r, ROWS)] = s.H1[kmaj(r, c, N_H)];
#pragma unroll
    for (int k = 0; k < K1; ++k) b.BT[kmaj(N_H + k, r, ROWS)] = s.X[kmaj(r, k, K1)];
    const uint32_t tb = s.taddr;
    // dH2 = dY W3 -> columns [0, 64)
    if (ok) ok = layer<K1>(s, tb, b.dY, b.W3T, idesc_bf16(ROWS, N_H), phase);
    if (ok) {
        float v[16];
#pragma unroll
        for (int c = 0; c < N_H; c += 16) {
            tmem_ld16(tmem_row(tb, c), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const bool on = __bfloat162float(s.H2[kmaj(r, c + j, N_H)]) > 0.0f;
                const __nv_bfloat16 d = __float2bfloat16_rn(on ? v[j] : 0.0f);
                b.dZ2[kmaj(r, c + j, N_H)] = d;
                b.AT[kmaj(c + j, r, ROWS)] = d;
            }
        }
    }
    // dH1 = dZ2 W2 -> columns [64, 128)
    if (ok) ok = layer<N_H>(s, tb + 64, b.dZ2, b.W2T, idesc_bf16(ROWS, N_H), phase);
    if (ok) {
        float v[16];
#pragma unroll
        for (int c = 0; c < N_H; c += 16) {
            tmem_ld16(tmem_row(tb, 64 + c), v);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const bool on = __bfloat162float(s.H1[kmaj(r, c + j, N_H)]) > 0.0f;
                b.AT[kmaj(N_H + c + j, r, ROWS)] = __float2bfloat16_rn(on ? v[j] : 0.0f);
            }
        }
    }
    // [dZ2^T; dZ1^T] [H1^T; X^T; 1]^T -> columns [128, 224)
    if (ok) ok = layer<ROWS>(s, tb + 128, b.AT, b.BT, idesc_bf16(ROWS, NB), phase);
    float* gp = part + (size_t)blockIdx.x * N_PARAMS;
    if (ok) {
        float v[16];
        if (r < N_H) {
#pragma unroll
            for (int c = 0; c < N_H; c += 16) {
                tmem_ld16(tmem_row(tb, 128 + c), v);
#pragma unroll
                for (int j = 0; j < 16; ++j) gp[P_W2 + r * N_H + c + j] = v[j];
            }
            tmem_ld16(tmem_row(tb, 128 + 80), v);
            gp[P_B2 + r] = v[0];
        } else {
            // warps 2 and 3: rows 64..127 are dW1 (columns 64..71) and db1 (72)
            const int o = r - N_H;
            tmem_ld16(tmem_row(tb, 128 + 64), v);
#pragma unroll
            for (int k = 0; k < N_IN; ++k) gp[P_W1 + o * N_IN + k] = v[k];
            gp[P_B1 + o] = v[N_IN];
        }
    }
    // layer-3 gradients on the CUDA cores: dW3 = dY^T H2, db3 = sum dY
    __syncthreads();
    {
        const int o = r >> 6, j = r & 63;
        float acc = 0.0f;
        for (int q = 0; q < ROWS; ++q)
            acc = fmaf(b.dYf[q * 2 + o], __bfloat162float(s.H2[kmaj(q, j, N_H)]), acc);
        gp[P_W3 + o * N_H + j] = acc;
        if (r < N_OUT) {
            float d = 0.0f;
            for (int q = 0; q < ROWS; ++q) d += b.dYf[q * 2 + r];
            gp[P_B3 + r] = d;
        }
    }
    // squared error of the CTA
    for (int o = 16; o > 0; o >>= 1) se += __shfl_down_sync(0xffffffffu, se, o);
    if ((r & 31) == 0) b.red[r >> 5] = se;
    if (finish_tiles(s, phase, 256) && r == 0) atomicOr(status, 1u);
    if (r == 0) part_loss[blockIdx.x] = b.red[0] + b.red[1] + b.red[2] + b.red[3];
}

// Sums the CTA partials in CTA order; then Adam (step > 0) or the plain
// gradient into g_out (step == 0).
__global__ void k_mlp_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                           const float* __restrict__ part, int nparts, int step, float lr,
                           float* __restrict__ g_out, const float* __restrict__ part_loss,
                           float loss_scale, float* __restrict__ loss_out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && loss_out) {
        float l = 0.0f;
        for (int c = 0; c < nparts; ++c) l += part_loss[c];
        *loss_out = l * loss_scale;
    }
    if (i >= N_PARAMS) return;
    float g = 0.0f;
    for (int c = 0; c < nparts; ++c) g += part[(size_t)c * N_PARAMS + i];
    if (g_out) g_out[i] = g;
    if (step <= 0) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - powf(b1, (float)step));
    const float vh = vi / (1.0f - powf(b2, (float)step));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

}  // namespace mlp
}  // namespace sfg

// ============================================================== C ABI

using namespace sfg::mlp;

struct sfg_mlp {
    int device = 0;
    float* d_params = nullptr;
    float* d_m = nullptr;
    float* d_v = nullptr;
    float* d_norm = nullptr;
    sfg::mlp::ModelDev* d_model = nullptr;
    float* d_part = nullptr;
    float* d_part_loss = nullptr;
    float* d_loss = nullptr;
    float* d_grad = nullptr;
    unsigned* d_status = nullptr;
    int part_cap = 0;
    int step = 0;
    bool model_dirty = true;
};

namespace {

int fail(int code, const std::string& msg) {
    sfg_host::set_error(msg);
    return code;
}

#define MCU(x)                                                                       \
    do {                                                                             \
        cudaError_t e_ = (x);                                                        \
        if (e_ != cudaSuccess)                                                       \
            return fail(SFG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int ensure_parts(sfg_mlp* m, int nparts) {
    if (nparts <= m->part_cap) return SFG_OK;
    if (m->d_part) cudaFree(m->d_part);
    if (m->d_part_loss) cudaFree(m->d_part_loss);
    m->d_part = nullptr;
    m->d_part_loss = nullptr;
    MCU(cudaMalloc(&m->d_part, sizeof(float) * (size_t)nparts * N_PARAMS));
    MCU(cudaMalloc(&m->d_part_loss, sizeof(float) * nparts));
    m->part_cap = nparts;
    return SFG_OK;
}

int check_status(sfg_mlp* m, cudaStream_t st, const char* who) {
    unsigned s = 0;
    MCU(cudaMemcpyAsync(&s, m->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    MCU(cudaStreamSynchronize(st));
    if (s) return fail(SFG_ERR_CUDA, std::string(who) + ": a tensor-core wait timed out");
    return SFG_OK;
}

int prepare_kernels(int device) {
    static unsigned long long done = 0;  // one bit per device ordinal below 64
    const unsigned long long bit = (device >= 0 && device < 64) ? (1ull << device) : 0ull;
    if (bit && (done & bit)) return SFG_OK;
    MCU(cudaFuncSetAttribute(k_mlp_train_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)TRAIN_SMEM));
    MCU(cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(FwdSmem)));
    done |= bit;
    return SFG_OK;
}

// one batch: partial gradients, then the reduction (+ Adam when step > 0)
int batch_step(sfg_mlp* m, const float* x, const float* t, int n, int step, float lr,
               float* g_out, float* loss_out, cudaStream_t st) {
    const int nparts = (n + ROWS - 1) / ROWS;
    int rc = ensure_parts(m, nparts);
    if (rc) return rc;
    k_mlp_train_tile<<<nparts, ROWS, TRAIN_SMEM, st>>>(m->d_params, m->d_norm, x, t, n,
                                                        1.0f / (float)n, m->d_part,
                                                        m->d_part_loss, m->d_status);
    MCU(cudaGetLastError());
    k_mlp_adam<<<(N_PARAMS + 255) / 256, 256, 0, st>>>(
        m->d_params, m->d_m, m->d_v, m->d_part, nparts, step, lr, g_out, m->d_part_loss,
        1.0f / (2.0f * (float)n), loss_out);
    MCU(cudaGetLastError());
    if (step > 0) m->model_dirty = true;
    return SFG_OK;
}

}  // namespace

extern "C" int sfg_mlp_create(int device, sfg_mlp** out) {
    if (!out) return fail(SFG_ERR_ARG, "sfg_mlp_create: null output");
    *out = nullptr;
    MCU(cudaSetDevice(device));
    int rc = prepare_kernels(device);
    if (rc) return rc;
    sfg_mlp* m = new sfg_mlp();
    m->device = device;
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&m->d_params, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_m, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_v, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_grad, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_norm, sizeof(float) * 20);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_model, sizeof(sfg::mlp::ModelDev));
    if (e == cudaSuccess) e = cudaMalloc(&m->d_loss, sizeof(float) * 4096);
    if (e == cudaSuccess) e = cudaMalloc(&m->d_status, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(m->d_params, 0, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMemset(m->d_m, 0, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMemset(m->d_v, 0, sizeof(float) * N_PARAMS);
    if (e == cudaSuccess) e = cudaMemset(m->d_status, 0, sizeof(unsigned));
    if (e == cudaSuccess) {
        float norm[20];
        for (int i = 0; i < 20; ++i) norm[i] = (i < 8 || (i >= 16 && i < 18)) ? 0.0f : 1.0f;
        e = cudaMemcpy(m->d_norm, norm, sizeof(norm), cudaMemcpyHostToDevice);
    }
    if (e != cudaSuccess) {
        sfg_mlp_destroy(m);
        return fail(SFG_ERR_CUDA, std::string("sfg_mlp_create: ") + cudaGetErrorString(e));
    }
    *out = m;
    return SFG_OK;
}

extern "C" int sfg_mlp_destroy(sfg_mlp* m) {
    if (!m) return SFG_OK;
    cudaSetDevice(m->device);
    for (void* p : {(void*)m->d_params, (void*)m->d_m, (void*)m->d_v, (void*)m->d_norm,
                    (void*)m->d_model, (void*)m->d_part, (void*)m->d_part_loss,
                    (void*)m->d_loss, (void*)m->d_grad, (void*)m->d_status})
        if (p) cudaFree(p);
    delete m;
    return SFG_OK;
}

extern "C" int sfg_mlp_set_params(sfg_mlp* m, const float* params) {
    if (!m || !params) return fail(SFG_ERR_ARG, "sfg_mlp_set_params: null argument");
    MCU(cudaSetDevice(m->device));
    MCU(cudaMemcpy(m->d_params, params, sizeof(float) * N_PARAMS, cudaMemcpyHostToDevice));
    MCU(cudaMemset(m->d_m, 0, sizeof(float) * N_PARAMS));
    MCU(cudaMemset(m->d_v, 0, sizeof(float) * N_PARAMS));
    m->step = 0;
    m->model_dirty = true;
    return SFG_OK;
}

extern "C" int sfg_mlp_get_params(sfg_mlp* m, float* params) {
    if (!m || !params) return fail(SFG_ERR_ARG, "sfg_mlp_get_params: null argument");
    MCU(cudaSetDevice(m->device));
    MCU(cudaDeviceSynchronize());
    MCU(cudaMemcpy(params, m->d_params, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost));
    return SFG_OK;
}

extern "C" int sfg_mlp_set_normalization(sfg_mlp* m, const float* in_mean, const float* in_std,
                                         const float* out_mean, const float* out_std) {
    if (!m || !in_mean || !in_std || !out_mean || !out_std)
        return fail(SFG_ERR_ARG, "sfg_mlp_set_normalization: null argument");
    float norm[20];
    for (int k = 0; k < 8; ++k) {
        if (!(in_std[k] > 0.0f)) return fail(SFG_ERR_ARG, "sfg_mlp_set_normalization: in_std <= 0");
        norm[k] = in_mean[k];
        norm[8 + k] = 1.0f / in_std[k];
    }
    for (int k = 0; k < 2; ++k) {
        if (!(out_std[k] > 0.0f)) return fail(SFG_ERR_ARG, "sfg_mlp_set_normalization: out_std <= 0");
        norm[16 + k] = out_mean[k];
        norm[18 + k] = out_std[k];
    }
    MCU(cudaSetDevice(m->device));
    MCU(cudaMemcpy(m->d_norm, norm, sizeof(norm), cudaMemcpyHostToDevice));
    m->model_dirty = true;
    return SFG_OK;
}

// Device image of the model in operand layout (built when parameters or
// normalisation changed); used by the forward kernel and the step.
int sfg_mlp_model_device(sfg_mlp* m, const void** model, cudaStream_t st) {
    if (m->model_dirty) {
        k_build_model<<<(N_H * N_H + 255) / 256, 256, 0, st>>>(m->d_params, m->d_norm, m->d_model);
        MCU(cudaGetLastError());
        m->model_dirty = false;
    }
    *model = m->d_model;
    return SFG_OK;
}

extern "C" int sfg_mlp_forward(sfg_mlp* m, const float* d_x, int n, float* d_y, void* stream) {
    if (!m || (n > 0 && (!d_x || !d_y))) return fail(SFG_ERR_ARG, "sfg_mlp_forward: null argument");
    if (n < 0) return fail(SFG_ERR_ARG, "sfg_mlp_forward: negative count");
    if (n == 0) return SFG_OK;
    MCU(cudaSetDevice(m->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const void* md = nullptr;
    int rc = sfg_mlp_model_device(m, &md, st);
    if (rc) return rc;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
    const int tiles = (n + ROWS - 1) / ROWS;
    const int grid = tiles < 4 * sms ? tiles : 4 * sms;
    k_mlp_forward<<<grid, ROWS, sizeof(FwdSmem), st>>>(
        static_cast<const sfg::mlp::ModelDev*>(md), d_x, n, d_y, m->d_status);
    MCU(cudaGetLastError());
    return check_status(m, st, "sfg_mlp_forward");
}

extern "C" int sfg_mlp_gradients(sfg_mlp* m, const float* d_x, const float* d_t, int n,
                                 float* grad, float* loss, void* stream) {
    if (!m || !d_x || !d_t || !grad) return fail(SFG_ERR_ARG, "sfg_mlp_gradients: null argument");
    if (n <= 0) return fail(SFG_ERR_ARG, "sfg_mlp_gradients: empty batch");
    MCU(cudaSetDevice(m->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = batch_step(m, d_x, d_t, n, 0, 0.0f, m->d_grad, m->d_loss, st);
    if (rc) return rc;
    if ((rc = check_status(m, st, "sfg_mlp_gradients"))) return rc;
    MCU(cudaMemcpy(grad, m->d_grad, sizeof(float) * N_PARAMS, cudaMemcpyDeviceToHost));
    if (loss) MCU(cudaMemcpy(loss, m->d_loss, sizeof(float), cudaMemcpyDeviceToHost));
    return SFG_OK;
}

extern "C" int sfg_mlp_train(sfg_mlp* m, const float* d_x, const float* d_t, int n, int batch,
                             float lr, float* losses, void* stream) {
    if (!m || !d_x || !d_t) return fail(SFG_ERR_ARG, "sfg_mlp_train: null argument");
    if (n <= 0 || batch <= 0) return fail(SFG_ERR_ARG, "sfg_mlp_train: empty data or batch");
    MCU(cudaSetDevice(m->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int nb = n / batch;
    if (nb < 1) return fail(SFG_ERR_ARG, "sfg_mlp_train: fewer samples than one batch");
    std::vector<float> hl;
    for (int b0 = 0; b0 < nb; b0 += 4096) {
        const int cnt = nb - b0 < 4096 ? nb - b0 : 4096;
        for (int k = 0; k < cnt; ++k) {
            const size_t off = (size_t)(b0 + k) * batch;
            int rc = batch_step(m, d_x + off * N_IN, d_t + off * N_OUT, batch, ++m->step, lr,
                                nullptr, m->d_loss + k, st);
            if (rc) return rc;
        }
        if (losses) {
            MCU(cudaMemcpyAsync(losses + b0, m->d_loss, sizeof(float) * cnt,
                                cudaMemcpyDeviceToHost, st));
        }
    }
    return check_status(m, st, "sfg_mlp_train");
}

extern "C" int sfg_mlp_step_count(sfg_mlp* m, int* steps) {
    if (!m || !steps) return fail(SFG_ERR_ARG, "sfg_mlp_step_count: null argument");
    *steps = m->step;
    return SFG_OK;
}
