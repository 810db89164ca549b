// learned_step.cu -- the learned form of multi-direct forcing inside the step.
//
// After the membrane-force spread, k_mdf_features interpolates the velocity
// at every marker of a learned channel (the same interpolation as the plain
// sweeps) and forms the network inputs in the marker's local frame;
// k_mdf_seed runs the network on the tensor cores for 128 markers per tile
// and writes the predicted correction back in the lattice frame.  The predictor is
// the odd part of the network in (slip, previous correction): the plain
// iteration's correction is linear in the slip field and vanishes with it.  The step then
// spreads it (seed), runs one plain sweep, and falls back to the plain
// iteration on channels whose no-slip residual is above the threshold.
//
// The network predicts the correction that the plain iteration of K sweeps
// has accumulated before its last sweep (sweeps 1..K-2).  With an exact
// prediction the seed reproduces the plain state before the last sweep (the
// force G that the collision uses), and the one plain sweep that follows is
// the plain iteration's last sweep: the step equals the plain step.
//
// k_harvest writes the inputs and that correction for every marker after
// the plain iteration: the network's training data.
#include "ibm_interp.cuh"
#include "mlp.cuh"
#include "sfg_internal.h"

namespace sfg {

__device__ __forceinline__ bool learned_marker(const ChannelDev* __restrict__ chans,
                                               const MarkerBufs& mb, int m) {
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    return ch.learned && ch.ibm_iterations > 1 && mb.valid[m];
}

// Interpolation after the membrane spread (with the step's tile moments) and
// the network inputs of every marker of a learned channel: u0, feat [M][8] and
// the local tangent frame [M].
template <typename R>
__global__ void k_mdf_features(const ChannelDev* __restrict__ chans,
                               const CapsuleDev* __restrict__ caps, int M, MarkerBufs mb,
                               const int* __restrict__ tile_slot,
                               const typename Mom4<R>::T* __restrict__ mom,
                               const double* __restrict__ acc, float* __restrict__ feat,
                               double2* __restrict__ frame) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M || !learned_marker(chans, mb, m)) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    double unused;
    const double2 u0 = interp_u_mom<R>(ch, mb, m, tile_slot, mom, acc, unused);
    float fe[8];
    double2 t, nrm;
    mdf_features(ch, caps[mb.mk_cap[m]], mb, m, u0, fe, t, nrm);
    float4* out = reinterpret_cast<float4*>(feat + 8 * (size_t)m);
    out[0] = make_float4(fe[0], fe[1], fe[2], fe[3]);
    out[1] = make_float4(fe[4], fe[5], fe[6], fe[7]);
    frame[m] = t;
    mb.u0[m] = u0;
}

// The network's seed for 128 markers per tile on the tensor cores.  The
// predictor is the odd part (N(x) - N(Px)) / 2, P negating the slip and the
// previous correction: no slip and no previous correction give no
// correction, as in the plain iteration.
__global__ void __launch_bounds__(mlp::ROWS)
k_mdf_seed(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
           const float* __restrict__ feat, const double2* __restrict__ frame,
           const mlp::ModelDev* __restrict__ model, unsigned* __restrict__ status) {
    using namespace mlp;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    FwdSmemDual& s = *reinterpret_cast<FwdSmemDual*>(smem_raw);
    load_model(s, model);
    start_tiles(s, DUAL_TMEM_COLS);
    uint32_t phase = 0;
    const int ntiles = (M + ROWS - 1) / ROWS;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int m = tile * ROWS + threadIdx.x;
        const bool active = m < M && learned_marker(chans, mb, m);
        if (!__syncthreads_or(active)) continue;  // uniform: no learned marker in the tile
        float fe[N_IN];
        if (active) {
            const float4* in = reinterpret_cast<const float4*>(feat + 8 * (size_t)m);
            const float4 a = in[0], b = in[1];
            fe[0] = a.x; fe[1] = a.y; fe[2] = a.z; fe[3] = a.w;
            fe[4] = b.x; fe[5] = b.y; fe[6] = b.z; fe[7] = b.w;
        } else {
#pragma unroll
            for (int k = 0; k < N_IN; ++k) fe[k] = 0.0f;
        }
        put_input_row_dual(s, 0, fe, active);
#pragma unroll
        for (int k = 0; k < 4; ++k) fe[k] = -fe[k];
        put_input_row_dual(s, 1, fe, active);
        float y[2], ym[2];
        if (!forward_tile_dual(s, s.taddr, phase, y, ym)) break;
        if (active) {
            const double a = 0.5 * (double)((y[0] - ym[0]) * s.out_std[0]);
            const double b = 0.5 * (double)((y[1] - ym[1]) * s.out_std[1]);
            const double2 t = frame[m];
            const double2 d = make_double2(a * t.x - b * t.y, a * t.y + b * t.x);
            mb.dF[m] = d;
            mb.dFsum[m] = d;
        }
    }
    if (finish_tiles(s, phase, DUAL_TMEM_COLS) && threadIdx.x == 0)
        atomicOr(status, ST_TENSOR_TIMEOUT);
}

__global__ void k_harvest(const ChannelDev* __restrict__ chans, const CapsuleDev* __restrict__ caps,
                          int M, MarkerBufs mb, float* __restrict__ feat,
                          float* __restrict__ label, int* __restrict__ valid) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    const bool ok = ch.ibm_iterations > 1 && mb.valid[m];
    float fe[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    float la[2] = {0, 0};
    if (ok) {
        double2 t, nrm;
        mdf_features(ch, caps[mb.mk_cap[m]], mb, m, mb.u0[m], fe, t, nrm);
        // label: the correction accumulated before the last sweep (the sum
        // minus that sweep's dF), which the seed stands in for
        const double2 d = make_double2(mb.dFsum[m].x - mb.dF[m].x, mb.dFsum[m].y - mb.dF[m].y);
        la[0] = (float)(d.x * t.x + d.y * t.y);
        la[1] = (float)(d.x * nrm.x + d.y * nrm.y);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) feat[(size_t)m * 8 + k] = fe[k];
    label[(size_t)m * 2 + 0] = la[0];
    label[(size_t)m * 2 + 1] = la[1];
    valid[m] = ok ? 1 : 0;
}

cudaError_t prepare_mdf_learned() {
    return cudaFuncSetAttribute(k_mdf_seed, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(mlp::FwdSmemDual));
}

template <typename S, typename R>
void launch_mdf_learned(const ChannelDev* chans, const CapsuleDev* caps, int M,
                        const MarkerBufs& mb, const S* f, TileBufs& tb, int parity,
                        const void* model, float* feat, double2* frame, int grid,
                        unsigned* status, cudaStream_t st) {
    if (M <= 0) return;
    (void)f;
    k_mdf_features<R><<<(M + tb.marker_block - 1) / tb.marker_block, tb.marker_block, 0, st>>>(
        chans, caps, M, mb, tb.tile_slot[parity], static_cast<const typename Mom4<R>::T*>(tb.mom),
        tb.acc0, feat, frame);   // a learned channel's sweep-0 force is in acc0
    const int tiles = (M + mlp::ROWS - 1) / mlp::ROWS;
    const int g = tiles < grid ? tiles : grid;
    k_mdf_seed<<<g, mlp::ROWS, sizeof(mlp::FwdSmemDual), st>>>(
        chans, M, mb, feat, frame, static_cast<const mlp::ModelDev*>(model), status);
}

void launch_harvest(const ChannelDev* chans, const CapsuleDev* caps, int M, const MarkerBufs& mb,
                    float* feat, float* label, int* valid, cudaStream_t st) {
    if (M <= 0) return;
    k_harvest<<<(M + 127) / 128, 128, 0, st>>>(chans, caps, M, mb, feat, label, valid);
}

#define SFG_INST(S, R)                                                                        \
    template void launch_mdf_learned<S, R>(const ChannelDev*, const CapsuleDev*, int,          \
                                           const MarkerBufs&, const S*, TileBufs&, int,        \
                                           const void*, float*, double2*, int, unsigned*,      \
                                           cudaStream_t);
SFG_INST(double, double)
SFG_INST(float, float)
SFG_INST(__half, float)
#undef SFG_INST

}  // namespace sfg
