// context.cu -- the C ABI (include/softflow_gpu.h): device context, channel
// and capsule registration, per-step kernel sequence (captured in CUDA
// graphs), and state transfer.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/softflow_gpu.h"
#include "lattice.cuh"
#include "sfg_internal.h"
#include "mlp.cuh"

using namespace sfg;

namespace sfg_host {
static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }
}  // namespace sfg_host

static int fail(int code, const std::string& msg) {
    sfg_host::set_error(msg);
    return code;
}

#define CU(x)                                                                           \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if (e_ != cudaSuccess)                                                          \
            return fail(SFG_ERR_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

struct CapsuleHost {
    int type = 0;
    sfg_membrane_params mp;
    sfg_capsule_rest rest;
    std::vector<double> pos, rest_len, rest_ang, rest_ds;
};

struct Pillar {
    int rect;            // 0 circle (a, b) radius c; 1 rectangle [a, c] x [b, d]
    double a, b, c, d;
};

struct ChanHost {
    sfg_channel_params p;
    ChannelDev d;
    std::vector<CapsuleHost> caps;
    std::vector<Pillar> pillars;
    bool has_chem = false;
    sfg_chemistry chem{};
    long long fluid_cells = 0;
};

// Obstacle::contains of CircleObstacle / RectObstacle
// (geometry/circle_obstacle.h:11-15, rect_obstacle.h:9-16).
bool pillar_contains(const Pillar& o, double x, double y) {
    if (o.rect) return x >= o.a && x <= o.c && y >= o.b && y <= o.d;
    const double dx = x - o.a, dy = y - o.b;
    return (dx * dx + dy * dy) <= o.c * o.c;
}

// Cell types of a channel with pillars: ChannelBuilder::applyToField
// (channel_builder.cpp:6-36) followed by LBMSolver::initialize's rows and
// columns (lbm_solver.cpp:130-160).
std::vector<unsigned char> pillar_mask(const sfg_channel_params& p,
                                       const std::vector<Pillar>& pillars) {
    const int nx = p.nx, ny = p.ny;
    std::vector<unsigned char> m((size_t)nx * ny, 0);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x)
            for (const Pillar& o : pillars)
                if (pillar_contains(o, (double)x, (double)y)) {
                    m[(size_t)y * nx + x] = 1;
                    break;
                }
    for (int x = 0; x < nx; ++x) m[x] = m[(size_t)(ny - 1) * nx + x] = 1;
    if (p.boundary_type == SFG_INLET_OUTLET) {
        for (int y = 1; y < ny - 1; ++y) {
            m[(size_t)y * nx] = 2;
            m[(size_t)y * nx + nx - 1] = 3;
        }
    } else if (p.boundary_type == SFG_CLOSED) {
        for (int y = 0; y < ny; ++y) m[(size_t)y * nx] = m[(size_t)y * nx + nx - 1] = 1;
    }
    if (p.periodic_y)
        for (int x = 0; x < nx; ++x) m[x] = m[(size_t)(ny - 1) * nx + x] = 0;
    return m;
}

// InterpolatedBounceBack::initialize (interpolated_bounce_back.cpp:7-54):
// links of non-SOLID nodes into SOLID nodes in (y, x, q) order, the wall
// fraction by 20 bisection steps against every pillar (1 if none is hit).
void build_ibb_links(int chan, const sfg_channel_params& p, const std::vector<unsigned char>& m,
                     const std::vector<Pillar>& pillars, std::vector<IbbLink>& out) {
    static const int CXh[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static const int CYh[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    const int nx = p.nx, ny = p.ny;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            if (m[(size_t)y * nx + x] == 1) continue;
            for (int q = 1; q < 9; ++q) {
                const int xn = x + CXh[q], yn = y + CYh[q];
                if (xn < 0 || xn >= nx || yn < 0 || yn >= ny) continue;
                if (m[(size_t)yn * nx + xn] != 1) continue;
                const double x0 = (double)x, y0 = (double)y;
                const double dx = (double)CXh[q], dy = (double)CYh[q];
                double min_q = 1.0;
                for (const Pillar& o : pillars) {
                    double lo = 0.0, hi = 1.0;
                    for (int it = 0; it < 20; ++it) {
                        const double mid = 0.5 * (lo + hi);
                        const double xm = x0 + mid * dx, ym = y0 + mid * dy;
                        if (pillar_contains(o, xm, ym)) hi = mid;
                        else lo = mid;
                    }
                    if (hi < min_q) min_q = hi;
                }
                out.push_back({chan, x, y, q, min_q});
            }
        }
}

__global__ void k_step_flags(const ChannelDev* __restrict__ chans, int nch, int* stepped,
                             int* adr_pending, int* c_fresh, unsigned* step_ctr,
                             const unsigned* __restrict__ resid_gate,
                             long long* __restrict__ learned_steps,
                             long long* __restrict__ fallbacks) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c == 0) *step_ctr += 1u;
    if (c >= nch) return;
    if (chans[c].learned && chans[c].cap_end > chans[c].cap_begin) {
        learned_steps[c] += 1;
        if (mdf_fallback(resid_gate[c], chans[c].mdf_threshold)) fallbacks[c] += 1;
    }
    if (chans[c].adr) {
        if (chans[c].adr_now) {
            c_fresh[c] = 0;          // this step's scalar step has run
        } else {
            if (adr_pending[c]) c_fresh[c] = 0;
            adr_pending[c] = 1;
        }
    }
    stepped[c] = 1;
}

__global__ void k_flush_flags(int nch, int* adr_pending, int* c_fresh) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    if (adr_pending[c]) c_fresh[c] = 0;
    adr_pending[c] = 0;
}

struct Feq9 {
    double v[9];
};

template <typename S, typename R>
__global__ void k_pop_fill(S* __restrict__ f, ChannelDev ch, Feq9 v) {
    const long long N = (long long)ch.plane;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 9 * N;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / N);
        PopIO<S, R>::store(f + ch.f_off + i, q, (R)v.v[q]);
    }
}

template <typename R>
__global__ void k_scalar_set(const double* __restrict__ C, R* __restrict__ g0, R* __restrict__ g1,
                             R* __restrict__ cf, ChannelDev ch) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / ch.nx), x = (int)(i % ch.nx);
        const long long n = (long long)y * ch.pitch + x;
        const double c = C[i];
        cf[ch.cell_off + n] = (R)c;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const R v = (R)(w_of(q) * c);
            g0[ch.g_off + q * ch.plane + n] = v;
            g1[ch.g_off + q * ch.plane + n] = v;
        }
    }
}

// Scalar state from a saved state: populations g [9][ny][nx] into both
// buffers and the concentration field the next collision reads.
template <typename R>
__global__ void k_scalar_import(const double* __restrict__ C, const double* __restrict__ g,
                                R* __restrict__ g0, R* __restrict__ g1, R* __restrict__ cf,
                                ChannelDev ch) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / ch.nx), x = (int)(i % ch.nx);
        const long long n = (long long)y * ch.pitch + x;
        cf[ch.cell_off + n] = (R)C[i];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const R v = (R)g[q * N + i];
            g0[ch.g_off + q * ch.plane + n] = v;
            g1[ch.g_off + q * ch.plane + n] = v;
        }
    }
}

template <typename R>
__global__ void k_scalar_export(const R* __restrict__ g, ChannelDev ch, double* __restrict__ C,
                                double* __restrict__ gout, const R* __restrict__ cfield,
                                const unsigned char* __restrict__ cov) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / ch.nx), x = (int)(i % ch.nx);
        const long long n = (long long)y * ch.pitch + x;
        R v[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = g[ch.g_off + q * ch.plane + n];
        const R s = v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7] + v[8];
        // a concentration the capsule chemistry overwrote is the stored one
        C[i] = (cov != nullptr && cov[ch.cell_off + n]) ? (double)cfield[ch.cell_off + n] : (double)s;
        if (gout)
            for (int q = 0; q < 9; ++q) gout[q * N + i] = (double)v[q];
    }
}

int io_blocks(long long n) {
    long long g = (n + 255) / 256;
    return (int)std::min<long long>(std::max<long long>(g, 1), 4096);
}

double phi_exact(double r) {
    // Peskin 4-point kernel (delta_function.h:18-26)
    const double ar = std::abs(r);
    if (ar <= 1.0) return 0.125 * (3.0 - 2.0 * ar + std::sqrt(1.0 + 4.0 * ar - 4.0 * ar * ar));
    if (ar <= 2.0) return 0.125 * (5.0 - 2.0 * ar - std::sqrt(-7.0 + 12.0 * ar - 4.0 * ar * ar));
    return 0.0;
}

}  // namespace

struct sfg_context {
    int device = 0;
    int precision = SFG_FP32;
    cudaStream_t stream = nullptr;
    std::vector<ChanHost> ch;
    bool initialized = false;

    // device state
    ChannelDev* d_chans = nullptr;
    RowItem* d_items = nullptr;
    int n_items = 0;
    RowItem* d_items4 = nullptr;
    int n_items4 = 0;
    bool use_vec4 = false;
    RowItem* d_items8 = nullptr;       // 256-cell runs (FP16-shifted storage)
    int n_items8 = 0;
    bool use_vec8 = false;
    bool any_bc = false;                // boundary-aware lattice kernel in use
    RowItem* d_zh_rows = nullptr;       // Zou-He rows (channel, y)
    int n_zh = 0;
    // independent launch groups at the start of a step (contact cell list,
    // force tiles + tile moments) run on side streams, joined by events
    cudaStream_t side[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_fork = nullptr, ev_contact = nullptr, ev_tiles = nullptr, ev_mom = nullptr;
    cudaEvent_t ev_lat1 = nullptr;      // the lattice pass over untouched force tiles
    cudaEvent_t ev_slots = nullptr;     // the step's slot records exist
    // the learned gate's fallback flag beside the last spread, the step's
    // flags beside the marker move
    cudaEvent_t ev_gate = nullptr, ev_pn = nullptr, ev_lat = nullptr, ev_flags = nullptr;
    bool split_lattice = false;         // that pass beside the forcing (8-cell kernel; off:
                                        // the concurrent pass slowed the forcing more than it
                                        // saved on the ensemble)
    // pipelined marker output: snapshots on the context stream, copied to
    // the host on a copy stream while later steps run
    cudaStream_t copy_stream = nullptr;
    // sfg_set_all_populations: upload stream, two staging buffers, events
    cudaStream_t up_stream = nullptr;
    double* d_up[2] = {nullptr, nullptr};
    size_t up_doubles = 0;
    cudaEvent_t up_copied[2] = {nullptr, nullptr}, up_free[2] = {nullptr, nullptr};
    double* d_snap[2] = {nullptr, nullptr};       // [M][2] positions, then [M][2] velocities
    cudaEvent_t ev_snap[2] = {nullptr, nullptr};
    cudaEvent_t ev_copy[2] = {nullptr, nullptr};
    bool copy_pending[2] = {false, false};
    // capsule chemistry of the scalar
    bool any_chem = false;              // also: the scalar step runs inside its step
    sfg_chemistry* d_chem = nullptr;    // [nch]
    double *d_released = nullptr, *d_absorbed = nullptr, *d_Mp = nullptr;   // [NC]
    double* d_gamma = nullptr;          // [M]
    unsigned char* d_cov = nullptr;     // [cells] stored concentration in cfield
    int* d_waves = nullptr;             // [2 NC]
    void* d_boxes = nullptr;            // [NC] footprints
    unsigned char* d_masks = nullptr;   // cell types of channels with pillars
    double* d_pillars = nullptr;        // [pillars][5] of every channel
    bool pillar_repulsion = false;      // some channel has pillars and capsules
    IbbLink* d_ibb = nullptr;           // interpolated bounce-back links by level
    std::vector<int> ibb_level_start;   // [levels + 1]
    void* f[2] = {nullptr, nullptr};
    void* g[2] = {nullptr, nullptr};
    void* cfield = nullptr;
    bool any_adr = false;
    CapsuleDev* d_caps = nullptr;
    int* d_has_prev = nullptr;
    MarkerBufs mb{};
    int M = 0, NC = 0, maxn = 0, Kmax = 1;
    TileBufs tb;
    ContactBufs cb;
    int ncells = 0;
    double* d_phi = nullptr;
    int* d_stepped = nullptr;
    int* d_adr_pending = nullptr;
    int* d_c_fresh = nullptr;
    unsigned* d_status = nullptr;
    unsigned* d_step_ctr = nullptr;
    double* d_io = nullptr;
    size_t io_doubles = 0;
    int spread_grid = 0;
    int persistent_ctas = 296;
    int shared_collision = -1;

    long long steps = 0;
    bool restored = false;              // state restored before the first step
    bool adr_pending_h = false;
    int g_cur = 0;
    cudaGraphExec_t gexec[2] = {nullptr, nullptr};
    bool use_graphs = true;
    bool force_scalar_lattice = false;  // diagnostics: use the one-cell-per-thread kernel
    bool force_vec4_lattice = false;    // diagnostics: four cells per lane in FP16S too
    // learned multi-direct forcing
    void* d_model = nullptr;            // mlp::ModelDev (the context's own copy)
    bool any_learned = false;
    int learned_grid = 592;
    // launch shapes (sfg_autotune): CTAs per SM of the persistent lattice
    // kernel, the spread and the learned seed; 0 = the largest resident count
    int nsm = 148;
    int lattice_cps = 0, spread_cps = 0, learned_cps = 4;
    long long* d_learned_steps = nullptr;  // [nch]
    long long* d_fallbacks = nullptr;      // [nch]
    bool harvest = false;
    float* d_hfeat = nullptr;           // [M][8]
    float* d_hlab = nullptr;            // [M][2]
    int* d_hvalid = nullptr;            // [M]
    int* d_plain_needed = nullptr;      // [1] see TileBufs::plain_needed
    float* d_feat = nullptr;            // [M][8] network inputs of the step
    double2* d_frame = nullptr;         // [M] local tangent of each marker
    // thermo reductions (allocated on first use)
    ThermoPart* d_thermo_parts = nullptr;  // [nch][thermo_bpc]
    int thermo_bpc = 0;                    // blocks per channel (from the largest channel)
    double* d_cap_stats = nullptr;         // [NC][6]
    sfg_thermo_record* d_thermo = nullptr;        // [nch]
    sfg_thermo_record* h_thermo = nullptr;        // pinned [nch]
    double* h_cap_stats = nullptr;         // pinned [NC][6]
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int launches = 0;
    // per-phase timing (profiling mode runs the step eagerly)
    bool profiling = false;
    std::vector<cudaEvent_t> pev;
    std::vector<int> pev_phase;
    float phase_ms[SFG_NUM_PHASES] = {0};

    size_t elem_size() const { return precision == SFG_FP64 ? 8 : (precision == SFG_FP32 ? 4 : 2); }
    size_t real_size() const { return precision == SFG_FP64 ? 8 : 4; }
};

namespace sfg {
int lattice_ctas_per_sm(int precision, bool adr, bool vec8) {
    if (precision == SFG_FP64) return lattice_ctas_per_sm_t<double, double>(adr, false);
    if (precision == SFG_FP32) return lattice_ctas_per_sm_t<float, float>(adr, false);
    return lattice_ctas_per_sm_t<__half, float>(adr, vec8);
}
}  // namespace sfg

// ------------------------------------------------------------------------
// library
// ------------------------------------------------------------------------
extern "C" int sfg_abi_version(void) { return SFG_ABI_VERSION; }
extern "C" const char* sfg_last_error(void) { return sfg_host::g_err.c_str(); }

extern "C" int sfg_create(int device, int precision, sfg_context** out) {
    if (!out) return fail(SFG_ERR_ARG, "sfg_create: null output");
    if (precision < SFG_FP64 || precision > SFG_FP16S)
        return fail(SFG_ERR_ARG, "sfg_create: unknown precision");
    int ndev = 0;
    CU(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return fail(SFG_ERR_ARG, "sfg_create: bad device ordinal");
    CU(cudaSetDevice(device));
    auto* c = new sfg_context();
    c->device = device;
    c->precision = precision;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev1);
    if (e != cudaSuccess) {
        delete c;
        return fail(SFG_ERR_CUDA, std::string("sfg_create: ") + cudaGetErrorString(e));
    }
    *out = c;
    return SFG_OK;
}

static void free_all(sfg_context* c) {
    auto F = [](void* p) {
        if (p) cudaFree(p);
    };
    for (int i = 0; i < 2; ++i) {
        if (c->gexec[i]) cudaGraphExecDestroy(c->gexec[i]);
        c->gexec[i] = nullptr;
        F(c->f[i]);
        F(c->g[i]);
        F(c->tb.tile_slot[i]);
        F(c->tb.fin[i]);
    }
    F(c->cfield);
    F(c->d_chans);
    F(c->d_items);
    F(c->d_items4);
    F(c->d_items8);
    F(c->d_caps);
    F(c->d_has_prev);
    F(c->mb.pos); F(c->mb.vel); F(c->mb.frc); F(c->mb.dF); F(c->mb.ds);
    F(c->mb.rest_len); F(c->mb.rest_ang); F(c->mb.rest_ds); F(c->mb.prev_len);
    F(c->mb.mk_cap); F(c->mb.mk_chan); F(c->mb.ix0); F(c->mb.iy0); F(c->mb.valid);
    F(c->mb.pair_count); F(c->mb.wx); F(c->mb.wy);
    F(c->tb.tile_chan); F(c->tb.tile_flag); F(c->tb.tile_cnt); F(c->tb.cursor);
    F(c->tb.slot_scan); F(c->tb.list_off); F(c->tb.slot_tile); F(c->tb.n_slots);
    F(c->tb.list); F(c->tb.scan_tmp); F(c->tb.acc); F(c->tb.gsnap); F(c->tb.capped);
    F(c->tb.fluid_touched); F(c->tb.acc0); F(c->tb.mom); F(c->tb.slot_info); F(c->tb.slot_order); F(c->tb.slot_rank); F(c->tb.cls_cnt); F(c->tb.spread_ctr); F(c->tb.resid_gate); F(c->tb.resid_plain);
    F(c->mb.u0); F(c->mb.dFsum); F(c->mb.dFprev); F(c->mb.slot8);
    F(c->d_model); F(c->d_learned_steps); F(c->d_fallbacks);
    F(c->d_hfeat); F(c->d_hlab); F(c->d_hvalid); F(c->d_feat); F(c->d_frame); F(c->d_plain_needed);
    F(c->cb.cell_of); F(c->cb.cell_cnt); F(c->cb.cell_start); F(c->cb.cursor); F(c->cb.list);
    F(c->cb.scan_tmp);
    F(c->d_phi); F(c->d_stepped); F(c->d_adr_pending); F(c->d_c_fresh); F(c->d_status);
    F(c->d_step_ctr);
    F(c->d_io);
    F(c->d_zh_rows);
    c->d_zh_rows = nullptr;
    F(c->d_masks);
    F(c->d_ibb);
    F(c->d_pillars);
    c->d_pillars = nullptr;
    F(c->d_chem); F(c->d_released); F(c->d_absorbed); F(c->d_Mp); F(c->d_gamma);
    F(c->d_cov); F(c->d_waves); F(c->d_boxes);
    c->d_chem = nullptr; c->d_released = c->d_absorbed = c->d_Mp = c->d_gamma = nullptr;
    c->d_cov = nullptr; c->d_waves = nullptr; c->d_boxes = nullptr;
    if (c->up_stream) {
        cudaStreamSynchronize(c->up_stream);
        cudaStreamDestroy(c->up_stream);
        c->up_stream = nullptr;
    }
    for (int i = 0; i < 2; ++i) {
        F(c->d_up[i]);
        c->d_up[i] = nullptr;
        if (c->up_copied[i]) cudaEventDestroy(c->up_copied[i]);
        if (c->up_free[i]) cudaEventDestroy(c->up_free[i]);
        c->up_copied[i] = c->up_free[i] = nullptr;
    }
    if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
    for (int i = 0; i < 2; ++i) {
        F(c->d_snap[i]);
        c->d_snap[i] = nullptr;
        if (c->ev_snap[i]) cudaEventDestroy(c->ev_snap[i]);
        if (c->ev_copy[i]) cudaEventDestroy(c->ev_copy[i]);
        c->ev_snap[i] = c->ev_copy[i] = nullptr;
        c->copy_pending[i] = false;
    }
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    c->copy_stream = nullptr;
    for (int i = 0; i < 3; ++i) {
        if (c->side[i]) {
            cudaStreamSynchronize(c->side[i]);
            cudaStreamDestroy(c->side[i]);
        }
        c->side[i] = nullptr;
    }
    for (cudaEvent_t* e : {&c->ev_fork, &c->ev_contact, &c->ev_tiles, &c->ev_mom, &c->ev_lat1, &c->ev_slots,
                           &c->ev_gate, &c->ev_pn, &c->ev_lat, &c->ev_flags}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    c->d_masks = nullptr;
    c->d_ibb = nullptr;
    F(c->d_thermo_parts); F(c->d_cap_stats); F(c->d_thermo);
    if (c->h_thermo) cudaFreeHost(c->h_thermo);
    if (c->h_cap_stats) cudaFreeHost(c->h_cap_stats);
    c->d_thermo_parts = nullptr; c->d_cap_stats = nullptr; c->d_thermo = nullptr;
    c->h_thermo = nullptr; c->h_cap_stats = nullptr;
}

extern "C" int sfg_destroy(sfg_context* c) {
    if (!c) return SFG_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_all(c);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    for (cudaEvent_t e : c->pev) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return SFG_OK;
}

extern "C" int sfg_add_channel(sfg_context* c, const sfg_channel_params* p, int* out) {
    if (!c || !p) return fail(SFG_ERR_ARG, "sfg_add_channel: null argument");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_add_channel: context already initialized");
    if (p->nx < 4 || p->ny < 3) return fail(SFG_ERR_ARG, "sfg_add_channel: need nx >= 4, ny >= 3");
    if (!(p->tau > 0.5)) return fail(SFG_ERR_ARG, "sfg_add_channel: tau must exceed 0.5");
    if (p->collision < 0 || p->collision > 2)
        return fail(SFG_ERR_ARG, "sfg_add_channel: unknown collision model");
    if (p->scalar_enabled && !(p->scalar_D > 0.0))
        return fail(SFG_ERR_ARG, "sfg_add_channel: scalar diffusivity must be positive");
    if (p->rep_r_cut <= 0.0) return fail(SFG_ERR_ARG, "sfg_add_channel: r_cut must be positive");
    if (p->boundary_type < 0 || p->boundary_type > 2)
        return fail(SFG_ERR_ARG, "sfg_add_channel: unknown boundary type");
    if (p->boundary_type == SFG_INLET_OUTLET && p->ny < 3)
        return fail(SFG_ERR_ARG, "sfg_add_channel: a Zou-He channel needs ny >= 3");
    if (p->boundary_type == SFG_INLET_OUTLET && !(p->outlet_density > 0.0))
        return fail(SFG_ERR_ARG, "sfg_add_channel: outlet density must be positive");
    {
        const bool moving = std::fabs(p->top_wall_velocity) > 1e-15 ||
                            std::fabs(p->bottom_wall_velocity) > 1e-15;
        if (p->scalar_enabled && (p->boundary_type != SFG_PERIODIC || moving))
            return fail(SFG_ERR_ARG, "sfg_add_channel: the scalar is supported on periodic "
                                     "channels with resting walls only");
    }
    ChanHost h;
    h.p = *p;
    c->ch.push_back(h);
    if (out) *out = (int)c->ch.size() - 1;
    return SFG_OK;
}

extern "C" int sfg_set_chemistry(sfg_context* c, int channel, const sfg_chemistry* chem) {
    if (!c || !chem) return fail(SFG_ERR_ARG, "sfg_set_chemistry: null argument");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_set_chemistry: context already initialized");
    if (channel < 0 || channel >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_set_chemistry: bad channel");
    if (!c->ch[channel].p.scalar_enabled)
        return fail(SFG_ERR_STATE, "sfg_set_chemistry: the channel has no scalar");
    const int counts[8] = {chem->n_release, chem->n_absorb, chem->n_k_leach, chem->n_C_eq,
                           chem->n_M_p, chem->n_k_adsorb, chem->n_k_desorb, chem->n_Gamma_max};
    for (int k : counts)
        if (k < 0 || k > SFG_CHEM_TYPES)
            return fail(SFG_ERR_ARG, "sfg_set_chemistry: vector lengths must be 0..8");
    c->ch[channel].chem = *chem;
    c->ch[channel].has_chem = true;
    return SFG_OK;
}

extern "C" int sfg_set_capsule_type(sfg_context* c, int channel, int capsule, int type) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_capsule_type: null context");
    if (c->initialized)
        return fail(SFG_ERR_STATE, "sfg_set_capsule_type: context already initialized");
    if (channel < 0 || channel >= (int)c->ch.size() || capsule < 0 ||
        capsule >= (int)c->ch[channel].caps.size() || type < 0)
        return fail(SFG_ERR_ARG, "sfg_set_capsule_type: bad argument");
    c->ch[channel].caps[capsule].type = type;
    return SFG_OK;
}

extern "C" int sfg_get_chemistry_state(sfg_context* c, int chi, double* released,
                                       double* absorbed, double* Mp, double* gamma) {
    if (!c || chi < 0 || chi >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_get_chemistry_state: bad channel");
    if (!c->initialized)
        return fail(SFG_ERR_STATE, "sfg_get_chemistry_state: context not initialized");
    const ChannelDev& d = c->ch[chi].d;
    const int nc = d.cap_end - d.cap_begin, nm = d.mk_end - d.mk_begin;
    CU(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < nc; ++i) {
        if (released) released[i] = 0.0;
        if (absorbed) absorbed[i] = 0.0;
        if (Mp) Mp[i] = -1.0;
    }
    for (int i = 0; i < nm; ++i)
        if (gamma) gamma[i] = 0.0;
    if (!c->any_chem || !c->ch[chi].has_chem) return SFG_OK;
    if (nc > 0) {
        if (released) CU(cudaMemcpy(released, c->d_released + d.cap_begin, sizeof(double) * nc, cudaMemcpyDeviceToHost));
        if (absorbed) CU(cudaMemcpy(absorbed, c->d_absorbed + d.cap_begin, sizeof(double) * nc, cudaMemcpyDeviceToHost));
        if (Mp) CU(cudaMemcpy(Mp, c->d_Mp + d.cap_begin, sizeof(double) * nc, cudaMemcpyDeviceToHost));
    }
    if (nm > 0 && gamma)
        CU(cudaMemcpy(gamma, c->d_gamma + d.mk_begin, sizeof(double) * nm, cudaMemcpyDeviceToHost));
    return SFG_OK;
}

extern "C" int sfg_add_pillar(sfg_context* c, int channel, int kind, double a, double b,
                              double cc, double d) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_add_pillar: null context");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_add_pillar: context already initialized");
    if (channel < 0 || channel >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_add_pillar: bad channel");
    if (kind != SFG_PILLAR_CIRCLE && kind != SFG_PILLAR_RECT)
        return fail(SFG_ERR_ARG, "sfg_add_pillar: unknown pillar kind");

    if (c->ch[channel].p.scalar_enabled)
        return fail(SFG_ERR_ARG, "sfg_add_pillar: pillars cannot share a channel with the scalar");
    Pillar o;
    if (kind == SFG_PILLAR_CIRCLE) {
        o = {0, a, b, cc, 0.0};
    } else {   // RectObstacle normalises its corners (rect_obstacle.h:9-11)
        o = {1, std::min(a, cc), std::min(b, d), std::max(a, cc), std::max(b, d)};
    }
    c->ch[channel].pillars.push_back(o);
    return SFG_OK;
}

extern "C" int sfg_add_capsule(sfg_context* c, int channel, const sfg_membrane_params* mp,
                               const sfg_capsule_rest* rest, const double* pos,
                               const double* rest_len, const double* rest_ang,
                               const double* rest_ds, int* out) {
    if (!c || !mp || !rest || !pos || !rest_len)
        return fail(SFG_ERR_ARG, "sfg_add_capsule: null argument");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_add_capsule: context already initialized");
    if (channel < 0 || channel >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_add_capsule: bad channel");
    if (c->ch[channel].p.boundary_type != SFG_PERIODIC)
        return fail(SFG_ERR_ARG, "sfg_add_capsule: capsules need a channel periodic in x");

    if (rest->num_nodes < 3) return fail(SFG_ERR_ARG, "sfg_add_capsule: need >= 3 nodes");
    if (mp->use_helfrich && (!rest_ang || !rest_ds))
        return fail(SFG_ERR_ARG, "sfg_add_capsule: Helfrich bending needs rest angles");
    CapsuleHost ch;
    ch.mp = *mp;
    ch.rest = *rest;
    const int n = rest->num_nodes;
    ch.pos.assign(pos, pos + 2 * n);
    ch.rest_len.assign(rest_len, rest_len + n);
    if (rest_ang) ch.rest_ang.assign(rest_ang, rest_ang + n);
    else ch.rest_ang.assign(n, 0.0);
    if (rest_ds) ch.rest_ds.assign(rest_ds, rest_ds + n);
    else ch.rest_ds.assign(n, 0.0);
    c->ch[channel].caps.push_back(std::move(ch));
    if (out) *out = (int)c->ch[channel].caps.size() - 1;
    return SFG_OK;
}

template <typename T>
static cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc((void**)p, std::max<size_t>(n, 1) * sizeof(T));
}

// ------------------------------------------------------------------------
// initialize
// ------------------------------------------------------------------------
// Grid sizes from the tuned CTAs-per-SM counts (0 = the resident maximum).
static void apply_launch_config(sfg_context* c) {
    const int lat_max = lattice_ctas_per_sm(c->precision, c->any_adr && !c->any_chem, c->use_vec8);
    const int spr_max = spread_blocks_per_sm(c->precision == SFG_FP64);
    const int lat = c->lattice_cps > 0 ? std::min(c->lattice_cps, lat_max) : lat_max;
    const int spr = c->spread_cps > 0 ? std::min(c->spread_cps, spr_max) : spr_max;
    c->persistent_ctas = c->nsm * lat;
    c->spread_grid = std::max(1, std::min((c->tb.max_slots + 7) / 8, c->nsm * spr));
    c->learned_grid = c->nsm * std::max(1, std::min(c->learned_cps, 6));
}

extern "C" int sfg_initialize(sfg_context* c) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_initialize: null context");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_initialize: already initialized");
    if (c->ch.empty()) return fail(SFG_ERR_STATE, "sfg_initialize: no channel");
    CU(cudaSetDevice(c->device));
    const int nch = (int)c->ch.size();
    long long cell_off = 0;
    int tile_base = 0, cell_base = 0, cap_base = 0, mk_base = 0;
    std::vector<RowItem> items, items4, items8, zh_rows;
    std::vector<unsigned char> masks;
    std::vector<long long> mask_off;
    std::vector<IbbLink> links;
    std::vector<CapsuleDev> caps;
    bool all_vec4 = true, all_vec8 = true;
    std::vector<double> pos, rest_len, rest_ang, rest_ds;
    std::vector<int> mk_cap, mk_chan, tile_chan;
    c->any_adr = false;
    c->any_bc = false;
    c->any_chem = false;
    c->maxn = 0;
    c->Kmax = 1;
    for (int ci = 0; ci < nch; ++ci) {
        ChanHost& h = c->ch[ci];
        const sfg_channel_params& p = h.p;
        ChannelDev d{};
        d.nx = p.nx;
        d.ny = p.ny;
        d.pitch = (p.nx + 31) / 32 * 32;
        d.periodic_y = p.periodic_y ? 1 : 0;
        d.plane = (long long)d.ny * d.pitch;
        d.cell_off = cell_off;
        d.f_off = 9 * cell_off;
        d.g_off = 9 * cell_off;
        cell_off += d.plane;
        d.collision = p.collision;
        d.ibm_iterations = p.ibm_iterations > 1 ? p.ibm_iterations : 1;
        d.tau = p.tau;
        d.omega = 1.0 / p.tau;
        d.mrt_se = p.mrt_se;
        d.mrt_s_eps = p.mrt_s_eps;
        d.mrt_sq = p.mrt_sq;
        d.body_fx = p.body_fx;
        d.body_fy = p.body_fy;
        d.max_force = p.max_lattice_force;
        {   // capped body force on FLUID cells away from the markers
            double fx = 0.0 + p.body_fx, fy = 0.0 + p.body_fy;
            const double Fm = p.max_lattice_force, f2 = fx * fx + fy * fy;
            if (f2 > Fm * Fm) {
                const double sc = Fm / std::sqrt(f2);
                fx *= sc;
                fy *= sc;
            }
            d.F_uni_x = fx;
            d.F_uni_y = fy;
        }
        d.dt = p.dt;
        d.bc_x = p.boundary_type;
        d.u_in = p.inlet_velocity;
        d.rho_out = p.outlet_density;
        d.u_top = p.top_wall_velocity;
        d.u_bot = p.bottom_wall_velocity;
        d.bc_active = (p.boundary_type != SFG_PERIODIC ||
                       (!p.periodic_y && (std::fabs(p.top_wall_velocity) > 1e-15 ||
                                          std::fabs(p.bottom_wall_velocity) > 1e-15))) ? 1 : 0;
        d.adr = p.scalar_enabled ? 1 : 0;
        d.adr_periodic_y = p.scalar_periodic_y ? 1 : 0;
        d.omega_s = 1.0 / (3.0 * p.scalar_D + 0.5);
        c->any_adr |= d.adr != 0;
        d.chem = h.has_chem ? 1 : 0;
        c->any_chem |= h.has_chem;
        d.tiles_x = (p.nx + TILE_W - 1) / TILE_W;
        d.tiles_y = (p.ny + TILE_H - 1) / TILE_H;
        d.tile_base = tile_base;
        tile_base += d.tiles_x * d.tiles_y;
        for (int t = 0; t < d.tiles_x * d.tiles_y; ++t) tile_chan.push_back(ci);
        // capsules of this channel, channel-major
        d.cap_begin = cap_base;
        d.mk_begin = mk_base;
        for (const CapsuleHost& cp : h.caps) {
            CapsuleDev cd{};
            cd.off = mk_base;
            cd.n = cp.rest.num_nodes;
            cd.chan = ci;
            cd.model = cp.mp.model;
            cd.use_helfrich = cp.mp.use_helfrich;
            cd.k_stretch = cp.mp.k_stretch;
            cd.G_s = cp.mp.G_s;
            cd.C_skalak = cp.mp.C_skalak;
            cd.wlc_L_max_ratio = cp.mp.wlc_L_max_ratio;
            cd.wlc_kBT_p = cp.rest.wlc_kBT_p;
            cd.wlc_k_pow = cp.rest.wlc_k_pow;
            cd.k_bend = cp.mp.k_bend;
            cd.k_area = cp.mp.k_area;
            cd.k_perimeter = cp.mp.k_perimeter;
            cd.gamma_visc = cp.mp.gamma_visc;
            cd.eta_membrane = cp.mp.eta_membrane;
            cd.rest_area = cp.rest.rest_area;
            cd.rest_perimeter = cp.rest.rest_perimeter;
            cd.periodic_nx = p.nx;
            cd.type = cp.type;
            caps.push_back(cd);
            c->maxn = std::max(c->maxn, cd.n);
            for (int k = 0; k < cd.n; ++k) {
                pos.push_back(cp.pos[2 * k]);
                pos.push_back(cp.pos[2 * k + 1]);
                rest_len.push_back(cp.rest_len[k]);
                rest_ang.push_back(cp.rest_ang[k]);
                rest_ds.push_back(cp.rest_ds[k]);
                mk_cap.push_back(cap_base);
                mk_chan.push_back(ci);
            }
            mk_base += cd.n;
            ++cap_base;
        }
        d.cap_end = cap_base;
        d.mk_end = mk_base;
        if (d.cap_end > d.cap_begin) c->Kmax = std::max(c->Kmax, d.ibm_iterations);
        // contact cell list geometry (cell_list.h:36-87, periodic in x)
        d.y_bot = 0.5;
        d.y_top = (double)p.ny - 1.5;
        {
            const double x_extent = (double)p.nx;
            d.ncx = std::max(1, (int)std::floor(x_extent / p.rep_r_cut));
            d.ncy = std::max(1, (int)std::floor((d.y_top - d.y_bot) / p.rep_r_cut));
            d.cdx = x_extent / (double)d.ncx;
            d.cdy = (d.y_top - d.y_bot) / (double)d.ncy;
        }
        d.brute_contact = (d.mk_end - d.mk_begin) <= 100 ? 1 : 0;
        d.cell_base = cell_base;
        if (!d.brute_contact) cell_base += d.ncx * d.ncy;
        d.rep_epsilon = p.rep_epsilon;
        d.rep_sigma = p.rep_sigma;
        d.rep_r_cut = p.rep_r_cut;
        d.rep_damping = p.rep_damping_normal;
        d.rep_friction = p.rep_friction;
        d.rep_power = p.rep_power;
        // lattice work items: 32-cell row runs (one warp each)
        const int y0 = p.periodic_y ? 0 : 1, y1 = p.periodic_y ? p.ny : p.ny - 1;
        for (int y = y0; y < y1; ++y)
            for (int x0 = 0; x0 < p.nx; x0 += ITEM_CELLS)
                items.push_back({ci, y, x0, std::min(ITEM_CELLS, p.nx - x0)});
        if (p.nx % 4 != 0) all_vec4 = false;
        if (p.nx % 8 != 0) all_vec8 = false;
        for (int y = y0; y < y1; ++y)
            for (int x0 = 0; x0 < p.nx; x0 += VEC_RUN)
                items4.push_back({ci, y, x0, std::min(VEC_RUN, p.nx - x0)});
        {   // 256-cell runs over the channel's rows in row-major order (a run
            // continues over row ends; nx % 8 == 0 keeps lanes inside rows)
            const long long ncell = (long long)(y1 - y0) * p.nx;
            for (long long o = 0; o < ncell; o += VEC8_RUN)
                items8.push_back({ci, y0 + (int)(o / p.nx), (int)(o % p.nx),
                                  (int)std::min<long long>(VEC8_RUN, ncell - o)});
        }
        h.fluid_cells = 0;
        if (!h.pillars.empty()) {
            const std::vector<unsigned char> m = pillar_mask(p, h.pillars);
            for (unsigned char k : m) h.fluid_cells += k == CK_FLUID;
            mask_off.push_back((long long)masks.size());
            masks.insert(masks.end(), m.begin(), m.end());
            d.bc_active = 1;
            if (p.use_interpolated_bb) build_ibb_links(ci, p, m, h.pillars, links);
        } else {
            mask_off.push_back(-1);
            for (int y = 0; y < p.ny; ++y)
                for (int x = 0; x < p.nx; ++x) h.fluid_cells += cell_kind(d, x, y) == CK_FLUID;
        }
        if (d.bc_active) c->any_bc = true;
        if (d.bc_x == SFG_INLET_OUTLET)
            for (int y = 1; y < p.ny - 1; ++y) zh_rows.push_back({ci, y, 0, 1});
        h.d = d;
    }
    c->M = mk_base;
    c->NC = cap_base;
    c->ncells = cell_base;
    c->n_items = (int)items.size();
    c->maxn = (c->maxn + 31) / 32 * 32;
    if (membrane_smem_bytes(c->maxn) > 227 * 1024)
        return fail(SFG_ERR_CAPACITY, "sfg_initialize: capsules with more than 640 nodes");
    if (c->maxn > 0) CU(prepare_membrane(c->maxn));
    CU(prepare_spread());

    {   // pillar shapes for the obstacle repulsion of the markers
        std::vector<double> pl;
        std::vector<int> pl_off(nch, 0);
        c->pillar_repulsion = false;
        for (int i = 0; i < nch; ++i) {
            pl_off[i] = (int)pl.size();
            for (const Pillar& o : c->ch[i].pillars) {
                pl.push_back((double)o.rect);
                pl.push_back(o.a);
                pl.push_back(o.b);
                pl.push_back(o.c);
                pl.push_back(o.d);
            }
            c->ch[i].d.n_pillars = (int)c->ch[i].pillars.size();
            if (!c->ch[i].pillars.empty() && !c->ch[i].caps.empty()) c->pillar_repulsion = true;
        }
        if (!pl.empty()) {
            CU(dalloc(&c->d_pillars, pl.size()));
            CU(cudaMemcpy(c->d_pillars, pl.data(), sizeof(double) * pl.size(),
                          cudaMemcpyHostToDevice));
            for (int i = 0; i < nch; ++i)
                if (c->ch[i].d.n_pillars > 0) c->ch[i].d.pillars = c->d_pillars + pl_off[i];
        }
    }
    if (!masks.empty()) {
        CU(dalloc(&c->d_masks, masks.size()));
        CU(cudaMemcpy(c->d_masks, masks.data(), masks.size(), cudaMemcpyHostToDevice));
        for (int i = 0; i < nch; ++i)
            if (mask_off[i] >= 0) c->ch[i].d.mask = c->d_masks + mask_off[i];
    }
    c->ibb_level_start.clear();
    if (!links.empty()) {
        // levels: a link runs after every earlier link that writes what it
        // reads or reads what it writes (the reference applies them in order)
        std::unordered_map<long long, int> max_w, max_r;
        std::vector<int> level(links.size());
        int nlev = 0;
        auto key = [&](const IbbLink& l, int x, int y, int q) {
            return ((long long)l.chan << 40) | ((long long)(y * c->ch[l.chan].p.nx + x) << 4) | q;
        };
        static const int CXh[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
        static const int CYh[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
        static const int OPh[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
        for (size_t i = 0; i < links.size(); ++i) {
            const IbbLink& l = links[i];
            const int nx = c->ch[l.chan].p.nx, ny = c->ch[l.chan].p.ny;
            std::vector<long long> reads = {key(l, l.x, l.y, l.q), key(l, l.x, l.y, OPh[l.q])};
            int xu = l.x - CXh[l.q];
            const int yu = l.y - CYh[l.q];
            if (c->ch[l.chan].p.boundary_type == SFG_PERIODIC) xu = ((xu % nx) + nx) % nx;
            if (xu >= 0 && xu < nx && yu >= 0 && yu < ny) reads.push_back(key(l, xu, yu, l.q));
            const long long w = key(l, l.x, l.y, OPh[l.q]);
            int lv = 0;
            for (long long r : reads) {
                auto it = max_w.find(r);
                if (it != max_w.end()) lv = std::max(lv, it->second + 1);
            }
            auto ir = max_r.find(w);
            if (ir != max_r.end()) lv = std::max(lv, ir->second + 1);
            auto iw = max_w.find(w);
            if (iw != max_w.end()) lv = std::max(lv, iw->second + 1);
            level[i] = lv;
            nlev = std::max(nlev, lv + 1);
            for (long long r : reads) max_r[r] = std::max(max_r.count(r) ? max_r[r] : 0, lv);
            max_w[w] = lv;
        }
        std::vector<IbbLink> sorted;
        sorted.reserve(links.size());
        c->ibb_level_start.push_back(0);
        for (int lv = 0; lv < nlev; ++lv) {
            for (size_t i = 0; i < links.size(); ++i)
                if (level[i] == lv) sorted.push_back(links[i]);
            c->ibb_level_start.push_back((int)sorted.size());
        }
        CU(dalloc(&c->d_ibb, sorted.size()));
        CU(cudaMemcpy(c->d_ibb, sorted.data(), sizeof(IbbLink) * sorted.size(),
                      cudaMemcpyHostToDevice));
    }
    // with capsule chemistry the scalar step runs inside its own step
    for (int i = 0; i < nch; ++i) c->ch[i].d.adr_now = (c->any_chem && c->ch[i].d.adr) ? 1 : 0;
    std::vector<ChannelDev> dch(nch);
    for (int i = 0; i < nch; ++i) dch[i] = c->ch[i].d;
    CU(dalloc(&c->d_chans, nch));
    CU(cudaMemcpy(c->d_chans, dch.data(), sizeof(ChannelDev) * nch, cudaMemcpyHostToDevice));
    CU(dalloc(&c->d_items, items.size()));
    CU(cudaMemcpy(c->d_items, items.data(), sizeof(RowItem) * items.size(), cudaMemcpyHostToDevice));
    c->use_vec4 = all_vec4 && !c->force_scalar_lattice && !c->any_bc;
    c->use_vec8 = c->use_vec4 && all_vec8 && c->precision == SFG_FP16S && !c->force_vec4_lattice;
    if (c->any_bc && c->any_adr)
        return fail(SFG_ERR_ARG, "sfg_initialize: the scalar cannot share a context with "
                                 "Zou-He, closed or moving-wall channels");
    c->n_zh = (int)zh_rows.size();
    if (c->n_zh > 0) {
        CU(dalloc(&c->d_zh_rows, zh_rows.size()));
        CU(cudaMemcpy(c->d_zh_rows, zh_rows.data(), sizeof(RowItem) * zh_rows.size(),
                      cudaMemcpyHostToDevice));
    }
    c->shared_collision = c->ch[0].p.collision;
    for (const ChanHost& h : c->ch)
        if (h.p.collision != c->shared_collision) c->shared_collision = -1;
    c->n_items8 = (int)items8.size();
    CU(dalloc(&c->d_items8, items8.size()));
    CU(cudaMemcpy(c->d_items8, items8.data(), sizeof(RowItem) * items8.size(),
                  cudaMemcpyHostToDevice));
    c->n_items4 = (int)items4.size();
    CU(dalloc(&c->d_items4, items4.size()));
    CU(cudaMemcpy(c->d_items4, items4.data(), sizeof(RowItem) * items4.size(),
                  cudaMemcpyHostToDevice));

    // populations
    const size_t nelem = 9 * (size_t)cell_off;
    for (int i = 0; i < 2; ++i) CU(cudaMalloc(&c->f[i], nelem * c->elem_size()));
    if (c->any_adr) {
        for (int i = 0; i < 2; ++i) {
            CU(cudaMalloc(&c->g[i], nelem * c->real_size()));
            CU(cudaMemset(c->g[i], 0, nelem * c->real_size()));
        }
        CU(cudaMalloc(&c->cfield, (size_t)cell_off * c->real_size()));
        CU(cudaMemset(c->cfield, 0, (size_t)cell_off * c->real_size()));
        if (c->any_chem) {
            CU(cudaMalloc(&c->d_cov, (size_t)cell_off));
            CU(cudaMemset(c->d_cov, 0, (size_t)cell_off));
        }
    }
    for (int ci = 0; ci < nch; ++ci) {
        const ChannelDev& d = c->ch[ci].d;
        Feq9 v;
        // feq(rho0, 0, 0) in the form of lattice.h:35-39
        const double cs2 = 1.0 / 3.0, cs4 = cs2 * cs2;
        for (int q = 0; q < 9; ++q) {
            const double eu = 0.0, uu = 0.0;
            v.v[q] = w_of(q) * c->ch[ci].p.rho0 *
                     (1.0 + eu / cs2 + (eu * eu) / (2.0 * cs4) - uu / (2.0 * cs2));
        }
        for (int i = 0; i < 2; ++i) {
            if (c->precision == SFG_FP64)
                k_pop_fill<double, double><<<io_blocks(9 * d.plane), 256, 0, c->stream>>>(
                    (double*)c->f[i], d, v);
            else if (c->precision == SFG_FP32)
                k_pop_fill<float, float><<<io_blocks(9 * d.plane), 256, 0, c->stream>>>(
                    (float*)c->f[i], d, v);
            else
                k_pop_fill<__half, float><<<io_blocks(9 * d.plane), 256, 0, c->stream>>>(
                    (__half*)c->f[i], d, v);
        }
    }
    CU(cudaGetLastError());

    // markers
    const int M = c->M;
    CU(dalloc(&c->mb.pos, M));
    CU(dalloc(&c->mb.vel, M));
    CU(dalloc(&c->mb.frc, M));
    CU(dalloc(&c->mb.dF, M));
    CU(dalloc(&c->mb.ds, M));
    CU(dalloc(&c->mb.rest_len, M));
    CU(dalloc(&c->mb.rest_ang, M));
    CU(dalloc(&c->mb.rest_ds, M));
    CU(dalloc(&c->mb.prev_len, M));
    CU(dalloc(&c->mb.mk_cap, M));
    CU(dalloc(&c->mb.mk_chan, M));
    CU(dalloc(&c->mb.ix0, M));
    CU(dalloc(&c->mb.iy0, M));
    CU(dalloc(&c->mb.valid, M));
    CU(dalloc(&c->mb.pair_count, M));
    CU(dalloc(&c->mb.wx, 4LL * M));
    CU(dalloc(&c->mb.wy, 4LL * M));
    CU(dalloc(&c->d_caps, c->NC));
    CU(dalloc(&c->d_has_prev, c->NC));
    if (c->any_chem) {
        // chemistry state as the reference sizes it at its first call
        // (advection_diffusion.cpp:300-316): nothing released or absorbed,
        // reservoirs infinite (-1) unless M_p_initial[type] > 0, no coverage
        std::vector<sfg_chemistry> chp(nch);
        for (int i = 0; i < nch; ++i) chp[i] = c->ch[i].chem;
        CU(dalloc(&c->d_chem, nch));
        CU(cudaMemcpy(c->d_chem, chp.data(), sizeof(sfg_chemistry) * nch, cudaMemcpyHostToDevice));
        const int NCc = std::max(c->NC, 1);
        CU(dalloc(&c->d_released, NCc));
        CU(dalloc(&c->d_absorbed, NCc));
        CU(dalloc(&c->d_Mp, NCc));
        CU(dalloc(&c->d_gamma, std::max(M, 1)));
        CU(dalloc(&c->d_waves, 2 * NCc));
        CU(cudaMalloc(&c->d_boxes, chem_box_bytes() * NCc));
        CU(cudaMemset(c->d_released, 0, sizeof(double) * NCc));
        CU(cudaMemset(c->d_absorbed, 0, sizeof(double) * NCc));
        CU(cudaMemset(c->d_gamma, 0, sizeof(double) * std::max(M, 1)));
        std::vector<double> mp(NCc, -1.0);
        for (int k = 0; k < c->NC; ++k) {
            const sfg_chemistry& ck = c->ch[caps[k].chan].chem;
            const int t = caps[k].type;
            if (t >= 0 && t < ck.n_M_p && ck.M_p_initial[t] > 0.0) mp[k] = ck.M_p_initial[t];
        }
        CU(cudaMemcpy(c->d_Mp, mp.data(), sizeof(double) * NCc, cudaMemcpyHostToDevice));
    }
    if (M > 0) {
        CU(cudaMemcpy(c->mb.pos, pos.data(), sizeof(double) * 2 * M, cudaMemcpyHostToDevice));
        CU(cudaMemset(c->mb.vel, 0, sizeof(double2) * M));
        CU(cudaMemset(c->mb.frc, 0, sizeof(double2) * M));
        CU(cudaMemset(c->mb.dF, 0, sizeof(double2) * M));
        CU(cudaMemset(c->mb.pair_count, 0, sizeof(int) * M));
        CU(cudaMemcpy(c->mb.rest_len, rest_len.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
        // Kelvin-Voigt previous lengths start at the rest lengths (capsule.cpp:85-86)
        CU(cudaMemcpy(c->mb.prev_len, rest_len.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(c->mb.rest_ang, rest_ang.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(c->mb.rest_ds, rest_ds.data(), sizeof(double) * M, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(c->mb.mk_cap, mk_cap.data(), sizeof(int) * M, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(c->mb.mk_chan, mk_chan.data(), sizeof(int) * M, cudaMemcpyHostToDevice));
        CU(cudaMemcpy(c->d_caps, caps.data(), sizeof(CapsuleDev) * c->NC, cudaMemcpyHostToDevice));
        CU(cudaMemset(c->d_has_prev, 0, sizeof(int) * c->NC));
    }

    // force tiles
    TileBufs& tb = c->tb;
    tb.T = tile_base;
    tb.max_slots = M > 0 ? (int)std::min<long long>(tile_base, 8LL * M) : 1;
    const int T = tb.T;
    CU(dalloc(&tb.tile_chan, T));
    CU(cudaMemcpy(tb.tile_chan, tile_chan.data(), sizeof(int) * T, cudaMemcpyHostToDevice));
    CU(dalloc(&tb.tile_flag, T));
    CU(dalloc(&tb.tile_cnt, T));
    CU(dalloc(&tb.cursor, T));
    CU(dalloc(&tb.slot_scan, T));
    CU(dalloc(&tb.list_off, T));
    for (int i = 0; i < 2; ++i) {
        CU(dalloc(&tb.tile_slot[i], T));
        CU(cudaMemset(tb.tile_slot[i], 0xff, sizeof(int) * std::max(T, 1)));
        CU(cudaMalloc(&tb.fin[i], (size_t)tb.max_slots * 2 * TILE_CELLS * c->real_size()));
    }
    CU(dalloc(&tb.slot_tile, tb.max_slots));
    CU(dalloc(&tb.slot_info, tb.max_slots));
    CU(dalloc(&tb.slot_order, tb.max_slots));
    CU(dalloc(&tb.slot_rank, tb.max_slots));
    CU(dalloc(&tb.cls_cnt, SLOT_CLASSES));
    tb.n_spread_ctr = c->Kmax + 3;
    CU(dalloc(&tb.spread_ctr, tb.n_spread_ctr));
    CU(dalloc(&tb.n_slots, 1));
    CU(cudaMemset(tb.n_slots, 0, sizeof(int)));
    CU(dalloc(&tb.list, 8LL * M));
    CU(dalloc(&tb.scan_tmp, scan_tmp_ints(T)));
    CU(dalloc(&tb.acc, (size_t)tb.max_slots * 2 * TILE_CELLS));
    CU(cudaMalloc(&tb.gsnap, (size_t)tb.max_slots * 2 * TILE_CELLS * c->real_size()));
    if (c->Kmax > 1) CU(cudaMalloc(&tb.mom, (size_t)tb.max_slots * TILE_CELLS * 4 * c->real_size()));
    CU(dalloc(&tb.capped, nch));
    CU(dalloc(&tb.fluid_touched, nch));
    CU(cudaMemset(tb.capped, 0, sizeof(int) * nch));
    CU(cudaMemset(tb.fluid_touched, 0, sizeof(int) * nch));
    CU(dalloc(&tb.resid_gate, nch));
    CU(dalloc(&tb.resid_plain, nch));
    CU(cudaMemset(tb.resid_gate, 0, sizeof(unsigned) * nch));
    CU(cudaMemset(tb.resid_plain, 0, sizeof(unsigned) * nch));
    CU(dalloc(&c->d_learned_steps, nch));
    CU(dalloc(&c->d_fallbacks, nch));
    CU(cudaMemset(c->d_learned_steps, 0, sizeof(long long) * nch));
    CU(cudaMemset(c->d_fallbacks, 0, sizeof(long long) * nch));
    // forcing state of the learned form (zero before the first step)
    CU(dalloc(&c->mb.u0, M));
    CU(dalloc(&c->mb.dFsum, M));
    CU(dalloc(&c->mb.dFprev, M));
    CU(dalloc(&c->mb.slot8, 8LL * M));
    if (M > 0) {
        CU(cudaMemset(c->mb.u0, 0, sizeof(double2) * M));
        CU(cudaMemset(c->mb.dFsum, 0, sizeof(double2) * M));
        CU(cudaMemset(c->mb.dFprev, 0, sizeof(double2) * M));
    }

    // contact cells
    CU(dalloc(&c->cb.cell_of, M));
    CU(dalloc(&c->cb.cell_cnt, c->ncells));
    CU(dalloc(&c->cb.cell_start, c->ncells));
    CU(dalloc(&c->cb.cursor, c->ncells));
    CU(dalloc(&c->cb.list, M));
    CU(dalloc(&c->cb.scan_tmp, scan_tmp_ints(c->ncells)));
    CU(cudaMemset(c->cb.cell_cnt, 0, sizeof(int) * std::max(c->ncells, 1)));
    CU(cudaMemset(c->cb.cell_start, 0, sizeof(int) * std::max(c->ncells, 1)));

    // Peskin table (delta_function.h:29-37)
    {
        std::vector<double> tbl(1025);
        for (int i = 0; i <= 1024; ++i) tbl[i] = phi_exact(2.0 * static_cast<double>(i) / 1024);
        CU(dalloc(&c->d_phi, 1025));
        CU(cudaMemcpy(c->d_phi, tbl.data(), sizeof(double) * 1025, cudaMemcpyHostToDevice));
    }
    CU(dalloc(&c->d_stepped, nch));
    CU(dalloc(&c->d_adr_pending, nch));
    CU(dalloc(&c->d_c_fresh, nch));
    CU(dalloc(&c->d_status, 1));
    CU(dalloc(&c->d_step_ctr, 1));
    CU(cudaMemset(c->d_step_ctr, 0, sizeof(unsigned)));
    CU(cudaMemset(c->d_stepped, 0, sizeof(int) * nch));
    CU(cudaMemset(c->d_adr_pending, 0, sizeof(int) * nch));
    CU(cudaMemset(c->d_c_fresh, 0, sizeof(int) * nch));
    CU(cudaMemset(c->d_status, 0, sizeof(unsigned)));

    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    c->nsm = nsm;
    apply_launch_config(c);
    CU(cudaStreamSynchronize(c->stream));
    if (c->M > 0 && !c->side[0]) {
        for (int i = 0; i < 3; ++i) CU(cudaStreamCreateWithFlags(&c->side[i], cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&c->ev_fork, &c->ev_contact, &c->ev_tiles, &c->ev_mom, &c->ev_lat1, &c->ev_slots,
                           &c->ev_gate, &c->ev_pn, &c->ev_lat, &c->ev_flags})
            CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    c->initialized = true;
    c->steps = 0;
    return SFG_OK;
}

// ------------------------------------------------------------------------
// one step
// ------------------------------------------------------------------------
static void mark(sfg_context* c, int phase) {
    if (!c->profiling) return;
    const size_t i = c->pev_phase.size();
    if (i >= c->pev.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        c->pev.push_back(e);
    }
    cudaEventRecord(c->pev[i], c->stream);
    c->pev_phase.push_back(phase);
}

template <typename S, typename R>
static int enqueue_step_t(sfg_context* c, int p) {
    cudaStream_t st = c->stream;
    const int nch = (int)c->ch.size();
    int launches = 0;
    mark(c, -1);
    LatticeLaunch L{c->d_items, c->n_items, c->d_chans, c->f[p], c->f[1 - p], c->g[p],
                    c->g[1 - p], c->cfield, c->d_stepped, c->d_adr_pending, c->d_c_fresh,
                    c->d_step_ctr, c->any_adr && !c->any_chem, c->d_items4, c->n_items4, c->use_vec4,
                    c->persistent_ctas, c->shared_collision, c->any_bc, c->d_zh_rows,
                    c->n_zh, c->d_ibb, c->ibb_level_start.data(),
                    (int)c->ibb_level_start.size() - 1, c->d_items8, c->n_items8, c->use_vec8,
                    0, nch, c->d_status};
    TileViewArgs tv{c->M > 0 ? c->tb.tile_slot[p] : nullptr,
                    c->M > 0 ? c->tb.tile_slot[1 - p] : nullptr, c->tb.fin[p], c->tb.gsnap,
                    c->tb.fin[1 - p]};
    // Optionally (lattice variant 3) the 8-cell lattice kernel in two passes:
    // cells of force tiles that no marker stencil touches this step take the
    // uniform force and do not depend on the forcing, so that pass runs
    // beside it on a side stream once the step's slot map exists; the
    // touched tiles follow the last spread.  The passes write disjoint cells
    // of the other population buffer.
    const bool split = c->M > 0 && !c->profiling && c->side[0] != nullptr && c->split_lattice &&
                       c->use_vec8 && !L.any_adr && !c->any_bc;
    if (c->M > 0) {
        cudaMemsetAsync(c->tb.capped, 0, sizeof(int) * nch, st);
        cudaMemsetAsync(c->tb.fluid_touched, 0, sizeof(int) * nch, st);
        cudaMemsetAsync(c->tb.resid_gate, 0, sizeof(unsigned) * nch, st);
        cudaMemsetAsync(c->tb.resid_plain, 0, sizeof(unsigned) * nch, st);
        cudaMemsetAsync(c->tb.spread_ctr, 0, sizeof(int) * c->tb.n_spread_ctr, st);
        const S* fp = static_cast<const S*>(c->f[p]);
        // The contact cell list and the force tiles read positions only, the
        // tile moments the populations: with profiling off they run beside
        // the membrane forces on side streams and join before their users.
        const bool par = !c->profiling && c->side[0] != nullptr;
        if (par) {
            CU(cudaEventRecord(c->ev_fork, st));
            CU(cudaStreamWaitEvent(c->side[0], c->ev_fork, 0));
            CU(cudaStreamWaitEvent(c->side[1], c->ev_fork, 0));
            launch_contact_prep(c->d_chans, c->M, c->mb, c->cb, c->ncells, c->side[0]);
            CU(cudaEventRecord(c->ev_contact, c->side[0]));
            launch_tiles(c->d_chans, c->d_caps, c->M, c->mb, c->tb, c->tb.T, p, c->d_phi,
                         c->d_status, c->side[1], c->Kmax > 1 ? c->ev_slots : nullptr);
            CU(cudaEventRecord(c->ev_tiles, c->side[1]));
            // the tile moments need the slot records only: they run beside
            // the work order and the marker lists
            if (c->Kmax > 1) {
                CU(cudaStreamWaitEvent(c->side[2], c->ev_slots, 0));
                launch_tile_moments<S, R>(c->d_chans, fp, c->tb, c->spread_grid, c->side[2]);
                CU(cudaEventRecord(c->ev_mom, c->side[2]));
            }
            if (split) {
                CU(cudaStreamWaitEvent(c->side[2], c->ev_tiles, 0));
                LatticeLaunch L1 = L;
                L1.pass = 1;
                launch_lattice_step<S, R>(L1, tv, c->side[2]);
                CU(cudaEventRecord(c->ev_lat1, c->side[2]));
                launches += 1;
            }
            launch_membrane(c->d_caps, c->NC, c->mb, c->d_has_prev, c->maxn, c->d_status, st);
            CU(cudaStreamWaitEvent(st, c->ev_contact, 0));
            launch_contact_force(c->d_chans, c->M, c->mb, c->cb, st);
            if (c->pillar_repulsion) {
                launch_obstacle_repulsion(c->d_chans, c->M, c->mb, st);
                launches += 1;
            }
            CU(cudaStreamWaitEvent(st, c->ev_tiles, 0));
            launch_spread<R>(c->d_chans, c->mb, c->tb, p, 0, MDF_PLAIN, 0, c->spread_grid,
                             c->d_status, st);
            if (c->Kmax > 1) CU(cudaStreamWaitEvent(st, c->ev_mom, 0));
            launches += 1 + (c->ncells > 0 ? 7 : 1) + 10 + 1 + (c->Kmax > 1 ? 1 : 0);
        } else {
            launch_membrane(c->d_caps, c->NC, c->mb, c->d_has_prev, c->maxn, c->d_status, st);
            mark(c, SFG_PHASE_MEMBRANE);
            launch_contact(c->d_chans, c->M, c->mb, c->cb, c->ncells, st);
            if (c->pillar_repulsion) {
                launch_obstacle_repulsion(c->d_chans, c->M, c->mb, st);
                launches += 1;
            }
            mark(c, SFG_PHASE_CONTACT);
            launch_tiles(c->d_chans, c->d_caps, c->M, c->mb, c->tb, c->tb.T, p, c->d_phi,
                         c->d_status, st);
            mark(c, SFG_PHASE_IBM_TILES);
            launch_spread<R>(c->d_chans, c->mb, c->tb, p, 0, MDF_PLAIN, 0, c->spread_grid,
                             c->d_status, st);
            mark(c, SFG_PHASE_IBM_SPREAD);
            launches += 1 + (c->ncells > 0 ? 7 : 1) + 10 + 1;
            if (c->Kmax > 1) {
                launch_tile_moments<S, R>(c->d_chans, fp, c->tb, c->spread_grid, st);
                mark(c, SFG_PHASE_MDF_INTERP);
                launches += 1;
            }
        }
        if (c->any_learned) {
            // seed, one plain sweep, gate; the plain sweeps below run only for
            // channels above the threshold
            launch_mdf_learned<S, R>(c->d_chans, c->d_caps, c->M, c->mb, fp, c->tb, p,
                                     c->d_model, c->d_feat, c->d_frame, c->learned_grid,
                                     c->d_status, st);
            mark(c, SFG_PHASE_MDF_LEARNED);
            launch_spread<R>(c->d_chans, c->mb, c->tb, p, 1, MDF_SEED, 1, c->spread_grid,
                             c->d_status, st);
            mark(c, SFG_PHASE_IBM_SPREAD);
            launch_mdf_interp<S, R>(c->d_chans, c->M, c->mb, fp, c->tb, p, 2, MDF_LEARNED, st);
            mark(c, SFG_PHASE_MDF_INTERP);
            // whether any channel falls back needs the gate residuals only:
            // it is found beside the last spread, and the plain sweeps wait
            if (par) {
                CU(cudaEventRecord(c->ev_gate, st));
                CU(cudaStreamWaitEvent(c->side[0], c->ev_gate, 0));
                launch_plain_needed(c->d_chans, nch, c->tb, c->side[0]);
                CU(cudaEventRecord(c->ev_pn, c->side[0]));
            } else {
                launch_plain_needed(c->d_chans, nch, c->tb, st);
            }
            launch_spread<R>(c->d_chans, c->mb, c->tb, p, 2, MDF_LEARNED, 2, c->spread_grid,
                             c->d_status, st);
            if (par) CU(cudaStreamWaitEvent(st, c->ev_pn, 0));
            mark(c, SFG_PHASE_IBM_SPREAD);
            launches += 6;
        }
        for (int k = 1; k < c->Kmax; ++k) {
            launch_mdf_interp<S, R>(c->d_chans, c->M, c->mb, fp, c->tb, p, k, MDF_PLAIN, st);
            mark(c, SFG_PHASE_MDF_INTERP);
            launch_spread<R>(c->d_chans, c->mb, c->tb, p, k, MDF_PLAIN, 2 + k, c->spread_grid,
                             c->d_status, st);
            mark(c, SFG_PHASE_IBM_SPREAD);
            launches += 2;
        }
        if (c->harvest) {
            launch_harvest(c->d_chans, c->d_caps, c->M, c->mb, c->d_hfeat, c->d_hlab, c->d_hvalid,
                           st);
            launches += 1;
        }
    }
    if (c->any_bc && c->n_zh > 0) launches += 1;
    if (c->any_bc && c->ibb_level_start.size() > 1) launches += (int)c->ibb_level_start.size() - 1;
    if (split) {
        L.pass = 2;
        launch_lattice_step<S, R>(L, tv, st);
        CU(cudaStreamWaitEvent(st, c->ev_lat1, 0));
    } else {
        launch_lattice_step<S, R>(L, tv, st);
    }
    if (c->any_chem) {
        // this step's scalar step, then the capsule chemistry
        // (simulation.cpp:636-653), before the markers move
        launch_scalar_now<S, R>(L, tv, c->d_cov, st);
        launch_chemistry<R>(c->d_chans, nch, c->d_chem, c->d_caps, c->mb.pos, c->d_phi,
                            c->g[1 - p], c->g[p], c->cfield, c->d_cov, c->d_released,
                            c->d_absorbed, c->d_Mp, c->d_gamma, c->d_waves, c->d_boxes,
                            std::max(c->NC, 1), c->d_status, st);
        launches += 2;
    }
    mark(c, SFG_PHASE_LATTICE);
    // the step's flags and the marker move are independent: the flags run
    // beside the move and join before the step ends
    const bool par_flags = c->M > 0 && !c->profiling && c->side[1] != nullptr;
    cudaStream_t fs = st;
    if (par_flags) {
        CU(cudaEventRecord(c->ev_lat, st));
        CU(cudaStreamWaitEvent(c->side[1], c->ev_lat, 0));
        fs = c->side[1];
    }
    k_step_flags<<<(nch + 127) / 128, 128, 0, fs>>>(c->d_chans, nch, c->d_stepped,
                                                    c->d_adr_pending, c->d_c_fresh,
                                                    c->d_step_ctr, c->tb.resid_gate,
                                                    c->d_learned_steps, c->d_fallbacks);
    if (par_flags) CU(cudaEventRecord(c->ev_flags, c->side[1]));
    mark(c, SFG_PHASE_BOOKKEEPING);
    launches += 2;
    if (c->M > 0) {
        launch_interp_move<S, R>(c->d_chans, c->d_caps, c->NC, c->M, c->mb,
                                 static_cast<const S*>(c->f[1 - p]), c->tb, p, c->d_phi, st);
        mark(c, SFG_PHASE_INTERP_MOVE);
        launches += 1;
    }
    if (par_flags) CU(cudaStreamWaitEvent(st, c->ev_flags, 0));
    c->launches = launches;
    return SFG_OK;
}

static int enqueue_step(sfg_context* c, int p) {
    if (c->precision == SFG_FP64) return enqueue_step_t<double, double>(c, p);
    if (c->precision == SFG_FP32) return enqueue_step_t<float, float>(c, p);
    return enqueue_step_t<__half, float>(c, p);
}

static int build_graphs(sfg_context* c) {
    for (int p = 0; p < 2; ++p) {
        cudaGraph_t g = nullptr;
        CU(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(c, p);
        CU(cudaStreamEndCapture(c->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&c->gexec[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess)
            return fail(SFG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    return SFG_OK;
}

extern "C" int sfg_step(sfg_context* c, int nsteps) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_step: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_step: context not initialized");
    if (nsteps < 0) return fail(SFG_ERR_ARG, "sfg_step: negative step count");
    CU(cudaSetDevice(c->device));
    if (c->use_graphs && !c->gexec[0]) {
        int rc = build_graphs(c);
        if (rc != SFG_OK) return rc;
    }
    CU(cudaEventRecord(c->ev0, c->stream));
    for (int i = 0; i < nsteps; ++i) {
        const int p = (int)(c->steps & 1);
        if (c->profiling) {
            c->pev_phase.clear();
            enqueue_step(c, p);
            CU(cudaStreamSynchronize(c->stream));
            for (size_t k = 1; k < c->pev_phase.size(); ++k) {
                float ms = 0.f;
                CU(cudaEventElapsedTime(&ms, c->pev[k - 1], c->pev[k]));
                const int ph = c->pev_phase[k];
                if (ph >= 0 && ph < SFG_NUM_PHASES) c->phase_ms[ph] += ms;
            }
        } else if (c->use_graphs) {
            CU(cudaGraphLaunch(c->gexec[p], c->stream));
        } else {
            enqueue_step(c, p);
        }
        if (c->any_adr) {
            if (c->any_chem) {
                c->g_cur = 1 - p;    // scalar step done inside the step
            } else {
                if (c->adr_pending_h) c->g_cur = 1 - p;
                c->adr_pending_h = true;
            }
        }
        ++c->steps;
    }
    CU(cudaEventRecord(c->ev1, c->stream));
    CU(cudaGetLastError());
    return SFG_OK;
}

extern "C" int sfg_synchronize(sfg_context* c, unsigned* status_out) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_synchronize: null context");
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    unsigned st = 0;
    if (c->d_status) CU(cudaMemcpy(&st, c->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (status_out) *status_out = st;
    if (st & ST_LATTICE_RUN)
        return fail(SFG_ERR_CUDA, "a lattice run record or cell was out of range (skipped)");
    if (st & (ST_LIST_OVERFLOW | ST_CAPSULE_TOO_BIG))
        return fail(SFG_ERR_CAPACITY,
                    st & ST_LIST_OVERFLOW ? "a force-tile marker list exceeded 4096 entries"
                                          : "a capsule exceeded the per-warp node capacity");
    return SFG_OK;
}

extern "C" int sfg_last_step_ms(sfg_context* c, float* ms) {
    if (!c || !ms) return fail(SFG_ERR_ARG, "sfg_last_step_ms: null argument");
    CU(cudaEventElapsedTime(ms, c->ev0, c->ev1));
    return SFG_OK;
}

// ------------------------------------------------------------------------
// learned multi-direct forcing
// ------------------------------------------------------------------------
int sfg_mlp_model_device(sfg_mlp* m, const void** model, cudaStream_t st);

static void drop_graphs(sfg_context* c) {
    for (int i = 0; i < 2; ++i) {
        if (c->gexec[i]) cudaGraphExecDestroy(c->gexec[i]);
        c->gexec[i] = nullptr;
    }
}

// ------------------------------------------------------------------------
// launch-shape autotuner
// ------------------------------------------------------------------------
static int time_steps(sfg_context* c, int n, float* ms_per_step) {
    drop_graphs(c);
    int rc = sfg_step(c, 2);
    if (rc) return rc;
    CU(cudaStreamSynchronize(c->stream));
    if ((rc = sfg_step(c, n))) return rc;
    CU(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    *ms_per_step = ms / (float)n;
    return SFG_OK;
}

extern "C" int sfg_autotune(sfg_context* c, int steps_per_trial, int* steps_run) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_autotune: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_autotune: context not initialized");
    if (steps_per_trial < 1) return fail(SFG_ERR_ARG, "sfg_autotune: steps_per_trial < 1");
    CU(cudaSetDevice(c->device));
    const bool prof = c->profiling;
    c->profiling = false;
    int run = 0;
    // coordinate descent over the tunables, each trial timed on real steps
    struct Knob {
        int* v;
        std::vector<int> cand;
    };
    std::vector<Knob> knobs;
    const int lat_max = lattice_ctas_per_sm(c->precision, c->any_adr && !c->any_chem, c->use_vec8);
    const int spr_max = spread_blocks_per_sm(c->precision == SFG_FP64);
    std::vector<int> lat, spr;
    for (int k = 1; k <= lat_max; ++k) lat.push_back(k);
    for (int k = 1; k <= spr_max; ++k) spr.push_back(k);
    knobs.push_back({&c->lattice_cps, lat});
    if (c->M > 0) {
        knobs.push_back({&c->spread_cps, spr});
        knobs.push_back({&c->tb.marker_block, {64, 128, 256}});
        if (c->any_learned) knobs.push_back({&c->learned_cps, {1, 2, 4, 6}});
    }
    if (c->lattice_cps == 0) c->lattice_cps = lat_max;
    if (c->spread_cps == 0) c->spread_cps = spr_max;
    for (auto& k : knobs) {
        int best = *k.v;
        float best_ms = 1e30f;
        for (int v : k.cand) {
            *k.v = v;
            apply_launch_config(c);
            float ms = 0.f;
            int rc = time_steps(c, steps_per_trial, &ms);
            run += 2 + steps_per_trial;
            if (rc) {
                c->profiling = prof;
                return rc;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = v;
            }
        }
        *k.v = best;
        apply_launch_config(c);
    }
    drop_graphs(c);
    c->profiling = prof;
    if (steps_run) *steps_run = run;
    return SFG_OK;
}

extern "C" int sfg_get_launch_config(sfg_context* c, int* lattice_cps, int* spread_cps,
                                     int* marker_block, int* learned_cps) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_get_launch_config: null context");
    // the chosen counts (the spread grid is further capped by the slot count)
    const int lat_max = lattice_ctas_per_sm(c->precision, c->any_adr && !c->any_chem, c->use_vec8);
    const int spr_max = spread_blocks_per_sm(c->precision == SFG_FP64);
    if (lattice_cps) *lattice_cps = c->lattice_cps > 0 ? std::min(c->lattice_cps, lat_max) : lat_max;
    if (spread_cps) *spread_cps = c->spread_cps > 0 ? std::min(c->spread_cps, spr_max) : spr_max;
    if (marker_block) *marker_block = c->tb.marker_block;
    if (learned_cps) *learned_cps = std::max(1, std::min(c->learned_cps, 6));
    return SFG_OK;
}

extern "C" int sfg_set_mdf_model(sfg_context* c, sfg_mlp* net, double residual_threshold) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_mdf_model: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_set_mdf_model: context not initialized");
    if (net && !(residual_threshold >= 0.0))
        return fail(SFG_ERR_ARG, "sfg_set_mdf_model: the threshold must be >= 0");
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    bool any = false;
    if (net) {
        static bool prepared[64] = {false};
        if (c->device >= 0 && c->device < 64 && !prepared[c->device]) {
            CU(prepare_mdf_learned());
            prepared[c->device] = true;
        }
        const void* md = nullptr;
        int rc = sfg_mlp_model_device(net, &md, c->stream);
        if (rc) return rc;
        if (!c->d_model) CU(cudaMalloc(&c->d_model, sizeof(sfg::mlp::ModelDev)));
        CU(cudaMemcpyAsync(c->d_model, md, sizeof(sfg::mlp::ModelDev), cudaMemcpyDeviceToDevice,
                           c->stream));
        if (!c->tb.acc0 && c->M > 0)
            CU(dalloc(&c->tb.acc0, (size_t)c->tb.max_slots * 2 * TILE_CELLS));
        if (!c->d_plain_needed) CU(dalloc(&c->d_plain_needed, 1));
        if (!c->d_feat && c->M > 0) {
            CU(dalloc(&c->d_feat, 8LL * c->M));
            CU(dalloc(&c->d_frame, c->M));
        }
    }
    for (auto& h : c->ch) {
        const bool on = net && h.d.ibm_iterations >= 3 && h.d.cap_end > h.d.cap_begin;
        h.d.learned = on ? 1 : 0;
        h.d.mdf_threshold = (float)residual_threshold;
        any = any || on;
    }
    std::vector<ChannelDev> dv;
    for (auto& h : c->ch) dv.push_back(h.d);
    CU(cudaMemcpyAsync(c->d_chans, dv.data(), sizeof(ChannelDev) * dv.size(),
                       cudaMemcpyHostToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->any_learned = any;
    c->tb.plain_needed = any ? c->d_plain_needed : nullptr;
    drop_graphs(c);
    return SFG_OK;
}

extern "C" int sfg_get_mdf_stats(sfg_context* c, int channel, float* resid_learned,
                                 float* resid_plain, long long* learned_steps,
                                 long long* fallbacks) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_get_mdf_stats: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_get_mdf_stats: context not initialized");
    if (channel < 0 || channel >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_get_mdf_stats: bad channel");
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    unsigned rg = 0, rp = 0;
    long long ls = 0, fb = 0;
    CU(cudaMemcpy(&rg, c->tb.resid_gate + channel, sizeof(unsigned), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&rp, c->tb.resid_plain + channel, sizeof(unsigned), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&ls, c->d_learned_steps + channel, sizeof(long long), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&fb, c->d_fallbacks + channel, sizeof(long long), cudaMemcpyDeviceToHost));
    float a, b;
    std::memcpy(&a, &rg, sizeof(float));
    std::memcpy(&b, &rp, sizeof(float));
    if (resid_learned) *resid_learned = a;
    if (resid_plain) *resid_plain = b;
    if (learned_steps) *learned_steps = ls;
    if (fallbacks) *fallbacks = fb;
    return SFG_OK;
}

extern "C" int sfg_set_harvest(sfg_context* c, int enabled) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_harvest: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_set_harvest: context not initialized");
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    if (enabled && c->M > 0 && !c->d_hfeat) {
        CU(dalloc(&c->d_hfeat, 8LL * c->M));
        CU(dalloc(&c->d_hlab, 2LL * c->M));
        CU(dalloc(&c->d_hvalid, c->M));
        CU(cudaMemset(c->d_hvalid, 0, sizeof(int) * c->M));
    }
    c->harvest = enabled != 0 && c->M > 0;
    drop_graphs(c);
    return SFG_OK;
}

extern "C" int sfg_get_harvest(sfg_context* c, float* features, float* labels, int* valid) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_get_harvest: null context");
    if (!c->harvest || !c->d_hfeat)
        return fail(SFG_ERR_STATE, "sfg_get_harvest: harvesting is not enabled");
    CU(cudaSetDevice(c->device));
    CU(cudaStreamSynchronize(c->stream));
    if (features)
        CU(cudaMemcpy(features, c->d_hfeat, sizeof(float) * 8 * c->M, cudaMemcpyDeviceToHost));
    if (labels)
        CU(cudaMemcpy(labels, c->d_hlab, sizeof(float) * 2 * c->M, cudaMemcpyDeviceToHost));
    if (valid) CU(cudaMemcpy(valid, c->d_hvalid, sizeof(int) * c->M, cudaMemcpyDeviceToHost));
    return SFG_OK;
}

// ------------------------------------------------------------------------
// state transfer
// ------------------------------------------------------------------------
static int check_chan(sfg_context* c, int ch, const char* who) {
    if (!c) return fail(SFG_ERR_ARG, std::string(who) + ": null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, std::string(who) + ": context not initialized");
    if (ch < 0 || ch >= (int)c->ch.size()) return fail(SFG_ERR_ARG, std::string(who) + ": bad channel");
    return SFG_OK;
}

static int ensure_io(sfg_context* c, size_t ndoubles) {
    if (c->io_doubles >= ndoubles) return SFG_OK;
    if (c->d_io) cudaFree(c->d_io);
    c->d_io = nullptr;
    c->io_doubles = 0;
    CU(cudaMalloc(&c->d_io, ndoubles * sizeof(double)));
    c->io_doubles = ndoubles;
    return SFG_OK;
}

static TileViewArgs last_view(sfg_context* c) {
    // the tile set of the last completed step (parity (steps - 1) & 1)
    const int lp = (int)((c->steps + 1) & 1);
    TileViewArgs tv{c->M > 0 ? c->tb.tile_slot[lp] : nullptr, c->M > 0 ? c->tb.tile_slot[1 - lp] : nullptr,
                    c->tb.fin[lp], c->tb.gsnap, c->tb.fin[1 - lp]};
    return tv;
}

extern "C" int sfg_get_populations(sfg_context* c, int chi, double* f) {
    int rc = check_chan(c, chi, "sfg_get_populations");
    if (rc) return rc;
    if (!f) return fail(SFG_ERR_ARG, "sfg_get_populations: null output");
    const ChannelDev& d = c->ch[chi].d;
    const size_t n = 9ULL * d.nx * d.ny;
    if ((rc = ensure_io(c, n))) return rc;
    const int p = (int)(c->steps & 1);
    if (c->precision == SFG_FP64) launch_pop_export<double, double>(c->f[p], c->d_io, d, c->stream);
    else if (c->precision == SFG_FP32) launch_pop_export<float, float>(c->f[p], c->d_io, d, c->stream);
    else launch_pop_export<__half, float>(c->f[p], c->d_io, d, c->stream);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(f, c->d_io, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_set_populations(sfg_context* c, int chi, const double* f) {
    int rc = check_chan(c, chi, "sfg_set_populations");
    if (rc) return rc;
    if (!f) return fail(SFG_ERR_ARG, "sfg_set_populations: null input");
    const ChannelDev& d = c->ch[chi].d;
    const size_t n = 9ULL * d.nx * d.ny;
    if ((rc = ensure_io(c, n))) return rc;
    CU(cudaMemcpyAsync(c->d_io, f, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    for (int i = 0; i < 2; ++i) {
        if (c->precision == SFG_FP64) launch_pop_import<double, double>(c->d_io, c->f[i], d, c->stream);
        else if (c->precision == SFG_FP32) launch_pop_import<float, float>(c->d_io, c->f[i], d, c->stream);
        else launch_pop_import<__half, float>(c->d_io, c->f[i], d, c->stream);
    }
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_set_all_populations(sfg_context* c, const double* f) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_all_populations: null context");
    if (!c->initialized)
        return fail(SFG_ERR_STATE, "sfg_set_all_populations: context not initialized");
    if (!f) return fail(SFG_ERR_ARG, "sfg_set_all_populations: null input");
    CU(cudaSetDevice(c->device));
    const int nch = (int)c->ch.size();
    size_t maxn = 0;
    for (int i = 0; i < nch; ++i)
        maxn = std::max(maxn, (size_t)9 * c->ch[i].d.nx * c->ch[i].d.ny);
    if (!c->up_stream) {
        CU(cudaStreamCreateWithFlags(&c->up_stream, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            CU(cudaEventCreateWithFlags(&c->up_copied[b], cudaEventDisableTiming));
            CU(cudaEventCreateWithFlags(&c->up_free[b], cudaEventDisableTiming));
        }
    }
    if (c->up_doubles < maxn) {
        for (int b = 0; b < 2; ++b) {
            if (c->d_up[b]) cudaFree(c->d_up[b]);
            c->d_up[b] = nullptr;
        }
        c->up_doubles = 0;
        for (int b = 0; b < 2; ++b) CU(cudaMalloc(&c->d_up[b], maxn * sizeof(double)));
        c->up_doubles = maxn;
    }
    size_t off = 0;
    for (int i = 0; i < nch; ++i) {
        const ChannelDev& d = c->ch[i].d;
        const size_t n = 9ULL * d.nx * d.ny;
        const int b = i & 1;
        // the buffer's previous import (channel i - 2) must have read it
        if (i >= 2) CU(cudaStreamWaitEvent(c->up_stream, c->up_free[b], 0));
        CU(cudaMemcpyAsync(c->d_up[b], f + off, n * sizeof(double), cudaMemcpyHostToDevice,
                           c->up_stream));
        CU(cudaEventRecord(c->up_copied[b], c->up_stream));
        CU(cudaStreamWaitEvent(c->stream, c->up_copied[b], 0));
        for (int k = 0; k < 2; ++k) {
            if (c->precision == SFG_FP64) launch_pop_import<double, double>(c->d_up[b], c->f[k], d, c->stream);
            else if (c->precision == SFG_FP32) launch_pop_import<float, float>(c->d_up[b], c->f[k], d, c->stream);
            else launch_pop_import<__half, float>(c->d_up[b], c->f[k], d, c->stream);
        }
        CU(cudaGetLastError());
        CU(cudaEventRecord(c->up_free[b], c->stream));
        off += n;
    }
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_get_macroscopic(sfg_context* c, int chi, double* rho, double* ux, double* uy,
                                   double* Fx, double* Fy) {
    int rc = check_chan(c, chi, "sfg_get_macroscopic");
    if (rc) return rc;
    const ChannelDev& d = c->ch[chi].d;
    const size_t N = (size_t)d.nx * d.ny;
    if ((rc = ensure_io(c, 5 * N))) return rc;
    const int p = (int)(c->steps & 1);
    const TileViewArgs tv = last_view(c);
    const int stepped = c->steps > 0 || c->restored;
    double* o = c->d_io;
    if (c->precision == SFG_FP64)
        launch_macro_export<double, double>(c->f[p], d, tv, stepped, o, o + N, o + 2 * N, o + 3 * N, o + 4 * N, c->stream);
    else if (c->precision == SFG_FP32)
        launch_macro_export<float, float>(c->f[p], d, tv, stepped, o, o + N, o + 2 * N, o + 3 * N, o + 4 * N, c->stream);
    else
        launch_macro_export<__half, float>(c->f[p], d, tv, stepped, o, o + N, o + 2 * N, o + 3 * N, o + 4 * N, c->stream);
    CU(cudaGetLastError());
    double* outs[5] = {rho, ux, uy, Fx, Fy};
    for (int k = 0; k < 5; ++k)
        if (outs[k])
            CU(cudaMemcpyAsync(outs[k], o + k * N, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_get_markers(sfg_context* c, int chi, double* pos, double* vel, double* force) {
    int rc = check_chan(c, chi, "sfg_get_markers");
    if (rc) return rc;
    const ChannelDev& d = c->ch[chi].d;
    const int n = d.mk_end - d.mk_begin;
    if (n > 0) {
        if (pos) CU(cudaMemcpyAsync(pos, c->mb.pos + d.mk_begin, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream));
        if (vel) CU(cudaMemcpyAsync(vel, c->mb.vel + d.mk_begin, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream));
        if (force) CU(cudaMemcpyAsync(force, c->mb.frc + d.mk_begin, sizeof(double2) * n, cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_wait_markers(sfg_context* c, int slot) {
    if (!c || slot < 0 || slot > 1) return fail(SFG_ERR_ARG, "sfg_wait_markers: bad argument");
    if (!c->copy_pending[slot]) return SFG_OK;
    CU(cudaSetDevice(c->device));
    CU(cudaEventSynchronize(c->ev_copy[slot]));
    c->copy_pending[slot] = false;
    return SFG_OK;
}

extern "C" int sfg_get_all_markers_async(sfg_context* c, int slot, double* pos, double* vel) {
    if (!c || slot < 0 || slot > 1)
        return fail(SFG_ERR_ARG, "sfg_get_all_markers_async: bad argument");
    if (!c->initialized)
        return fail(SFG_ERR_STATE, "sfg_get_all_markers_async: context not initialized");
    if (c->M == 0) return SFG_OK;
    CU(cudaSetDevice(c->device));
    if (!c->copy_stream) {
        CU(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2; ++i) {
            CU(cudaMalloc(&c->d_snap[i], sizeof(double) * 4 * (size_t)c->M));
            CU(cudaEventCreateWithFlags(&c->ev_snap[i], cudaEventDisableTiming));
            CU(cudaEventCreateWithFlags(&c->ev_copy[i], cudaEventDisableTiming));
        }
    }
    // the slot's previous copy must have left its snapshot buffer
    int rc = sfg_wait_markers(c, slot);
    if (rc) return rc;
    double* snap = c->d_snap[slot];
    const size_t bytes = sizeof(double2) * (size_t)c->M;
    CU(cudaMemcpyAsync(snap, c->mb.pos, bytes, cudaMemcpyDeviceToDevice, c->stream));
    CU(cudaMemcpyAsync(snap + 2 * (size_t)c->M, c->mb.vel, bytes, cudaMemcpyDeviceToDevice,
                       c->stream));
    CU(cudaEventRecord(c->ev_snap[slot], c->stream));
    CU(cudaStreamWaitEvent(c->copy_stream, c->ev_snap[slot], 0));
    if (pos) CU(cudaMemcpyAsync(pos, snap, bytes, cudaMemcpyDeviceToHost, c->copy_stream));
    if (vel)
        CU(cudaMemcpyAsync(vel, snap + 2 * (size_t)c->M, bytes, cudaMemcpyDeviceToHost,
                           c->copy_stream));
    CU(cudaEventRecord(c->ev_copy[slot], c->copy_stream));
    c->copy_pending[slot] = true;
    return SFG_OK;
}

extern "C" int sfg_get_all_markers(sfg_context* c, double* pos, double* vel) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_get_all_markers: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_get_all_markers: context not initialized");
    if (c->M > 0) {
        if (pos) CU(cudaMemcpyAsync(pos, c->mb.pos, sizeof(double2) * c->M, cudaMemcpyDeviceToHost, c->stream));
        if (vel) CU(cudaMemcpyAsync(vel, c->mb.vel, sizeof(double2) * c->M, cudaMemcpyDeviceToHost, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_set_markers(sfg_context* c, int chi, const double* pos, const double* vel) {
    int rc = check_chan(c, chi, "sfg_set_markers");
    if (rc) return rc;
    const ChannelDev& d = c->ch[chi].d;
    const int n = d.mk_end - d.mk_begin;
    if (n > 0) {
        if (pos) CU(cudaMemcpyAsync(c->mb.pos + d.mk_begin, pos, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream));
        if (vel) CU(cudaMemcpyAsync(c->mb.vel + d.mk_begin, vel, sizeof(double2) * n, cudaMemcpyHostToDevice, c->stream));
    }
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

// Runs the pending scalar step of the last lattice step, if any.
template <typename S, typename R>
static int flush_scalar_t(sfg_context* c) {
    const int P = (int)(c->steps & 1);
    LatticeLaunch L{c->d_items, c->n_items, c->d_chans, c->f[P], nullptr, c->g[P], c->g[1 - P],
                    c->cfield, c->d_stepped, c->d_adr_pending, c->d_c_fresh, c->d_step_ctr,
                    c->any_adr, c->d_items4, c->n_items4, false, 0, -1};
    launch_scalar_flush<S, R>(L, last_view(c), c->stream);
    const int nch = (int)c->ch.size();
    k_flush_flags<<<(nch + 127) / 128, 128, 0, c->stream>>>(nch, c->d_adr_pending, c->d_c_fresh);
    CU(cudaGetLastError());
    c->g_cur = 1 - P;
    c->adr_pending_h = false;
    return SFG_OK;
}

static int flush_scalar(sfg_context* c) {
    if (!c->any_adr || !c->adr_pending_h) return SFG_OK;
    if (c->precision == SFG_FP64) return flush_scalar_t<double, double>(c);
    if (c->precision == SFG_FP32) return flush_scalar_t<float, float>(c);
    return flush_scalar_t<__half, float>(c);
}

extern "C" int sfg_set_concentration(sfg_context* c, int chi, const double* C) {
    int rc = check_chan(c, chi, "sfg_set_concentration");
    if (rc) return rc;
    if (!C) return fail(SFG_ERR_ARG, "sfg_set_concentration: null input");
    const ChannelDev& d = c->ch[chi].d;
    if (!d.adr) return fail(SFG_ERR_STATE, "sfg_set_concentration: scalar transport is off");
    if ((rc = flush_scalar(c))) return rc;
    const size_t N = (size_t)d.nx * d.ny;
    if ((rc = ensure_io(c, N))) return rc;
    CU(cudaMemcpyAsync(c->d_io, C, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (c->precision == SFG_FP64)
        k_scalar_set<double><<<io_blocks(N), 256, 0, c->stream>>>(c->d_io, (double*)c->g[0], (double*)c->g[1], (double*)c->cfield, d);
    else
        k_scalar_set<float><<<io_blocks(N), 256, 0, c->stream>>>(c->d_io, (float*)c->g[0], (float*)c->g[1], (float*)c->cfield, d);
    const int one = 1;
    CU(cudaMemcpyAsync(c->d_c_fresh + chi, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (c->d_cov) CU(cudaMemsetAsync(c->d_cov + d.cell_off, 0, (size_t)d.plane, c->stream));
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_set_scalar_state(sfg_context* c, int chi, const double* C, const double* g) {
    int rc = check_chan(c, chi, "sfg_set_scalar_state");
    if (rc) return rc;
    if (!C || !g) return fail(SFG_ERR_ARG, "sfg_set_scalar_state: null input");
    const ChannelDev& d = c->ch[chi].d;
    if (!d.adr) return fail(SFG_ERR_STATE, "sfg_set_scalar_state: scalar transport is off");
    if ((rc = flush_scalar(c))) return rc;
    const size_t N = (size_t)d.nx * d.ny;
    if ((rc = ensure_io(c, 10 * N))) return rc;
    CU(cudaMemcpyAsync(c->d_io, C, N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CU(cudaMemcpyAsync(c->d_io + N, g, 9 * N * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    if (c->precision == SFG_FP64)
        k_scalar_import<double><<<io_blocks(N), 256, 0, c->stream>>>(c->d_io, c->d_io + N, (double*)c->g[0], (double*)c->g[1], (double*)c->cfield, d);
    else
        k_scalar_import<float><<<io_blocks(N), 256, 0, c->stream>>>(c->d_io, c->d_io + N, (float*)c->g[0], (float*)c->g[1], (float*)c->cfield, d);
    const int one = 1;
    CU(cudaMemcpyAsync(c->d_c_fresh + chi, &one, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    if (c->d_cov) CU(cudaMemsetAsync(c->d_cov + d.cell_off, 0, (size_t)d.plane, c->stream));
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_mark_restored(sfg_context* c) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_mark_restored: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_mark_restored: context not initialized");
    if (c->steps != 0)
        return fail(SFG_ERR_STATE, "sfg_mark_restored: only before the first step");
    CU(cudaSetDevice(c->device));
    const int nch = (int)c->ch.size();
    std::vector<int> ones(nch, 1);
    CU(cudaMemcpyAsync(c->d_stepped, ones.data(), sizeof(int) * nch, cudaMemcpyHostToDevice, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    c->restored = true;
    return SFG_OK;
}

extern "C" int sfg_get_concentration(sfg_context* c, int chi, double* C, double* g) {
    int rc = check_chan(c, chi, "sfg_get_concentration");
    if (rc) return rc;
    const ChannelDev& d = c->ch[chi].d;
    if (!d.adr) return fail(SFG_ERR_STATE, "sfg_get_concentration: scalar transport is off");
    if ((rc = flush_scalar(c))) return rc;
    const size_t N = (size_t)d.nx * d.ny;
    if ((rc = ensure_io(c, 10 * N))) return rc;
    double* o = c->d_io;
    if (c->precision == SFG_FP64)
        k_scalar_export<double><<<io_blocks(N), 256, 0, c->stream>>>((const double*)c->g[c->g_cur], d, o, g ? o + N : nullptr, (const double*)c->cfield, c->d_cov);
    else
        k_scalar_export<float><<<io_blocks(N), 256, 0, c->stream>>>((const float*)c->g[c->g_cur], d, o, g ? o + N : nullptr, (const float*)c->cfield, c->d_cov);
    CU(cudaGetLastError());
    if (C) CU(cudaMemcpyAsync(C, o, N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (g) CU(cudaMemcpyAsync(g, o + N, 9 * N * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

// ------------------------------------------------------------------------
// thermo: device-side reductions and the multi-step run
// ------------------------------------------------------------------------
// One thread per channel: combines the channel's block partials in block
// order, sums the capsule deformations in capsule order
// (global_stats_writer.cpp:84-90) and counts the capped cells as
// sfg_get_capped_count does.
__global__ void k_thermo_final(const ChannelDev* __restrict__ chans, int nch, int bpc,
                               const ThermoPart* __restrict__ parts,
                               const double* __restrict__ cap_stats, const int* __restrict__ capped,
                               const int* __restrict__ fluid_touched, int stepped,
                               sfg_thermo_record* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nch) return;
    const ChannelDev& ch = chans[c];
    ThermoPart p;
    thermo_init(p);
    for (int b = 0; b < bpc; ++b) thermo_merge(p, parts[(long long)c * bpc + b]);
    sfg_thermo_record t;
    const double n = (double)p.count;
    t.max_speed = __dsqrt_rn(p.max_v2);
    t.mean_rho = p.count > 0 ? __ddiv_rn(p.sum_rho, n) : 0.0;
    t.mean_velocity = p.count > 0 ? __ddiv_rn(p.sum_vel, n) : 0.0;
    t.kinetic_energy = p.ke;
    t.min_rho = p.min_rho;
    t.max_rho = p.max_rho;
    t.total_scalar = p.sum_c;
    t.fluid_cells = p.count;
    t.first_nonfinite = p.first_bad == THERMO_NONE ? -1 : p.first_bad;
    const int nc = ch.cap_end - ch.cap_begin;
    double mean_def = 0.0, max_def = 0.0;
    for (int k = ch.cap_begin; k < ch.cap_end; ++k) {
        const double D = cap_stats[6LL * k + 4];
        mean_def = __dadd_rn(mean_def, D);
        if (D > max_def) max_def = D;
    }
    if (nc > 0) mean_def = __ddiv_rn(mean_def, (double)nc);
    t.mean_deformation = mean_def;
    t.max_deformation = max_def;
    t.num_capsules = nc;
    t.reserved = 0;
    long long cap_n = 0;
    if (stepped && capped != nullptr) {
        cap_n = capped[c];
        const double bx = 0.0 + ch.body_fx, by = 0.0 + ch.body_fy, Fm = ch.max_force;
        if (__dadd_rn(__dmul_rn(bx, bx), __dmul_rn(by, by)) > __dmul_rn(Fm, Fm))
            cap_n += p.fluid - fluid_touched[c];
    }
    t.capped_nodes = cap_n;
    out[c] = t;
}

// Enqueues the thermo reductions of the current state on the context stream
// and the copies of their results into the pinned host records.
static int enqueue_thermo(sfg_context* c) {
    const int nch = (int)c->ch.size();
    if (!c->d_thermo) {
        long long maxN = 1;
        for (const ChanHost& h : c->ch) maxN = std::max(maxN, (long long)h.d.nx * h.d.ny);
        // about 16 cells per thread on the largest channel, at most 512 blocks
        c->thermo_bpc = (int)std::min<long long>(512, std::max<long long>(1, (maxN + 4095) / 4096));
        CU(cudaMalloc(&c->d_thermo_parts, sizeof(ThermoPart) * (size_t)nch * c->thermo_bpc));
        CU(cudaMalloc(&c->d_thermo, sizeof(sfg_thermo_record) * nch));
        CU(cudaMallocHost(&c->h_thermo, sizeof(sfg_thermo_record) * nch));
        if (c->NC > 0) {
            CU(cudaMalloc(&c->d_cap_stats, sizeof(double) * 6 * c->NC));
            CU(cudaMallocHost(&c->h_cap_stats, sizeof(double) * 6 * c->NC));
        }
    }
    int rc = flush_scalar(c);
    if (rc) return rc;
    const int p = (int)(c->steps & 1);
    const TileViewArgs tv = last_view(c);
    const int stepped = c->steps > 0 || c->restored;
    const void* g = c->any_adr ? c->g[c->g_cur] : nullptr;
    if (c->precision == SFG_FP64)
        launch_thermo_cells<double, double>(c->f[p], g, c->d_chans, nch, c->thermo_bpc, tv, stepped, c->d_thermo_parts, c->cfield, c->d_cov, c->stream);
    else if (c->precision == SFG_FP32)
        launch_thermo_cells<float, float>(c->f[p], g, c->d_chans, nch, c->thermo_bpc, tv, stepped, c->d_thermo_parts, c->cfield, c->d_cov, c->stream);
    else
        launch_thermo_cells<__half, float>(c->f[p], g, c->d_chans, nch, c->thermo_bpc, tv, stepped, c->d_thermo_parts, c->cfield, c->d_cov, c->stream);
    if (c->NC > 0) launch_capsule_stats(c->d_caps, c->NC, c->mb.pos, c->d_cap_stats, c->stream);
    k_thermo_final<<<(nch + 127) / 128, 128, 0, c->stream>>>(
        c->d_chans, nch, c->thermo_bpc, c->d_thermo_parts, c->d_cap_stats, c->tb.capped,
        c->tb.fluid_touched, stepped, c->d_thermo);
    CU(cudaGetLastError());
    CU(cudaMemcpyAsync(c->h_thermo, c->d_thermo, sizeof(sfg_thermo_record) * nch, cudaMemcpyDeviceToHost,
                       c->stream));
    if (c->NC > 0)
        CU(cudaMemcpyAsync(c->h_cap_stats, c->d_cap_stats, sizeof(double) * 6 * c->NC,
                           cudaMemcpyDeviceToHost, c->stream));
    return SFG_OK;
}

extern "C" int sfg_thermo(sfg_context* c, sfg_thermo_record* chans, sfg_capsule_stats* caps) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_thermo: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_thermo: context not initialized");
    CU(cudaSetDevice(c->device));
    int rc = enqueue_thermo(c);
    if (rc) return rc;
    if ((rc = sfg_synchronize(c, nullptr))) return rc;
    const int nch = (int)c->ch.size();
    if (chans) std::memcpy(chans, c->h_thermo, sizeof(sfg_thermo_record) * nch);
    if (caps && c->NC > 0) std::memcpy(caps, c->h_cap_stats, sizeof(double) * 6 * c->NC);
    return SFG_OK;
}

extern "C" int sfg_run(sfg_context* c, int nsteps, int thermo_every, sfg_thermo_fn cb, void* user,
                       int* steps_done) {
    if (steps_done) *steps_done = 0;
    if (!c) return fail(SFG_ERR_ARG, "sfg_run: null context");
    if (!c->initialized) return fail(SFG_ERR_STATE, "sfg_run: context not initialized");
    if (nsteps < 0) return fail(SFG_ERR_ARG, "sfg_run: negative step count");
    CU(cudaSetDevice(c->device));
    int rc;
    if (cb == nullptr) {
        if ((rc = sfg_step(c, nsteps))) return rc;
        if ((rc = sfg_synchronize(c, nullptr))) return rc;
        if (steps_done) *steps_done = nsteps;
        return SFG_OK;
    }
    const int every = thermo_every > 0 ? thermo_every : std::max(nsteps, 1);
    const int nch = (int)c->ch.size();
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(every, nsteps - done);
        if ((rc = sfg_step(c, n))) return rc;
        done += n;
        if (steps_done) *steps_done = done;
        if ((rc = enqueue_thermo(c))) return rc;
        if ((rc = sfg_synchronize(c, nullptr))) return rc;
        if (cb(c->steps, c->h_thermo, nch, reinterpret_cast<const sfg_capsule_stats*>(c->h_cap_stats),
               c->NC, user) != 0)
            break;
    }
    return SFG_OK;
}

extern "C" int sfg_get_capped_count(sfg_context* c, int chi, int* count) {
    int rc = check_chan(c, chi, "sfg_get_capped_count");
    if (rc) return rc;
    if (!count) return fail(SFG_ERR_ARG, "sfg_get_capped_count: null output");
    CU(cudaStreamSynchronize(c->stream));
    if (c->steps == 0) { *count = 0; return SFG_OK; }
    const ChanHost& h = c->ch[chi];
    int capped = 0, touched = 0;
    CU(cudaMemcpy(&capped, c->tb.capped + chi, sizeof(int), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&touched, c->tb.fluid_touched + chi, sizeof(int), cudaMemcpyDeviceToHost));
    const double bx = 0.0 + h.p.body_fx, by = 0.0 + h.p.body_fy;
    const double Fm = h.p.max_lattice_force;
    const bool body_capped = bx * bx + by * by > Fm * Fm;
    long long total = capped;
    if (body_capped) total += h.fluid_cells - touched;
    *count = (int)total;
    return SFG_OK;
}

extern "C" int sfg_get_contact_counts(sfg_context* c, int chi, int* counts) {
    int rc = check_chan(c, chi, "sfg_get_contact_counts");
    if (rc) return rc;
    const ChannelDev& d = c->ch[chi].d;
    const int n = d.mk_end - d.mk_begin;
    if (n > 0 && counts)
        CU(cudaMemcpyAsync(counts, c->mb.pair_count + d.mk_begin, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream));
    CU(cudaStreamSynchronize(c->stream));
    return SFG_OK;
}

extern "C" int sfg_num_channels(const sfg_context* c, int* n) {
    if (!c || !n) return fail(SFG_ERR_ARG, "sfg_num_channels: null argument");
    *n = (int)c->ch.size();
    return SFG_OK;
}

extern "C" int sfg_channel_counts(const sfg_context* c, int chi, int* ncaps, int* nmk) {
    if (!c || chi < 0 || chi >= (int)c->ch.size()) return fail(SFG_ERR_ARG, "sfg_channel_counts: bad argument");
    int m = 0;
    for (const auto& cp : c->ch[chi].caps) m += cp.rest.num_nodes;
    if (ncaps) *ncaps = (int)c->ch[chi].caps.size();
    if (nmk) *nmk = m;
    return SFG_OK;
}

extern "C" int sfg_get_channel_params(const sfg_context* c, int chi, sfg_channel_params* out) {
    if (!c || !out || chi < 0 || chi >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_get_channel_params: bad argument");
    *out = c->ch[chi].p;
    return SFG_OK;
}

extern "C" int sfg_get_capsule_nodes(const sfg_context* c, int chi, int* nodes) {
    if (!c || !nodes || chi < 0 || chi >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_get_capsule_nodes: bad argument");
    int k = 0;
    for (const auto& cp : c->ch[chi].caps) nodes[k++] = cp.rest.num_nodes;
    return SFG_OK;
}

extern "C" int sfg_get_capsule_base(const sfg_context* c, int chi, int* first_capsule) {
    if (!c || !first_capsule || chi < 0 || chi >= (int)c->ch.size())
        return fail(SFG_ERR_ARG, "sfg_get_capsule_base: bad argument");
    int k = 0;
    for (int i = 0; i < chi; ++i) k += (int)c->ch[i].caps.size();
    *first_capsule = k;
    return SFG_OK;
}

extern "C" int sfg_step_count(const sfg_context* c, long long* s) {
    if (!c || !s) return fail(SFG_ERR_ARG, "sfg_step_count: null argument");
    *s = c->steps;
    return SFG_OK;
}

extern "C" int sfg_launches_per_step(const sfg_context* c, int* l) {
    if (!c || !l) return fail(SFG_ERR_ARG, "sfg_launches_per_step: null argument");
    *l = c->launches;
    return SFG_OK;
}

extern "C" int sfg_set_profiling(sfg_context* c, int on) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_profiling: null context");
    c->profiling = on != 0;
    return SFG_OK;
}

extern "C" int sfg_get_phase_times(sfg_context* c, float* ms, int n) {
    if (!c || !ms) return fail(SFG_ERR_ARG, "sfg_get_phase_times: null argument");
    for (int i = 0; i < n && i < SFG_NUM_PHASES; ++i) ms[i] = c->phase_ms[i];
    return SFG_OK;
}

extern "C" int sfg_reset_phase_times(sfg_context* c) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_reset_phase_times: null context");
    for (int i = 0; i < SFG_NUM_PHASES; ++i) c->phase_ms[i] = 0.f;
    return SFG_OK;
}

extern "C" int sfg_set_lattice_variant(sfg_context* c, int variant) {
    if (!c) return fail(SFG_ERR_ARG, "sfg_set_lattice_variant: null context");
    if (c->initialized) return fail(SFG_ERR_STATE, "sfg_set_lattice_variant: before sfg_initialize");
    if (variant < 0 || variant > 3)
        return fail(SFG_ERR_ARG, "sfg_set_lattice_variant: 0, 1, 2 or 3");
    c->force_scalar_lattice = variant == 1;
    c->force_vec4_lattice = variant == 2;
    c->split_lattice = variant == 3;
    return SFG_OK;
}

extern "C" int sfg_get_stream(const sfg_context* c, void** s) {
    if (!c || !s) return fail(SFG_ERR_ARG, "sfg_get_stream: null argument");
    *s = (void*)c->stream;
    return SFG_OK;
}
