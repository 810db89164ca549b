// common.cuh -- shared device types and constants for the SoftFlow B200 path.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sfg {

// D2Q9 velocity set in the reference's numbering (src/lbm/lattice.h:12-27):
//   6 2 5
//   3 0 1
//   7 4 8
__host__ __device__ constexpr int cx_of(int q) {
    return q == 1 || q == 5 || q == 8 ? 1 : (q == 3 || q == 6 || q == 7 ? -1 : 0);
}
__host__ __device__ constexpr int cy_of(int q) {
    return q == 2 || q == 5 || q == 6 ? 1 : (q == 4 || q == 7 || q == 8 ? -1 : 0);
}
__host__ __device__ constexpr int opp_of(int q) {
    return q == 0 ? 0 : (q <= 4 ? ((q + 1) % 4) + 1 : ((q - 5 + 2) % 4) + 5);
}
__host__ __device__ constexpr double w_of(int q) {
    return q == 0 ? 4.0 / 9.0 : (q <= 4 ? 1.0 / 9.0 : 1.0 / 36.0);
}
static_assert(opp_of(1) == 3 && opp_of(2) == 4 && opp_of(3) == 1 && opp_of(4) == 2, "opp");
static_assert(opp_of(5) == 7 && opp_of(6) == 8 && opp_of(7) == 5 && opp_of(8) == 6, "opp");

// Force-tile geometry: lattice forces from the immersed boundary live in
// 32 x 8 tiles that are only materialised where markers touch the lattice.
constexpr int TILE_W = 32;
constexpr int TILE_H = 8;
constexpr int TILE_CELLS = TILE_W * TILE_H;
// Classes of force tiles by list length for the spread's work order: the
// passes of 8 markers a tile takes, the last class open-ended.
constexpr int SLOT_CLASSES = 16;
__host__ __device__ __forceinline__ int slot_class(int cnt) {
    const int p = (cnt + 7) >> 3;
    return p < SLOT_CLASSES - 1 ? p : SLOT_CLASSES - 1;
}

// Storage precision of the populations.
enum Precision : int { PREC_FP64 = 0, PREC_FP32 = 1, PREC_FP16S = 2 };

// Per-channel constants, read by every kernel (device copy in global memory).
struct ChannelDev {
    int nx, ny, pitch;          // pitch: row stride in elements
    int periodic_y;             // 0: rows 0 and ny-1 are SOLID walls
    long long plane;            // elements per population plane (ny * pitch)
    long long cell_off;         // offset of this channel in one-plane arrays
    long long f_off;            // = 9 * cell_off: plane 0 in the population buffers
    long long g_off;            // = 9 * cell_off: plane 0 in the scalar buffers
    int collision;              // 0 BGK, 1 MRT, 2 regularized
    int ibm_iterations;
    double omega, tau;
    double mrt_se, mrt_s_eps, mrt_sq;
    double body_fx, body_fy;
    double max_force;
    double F_uni_x, F_uni_y;    // capped body force (FLUID cells, untouched tiles)
    double dt;
    // scalar transport
    int adr, adr_periodic_y;
    double omega_s;
    // force tiles
    int tiles_x, tiles_y;
    int tile_base;              // first global tile index of this channel
    // markers / capsules
    int cap_begin, cap_end;
    int mk_begin, mk_end;
    // contact grid (reference cell_list.h:36-87)
    int ncx, ncy, cell_base;
    double cdx, cdy, y_bot, y_top;
    double rep_epsilon, rep_sigma, rep_r_cut, rep_damping, rep_friction;
    int rep_power;
    int brute_contact;          // <= 100 markers: all pairs, one-sided
    // learned multi-direct forcing
    int learned;                // 1: network seed + one sweep, plain sweeps as fallback
    float mdf_threshold;        // no-slip residual (lu/step) above which it falls back
    // fluid boundaries: x columns as BoundaryType (0 Zou-He inlet / outlet,
    // 1 periodic, 2 SOLID); Zou-He inlet centre-line speed and outlet
    // density; moving top / bottom wall speeds (0 when at rest)
    int bc_x;
    int bc_active;              // needs the boundary-aware lattice kernel
    double u_in, rho_out, u_top, u_bot;
    const unsigned char* mask;  // device cell types [ny][nx] of a channel with
                                // pillars, null otherwise
    int chem;                   // capsule chemistry after the scalar step
    int adr_now;                // scalar step inside its own step (not lagged)
    const double* pillars;      // [n_pillars][5]: kind (0 circle, 1 rectangle), a, b, c, d
    int n_pillars;
};

// Cell types of a channel (reference CellType, core/types.h:48-56), as
// LBMSolver::initialize sets them (lbm_solver.cpp:130-160): rows 0 and ny-1
// SOLID unless periodic in y; Zou-He channels have an INLET column at x = 0
// and an OUTLET column at x = nx-1 (rows 1..ny-2); closed boxes SOLID
// columns 0 and nx-1.  Channels with pillars read the types from a mask
// built on the host (device code only; host code uses the mask array).
enum CellKind : int { CK_FLUID = 0, CK_SOLID = 1, CK_INLET = 2, CK_OUTLET = 3 };
__host__ __device__ __forceinline__ int cell_kind(const ChannelDev& ch, int x, int y) {
#ifdef __CUDA_ARCH__
    if (ch.mask != nullptr) return ch.mask[y * ch.nx + x];
#endif
    if (y == 0 || y == ch.ny - 1) return ch.periodic_y ? CK_FLUID : CK_SOLID;
    if (ch.bc_x == 0) {
        if (x == 0) return CK_INLET;
        if (x == ch.nx - 1) return CK_OUTLET;
    } else if (ch.bc_x == 2) {
        if (x == 0 || x == ch.nx - 1) return CK_SOLID;
    }
    return CK_FLUID;
}

// Per-capsule constants (reference Capsule members, capsule.h:77-142).
struct CapsuleDev {
    int off, n, chan, model;
    int type;                   // Capsule::getTypeId (chemistry parameters)
    int use_helfrich;
    double k_stretch, G_s, C_skalak;
    double wlc_L_max_ratio, wlc_kBT_p, wlc_k_pow;
    double k_bend, k_area, k_perimeter, gamma_visc, eta_membrane;
    double rest_area, rest_perimeter;
    int periodic_nx;
};

// One interpolated bounce-back link (reference InterpolatedBounceBack::Link):
// non-SOLID node (x, y) of channel chan whose direction q points into a
// SOLID node, wall at the fraction qf of the link.
struct IbbLink {
    int chan, x, y, q;
    double qf;
};

// Partial thermo sums of one block of cells (see k_thermo_cells).
constexpr int THERMO_THREADS = 256;
struct ThermoPart {
    double sum_rho, min_rho, max_rho, max_v2, sum_vel, ke, sum_c;
    long long count, first_bad, fluid;
};
constexpr long long THERMO_NONE = 0x7fffffffffffffffLL;

__device__ __forceinline__ void thermo_init(ThermoPart& p) {
    p.sum_rho = p.sum_vel = p.ke = p.sum_c = p.max_v2 = 0.0;
    p.min_rho = 1e30;
    p.max_rho = -1e30;
    p.count = 0;
    p.fluid = 0;
    p.first_bad = THERMO_NONE;
}

// Comparisons as the reference writes them: a NaN never replaces a value.
__device__ __forceinline__ void thermo_merge(ThermoPart& a, const ThermoPart& b) {
    a.sum_rho = __dadd_rn(a.sum_rho, b.sum_rho);
    a.sum_vel = __dadd_rn(a.sum_vel, b.sum_vel);
    a.ke = __dadd_rn(a.ke, b.ke);
    a.sum_c = __dadd_rn(a.sum_c, b.sum_c);
    if (b.min_rho < a.min_rho) a.min_rho = b.min_rho;
    if (b.max_rho > a.max_rho) a.max_rho = b.max_rho;
    if (b.max_v2 > a.max_v2) a.max_v2 = b.max_v2;
    a.count += b.count;
    a.fluid += b.fluid;
    if (b.first_bad < a.first_bad) a.first_bad = b.first_bad;
}

// Work item of the lattice kernels: one row segment of one channel.
struct RowItem {
    int chan, y, x0, len;
};

// Multi-direct forcing launch modes.
//   MDF_PLAIN   : the reference sweeps; on a learned channel only when its
//                 gate residual exceeded the threshold (fallback), restarting
//                 from the force after the membrane spread (acc0);
//   MDF_SEED    : spread of the network's correction (learned channels);
//   MDF_LEARNED : the one plain sweep after the seed (learned channels); its
//                 interpolation gives the gate residual, its spread finishes
//                 the step's force unless the channel falls back.
enum MdfMode : int { MDF_PLAIN = 0, MDF_SEED = 1, MDF_LEARNED = 2 };

// A learned channel falls back when its residual is above the threshold or
// not a number (the residual is kept as the bits of a non-negative float).
__device__ __forceinline__ bool mdf_fallback(unsigned resid_bits, float thr) {
    return !(__uint_as_float(resid_bits) <= thr);
}

// Whether a channel takes part in a correction sweep (sweep >= 1) of the
// given mode.
__device__ __forceinline__ bool mdf_active(const ChannelDev& ch, int mode,
                                           const unsigned* resid_gate, int chan) {
    if (mode != MDF_PLAIN) return ch.learned != 0;
    return !ch.learned || mdf_fallback(resid_gate[chan], ch.mdf_threshold);
}

// Status word bits written by kernels (host reads them after a sync).
enum StatusBits : unsigned {
    ST_NAN_MARKER = 1u,         // non-finite marker position seen
    ST_LIST_OVERFLOW = 2u,      // a per-tile marker list exceeded its capacity
    ST_CAPSULE_TOO_BIG = 4u,    // a capsule exceeded the per-warp node capacity
    ST_TENSOR_TIMEOUT = 8u,     // a tensor-core completion wait gave up
    ST_LATTICE_RUN = 16u,       // a lattice run record or cell out of range (skipped)
};

}  // namespace sfg
