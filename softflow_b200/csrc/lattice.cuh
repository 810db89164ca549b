// lattice.cuh -- fused lattice step (collide + push-stream + halfway bounce-back),
// the lagged fused scalar step, and the population/macroscopic I/O kernels.
//
// State between steps is the post-stream population field (the reference's
// LatticeField::f_ after LBMSolver::step, lbm_solver.cpp:172-207).  One
// kernel launch reads every population once (own cell, aligned) and writes
// it once (to the downstream neighbour, or reflected into the own cell when
// that neighbour is a wall: the halfway bounce-back of bounce_back.cpp:12-41
// folded into the store).
//
// Storage types: double (FP64), float (FP32), or __half holding f - w
// (FP16-shifted), with FP32 arithmetic for the last two.
#pragma once
#include <type_traits>

#include "collide.cuh"

namespace sfg {

// FP16-shifted storage: h = (f - w_q) * 2^12 in binary16.  The power-of-two
// scale moves the deviations (|f - w| <= ~0.6) away from the subnormal range
// without changing their relative precision.  Stores inside the time loop
// round stochastically: the 13 float mantissa bits below the binary16 LSB
// are dithered with hashed bits before truncation, so rounding errors are
// unbiased and uncorrelated between cells (round-to-nearest gives every cell
// of a uniform row the same error, which acts as a spurious body force).
// Values below the binary16 normal range round to nearest.
constexpr float FP16S_SCALE = 4096.0f;
constexpr float FP16S_UNSCALE = 1.0f / 4096.0f;

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ __half f2h_stochastic(float v, uint32_t r) {
    // branch-free: both roundings, then a select
    const uint32_t u = (__float_as_uint(v) + (r & 0x1FFFu)) & ~0x1FFFu;
    const __half hs = __float2half_rz(__uint_as_float(u));
    const __half hn = __float2half_rn(v);
    return fabsf(v) < 6.103515625e-05f ? hn : hs;
}

template <typename S, typename R>
struct PopIO;
// load / store: populations f (fill, import, export).  ld / st_sr: the
// lattice kernels' working representation -- f for FP64, the deviation
// d = f - w for FP32 arithmetic (FP32 and FP16 storage both keep d).
template <>
struct PopIO<double, double> {
    static __device__ __forceinline__ double ld(const double* p, int) { return __ldg(p); }
    static __device__ __forceinline__ void st_sr(double* p, int, double v, uint32_t) { *p = v; }
    static __device__ __forceinline__ double load(const double* p, int) { return __ldg(p); }
    static __device__ __forceinline__ void store(double* p, int, double v) { *p = v; }
};
// FP32 storage keeps the deviation f - w (the populations stay close to
// their weights, so the stored deviation carries far more significant bits
// than f itself).
template <>
struct PopIO<float, float> {
    static __device__ __forceinline__ float load(const float* p, int q) {
        return float(w_of(q)) + __ldg(p);
    }
    static __device__ __forceinline__ void store(float* p, int q, float v) {
        *p = v - float(w_of(q));
    }
    static __device__ __forceinline__ float ld(const float* p, int) { return __ldg(p); }
    static __device__ __forceinline__ void st_sr(float* p, int, float v, uint32_t) { *p = v; }
};
template <>
struct PopIO<__half, float> {
    static __device__ __forceinline__ float load(const __half* p, int q) {
        return float(w_of(q)) + __half2float(__ldg(p)) * FP16S_UNSCALE;
    }
    static __device__ __forceinline__ void store(__half* p, int q, float v) {
        *p = __float2half_rn((v - float(w_of(q))) * FP16S_SCALE);
    }
    static __device__ __forceinline__ float ld(const __half* p, int) {
        return __half2float(__ldg(p)) * FP16S_UNSCALE;
    }
    // r: per-cell seed; each direction draws its own 13 dither bits
    static __device__ __forceinline__ void st_sr(__half* p, int q, float v, uint32_t r) {
        const uint32_t d = (r + (uint32_t)q * 0x9E3779B9u) * 1664525u + 1013904223u;
        *p = f2h_stochastic(v * FP16S_SCALE, d >> 19);
    }
};

// Per-cell forces of one step: Guo force F, the force G that entered the
// macroscopic velocity the reference's collide reads, and the previous
// step's force P (for the scalar step's velocity).
template <typename R>
struct CellForces {
    R Fx, Fy, Gx, Gy, Px, Py;
};

struct TileView {
    const int* cur_slot;   // global tile -> slot of this step (-1: untouched)
    const int* prev_slot;  // same for the previous step
    const void* cur_fin;   // [slot][2][TILE_CELLS] capped total force, R
    const void* cur_G;     // [slot][2][TILE_CELLS] force before the last MDF sweep, R
    const void* prev_fin;
};

template <typename R>
__device__ __forceinline__ CellForces<R> cell_forces(const ChannelDev& ch, int x, int y,
                                                     const TileView& tv, int stepped) {
    CellForces<R> cf;
    const R Fux = R(ch.F_uni_x), Fuy = R(ch.F_uni_y);
    const R Pux = stepped ? Fux : R(0), Puy = stepped ? Fuy : R(0);
    const bool mdf = ch.ibm_iterations > 1;
    if (ch.cap_end > ch.cap_begin && tv.cur_slot != nullptr) {
        const int t = ch.tile_base + (y / TILE_H) * ch.tiles_x + (x / TILE_W);
        const int cell = (y % TILE_H) * TILE_W + (x % TILE_W);
        const int s = tv.cur_slot[t];
        // the previous step's force is only read where it is used: as G
        // without MDF, and by the scalar step
        const int ps = (!mdf || ch.adr) ? tv.prev_slot[t] : -1;
        const R* fin = static_cast<const R*>(tv.cur_fin);
        const R* gs = static_cast<const R*>(tv.cur_G);
        const R* pfin = static_cast<const R*>(tv.prev_fin);
        if (s >= 0) {
            cf.Fx = fin[(size_t)s * 2 * TILE_CELLS + cell];
            cf.Fy = fin[(size_t)s * 2 * TILE_CELLS + TILE_CELLS + cell];
        } else {
            cf.Fx = Fux;
            cf.Fy = Fuy;
        }
        if (ps >= 0) {
            cf.Px = pfin[(size_t)ps * 2 * TILE_CELLS + cell];
            cf.Py = pfin[(size_t)ps * 2 * TILE_CELLS + TILE_CELLS + cell];
        } else {
            cf.Px = Pux;
            cf.Py = Puy;
        }
        if (mdf) {
            if (s >= 0) {
                cf.Gx = gs[(size_t)s * 2 * TILE_CELLS + cell];
                cf.Gy = gs[(size_t)s * 2 * TILE_CELLS + TILE_CELLS + cell];
            } else {
                cf.Gx = R(0);
                cf.Gy = R(0);
            }
        } else {
            cf.Gx = cf.Px;
            cf.Gy = cf.Py;
        }
    } else {
        cf.Fx = Fux;
        cf.Fy = Fuy;
        cf.Px = Pux;
        cf.Py = Puy;
        // with MDF the reference recomputes the moments with the (empty)
        // immersed-boundary force before colliding
        cf.Gx = mdf ? R(0) : Pux;
        cf.Gy = mdf ? R(0) : Puy;
    }
    return cf;
}

// Lattice work items are 32-cell row runs, one per warp.
constexpr int ITEM_CELLS = 32;
constexpr int ITEMS_PER_CTA = 8;

// Neighbour columns/rows of a cell and the wall flags of its two
// neighbouring rows.  y-wall modes: 0 = SOLID rows 0 and ny-1, 1 = periodic,
// 2 = reflection at the domain edge (scalar with open y).
struct Nbr {
    int xm, xp, ym, yp;
    bool wall_m, wall_p;
};

__device__ __forceinline__ Nbr neighbours(int x, int y, int nx, int ny, int mode) {
    Nbr b;
    b.xm = (x == 0) ? nx - 1 : x - 1;
    b.xp = (x == nx - 1) ? 0 : x + 1;
    if (mode == 1) {
        b.ym = (y == 0) ? ny - 1 : y - 1;
        b.yp = (y == ny - 1) ? 0 : y + 1;
        b.wall_m = b.wall_p = false;
    } else if (mode == 0) {
        b.ym = y - 1;
        b.yp = y + 1;
        b.wall_m = (b.ym == 0);
        b.wall_p = (b.yp == ny - 1);
    } else {
        b.ym = y - 1;
        b.yp = y + 1;
        b.wall_m = (b.ym < 0);
        b.wall_p = (b.yp >= ny);
    }
    return b;
}

// Push the nine post-collision values of cell (x, y): to the downstream
// neighbour, or reflected into the own cell when that neighbour is a wall.
template <typename S, typename R, bool POP = true>
__device__ __forceinline__ void push_cell(S* __restrict__ fd, const R f[9], int x, int y, int n,
                                          int pitch, int plane, const Nbr& b, uint32_t seed) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int cx = cx_of(q), cy = cy_of(q);
        const bool wall = (cy > 0 && b.wall_p) || (cy < 0 && b.wall_m);
        const int xd = cx == 0 ? x : (cx > 0 ? b.xp : b.xm);
        const int yd = cy == 0 ? y : (cy > 0 ? b.yp : b.ym);
        S* p = wall ? fd + opp_of(q) * plane + n : fd + q * plane + yd * pitch + xd;
        const int qs = wall ? opp_of(q) : q;
        if (POP) PopIO<S, R>::st_sr(p, qs, f[q], seed);
        else *p = (S)f[q];
    }
}

template <typename S, typename R, bool ADR>
__global__ void __launch_bounds__(256)
k_lattice_step(const RowItem* __restrict__ items, int n_items, const ChannelDev* __restrict__ chans,
               const S* __restrict__ src, S* __restrict__ dst, const R* __restrict__ gsrc,
               R* __restrict__ gdst, const R* __restrict__ cfield, TileView tv,
               const int* __restrict__ stepped, const int* __restrict__ adr_pending,
               const int* __restrict__ c_fresh, const unsigned* __restrict__ step_ctr) {
    const int item = blockIdx.x * ITEMS_PER_CTA + (threadIdx.x >> 5);
    if (item >= n_items) return;
    const RowItem it = items[item];
    const int lane = threadIdx.x & 31;
    if (lane >= it.len) return;
    const ChannelDev& ch = chans[it.chan];
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x = it.x0 + lane, y = it.y;
    const int n = y * pitch + x;
    const S* __restrict__ fs = src + ch.f_off + n;
    R f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = PopIO<S, R>::ld(fs + q * plane, q);
    R rho, jx, jy;
    lattice_moments(f, rho, jx, jy);
    const int st = stepped[it.chan];
    const CellForces<R> cf = cell_forces<R>(ch, x, y, tv, st);
    R ux, uy;
    cell_velocity(rho, jx, jy, cf.Gx, cf.Gy, ux, uy);
    const int coll = ch.collision;
    if (coll == 2) {
        collide_regularized(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega));
    } else if (coll == 1) {
        collide_mrt(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega), R(ch.mrt_se), R(ch.mrt_s_eps),
                    R(ch.mrt_sq));
    } else {
        collide_bgk(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega));
    }
    const Nbr b = neighbours(x, y, nx, ny, ch.periodic_y ? 1 : 0);
    const uint32_t seed = mix32((uint32_t)n ^ mix32(*step_ctr + 0x51ED270Bu));
    push_cell<S, R>(dst + ch.f_off, f, x, y, n, pitch, plane, b, seed);
    if (ADR) {
        // Scalar step of the previous lattice step (it needs that step's
        // final velocity, which is only known once its populations have been
        // streamed): advection_diffusion.cpp:84-223.
        if (ch.adr && adr_pending[it.chan]) {
            R g[9];
            const R* gp = gsrc + ch.g_off + n;
#pragma unroll
            for (int q = 0; q < 9; ++q) g[q] = gp[q * plane];
            R C;
            if (c_fresh[it.chan]) C = cfield[ch.cell_off + n];
            else C = g[0] + g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8];
            R vx, vy;
            cell_velocity(rho, jx, jy, cf.Px, cf.Py, vx, vy);
            collide_scalar(g, C, vx, vy, R(ch.omega_s));
            const int gmode = ch.periodic_y ? (ch.adr_periodic_y ? 1 : 2) : 0;
            const Nbr gb = gmode == (ch.periodic_y ? 1 : 0) ? b : neighbours(x, y, nx, ny, gmode);
            push_cell<R, R, false>(gdst + ch.g_off, g, x, y, n, pitch, plane, gb, 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// Lattice step of contexts with fluid boundaries other than the periodic
// channel with resting walls: Zou-He inlet / outlet columns, closed boxes,
// moving top / bottom walls (reference lbm_solver.cpp:172-207 with
// moving_wall.cpp:14-64 and the INLET / OUTLET cell types).  One cell per
// thread, push scheme:
//   * SOLID cells do nothing; INLET / OUTLET cells do not collide (the
//     reference collides FLUID cells only) and push their populations as
//     they are;
//   * a population bound for a SOLID cell is reflected into the own cell
//     (halfway bounce-back); bound for a moving wall row it loses
//     2 w_q rho (e_q . u_wall) / cs^2, rho the cell's own density;
//   * without periodic x a population leaving the lattice is dropped (the
//     reference's pull falls back to the node itself there, and Zou-He
//     overwrites exactly those populations afterwards: k_zou_he).
// The working representation (f in FP64, f - w otherwise) reflects the same
// way since w_q = w_opp(q).
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R wall_correction(int q, R rho, double vel) {
    // 2.0 * w[q] * rho * eu_wall / cs2 in the reference's order
    const R eu = R((double)cx_of(q) * vel);
    const R cs2 = R(1.0) / R(3.0);
    return R(2.0) * R(w_of(q)) * rho * eu / cs2;
}

template <typename S, typename R>
__global__ void __launch_bounds__(256)
k_lattice_step_bc(const RowItem* __restrict__ items, int n_items,
                  const ChannelDev* __restrict__ chans, const S* __restrict__ src,
                  S* __restrict__ dst, TileView tv, const int* __restrict__ stepped,
                  const unsigned* __restrict__ step_ctr) {
    const int item = blockIdx.x * ITEMS_PER_CTA + (threadIdx.x >> 5);
    if (item >= n_items) return;
    const RowItem it = items[item];
    const int lane = threadIdx.x & 31;
    if (lane >= it.len) return;
    const ChannelDev& ch = chans[it.chan];
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x = it.x0 + lane, y = it.y;
    const int kind = cell_kind(ch, x, y);
    if (kind == CK_SOLID) return;
    const int n = y * pitch + x;
    const S* __restrict__ fs = src + ch.f_off + n;
    R f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = PopIO<S, R>::ld(fs + q * plane, q);
    R rho, jx, jy;
    lattice_moments(f, rho, jx, jy);
    if (kind == CK_FLUID) {
        const CellForces<R> cf = cell_forces<R>(ch, x, y, tv, stepped[it.chan]);
        R ux, uy;
        cell_velocity(rho, jx, jy, cf.Gx, cf.Gy, ux, uy);
        const int coll = ch.collision;
        if (coll == 2) {
            collide_regularized(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega));
        } else if (coll == 1) {
            collide_mrt(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega), R(ch.mrt_se),
                        R(ch.mrt_s_eps), R(ch.mrt_sq));
        } else {
            collide_bgk(f, rho, ux, uy, cf.Fx, cf.Fy, R(ch.omega));
        }
    }
    const uint32_t seed = mix32((uint32_t)n ^ mix32(*step_ctr + 0x51ED270Bu));
    S* __restrict__ fd = dst + ch.f_off;
    const bool per_x = ch.bc_x == 1;
    const bool mw_bot = !ch.periodic_y && fabs(ch.u_bot) > 1e-15;
    const bool mw_top = !ch.periodic_y && fabs(ch.u_top) > 1e-15;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        int xt = x + cx_of(q), yt = y + cy_of(q);
        if (per_x) xt = xt < 0 ? xt + nx : (xt >= nx ? xt - nx : xt);
        else if (xt < 0 || xt >= nx) continue;
        if (ch.periodic_y) yt = yt < 0 ? yt + ny : (yt >= ny ? yt - ny : yt);
        if (cell_kind(ch, xt, yt) == CK_SOLID) {
            R v = f[q];
            if (yt == 0 && mw_bot) v = v - wall_correction<R>(q, rho, ch.u_bot);
            else if (yt == ny - 1 && mw_top) v = v - wall_correction<R>(q, rho, ch.u_top);
            PopIO<S, R>::st_sr(fd + opp_of(q) * plane + n, opp_of(q), v, seed);
        } else {
            PopIO<S, R>::st_sr(fd + q * plane + yt * pitch + xt, q, f[q], seed);
        }
    }
    if (!per_x) {
        // a direction whose source lies outside the lattice keeps the node's
        // own value, as the reference's pull falls back to the node itself
        // (lbm_solver.cpp:86-96); Zou-He overwrites these at the INLET /
        // OUTLET columns, but interpolated bounce-back reads them first
#pragma unroll
        for (int q = 1; q < 9; ++q) {
            const int xs = x - cx_of(q);
            if (xs < 0 || xs >= nx)
                PopIO<S, R>::st_sr(fd + q * plane + n, q, f[q], seed);
        }
    }
}

// Bouzidi interpolated bounce-back on the streamed populations (reference
// InterpolatedBounceBack::apply, interpolated_bounce_back.cpp:56-96), one
// thread per link.  The reference applies its links one after the other;
// links are launched in levels built on the host so that a link that reads
// what an earlier link writes (or writes what an earlier link reads) runs in
// a later launch, which reproduces that order.  Linear in f with weights
// summing to one, so the working representation (f - w) takes the same
// formula.
template <typename S, typename R>
__global__ void k_ibb(const IbbLink* __restrict__ links, int n,
                      const ChannelDev* __restrict__ chans, S* __restrict__ dst,
                      const unsigned* __restrict__ step_ctr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const IbbLink L = links[i];
    const ChannelDev& ch = chans[L.chan];
    const int nx = ch.nx, ny = ch.ny, plane = (int)ch.plane, pitch = ch.pitch;
    const int q = L.q, o = opp_of(q);
    S* __restrict__ fd = dst + ch.f_off;
    const R fq = PopIO<S, R>::ld(fd + q * plane + L.y * pitch + L.x, q);
    R v;
    if (L.qf < 0.5) {
        int xu = L.x - cx_of(q);
        const int yu = L.y - cy_of(q);
        if (ch.bc_x == 1) xu = ((xu % nx) + nx) % nx;
        if (xu >= 0 && xu < nx && yu >= 0 && yu < ny) {
            const R fu = PopIO<S, R>::ld(fd + q * plane + yu * pitch + xu, q);
            v = R(2.0 * L.qf) * fq + R(1.0 - 2.0 * L.qf) * fu;
        } else {
            v = fq;
        }
    } else {
        const double inv2q = 1.0 / (2.0 * L.qf);
        const R fo = PopIO<S, R>::ld(fd + o * plane + L.y * pitch + L.x, o);
        v = R(inv2q) * fq + R(1.0 - inv2q) * fo;
    }
    const uint32_t seed = mix32((uint32_t)(L.y * pitch + L.x) ^
                                mix32(*step_ctr + 0x6A09E667u + (uint32_t)q));
    PopIO<S, R>::st_sr(fd + o * plane + L.y * pitch + L.x, o, v, seed);
}

// Zou-He velocity inlet (parabolic profile) at x = 0 and pressure outlet at
// x = nx-1 on the streamed populations (reference zou_he_boundary.cpp:17-85),
// one thread per row item (chan, y).  The expressions keep the reference's
// order; in FP32 arithmetic they act on deviations f - w, where the known
// weights sum to 1 and opposite weights cancel.
template <typename S, typename R>
__global__ void k_zou_he(const RowItem* __restrict__ rows, int n_rows,
                         const ChannelDev* __restrict__ chans, S* __restrict__ dst,
                         const unsigned* __restrict__ step_ctr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_rows) return;
    const RowItem it = rows[i];
    const ChannelDev& ch = chans[it.chan];
    const int y = it.y, ny = ch.ny, plane = (int)ch.plane;
    const R base = sizeof(R) == sizeof(double) ? R(0) : R(1);
    S* __restrict__ fd = dst + ch.f_off;
    const uint32_t seed = mix32((uint32_t)y ^ mix32(*step_ctr + 0x2E5BF271u));
    {   // inlet
        const int n = y * ch.pitch;
        R f0 = PopIO<S, R>::ld(fd + 0 * plane + n, 0), f2 = PopIO<S, R>::ld(fd + 2 * plane + n, 2);
        R f3 = PopIO<S, R>::ld(fd + 3 * plane + n, 3), f4 = PopIO<S, R>::ld(fd + 4 * plane + n, 4);
        R f6 = PopIO<S, R>::ld(fd + 6 * plane + n, 6), f7 = PopIO<S, R>::ld(fd + 7 * plane + n, 7);
        const double y_center = (double)ny * 0.5;
        const double H = (double)(ny - 2);
        const double y_norm = ((double)y - y_center) / (H * 0.5);
        const R ux = R(ch.u_in * (1.0 - y_norm * y_norm));
        const R uy = R(0);
        const R rho = (base + (f0 + f2 + f4 + R(2.0) * (f3 + f6 + f7))) / (R(1.0) - ux);
        const R f1 = f3 + (R(2.0) / R(3.0)) * rho * ux;
        const R f5 = f7 + R(0.5) * (f4 - f2) + (R(1.0) / R(6.0)) * rho * ux + R(0.5) * rho * uy;
        const R f8 = f6 - R(0.5) * (f4 - f2) + (R(1.0) / R(6.0)) * rho * ux - R(0.5) * rho * uy;
        PopIO<S, R>::st_sr(fd + 1 * plane + n, 1, f1, seed);
        PopIO<S, R>::st_sr(fd + 5 * plane + n, 5, f5, seed ^ 0x5bd1e995u);
        PopIO<S, R>::st_sr(fd + 8 * plane + n, 8, f8, seed ^ 0x27d4eb2fu);
    }
    {   // outlet
        const int n = y * ch.pitch + ch.nx - 1;
        const R rho = R(ch.rho_out);
        R f0 = PopIO<S, R>::ld(fd + 0 * plane + n, 0), f1 = PopIO<S, R>::ld(fd + 1 * plane + n, 1);
        R f2 = PopIO<S, R>::ld(fd + 2 * plane + n, 2), f4 = PopIO<S, R>::ld(fd + 4 * plane + n, 4);
        R f5 = PopIO<S, R>::ld(fd + 5 * plane + n, 5), f8 = PopIO<S, R>::ld(fd + 8 * plane + n, 8);
        const R ux = R(-1.0) + (base + (f0 + f2 + f4 + R(2.0) * (f1 + f5 + f8))) / rho;
        const R uy = R(0);
        const R f3 = f1 - (R(2.0) / R(3.0)) * rho * ux;
        const R f7 = f5 - R(0.5) * (f4 - f2) - (R(1.0) / R(6.0)) * rho * ux - R(0.5) * rho * uy;
        const R f6 = f8 + R(0.5) * (f4 - f2) - (R(1.0) / R(6.0)) * rho * ux + R(0.5) * rho * uy;
        PopIO<S, R>::st_sr(fd + 3 * plane + n, 3, f3, seed ^ 0x165667b1u);
        PopIO<S, R>::st_sr(fd + 7 * plane + n, 7, f7, seed ^ 0xd3a2646cu);
        PopIO<S, R>::st_sr(fd + 6 * plane + n, 6, f6, seed ^ 0xfd7046c5u);
    }
}

// ---------------------------------------------------------------------------
// Vectorised lattice step: each lane owns 4 consecutive cells of a row, loads
// every population plane with one aligned vector load (16 B for FP32, 8 B for
// FP16-shifted, 2 x 16 B for FP64), collides the 4 cells, and stores.  Planes
// without an x shift (q = 0, 2, 4, and every reflected population) are stored
// as aligned vectors in place.  For the x-shifted planes the lane takes the
// one value that crosses its 4-cell boundary from its neighbour with a warp
// shuffle, so these stores are aligned vectors too; only the ends of each
// 128-cell run use narrow stores.  Needs nx % 4 == 0.
// ---------------------------------------------------------------------------
constexpr int VEC_RUN = 128;   // cells per warp work item

template <typename S>
struct Vec;
template <>
struct Vec<float> {
    static __device__ __forceinline__ void load4(const float* p, float v[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    }
    static __device__ __forceinline__ void store4(float* p, float a, float b, float c, float d) {
        *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
    }
    static __device__ __forceinline__ void store2(float* p, float a, float b) {
        *reinterpret_cast<float2*>(p) = make_float2(a, b);
    }
};
template <>
struct Vec<double> {
    static __device__ __forceinline__ void load4(const double* p, double v[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
    static __device__ __forceinline__ void store4(double* p, double a, double b, double c,
                                                  double d) {
        reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
        reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
    }
    static __device__ __forceinline__ void store2(double* p, double a, double b) {
        *reinterpret_cast<double2*>(p) = make_double2(a, b);
    }
};
template <>
struct Vec<__half> {
    static __device__ __forceinline__ void load4(const __half* p, __half v[4]) {
        const uint2 a = __ldg(reinterpret_cast<const uint2*>(p));
        const __half2 lo = *reinterpret_cast<const __half2*>(&a.x);
        const __half2 hi = *reinterpret_cast<const __half2*>(&a.y);
        v[0] = __low2half(lo); v[1] = __high2half(lo);
        v[2] = __low2half(hi); v[3] = __high2half(hi);
    }
    static __device__ __forceinline__ void store4(__half* p, __half a, __half b, __half c,
                                                  __half d) {
        const __half2 lo = __halves2half2(a, b), hi = __halves2half2(c, d);
        uint2 u;
        u.x = *reinterpret_cast<const unsigned*>(&lo);
        u.y = *reinterpret_cast<const unsigned*>(&hi);
        *reinterpret_cast<uint2*>(p) = u;
    }
    static __device__ __forceinline__ void store2(__half* p, __half a, __half b) {
        *reinterpret_cast<__half2*>(p) = __halves2half2(a, b);
    }
};

// Storage encoding of the generic 4-cell run (FP64, and the identity for the
// FP32 deviations).  FP32-arithmetic runs use load_pairs / store_pairs
// (FP16-shifted: enc4_words) instead.
template <typename S, typename R>
struct Enc {
    static __device__ __forceinline__ R dec(S s, int) { return (R)s; }
    static __device__ __forceinline__ void dec4(const S s[4], int, R out[4]) {
#pragma unroll
        for (int i = 0; i < 4; ++i) out[i] = (R)s[i];
    }
    static __device__ __forceinline__ S enc(R v, int, uint32_t) { return (S)v; }
    static __device__ __forceinline__ void enc4(const R v[4], int, uint32_t, S e[4]) {
#pragma unroll
        for (int i = 0; i < 4; ++i) e[i] = (S)v[i];
    }
};


// Odd 32-bit multipliers for the dither words of the paired FP16 encode,
// one per (direction, pair): murmur3's finaliser of the index, evaluated at
// compile time.
__host__ __device__ constexpr uint32_t dither_mult(uint32_t j) {
    uint32_t x = j * 0x9E3779B9u + 0x632BE5ABu;
    x ^= x >> 16;
    x *= 0x85EBCA6Bu;
    x ^= x >> 13;
    x *= 0xC2B2AE35u;
    x ^= x >> 16;
    return x | 1u;
}

// FP16-shifted encode of four consecutive cells of direction q into two
// words (cells 0, 1 and 2, 3; the first cell in the low half).  The hardware
// stochastic rounding (cvt.rs.f16x2.f32) takes its random bits (0-12 for the
// low half, 16-28 for the high half) from the cell's seed r times a
// per-(q, pair) odd multiplier: one instruction per word, and a bijection of
// r, so every dither field stays exactly uniform (rounding unbiased).  The
// high word of the product would not be: it is bounded by the multiplier.
__device__ __forceinline__ void enc4_words(F2 a, F2 b, int q, uint32_t r, uint32_t& w0,
                                           uint32_t& w1) {
    const F2 sa = vmul(a, vc<F2>(FP16S_SCALE)), sb = vmul(b, vc<F2>(FP16S_SCALE));
    const uint32_t h0 = r * dither_mult((uint32_t)(2 * q)),
                   h1 = r * dither_mult((uint32_t)(2 * q + 1));
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(w0) : "f"(sa.v.y), "f"(sa.v.x), "r"(h0));
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(w1) : "f"(sb.v.y), "f"(sb.v.x), "r"(h1));
}
__device__ __forceinline__ void enc4_words(const float v[4], int q, uint32_t r, uint32_t& w0,
                                           uint32_t& w1) {
    enc4_words(mk2(v[0], v[1]), mk2(v[2], v[3]), q, r, w0, w1);
}

// Stores the encoded words of one plane of a run (FP16 storage): w0 holds
// cells x, x + 1 and w1 cells x + 2, x + 3 of the lane.  dx is the x shift
// (-1, 0, +1); the shifted forms assemble the target words with byte
// permutes from the lane's words and one neighbour word.  All lanes of the
// warp must call this (shuffles).
__device__ __forceinline__ void store_plane4h(__half* __restrict__ row, uint32_t w0, uint32_t w1,
                                              int dx, int x, int x0, int len, int nx, bool active,
                                              int lane, int last_lane) {
    // straight-line code: every store is a single predicated instruction
    if (dx == 0) {
        if (active) *reinterpret_cast<uint2*>(row + x) = make_uint2(w0, w1);
        return;
    }
    const unsigned short lo0 = (unsigned short)(w0 & 0xFFFFu), hi1 = (unsigned short)(w1 >> 16);
    if (dx > 0) {
        const uint32_t prev = __shfl_up_sync(0xffffffffu, w1, 1);
        const uint32_t a = __byte_perm(prev, w0, 0x5432), b = __byte_perm(w0, w1, 0x5432);
        int xe = x0 + len;
        xe = xe >= nx ? xe - nx : xe;
        const bool first = lane == 0;
        if (active && !first) *reinterpret_cast<uint2*>(row + x) = make_uint2(a, b);
        if (active && first) row[x + 1] = __ushort_as_half(lo0);
        if (active && first) *reinterpret_cast<uint32_t*>(row + x + 2) = b;
        if (active && lane == last_lane) row[xe] = __ushort_as_half(hi1);
    } else {
        const uint32_t next = __shfl_down_sync(0xffffffffu, w0, 1);
        const uint32_t a = __byte_perm(w0, w1, 0x5432), b = __byte_perm(w1, next, 0x5432);
        int xb = x0 - 1;
        xb = xb < 0 ? xb + nx : xb;
        const bool last = lane == last_lane;
        if (active && !last) *reinterpret_cast<uint2*>(row + x) = make_uint2(a, b);
        if (active && last) *reinterpret_cast<uint32_t*>(row + x) = a;
        if (active && last) row[x + 2] = __ushort_as_half(hi1);
        if (active && lane == 0) row[xb] = __ushort_as_half(lo0);
    }
}

template <typename S>
__device__ __forceinline__ S shfl_up1(S v) { return __shfl_up_sync(0xffffffffu, v, 1); }
template <typename S>
__device__ __forceinline__ S shfl_down1(S v) { return __shfl_down_sync(0xffffffffu, v, 1); }
template <>
__device__ __forceinline__ __half shfl_up1<__half>(__half v) {
    unsigned short u = __half_as_ushort(v);
    return __ushort_as_half((unsigned short)__shfl_up_sync(0xffffffffu, (unsigned)u, 1));
}
template <>
__device__ __forceinline__ __half shfl_down1<__half>(__half v) {
    unsigned short u = __half_as_ushort(v);
    return __ushort_as_half((unsigned short)__shfl_down_sync(0xffffffffu, (unsigned)u, 1));
}

// Stores 4 encoded values of one plane.  `row` points at the target row of
// the plane, `x` is the lane's first cell, dx the x shift (-1, 0, +1); run
// covers cells [x0, x0 + len) of an nx-periodic row.  All lanes of the warp
// must call this (shuffles).
template <typename S>
__device__ __forceinline__ void store_plane4(S* __restrict__ row, const S v[4], int dx, int x,
                                             int x0, int len, int nx, bool active, int lane,
                                             int last_lane) {
    if (dx == 0) {
        if (active) Vec<S>::store4(row + x, v[0], v[1], v[2], v[3]);
        return;
    }
    if (dx > 0) {
        const S prev = shfl_up1(v[3]);
        if (!active) return;
        if (lane > 0) {
            Vec<S>::store4(row + x, prev, v[0], v[1], v[2]);
        } else {
            row[x + 1] = v[0];
            Vec<S>::store2(row + x + 2, v[1], v[2]);
        }
        if (lane == last_lane) {
            int xe = x0 + len;
            if (xe >= nx) xe -= nx;
            row[xe] = v[3];
        }
    } else {
        const S next = shfl_down1(v[0]);
        if (!active) return;
        if (lane < last_lane) {
            Vec<S>::store4(row + x, v[1], v[2], v[3], next);
        } else {
            Vec<S>::store2(row + x, v[1], v[2]);
            row[x + 2] = v[3];
        }
        if (lane == 0) {
            int xb = x0 - 1;
            if (xb < 0) xb += nx;
            row[xb] = v[0];
        }
    }
}

// POP: f are lattice populations (stored through the population codec);
// otherwise raw values (the scalar's distributions).
template <typename S, typename R, bool POP = true>
__device__ __forceinline__ void push_vec4(S* __restrict__ fd, R f[9][4], int x, int x0, int len,
                                          int nx, int y, int ym, int yp, bool wall_m, bool wall_p,
                                          int pitch, int plane, bool active, int lane,
                                          int last_lane, uint32_t seed) {
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int cx = cx_of(q), cy = cy_of(q);
        const bool wall = (cy > 0 && wall_p) || (cy < 0 && wall_m);
        const int qq = wall ? opp_of(q) : q;
        if constexpr (POP && std::is_same<S, __half>::value && std::is_same<R, float>::value) {
            uint32_t w0, w1;
            enc4_words(f[q], qq, seed, w0, w1);
            if (wall) {
                store_plane4h(fd + qq * plane + y * pitch, w0, w1, 0, x, x0, len, nx, active,
                              lane, last_lane);
            } else {
                const int yd = cy == 0 ? y : (cy > 0 ? yp : ym);
                store_plane4h(fd + q * plane + yd * pitch, w0, w1, cx, x, x0, len, nx, active,
                              lane, last_lane);
            }
            continue;
        }
        S e[4];
        if (POP) {
            Enc<S, R>::enc4(f[q], qq, seed, e);
        } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) e[i] = (S)f[q][i];
        }
        if (wall) {
            store_plane4<S>(fd + qq * plane + y * pitch, e, 0, x, x0, len, nx, active, lane,
                            last_lane);
        } else {
            const int yd = cy == 0 ? y : (cy > 0 ? yp : ym);
            store_plane4<S>(fd + q * plane + yd * pitch, e, cx, x, x0, len, nx, active, lane,
                            last_lane);
        }
    }
}

// Force-tile slots of a 4-cell run (the 4 cells share a tile: x % 4 == 0).
struct RunTiles {
    int s, ps;      // current / previous slot, -1 when untouched (or no tiles)
    int cell;       // index of the run's first cell inside the tile
};

__device__ __forceinline__ RunTiles run_tiles(const ChannelDev& ch, int x, int y,
                                              const TileView& tv) {
    RunTiles r{-1, -1, 0};
    if (ch.cap_end > ch.cap_begin && tv.cur_slot != nullptr) {
        const int t = ch.tile_base + (y / TILE_H) * ch.tiles_x + (x / TILE_W);
        r.cell = (y % TILE_H) * TILE_W + (x % TILE_W);
        r.s = tv.cur_slot[t];
        const bool mdf = ch.ibm_iterations > 1;
        r.ps = (!mdf || ch.adr) ? tv.prev_slot[t] : -1;
    }
    return r;
}

// Forces of cell i of a run (same rules as cell_forces).
template <typename R>
__device__ __forceinline__ CellForces<R> run_forces(const ChannelDev& ch, const RunTiles& rt,
                                                    int i, const TileView& tv, int stepped) {
    CellForces<R> cf;
    const R Fux = R(ch.F_uni_x), Fuy = R(ch.F_uni_y);
    const R Pux = stepped ? Fux : R(0), Puy = stepped ? Fuy : R(0);
    const bool mdf = ch.ibm_iterations > 1;
    const int c = rt.cell + i;
    if (rt.s >= 0) {
        const R* fin = static_cast<const R*>(tv.cur_fin) + (size_t)rt.s * 2 * TILE_CELLS;
        cf.Fx = fin[c];
        cf.Fy = fin[TILE_CELLS + c];
    } else {
        cf.Fx = Fux;
        cf.Fy = Fuy;
    }
    if (rt.ps >= 0) {
        const R* pf = static_cast<const R*>(tv.prev_fin) + (size_t)rt.ps * 2 * TILE_CELLS;
        cf.Px = pf[c];
        cf.Py = pf[TILE_CELLS + c];
    } else {
        cf.Px = Pux;
        cf.Py = Puy;
    }
    if (mdf) {
        if (rt.s >= 0) {
            const R* gs = static_cast<const R*>(tv.cur_G) + (size_t)rt.s * 2 * TILE_CELLS;
            cf.Gx = gs[c];
            cf.Gy = gs[TILE_CELLS + c];
        } else {
            cf.Gx = R(0);
            cf.Gy = R(0);
        }
    } else {
        cf.Gx = cf.Px;
        cf.Gy = cf.Py;
    }
    return cf;
}

// Forces of cells (i, i + 1) of a run in FP32, one 8-byte load per
// component (i is even, the run's first cell a multiple of 4 inside its
// tile): F (Guo force), G (force in the collision's velocity) and P
// (previous step's force, for the scalar step), with the rules of
// run_forces.
struct PairForces {
    F2 Fx, Fy, Gx, Gy, Px, Py;
};
__device__ __forceinline__ F2 ld2(const float* p) {
    F2 r;
    r.v = *reinterpret_cast<const float2*>(p);
    return r;
}
template <bool NEED_P>
__device__ __forceinline__ PairForces pair_forces(const ChannelDev& ch, const RunTiles& rt, int i,
                                                  const TileView& tv, int stepped) {
    PairForces r;
    const float Fux = float(ch.F_uni_x), Fuy = float(ch.F_uni_y);
    const float Pux = stepped ? Fux : 0.f, Puy = stepped ? Fuy : 0.f;
    const bool mdf = ch.ibm_iterations > 1;
    const int c = rt.cell + i;
    if (rt.s >= 0) {
        const float* fin = static_cast<const float*>(tv.cur_fin) + (size_t)rt.s * 2 * TILE_CELLS;
        r.Fx = ld2(fin + c);
        r.Fy = ld2(fin + TILE_CELLS + c);
    } else {
        r.Fx = vc<F2>(Fux);
        r.Fy = vc<F2>(Fuy);
    }
    if (NEED_P || !mdf) {
        if (rt.ps >= 0) {
            const float* pf =
                static_cast<const float*>(tv.prev_fin) + (size_t)rt.ps * 2 * TILE_CELLS;
            r.Px = ld2(pf + c);
            r.Py = ld2(pf + TILE_CELLS + c);
        } else {
            r.Px = vc<F2>(Pux);
            r.Py = vc<F2>(Puy);
        }
    }
    if (mdf) {
        if (rt.s >= 0) {
            const float* gs = static_cast<const float*>(tv.cur_G) + (size_t)rt.s * 2 * TILE_CELLS;
            r.Gx = ld2(gs + c);
            r.Gy = ld2(gs + TILE_CELLS + c);
        } else {
            r.Gx = vc<F2>(0.f);
            r.Gy = r.Gx;
        }
    } else {
        r.Gx = r.Px;
        r.Gy = r.Py;
    }
    return r;
}

// Collision of two cells (paired FP32), bit-identical to collide_cell<float>.
template <int COLL>
__device__ __forceinline__ void collide_cell2(F2 d[9], const DevMoments<F2>& m, F2 rho, F2 ux,
                                              F2 uy, F2 Fx, F2 Fy, const ChannelDev& ch) {
    const int coll = COLL >= 0 ? COLL : ch.collision;
    if (coll == 2)
        reg_collide_v(d, m, rho, ux, uy, Fx, Fy, reg_const<F2>(float(ch.omega)));
    else if (coll == 1)
        mrt_collide_v(d, rho, ux, uy, Fx, Fy,
                      mrt_const<F2>(float(ch.omega), float(ch.mrt_se), float(ch.mrt_s_eps),
                                    float(ch.mrt_sq)));
    else
        bgk_collide_v(d, m.drho, rho, ux, uy, Fx, Fy, bgk_const<F2>(float(ch.omega)));
}

// Forces of 4 consecutive cells (same force tile: x is a multiple of 4).
template <typename R>
__device__ __forceinline__ void cell_forces4(const ChannelDev& ch, int x, int y,
                                             const TileView& tv, int stepped,
                                             CellForces<R> cf[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i) cf[i] = cell_forces<R>(ch, x + i, y, tv, stepped);
}

// Collision of one cell: COLL >= 0 fixes the operator at compile time (one
// operator per kernel keeps the code small); COLL < 0 selects per channel.
template <typename R, int COLL>
__device__ __forceinline__ void collide_cell(R c[9], R rho, R ux, R uy, R Fx, R Fy,
                                             const ChannelDev& ch) {
    const int coll = COLL >= 0 ? COLL : ch.collision;
    if (coll == 2)
        collide_regularized(c, rho, ux, uy, Fx, Fy, R(ch.omega));
    else if (coll == 1)
        collide_mrt(c, rho, ux, uy, Fx, Fy, R(ch.omega), R(ch.mrt_se), R(ch.mrt_s_eps),
                    R(ch.mrt_sq));
    else
        collide_bgk(c, rho, ux, uy, Fx, Fy, R(ch.omega));
}

// Loads and decodes the 4 cells of direction q of a run as two pairs
// (cells 0, 1 and 2, 3): FP32 storage as one 16-byte load, FP16-shifted
// storage as one 8-byte load whose half pairs convert and unscale in pairs.
template <typename S>
__device__ __forceinline__ void load_pairs(const S* p, F2& a, F2& b);
template <>
__device__ __forceinline__ void load_pairs<float>(const float* p, F2& a, F2& b) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    a = mk2(v.x, v.y);
    b = mk2(v.z, v.w);
}
template <>
__device__ __forceinline__ void load_pairs<__half>(const __half* p, F2& a, F2& b) {
    const uint2 w = __ldg(reinterpret_cast<const uint2*>(p));
    F2 u, v;
    u.v = __half22float2(*reinterpret_cast<const __half2*>(&w.x));
    v.v = __half22float2(*reinterpret_cast<const __half2*>(&w.y));
    a = vmul(u, vc<F2>(FP16S_UNSCALE));
    b = vmul(v, vc<F2>(FP16S_UNSCALE));
}

// Stores plane q of a run from its two pairs (see push_vec4).
template <typename S>
__device__ __forceinline__ void store_pairs(S* row, F2 a, F2 b, int q, uint32_t seed, int dx,
                                            int x, int x0, int len, int nx, bool active,
                                            int lane, int last_lane);
template <>
__device__ __forceinline__ void store_pairs<__half>(__half* row, F2 a, F2 b, int q,
                                                    uint32_t seed, int dx, int x, int x0, int len,
                                                    int nx, bool active, int lane,
                                                    int last_lane) {
    uint32_t w0, w1;
    enc4_words(a, b, q, seed, w0, w1);
    store_plane4h(row, w0, w1, dx, x, x0, len, nx, active, lane, last_lane);
}
template <>
__device__ __forceinline__ void store_pairs<float>(float* row, F2 a, F2 b, int, uint32_t, int dx,
                                                   int x, int x0, int len, int nx, bool active,
                                                   int lane, int last_lane) {
    const float v[4] = {a.v.x, a.v.y, b.v.x, b.v.y};
    store_plane4<float>(row, v, dx, x, x0, len, nx, active, lane, last_lane);
}

// lattice_run4 for FP32 arithmetic (FP32 and FP16-shifted storage): the
// populations stay in register pairs from the load to the store, two cells
// per paired instruction.
template <typename S, bool ADR, int COLL>
__device__ __forceinline__ void lattice_run4f(const RowItem& it, const ChannelDev& ch, int st,
                                              const S* __restrict__ src, S* __restrict__ dst,
                                              const float* __restrict__ gsrc,
                                              float* __restrict__ gdst,
                                              const float* __restrict__ cfield,
                                              const TileView& tv, bool adr_on, bool fresh,
                                              uint32_t step_mix, int lane) {
    const bool active = 4 * lane < it.len;
    const int last_lane = (it.len >> 2) - 1;
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x0 = it.x0, y = it.y;
    const int x = x0 + 4 * lane;
    const int n = y * pitch + (active ? x : x0);
    F2 d[2][9];   // [pair][direction]
    {
        const S* fs = src + ch.f_off + n;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            if (active) {
                load_pairs<S>(fs + q * plane, d[0][q], d[1][q]);
            } else {
                d[0][q] = vc<F2>(0.f);
                d[1][q] = vc<F2>(0.f);
            }
        }
    }
    float rho[ADR ? 4 : 1], jx[ADR ? 4 : 1], jy[ADR ? 4 : 1], Px[ADR ? 4 : 1], Py[ADR ? 4 : 1];
    const RunTiles rt = active ? run_tiles(ch, x, y, tv) : RunTiles{-1, -1, 0};
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        const DevMoments<F2> m = dev_moments(d[p]);
        const F2 r = vadd(m.drho, vc<F2>(1.f));
        if (active) {
            const PairForces pf = pair_forces<ADR>(ch, rt, 2 * p, tv, st);
            F2 ux, uy;
            cell_velocity2(r, m.jx, m.jy, pf.Gx, pf.Gy, ux, uy);
            collide_cell2<COLL>(d[p], m, r, ux, uy, pf.Fx, pf.Fy, ch);
            if (ADR) {
                Px[2 * p] = pf.Px.v.x;
                Px[2 * p + 1] = pf.Px.v.y;
                Py[2 * p] = pf.Py.v.x;
                Py[2 * p + 1] = pf.Py.v.y;
            }
        }
        if (ADR) {
            rho[2 * p] = r.v.x;
            rho[2 * p + 1] = r.v.y;
            jx[2 * p] = m.jx.v.x;
            jx[2 * p + 1] = m.jx.v.y;
            jy[2 * p] = m.jy.v.x;
            jy[2 * p + 1] = m.jy.v.y;
        }
    }
    {
        const Nbr b = neighbours(0, y, nx, ny, ch.periodic_y ? 1 : 0);
        const uint32_t seed = mix32((uint32_t)n ^ step_mix);
        S* fd = dst + ch.f_off;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int cx = cx_of(q), cy = cy_of(q);
            const bool wall = (cy > 0 && b.wall_p) || (cy < 0 && b.wall_m);
            const int qq = wall ? opp_of(q) : q;
            if (wall) {
                store_pairs<S>(fd + qq * plane + y * pitch, d[0][q], d[1][q], qq, seed, 0, x, x0,
                               it.len, nx, active, lane, last_lane);
            } else {
                const int yd = cy == 0 ? y : (cy > 0 ? b.yp : b.ym);
                store_pairs<S>(fd + q * plane + yd * pitch, d[0][q], d[1][q], q, seed, cx, x, x0,
                               it.len, nx, active, lane, last_lane);
            }
        }
    }
    if (ADR) {
        if (adr_on) {   // warp-uniform
            float g[9][4];
            const float* gp = gsrc + ch.g_off + n;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                if (active) Vec<float>::load4(gp + q * plane, g[q]);
                else g[q][0] = g[q][1] = g[q][2] = g[q][3] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                float c[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) c[q] = g[q][i];
                if (active) {
                    float C = fresh ? cfield[ch.cell_off + n + i]
                                    : c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7] + c[8];
                    float vx, vy;
                    cell_velocity(rho[i], jx[i], jy[i], Px[i], Py[i], vx, vy);
                    collide_scalar(c, C, vx, vy, float(ch.omega_s));
                }
#pragma unroll
                for (int q = 0; q < 9; ++q) g[q][i] = c[q];
            }
            const int gmode = ch.periodic_y ? (ch.adr_periodic_y ? 1 : 2) : 0;
            const Nbr gb = neighbours(0, y, nx, ny, gmode);
            push_vec4<float, float, false>(gdst + ch.g_off, g, x, x0, it.len, nx, y, gb.ym,
                                           gb.yp, gb.wall_m, gb.wall_p, pitch, plane, active,
                                           lane, last_lane, 0u);
        }
    }
}

template <typename S, typename R, bool ADR, int COLL>
__device__ __forceinline__ void lattice_run4(const RowItem& it, const ChannelDev& ch, int st,
                                             const S* __restrict__ src, S* __restrict__ dst,
                                             const R* __restrict__ gsrc, R* __restrict__ gdst,
                                             const R* __restrict__ cfield, const TileView& tv,
                                             bool adr_on, bool fresh, uint32_t step_mix,
                                             int lane) {
    if constexpr (std::is_same<R, float>::value) {
        lattice_run4f<S, ADR, COLL>(it, ch, st, src, dst, gsrc, gdst, cfield, tv, adr_on, fresh,
                                    step_mix, lane);
        return;
    }
    const bool active = 4 * lane < it.len;
    const int last_lane = (it.len >> 2) - 1;
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x0 = it.x0, y = it.y;
    const int x = x0 + 4 * lane;
    const int n = y * pitch + (active ? x : x0);
    R f[9][4];
    {
        const S* fs = src + ch.f_off + n;
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            S v[4];
            if (active) {
                Vec<S>::load4(fs + q * plane, v);
            } else {
                v[0] = v[1] = v[2] = v[3] = S(0);
            }
            Enc<S, R>::dec4(v, q, f[q]);
        }
    }
    // per cell: forces, moments and collision; the scalar step keeps only
    // the moments and the previous force it needs
    R rho[ADR ? 4 : 1], jx[ADR ? 4 : 1], jy[ADR ? 4 : 1], Px[ADR ? 4 : 1], Py[ADR ? 4 : 1];
    const RunTiles rt = active ? run_tiles(ch, x, y, tv) : RunTiles{-1, -1, 0};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        R c[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) c[q] = f[q][i];
        R r, a, bj;
        lattice_moments(c, r, a, bj);
        if (active) {
            const CellForces<R> cf = run_forces<R>(ch, rt, i, tv, st);
            R ux, uy;
            cell_velocity(r, a, bj, cf.Gx, cf.Gy, ux, uy);
            collide_cell<R, COLL>(c, r, ux, uy, cf.Fx, cf.Fy, ch);
            if (ADR) {
                Px[i] = cf.Px;
                Py[i] = cf.Py;
            }
        }
        if (ADR) {
            rho[i] = r;
            jx[i] = a;
            jy[i] = bj;
        }
#pragma unroll
        for (int q = 0; q < 9; ++q) f[q][i] = c[q];
    }
    const Nbr b = neighbours(0, y, nx, ny, ch.periodic_y ? 1 : 0);
    const uint32_t seed = mix32((uint32_t)n ^ step_mix);
    push_vec4<S, R>(dst + ch.f_off, f, x, x0, it.len, nx, y, b.ym, b.yp, b.wall_m, b.wall_p,
                    pitch, plane, active, lane, last_lane, seed);
    if (ADR) {
        if (adr_on) {   // warp-uniform
            R g[9][4];
            const R* gp = gsrc + ch.g_off + n;
#pragma unroll
            for (int q = 0; q < 9; ++q) {
                if (active) Vec<R>::load4(gp + q * plane, g[q]);
                else g[q][0] = g[q][1] = g[q][2] = g[q][3] = R(0);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                R c[9];
#pragma unroll
                for (int q = 0; q < 9; ++q) c[q] = g[q][i];
                if (active) {
                    R C = fresh ? cfield[ch.cell_off + n + i]
                                : c[0] + c[1] + c[2] + c[3] + c[4] + c[5] + c[6] + c[7] + c[8];
                    R vx, vy;
                    cell_velocity(rho[i], jx[i], jy[i], Px[i], Py[i], vx, vy);
                    collide_scalar(c, C, vx, vy, R(ch.omega_s));
                }
#pragma unroll
                for (int q = 0; q < 9; ++q) g[q][i] = c[q];
            }
            const int gmode = ch.periodic_y ? (ch.adr_periodic_y ? 1 : 2) : 0;
            const Nbr gb = neighbours(0, y, nx, ny, gmode);
            push_vec4<R, R, false>(gdst + ch.g_off, g, x, x0, it.len, nx, y, gb.ym, gb.yp, gb.wall_m,
                            gb.wall_p, pitch, plane, active, lane, last_lane, 0u);
        }
    }
}

// ---------------------------------------------------------------------------
// FP16-shifted storage, eight cells per lane (256-cell runs).  Each lane
// moves 16 bytes per plane per load and store, as the FP32 form does with
// four cells, so the bytes in flight per instruction match FP32 while the
// per-run work (run record, channel record, force-tile slots, neighbour
// shuffles, loads and stores) is spread over twice the cells.  The cells
// are processed as four register pairs: decode (binary16 pair -> FP32 pair),
// moments, velocity, collision, stochastic encode back into the same word,
// so the populations stay packed while the next pair is worked on.
// ---------------------------------------------------------------------------
constexpr int VEC8_RUN = 256;   // cells per warp work item of the 8-cell form (row-major,
                                // continuing over row ends)

__device__ __forceinline__ uint32_t u4_get(const uint4& v, int k) {
    return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w));
}
__device__ __forceinline__ void u4_set(uint4& v, int k, uint32_t w) {
    if (k == 0) v.x = w;
    else if (k == 1) v.y = w;
    else if (k == 2) v.z = w;
    else v.w = w;
}
// binary16 pair (first cell in the low half) -> FP32 deviations
__device__ __forceinline__ F2 dec_word(uint32_t w) {
    F2 u;
    u.v = __half22float2(*reinterpret_cast<const __half2*>(&w));
    return vmul(u, vc<F2>(FP16S_UNSCALE));
}
// FP32 deviations -> binary16 pair, rounded stochastically with the 13-bit
// fields of `bits` (0-12 for the low half, 16-28 for the high half)
__device__ __forceinline__ uint32_t enc_word(F2 a, uint32_t bits) {
    const F2 s = vmul(a, vc<F2>(FP16S_SCALE));
    uint32_t w;
    asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(w) : "f"(s.v.y), "f"(s.v.x), "r"(bits));
    return w;
}

// Stores the eight encoded cells (four words) of one plane of a 256-cell
// run: v holds cells x .. x + 7 of the lane, cell x in the low half of v.x.
// CX is the plane's x shift (-1, 0, +1), the same for every lane: the
// neighbour word it needs is shuffled by all lanes of the warp, whatever
// their own store does (lanes of one run can sit on different rows, so
// some reflect the plane at a wall while others push it).  dx is the lane's
// own shift: CX when it pushes, 0 when it reflects.  The shifted forms build
// the target's aligned 16-byte block from the lane's words and that
// neighbour word (byte permutes).  A segment of consecutive active lanes
// stores the cells at its ends singly: `first` (no active lane of its row
// before it) leaves the block cell its left neighbour pushes in and, for
// dx < 0, stores its first cell at xb; `last` (no active lane of its row
// after it) stores, for dx > 0, its last cell at xe and, for dx < 0, leaves
// the block cell its right neighbour pushes in.
template <int CX>
__device__ __forceinline__ void store_plane8h(__half* __restrict__ row, const uint4 v, int dx,
                                              int x, int xb, int xe, bool active, bool first,
                                              bool last) {
    uint32_t nb = 0u;   // CX > 0: the previous lane's last word; CX < 0: the next lane's first
    if (CX > 0) nb = __shfl_up_sync(0xffffffffu, v.w, 1);
    if (CX < 0) nb = __shfl_down_sync(0xffffffffu, v.x, 1);
    if (dx == 0) {
        if (active) *reinterpret_cast<uint4*>(row + x) = v;
        return;
    }
    if (dx > 0) {
        // block x .. x + 7 receives cells x - 1 .. x + 6
        const uint32_t a0 = __byte_perm(nb, v.x, 0x5432), a1 = __byte_perm(v.x, v.y, 0x5432),
                       a2 = __byte_perm(v.y, v.z, 0x5432), a3 = __byte_perm(v.z, v.w, 0x5432);
        if (active && !first) *reinterpret_cast<uint4*>(row + x) = make_uint4(a0, a1, a2, a3);
        if (active && first) row[x + 1] = __ushort_as_half((unsigned short)(v.x & 0xFFFFu));
        if (active && first) *reinterpret_cast<uint32_t*>(row + x + 2) = a1;
        if (active && first) *reinterpret_cast<uint2*>(row + x + 4) = make_uint2(a2, a3);
        if (active && last) row[xe] = __ushort_as_half((unsigned short)(v.w >> 16));
    } else {
        // block x .. x + 7 receives cells x + 1 .. x + 8
        const uint32_t b0 = __byte_perm(v.x, v.y, 0x5432), b1 = __byte_perm(v.y, v.z, 0x5432),
                       b2 = __byte_perm(v.z, v.w, 0x5432), b3 = __byte_perm(v.w, nb, 0x5432);
        if (active && !last) *reinterpret_cast<uint4*>(row + x) = make_uint4(b0, b1, b2, b3);
        if (active && last) *reinterpret_cast<uint2*>(row + x) = make_uint2(b0, b1);
        if (active && last) *reinterpret_cast<uint32_t*>(row + x + 4) = b2;
        if (active && last) row[x + 6] = __ushort_as_half((unsigned short)(v.w >> 16));
        if (active && first) row[xb] = __ushort_as_half((unsigned short)(v.x & 0xFFFFu));
    }
}

// Forces of cells c .. c + 3 of a run (c = rt.cell + i, i a multiple of 4),
// one 16-byte load per component, with the rules of pair_forces for the
// fluid step without the scalar: F (Guo force) and G (the force in the
// collision's velocity).
struct QuadForces {
    float4 Fx, Fy, Gx, Gy;
};
__device__ __forceinline__ float4 ld4f(const float* p) {
    return __ldg(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ float4 splat4(float a) { return make_float4(a, a, a, a); }
__device__ __forceinline__ QuadForces quad_forces(const ChannelDev& ch, const RunTiles& rt, int i,
                                                  const TileView& tv, int stepped) {
    QuadForces r;
    const bool mdf = ch.ibm_iterations > 1;
    const int c = rt.cell + i;
    if (rt.s >= 0) {
        const float* fin = static_cast<const float*>(tv.cur_fin) + (size_t)rt.s * 2 * TILE_CELLS;
        r.Fx = ld4f(fin + c);
        r.Fy = ld4f(fin + TILE_CELLS + c);
    } else {
        r.Fx = splat4(float(ch.F_uni_x));
        r.Fy = splat4(float(ch.F_uni_y));
    }
    if (mdf) {
        if (rt.s >= 0) {
            const float* gs = static_cast<const float*>(tv.cur_G) + (size_t)rt.s * 2 * TILE_CELLS;
            r.Gx = ld4f(gs + c);
            r.Gy = ld4f(gs + TILE_CELLS + c);
        } else {
            r.Gx = splat4(0.f);
            r.Gy = r.Gx;
        }
    } else if (rt.ps >= 0) {
        const float* pf = static_cast<const float*>(tv.prev_fin) + (size_t)rt.ps * 2 * TILE_CELLS;
        r.Gx = ld4f(pf + c);
        r.Gy = ld4f(pf + TILE_CELLS + c);
    } else {
        r.Gx = splat4(stepped ? float(ch.F_uni_x) : 0.f);
        r.Gy = splat4(stepped ? float(ch.F_uni_y) : 0.f);
    }
    return r;
}
__device__ __forceinline__ F2 quad_pair(const float4& v, int p) {
    return p == 0 ? mk2(v.x, v.y) : mk2(v.z, v.w);
}

// One 256-cell run of the fluid step in FP16-shifted storage (no scalar):
// collide + push stream + halfway bounce-back, the arithmetic of
// lattice_run4f (paired FP32 on deviations).  The dither word of the
// stochastic encode of pair k of plane q is the lane's seed times an odd
// multiplier per (q, k): a bijection of the seed, so each 13-bit field is
// uniform.
// A run is `len` consecutive fluid cells of one channel in row-major order
// starting at (x0, y), so it may continue over row ends (each row's nx is a
// multiple of 8: a lane's eight cells never straddle one): lane i takes
// cells 8i .. 8i + 7 of the run, on its own row.  A segment of active lanes
// ends at a row end, where the stream wraps around the periodic row.
// `pass` selects the lanes (eight cells of one force tile each): 0 all, 1
// those whose tile has no force slot this step (uniform force: they do not
// depend on the step's forcing), 2 those whose tile has one.  Passes 1 and 2
// together write exactly what pass 0 writes.
template <int COLL>
__device__ __forceinline__ void lattice_run8h(const RowItem& it, const ChannelDev& ch, int st,
                                              const __half* __restrict__ src,
                                              __half* __restrict__ dst, const TileView& tv,
                                              uint32_t step_mix, int lane, int pass,
                                              unsigned* __restrict__ status) {
    bool in_run = 8 * lane < it.len;
    const int last_lane = (it.len >> 3) - 1;
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    int x = it.x0 + 8 * lane, y = it.y;
    // row wrap: at most 256 / nx + 1 times for a valid run (bounded; a cell
    // outside the channel is flagged and skipped)
    for (int k = 0; k < 40 && nx > 0 && x >= nx; ++k) {
        x -= nx;
        ++y;
    }
    if (in_run && (nx < 8 || x < 0 || x + 8 > nx || y < 0 || y >= ny)) {
        atomicOr(status, (unsigned)ST_LATTICE_RUN);
        in_run = false;
    }
    const RunTiles rt = in_run ? run_tiles(ch, x, y, tv) : RunTiles{-1, -1, 0};
    const bool active = in_run && (pass == 0 || ((rt.s >= 0) == (pass == 2)));
    const unsigned am = __ballot_sync(0xffffffffu, active);
    if (am == 0u) return;                      // warp-uniform
    const bool first = active && (lane == 0 || x == 0 || !((am >> (lane - 1)) & 1u));
    const bool last = active && (lane == last_lane || x + 8 == nx || !((am >> (lane + 1)) & 1u));
    const int xb = x == 0 ? nx - 1 : x - 1;    // the row's ends wrap (periodic x)
    const int xe = x + 8 == nx ? 0 : x + 8;
    const int n = y * pitch + x;
    uint4 w[9];
    {
        const __half* fs = src + ch.f_off + n;
#pragma unroll
        for (int q = 0; q < 9; ++q)
            w[q] = active ? __ldg(reinterpret_cast<const uint4*>(fs + (size_t)q * plane))
                          : make_uint4(0u, 0u, 0u, 0u);
    }
    const uint32_t seed = mix32((uint32_t)n ^ step_mix);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const QuadForces qf = quad_forces(ch, rt, 4 * h, tv, st);
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int k = 2 * h + p;
            F2 d[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) d[q] = dec_word(u4_get(w[q], k));
            const DevMoments<F2> m = dev_moments(d);
            const F2 r = vadd(m.drho, vc<F2>(1.f));
            F2 ux, uy;
            cell_velocity2(r, m.jx, m.jy, quad_pair(qf.Gx, p), quad_pair(qf.Gy, p), ux, uy);
            collide_cell2<COLL>(d, m, r, ux, uy, quad_pair(qf.Fx, p), quad_pair(qf.Fy, p), ch);
#pragma unroll
            for (int q = 0; q < 9; ++q)
                u4_set(w[q], k, enc_word(d[q], seed * dither_mult((uint32_t)(4 * q + k))));
        }
    }
    // per-lane rows: a plane bound for a wall row is reflected into the own
    // cell (dx = 0); every lane still takes part in the plane's shuffle
    const Nbr b = neighbours(0, in_run ? y : it.y, nx, ny, ch.periodic_y ? 1 : 0);
    __half* fd = dst + ch.f_off;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int cy = cy_of(q);
        const bool wall = (cy > 0 && b.wall_p) || (cy < 0 && b.wall_m);
        const int yd = wall || cy == 0 ? y : (cy > 0 ? b.yp : b.ym);
        __half* row = fd + (wall ? opp_of(q) : q) * plane + yd * pitch;
        const int dx = wall ? 0 : cx_of(q);
        if (cx_of(q) > 0)
            store_plane8h<1>(row, w[q], dx, x, xb, xe, active, first, last);
        else if (cx_of(q) < 0)
            store_plane8h<-1>(row, w[q], dx, x, xb, xe, active, first, last);
        else
            store_plane8h<0>(row, w[q], dx, x, xb, xe, active, first, last);
    }
}

// Persistent 8-cell form (FP16-shifted storage, no scalar): every warp walks
// a contiguous chunk of 256-cell runs, prefetching the next run record.
// `pass` as in lattice_run8h.
template <int COLL>
__global__ void __launch_bounds__(256, 2)
k_lattice_step8h(const RowItem* __restrict__ items, int n_items,
                 const ChannelDev* __restrict__ chans, int n_chans,
                 const __half* __restrict__ src, __half* __restrict__ dst, TileView tv,
                 const int* __restrict__ stepped, const unsigned* __restrict__ step_ctr,
                 int pass, unsigned* __restrict__ status) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int chunk = (n_items + nwarps - 1) / nwarps;
    const int i0 = gwarp * chunk;
    const int i1 = min(n_items, i0 + chunk);
    if (i0 >= i1) return;                      // warp-uniform
    const uint32_t step_mix = mix32(*step_ctr + 0x51ED270Bu);
    RowItem next = items[i0];
    for (int item = i0; item < i1; ++item) {
        const RowItem it = next;
        if (item + 1 < i1) next = items[item + 1];
        if (it.chan < 0 || it.chan >= n_chans || it.len <= 0 || it.len > VEC8_RUN ||
            it.x0 < 0) {                       // warp-uniform: a bad record is skipped
            if (lane == 0) atomicOr(status, (unsigned)ST_LATTICE_RUN);
            continue;
        }
        const ChannelDev& ch = chans[it.chan];
        lattice_run8h<COLL>(it, ch, stepped[it.chan], src, dst, tv, step_mix, lane, pass,
                            status);
    }
}

// Persistent form: every warp walks a contiguous chunk of 128-cell runs,
// prefetching the next run descriptor, so the dependent loads of a run's
// metadata overlap the previous run's work.
// Resident CTAs per SM requested from the compiler: 3 (80 registers) for the
// FP32-arithmetic fluid step, 2 with the fused scalar step, 1 for FP64.
template <typename R, bool ADR>
constexpr int lattice_min_ctas() { return sizeof(R) == 8 ? 1 : (ADR ? 2 : 3); }

template <typename S, typename R, bool ADR, int COLL>
__global__ void __launch_bounds__(256, lattice_min_ctas<R, ADR>())
k_lattice_step4(const RowItem* __restrict__ items, int n_items,
                const ChannelDev* __restrict__ chans, const S* __restrict__ src,
                S* __restrict__ dst, const R* __restrict__ gsrc, R* __restrict__ gdst,
                const R* __restrict__ cfield, TileView tv, const int* __restrict__ stepped,
                const int* __restrict__ adr_pending, const int* __restrict__ c_fresh,
                const unsigned* __restrict__ step_ctr) {
    const int lane = threadIdx.x & 31;
    const int gwarp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int chunk = (n_items + nwarps - 1) / nwarps;
    const int i0 = gwarp * chunk;
    const int i1 = min(n_items, i0 + chunk);
    if (i0 >= i1) return;                      // warp-uniform
    const uint32_t step_mix = mix32(*step_ctr + 0x51ED270Bu);
    RowItem next = items[i0];
    for (int item = i0; item < i1; ++item) {
        const RowItem it = next;
        if (item + 1 < i1) next = items[item + 1];
        const ChannelDev& ch = chans[it.chan];
        const int st = stepped[it.chan];
        bool adr_on = false, fresh = false;
        if (ADR) {
            adr_on = ch.adr && adr_pending[it.chan];
            fresh = adr_on && c_fresh[it.chan] != 0;
        }
        lattice_run4<S, R, ADR, COLL>(it, ch, st, src, dst, gsrc, gdst, cfield, tv, adr_on,
                                      fresh, step_mix, lane);
    }
}

// Scalar step alone (brings the scalar up to date before a host read).
template <typename S, typename R>
__global__ void __launch_bounds__(256)
k_scalar_flush(const RowItem* __restrict__ items, int n_items, const ChannelDev* __restrict__ chans,
               const S* __restrict__ src, const R* __restrict__ gsrc, R* __restrict__ gdst,
               const R* __restrict__ cfield, TileView tv_last, const int* __restrict__ adr_pending,
               const int* __restrict__ c_fresh) {
    const int item = blockIdx.x * ITEMS_PER_CTA + (threadIdx.x >> 5);
    if (item >= n_items) return;
    const RowItem it = items[item];
    const int lane = threadIdx.x & 31;
    if (lane >= it.len) return;
    const ChannelDev& ch = chans[it.chan];
    if (!ch.adr || !adr_pending[it.chan]) return;
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x = it.x0 + lane, y = it.y;
    const int n = y * pitch + x;
    const S* fs = src + ch.f_off + n;
    R f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = PopIO<S, R>::ld(fs + q * plane, q);
    R rho, jx, jy;
    lattice_moments(f, rho, jx, jy);
    // the force of the last completed step (its "cur" tile set)
    const CellForces<R> cf = cell_forces<R>(ch, x, y, tv_last, 1);
    R g[9];
    const R* gp = gsrc + ch.g_off + n;
#pragma unroll
    for (int q = 0; q < 9; ++q) g[q] = gp[q * plane];
    R C;
    if (c_fresh[it.chan]) C = cfield[ch.cell_off + n];
    else C = g[0] + g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8];
    R vx, vy;
    cell_velocity(rho, jx, jy, cf.Fx, cf.Fy, vx, vy);
    collide_scalar(g, C, vx, vy, R(ch.omega_s));
    const int gmode = ch.periodic_y ? (ch.adr_periodic_y ? 1 : 2) : 0;
    push_cell<R, R, false>(gdst + ch.g_off, g, x, y, n, pitch, plane, neighbours(x, y, nx, ny, gmode),
                    0u);
}

// Scalar step of this step right after its lattice step, for contexts with
// capsule chemistry (the chemistry follows it within the step, as in
// Simulation::step, simulation.cpp:636-653).  src: the streamed populations
// of this step; tv: this step's forces.  The concentration of a node whose
// value the chemistry overwrote (cov) is the stored one; the flag is
// consumed here.
template <typename S, typename R>
__global__ void __launch_bounds__(256)
k_scalar_now(const RowItem* __restrict__ items, int n_items, const ChannelDev* __restrict__ chans,
             const S* __restrict__ src, const R* __restrict__ gsrc, R* __restrict__ gdst,
             const R* __restrict__ cfield, unsigned char* __restrict__ cov, TileView tv,
             const int* __restrict__ c_fresh) {
    const int item = blockIdx.x * ITEMS_PER_CTA + (threadIdx.x >> 5);
    if (item >= n_items) return;
    const RowItem it = items[item];
    const int lane = threadIdx.x & 31;
    if (lane >= it.len) return;
    const ChannelDev& ch = chans[it.chan];
    if (!ch.adr) return;
    const int nx = ch.nx, ny = ch.ny, pitch = ch.pitch, plane = (int)ch.plane;
    const int x = it.x0 + lane, y = it.y;
    const int n = y * pitch + x;
    const S* fs = src + ch.f_off + n;
    R f[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = PopIO<S, R>::ld(fs + q * plane, q);
    R rho, jx, jy;
    lattice_moments(f, rho, jx, jy);
    const CellForces<R> cf = cell_forces<R>(ch, x, y, tv, 1);
    R g[9];
    const R* gp = gsrc + ch.g_off + n;
#pragma unroll
    for (int q = 0; q < 9; ++q) g[q] = gp[q * plane];
    R C;
    const bool stored = c_fresh[it.chan] || (cov != nullptr && cov[ch.cell_off + n]);
    if (stored) C = cfield[ch.cell_off + n];
    else C = g[0] + g[1] + g[2] + g[3] + g[4] + g[5] + g[6] + g[7] + g[8];
    if (cov != nullptr) cov[ch.cell_off + n] = 0;
    R vx, vy;
    cell_velocity(rho, jx, jy, cf.Fx, cf.Fy, vx, vy);
    collide_scalar(g, C, vx, vy, R(ch.omega_s));
    const int gmode = ch.periodic_y ? (ch.adr_periodic_y ? 1 : 2) : 0;
    push_cell<R, R, false>(gdst + ch.g_off, g, x, y, n, pitch, plane,
                           neighbours(x, y, nx, ny, gmode), 0u);
}

// ---- host <-> device population transfer (canonical FP64 [9][ny][nx]) ----

template <typename S, typename R>
__global__ void k_pop_import(const double* __restrict__ in, S* __restrict__ out, ChannelDev ch) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 9 * N;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / N);
        const long long r = i % N;
        const int y = (int)(r / ch.nx), x = (int)(r % ch.nx);
        PopIO<S, R>::store(out + ch.f_off + q * ch.plane + (long long)y * ch.pitch + x, q,
                           (R)in[i]);
    }
}

template <typename S>
__device__ __forceinline__ double pop_export_one(const S* p, int q);
template <>
__device__ __forceinline__ double pop_export_one<double>(const double* p, int) { return *p; }
template <>
__device__ __forceinline__ double pop_export_one<float>(const float* p, int) { return (double)*p; }
template <>
__device__ __forceinline__ double pop_export_one<__half>(const __half* p, int q) {
    return w_of(q) + (double)__half2float(*p) * (double)FP16S_UNSCALE;
}

template <typename S>
__global__ void k_pop_export(const S* __restrict__ in, double* __restrict__ out, ChannelDev ch) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 9 * N;
         i += (long long)gridDim.x * blockDim.x) {
        const int q = (int)(i / N);
        const long long r = i % N;
        const int y = (int)(r / ch.nx), x = (int)(r % ch.nx);
        out[i] = pop_export_one<S>(in + ch.f_off + q * ch.plane + (long long)y * ch.pitch + x, q);
    }
}

// Macroscopic state of cell (x, y): rho and u of the current populations with
// the force of the last step, as the reference's LatticeField::
// computeMacroscopic leaves them (lattice_field.cpp:28-73; rho = u = 0 on
// SOLID cells), and that force.  Returns whether the cell is SOLID.
template <typename S, typename R>
__device__ __forceinline__ bool cell_macro(const S* __restrict__ in, const ChannelDev& ch,
                                           const TileView& tv_last, int stepped, int x, int y,
                                           R& rho, R& ux, R& uy, R& Fx, R& Fy) {
    const int kind = cell_kind(ch, x, y);
    const bool solid = kind == CK_SOLID;
    // last step's force (the "cur" tile set of that step); the body force
    // is on FLUID cells only (simulation.cpp:556-560)
    if (!stepped) {
        Fx = R(0);
        Fy = R(0);
    } else {
        CellForces<R> cf = cell_forces<R>(ch, x, y, tv_last, 1);
        Fx = cf.Fx;
        Fy = cf.Fy;
        if (kind != CK_FLUID) {
            bool touched = false;
            if (ch.cap_end > ch.cap_begin && tv_last.cur_slot != nullptr) {
                const int t = ch.tile_base + (y / TILE_H) * ch.tiles_x + (x / TILE_W);
                touched = tv_last.cur_slot[t] >= 0;
            }
            if (!touched) {
                Fx = R(0);
                Fy = R(0);
            }
        }
    }
    if (solid) {
        rho = ux = uy = R(0);
        return true;
    }
    R f[9];
    const long long n = (long long)y * ch.pitch + x;
#pragma unroll
    for (int q = 0; q < 9; ++q) f[q] = PopIO<S, R>::ld(in + ch.f_off + q * ch.plane + n, q);
    R jx, jy;
    lattice_moments(f, rho, jx, jy);
    cell_velocity(rho, jx, jy, Fx, Fy, ux, uy);
    return false;
}

// Macroscopic fields and the last step's force field of one channel.
template <typename S, typename R>
__global__ void k_macro_export(const S* __restrict__ in, ChannelDev ch, TileView tv_last,
                               int stepped, double* __restrict__ rho_o, double* __restrict__ ux_o,
                               double* __restrict__ uy_o, double* __restrict__ Fx_o,
                               double* __restrict__ Fy_o) {
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N;
         i += (long long)gridDim.x * blockDim.x) {
        const int y = (int)(i / ch.nx), x = (int)(i % ch.nx);
        R rho, ux, uy, Fx, Fy;
        cell_macro<S, R>(in, ch, tv_last, stepped, x, y, rho, ux, uy, Fx, Fy);
        if (Fx_o) {
            Fx_o[i] = (double)Fx;
            Fy_o[i] = (double)Fy;
        }
        rho_o[i] = (double)rho;
        ux_o[i] = (double)ux;
        uy_o[i] = (double)uy;
    }
}

// ---------------- thermo reductions over the cells --------------------------
// Partial sums of one block (GlobalStatsWriter::writeTimestep,
// global_stats_writer.cpp:52-81, and Simulation::getMaxSpeed /
// checkStability, simulation.cpp:818-907, over non-SOLID cells).  The double
// products and sums use explicit round-to-nearest intrinsics, so no FMA
// contraction changes them in either translation unit; rho and u are those
// of k_macro_export to the bit.

// Grid (blocks per channel, channels).  Thread t of block b visits cells
// b * 256 + t + k * (256 * blocks per channel) in order; the block's
// partials are combined in a fixed tree, so the result depends only on the
// channel sizes.  parts[channel * gridDim.x + b].
template <typename S, typename R>
__global__ void __launch_bounds__(THERMO_THREADS)
k_thermo_cells(const S* __restrict__ in, const R* __restrict__ g, const ChannelDev* __restrict__ chans,
               TileView tv_last, int stepped, ThermoPart* __restrict__ parts,
               const R* __restrict__ cfield, const unsigned char* __restrict__ cov) {
    __shared__ ThermoPart sp[THERMO_THREADS];
    const ChannelDev& ch = chans[blockIdx.y];
    ThermoPart p;
    thermo_init(p);
    const long long N = (long long)ch.nx * ch.ny;
    for (long long i = blockIdx.x * (long long)THERMO_THREADS + threadIdx.x; i < N;
         i += (long long)gridDim.x * THERMO_THREADS) {
        const int y = (int)(i / ch.nx), x = (int)(i % ch.nx);
        R rho, ux, uy, Fx, Fy;
        if (!cell_macro<S, R>(in, ch, tv_last, stepped, x, y, rho, ux, uy, Fx, Fy)) {
            if (cell_kind(ch, x, y) == CK_FLUID) ++p.fluid;
            const double r = (double)rho, vx = (double)ux, vy = (double)uy;
            if (isnan(r) || isinf(r) || isnan(vx) || isinf(vx) || isnan(vy) || isinf(vy))
                if (i < p.first_bad) p.first_bad = i;
            const double v2 = __dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vy, vy));
            p.sum_rho = __dadd_rn(p.sum_rho, r);
            if (r < p.min_rho) p.min_rho = r;
            if (r > p.max_rho) p.max_rho = r;
            if (v2 > p.max_v2) p.max_v2 = v2;
            p.sum_vel = __dadd_rn(p.sum_vel, __dsqrt_rn(v2));
            p.ke = __dadd_rn(p.ke, __dmul_rn(__dmul_rn(0.5, r), v2));
            ++p.count;
        }
        if (g != nullptr && ch.adr) {
            const long long n = (long long)y * ch.pitch + x;
            R v[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) v[q] = g[ch.g_off + q * ch.plane + n];
            const R c = v[0] + v[1] + v[2] + v[3] + v[4] + v[5] + v[6] + v[7] + v[8];
            const double cc = (cov != nullptr && cov[ch.cell_off + n])
                                  ? (double)cfield[ch.cell_off + n] : (double)c;
            p.sum_c = __dadd_rn(p.sum_c, cc);
        }
    }
    sp[threadIdx.x] = p;
    __syncthreads();
    for (int s = THERMO_THREADS / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) thermo_merge(sp[threadIdx.x], sp[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) parts[(long long)blockIdx.y * gridDim.x + blockIdx.x] = sp[0];
}

}  // namespace sfg
