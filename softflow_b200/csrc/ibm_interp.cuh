// ibm_interp.cuh -- interpolation of the lattice velocity at a marker with
// the force accumulated so far, and the per-marker inputs of the learned
// multi-direct forcing network.  Shared by the plain forcing sweeps and the
// learned seed so that both interpolate identically.
#pragma once
#include <type_traits>
#include "markers.cuh"
#include "lattice.cuh"

namespace sfg {

// u = (j + F/2)/rho at the marker's 4 x 4 stencil with the accumulated force
// acc (immersed_boundary.cpp:174-229 with the stencil weights of the step;
// SOLID rows and rho <= 1e-15 contribute zero).
// Slot of stencil cell (sx, jy) from the marker's slot record (k_tile_fill).
struct StencilSlots {
    int s[8];
    int ty0;
    __device__ __forceinline__ StencilSlots(const MarkerBufs& mb, int m, int iy0) {
        const int4* p = reinterpret_cast<const int4*>(mb.slot8 + 8 * (size_t)m);
        const int4 a = p[0], b = p[1];
        s[0] = a.x; s[1] = a.y; s[2] = a.z; s[3] = a.w;
        s[4] = b.x; s[5] = b.y; s[6] = b.z; s[7] = b.w;
        ty0 = max(iy0 - 1, 0) / TILE_H;
    }
    __device__ __forceinline__ int slot(int sx, int jy) const {
        return s[(jy / TILE_H != ty0 ? 4 : 0) + sx];
    }
};

template <typename S, typename R, typename A = double>
__device__ __forceinline__ double2 interp_u_acc(const ChannelDev& ch, const MarkerBufs& mb, int m,
                                               const S* __restrict__ f,
                                               const int* __restrict__ tile_slot,
                                               const A* __restrict__ acc) {
    (void)tile_slot;
    // compute type: double in FP64 contexts (the reference's arithmetic),
    // float in the FP32-arithmetic modes
    using C = typename std::conditional<sizeof(R) == 8, double, float>::type;
    const int ix0 = mb.ix0[m], iy0 = mb.iy0[m];
    const StencilSlots ss(mb, m, iy0);
    const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
    const double2* wy2 = reinterpret_cast<const double2*>(mb.wy + 4 * (size_t)m);
    const double2 wxa = wx2[0], wxb = wx2[1], wya = wy2[0], wyb = wy2[1];
    const C wxs[4] = {(C)wxa.x, (C)wxa.y, (C)wxb.x, (C)wxb.y};
    const C wys[4] = {(C)wya.x, (C)wya.y, (C)wyb.x, (C)wyb.y};
    int jxs[4];
#pragma unroll
    for (int sx = 0; sx < 4; ++sx) {
        int jx = ix0 - 1 + sx;
        if (jx < 0) jx += ch.nx;
        if (jx >= ch.nx) jx -= ch.nx;
        jxs[sx] = jx;
    }
    C ux = 0, uy = 0;
    // one stencil row at a time: the populations and forces of its four
    // cells are loaded together, then its terms are added in order
#pragma unroll
    for (int sy = 0; sy < 4; ++sy) {
        const int jy = iy0 - 1 + sy;
        R v[4][9];
        A fx[4], fy[4];
        bool in[4], solid[4];
#pragma unroll
        for (int sx = 0; sx < 4; ++sx) {
            const int jx = jxs[sx];
            in[sx] = jy >= 0 && jy < ch.ny && jx >= 0 && jx < ch.nx;
            solid[sx] = in[sx] && cell_kind(ch, jx, jy) == CK_SOLID;
            if (in[sx] && !solid[sx]) {
                const long long n = (long long)jy * ch.pitch + jx;
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    v[sx][q] = PopIO<S, R>::ld(f + ch.f_off + q * ch.plane + n, q);
                const size_t ci = (size_t)ss.slot(sx, jy) * 2 * TILE_CELLS +
                                  (jy % TILE_H) * TILE_W + (jx % TILE_W);
                fx[sx] = acc[ci];
                fy[sx] = acc[ci + TILE_CELLS];
            }
        }
#pragma unroll
        for (int sx = 0; sx < 4; ++sx) {
            if (!in[sx]) continue;
            const C w = wxs[sx] * wys[sy];
            if (w > (C)1e-15) {
                C rho = 0, jxm = 0, jym = 0;
                if (!solid[sx]) {
                    R r, a, b;
                    lattice_moments(v[sx], r, a, b);
                    rho = (C)r;
                    jxm = (C)a;
                    jym = (C)b;
                }
                C cu = 0, cv = 0;
                if (!solid[sx] && rho > (C)1e-15) {
                    if constexpr (sizeof(R) == 8) {
                        cu = (jxm + 0.5 * (double)fx[sx]) / rho;
                        cv = (jym + 0.5 * (double)fy[sx]) / rho;
                    } else {
                        const float inv = __frcp_rn(rho);
                        cu = (jxm + 0.5f * (float)fx[sx]) * inv;
                        cv = (jym + 0.5f * (float)fy[sx]) * inv;
                    }
                }
                ux += cu * w;
                uy += cv * w;
            }
        }
    }
    return make_double2((double)ux, (double)uy);
}

// Moments (rho, jx, jy) of a force tile's cells, computed once per step
// (k_tile_moments) because the populations do not change during the forcing
// sweeps: [slot][TILE_CELLS] records of R, rho = 0 on SOLID rows (where the
// reference's interpolation and density lookup give 0) and outside the
// channel.
template <typename R> struct Mom4;
template <> struct Mom4<double> { using T = double4; };
template <> struct Mom4<float> { using T = float4; };

// interp_u_acc with the step's tile moments and the accumulated force acc
// ([slot][TILE_CELLS] (x, y) pairs): the same terms in the same order.  The loads of a stencil row (moments and force of four cells) are
// issued together before any of their terms is formed, so a marker waits
// for one round of gathers per row instead of one per cell.  FP64
// divides by rho as the reference does (bit for bit); FP32-arithmetic modes
// multiply by one reciprocal per cell.  With NEAR, also the density
// at the node nearest to the marker (immersed_boundary.cpp:262-270: the
// node (int)(x + 0.5), (int)(y + 0.5), density 1 outside the lattice rows),
// taken from the stencil's moments already loaded (the node is stencil
// column and row 1 or 2).
template <typename R, bool NEAR = false>
__device__ __forceinline__ double2 interp_u_mom(const ChannelDev& ch, const MarkerBufs& mb, int m,
                                               const int* __restrict__ tile_slot,
                                               const typename Mom4<R>::T* __restrict__ mom,
                                               const double* __restrict__ acc,
                                               double& rho_near) {
    (void)tile_slot;
    // compute type: double in FP64 contexts (the reference's arithmetic),
    // float in the FP32-arithmetic modes (fewer registers, more resident
    // warps for this latency-bound gather)
    using C = typename std::conditional<sizeof(R) == 8, double, float>::type;
    const int ix0 = mb.ix0[m], iy0 = mb.iy0[m];
    const StencilSlots ss(mb, m, iy0);
    const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
    const double2* wy2 = reinterpret_cast<const double2*>(mb.wy + 4 * (size_t)m);
    const double2 wxa = wx2[0], wxb = wx2[1], wya = wy2[0], wyb = wy2[1];
    const C wxs[4] = {(C)wxa.x, (C)wxa.y, (C)wxb.x, (C)wxb.y};
    const C wys[4] = {(C)wya.x, (C)wya.y, (C)wyb.x, (C)wyb.y};
    int jxs[4];
#pragma unroll
    for (int sx = 0; sx < 4; ++sx) {
        int jx = ix0 - 1 + sx;
        if (jx < 0) jx += ch.nx;
        if (jx >= ch.nx) jx -= ch.nx;
        jxs[sx] = jx;
    }
    // the nearest node's stencil column and row (-1: not wanted, or the
    // density is 1 outside the lattice rows)
    int sxn = -1, syn = -1;
    if (NEAR) {
        rho_near = 1.0;
        const double2 p = mb.pos[m];
        int ixr = (int)(p.x + 0.5);
        const int iyr = (int)(p.y + 0.5);
        if (ixr < 0) ixr += ch.nx;
        if (ixr >= ch.nx) ixr -= ch.nx;
        if (iyr >= 0 && iyr < ch.ny && ixr >= 0 && ixr < ch.nx) {
            sxn = (int)(p.x + 0.5) - ix0 + 1;
            syn = iyr - (iy0 - 1);
            // (always column and row 1 or 2 for a finite position; a
            // non-finite one keeps the density 1)
            if (sxn < 0 || sxn > 3 || syn < 0 || syn > 3) sxn = syn = -1;
        }
    }
    C ux = 0, uy = 0;
#pragma unroll
    for (int row = 0; row < 4; ++row) {
        typename Mom4<R>::T q[4];
        C fx[4], fy[4];
        bool in[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int sy = row, sx = i;
            const int jx = jxs[sx], jy = iy0 - 1 + sy;
            in[i] = jy >= 0 && jy < ch.ny && jx >= 0 && jx < ch.nx;
            const int sl = in[i] ? ss.slot(sx, jy) : -1;
            in[i] = in[i] && sl >= 0;
            if (in[i]) {
                const int cell = (jy % TILE_H) * TILE_W + (jx % TILE_W);
                q[i] = mom[(size_t)sl * TILE_CELLS + cell];
                // (x, y) pairs of R: double2 in FP64 contexts, float2 otherwise
                if constexpr (sizeof(R) == 8) {
                    const double2 a =
                        reinterpret_cast<const double2*>(acc)[(size_t)sl * TILE_CELLS + cell];
                    fx[i] = a.x;
                    fy[i] = a.y;
                } else {
                    const float2 a =
                        reinterpret_cast<const float2*>(acc)[(size_t)sl * TILE_CELLS + cell];
                    fx[i] = a.x;
                    fy[i] = a.y;
                }
            }
        }
        if (NEAR && row == syn) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
                if (i == sxn && in[i]) rho_near = (double)q[i].x;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int sy = row, sx = i;
            if (!in[i]) continue;
            const C w = wxs[sx] * wys[sy];
            if (w > (C)1e-15) {
                const C rho = (C)q[i].x;
                C cu = 0, cv = 0;
                if (rho > (C)1e-15) {
                    if constexpr (sizeof(R) == 8) {
                        cu = ((double)q[i].y + 0.5 * fx[i]) / rho;
                        cv = ((double)q[i].z + 0.5 * fy[i]) / rho;
                    } else {
                        const float inv = __frcp_rn(rho);
                        cu = (q[i].y + 0.5f * fx[i]) * inv;
                        cv = (q[i].z + 0.5f * fy[i]) * inv;
                    }
                }
                ux += cu * w;
                uy += cv * w;
            }
        }
    }
    return make_double2((double)ux, (double)uy);
}

// Inputs of the forcing network in the marker's local frame (tangent t along
// e_prev + e_next, normal n = (-t_y, t_x)):
//   [slip.t, slip.n, dF_prev.t, dF_prev.n, stretch, curvature, u_target.t,
//    u_target.n], slip = u_interp - u_target, u_target = the marker velocity
//   of the previous step (the forcing target, immersed_boundary.cpp:255),
//   stretch = (|e_prev| + |e_next|) / (L0_prev + L0_next) - 1,
//   curvature = atan2(e_prev x e_next, e_prev . e_next) / (0.5 (|e_prev| + |e_next|)).
__device__ __forceinline__ void mdf_features(const ChannelDev& ch, const CapsuleDev& cp,
                                             const MarkerBufs& mb, int m, double2 u_interp,
                                             float* feat, double2& t, double2& nrm) {
    const int k = m - cp.off, n = cp.n;
    const int kp = cp.off + (k - 1 + n) % n, kn = cp.off + (k + 1) % n;
    const double Lx = (double)ch.nx;
    const double2 p = mb.pos[m];
    const double2 ep = min_image_d(p, mb.pos[kp], Lx);
    const double2 en = min_image_d(mb.pos[kn], p, Lx);
    const double tx = ep.x + en.x, ty = ep.y + en.y;
    const double tl = sqrt(tx * tx + ty * ty);
    t = tl > 0.0 ? make_double2(tx / tl, ty / tl) : make_double2(1.0, 0.0);
    nrm = make_double2(-t.y, t.x);
    const double lp = norm_d(ep), ln = norm_d(en);
    const double stretch = (lp + ln) / (mb.rest_len[kp] + mb.rest_len[m]) - 1.0;
    const double curv = atan2(ep.x * en.y - ep.y * en.x, ep.x * en.x + ep.y * en.y) /
                        (0.5 * (lp + ln));
    const double2 ut = mb.vel[m];
    const double2 dp = mb.dFprev[m];
    const double sx = u_interp.x - ut.x, sy = u_interp.y - ut.y;
    feat[0] = (float)(sx * t.x + sy * t.y);
    feat[1] = (float)(sx * nrm.x + sy * nrm.y);
    feat[2] = (float)(dp.x * t.x + dp.y * t.y);
    feat[3] = (float)(dp.x * nrm.x + dp.y * nrm.y);
    feat[4] = (float)stretch;
    feat[5] = (float)curv;
    feat[6] = (float)(ut.x * t.x + ut.y * t.y);
    feat[7] = (float)(ut.x * nrm.x + ut.y * nrm.y);
}

// Per-channel maximum of a non-negative residual kept as float bits (NaN
// becomes the largest value, so it triggers the fallback).
__device__ __forceinline__ void atomic_max_resid(unsigned* slot, double r) {
    const float rf = (float)r;
    atomicMax(slot, isnan(rf) ? 0x7fc00000u : __float_as_uint(rf));
}

// atomic_max_resid for the active lanes of a warp (each calls it once, `on`
// lanes carry a residual; lanes that left the kernel take no part): lanes of
// one channel are reduced first and one lane per channel updates the slot (the max of non-negative floats is the max of their bit
// patterns, NaN mapped above every finite value as in atomic_max_resid).
__device__ __forceinline__ void warp_max_resid(unsigned* slots, int chan, bool on, double r) {
    const float rf = (float)r;
    const unsigned v = on ? (isnan(rf) ? 0x7fc00000u : __float_as_uint(rf)) : 0u;
    const unsigned key = on ? (unsigned)chan : 0xffffffffu;
    const unsigned peers = __match_any_sync(__activemask(), key);
    const unsigned m = __reduce_max_sync(peers, v);   // over the lanes of one key
    const int leader = __ffs(peers) - 1;
    if (on && (threadIdx.x & 31) == leader) atomicMax(&slots[chan], m);
}

}  // namespace sfg
