// markers.cu -- marker-side kernels (FP64, compiled with --fmad=false).
//
// Membrane mechanics follow reference src/membrane/capsule.cpp:149-671,
// contact follows src/membrane/repulsion.cpp:6-284 with the cell list of
// src/membrane/cell_list.h:36-146, and the immersed-boundary coupling
// follows src/coupling/immersed_boundary.cpp:25-286.
//
// Spreading is a deterministic gather: every lattice cell of a touched
// 32 x 8 force tile sums the contributions of the markers whose 4 x 4
// stencil covers it, in ascending marker order (the reference's serial
// order), with no floating-point atomics.
#include <climits>

#include "markers.cuh"
#include "lattice.cuh"
#include "sfg_internal.h"
#include "ibm_interp.cuh"

namespace sfg {

// ============================ membrane forces ==============================
// One warp per capsule.  Nodes are staged in shared memory; lanes work on
// nodes/edges in parallel; the ring reductions (area, perimeter) run
// sequentially in lane 0 in the reference's order.  Each node applies the
// contributions of its two edges (or three bending stencils) in the order
// in which the reference's edge loop reaches them.

constexpr int MEM_WARPS = 4;
constexpr int MEM_DOUBLES_PER_NODE = 11;  // P, F, E, GN, GP (2 each) + OK

__device__ __forceinline__ void apply_edges(double2* F, const double2* E, const double* OK, int n,
                                            int k, double s_first, double s_second) {
    // node k is the first node of edge k and the second node of edge k-1
    double2 a = F[k];
    if (k == 0) {
        if (OK[0] != 0.0) { a.x = a.x + s_first * E[0].x; a.y = a.y + s_first * E[0].y; }
        if (n > 1 && OK[n - 1] != 0.0) {
            a.x = a.x + s_second * E[n - 1].x;
            a.y = a.y + s_second * E[n - 1].y;
        }
    } else {
        if (OK[k - 1] != 0.0) {
            a.x = a.x + s_second * E[k - 1].x;
            a.y = a.y + s_second * E[k - 1].y;
        }
        if (OK[k] != 0.0) { a.x = a.x + s_first * E[k].x; a.y = a.y + s_first * E[k].y; }
    }
    F[k] = a;
}
// s_first / s_second are +1 or -1: multiplying by them is exact, so
// a + (-1) * e == a - e bit for bit.

__global__ void k_membrane(const CapsuleDev* __restrict__ caps, int ncaps, MarkerBufs mb,
                           int* __restrict__ has_prev, int maxn, unsigned* status) {
    extern __shared__ double smem[];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const int c = blockIdx.x * MEM_WARPS + warp;
    if (c >= ncaps) return;
    double* base = smem + (size_t)warp * MEM_DOUBLES_PER_NODE * maxn;
    double2* P = reinterpret_cast<double2*>(base);
    double2* F = P + maxn;
    double2* E = F + maxn;
    double2* GN = E + maxn;
    double2* GP = GN + maxn;
    double* OK = reinterpret_cast<double*>(GP + maxn);
    const CapsuleDev cp = caps[c];
    const int n = cp.n, off = cp.off;
    if (n > maxn) {
        if (lane == 0) atomicOr(status, (unsigned)ST_CAPSULE_TOO_BIG);
        return;
    }
    const double Lx = (double)cp.periodic_nx;
    for (int k = lane; k < n; k += 32) {
        P[k] = mb.pos[off + k];
        F[k] = make_double2(0.0, 0.0);
    }
    __syncwarp();

    // ---- stretching (capsule.cpp:338-470) ----
    for (int i = lane; i < n; i += 32) {
        const int j = (i + 1) % n;
        const double2 diff = min_image_d(P[j], P[i], Lx);
        const double L = norm_d(diff);
        if (L < 1e-15) { OK[i] = 0.0; continue; }
        const double L0 = mb.rest_len[off + i];
        double F_mag;
        if (cp.model == 1) {            // Neo-Hookean
            double lambda = L / L0;
            double inv3 = 1.0 / (lambda * lambda * lambda);
            F_mag = cp.G_s * (lambda - inv3);
        } else if (cp.model == 2) {     // Skalak
            double lambda = L / L0;
            double l2 = lambda * lambda;
            F_mag = cp.G_s * lambda * (l2 - 1.0) * (1.0 + cp.C_skalak);
        } else if (cp.model == 3) {     // WLC + power-law repulsion
            double L_max = cp.wlc_L_max_ratio * L0;
            double x = L / L_max;
            if (x > 0.99) x = 0.99;
            double F_wlc = cp.wlc_kBT_p * (1.0 / (4.0 * (1.0 - x) * (1.0 - x)) - 0.25 + x);
            double F_pow = -cp.wlc_k_pow / L;
            F_mag = F_wlc + F_pow;
        } else {                        // Hookean
            F_mag = cp.k_stretch * (L / L0 - 1.0);
        }
        const double2 dir = make_double2(diff.x / L, diff.y / L);
        E[i] = make_double2(dir.x * F_mag, dir.y * F_mag);
        OK[i] = 1.0;
    }
    __syncwarp();
    for (int k = lane; k < n; k += 32) apply_edges(F, E, OK, n, k, 1.0, -1.0);
    __syncwarp();

    // ---- bending (capsule.cpp:476-541) ----
    if (cp.use_helfrich) {
        for (int i = lane; i < n; i += 32) {
            const int ip = (i - 1 + n) % n, in = (i + 1) % n;
            const double2 ep = min_image_d(P[i], P[ip], Lx);
            const double2 en = min_image_d(P[in], P[i], Lx);
            const double lp2 = ep.x * ep.x + ep.y * ep.y, ln2 = en.x * en.x + en.y * en.y;
            if (lp2 < 1e-30 || ln2 < 1e-30) { OK[i] = 0.0; continue; }
            const double dth = atan2(ep.x * en.y - ep.y * en.x, ep.x * en.x + ep.y * en.y) -
                               mb.rest_ang[off + i];
            const double cc = -cp.k_bend * dth / mb.rest_ds[off + i];
            const double2 gn = make_double2(-en.y / ln2, en.x / ln2);
            const double2 gp = make_double2(-ep.y / lp2, ep.x / lp2);
            GN[i] = make_double2(gn.x * cc, gn.y * cc);
            GP[i] = make_double2(gp.x * cc, gp.y * cc);
            E[i] = make_double2((gn.x + gp.x) * cc, (gn.y + gp.y) * cc);
            OK[i] = 1.0;
        }
        __syncwarp();
        for (int k = lane; k < n; k += 32) {
            // stencils i in {k-1, k, k+1} touch node k; apply in loop order
            int ids[3] = {(k - 1 + n) % n, k, (k + 1) % n};
            for (int a = 0; a < 3; ++a)
                for (int b = a + 1; b < 3; ++b)
                    if (ids[b] < ids[a]) { int t = ids[a]; ids[a] = ids[b]; ids[b] = t; }
            double2 acc = F[k];
            for (int a = 0; a < 3; ++a) {
                const int i = ids[a];
                if (a > 0 && i == ids[a - 1]) continue;
                if (OK[i] == 0.0) continue;
                if ((i + 1) % n == k) { acc.x = acc.x + GN[i].x; acc.y = acc.y + GN[i].y; }
                if ((i - 1 + n) % n == k) { acc.x = acc.x + GP[i].x; acc.y = acc.y + GP[i].y; }
                if (i == k) { acc.x = acc.x - E[i].x; acc.y = acc.y - E[i].y; }
            }
            F[k] = acc;
        }
    } else {
        for (int i = lane; i < n; i += 32) {
            const double2 dp = min_image_d(P[(i - 1 + n) % n], P[i], Lx);
            const double2 dn = min_image_d(P[(i + 1) % n], P[i], Lx);
            const double2 lap = make_double2(dp.x + dn.x, dp.y + dn.y);
            F[i] = make_double2(F[i].x + lap.x * cp.k_bend, F[i].y + lap.y * cp.k_bend);
        }
    }
    __syncwarp();

    // ---- ring reductions in the reference's order (capsule.cpp:175-204) ----
    // The per-edge terms (minimum-image edge vector, edge length) are formed
    // by the lanes in parallel, with the same expressions; lane 0 then sums
    // them in the reference's order, so the sums are the same bit for bit.
    for (int i = lane; i < n; i += 32) {
        const double2 d = min_image_d(P[(i + 1) % n], P[i], Lx);
        GN[i] = d;
        E[i].x = norm_d(d);
    }
    __syncwarp();
    double sarea = 0.0, perim = 0.0;
    if (lane == 0) {
        if (Lx > 0.0) {
            double2 cur = P[0];
            for (int i = 0; i < n; ++i) {
                double2 nxt;
                if (i + 1 < n) {
                    const double2 d = GN[i];
                    nxt = make_double2(cur.x + d.x, cur.y + d.y);
                } else {
                    nxt = P[0];
                }
                sarea += cur.x * nxt.y - cur.y * nxt.x;
                cur = nxt;
            }
        } else {
            for (int i = 0; i < n; ++i) {
                const double2 a = P[i], b = P[(i + 1) % n];
                sarea += a.x * b.y - a.y * b.x;
            }
        }
        for (int i = 0; i < n; ++i) perim += E[i].x;
    }
    sarea = __shfl_sync(0xffffffffu, sarea, 0);
    perim = __shfl_sync(0xffffffffu, perim, 0);

    // ---- area penalty (capsule.cpp:547-586) ----
    {
        const double A = 0.5 * fabs(sarea), A0 = cp.rest_area;
        if (!(A0 < 1e-15)) {
            const double coeff = -cp.k_area * (A - A0) / A0;
            const double sign = (sarea >= 0.0) ? 1.0 : -1.0;
            for (int i = lane; i < n; i += 32) {
                const double2 ep = min_image_d(P[i], P[(i - 1 + n) % n], Lx);
                const double2 en = min_image_d(P[(i + 1) % n], P[i], Lx);
                double2 o = make_double2((ep.y + en.y) * 0.5, (-ep.x + -en.x) * 0.5);
                const double len = norm_d(o);
                if (len < 1e-15) continue;
                o = make_double2(o.x / len * sign, o.y / len * sign);
                F[i] = make_double2(F[i].x + o.x * coeff, F[i].y + o.y * coeff);
            }
        }
    }
    __syncwarp();

    // ---- perimeter penalty (capsule.cpp:588-604) ----
    {
        const double P0 = cp.rest_perimeter;
        if (!(P0 < 1e-15)) {
            const double coeff = -cp.k_perimeter * (perim - P0) / P0;
            for (int i = lane; i < n; i += 32) {
                const double2 diff = min_image_d(P[(i + 1) % n], P[i], Lx);
                const double L = norm_d(diff);
                if (L < 1e-15) { OK[i] = 0.0; continue; }
                E[i] = make_double2(diff.x / L * coeff, diff.y / L * coeff);
                OK[i] = 1.0;
            }
            __syncwarp();
            for (int k = lane; k < n; k += 32) apply_edges(F, E, OK, n, k, -1.0, 1.0);
            __syncwarp();
        }
    }

    // ---- lab-frame damping (capsule.cpp:606-610) ----
    for (int k = lane; k < n; k += 32) {
        const double2 v = mb.vel[off + k];
        F[k] = make_double2(F[k].x - v.x * cp.gamma_visc, F[k].y - v.y * cp.gamma_visc);
    }
    __syncwarp();

    // ---- Kelvin-Voigt membrane viscosity (capsule.cpp:612-671) ----
    if (cp.eta_membrane > 0.0) {
        if (!has_prev[c]) {
            for (int i = lane; i < n; i += 32)
                mb.prev_len[off + i] = norm_d(min_image_d(P[(i + 1) % n], P[i], Lx));
            __syncwarp();
            if (lane == 0) has_prev[c] = 1;
        } else {
            for (int i = lane; i < n; i += 32) {
                const double2 diff = min_image_d(P[(i + 1) % n], P[i], Lx);
                const double L = norm_d(diff);
                if (L < 1e-15) { OK[i] = 0.0; continue; }
                const double strain = (L - mb.prev_len[off + i]) / mb.rest_len[off + i];
                const double Fv = cp.eta_membrane * strain;
                E[i] = make_double2(diff.x / L * Fv, diff.y / L * Fv);
                OK[i] = 1.0;
                mb.prev_len[off + i] = L;
            }
            __syncwarp();
            for (int k = lane; k < n; k += 32) apply_edges(F, E, OK, n, k, 1.0, -1.0);
            __syncwarp();
        }
    }
    for (int k = lane; k < n; k += 32) mb.frc[off + k] = F[k];
}

// ================================ contact ==================================

__device__ __forceinline__ int contact_cell(const ChannelDev& ch, double2 p) {
    if (!finite2(p)) return 0;
    const double Lx = (double)ch.nx;
    double px = p.x - 0.0;
    px = fmod(px, Lx);
    if (px < 0.0) px += Lx;
    int cx = (int)floor(px / ch.cdx);
    int cy = (int)floor((p.y - ch.y_bot) / ch.cdy);
    if (cx < 0) cx = 0;
    if (cx >= ch.ncx) cx = ch.ncx - 1;
    if (cy < 0) cy = 0;
    if (cy >= ch.ncy) cy = ch.ncy - 1;
    return cy * ch.ncx + cx;
}

__device__ __forceinline__ double2 pair_force(const ChannelDev& ch, double2 pa, double2 va,
                                              double2 pb, double2 vb) {
    const double Lx = (double)ch.nx;
    double2 diff = make_double2(pa.x - pb.x, pa.y - pb.y);
    if (Lx > 0.0) {
        if (diff.x > 0.5 * Lx) diff.x -= Lx;
        if (diff.x < -0.5 * Lx) diff.x += Lx;
    }
    const double r = norm_d(diff);
    if (r < 1e-15 || r >= ch.rep_r_cut) return make_double2(0.0, 0.0);
    const double2 nrm = make_double2(diff.x / r, diff.y / r);
    const double F_rep = ch.rep_epsilon * pow(ch.rep_sigma / r, (double)ch.rep_power);
    double F_n = F_rep;
    double2 F_t = make_double2(0.0, 0.0);
    if (ch.rep_damping > 0.0 || ch.rep_friction > 0.0) {
        const double2 vr = make_double2(va.x - vb.x, va.y - vb.y);
        const double v_n = vr.x * nrm.x + vr.y * nrm.y;
        F_n = F_rep - ch.rep_damping * v_n;
        if (F_n < 0.0) F_n = 0.0;
        if (ch.rep_friction > 0.0) {
            const double2 vt = make_double2(vr.x - nrm.x * v_n, vr.y - nrm.y * v_n);
            const double vtm = norm_d(vt);
            if (vtm > 1e-12) {
                const double s = -ch.rep_friction * F_n;
                F_t = make_double2(vt.x / vtm * s, vt.y / vtm * s);
            }
        }
    }
    return make_double2(nrm.x * F_n + F_t.x, nrm.y * F_n + F_t.y);
}

__global__ void k_contact_bin(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                              int* __restrict__ cell_of, int* __restrict__ cell_cnt) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    if (ch.brute_contact) return;
    const int c = ch.cell_base + contact_cell(ch, mb.pos[m]);
    cell_of[m] = c;
    atomicAdd(&cell_cnt[c], 1);
}

__global__ void k_contact_fill(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                               const int* __restrict__ cell_of, const int* __restrict__ cell_start,
                               int* __restrict__ cursor, int* __restrict__ list) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    if (ch.brute_contact) return;
    const int c = cell_of[m];
    list[cell_start[c] + atomicAdd(&cursor[c], 1)] = m;
}

// Cells hold a handful of markers: insertion sort restores the reference's
// insertion order (capsule-major, node-minor = ascending marker index).
__global__ void k_contact_sort(int ncells, const int* __restrict__ cell_start,
                               const int* __restrict__ cell_cnt, int* __restrict__ list) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int* a = list + cell_start[c];
    const int n = cell_cnt[c];
    for (int i = 1; i < n; ++i) {
        const int v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
        a[j + 1] = v;
    }
}

__global__ void k_contact_force(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                                const int* __restrict__ cell_of, const int* __restrict__ cell_start,
                                const int* __restrict__ cell_cnt, const int* __restrict__ list) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    const int cap = mb.mk_cap[m];
    const double2 pa = mb.pos[m], va = mb.vel[m];
    double2 F = mb.frc[m];
    int count = 0;
    if (ch.brute_contact) {
        for (int b = ch.mk_begin; b < ch.mk_end; ++b) {
            if (mb.mk_cap[b] == cap) continue;
            const double2 f = pair_force(ch, pa, va, mb.pos[b], mb.vel[b]);
            F.x = F.x + f.x;
            F.y = F.y + f.y;
            ++count;
        }
    } else {
        const int ci = cell_of[m] - ch.cell_base;
        const int cx = ci % ch.ncx, cy = ci / ch.ncx;
        for (int dy = -1; dy <= 1; ++dy) {
            const int yy = cy + dy;
            if (yy < 0 || yy >= ch.ncy) continue;
            for (int dx = -1; dx <= 1; ++dx) {
                int xx = cx + dx;
                if (xx < 0) xx += ch.ncx;
                if (xx >= ch.ncx) xx -= ch.ncx;
                const int cell = ch.cell_base + yy * ch.ncx + xx;
                const int s = cell_start[cell], e = s + cell_cnt[cell];
                for (int k = s; k < e; ++k) {
                    const int b = list[k];
                    if (mb.mk_cap[b] == cap) continue;
                    const double2 f = pair_force(ch, pa, va, mb.pos[b], mb.vel[b]);
                    F.x = F.x + f.x;
                    F.y = F.y + f.y;
                    ++count;
                }
            }
        }
    }
    const double2 z = make_double2(0.0, 0.0);
    double2 f = pair_force(ch, pa, va, make_double2(pa.x, ch.y_bot), z);
    F.x = F.x + f.x;
    F.y = F.y + f.y;
    f = pair_force(ch, pa, va, make_double2(pa.x, ch.y_top), z);
    F.x = F.x + f.x;
    F.y = F.y + f.y;
    mb.frc[m] = F;
    mb.pair_count[m] = count;
}

// ====================== immersed-boundary force tiles ======================

// Tiles covered by the stencil of a marker (at most 4 columns x 2 rows).
__device__ __forceinline__ int stencil_tiles(const ChannelDev& ch, int ix0, int iy0, int out[8]) {
    int tys[2], nty = 0;
    for (int iy = iy0 - 1; iy <= iy0 + 2; ++iy) {
        if (iy < 0 || iy >= ch.ny) continue;
        const int ty = iy / TILE_H;
        if (nty == 0 || tys[nty - 1] != ty) tys[nty++] = ty;
    }
    int txs[4], ntx = 0;
    for (int ix = ix0 - 1; ix <= ix0 + 2; ++ix) {
        int jx = ix;
        if (jx < 0) jx += ch.nx;
        if (jx >= ch.nx) jx -= ch.nx;
        if (jx < 0 || jx >= ch.nx) continue;
        const int tx = jx / TILE_W;
        bool dup = false;
        for (int a = 0; a < ntx; ++a) dup |= (txs[a] == tx);
        if (!dup) txs[ntx++] = tx;
    }
    int n = 0;
    for (int a = 0; a < nty; ++a)
        for (int b = 0; b < ntx; ++b) out[n++] = ch.tile_base + tys[a] * ch.tiles_x + txs[b];
    return n;
}

// Per-marker preparation: arc length ds (min-image, immersed_boundary.cpp:
// 164-173), stencil origin, validity, and the tile occupancy counts.
__global__ void k_ibm_prep(const ChannelDev* __restrict__ chans,
                           const CapsuleDev* __restrict__ caps, int M, MarkerBufs mb,
                           const double* __restrict__ phi_tbl, int* __restrict__ tile_flag,
                           int* __restrict__ tile_cnt, unsigned* status) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    const CapsuleDev& cp = caps[mb.mk_cap[m]];
    const int k = m - cp.off, n = cp.n;
    const int kp = cp.off + (k - 1 + n) % n, kn = cp.off + (k + 1) % n;
    const double Lx = (double)ch.nx;
    const double2 p = mb.pos[m];
    const double dp = norm_d(min_image_d(p, mb.pos[kp], Lx));
    const double dn = norm_d(min_image_d(mb.pos[kn], p, Lx));
    mb.ds[m] = 0.5 * (dp + dn);
    int ok = finite2(p);
    int ix0 = 0, iy0 = 0;
    if (ok) {
        // markers more than one period outside the lattice are skipped (the
        // reference indexes out of range there); wrapped x stays in [0, nx)
        if (p.x < -(double)ch.nx + 2.0 || p.x >= 2.0 * (double)ch.nx - 3.0) ok = 0;
        if (fabs(p.y) > 1e9) ok = 0;
    }
    if (ok) {
        ix0 = (int)floor(p.x);
        iy0 = (int)floor(p.y);
        if (iy0 < -2 || iy0 >= ch.ny + 2) ok = 0;
    } else if (!finite2(p)) {
        atomicOr(status, (unsigned)ST_NAN_MARKER);
    }
    mb.ix0[m] = ix0;
    mb.iy0[m] = iy0;
    mb.valid[m] = ok;
    if (!ok) return;
    // Peskin weights of the stencil, evaluated once per step (delta_function.h:44-59)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        mb.wx[4 * m + k] = phi_lut(phi_tbl, p.x - (double)(ix0 - 1 + k));
        mb.wy[4 * m + k] = phi_lut(phi_tbl, p.y - (double)(iy0 - 1 + k));
    }
    int t[8];
    const int nt = stencil_tiles(ch, ix0, iy0, t);
    // consecutive markers share tiles: one atomic per distinct tile and warp
    for (int a = 0; a < 8; ++a) {
        const int key = a < nt ? t[a] : -1;
        const unsigned peers = __match_any_sync(__activemask(), key);
        if (key >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) {
            tile_flag[key] = 1;
            atomicAdd(&tile_cnt[key], __popc(peers));
        }
    }
}

// Slot map of the step, and per slot the record the spread reads first
// (SlotInfo: tile, channel, tile origin, list length and offset, nx, ny), so
// that a spread warp starts a slot with one 32-byte load.
__global__ void k_tile_slots(int T, const int* __restrict__ tile_flag,
                             const int* __restrict__ slot_scan, int* __restrict__ tile_slot,
                             int* __restrict__ slot_tile, const ChannelDev* __restrict__ chans,
                             const int* __restrict__ tile_chan, const int* __restrict__ tile_cnt,
                             const int* __restrict__ list_off, SlotInfo* __restrict__ info,
                             int* __restrict__ cls_cnt, int* __restrict__ slot_rank) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    if (tile_flag[t]) {
        const int s = slot_scan[t];
        tile_slot[t] = s;
        slot_tile[s] = t;
        const int chan = tile_chan[t];
        const ChannelDev& ch = chans[chan];
        const int local = t - ch.tile_base;
        SlotInfo si;
        si.tile = t;
        si.chan = chan;
        si.x0 = (local % ch.tiles_x) * TILE_W;
        si.y0 = (local / ch.tiles_x) * TILE_H;
        si.cnt = tile_cnt[t];
        si.off = list_off[t];
        si.nx = ch.nx;
        si.ny = ch.ny;
        info[s] = si;
        // rank within the list-length class: one atomic per class and warp
        const int cls = slot_class(si.cnt);
        const unsigned peers = __match_any_sync(__activemask(), cls);
        const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(&cls_cnt[cls], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        slot_rank[s] = base + __popc(peers & ((1u << lane) - 1u));
    } else {
        tile_slot[t] = -1;
    }
}

// The spread's work order: slots by descending class, any order within a
// class (every slot's result is independent of the warp and of the order).
__global__ void k_slot_order(const int* __restrict__ n_slots_p, const SlotInfo* __restrict__ info,
                             const int* __restrict__ cls_cnt, const int* __restrict__ slot_rank,
                             int* __restrict__ order) {
    __shared__ int start[SLOT_CLASSES];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = SLOT_CLASSES - 1; c >= 0; --c) {
            start[c] = acc;
            acc += cls_cnt[c];
        }
    }
    __syncthreads();
    const int n = *n_slots_p;
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        order[start[slot_class(info[s].cnt)] + slot_rank[s]] = s;
}

__global__ void k_tile_fill(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                            const int* __restrict__ list_off, int* __restrict__ cursor,
                            int* __restrict__ list, const int* __restrict__ tile_slot) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M || !mb.valid[m]) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    const int ix0 = mb.ix0[m], iy0 = mb.iy0[m];
    int t[8];
    const int nt = stencil_tiles(ch, ix0, iy0, t);
    // one atomic per distinct tile and warp; the lanes of a tile take
    // consecutive list entries (the order is restored by the sweep-0 sort)
    const int lane = threadIdx.x & 31;
    for (int a = 0; a < 8; ++a) {
        const int key = a < nt ? t[a] : -1;
        const unsigned peers = __match_any_sync(__activemask(), key);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (key >= 0 && lane == leader) base = atomicAdd(&cursor[key], __popc(peers));
        base = __shfl_sync(peers, base, leader);
        if (key >= 0) list[list_off[key] + base + __popc(peers & ((1u << lane) - 1u))] = m;
    }
    // the slot of every stencil cell, by row tile and stencil column, for the
    // interpolations of the step (one 32-byte record instead of 16 lookups)
    int s8[8];
    const int ty0 = max(iy0 - 1, 0) / TILE_H, ty1 = min(iy0 + 2, ch.ny - 1) / TILE_H;
#pragma unroll
    for (int sx = 0; sx < 4; ++sx) {
        int jx = ix0 - 1 + sx;
        if (jx < 0) jx += ch.nx;
        if (jx >= ch.nx) jx -= ch.nx;
        const bool in = jx >= 0 && jx < ch.nx;
        const int tx = in ? jx / TILE_W : 0;
        s8[sx] = in ? tile_slot[ch.tile_base + ty0 * ch.tiles_x + tx] : -1;
        s8[4 + sx] = in ? tile_slot[ch.tile_base + ty1 * ch.tiles_x + tx] : -1;
    }
    int4* o = reinterpret_cast<int4*>(mb.slot8 + 8 * (size_t)m);
    o[0] = make_int4(s8[0], s8[1], s8[2], s8[3]);
    o[1] = make_int4(s8[4], s8[5], s8[6], s8[7]);
}

// Stencil column of lattice column jx for a marker with origin ix0 (the
// unwrapped index the reference uses in rx = x - ix); false if uncovered.
__device__ __forceinline__ bool stencil_ix(int jx, int ix0, int nx, int& ix) {
    int d = jx - ix0;
    if (d >= -1 && d <= 2) { ix = jx; return true; }
    d = jx - nx - ix0;
    if (d >= -1 && d <= 2) { ix = jx - nx; return true; }
    d = jx + nx - ix0;
    if (d >= -1 && d <= 2) { ix = jx + nx; return true; }
    return false;
}

constexpr int SPREAD_WARPS = 8;       // force tiles processed per CTA (one per warp)
constexpr int SPREAD_LCAP = 256;      // list entries sorted in shared memory per warp
                                      // (a power of two: the bitonic sort pads to one)
constexpr int SPREAD_LIST_MAX = 4096; // longer lists are clamped and flagged

// Shared memory of one spread warp: the tile's accumulators, the sort buffer
// of its marker list (sweep 0) and a staged chunk of markers.
constexpr int SPREAD_CHUNK = 16;      // markers staged per chunk
// Channels narrower than a tile: the stencil data of each marker.
struct SpreadChunkNarrow {
    double2 f[SPREAD_CHUNK];
    double ds[SPREAD_CHUNK];
    double wx[SPREAD_CHUNK][4], wy[SPREAD_CHUNK][4];
    int ix[SPREAD_CHUNK], iy[SPREAD_CHUNK], ok[SPREAD_CHUNK];
};
// Otherwise: each marker's 16 stencil contributions (f w ds, in the
// reference's rounding order), the lanes that own a valid point of it, and
// its stencil origin in tile coordinates.
// (x, y) pair of the accumulation type: double2 in FP64 contexts (the
// reference's arithmetic, bit for bit), float2 in the FP32-arithmetic modes.
template <typename A> struct APair;
template <> struct APair<double> {
    using T = double2;
    static __device__ __forceinline__ T make(double x, double y) { return make_double2(x, y); }
};
template <> struct APair<float> {
    using T = float2;
    static __device__ __forceinline__ T make(double x, double y) {
        return make_float2((float)x, (float)y);
    }
};
// Markers staged per chunk on the wide path: four lanes per marker, one
// stencil row each.  A staged point goes to the slot of the lane that owns
// its cell (lane (a, b) owns the tile cells whose column is a mod 8 and row
// b mod 4): its contribution and its accumulator index.
constexpr int WIDE_CHUNK = 8;
template <typename A>
struct SpreadChunkWide {
    typename APair<A>::T v[WIDE_CHUNK][33];    // [marker][owner lane] (padded row)
    unsigned short cell[WIDE_CHUNK][32];       // accumulator index of that point
    unsigned mask[WIDE_CHUNK];                 // owner lanes holding a point
};
// The tile accumulators keep rows of TILE_W + 4 doubles: the 4 x 4 stencil
// points of a marker (4 consecutive rows and columns) then fall on 16
// distinct bank pairs (a row stride of 32 doubles puts all 4 rows on the same
// banks: 4-way conflicts on every accumulation).
constexpr int ACC_W = TILE_W + 4;
constexpr int ACC_CELLS = TILE_H * ACC_W;
__device__ __forceinline__ int acc_at(int c) { return (c / TILE_W) * ACC_W + (c % TILE_W); }
template <typename A>
struct SpreadWarpSmem {
    A ax[ACC_CELLS], ay[ACC_CELLS];
    union {
        int list[SPREAD_LCAP];                 // sweep 0: the bitonic sort of long lists
        SpreadChunkNarrow n;                   // (the sort ends before the first chunk)
        SpreadChunkWide<A> w;
    } ck;
};
template <typename A>
constexpr size_t spread_smem() { return sizeof(SpreadWarpSmem<A>) * SPREAD_WARPS; }

// Deterministic spread into force tiles for MDF sweep `sweep`.  Sweep 0
// spreads the membrane + contact forces (immersed_boundary.cpp:25-100);
// sweep k >= 1 adds the corrections dF (:231-286).  One warp owns one tile:
// it sorts the tile's marker list (ascending marker index = the reference's
// loop order), then applies the markers one after the other, 16 lanes
// covering the 4 x 4 stencil, so every cell receives its contributions in
// the reference's order.  On a channel's last sweep the warp also adds the
// body force on FLUID cells, applies the force cap and counts capped cells
// (simulation.cpp:540-609), writing the final tile force `fin` (type R).
// The tile accumulates in R; the step launches it for FP64 contexts (double,
// bit for bit), the FP32-arithmetic modes run k_spread_fx.
// Resident CTAs per SM asked of the compiler: 3 for the double form (4 for a
// float instantiation).
template <typename R>
constexpr int spread_min_ctas() { return sizeof(R) == 4 ? 4 : 3; }

template <typename R>
__global__ void __launch_bounds__(SPREAD_WARPS * 32, spread_min_ctas<R>())
k_spread(const ChannelDev* __restrict__ chans, const SlotInfo* __restrict__ slot_info,
         const int* __restrict__ slot_order, const int* __restrict__ n_slots_p,
         int* __restrict__ slot_ctr,
         int* __restrict__ list, MarkerBufs mb, double* __restrict__ acc,
         double* __restrict__ acc0, R* __restrict__ gsnap, R* __restrict__ fin, int sweep,
         int mode, const unsigned* __restrict__ resid_gate,
         const int* __restrict__ plain_needed, int* __restrict__ capped,
         int* __restrict__ fluid_touched, unsigned* status) {
    if (sweep > 0 && mode == MDF_PLAIN && plain_needed && !*plain_needed) return;
    extern __shared__ __align__(16) unsigned char spread_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    using A = R;
    using A2 = typename APair<A>::T;
    SpreadWarpSmem<A>& W = reinterpret_cast<SpreadWarpSmem<A>*>(spread_smem)[warp];
    A* ax = W.ax;
    A* ay = W.ay;
    int* sl = W.ck.list;
    const int n_slots = *n_slots_p;
    // slots are dealt to the warps in rounds over the work order (longest
    // lists first, alternating direction, so each warp's share sums to
    // about the same work; a shared claim counter serialises on one L2
    // address); the next slot's record is fetched while the current one is
    // processed
    const int nwarps = gridDim.x * SPREAD_WARPS;
    // round k takes work-order positions k nwarps .. (k + 1) nwarps - 1,
    // the warps in reverse order on odd rounds
    const int wid = blockIdx.x * SPREAD_WARPS + warp;
    int round = 0, next = wid;
    int nslot = next < n_slots ? slot_order[next] : 0;
    SlotInfo nfo{};
    if (next < n_slots) nfo = slot_info[nslot];
    while (next < n_slots) {
        const int slot = nslot;
        const SlotInfo si = nfo;
        ++round;
        next = round * nwarps + ((round & 1) ? nwarps - 1 - wid : wid);
        if (next < n_slots) {
            nslot = slot_order[next];
            nfo = slot_info[nslot];
        }
        const int chan = si.chan;
        const ChannelDev& ch = chans[chan];
        const int K = ch.ibm_iterations > 1 ? ch.ibm_iterations : 1;
        if (sweep >= K) continue;  // warp-uniform
        if (sweep > 0 && !mdf_active(ch, mode, resid_gate, chan)) continue;  // sweep 0: all
        const int nx = si.nx, ny = si.ny;
        const int x0 = si.x0, y0 = si.y0;
        int cnt = si.cnt;
        const int off = si.off;
        const int* lst;
        // the lists are sorted by the step's first spread (sweep 0) and
        // written back; later sweeps read them in order
        const bool do_sort = (sweep == 0);
        if (cnt <= SPREAD_LCAP && !do_sort) {
            lst = list + off;
        } else if (cnt <= 32) {
            // bitonic sort across the warp's registers (ascending by lane)
            int v = lane < cnt ? list[off + lane] : INT_MAX;
#pragma unroll
            for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
                for (int j = k >> 1; j > 0; j >>= 1) {
                    const int o = __shfl_xor_sync(0xffffffffu, v, j);
                    const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
                    v = take_min ? min(v, o) : max(v, o);
                }
            if (lane < cnt) list[off + lane] = v;
            __syncwarp();
            lst = list + off;
        } else if (cnt <= SPREAD_LCAP) {
            int pow2 = 1;
            while (pow2 < cnt) pow2 <<= 1;
            for (int i = lane; i < pow2; i += 32) sl[i] = i < cnt ? list[off + i] : INT_MAX;
            __syncwarp();
            for (int k = 2; k <= pow2; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = lane; i < pow2; i += 32) {
                        const int l = i ^ j;
                        if (l > i) {
                            const int a = sl[i], b = sl[l];
                            if ((a > b) == ((i & k) == 0)) { sl[i] = b; sl[l] = a; }
                        }
                    }
                    __syncwarp();
                }
            for (int i = lane; i < cnt; i += 32) list[off + i] = sl[i];
            __syncwarp();
            lst = list + off;
        } else {
            if (cnt > SPREAD_LIST_MAX) {
                if (lane == 0) atomicOr(status, (unsigned)ST_LIST_OVERFLOW);
                cnt = SPREAD_LIST_MAX;
            }
            if (lane == 0 && do_sort) {  // long lists are rare: sort in place
                int* a = list + off;
                for (int i = 1; i < cnt; ++i) {
                    const int v = a[i];
                    int j = i - 1;
                    while (j >= 0 && a[j] > v) { a[j + 1] = a[j]; --j; }
                    a[j + 1] = v;
                }
            }
            __syncwarp();
            lst = list + off;
        }
        const size_t base = (size_t)slot * 2 * TILE_CELLS;
        const bool last = mode == MDF_LEARNED ? true : (mode == MDF_SEED ? false : sweep == K - 1);
        // a learned channel's membrane-only force lives in acc0 only: the
        // seed sweep and a fallback's restart read it there.  The
        // accumulators hold (x, y) pairs per cell: [slot][TILE_CELLS] double2.
        const A2* src = reinterpret_cast<const A2*>(
            (ch.learned && (mode == MDF_SEED || (mode == MDF_PLAIN && sweep == 1))) ? acc0 : acc);
        const size_t base2 = (size_t)slot * TILE_CELLS;
        for (int c = lane; c < TILE_CELLS; c += 32) {
            const A2 a = sweep > 0 ? src[base2 + c] : APair<A>::make(0.0, 0.0);
            const A vx = a.x, vy = a.y;
            ax[acc_at(c)] = vx;
            ay[acc_at(c)] = vy;
            if (last && K > 1) {
                gsnap[base + c] = (R)vx;
                gsnap[base + TILE_CELLS + c] = (R)vy;
            }
        }
        __syncwarp();
        const int la = lane & 7, lb = lane >> 3;
        if (nx > TILE_W) {
            // Markers in list order, WIDE_CHUNK at a time.  Staging: lanes
            // 4j .. 4j + 3 take marker j of the chunk, one stencil row each
            // (sy = lane & 3), and evaluate its four points: the weight
            // w = phi(rx) phi(ry), the contribution (f w) ds and the lane that
            // owns the point's cell, into whose slot the contribution and the
            // cell's accumulator index go.  Lane (a, b) = (lane & 7, lane >> 3)
            // owns the tile cells of column a mod 8 and row b mod 4; the 4 x 4
            // stencil has 4 consecutive columns and rows, so its 16 points
            // fall on 16 distinct lanes.  Then every lane adds its own point of
            // each marker to its own cell, marker after marker, so every cell
            // receives its terms in the reference's order.  A lane with no
            // point of a marker adds zero to a padding cell of its own (the
            // accumulator rows carry four padding columns: 8 x 4 = 32 cells,
            // one per lane), so the additions carry no branches.
            const int jm = lane >> 2, sy = lane & 3;
            double2 rf = make_double2(0.0, 0.0), rw0 = rf, rw1 = rf;
            double rds = 0.0, rwy = 0.0;
            int rix = 0, riy = 0;
            auto fetch = [&](int c) {
                if (c + jm < cnt) {
                    const int m = lst[c + jm];
                    rf = sweep == 0 ? mb.frc[m] : mb.dF[m];
                    rix = mb.ix0[m];
                    riy = mb.iy0[m];
                    rds = mb.ds[m];
                    const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
                    rw0 = wx2[0];
                    rw1 = wx2[1];
                    rwy = mb.wy[4 * (size_t)m + sy];
                }
            };
            const int pad = (lane >> 2) * ACC_W + TILE_W + (lane & 3);   // this lane's padding cell
            fetch(0);
            for (int c0 = 0; c0 < cnt; c0 += WIDE_CHUNK) {
                const int nb = cnt - c0 < WIDE_CHUNK ? cnt - c0 : WIDE_CHUNK;
                __syncwarp();
                unsigned bits = 0u;
                if (jm < nb) {
                    const bool ok = !(isnan(rf.x) || isnan(rf.y));
                    const int cyl = riy - 1 + sy - y0, iy = riy - 1 + sy;
                    const bool vrow = ok && cyl >= 0 && cyl < TILE_H && iy >= 0 && iy < ny;
                    const double wxk[4] = {rw0.x, rw0.y, rw1.x, rw1.y};
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        int jx = rix - 1 + k;
                        if (jx < 0) jx += nx;
                        if (jx >= nx) jx -= nx;
                        const int cl = jx - x0;
                        const double w = wxk[k] * rwy;
                        if (vrow && jx >= 0 && jx < nx && cl >= 0 && cl < TILE_W && w > 1e-15) {
                            const int t = (cl & 7) + 8 * (cyl & 3);
                            // FP64: (f w) ds in the reference's order; the
                            // float form rounds f, w, ds once and works in float
                            if constexpr (sizeof(A) == 8)
                                W.ck.w.v[jm][t] = APair<A>::make(rf.x * w * rds, rf.y * w * rds);
                            else
                                W.ck.w.v[jm][t] = make_float2((float)rf.x * (float)w * (float)rds,
                                                              (float)rf.y * (float)w * (float)rds);
                            W.ck.w.cell[jm][t] = (unsigned short)(cyl * ACC_W + cl);
                            bits |= 1u << t;
                        }
                    }
                }
                bits |= __shfl_xor_sync(0xffffffffu, bits, 1);
                bits |= __shfl_xor_sync(0xffffffffu, bits, 2);
                if (sy == 0 && jm < nb) W.ck.w.mask[jm] = bits;
                __syncwarp();
                fetch(c0 + WIDE_CHUNK);   // in flight while this chunk is added
                const A2 zero = APair<A>::make(0.0, 0.0);
                // this lane's point of marker j (or zero into its padding cell)
                auto point = [&](int j, int& c, A2& v) {
                    const bool h = (W.ck.w.mask[j] >> lane) & 1u;
                    const int ci = W.ck.w.cell[j][lane];
                    const A2 vi = W.ck.w.v[j][lane];
                    c = h ? ci : pad;
                    v = h ? vi : zero;
                };
                int j = 0;
                // two markers at a time: both cells are read before either is
                // written, the second addition taking the first's sum when
                // both points are the same cell (same order, same rounding)
                for (; j + 1 < nb; j += 2) {
                    int c0i, c1i;
                    A2 v0, v1;
                    point(j, c0i, v0);
                    point(j + 1, c1i, v1);
                    A a0x = ax[c0i], a0y = ay[c0i];
                    A a1x = ax[c1i], a1y = ay[c1i];
                    a0x += v0.x;
                    a0y += v0.y;
                    ax[c0i] = a0x;
                    ay[c0i] = a0y;
                    const bool same = c1i == c0i;
                    a1x = same ? a0x : a1x;
                    a1y = same ? a0y : a1y;
                    ax[c1i] = a1x + v1.x;
                    ay[c1i] = a1y + v1.y;
                }
                if (j < nb) {
                    int c;
                    A2 v;
                    point(j, c, v);
                    ax[c] += v.x;
                    ay[c] += v.y;
                }
            }
        } else {
        // One tile holds both sides of the periodic seam: two stencil
        // columns can share a residue, so a lane applies each of its points.
        SpreadChunkNarrow& N = W.ck.n;
        double2 rf = make_double2(0.0, 0.0), rw0 = rf, rw1 = rf, rv0 = rf, rv1 = rf;
        double rds = 0.0;
        int rix = 0, riy = 0;
        auto fetch = [&](int c) {
            if (lane < SPREAD_CHUNK && c + lane < cnt) {
                const int m = lst[c + lane];
                rf = sweep == 0 ? mb.frc[m] : mb.dF[m];
                rix = mb.ix0[m];
                riy = mb.iy0[m];
                rds = mb.ds[m];
                const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
                const double2* wy2 = reinterpret_cast<const double2*>(mb.wy + 4 * (size_t)m);
                rw0 = wx2[0]; rw1 = wx2[1]; rv0 = wy2[0]; rv1 = wy2[1];
            }
        };
        fetch(0);
        for (int c0 = 0; c0 < cnt; c0 += SPREAD_CHUNK) {
            const int nb = cnt - c0 < SPREAD_CHUNK ? cnt - c0 : SPREAD_CHUNK;
            __syncwarp();
            if (lane < nb) {
                N.f[lane] = rf;
                N.ok[lane] = !(isnan(rf.x) || isnan(rf.y));
                N.ds[lane] = rds;
                N.ix[lane] = rix;
                N.iy[lane] = riy;
                N.wx[lane][0] = rw0.x; N.wx[lane][1] = rw0.y; N.wx[lane][2] = rw1.x; N.wx[lane][3] = rw1.y;
                N.wy[lane][0] = rv0.x; N.wy[lane][1] = rv0.y; N.wy[lane][2] = rv1.x; N.wy[lane][3] = rv1.y;
            }
            __syncwarp();
            fetch(c0 + SPREAD_CHUNK);   // in flight while this chunk is added
            for (int j = 0; j < nb; ++j) {
                if (!N.ok[j]) continue;  // warp-uniform
                const int jx0 = N.ix[j] - 1;
                const int r0n = N.iy[j] - 1 - y0;
                const int syn = (lb - r0n) & 3;
                const int cyn = r0n + syn;
                if (cyn >= 0 && cyn < TILE_H && cyn + y0 >= 0 && cyn + y0 < ny) {
                    for (int k = 0; k < 4; ++k) {
                        int jx = jx0 + k;
                        if (jx < 0) jx += nx;
                        if (jx >= nx) jx -= nx;
                        const int cl = jx - x0;
                        if (cl < 0 || cl >= TILE_W || (cl & 7) != la) continue;
                        const double w = N.wx[j][k] * N.wy[j][syn];
                        if (w > 1e-15) {
                            const double ds = N.ds[j];
                            const double2 fo = N.f[j];
                            const int c = cyn * ACC_W + cl;
                            ax[c] += (A)(fo.x * w * ds);
                            ay[c] += (A)(fo.y * w * ds);
                        }
                    }
                }
            }
        }
        }
        __syncwarp();
        if (!last) {
            A2* out = reinterpret_cast<A2*>((sweep == 0 && ch.learned) ? acc0 : acc);
            for (int c = lane; c < TILE_CELLS; c += 32) {
                A2 o;
                o.x = ax[acc_at(c)];
                o.y = ay[acc_at(c)];
                out[base2 + c] = o;
            }
            __syncwarp();
            continue;
        }
        // finalize: body force on FLUID cells, then the force cap
        int n_cap = 0, n_fluid = 0;
        const double Fm = ch.max_force, Fm2 = Fm * Fm;
        const bool body = (ch.body_fx != 0.0 || ch.body_fy != 0.0);
        for (int c = lane; c < TILE_CELLS; c += 32) {
            const int jx = x0 + (c % TILE_W), jy = y0 + (c / TILE_W);
            double vx = (double)ax[acc_at(c)], vy = (double)ay[acc_at(c)];
            if (jx < nx && jy < ny) {
                const bool fluid = cell_kind(ch, jx, jy) == CK_FLUID;
                if (fluid && body) {
                    vx += ch.body_fx;
                    vy += ch.body_fy;
                }
                const double f2 = vx * vx + vy * vy;
                if (f2 > Fm2) {
                    const double sc = Fm / sqrt(f2);
                    vx *= sc;
                    vy *= sc;
                    ++n_cap;
                }
                n_fluid += fluid ? 1 : 0;
            }
            // (no sweep reads acc after a channel's last one)
            fin[base + c] = (R)vx;
            fin[base + TILE_CELLS + c] = (R)vy;
        }
        for (int o = 16; o > 0; o >>= 1) {
            n_cap += __shfl_down_sync(0xffffffffu, n_cap, o);
            n_fluid += __shfl_down_sync(0xffffffffu, n_fluid, o);
        }
        if (lane == 0) {
            if (n_cap) atomicAdd(&capped[chan], n_cap);
            if (n_fluid) atomicAdd(&fluid_touched[chan], n_fluid);
        }
        __syncwarp();
    }
}

// The spread of the FP32-arithmetic modes (FP32 and FP16-shifted storage):
// the reference's contributions (f w) ds of each stencil point with
// w > 1e-15, formed as (float)f (float)w (float)ds and summed per cell
// exactly in fixed point.  Integer addition does not depend on the order of the
// terms, so the lanes of a warp add any markers' points in any order, with
// 32-bit shared-memory atomics, and the result is the same on every run, in
// every launch shape and whether a channel runs alone or in an ensemble; the
// marker lists need no sort.  Each value is v = q 2^-38 with the integer q
// split into a low part of 20 bits (unsigned, in [0, 2^20)) and a high part
// (signed).  A cell takes at most one term per list entry (channels at
// least 4 cells wide), so at most SPREAD_LIST_MAX = 4,096 low parts a sweep,
// whose sum stays below 2^32; the high parts are summed modulo 2^32, exact
// while the cell's sum stays below 2^13 in magnitude, far beyond any
// lattice force.
//
// A cell that no stencil point of the tile's markers reaches (with weight
// above 1e-15) receives nothing in any sweep of the step (the lists do not
// change between sweeps) and so holds zero throughout; about five in six
// cells of a tile are such.  The accumulators are therefore read and written
// only at the touched cells: a sweep adds its sum, rounded to float once, to
// the previous sweep's value there, and the readers of the accumulators (the
// interpolations, at the same stencil points) read nothing else.  The last
// sweep writes every cell of the tile's final force and of the force before
// that sweep, zero plus the body force where untouched.  The shared
// accumulators start at zero once per kernel and are cleared again at the
// touched cells after each tile.  FP64 contexts keep k_spread (the
// reference's serial order, bit for bit).
constexpr int FX_LO_BITS = 20;
constexpr float FX_SCALE = 274877906944.0f;          // 2^38
constexpr float FX_UNSCALE = 1.0f / 274877906944.0f;  // 2^-38 (exact)
struct SpreadFxWarp {
    unsigned lo[2][ACC_CELLS];        // x, y; rows of ACC_W cells
    int hi[2][ACC_CELLS];
    unsigned char hit[ACC_CELLS];     // touched this tile
    unsigned short idx[TILE_CELLS];   // the touched cells, compacted
};
constexpr size_t spread_fx_smem() { return sizeof(SpreadFxWarp) * SPREAD_WARPS; }
__device__ __forceinline__ long long fx_quant(float v) { return __float2ll_rn(v * FX_SCALE); }
__device__ __forceinline__ unsigned fx_lo(long long q) {
    return (unsigned)(q & ((1LL << FX_LO_BITS) - 1));
}
__device__ __forceinline__ int fx_hi(long long q) { return (int)(q >> FX_LO_BITS); }
__device__ __forceinline__ float fx_value(unsigned lo, int hi) {
    return __ll2float_rn((long long)hi * (1LL << FX_LO_BITS) + (long long)lo) * FX_UNSCALE;
}

__global__ void __launch_bounds__(SPREAD_WARPS * 32, 4)
k_spread_fx(const ChannelDev* __restrict__ chans, const SlotInfo* __restrict__ slot_info,
            const int* __restrict__ slot_order, const int* __restrict__ n_slots_p,
            const int* __restrict__ list, MarkerBufs mb,
            double* __restrict__ acc, double* __restrict__ acc0, float* __restrict__ gsnap,
            float* __restrict__ fin, int sweep, int mode, const unsigned* __restrict__ resid_gate,
            const int* __restrict__ plain_needed, int* __restrict__ capped,
            int* __restrict__ fluid_touched, unsigned* status) {
    if (sweep > 0 && mode == MDF_PLAIN && plain_needed && !*plain_needed) return;
    extern __shared__ __align__(16) unsigned char spread_fx_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    SpreadFxWarp& W = reinterpret_cast<SpreadFxWarp*>(spread_fx_raw)[warp];
    for (int i = lane; i < ACC_CELLS; i += 32) {
        W.lo[0][i] = W.lo[1][i] = 0u;
        W.hi[0][i] = W.hi[1][i] = 0;
        W.hit[i] = 0;
    }
    __syncwarp();
    const int n_slots = *n_slots_p;
    const int nwarps = gridDim.x * SPREAD_WARPS;
    // round k takes work-order positions k nwarps .. (k + 1) nwarps - 1,
    // the warps in reverse order on odd rounds
    const int wid = blockIdx.x * SPREAD_WARPS + warp;
    int round = 0, next = wid;
    int nslot = next < n_slots ? slot_order[next] : 0;
    SlotInfo nfo{};
    if (next < n_slots) nfo = slot_info[nslot];
    while (next < n_slots) {
        const int slot = nslot;
        const SlotInfo si = nfo;
        ++round;
        next = round * nwarps + ((round & 1) ? nwarps - 1 - wid : wid);
        if (next < n_slots) {
            nslot = slot_order[next];
            nfo = slot_info[nslot];
        }
        const int chan = si.chan;
        const ChannelDev& ch = chans[chan];
        const int K = ch.ibm_iterations > 1 ? ch.ibm_iterations : 1;
        if (sweep >= K) continue;  // warp-uniform
        if (sweep > 0 && !mdf_active(ch, mode, resid_gate, chan)) continue;  // sweep 0: all
        const int nx = si.nx, ny = si.ny;
        const int x0 = si.x0, y0 = si.y0;
        int cnt = si.cnt;
        if (cnt > SPREAD_LIST_MAX) {
            if (lane == 0) atomicOr(status, (unsigned)ST_LIST_OVERFLOW);
            cnt = SPREAD_LIST_MAX;
        }
        const int* lst = list + si.off;
        const size_t base = (size_t)slot * 2 * TILE_CELLS;
        const bool last = mode == MDF_LEARNED ? true : (mode == MDF_SEED ? false : sweep == K - 1);
        // a learned channel's membrane-only force lives in acc0 only (k_spread)
        const float2* src = reinterpret_cast<const float2*>(
            (ch.learned && (mode == MDF_SEED || (mode == MDF_PLAIN && sweep == 1))) ? acc0 : acc);
        const size_t base2 = (size_t)slot * TILE_CELLS;
        // four lanes per marker, one stencil row each, eight markers a pass;
        // the next pass's marker data is loaded before this pass's points
        const int jm = lane >> 2, sy = lane & 3;
        struct Mk {
            double2 f, w0, w1;
            double ds, wy;
            int ix, iy;
        };
        auto fetch = [&](int c, Mk& k) {
            if (c + jm < cnt) {
                const int m = lst[c + jm];
                k.f = sweep == 0 ? mb.frc[m] : mb.dF[m];
                k.ix = mb.ix0[m];
                k.iy = mb.iy0[m];
                k.ds = mb.ds[m];
                const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
                k.w0 = wx2[0];
                k.w1 = wx2[1];
                k.wy = mb.wy[4 * (size_t)m + sy];
            }
        };
        Mk cur{}, nxt{};
        fetch(0, cur);
        for (int c0 = 0; c0 < cnt; c0 += 8) {
            fetch(c0 + 8, nxt);
            if (c0 + jm < cnt) {
                const bool ok = !(isnan(cur.f.x) || isnan(cur.f.y));
                const int iy = cur.iy - 1 + sy, cyl = iy - y0;
                const bool vrow = cyl >= 0 && cyl < TILE_H && iy >= 0 && iy < ny;
                const double wxk[4] = {cur.w0.x, cur.w0.y, cur.w1.x, cur.w1.y};
                const float fx = (float)cur.f.x, fy = (float)cur.f.y, ds = (float)cur.ds;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    int jx = cur.ix - 1 + k;
                    if (jx < 0) jx += nx;
                    if (jx >= nx) jx -= nx;
                    const int cl = jx - x0;
                    const double w = wxk[k] * cur.wy;
                    // touched: a superset of the points that the
                    // interpolations read (they test the weight in float)
                    if (vrow && jx >= 0 && jx < nx && cl >= 0 && cl < TILE_W && w > 0.5e-15) {
                        const int i = cyl * ACC_W + cl;
                        W.hit[i] = 1;   // (lanes that meet here all store 1)
                        if (!ok || !(w > 1e-15)) continue;
                        const float wf = (float)w;
                        const long long qx = fx_quant(fx * wf * ds), qy = fx_quant(fy * wf * ds);
                        atomicAdd(&W.lo[0][i], fx_lo(qx));
                        atomicAdd(&W.hi[0][i], fx_hi(qx));
                        atomicAdd(&W.lo[1][i], fx_lo(qy));
                        atomicAdd(&W.hi[1][i], fx_hi(qy));
                    }
                }
            }
            cur = nxt;
        }
        __syncwarp();
        if (!last) {
            // the touched cells, compacted row by row
            int n = 0;
#pragma unroll
            for (int r = 0; r < TILE_H; ++r) {
                const bool h = W.hit[r * ACC_W + lane] != 0;
                const unsigned b = __ballot_sync(0xffffffffu, h);
                if (h) W.idx[n + __popc(b & ((1u << lane) - 1u))] = (unsigned short)(r * TILE_W + lane);
                n += __popc(b);
            }
            __syncwarp();
            float2* out = reinterpret_cast<float2*>((sweep == 0 && ch.learned) ? acc0 : acc);
            for (int k = lane; k < n; k += 32) {
                const int c = W.idx[k], i = acc_at(c);
                float2 v = make_float2(fx_value(W.lo[0][i], W.hi[0][i]),
                                       fx_value(W.lo[1][i], W.hi[1][i]));
                if (sweep > 0) {
                    const float2 a = src[base2 + c];
                    v.x = a.x + v.x;
                    v.y = a.y + v.y;
                }
                out[base2 + c] = v;
                W.lo[0][i] = W.lo[1][i] = 0u;
                W.hi[0][i] = W.hi[1][i] = 0;
                W.hit[i] = 0;
            }
            __syncwarp();
            continue;
        }
        // finalize every cell, two adjacent cells a lane: the value before
        // this sweep (zero where untouched) plus this sweep's sum, the body
        // force on FLUID cells, then the force cap with the capped-cell
        // count (as k_spread, in float).  Cell kinds follow from the row
        // alone unless the channel has a cell-type mask or x boundaries.
        int n_cap = 0, n_fluid = 0;
        const float Fm = (float)ch.max_force, Fm2 = Fm * Fm;
        const float bfx = (float)ch.body_fx, bfy = (float)ch.body_fy;
        const bool body = (ch.body_fx != 0.0 || ch.body_fy != 0.0);
        const bool row_kinds = ch.mask == nullptr && ch.bc_x != 0 && ch.bc_x != 2;
        const float2 zero = make_float2(0.f, 0.f);
#pragma unroll 2
        for (int it = 0; it < TILE_H / 2; ++it) {
            const int r = 2 * it + (lane >> 4), cx = 2 * (lane & 15);
            const int c = r * TILE_W + cx, i = r * ACC_W + cx;
            const int jx = x0 + cx, jy = y0 + r;
            const bool h0 = W.hit[i] != 0, h1 = W.hit[i + 1] != 0;
            float2 a0 = zero, a1 = zero, v0 = zero, v1 = zero;
            if (h0 || h1) {
                if (sweep > 0) {
                    const float4 a = *reinterpret_cast<const float4*>(src + base2 + c);
                    if (h0) a0 = make_float2(a.x, a.y);
                    if (h1) a1 = make_float2(a.z, a.w);
                }
                if (h0) {
                    v0 = make_float2(a0.x + fx_value(W.lo[0][i], W.hi[0][i]),
                                     a0.y + fx_value(W.lo[1][i], W.hi[1][i]));
                    W.lo[0][i] = W.lo[1][i] = 0u;
                    W.hi[0][i] = W.hi[1][i] = 0;
                    W.hit[i] = 0;
                }
                if (h1) {
                    v1 = make_float2(a1.x + fx_value(W.lo[0][i + 1], W.hi[0][i + 1]),
                                     a1.y + fx_value(W.lo[1][i + 1], W.hi[1][i + 1]));
                    W.lo[0][i + 1] = W.lo[1][i + 1] = 0u;
                    W.hi[0][i + 1] = W.hi[1][i + 1] = 0;
                    W.hit[i + 1] = 0;
                }
            }
            if (K > 1) {
                *reinterpret_cast<float2*>(gsnap + base + c) = make_float2(a0.x, a1.x);
                *reinterpret_cast<float2*>(gsnap + base + TILE_CELLS + c) = make_float2(a0.y, a1.y);
            }
            float2 v[2] = {v0, v1};
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                if (jx + e < nx && jy < ny) {
                    const bool fluid =
                        row_kinds ? (ch.periodic_y || (jy != 0 && jy != ny - 1))
                                  : cell_kind(ch, jx + e, jy) == CK_FLUID;
                    if (fluid && body) {
                        v[e].x += bfx;
                        v[e].y += bfy;
                    }
                    const float f2 = v[e].x * v[e].x + v[e].y * v[e].y;
                    if (f2 > Fm2) {
                        const float sc = Fm / sqrtf(f2);
                        v[e].x *= sc;
                        v[e].y *= sc;
                        ++n_cap;
                    }
                    n_fluid += fluid ? 1 : 0;
                }
            }
            *reinterpret_cast<float2*>(fin + base + c) = make_float2(v[0].x, v[1].x);
            *reinterpret_cast<float2*>(fin + base + TILE_CELLS + c) = make_float2(v[0].y, v[1].y);
        }
        for (int o = 16; o > 0; o >>= 1) {
            n_cap += __shfl_down_sync(0xffffffffu, n_cap, o);
            n_fluid += __shfl_down_sync(0xffffffffu, n_fluid, o);
        }
        if (lane == 0) {
            if (n_cap) atomicAdd(&capped[chan], n_cap);
            if (n_fluid) atomicAdd(&fluid_touched[chan], n_fluid);
        }
        __syncwarp();
    }
}

// MDF correction of one sweep (immersed_boundary.cpp:231-286): interpolate
// u = (j + F/2)/rho with the force spread so far, then
// dF = 2 rho(nearest node) (U_prev - U_interp).  Also keeps the step's total
// correction (dFsum), the first sweep's interpolation (u0) and the no-slip
// residual max |U_prev - U_interp| per channel: at the learned form's sweep
// (resid_gate) and at a plain iteration's last sweep (resid_plain).
template <typename S, typename R>
__global__ void k_mdf_interp(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                             const int* __restrict__ tile_slot,
                             const typename Mom4<R>::T* __restrict__ mom,
                             const double* __restrict__ acc, const double* __restrict__ acc0,
                             int sweep, int mode, unsigned* __restrict__ resid_gate,
                             unsigned* __restrict__ resid_plain,
                             const int* __restrict__ plain_needed) {
    if (mode == MDF_PLAIN && plain_needed && !*plain_needed) return;  // no channel needs it
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const int chan = mb.mk_chan[m];
    const ChannelDev& ch = chans[chan];
    if (sweep >= ch.ibm_iterations || !mb.valid[m]) return;
    if (!mdf_active(ch, mode, resid_gate, chan)) return;
    const double* base = (mode == MDF_PLAIN && ch.learned && sweep == 1) ? acc0 : acc;
    double rho_local;
    const double2 u = interp_u_mom<R, true>(ch, mb, m, tile_slot, mom, base, rho_local);
    const double2 v = mb.vel[m];
    const double dux = v.x - u.x, duy = v.y - u.y;
    const double2 d = make_double2(dux * (2.0 * rho_local), duy * (2.0 * rho_local));
    mb.dF[m] = d;
    if (mode == MDF_PLAIN && sweep == 1) {
        mb.u0[m] = u;
        mb.dFsum[m] = d;
    } else {
        const double2 s0 = mb.dFsum[m];
        mb.dFsum[m] = make_double2(s0.x + d.x, s0.y + d.y);
    }
    // the per-channel residual max, one atomic per channel and warp
    const bool want = mode == MDF_LEARNED || sweep == ch.ibm_iterations - 1;
    warp_max_resid(mode == MDF_LEARNED ? resid_gate : resid_plain, chan, want,
                   sqrt(dux * dux + duy * duy));
}

// Whether any channel needs the plain correction sweeps this step: a forcing
// channel that is not learned, or a learned one whose gate residual is above
// its threshold.  One CTA; runs after the learned sweep's interpolation.
__global__ void k_plain_needed(const ChannelDev* __restrict__ chans, int nch,
                               const unsigned* __restrict__ resid_gate, int* __restrict__ flag) {
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    int mine = 0;
    for (int c = threadIdx.x; c < nch; c += blockDim.x) {
        const ChannelDev& ch = chans[c];
        if (ch.cap_end > ch.cap_begin && ch.ibm_iterations > 1 &&
            (!ch.learned || mdf_fallback(resid_gate[c], ch.mdf_threshold)))
            mine = 1;
    }
    if (mine) any = 1;
    __syncthreads();
    if (threadIdx.x == 0) *flag = any;
}

void launch_plain_needed(const ChannelDev* chans, int nch, TileBufs& tb, cudaStream_t st) {
    k_plain_needed<<<1, 256, 0, st>>>(chans, nch, tb.resid_gate, tb.plain_needed);
}

// (rho, jx, jy) of every cell of the step's force tiles, one warp per tile
// (rows of 32 cells: coalesced population loads).
template <typename S, typename R>
__global__ void k_tile_moments(const ChannelDev* __restrict__ chans,
                               const SlotInfo* __restrict__ slot_info,
                               const int* __restrict__ n_slots_p, const S* __restrict__ f,
                               typename Mom4<R>::T* __restrict__ mom) {
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int n_slots = *n_slots_p;
    for (int slot = warp; slot < n_slots; slot += nwarps) {
        const SlotInfo si = slot_info[slot];
        const ChannelDev& ch = chans[si.chan];
        const int x0 = si.x0, y0 = si.y0;
        const int jx = x0 + lane;
        // four rows at a time: their 36 population loads are issued together
#pragma unroll
        for (int rb = 0; rb < TILE_H; rb += 4) {
            R v[4][9];
            bool use[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int jy = y0 + rb + i;
                use[i] = jx < ch.nx && jy < ch.ny && cell_kind(ch, jx, jy) != CK_SOLID;
                if (use[i]) {
                    const long long n = (long long)jy * ch.pitch + jx;
#pragma unroll
                    for (int q = 0; q < 9; ++q)
                        v[i][q] = PopIO<S, R>::ld(f + ch.f_off + q * ch.plane + n, q);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                typename Mom4<R>::T q;
                q.x = 0; q.y = 0; q.z = 0; q.w = 0;
                if (use[i]) {   // the cell's moments, in the working precision
                    R r, a, b;
                    lattice_moments(v[i], r, a, b);
                    q.x = (R)(double)r;
                    q.y = (R)(double)a;
                    q.z = (R)(double)b;
                }
                mom[(size_t)slot * TILE_CELLS + (rb + i) * TILE_W + lane] = q;
            }
        }
    }
}

// Move marker m with its interpolated velocity u (simulation.cpp:656-675,
// capsule.cpp:267-297).
__device__ __forceinline__ void move_marker(const ChannelDev& ch, const MarkerBufs& mb, int m,
                                            double2 u) {
    double2 p = mb.pos[m];
    const double ux = u.x, uy = u.y;
    mb.vel[m] = make_double2(ux, uy);
    // the step's correction before its last sweep (the network's label, or
    // on a learned step its seed) becomes the next step's network input
    mb.dFprev[m] = (mb.valid[m] && ch.ibm_iterations > 1)
                       ? make_double2(mb.dFsum[m].x - mb.dF[m].x, mb.dFsum[m].y - mb.dF[m].y)
                       : make_double2(0.0, 0.0);
    p.x = p.x + ux * ch.dt;
    p.y = p.y + uy * ch.dt;
    const double Lx = (double)ch.nx;
    if (isfinite(p.x)) {
        // the reference wraps with while-loops (capsule.cpp:287-296); moves
        // are far below one period, so a bounded loop gives the same result
        int it = 0;
        while (p.x < 0.0 && it < 8) { p.x += Lx; ++it; }
        while (p.x >= Lx && it < 16) { p.x -= Lx; ++it; }
        if (p.x < 0.0 || p.x >= Lx) {
            p.x = fmod(p.x, Lx);
            if (p.x < 0.0) p.x += Lx;
        }
    }
    if (!ch.periodic_y) {
        const double ymin = 1.5, ymax = (double)ch.ny - 1.5;
        if (p.y < ymin) p.y = ymin;
        if (p.y > ymax) p.y = ymax;
    }
    mb.pos[m] = p;
}

// Interpolate the new velocity and move the markers (FP64 contexts), one
// thread per marker.
template <typename S, typename R>
__global__ void k_interp_move(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb,
                              const S* __restrict__ f, const int* __restrict__ tile_slot,
                              const R* __restrict__ fin, const double* __restrict__ phi_tbl) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    double2 u = make_double2(0.0, 0.0);
    if (mb.valid[m]) u = interp_u_acc<S, R, R>(ch, mb, m, f, tile_slot, fin);
    move_marker(ch, mb, m, u);
}

// The marker move of the FP32-arithmetic modes, one warp per capsule: the
// warp first forms, for every cell of the box that holds its markers'
// stencils, the new state's moments (rho, jx, jy; zero on SOLID cells) and
// the cell's final force, into shared memory, the lanes running along the
// box's rows (each cell's nine populations are read once, coalesced, where
// the markers' stencils overlap); then each lane interpolates its markers
// from there with the terms, order and arithmetic of interp_u_acc (the same
// values, so the same result bit for bit), and moves them.  A capsule whose
// box exceeds MOVE_BOX_MAX cells interpolates from global memory as
// k_interp_move does.
// (out of line: the rare large capsule keeps its registers out of the box path)
template <typename S>
__device__ __noinline__ double2 interp_u_acc_global(const ChannelDev& ch, const MarkerBufs& mb,
                                                    int m, const S* __restrict__ f,
                                                    const int* __restrict__ tile_slot,
                                                    const float* __restrict__ fin) {
    return interp_u_acc<S, float, float>(ch, mb, m, f, tile_slot, fin);
}
constexpr int MOVE_WARPS = 4;
constexpr int MOVE_BOX_MAX = 512;
struct MoveBox {
    float rho[MOVE_BOX_MAX], jx[MOVE_BOX_MAX], jy[MOVE_BOX_MAX];
    float fx[MOVE_BOX_MAX], fy[MOVE_BOX_MAX];
};
template <typename S>
__global__ void __launch_bounds__(MOVE_WARPS * 32)
k_interp_move_caps(const CapsuleDev* __restrict__ caps, int ncaps,
                   const ChannelDev* __restrict__ chans, MarkerBufs mb, const S* __restrict__ f,
                   const int* __restrict__ tile_slot, const float* __restrict__ fin) {
    extern __shared__ __align__(16) unsigned char move_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * MOVE_WARPS + warp;
    if (c >= ncaps) return;
    MoveBox& B = reinterpret_cast<MoveBox*>(move_smem)[warp];
    const CapsuleDev cp = caps[c];
    const ChannelDev& ch = chans[cp.chan];
    const int nx = ch.nx, ny = ch.ny, n = cp.n, off = cp.off;
    // the stencils' box: x relative to the first marker (minimum image)
    int ref = 0;
    for (int k = 0; k < n; ++k)
        if (mb.valid[off + k]) { ref = mb.ix0[off + k]; break; }
    int dmin = INT_MAX, dmax = INT_MIN, ymin = INT_MAX, ymax = INT_MIN;
    for (int k = lane; k < n; k += 32) {
        if (!mb.valid[off + k]) continue;
        int d = mb.ix0[off + k] - ref;
        if (2 * d > nx) d -= nx;
        if (2 * d < -nx) d += nx;
        const int y = mb.iy0[off + k];
        dmin = min(dmin, d);
        dmax = max(dmax, d);
        ymin = min(ymin, y);
        ymax = max(ymax, y);
    }
    dmin = __reduce_min_sync(0xffffffffu, dmin);
    dmax = __reduce_max_sync(0xffffffffu, dmax);
    ymin = __reduce_min_sync(0xffffffffu, ymin);
    ymax = __reduce_max_sync(0xffffffffu, ymax);
    const bool any = dmin <= dmax;
    const int bw = dmax - dmin + 4, bh = ymax - ymin + 4;
    const bool boxed = any && (long long)bw * bh <= MOVE_BOX_MAX;
    if (boxed) {
        const int bx0 = ref + dmin - 1, by0 = ymin - 1;
        for (int i = lane; i < bw * bh; i += 32) {
            const int by = i / bw, bx = i - by * bw;
            int jx = (bx0 + bx) % nx;
            if (jx < 0) jx += nx;
            const int jy = by0 + by;
            float r = 0.f, a = 0.f, b = 0.f, gx = 0.f, gy = 0.f;
            if (jy >= 0 && jy < ny && cell_kind(ch, jx, jy) != CK_SOLID) {
                const long long nn = (long long)jy * ch.pitch + jx;
                float v[9];
#pragma unroll
                for (int q = 0; q < 9; ++q)
                    v[q] = PopIO<S, float>::ld(f + ch.f_off + q * ch.plane + nn, q);
                lattice_moments(v, r, a, b);
                const int t = ch.tile_base + (jy / TILE_H) * ch.tiles_x + jx / TILE_W;
                const int sl = tile_slot[t];
                if (sl >= 0) {
                    const int cell = (jy % TILE_H) * TILE_W + (jx % TILE_W);
                    gx = fin[(size_t)sl * 2 * TILE_CELLS + cell];
                    gy = fin[(size_t)sl * 2 * TILE_CELLS + TILE_CELLS + cell];
                }
            }
            B.rho[i] = r;
            B.jx[i] = a;
            B.jy[i] = b;
            B.fx[i] = gx;
            B.fy[i] = gy;
        }
        __syncwarp();
    }
    for (int k = lane; k < n; k += 32) {
        const int m = off + k;
        double2 u = make_double2(0.0, 0.0);
        if (mb.valid[m]) {
            if (!boxed) {
                u = interp_u_acc_global<S>(ch, mb, m, f, tile_slot, fin);
            } else {
                const int ix0 = mb.ix0[m], iy0 = mb.iy0[m];
                int d = ix0 - ref;
                if (2 * d > nx) d -= nx;
                if (2 * d < -nx) d += nx;
                const double2* wx2 = reinterpret_cast<const double2*>(mb.wx + 4 * (size_t)m);
                const double2* wy2 = reinterpret_cast<const double2*>(mb.wy + 4 * (size_t)m);
                const double2 wxa = wx2[0], wxb = wx2[1], wya = wy2[0], wyb = wy2[1];
                const float wxs[4] = {(float)wxa.x, (float)wxa.y, (float)wxb.x, (float)wxb.y};
                const float wys[4] = {(float)wya.x, (float)wya.y, (float)wyb.x, (float)wyb.y};
                float ux = 0.f, uy = 0.f;
#pragma unroll
                for (int sy = 0; sy < 4; ++sy) {
                    const int jy = iy0 - 1 + sy;
                    if (jy < 0 || jy >= ny) continue;
                    const int row = (iy0 - ymin + sy) * bw + (d - dmin);
#pragma unroll
                    for (int sx = 0; sx < 4; ++sx) {
                        const float w = wxs[sx] * wys[sy];
                        if (w > 1e-15f) {
                            const int i = row + sx;
                            const float rho = B.rho[i];
                            float cu = 0.f, cv = 0.f;
                            if (rho > 1e-15f) {
                                const float inv = __frcp_rn(rho);
                                cu = (B.jx[i] + 0.5f * B.fx[i]) * inv;
                                cv = (B.jy[i] + 0.5f * B.fy[i]) * inv;
                            }
                            ux += cu * w;
                            uy += cv * w;
                        }
                    }
                }
                u = make_double2((double)ux, (double)uy);
            }
        }
        move_marker(ch, mb, m, u);
    }
}

// ============================ launch wrappers ==============================

size_t membrane_smem_bytes(int maxn) {
    return (size_t)MEM_WARPS * MEM_DOUBLES_PER_NODE * maxn * sizeof(double);
}

int spread_blocks_per_sm(bool fp64) {
    int b = 0;
    const cudaError_t e =
        fp64 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_spread<double>,
                                                             SPREAD_WARPS * 32,
                                                             spread_smem<double>())
             : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_spread_fx,
                                                             SPREAD_WARPS * 32,
                                                             spread_fx_smem());
    if (e != cudaSuccess || b < 1) b = 1;
    return b;
}

cudaError_t prepare_spread() {
    cudaError_t e = cudaFuncSetAttribute(k_spread<double>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)spread_smem<double>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_spread_fx, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)spread_fx_smem());
    return e;
}

// ---------------- capsule geometry (thermo) ---------------------------------
// One thread per capsule, FP64 in the reference's serial order:
// Capsule::centroid, area, perimeter, secondMoments, deformationIndex and
// inclinationAngle (capsule.cpp:159-266).  Unwrapped nodes are regenerated
// on the fly (p_0 = X_0, p_i = p_{i-1} + minImage(X_i - X_{i-1})).
__device__ __forceinline__ double2 unwrap_next(const double2* X, int i, double2 p, double Lx) {
    const double2 d = min_image_d(X[i], X[i - 1], Lx);
    return make_double2(p.x + d.x, p.y + d.y);
}

__device__ void capsule_moments(const double2* X, int n, double Lx, double& mxx, double& myy,
                                double& mxy) {
    // capsule.cpp:209-247
    double A = 0.0, cx = 0.0, cy = 0.0;
    double2 a = X[0];
    const double2 p0 = a;
    for (int i = 0; i < n; ++i) {
        const double2 b = (i + 1 < n) ? unwrap_next(X, i + 1, a, Lx) : p0;
        const double cr = a.x * b.y - b.x * a.y;
        A += cr;
        cx += (a.x + b.x) * cr;
        cy += (a.y + b.y) * cr;
        a = b;
    }
    A *= 0.5;
    mxx = myy = mxy = 0.0;
    if (fabs(A) < 1e-15) return;
    cx /= (6.0 * A);
    cy /= (6.0 * A);
    a = p0;
    for (int i = 0; i < n; ++i) {
        const double2 q = (i + 1 < n) ? unwrap_next(X, i + 1, a, Lx) : p0;
        const double x0 = a.x - cx, y0 = a.y - cy;
        const double x1 = q.x - cx, y1 = q.y - cy;
        const double cr = x0 * y1 - x1 * y0;
        mxx += (x0 * x0 + x0 * x1 + x1 * x1) * cr;
        myy += (y0 * y0 + y0 * y1 + y1 * y1) * cr;
        mxy += (x0 * y1 + 2.0 * x0 * y0 + 2.0 * x1 * y1 + x1 * y0) * cr;
        a = q;
    }
    const double sgn = (A > 0.0) ? 1.0 : -1.0;
    mxx *= sgn / 12.0;
    myy *= sgn / 12.0;
    mxy *= sgn / 24.0;
}

__global__ void k_capsule_stats(const CapsuleDev* __restrict__ caps, int ncaps,
                                const double2* __restrict__ pos, double* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncaps) return;
    const CapsuleDev cd = caps[c];
    const double2* X = pos + cd.off;
    const int n = cd.n;
    const double Lx = (double)cd.periodic_nx;
    double* o = out + 6LL * c;
    // centroid (capsule.cpp:159-172)
    double2 cen = make_double2(0.0, 0.0);
    if (cd.periodic_nx > 0 && n > 0) {
        const double2 ref = X[0];
        double2 sum = ref;
        for (int i = 1; i < n; ++i) {
            const double2 d = min_image_d(X[i], ref, Lx);
            sum.x += ref.x + d.x;
            sum.y += ref.y + d.y;
        }
        cen = make_double2(sum.x / (double)n, sum.y / (double)n);
    } else if (n > 0) {
        for (int i = 0; i < n; ++i) {
            cen.x += X[i].x;
            cen.y += X[i].y;
        }
        cen = make_double2(cen.x / (double)n, cen.y / (double)n);
    }
    // area (capsule.cpp:174-195)
    double A = 0.0;
    if (cd.periodic_nx > 0 && n > 0) {
        double2 a = X[0];
        const double2 p0 = a;
        for (int i = 0; i < n; ++i) {
            const double2 b = (i + 1 < n) ? unwrap_next(X, i + 1, a, Lx) : p0;
            A += a.x * b.y - a.y * b.x;
            a = b;
        }
    } else {
        for (int i = 0; i < n; ++i) {
            const double2 a = X[i], b = X[(i + 1) % n];
            A += a.x * b.y - a.y * b.x;
        }
    }
    // perimeter (capsule.cpp:197-204)
    double P = 0.0;
    for (int i = 0; i < n; ++i) P += norm_d(min_image_d(X[(i + 1) % n], X[i], Lx));
    // deformation index and inclination (capsule.cpp:249-266)
    double D = 0.0, th = 0.0;
    if (n >= 3) {
        double mxx, myy, mxy;
        capsule_moments(X, n, Lx, mxx, myy, mxy);
        const double tr = 0.5 * (mxx + myy);
        const double dd = sqrt(0.25 * (mxx - myy) * (mxx - myy) + mxy * mxy);
        const double J1 = tr + dd;
        const double t2 = tr - dd;
        const double J2 = (t2 < 0.0) ? 0.0 : t2;
        const double s1 = sqrt(J1), s2 = sqrt(J2);
        D = (s1 + s2 > 1e-15) ? (s1 - s2) / (s1 + s2) : 0.0;
        th = 0.5 * atan2(2.0 * mxy, mxx - myy);
    }
    o[0] = cen.x;
    o[1] = cen.y;
    o[2] = 0.5 * fabs(A);
    o[3] = P;
    o[4] = D;
    o[5] = th;
}

void launch_capsule_stats(const CapsuleDev* caps, int ncaps, const double2* pos, double* out,
                          cudaStream_t st) {
    if (ncaps == 0) return;
    k_capsule_stats<<<(ncaps + 127) / 128, 128, 0, st>>>(caps, ncaps, pos, out);
}

cudaError_t prepare_membrane(int maxn) {
    const size_t smem = membrane_smem_bytes(maxn);
    if (smem <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(k_membrane, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
}

void launch_membrane(const CapsuleDev* caps, int ncaps, const MarkerBufs& mb, int* has_prev,
                     int maxn, unsigned* status, cudaStream_t st) {
    if (ncaps == 0) return;
    const size_t smem = membrane_smem_bytes(maxn);
    const int blocks = (ncaps + MEM_WARPS - 1) / MEM_WARPS;
    k_membrane<<<blocks, MEM_WARPS * 32, smem, st>>>(caps, ncaps, mb, has_prev, maxn, status);
}

// ---------------- obstacle repulsion (pillars) -------------------------------
// Obstacle::signedDistance / normalAt of CircleObstacle and RectObstacle
// (geometry/circle_obstacle.h:17-37, rect_obstacle.h:18-59) with the
// first-extremum semantics of std::min / std::max over initializer lists.
__device__ __forceinline__ double max3(double a, double b, double c) {
    double m = a;
    if (m < b) m = b;
    if (m < c) m = c;
    return m;
}
__device__ __forceinline__ double min4(double a, double b, double c, double d) {
    double m = a;
    if (b < m) m = b;
    if (c < m) m = c;
    if (d < m) m = d;
    return m;
}

__device__ void pillar_geometry(const double* o, double x, double y, double& sd, double2& nrm) {
    if (o[0] == 0.0) {   // circle (a, b) radius c
        const double dx = x - o[1], dy = y - o[2];
        const double d = sqrt(dx * dx + dy * dy);
        sd = d - o[3];
        nrm = (d < 1e-15) ? make_double2(1.0, 0.0) : make_double2(dx / d, dy / d);
        return;
    }
    const double x0 = o[1], y0 = o[2], x1 = o[3], y1 = o[4];
    {
        const double dx = max3(x0 - x, x - x1, 0.0);
        const double dy = max3(y0 - y, y - y1, 0.0);
        const double outside = sqrt(dx * dx + dy * dy);
        sd = (outside > 1e-15) ? outside : -min4(x - x0, x1 - x, y - y0, y1 - y);
    }
    // nearestPoint
    const double cx = (x < x0) ? x0 : ((x1 < x) ? x1 : x);
    const double cy = (y < y0) ? y0 : ((y1 < y) ? y1 : y);
    double2 np;
    if (cx == x && cy == y) {
        const double dl = x - x0, dr = x1 - x, db = y - y0, dt = y1 - y;
        const double dmin = min4(dl, dr, db, dt);
        if (dmin == dl) np = make_double2(x0, y);
        else if (dmin == dr) np = make_double2(x1, y);
        else if (dmin == db) np = make_double2(x, y0);
        else np = make_double2(x, y1);
    } else {
        np = make_double2(cx, cy);
    }
    const double ddx = x - np.x, ddy = y - np.y;
    const double d = sqrt(ddx * ddx + ddy * ddy);
    if (d < 1e-15) {
        const double dl = fabs(x - x0), dr = fabs(x - x1), db = fabs(y - y0), dt = fabs(y - y1);
        const double dmin = min4(dl, dr, db, dt);
        if (dmin == dl) nrm = make_double2(-1.0, 0.0);
        else if (dmin == dr) nrm = make_double2(1.0, 0.0);
        else if (dmin == db) nrm = make_double2(0.0, -1.0);
        else nrm = make_double2(0.0, 1.0);
    } else {
        nrm = make_double2(ddx / d, ddy / d);
    }
}

// RepulsionForce::computeObstacleRepulsion (repulsion.cpp:180-235) for every
// pillar of the marker's channel in order, after the pair contact.
__global__ void k_obstacle_repulsion(const ChannelDev* __restrict__ chans, int M, MarkerBufs mb) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    const ChannelDev& ch = chans[mb.mk_chan[m]];
    if (ch.n_pillars == 0) return;
    const double2 p = mb.pos[m], v = mb.vel[m];
    double2 f = mb.frc[m];
    const double r_cut = ch.rep_r_cut, eps = ch.rep_epsilon, sigma = ch.rep_sigma;
    const double gamma_n = ch.rep_damping, mu = ch.rep_friction;
    for (int k = 0; k < ch.n_pillars; ++k) {
        double sd;
        double2 nrm;
        pillar_geometry(ch.pillars + 5 * k, p.x, p.y, sd, nrm);
        if (sd >= r_cut) continue;
        double r = fabs(sd);
        if (r < 1e-15) r = 1e-15;
        const double F_rep = eps * pow(sigma / r, (double)ch.rep_power);
        if (sd < 0.0) {
            const double s = F_rep * 10.0;
            f.x += nrm.x * s;
            f.y += nrm.y * s;
            continue;
        }
        double F_n = F_rep;
        double2 F_t = make_double2(0.0, 0.0);
        if (gamma_n > 0.0 || mu > 0.0) {
            const double v_n = v.x * nrm.x + v.y * nrm.y;
            F_n = F_rep - gamma_n * v_n;
            if (F_n < 0.0) F_n = 0.0;
            if (mu > 0.0) {
                const double2 v_t = make_double2(v.x - nrm.x * v_n, v.y - nrm.y * v_n);
                const double v_t_mag = sqrt(v_t.x * v_t.x + v_t.y * v_t.y);
                if (v_t_mag > 1e-12) {
                    const double s = -mu * F_n;
                    F_t = make_double2((v_t.x / v_t_mag) * s, (v_t.y / v_t_mag) * s);
                }
            }
        }
        f.x += nrm.x * F_n + F_t.x;
        f.y += nrm.y * F_n + F_t.y;
    }
    mb.frc[m] = f;
}

void launch_obstacle_repulsion(const ChannelDev* chans, int M, const MarkerBufs& mb,
                               cudaStream_t st) {
    if (M == 0) return;
    k_obstacle_repulsion<<<(M + 255) / 256, 256, 0, st>>>(chans, M, mb);
}

void launch_contact(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                    int ncells, cudaStream_t st) {
    launch_contact_prep(chans, M, mb, cb, ncells, st);
    launch_contact_force(chans, M, mb, cb, st);
}

void launch_contact_force(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                          cudaStream_t st) {
    if (M == 0) return;
    const int B = 256, G = (M + B - 1) / B;
    k_contact_force<<<G, B, 0, st>>>(chans, M, mb, cb.cell_of, cb.cell_start, cb.cell_cnt,
                                     cb.list);
}

void launch_contact_prep(const ChannelDev* chans, int M, const MarkerBufs& mb, ContactBufs& cb,
                         int ncells, cudaStream_t st) {
    if (M == 0) return;
    const int B = 256, G = (M + B - 1) / B;
    if (ncells > 0) {
        cudaMemsetAsync(cb.cell_cnt, 0, sizeof(int) * ncells, st);
        cudaMemsetAsync(cb.cursor, 0, sizeof(int) * ncells, st);
        k_contact_bin<<<G, B, 0, st>>>(chans, M, mb, cb.cell_of, cb.cell_cnt);
        scan_exclusive(cb.cell_cnt, cb.cell_start, ncells, cb.scan_tmp, nullptr, st);
        k_contact_fill<<<G, B, 0, st>>>(chans, M, mb, cb.cell_of, cb.cell_start, cb.cursor,
                                        cb.list);
        k_contact_sort<<<(ncells + B - 1) / B, B, 0, st>>>(ncells, cb.cell_start, cb.cell_cnt,
                                                           cb.list);
    }
}

void launch_tiles(const ChannelDev* chans, const CapsuleDev* caps, int M, const MarkerBufs& mb,
                  TileBufs& tb, int T, int parity, const double* phi_tbl, unsigned* status,
                  cudaStream_t st, cudaEvent_t slots_ready) {
    const int B = 256, G = (M + B - 1) / B;
    cudaMemsetAsync(tb.tile_flag, 0, sizeof(int) * T, st);
    cudaMemsetAsync(tb.tile_cnt, 0, sizeof(int) * T, st);
    cudaMemsetAsync(tb.cursor, 0, sizeof(int) * T, st);
    cudaMemsetAsync(tb.cls_cnt, 0, sizeof(int) * SLOT_CLASSES, st);
    k_ibm_prep<<<G, B, 0, st>>>(chans, caps, M, mb, phi_tbl, tb.tile_flag, tb.tile_cnt, status);
    scan_exclusive(tb.tile_flag, tb.slot_scan, T, tb.scan_tmp, tb.n_slots, st);
    scan_exclusive(tb.tile_cnt, tb.list_off, T, tb.scan_tmp, nullptr, st);
    k_tile_slots<<<(T + B - 1) / B, B, 0, st>>>(T, tb.tile_flag, tb.slot_scan,
                                                tb.tile_slot[parity], tb.slot_tile, chans,
                                                tb.tile_chan, tb.tile_cnt, tb.list_off,
                                                tb.slot_info, tb.cls_cnt, tb.slot_rank);
    if (slots_ready) cudaEventRecord(slots_ready, st);
    k_slot_order<<<148, 256, 0, st>>>(tb.n_slots, tb.slot_info, tb.cls_cnt, tb.slot_rank,
                                      tb.slot_order);
    k_tile_fill<<<G, B, 0, st>>>(chans, M, mb, tb.list_off, tb.cursor, tb.list,
                                 tb.tile_slot[parity]);
}

template <typename R>
void launch_spread(const ChannelDev* chans, const MarkerBufs& mb, TileBufs& tb, int parity,
                   int sweep, int mode, int launch_idx, int grid, unsigned* status,
                   cudaStream_t st) {
    if constexpr (sizeof(R) == 4) {
        k_spread_fx<<<grid, SPREAD_WARPS * 32, spread_fx_smem(), st>>>(
            chans, tb.slot_info, tb.slot_order, tb.n_slots, tb.list, mb, tb.acc, tb.acc0,
            static_cast<float*>(tb.gsnap), static_cast<float*>(tb.fin[parity]), sweep, mode,
            tb.resid_gate, tb.plain_needed, tb.capped, tb.fluid_touched, status);
    } else {
        k_spread<R><<<grid, SPREAD_WARPS * 32, spread_smem<R>(), st>>>(
            chans, tb.slot_info, tb.slot_order, tb.n_slots, tb.spread_ctr + launch_idx, tb.list,
            mb, tb.acc,
            tb.acc0, static_cast<R*>(tb.gsnap), static_cast<R*>(tb.fin[parity]), sweep, mode,
            tb.resid_gate, tb.plain_needed, tb.capped, tb.fluid_touched, status);
    }
}
template void launch_spread<double>(const ChannelDev*, const MarkerBufs&, TileBufs&, int, int,
                                    int, int, int, unsigned*, cudaStream_t);
template void launch_spread<float>(const ChannelDev*, const MarkerBufs&, TileBufs&, int, int, int,
                                   int, int, unsigned*, cudaStream_t);

template <typename S, typename R>
void launch_mdf_interp(const ChannelDev* chans, int M, const MarkerBufs& mb, const S* f,
                       TileBufs& tb, int parity, int sweep, int mode, cudaStream_t st) {
    (void)f;
    const int B = tb.marker_block, G = (M + B - 1) / B;
    k_mdf_interp<S, R><<<G, B, 0, st>>>(chans, M, mb, tb.tile_slot[parity],
                                        static_cast<const typename Mom4<R>::T*>(tb.mom), tb.acc,
                                        tb.acc0, sweep, mode, tb.resid_gate, tb.resid_plain,
                                        tb.plain_needed);
}

template <typename S, typename R>
void launch_tile_moments(const ChannelDev* chans, const S* f, TileBufs& tb, int grid,
                         cudaStream_t st) {
    k_tile_moments<S, R><<<grid, 256, 0, st>>>(chans, tb.slot_info, tb.n_slots, f,
                                               static_cast<typename Mom4<R>::T*>(tb.mom));
}

template <typename S, typename R>
void launch_interp_move(const ChannelDev* chans, const CapsuleDev* caps, int ncaps, int M,
                        const MarkerBufs& mb, const S* f, TileBufs& tb, int parity,
                        const double* phi_tbl, cudaStream_t st) {
    if constexpr (sizeof(R) == 4) {
        (void)phi_tbl;
        if (ncaps == 0) return;
        k_interp_move_caps<S><<<(ncaps + MOVE_WARPS - 1) / MOVE_WARPS, MOVE_WARPS * 32,
                                MOVE_WARPS * sizeof(MoveBox), st>>>(
            caps, ncaps, chans, mb, f, tb.tile_slot[parity],
            static_cast<const float*>(tb.fin[parity]));
    } else {
        const int B = tb.marker_block, G = (M + B - 1) / B;
        k_interp_move<S, R><<<G, B, 0, st>>>(chans, M, mb, f, tb.tile_slot[parity],
                                             static_cast<const R*>(tb.fin[parity]), phi_tbl);
    }
}

#define SFG_INST(S, R)                                                                          \
    template void launch_mdf_interp<S, R>(const ChannelDev*, int, const MarkerBufs&, const S*,  \
                                          TileBufs&, int, int, int, cudaStream_t);              \
    template void launch_tile_moments<S, R>(const ChannelDev*, const S*, TileBufs&, int,       \
                                            cudaStream_t);                                      \
    template void launch_interp_move<S, R>(const ChannelDev*, const CapsuleDev*, int, int,     \
                                           const MarkerBufs&, const S*, TileBufs&, int,        \
                                           const double*, cudaStream_t);
SFG_INST(double, double)
SFG_INST(float, float)
SFG_INST(__half, float)
#undef SFG_INST

}  // namespace sfg
