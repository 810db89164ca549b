// chemistry.cu -- capsule chemistry of the scalar after each scalar step:
// constant release / absorption at the nearest node
// (AdvectionDiffusion::applySourceSink, advection_diffusion.cpp:225-271) or
// Fick leaching from finite reservoirs with Langmuir adsorption and
// Peskin-weighted exchange (applyChemistry, :273-437).
//
// The reference walks capsules and nodes one after the other, and every
// node reads the concentration its predecessors have just changed.  Here
// one CTA serves one channel: each capsule's nodes run in order in one
// thread, and capsules run in waves -- a capsule joins the wave after the
// last earlier capsule whose stencil footprint overlaps its own -- so every
// read sees exactly the writes the serial loop would have made before it.
// FP64 state and arithmetic in the reference's order (compiled without FMA
// contraction); the scalar fields are stored in the lattice's arithmetic
// type R.
//
// Concentration: after a scalar step the reference keeps C = sum_q g per
// node; chemistry overwrites C at the nodes it touches and resets their g
// to w C.  A per-node flag marks such overwritten values (the field is
// then the stored C, not sum g) until the next scalar step consumes them.
#include <cstdio>

#include "../../include/softflow_gpu.h"
#include "common.cuh"
#include "markers.cuh"
#include "sfg_internal.h"

namespace sfg {

constexpr int CHEM_THREADS = 256;

struct ChemBox {
    int x0, x1, y0, y1;   // stencil footprint, x unwrapped around node 0
};

__device__ __forceinline__ bool chem_overlap(const ChemBox& a, const ChemBox& b, int nx) {
    if (a.y1 < b.y0 || b.y1 < a.y0) return false;
    if (a.x1 - a.x0 + 1 >= nx || b.x1 - b.x0 + 1 >= nx) return true;
    for (int k = -2; k <= 2; ++k) {
        const int c0 = b.x0 + k * nx, c1 = b.x1 + k * nx;
        if (!(c1 < a.x0 || c0 > a.x1)) return true;
    }
    return false;
}

template <typename R>
struct ChemField {
    R* g;                     // scalar populations after this step's scalar step
    R* g_other;               // the other buffer (SOLID nodes are never streamed)
    R* cf;                    // stored concentration of overwritten nodes
    unsigned char* cov;       // 1: cf holds the node's concentration
    ChannelDev ch;

    __device__ double C(int x, int y) const {
        const long long n = (long long)y * ch.pitch + x;
        if (cov[ch.cell_off + n]) return (double)cf[ch.cell_off + n];
        const R* p = g + ch.g_off + n;
        const long long P = ch.plane;
        const R s = p[0] + p[P] + p[2 * P] + p[3 * P] + p[4 * P] + p[5 * P] + p[6 * P] +
                    p[7 * P] + p[8 * P];
        return (double)s;
    }
    // C(x, y) = c and g = w c (advection_diffusion.cpp:265-268, 421-423)
    __device__ void set(int x, int y, double c) const {
        const long long n = (long long)y * ch.pitch + x;
        cf[ch.cell_off + n] = (R)c;
        cov[ch.cell_off + n] = 1;
        const bool solid = !ch.periodic_y && (y == 0 || y == ch.ny - 1);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const R v = (R)(w_of(q) * c);
            g[ch.g_off + q * ch.plane + n] = v;
            if (solid) g_other[ch.g_off + q * ch.plane + n] = v;
        }
    }
};

__device__ __forceinline__ double chem_param(const double* v, int n, int type, double dflt) {
    return type < n ? v[type] : dflt;
}

template <typename R>
__device__ void chem_capsule_source(const ChemField<R>& F, const sfg_chemistry& P,
                                    const CapsuleDev& cd, const double2* __restrict__ pos,
                                    double* released, double* absorbed, int c) {
    const int nx = F.ch.nx, ny = F.ch.ny;
    const double release = chem_param(P.release, P.n_release, cd.type, 0.0);
    const double absorb = chem_param(P.absorb, P.n_absorb, cd.type, 0.0);
    for (int ni = 0; ni < cd.n; ++ni) {
        const double2 p = pos[cd.off + ni];
        int ix = (int)(p.x + 0.5);
        int iy = (int)(p.y + 0.5);
        ix = ix < 0 ? 0 : (ix > nx - 1 ? nx - 1 : ix);
        iy = iy < 0 ? 0 : (iy > ny - 1 ? ny - 1 : iy);
        double C = F.C(ix, iy);
        C += release;
        released[c] += release;
        const double actual = (C < absorb) ? C : absorb;   // std::min(absorb, C)
        C -= actual;
        absorbed[c] += actual;
        F.set(ix, iy, C);
    }
}

template <typename R>
__device__ void chem_capsule_physics(const ChemField<R>& F, const sfg_chemistry& P,
                                     const CapsuleDev& cd, const double2* __restrict__ pos,
                                     const double* __restrict__ phi, double* released,
                                     double* absorbed, double* Mp, double* gamma, int c) {
    const int nx = F.ch.nx, ny = F.ch.ny, Lx = nx;
    const int type = cd.type, Nn = cd.n;
    const double k_L = chem_param(P.k_leach, P.n_k_leach, type, 0.0);
    const double Ceq = chem_param(P.C_eq, P.n_C_eq, type, 0.0);
    const double k_a = chem_param(P.k_adsorb, P.n_k_adsorb, type, 0.0);
    const double k_d = chem_param(P.k_desorb, P.n_k_desorb, type, 0.0);
    const double Gmax = chem_param(P.Gamma_max, P.n_Gamma_max, type, 1.0);
    const double const_release = chem_param(P.release, P.n_release, type, 0.0);
    const double const_absorb = chem_param(P.absorb, P.n_absorb, type, 0.0);
    for (int k = 0; k < Nn; ++k) {
        const double2 ps = pos[cd.off + k];
        const double2 pp = pos[cd.off + (k + 1) % Nn];
        const double2 pm = pos[cd.off + (k - 1 + Nn) % Nn];
        const double dxp = pp.x - ps.x, dyp = pp.y - ps.y;
        const double dxm = ps.x - pm.x, dym = ps.y - pm.y;
        double ds = 0.5 * (sqrt(dxp * dxp + dyp * dyp) + sqrt(dxm * dxm + dym * dym));
        if (ds < 1e-12) ds = 1.0;
        const int ix0 = (int)floor(ps.x), iy0 = (int)floor(ps.y);
        double C_surf = 0.0;
        for (int dy = -1; dy <= 2; ++dy) {
            const int jy = iy0 + dy;
            if (jy < 0 || jy >= ny) continue;
            for (int dx = -1; dx <= 2; ++dx) {
                const int jx = (((ix0 + dx) % Lx) + Lx) % Lx;
                const double rx = ps.x - (double)(ix0 + dx);
                const double ry = ps.y - (double)jy;
                const double w = phi_lut(phi, rx) * phi_lut(phi, ry);
                C_surf += F.C(jx, jy) * w;
            }
        }
        double dC_leach = 0.0;
        if (k_L > 0.0) {
            dC_leach = k_L * (Ceq - C_surf);
            if (Mp[c] >= 0.0) {
                if (dC_leach > 0.0) {
                    const double available_per_ds = Mp[c] / ds;
                    dC_leach = (available_per_ds < dC_leach) ? available_per_ds : dC_leach;
                    Mp[c] -= dC_leach * ds;
                    if (Mp[c] < 0.0) Mp[c] = 0.0;
                }
            }
        } else {
            const double absorb_now = (C_surf < const_absorb) ? C_surf : const_absorb;
            dC_leach = const_release - absorb_now;
        }
        double dC_adsorb = 0.0;
        if (k_a > 0.0 || k_d > 0.0) {
            double G = gamma[cd.off + k];
            const double dGamma = k_a * C_surf * (1.0 - G / Gmax) - k_d * G;
            double t = G + dGamma;
            t = (t < Gmax) ? t : Gmax;
            G = (0.0 < t) ? t : 0.0;
            gamma[cd.off + k] = G;
            dC_adsorb = -dGamma;
        }
        const double total_flux = dC_leach + dC_adsorb;
        if (total_flux == 0.0) continue;
        for (int dy = -1; dy <= 2; ++dy) {
            const int jy = iy0 + dy;
            if (jy < 0 || jy >= ny) continue;
            for (int dx = -1; dx <= 2; ++dx) {
                const int jx = (((ix0 + dx) % Lx) + Lx) % Lx;
                const double rx = ps.x - (double)(ix0 + dx);
                const double ry = ps.y - (double)jy;
                const double w = phi_lut(phi, rx) * phi_lut(phi, ry);
                if (w < 1e-15) continue;
                double C = F.C(jx, jy);
                C += total_flux * w * ds;
                if (C < 0.0) C = 0.0;
                F.set(jx, jy, C);
            }
        }
        if (total_flux > 0.0) released[c] += total_flux * ds;
        else absorbed[c] -= total_flux * ds;
    }
}

// One CTA per channel.  Capsules of the channel: footprints, waves by
// relaxation (wave = 1 + the largest wave of an earlier overlapping
// capsule; Jacobi sweeps converge in as many sweeps as the longest chain,
// bounded by the capsule count), then the waves in order.
template <typename R>
__global__ void __launch_bounds__(CHEM_THREADS)
k_chemistry(const ChannelDev* __restrict__ chans, const sfg_chemistry* __restrict__ params,
            const CapsuleDev* __restrict__ caps, const double2* __restrict__ pos,
            const double* __restrict__ phi, R* g_new, R* g_old, R* cfield,
            unsigned char* cov, double* released, double* absorbed, double* Mp,
            double* gamma, int* wave_buf, ChemBox* box_buf, int box_cap,
            unsigned* status) {
    const ChannelDev ch = chans[blockIdx.x];
    if (!ch.chem || ch.cap_end <= ch.cap_begin) return;
    const sfg_chemistry& P = params[blockIdx.x];
    const int c0 = ch.cap_begin, nc = ch.cap_end - ch.cap_begin;
    if (nc > box_cap) {
        if (threadIdx.x == 0) atomicOr(status, ST_CAPSULE_TOO_BIG);
        return;
    }
    // SOLID rows are not visited by the scalar step: a value the previous
    // chemistry stored there became sum g at the reference's concentration
    // update of this step (advection_diffusion.cpp:212-223)
    if (!ch.periodic_y) {
        for (int x = threadIdx.x; x < ch.nx; x += blockDim.x) {
            cov[ch.cell_off + x] = 0;
            cov[ch.cell_off + (long long)(ch.ny - 1) * ch.pitch + x] = 0;
        }
    }
    __syncthreads();
    ChemBox* box = box_buf + c0;
    int* wave = wave_buf + 2 * c0;        // [nc] current, [nc] next
    int* wnext = wave + nc;
    for (int i = threadIdx.x; i < nc; i += blockDim.x) {
        const CapsuleDev cd = caps[c0 + i];
        const double2 p0 = pos[cd.off];
        double xmin = p0.x, xmax = p0.x, ymin = p0.y, ymax = p0.y;
        const double Lx = (double)ch.nx;
        for (int k = 1; k < cd.n; ++k) {
            const double2 p = pos[cd.off + k];
            double x = p.x;
            if (x - p0.x > 0.5 * Lx) x -= Lx;
            if (x - p0.x < -0.5 * Lx) x += Lx;
            xmin = fmin(xmin, x);
            xmax = fmax(xmax, x);
            ymin = fmin(ymin, p.y);
            ymax = fmax(ymax, p.y);
        }
        ChemBox b;
        b.x0 = (int)floor(xmin) - 1;
        b.x1 = (int)floor(xmax) + 2;
        b.y0 = (int)floor(ymin) - 1;
        b.y1 = (int)floor(ymax) + 2;
        // non-finite positions: one footprint over everything (serial)
        if (!(xmin == xmin) || !(xmax == xmax) || !(ymin == ymin) || !(ymax == ymax)) {
            b.x0 = 0;
            b.x1 = ch.nx;
            b.y0 = -1000000000;
            b.y1 = 1000000000;
        }
        box[i] = b;
        wave[i] = 0;
    }
    __syncthreads();
    __shared__ int changed;
    for (int it = 0; it <= nc; ++it) {
        if (threadIdx.x == 0) changed = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            int w = 0;
            for (int j = 0; j < i; ++j)
                if (chem_overlap(box[i], box[j], ch.nx)) w = max(w, wave[j] + 1);
            wnext[i] = w;
            if (w != wave[i]) changed = 1;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nc; i += blockDim.x) wave[i] = wnext[i];
        // every thread takes the flag before thread 0 may clear it again
        const int done = !changed;
        __syncthreads();
        if (done) break;
    }
    __shared__ int maxw;
    if (threadIdx.x == 0) maxw = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < nc; i += blockDim.x) atomicMax(&maxw, wave[i]);
    __syncthreads();
    ChemField<R> F{g_new, g_old, cfield, cov, ch};
    const bool physics = P.n_k_leach > 0 || P.n_k_adsorb > 0;
    for (int w = 0; w <= maxw; ++w) {
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            if (wave[i] != w) continue;
            const CapsuleDev cd = caps[c0 + i];
            if (physics)
                chem_capsule_physics<R>(F, P, cd, pos, phi, released, absorbed, Mp, gamma, c0 + i);
            else
                chem_capsule_source<R>(F, P, cd, pos, released, absorbed, c0 + i);
        }
        __syncthreads();
    }
}

template <typename R>
void launch_chemistry(const ChannelDev* chans, int nch, const sfg_chemistry* params,
                      const CapsuleDev* caps, const double2* pos, const double* phi, void* g_new,
                      void* g_old, void* cfield, unsigned char* cov, double* released,
                      double* absorbed, double* Mp, double* gamma, int* wave_buf,
                      void* box_buf, int box_cap, unsigned* status, cudaStream_t st) {
    k_chemistry<R><<<nch, CHEM_THREADS, 0, st>>>(
        chans, params, caps, pos, phi, static_cast<R*>(g_new), static_cast<R*>(g_old),
        static_cast<R*>(cfield), cov, released, absorbed, Mp, gamma, wave_buf,
        static_cast<ChemBox*>(box_buf), box_cap, status);
}

size_t chem_box_bytes() { return sizeof(ChemBox); }

template void launch_chemistry<double>(const ChannelDev*, int, const sfg_chemistry*,
                                       const CapsuleDev*, const double2*, const double*, void*,
                                       void*, void*, unsigned char*, double*, double*, double*,
                                       double*, int*, void*, int, unsigned*, cudaStream_t);
template void launch_chemistry<float>(const ChannelDev*, int, const sfg_chemistry*,
                                      const CapsuleDev*, const double2*, const double*, void*,
                                      void*, void*, unsigned char*, double*, double*, double*,
                                      double*, int*, void*, int, unsigned*, cudaStream_t);

}  // namespace sfg
