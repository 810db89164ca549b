// markers.cuh -- Lagrangian-side kernels: membrane forces, soft contact,
// immersed-boundary force tiles, deterministic spreading, multi-direct
// forcing, and interpolate + move.
//
// All marker arithmetic is FP64 and is compiled without FMA contraction, so
// with the reference's evaluation order the results agree with the
// reference engine to the last bit wherever the same libm-class functions are
// not involved (atan2 in Helfrich bending and pow in the contact law are the
// exceptions, agreeing to a few ulp).
#pragma once
#include "common.cuh"

namespace sfg {

struct MarkerBufs {
    double2* pos;
    double2* vel;
    double2* frc;       // membrane + contact force (reference Capsule::forces_)
    double2* dF;        // MDF correction of the current sweep
    double* ds;         // arc length per marker (min-image)
    double* rest_len;
    double* rest_ang;
    double* rest_ds;
    double* prev_len;
    int* mk_cap;        // capsule of each marker
    int* mk_chan;       // channel of each marker
    int* ix0;           // floor(x), floor(y) of the current step
    int* iy0;
    int* valid;         // finite position with its stencil rows near the lattice
    int* pair_count;    // contact pairs visited per marker (bookkeeping)
    double* wx;         // [M][4] phi(x - ix) for ix = ix0-1 .. ix0+2 (this step)
    double* wy;         // [M][4] phi(y - iy) for iy = iy0-1 .. iy0+2
    // multi-direct forcing state of the learned form and its training data
    double2* u0;        // velocity interpolated after the membrane-force spread
    double2* dFsum;     // forcing correction of this step summed over its sweeps
    double2* dFprev;    // previous step's correction before its last sweep
    // force-tile slots of the marker's stencil, this step: [M][2][4] =
    // [row tile (of the first / last stencil row)][stencil column sx]
    int* slot8;
};

// ---------------- Peskin 4-point delta via the 1024-bin table --------------
// reference delta_function.h:44-54 (table built on the host from :18-26)
__device__ __forceinline__ double phi_lut(const double* __restrict__ tbl, double r) {
    double ar = fabs(r);
    if (ar >= 2.0) return 0.0;
    double idx = ar * (1024 * 0.5);
    int i = (int)idx;
    if (i >= 1024) return 0.0;
    double frac = idx - (double)i;
    return tbl[i] * (1.0 - frac) + tbl[i + 1] * frac;
}

__device__ __forceinline__ double2 min_image_d(double2 a, double2 b, double Lx) {
    double2 d = make_double2(a.x - b.x, a.y - b.y);
    if (Lx > 0.0) {
        if (d.x > 0.5 * Lx) d.x -= Lx;
        if (d.x < -0.5 * Lx) d.x += Lx;
    }
    return d;
}
__device__ __forceinline__ double norm_d(double2 a) { return sqrt(a.x * a.x + a.y * a.y); }

__device__ __forceinline__ bool finite2(double2 p) {
    return !(isnan(p.x) || isnan(p.y) || isinf(p.x) || isinf(p.y));
}

}  // namespace sfg
