// collide.cuh -- D2Q9 collision operators with Guo forcing, one cell in registers.
//
// The arithmetic keeps the reference's evaluation order (bgk_collision.cpp:42-85,
// regularized_bgk.cpp:123-180, mrt_collision.cpp:239-322) so that the FP64
// instantiation, compiled without FMA contraction, reproduces the reference
// bit for bit; the FP32 instantiation uses the same formulas in float.
#pragma once
#include "common.cuh"

namespace sfg {

// Moments of one cell in the reference's summation order
// (lattice_field.cpp:220-227): rho = sum f_q, j = sum f_q e_q, q = 0..8.
template <typename R>
__device__ __forceinline__ void cell_moments(const R f[9], R& rho, R& jx, R& jy) {
    rho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    jx = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    jy = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
}

// Moments in the lattice kernels' representation: populations (FP64) or
// deviations d = f - w (FP32 arithmetic: rho = 1 + sum d, j = sum e d).
template <typename R>
__device__ __forceinline__ void lattice_moments(const R c[9], R& rho, R& jx, R& jy) {
    cell_moments(c, rho, jx, jy);
}
template <>
__device__ __forceinline__ void lattice_moments<float>(const float c[9], float& rho, float& jx,
                                                       float& jy) {
    cell_moments(c, rho, jx, jy);
    rho += 1.f;
}

// u = (j + F/2) / rho, zero for rho <= 1e-15 (lattice_field.cpp:229-237).
template <typename R>
__device__ __forceinline__ void cell_velocity(R rho, R jx, R jy, R Gx, R Gy, R& ux, R& uy) {
    if (rho > R(1e-15)) {
        ux = (jx + R(0.5) * Gx) / rho;
        uy = (jy + R(0.5) * Gy) / rho;
    } else {
        ux = R(0);
        uy = R(0);
    }
}
// FP32 form: one correctly rounded reciprocal and two products.
template <>
__device__ __forceinline__ void cell_velocity<float>(float rho, float jx, float jy, float Gx,
                                                     float Gy, float& ux, float& uy) {
    const float inv = rho > 1e-15f ? __frcp_rn(rho) : 0.0f;
    ux = (jx + 0.5f * Gx) * inv;
    uy = (jy + 0.5f * Gy) * inv;
}

template <typename R>
__device__ __forceinline__ void collide_bgk(R f[9], R r, R vx, R vy, R fx, R fy, R om) {
    const R om1 = R(1) - om;
    const R guo = R(1) - R(0.5) * om;
    const R inv_cs2 = R(3), inv_cs4 = R(9);
    const R uu = vx * vx + vy * vy;
    const R uu_term = R(-0.5) * inv_cs2 * uu;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const R ex = R(cx_of(q)), ey = R(cy_of(q));
        const R eu = ex * vx + ey * vy;
        const R w = R(w_of(q));
        R feq = w * r * (R(1) + eu * inv_cs2 + R(0.5) * eu * eu * inv_cs4 + uu_term);
        R tx = (ex - vx) * inv_cs2 + (eu * inv_cs4) * ex;
        R ty = (ey - vy) * inv_cs2 + (eu * inv_cs4) * ey;
        R Fi = guo * w * (tx * fx + ty * fy);
        f[q] = om1 * f[q] + om * feq + Fi;
    }
}

// Equilibrium in the form of reference lattice.h:35-39.
template <typename R>
__device__ __forceinline__ R feq_ref(int q, R rho, R ux, R uy) {
    const R cs2 = R(1.0 / 3.0);
    const R cs4 = cs2 * cs2;
    R eu = R(cx_of(q)) * ux + R(cy_of(q)) * uy;
    R uu = ux * ux + uy * uy;
    return R(w_of(q)) * rho * (R(1) + eu / cs2 + (eu * eu) / (R(2) * cs4) - uu / (R(2) * cs2));
}

// Regularized BGK keeping the first-order non-equilibrium moment.
template <typename R>
__device__ __forceinline__ void collide_regularized(R f[9], R rho, R ux, R uy, R Fx, R Fy, R omega) {
    const R cs2 = R(1.0 / 3.0);
    const R cs4_2 = R(2) * cs2 * cs2;
    R fe[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) fe[q] = feq_ref(q, rho, ux, uy);
    R jx = R(0), jy = R(0), pxx = R(0), pxy = R(0), pyy = R(0);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const R cx = R(cx_of(q)), cy = R(cy_of(q));
        R fneq = f[q] - fe[q];
        jx += fneq * cx;
        jy += fneq * cy;
        pxx += fneq * cx * cx;
        pxy += fneq * cx * cy;
        pyy += fneq * cy * cy;
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const int icx = cx_of(q), icy = cy_of(q);
        const R cx = R(icx), cy = R(icy);
        R Qxx = R(icx * icx) - cs2;
        R Qxy = R(icx * icy);
        R Qyy = R(icy * icy) - cs2;
        R fneq_reg = R(w_of(q)) * ((cx * jx + cy * jy) / cs2 +
                                   (Qxx * pxx + R(2) * Qxy * pxy + Qyy * pyy) / cs4_2);
        R eu = cx * ux + cy * uy;
        R Fi = (R(1) - R(0.5) * omega) * R(w_of(q)) *
               ((cx - ux + eu * cx / cs2) * Fx / cs2 + (cy - uy + eu * cy / cs2) * Fy / cs2);
        f[q] = fe[q] + (R(1) - omega) * fneq_reg + Fi;
    }
}

// D2Q9 MRT (Lallemand-Luo basis) with the Guo source in moment space.
template <typename R>
__device__ __forceinline__ void collide_mrt(R f[9], R r, R vx, R vy, R fx, R fy, R sn, R s1, R s2,
                                            R s4) {
    const R s6 = s4;
    R m0 = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    R m1 = R(-4) * f[0] - f[1] - f[2] - f[3] - f[4] + R(2) * f[5] + R(2) * f[6] + R(2) * f[7] +
           R(2) * f[8];
    R m2 = R(4) * f[0] - R(2) * f[1] - R(2) * f[2] - R(2) * f[3] - R(2) * f[4] + f[5] + f[6] +
           f[7] + f[8];
    R m3 = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    R m4 = R(-2) * f[1] + R(2) * f[3] + f[5] - f[6] - f[7] + f[8];
    R m5 = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    R m6 = R(-2) * f[2] + R(2) * f[4] + f[5] + f[6] - f[7] - f[8];
    R m7 = f[1] - f[2] + f[3] - f[4];
    R m8 = f[5] - f[6] + f[7] - f[8];
    R uu = vx * vx + vy * vy;
    R meq1 = R(-2) * r + R(3) * r * uu;
    R meq2 = r - R(3) * r * uu;
    R meq4 = -r * vx;
    R meq6 = -r * vy;
    R meq7 = r * (vx * vx - vy * vy);
    R meq8 = r * vx * vy;
    R uF = vx * fx + vy * fy;
    R Sb1 = R(6) * uF, Sb2 = R(-6) * uF;
    R Sb3 = fx, Sb4 = -fx, Sb5 = fy, Sb6 = -fy;
    R Sb7 = R(2) * (vx * fx - vy * fy);
    R Sb8 = vx * fy + vy * fx;
    m1 = m1 - s1 * (m1 - meq1) + (R(1) - s1 * R(0.5)) * Sb1;
    m2 = m2 - s2 * (m2 - meq2) + (R(1) - s2 * R(0.5)) * Sb2;
    m3 = m3 + Sb3;
    m4 = m4 - s4 * (m4 - meq4) + (R(1) - s4 * R(0.5)) * Sb4;
    m5 = m5 + Sb5;
    m6 = m6 - s6 * (m6 - meq6) + (R(1) - s6 * R(0.5)) * Sb6;
    m7 = m7 - sn * (m7 - meq7) + (R(1) - sn * R(0.5)) * Sb7;
    m8 = m8 - sn * (m8 - meq8) + (R(1) - sn * R(0.5)) * Sb8;
    const R k9 = R(9), k36 = R(36), k18 = R(18), k6 = R(6), k4 = R(4), k12 = R(12);
    f[0] = m0 / k9 - m1 / k9 + m2 / k9;
    f[1] = m0 / k9 - m1 / k36 - m2 / k18 + m3 / k6 - m4 / k6 + m7 / k4;
    f[2] = m0 / k9 - m1 / k36 - m2 / k18 + m5 / k6 - m6 / k6 - m7 / k4;
    f[3] = m0 / k9 - m1 / k36 - m2 / k18 - m3 / k6 + m4 / k6 + m7 / k4;
    f[4] = m0 / k9 - m1 / k36 - m2 / k18 - m5 / k6 + m6 / k6 - m7 / k4;
    f[5] = m0 / k9 + m1 / k18 + m2 / k36 + m3 / k6 + m4 / k12 + m5 / k6 + m6 / k12 + m8 / k4;
    f[6] = m0 / k9 + m1 / k18 + m2 / k36 - m3 / k6 - m4 / k12 + m5 / k6 + m6 / k12 - m8 / k4;
    f[7] = m0 / k9 + m1 / k18 + m2 / k36 - m3 / k6 - m4 / k12 - m5 / k6 - m6 / k12 + m8 / k4;
    f[8] = m0 / k9 + m1 / k18 + m2 / k36 + m3 / k6 + m4 / k12 - m5 / k6 - m6 / k12 - m8 / k4;
}

// ---------------------------------------------------------------------------
// FP32 forms.  The FP32 path is checked against the FP64 oracle with a
// tolerance, so it uses algebraically equal, division-free expressions
// (1/cs^2 = 3, 1/(2 cs^4) = 4.5, reciprocals of the inverse-transform
// denominators) instead of the reference's evaluation order.
// ---------------------------------------------------------------------------
// FP32-arithmetic forms work on the deviations d = f - w (the lattice
// kernels' representation for FP32 and FP16 storage): the collision reads d
// and writes d, so no value near a weight is ever formed or rounded.

// MRT on deviations: M w = (1, -2, 1, 0, ..., 0), so the conserved moment is
// rho - 1 and the two energy equilibria shift by the rest state:
// e_eq + 2 = -2 (rho - 1) + 3 rho u^2, eps_eq - 1 = (rho - 1) - 3 rho u^2.
template <>
__device__ __forceinline__ void collide_mrt<float>(float f[9], float r, float vx, float vy,
                                                   float fx, float fy, float sn, float s1,
                                                   float s2, float s4) {
    const float m0 = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];  // rho - 1
    const float a = f[1] + f[2] + f[3] + f[4];
    const float d = f[5] + f[6] + f[7] + f[8];
    float m1 = -4.f * f[0] - a + 2.f * d;
    float m2 = 4.f * f[0] - 2.f * a + d;
    const float m3 = f[1] - f[3] + f[5] - f[6] - f[7] + f[8] + fx;   // + Sb3
    float m4 = -2.f * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
    const float m5 = f[2] - f[4] + f[5] + f[6] - f[7] - f[8] + fy;   // + Sb5
    float m6 = -2.f * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
    float m7 = f[1] - f[2] + f[3] - f[4];
    float m8 = f[5] - f[6] + f[7] - f[8];
    const float uu = vx * vx + vy * vy;
    const float uF = vx * fx + vy * fy;
    const float ru3 = 3.f * r * uu;
    m1 = m1 - s1 * (m1 - (-2.f * m0 + ru3)) + (1.f - 0.5f * s1) * (6.f * uF);
    m2 = m2 - s2 * (m2 - (m0 - ru3)) - (1.f - 0.5f * s2) * (6.f * uF);
    m4 = m4 - s4 * (m4 + r * vx) - (1.f - 0.5f * s4) * fx;
    m6 = m6 - s4 * (m6 + r * vy) - (1.f - 0.5f * s4) * fy;
    m7 = m7 - sn * (m7 - r * (vx * vx - vy * vy)) + (1.f - 0.5f * sn) * (2.f * (vx * fx - vy * fy));
    m8 = m8 - sn * (m8 - r * vx * vy) + (1.f - 0.5f * sn) * (vx * fy + vy * fx);
    const float c9 = 1.f / 9.f, c18 = 1.f / 18.f, c36 = 1.f / 36.f, c6 = 1.f / 6.f,
                c12 = 1.f / 12.f;
    const float b0 = c9 * m0;
    const float bA = b0 - c36 * m1 - c18 * m2;   // axis directions
    const float bD = b0 + c18 * m1 + c36 * m2;   // diagonals
    f[0] = c9 * (m0 - m1 + m2);
    f[1] = bA + c6 * (m3 - m4) + 0.25f * m7;
    f[2] = bA + c6 * (m5 - m6) - 0.25f * m7;
    f[3] = bA - c6 * (m3 - m4) + 0.25f * m7;
    f[4] = bA - c6 * (m5 - m6) - 0.25f * m7;
    const float px = c6 * m3 + c12 * m4, py = c6 * m5 + c12 * m6;
    f[5] = bD + px + py + 0.25f * m8;
    f[6] = bD - px + py - 0.25f * m8;
    f[7] = bD - px - py + 0.25f * m8;
    f[8] = bD + px - py - 0.25f * m8;
}

// Regularized BGK on deviations, by opposite direction pairs.  The
// non-equilibrium first moment and stress come from the moments minus their
// values for the
// second-order equilibrium (sum e feq = rho u, sum e e feq = rho/3 I +
// rho u u), and every pair (e, -e) shares the even part of the update
// (equilibrium, stress projection, second-order Guo term) while the odd part
// (3 e.u, 3 e.j_neq, 3 e.F) changes sign.
template <>
__device__ __forceinline__ void collide_regularized<float>(float f[9], float rho, float ux,
                                                           float uy, float Fx, float Fy,
                                                           float omega) {
    // f holds deviations d = f - w: sum_{cx!=0} w = 1/3 and the odd weight
    // moments vanish
    const float* d = f;
    const float drho = d[0] + d[1] + d[2] + d[3] + d[4] + d[5] + d[6] + d[7] + d[8];
    const float jx = d[1] - d[3] + d[5] - d[6] - d[7] + d[8];
    const float jy = d[2] - d[4] + d[5] + d[6] - d[7] - d[8];
    const float sxx = d[1] + d[3] + d[5] + d[6] + d[7] + d[8];
    const float syy = d[2] + d[4] + d[5] + d[6] + d[7] + d[8];
    const float sxy = d[5] - d[6] + d[7] - d[8];
    const float rux = rho * ux, ruy = rho * uy;
    const float jnx = jx - rux, jny = jy - ruy;
    const float dr3 = drho * (1.f / 3.f);
    const float pxx = sxx - dr3 - rux * ux;
    const float pyy = syy - dr3 - ruy * uy;
    const float pxy = sxy - rux * uy;
    const float om1 = 1.f - omega, guo = 1.f - 0.5f * omega;
    const float bm = -1.5f * (ux * ux + uy * uy);
    const float uF3 = 3.f * (ux * Fx + uy * Fy);
    const float trP3 = (pxx + pyy) * (1.f / 3.f);
    const float ane = 4.5f * om1, aj = 3.f * om1, g3 = 3.f * guo, g9 = 9.f * guo;
    f[0] = (4.f / 9.f) * (drho + rho * bm - ane * trP3 - guo * uF3);
    auto pair = [&](int q, int o, float eu, float eF, float ej, float QP, float w) {
        const float E = w * (drho + rho * (bm + 4.5f * eu * eu) + ane * QP + g9 * eu * eF -
                             guo * uF3);
        const float O = w * (3.f * rho * eu + aj * ej + g3 * eF);
        f[q] = E + O;
        f[o] = E - O;
    };
    pair(1, 3, ux, Fx, jnx, pxx - trP3, 1.f / 9.f);
    pair(2, 4, uy, Fy, jny, pyy - trP3, 1.f / 9.f);
    pair(5, 7, ux + uy, Fx + Fy, jnx + jny, pxx + pyy + 2.f * pxy - trP3, 1.f / 36.f);
    pair(6, 8, uy - ux, Fy - Fx, jny - jnx, pxx + pyy - 2.f * pxy - trP3, 1.f / 36.f);
}

// BGK on deviations, by opposite direction pairs:
// d' = (1 - omega) d + omega (feq - w) + F with
// feq - w = w ((rho - 1) + rho (-1.5 u^2 + 4.5 (e.u)^2) + 3 rho e.u).
template <>
__device__ __forceinline__ void collide_bgk<float>(float f[9], float r, float vx, float vy,
                                                   float fx, float fy, float om) {
    const float drho = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    const float om1 = 1.f - om, guo = 1.f - 0.5f * om;
    const float bm = -1.5f * (vx * vx + vy * vy);
    const float uF3 = 3.f * (vx * fx + vy * fy);
    const float g3 = 3.f * guo, g9 = 9.f * guo, orr = om * r;
    f[0] = om1 * f[0] + (4.f / 9.f) * (om * drho + orr * bm - guo * uF3);
    auto pair = [&](int q, int o, float eu, float eF, float w) {
        const float E = w * (om * drho + orr * (bm + 4.5f * eu * eu) + g9 * eu * eF - guo * uF3);
        const float O = w * (3.f * orr * eu + g3 * eF);
        f[q] = om1 * f[q] + (E + O);
        f[o] = om1 * f[o] + (E - O);
    };
    pair(1, 3, vx, fx, 1.f / 9.f);
    pair(2, 4, vy, fy, 1.f / 9.f);
    pair(5, 7, vx + vy, fx + fy, 1.f / 36.f);
    pair(6, 8, vy - vx, fy - fx, 1.f / 36.f);
}

// Passive-scalar BGK collision with the first-order equilibrium
// (advection_diffusion.cpp:137-151): g* = g - w_s (g - w C (1 + 3 e.u)).
template <typename R>
__device__ __forceinline__ void collide_scalar(R g[9], R C, R ux, R uy, R omega_s) {
    const R inv_cs2 = R(3);
#pragma unroll
    for (int q = 0; q < 9; ++q) {
        const R eu = R(cx_of(q)) * ux + R(cy_of(q)) * uy;
        const R geq = R(w_of(q)) * C * (R(1) + eu * inv_cs2);
        g[q] = g[q] - omega_s * (g[q] - geq);
    }
}

}  // namespace sfg
