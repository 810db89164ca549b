// collide.cuh -- D2Q9 collision operators with Guo forcing, one cell in registers.
//
// The arithmetic keeps the reference's evaluation order (bgk_collision.cpp:42-85,
// regularized_bgk.cpp:123-180, mrt_collision.cpp:239-322) so that the FP64
// instantiation, compiled without FMA contraction, reproduces the reference
// bit for bit; the FP32 instantiation uses the same formulas in float.
#pragma once
#include "common.cuh"

namespace sfg {

// ---------------------------------------------------------------------------
// FP32 arithmetic of the lattice kernels, written once for a single cell
// (V = float) and for two cells packed in one register pair (V = F2: the
// sm_100 paired FP32 instructions FADD2 / FMUL2 / FFMA2, which round each
// half exactly like the scalar instruction).  Every operation is explicit
// (no contraction left to the compiler), so the one-cell and the paired
// kernels give bit-identical results.
// ---------------------------------------------------------------------------
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 mk2(float a, float b) {
    F2 r;
    r.v = make_float2(a, b);
    return r;
}
template <typename V>
__device__ __forceinline__ V vc(float a);
template <>
__device__ __forceinline__ float vc<float>(float a) { return a; }
template <>
__device__ __forceinline__ F2 vc<F2>(float a) { return mk2(a, a); }

__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ F2 vadd(F2 a, F2 b) {
    F2 r;
    r.v = __fadd2_rn(a.v, b.v);
    return r;
}
__device__ __forceinline__ F2 vmul(F2 a, F2 b) {
    F2 r;
    r.v = __fmul2_rn(a.v, b.v);
    return r;
}
__device__ __forceinline__ F2 vfma(F2 a, F2 b, F2 c) {
    F2 r;
    r.v = __ffma2_rn(a.v, b.v, c.v);
    return r;
}
// a - b = fma(b, -1, a), rounded once like the scalar subtraction
__device__ __forceinline__ F2 vsub(F2 a, F2 b) { return vfma(b, vc<F2>(-1.f), a); }

// Moments of the deviations d = f - w: rho - 1, j and the second-moment sums
// sxx = sum d cx^2, syy = sum d cy^2, sxy = sum d cx cy, through the
// opposite-direction sums and differences.
template <typename V>
struct DevMoments {
    V drho, jx, jy, sxx, syy, sxy;
};
template <typename V>
__device__ __forceinline__ DevMoments<V> dev_moments(const V d[9]) {
    const V a13 = vadd(d[1], d[3]), m13 = vsub(d[1], d[3]);
    const V a24 = vadd(d[2], d[4]), m24 = vsub(d[2], d[4]);
    const V a57 = vadd(d[5], d[7]), m57 = vsub(d[5], d[7]);
    const V a68 = vadd(d[6], d[8]), m68 = vsub(d[6], d[8]);
    const V sd = vadd(a57, a68);
    DevMoments<V> m;
    m.drho = vadd(vadd(d[0], a13), vadd(a24, sd));
    m.jx = vsub(vadd(m13, m57), m68);
    m.jy = vadd(vadd(m24, m57), m68);
    m.sxx = vadd(a13, sd);
    m.syy = vadd(a24, sd);
    m.sxy = vsub(a57, a68);
    return m;
}

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
    const DevMoments<float> m = dev_moments(c);
    rho = vadd(m.drho, 1.f);
    jx = m.jx;
    jy = m.jy;
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
// FP32 reciprocal of the density: the hardware approximation (relative
// error below 2^-22, no special-case path; rho stays near 1).
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
template <>
__device__ __forceinline__ void cell_velocity<float>(float rho, float jx, float jy, float Gx,
                                                     float Gy, float& ux, float& uy) {
    const float inv = rho > 1e-15f ? rcp_approx(rho) : 0.0f;
    ux = vmul(vfma(0.5f, Gx, jx), inv);
    uy = vmul(vfma(0.5f, Gy, jy), inv);
}
// Two cells: the reciprocal per half, the rest paired.
__device__ __forceinline__ void cell_velocity2(F2 rho, F2 jx, F2 jy, F2 Gx, F2 Gy, F2& ux,
                                               F2& uy) {
    const F2 inv = mk2(rho.v.x > 1e-15f ? rcp_approx(rho.v.x) : 0.0f,
                       rho.v.y > 1e-15f ? rcp_approx(rho.v.y) : 0.0f);
    ux = vmul(vfma(vc<F2>(0.5f), Gx, jx), inv);
    uy = vmul(vfma(vc<F2>(0.5f), Gy, jy), inv);
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
// denominators) instead of the reference's evaluation order.  They work on
// the deviations d = f - w (the lattice kernels' representation for FP32
// and FP16 storage), so no value near a weight is ever formed or rounded,
// and are written for V = float (one cell) and V = F2 (two cells).
// ---------------------------------------------------------------------------

// Per-channel constants, computed in scalar FP32 with explicit rounding so
// both forms see the same values.
template <typename V>
struct RegConst {
    V ane, aj, g3, g9, nguo, nane;
};
template <typename V>
__device__ __forceinline__ RegConst<V> reg_const(float omega) {
    const float om1 = __fsub_rn(1.f, omega), guo = __fmaf_rn(-0.5f, omega, 1.f);
    const float ane = __fmul_rn(4.5f, om1);
    RegConst<V> c;
    c.ane = vc<V>(ane);
    c.nane = vc<V>(-ane);
    c.aj = vc<V>(__fmul_rn(3.f, om1));
    c.g3 = vc<V>(__fmul_rn(3.f, guo));
    c.g9 = vc<V>(__fmul_rn(9.f, guo));
    c.nguo = vc<V>(-guo);
    return c;
}

template <typename V>
struct BgkConst {
    V om, om1, g3, g9, nguo;
};
template <typename V>
__device__ __forceinline__ BgkConst<V> bgk_const(float omega) {
    const float guo = __fmaf_rn(-0.5f, omega, 1.f);
    BgkConst<V> c;
    c.om = vc<V>(omega);
    c.om1 = vc<V>(__fsub_rn(1.f, omega));
    c.g3 = vc<V>(__fmul_rn(3.f, guo));
    c.g9 = vc<V>(__fmul_rn(9.f, guo));
    c.nguo = vc<V>(-guo);
    return c;
}

// MRT rates: sn (stress), s1 (energy), s2 (energy square), s4 (heat flux);
// h = 1 - s/2 the Guo factors.
template <typename V>
struct MrtConst {
    V ns1, h1, ns2, nh2, ns4, nh4, nsn, hn, hn2;
};
template <typename V>
__device__ __forceinline__ MrtConst<V> mrt_const(float sn, float s1, float s2, float s4) {
    const float h1 = __fmaf_rn(-0.5f, s1, 1.f), h2 = __fmaf_rn(-0.5f, s2, 1.f);
    const float h4 = __fmaf_rn(-0.5f, s4, 1.f), hn = __fmaf_rn(-0.5f, sn, 1.f);
    MrtConst<V> c;
    c.ns1 = vc<V>(-s1);
    c.h1 = vc<V>(h1);
    c.ns2 = vc<V>(-s2);
    c.nh2 = vc<V>(-h2);
    c.ns4 = vc<V>(-s4);
    c.nh4 = vc<V>(-h4);
    c.nsn = vc<V>(-sn);
    c.hn = vc<V>(hn);
    c.hn2 = vc<V>(__fmul_rn(2.f, hn));
    return c;
}

// Regularized BGK on deviations, by opposite direction pairs.  The
// non-equilibrium first moment and stress come from the moments minus their
// values for the second-order equilibrium (sum e feq = rho u,
// sum e e feq = rho/3 I + rho u u), and every pair (e, -e) shares the even
// part of the update (equilibrium, stress projection, second-order Guo term)
// while the odd part (3 e.u, 3 e.j_neq, 3 e.F) changes sign.  Sums over d
// use sum_{cx != 0} w = 1/3 and the vanishing odd weight moments.
template <typename V>
__device__ __forceinline__ void reg_collide_v(V d[9], const DevMoments<V>& m, V rho, V ux, V uy,
                                              V Fx, V Fy, const RegConst<V>& c) {
    const V rux = vmul(rho, ux), ruy = vmul(rho, uy);
    const V jnx = vsub(m.jx, rux), jny = vsub(m.jy, ruy);
    const V dr3 = vmul(m.drho, vc<V>(1.f / 3.f));
    const V pxx = vsub(m.sxx, vfma(rux, ux, dr3));
    const V pyy = vsub(m.syy, vfma(ruy, uy, dr3));
    const V pxy = vsub(m.sxy, vmul(rux, uy));
    const V bm = vmul(vfma(ux, ux, vmul(uy, uy)), vc<V>(-1.5f));
    const V uF3 = vmul(vfma(ux, Fx, vmul(uy, Fy)), vc<V>(3.f));
    const V sP = vadd(pxx, pyy);
    const V trP3 = vmul(sP, vc<V>(1.f / 3.f));
    const V C0 = vfma(c.nguo, uF3, vfma(rho, bm, m.drho));
    d[0] = vmul(vc<V>(4.f / 9.f), vfma(c.nane, trP3, C0));
    const V r45 = vmul(rho, vc<V>(4.5f)), r3 = vmul(rho, vc<V>(3.f));
    auto pair = [&](int q, int o, V eu, V eF, V ej, V QP, float w) {
        const V E = vmul(vc<V>(w), vfma(c.ane, QP, vfma(eu, vfma(r45, eu, vmul(c.g9, eF)), C0)));
        const V O = vmul(vc<V>(w), vfma(r3, eu, vfma(c.aj, ej, vmul(c.g3, eF))));
        d[q] = vadd(E, O);
        d[o] = vsub(E, O);
    };
    pair(1, 3, ux, Fx, jnx, vsub(pxx, trP3), 1.f / 9.f);
    pair(2, 4, uy, Fy, jny, vsub(pyy, trP3), 1.f / 9.f);
    pair(5, 7, vadd(ux, uy), vadd(Fx, Fy), vadd(jnx, jny),
         vsub(vfma(vc<V>(2.f), pxy, sP), trP3), 1.f / 36.f);
    pair(6, 8, vsub(uy, ux), vsub(Fy, Fx), vsub(jny, jnx),
         vsub(vfma(vc<V>(-2.f), pxy, sP), trP3), 1.f / 36.f);
}

// BGK on deviations, by opposite direction pairs:
// d' = (1 - omega) d + omega (feq - w) + F with
// feq - w = w ((rho - 1) + rho (-1.5 u^2 + 4.5 (e.u)^2) + 3 rho e.u).
template <typename V>
__device__ __forceinline__ void bgk_collide_v(V d[9], V drho, V rho, V ux, V uy, V Fx, V Fy,
                                              const BgkConst<V>& c) {
    const V bm = vmul(vfma(ux, ux, vmul(uy, uy)), vc<V>(-1.5f));
    const V uF3 = vmul(vfma(ux, Fx, vmul(uy, Fy)), vc<V>(3.f));
    const V orr = vmul(c.om, rho);
    const V C0 = vfma(c.nguo, uF3, vfma(orr, bm, vmul(c.om, drho)));
    d[0] = vfma(c.om1, d[0], vmul(vc<V>(4.f / 9.f), C0));
    const V o45 = vmul(orr, vc<V>(4.5f)), o3 = vmul(orr, vc<V>(3.f));
    auto pair = [&](int q, int o, V eu, V eF, float w) {
        const V E = vmul(vc<V>(w), vfma(eu, vfma(o45, eu, vmul(c.g9, eF)), C0));
        const V O = vmul(vc<V>(w), vfma(o3, eu, vmul(c.g3, eF)));
        d[q] = vfma(c.om1, d[q], vadd(E, O));
        d[o] = vfma(c.om1, d[o], vsub(E, O));
    };
    pair(1, 3, ux, Fx, 1.f / 9.f);
    pair(2, 4, uy, Fy, 1.f / 9.f);
    pair(5, 7, vadd(ux, uy), vadd(Fx, Fy), 1.f / 36.f);
    pair(6, 8, vsub(uy, ux), vsub(Fy, Fx), 1.f / 36.f);
}

// MRT on deviations: M w = (1, -2, 1, 0, ..., 0), so the conserved moment is
// rho - 1 and the two energy equilibria shift by the rest state:
// e_eq + 2 = -2 (rho - 1) + 3 rho u^2, eps_eq - 1 = (rho - 1) - 3 rho u^2.
template <typename V>
__device__ __forceinline__ void mrt_collide_v(V d[9], V rho, V vx, V vy, V fx, V fy,
                                              const MrtConst<V>& c) {
    const V a13 = vadd(d[1], d[3]), m13 = vsub(d[1], d[3]);
    const V a24 = vadd(d[2], d[4]), m24 = vsub(d[2], d[4]);
    const V a57 = vadd(d[5], d[7]), m57 = vsub(d[5], d[7]);
    const V a68 = vadd(d[6], d[8]), m68 = vsub(d[6], d[8]);
    const V sd = vadd(a57, a68), sa = vadd(a13, a24);
    const V m0 = vadd(vadd(d[0], a13), vadd(a24, sd));          // rho - 1
    const V jx = vsub(vadd(m13, m57), m68), jy = vadd(vadd(m24, m57), m68);
    V m1 = vsub(vfma(vc<V>(2.f), sd, vmul(vc<V>(-4.f), d[0])), sa);
    V m2 = vadd(vfma(vc<V>(-2.f), sa, vmul(vc<V>(4.f), d[0])), sd);
    const V m3 = vadd(jx, fx);                                   // + Sb3
    V m4 = vfma(vc<V>(-3.f), m13, jx);
    const V m5 = vadd(jy, fy);                                   // + Sb5
    V m6 = vfma(vc<V>(-3.f), m24, jy);
    V m7 = vsub(a13, a24);
    V m8 = vsub(a57, a68);
    const V uu = vfma(vx, vx, vmul(vy, vy));
    const V uF6 = vmul(vfma(vx, fx, vmul(vy, fy)), vc<V>(6.f));
    const V ru3 = vmul(vmul(rho, vc<V>(3.f)), uu);
    m1 = vfma(c.h1, uF6, vfma(c.ns1, vsub(m1, vfma(vc<V>(-2.f), m0, ru3)), m1));
    m2 = vfma(c.nh2, uF6, vfma(c.ns2, vsub(m2, vsub(m0, ru3)), m2));
    m4 = vfma(c.nh4, fx, vfma(c.ns4, vfma(rho, vx, m4), m4));
    m6 = vfma(c.nh4, fy, vfma(c.ns4, vfma(rho, vy, m6), m6));
    const V A = vsub(vmul(vx, vx), vmul(vy, vy));
    const V B = vsub(vmul(vx, fx), vmul(vy, fy));
    m7 = vfma(c.hn2, B, vfma(c.nsn, vsub(m7, vmul(rho, A)), m7));
    const V Cxy = vmul(vx, vy);
    const V D = vfma(vx, fy, vmul(vy, fx));
    m8 = vfma(c.hn, D, vfma(c.nsn, vsub(m8, vmul(rho, Cxy)), m8));
    const float c9 = 1.f / 9.f, c18 = 1.f / 18.f, c36 = 1.f / 36.f, c6 = 1.f / 6.f,
                c12 = 1.f / 12.f;
    const V b0 = vmul(vc<V>(c9), m0);
    const V bA = vfma(vc<V>(-c18), m2, vfma(vc<V>(-c36), m1, b0));   // axis directions
    const V bD = vfma(vc<V>(c36), m2, vfma(vc<V>(c18), m1, b0));     // diagonals
    d[0] = vmul(vc<V>(c9), vadd(vsub(m0, m1), m2));
    const V t1 = vmul(vc<V>(c6), vsub(m3, m4)), t2 = vmul(vc<V>(c6), vsub(m5, m6));
    const V q7 = vmul(vc<V>(0.25f), m7);
    const V bAp = vadd(bA, q7), bAm = vsub(bA, q7);
    d[1] = vadd(bAp, t1);
    d[3] = vsub(bAp, t1);
    d[2] = vadd(bAm, t2);
    d[4] = vsub(bAm, t2);
    const V px = vfma(vc<V>(c12), m4, vmul(vc<V>(c6), m3));
    const V py = vfma(vc<V>(c12), m6, vmul(vc<V>(c6), m5));
    const V q8 = vmul(vc<V>(0.25f), m8);
    const V bDp = vadd(bD, q8), bDm = vsub(bD, q8);
    const V spp = vadd(px, py), smp = vsub(py, px);
    d[5] = vadd(bDp, spp);
    d[7] = vsub(bDp, spp);
    d[6] = vadd(bDm, smp);
    d[8] = vsub(bDm, smp);
}

template <>
__device__ __forceinline__ void collide_mrt<float>(float f[9], float r, float vx, float vy,
                                                   float fx, float fy, float sn, float s1,
                                                   float s2, float s4) {
    mrt_collide_v(f, r, vx, vy, fx, fy, mrt_const<float>(sn, s1, s2, s4));
}

template <>
__device__ __forceinline__ void collide_regularized<float>(float f[9], float rho, float ux,
                                                           float uy, float Fx, float Fy,
                                                           float omega) {
    const DevMoments<float> m = dev_moments(f);
    reg_collide_v(f, m, rho, ux, uy, Fx, Fy, reg_const<float>(omega));
}

template <>
__device__ __forceinline__ void collide_bgk<float>(float f[9], float r, float vx, float vy,
                                                   float fx, float fy, float om) {
    const DevMoments<float> m = dev_moments(f);
    bgk_collide_v(f, m.drho, r, vx, vy, fx, fy, bgk_const<float>(om));
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
