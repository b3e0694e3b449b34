// itlbm_site.cuh -- per-site device physics of the colour-gradient step.
//
// Two forms of the same site update:
//   * collide_f64: the populations f_R, f_B in FP64, with the reference's arithmetic in the
//     reference's operation order (colisao_comum, Operadores_tensao.cpp:340-373, and the library
//     functions it calls).  Velocity components equal to zero are skipped in the dot products; with
//     round-to-nearest that changes no finite result (adding a signed zero to a non-zero partial sum
//     is exact), and the paired directions c_i, -c_i share one division because negation commutes
//     with rounding.
//   * collide_f32: FP32 storage of e_i = f_i - w_i rho0 (the deviation of the total population) and
//     d_i = f_R,i - f_B,i (the colour difference).  Both are linear in (f_R, f_B), so streaming is
//     unchanged; rho^N = sum d_i / rho, and the BGK update is applied to the deviation so that the
//     pressure keeps FP32 relative precision on rho - rho0 instead of on rho.
#pragma once

#include "itlbm_internal.h"

namespace itlbm {

// ---------------------------------------------------------------------------------------------
// FP64 plain form
// ---------------------------------------------------------------------------------------------

// c_i . (a, b, c) summing the non-zero terms in index order (dot_product, LBM_functions.cpp:865-876)
template <int i, class T>
__device__ __forceinline__ T cdot(T a, T b, T c3) {
    T s = T(0);
    bool first = true;
    auto add = [&](int ci, T v) {
        if (ci == 0) return;
        const T t = ci > 0 ? v : -v;
        s = first ? t : s + t;
        first = false;
    };
    add(cx(i), a);
    add(cy(i), b);
    add(cz(i), c3);
    return s;
}

// Guo source term S_i (source, LBM_functions.cpp:1603-1673):
//   S_i = (1 - 1/2tau) w_i 3 (c_i.F + 3 (c_i.F)(c_i.v) - v.F)
template <int i>
__device__ __forceinline__ double guo_source_f64(double factor, double Fx, double Fy, double Fz,
                                                 double cv, double vF) {
    const double cF = cdot<i>(Fx, Fy, Fz);
    return ((factor * wgt<double>(i)) * 3.0) * ((cF + ((3.0 * cF) * cv)) - vF);
}

// Class-P perturbation (perturbacao, Operadores_tensao.cpp:116-133):
//   f_i += A |g| (w_i (c_i.g)^2 / |g|^2 - B_i), skipped when |g|^2 <= 1e-60 or A == 0.
// The 9 direction pairs share (c_i.g)^2; c_i.g is summed in the reference's order.
__device__ __forceinline__ void perturb_f64(double (&f)[NV], double gmx, double gmy, double gmz,
                                            double A, double B0, double B1, double B2) {
    const double mod2 = gmx * gmx + gmy * gmy + gmz * gmz;
    if (mod2 <= 1.0e-60 || A == 0.0) return;
    const double amod = A * sqrt(mod2);
    const double q0 = 0.0;
    const double qx = ((wgt<double>(1) * gmx) * gmx) / mod2;
    const double qy = ((wgt<double>(3) * gmy) * gmy) / mod2;
    const double qz = ((wgt<double>(5) * gmz) * gmz) / mod2;
    const double s7 = gmx + gmy, s9 = gmx - gmy, s11 = gmx + gmz, s13 = gmx - gmz;
    const double s16 = gmy + gmz, s17 = -gmy + gmz;
    const double d7 = ((wgt<double>(7) * s7) * s7) / mod2;
    const double d9 = ((wgt<double>(9) * s9) * s9) / mod2;
    const double d11 = ((wgt<double>(11) * s11) * s11) / mod2;
    const double d13 = ((wgt<double>(13) * s13) * s13) / mod2;
    const double d16 = ((wgt<double>(16) * s16) * s16) / mod2;
    const double d17 = ((wgt<double>(17) * s17) * s17) / mod2;
    const double Q[NV] = {q0, qx,  qx,  qy,  qy,  qz,  qz,  d7,  d7, d9,
                          d9, d11, d11, d13, d13, d16, d16, d17, d17};
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const double B = cc(i) == 0 ? B0 : (cc(i) == 1 ? B1 : B2);
        f[i] += amod * (Q[i] - B);
    });
}

// Result of the collision of one site: the recolouring split of the post-collision total f_i
// (recolloring, LBM_functions.cpp:1713-1746):
//   f_R,0 = c_R f_0, f_B,0 = c_B f_0; for i >= 1: f_R,i = c_R f_i - t_i, f_B,i = c_B f_i + t_i with
//   t_i = ((beta c_R c_B) w_i rho) cos(phi_i), cos(phi_i) = (c_i . g) / (|g| |c_i|).
struct Recolour64 {
    double cR, cB, frho;   // frho = (beta c_R c_B)... times rho: t_i = (frho_w_i) cos_i
    double fator, rho;
    double k[9];           // cos(phi) of the directions 1, 3, 5, 7, 9, 11, 13, 16, 17
    bool skip;             // rho <= 1e-30: the reference leaves the site unchanged
};

// cos(phi_i) for i = 0..18 from the 9 independent values (pairs i, i+1 are opposite directions)
__device__ __forceinline__ double cos_of(const Recolour64 &r, int i) {
    switch (i) {
        case 1: return r.k[0];  case 2: return -r.k[0];
        case 3: return r.k[1];  case 4: return -r.k[1];
        case 5: return r.k[2];  case 6: return -r.k[2];
        case 7: return r.k[3];  case 8: return -r.k[3];
        case 9: return r.k[4];  case 10: return -r.k[4];
        case 11: return r.k[5]; case 12: return -r.k[5];
        case 13: return r.k[6]; case 14: return -r.k[6];
        case 15: return -r.k[7]; case 16: return r.k[7];
        case 17: return r.k[8]; case 18: return -r.k[8];
        default: return 0.0;
    }
}

// Post-collision colour populations of direction i from the collided total f_i.
template <int i>
__device__ __forceinline__ void split64(const Recolour64 &r, double fi, double &fR, double &fB) {
    if constexpr (i == 0) {
        fR = r.cR * fi;
        fB = r.cB * fi;
    } else {
        constexpr double w = wgt<double>(i);
        const double t = ((r.fator * w) * r.rho) * cos_of(r, i);
        fR = r.cR * fi - t;
        fB = r.cB * fi + t;
    }
}

// Guo forcing, BGK relaxation and class-P perturbation of one site (colisao_comum,
// Operadores_tensao.cpp:340-373, and the library functions it calls).  On entry f holds
// f_i = f_R,i + f_B,i (Operadores_tensao.cpp:360) and rho_R, rho_B the colour sums (density(),
// LBM_functions.cpp:1582-1590, index order).  gm is the mediator momentum (= -grad rho^N), F the force
// (class F only).  On exit f is the post-BGK total and r holds the recolouring split.
template <bool FORCE>
__device__ __forceinline__ void collide_f64(double (&f)[NV], double rho_R, double rho_B, double gmx,
                                            double gmy, double gmz, double Fx, double Fy, double Fz,
                                            const CaseDev &c, Recolour64 &rc) {
    const double rho = rho_R + rho_B;
    rc.skip = !(rho > 1.0e-30);  // Operadores_tensao.cpp:347 (rho <= 1e-30: return)
    if (rc.skip) return;
    const double conc_R = rho_R / rho;
    const double conc_B = 1.0 - conc_R;
    const double mod = sqrt(gmx * gmx + gmy * gmy + gmz * gmz);

    // coll_BGK (Collision_operators.cpp:8-46) with acc = F / rho (class F) or 0 (class P)
    double ax = 0.0, ay = 0.0, az = 0.0;
    if constexpr (FORCE) {
        ax = Fx / rho;
        ay = Fy / rho;
        az = Fz / rho;
    }
    // calcula (LBM_functions.cpp:1100-1171)
    double r = 0.0, mx = 0.0, my = 0.0, mz = 0.0;
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        r = r + f[i];
        if constexpr (cx(i) == 1) mx = mx + f[i];
        if constexpr (cx(i) == -1) mx = mx - f[i];
        if constexpr (cy(i) == 1) my = my + f[i];
        if constexpr (cy(i) == -1) my = my - f[i];
        if constexpr (cz(i) == 1) mz = mz + f[i];
        if constexpr (cz(i) == -1) mz = mz - f[i];
    });
    double vx = 0., vy = 0., vz = 0.;
    if (r != 0.0) {
        const double inv = 1.0 / (r);
        vx = mx * inv;
        vy = my * inv;
        vz = mz * inv;
    }
    const double vxa = vx + 0.5 * ax, vya = vy + 0.5 * ay, vza = vz + 0.5 * az;
    // dist_eq (LBM_functions.cpp:890-945) and source (LBM_functions.cpp:1603-1673)
    const double vquad = (vxa * vxa + vya * vya + vza * vza);
    const double t_vq = (0.5 * vquad) * 3.0;
    const double inv_tau = c.inv_tau;
    double Fxr = 0, Fyr = 0, Fzr = 0, vF = 0, fac3 = 0;
    if constexpr (FORCE) {
        Fxr = ax * r;
        Fyr = ay * r;
        Fzr = az * r;
        vF = Fxr * vxa + Fyr * vya + Fzr * vza;
        fac3 = c.src_factor;
    }
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const double cv = cdot<i>(vxa, vya, vza);
        constexpr double w = wgt<double>(i);
        const double feq = (w * r) * (((1.0 + cv * 3.0) + (((0.5 * cv) * cv) * 3.0) * 3.0) - t_vq);
        const double op = (feq - f[i]) * inv_tau;
        if constexpr (FORCE) {
            f[i] = f[i] + op + guo_source_f64<i>(fac3, Fxr, Fyr, Fzr, cv, vF);
        } else {
            f[i] = f[i] + op;
        }
    });

    // perturbacao (Operadores_tensao.cpp:116-133), class P only; the sign of g is irrelevant
    if constexpr (!FORCE) perturb_f64(f, gmx, gmy, gmz, c.A, c.B0, c.B1, c.B2);

    // recolloring (LBM_functions.cpp:1713-1746) with grad = gm, |c_i| = 1 or sqrt(2)
    rc.cR = conc_R;
    rc.cB = conc_B;
    rc.rho = rho;
    rc.fator = (c.beta * conc_R) * conc_B;
    const double den1 = mod * 1.0;
    const double den2 = mod * sqrt(2.0);
    const bool nz = (mod != 0.0);
    rc.k[0] = nz ? gmx / den1 : 0.0;
    rc.k[1] = nz ? gmy / den1 : 0.0;
    rc.k[2] = nz ? gmz / den1 : 0.0;
    rc.k[3] = nz ? (gmx + gmy) / den2 : 0.0;
    rc.k[4] = nz ? (gmx - gmy) / den2 : 0.0;
    rc.k[5] = nz ? (gmx + gmz) / den2 : 0.0;
    rc.k[6] = nz ? (gmx - gmz) / den2 : 0.0;
    rc.k[7] = nz ? (gmy + gmz) / den2 : 0.0;
    rc.k[8] = nz ? (-gmy + gmz) / den2 : 0.0;
}

// The whole site update on arrays, for the per-site seam entry points.
template <bool FORCE>
__device__ __forceinline__ void colisao_site_f64(double (&fR)[NV], double (&fB)[NV], double gmx,
                                                 double gmy, double gmz, double Fx, double Fy,
                                                 double Fz, const CaseDev &c) {
    double f[NV], sa = 0.0, sb = 0.0;
#pragma unroll
    for (int i = 0; i < NV; i++) sa = sa + fR[i];
#pragma unroll
    for (int i = 0; i < NV; i++) sb = sb + fB[i];
#pragma unroll
    for (int i = 0; i < NV; i++) f[i] = fR[i] + fB[i];
    Recolour64 rc;
    collide_f64<FORCE>(f, sa, sb, gmx, gmy, gmz, Fx, Fy, Fz, c, rc);
    if (rc.skip) return;
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        split64<i>(rc, f[i], fR[i], fB[i]);
    });
}

// The shift s of a direction (or class) with x velocity ex: w (s0 + 3 c.J0 + 4.5 (c.J0)(c.U0)), the
// equilibrium at rho0 and U0 = (u0x, 0) (CaseDev).
template <int ex>
__device__ __forceinline__ float shift_of(const CaseDev::F32Par &p, float w) {
    if constexpr (ex == 0) return w * p.s0;
    else if constexpr (ex > 0) return w * (p.sx + p.j3);
    else return w * (p.sx - p.j3);
}

// ---------------------------------------------------------------------------------------------
// FP32 shifted form: e_i = f_i - s_i, d_i = f_R,i - f_B,i, with s_i the equilibrium at the case's
// reference density rho0 and initial flow velocity U0 (CaseDev::sh); U0 = 0 gives s_i = w_i rho0.
// With P = rho u* (u* the velocity with half the force) and Delta = P - rho0 U0 = sum c_i e_i + F/2,
// the equilibrium minus the shift is, per direction,
//   f_eq,i - s_i = w_i (drho + 3 c.Delta + 4.5 ((c.P)^2 / rho - rho0 (c.U0)^2) - 1.5 (P^2 / rho - rho0 U0^2))
// and each difference of squares is formed from the small deviations only (U0 = (u0x, 0)):
//   (c.P)^2 / rho - rho0 (c.U0)^2 = (c.Delta (2 rho0 c.U0 + c.Delta) - drho rho0 (c.U0)^2) / rho,
//   P^2 / rho - rho0 U0^2        = (Delta.(2 rho0 U0 + Delta) - drho rho0 U0^2) / rho,
// so the stored values and every rounding stay at the scale of the deviations from the initial flow.
// ---------------------------------------------------------------------------------------------
// The FP32 form is evaluated by opposite-direction pairs: c_{2m} = -c_{2m-1} (m = 1..9), so the
// pair shares c.u, the symmetric part of f_eq, c.F, (c.g)^2 and the recolouring term; the rest
// population comes out as a complement.  (The FP64 form keeps the reference's per-direction order.)
template <int i, class T>
__device__ __forceinline__ T cdotp(T a, T b, T c3) {  // c_i . (a, b, c3), non-zero terms only
    T s = T(0);
    if constexpr (cx(i) == 1) s = a;
    if constexpr (cx(i) == -1) s = -a;
    if constexpr (cy(i) == 1) s = (cx(i) == 0) ? b : s + b;
    if constexpr (cy(i) == -1) s = (cx(i) == 0) ? -b : s - b;
    if constexpr (cz(i) == 1) s = (cx(i) == 0 && cy(i) == 0) ? c3 : s + c3;
    if constexpr (cz(i) == -1) s = (cx(i) == 0 && cy(i) == 0) ? -c3 : s - c3;
    return s;
}

// Recolouring split of the FP32 form: d_i = rho^N f_i - fat2 w_i cos(phi_i), f_i = s_i + e_i, with
// fat2 = 2 beta c_R c_B rho = beta (1 - rho^N^2) rho / 2 (c_R - c_B = rho^N) and
// cos(phi_i) = (c_i . g) / (|c_i| |g|); k1 and k2 fold fat2 w_i / (|c_i| |g|) of the two speeds.
// d_0 is the complement D - sum_{i>=1} d_i, formed by the step kernel with FP64 sums.
struct Recolour32 {
    float phi, k1, k2, gx, gy, gz;
    bool skip;
};

// d_i and d_{i+1} of the pair (i, i + 1), i odd, from the post-collision e_i, e_{i+1} and the shifts
// s_i, s_{i+1}.
template <int i>
__device__ __forceinline__ void split32_pair(const Recolour32 &r, float ei, float ej, float si, float sj,
                                             float &di, float &dj) {
    const float K = cdotp<i>(r.gx, r.gy, r.gz) * (cc(i) == 1 ? r.k1 : r.k2);
    di = fmaf(r.phi, si + ei, -K);
    dj = fmaf(r.phi, sj + ej, K);
}

// e_i = f_i - s_i in, post-collision e_i out; drho = sum e_i, D = sum d_i = rho_R - rho_B.
template <bool FORCE>
__device__ __forceinline__ void collide_f32(float (&e)[NV], float drho, float D, float gmx,
                                            float gmy, float gmz, float Fx, float Fy, float Fz,
                                            const CaseDev::F32Par &p, Recolour32 &rc) {
    const float rho0 = p.rho0;
    const float rho = rho0 + drho;
    rc.skip = !(rho > 1.0e-30f);
    if (rc.skip) return;
    const float inv_rho = 1.0f / rho;
    const float phi = D * inv_rho;  // rho^N = (rho_R - rho_B) / rho
    float ax = 0.f, ay = 0.f, az = 0.f;
    if constexpr (FORCE) {
        ax = Fx * inv_rho;
        ay = Fy * inv_rho;
        az = Fz * inv_rho;
    }
    float jx = 0.f, jy = 0.f, jz = 0.f;
    sfor<0, 9>([&](auto M) {
        constexpr int i = 2 * decltype(M)::value + 1;
        const float p = e[i] - e[i + 1];
        if constexpr (cx(i) == 1) jx += p;
        if constexpr (cx(i) == -1) jx -= p;
        if constexpr (cy(i) == 1) jy += p;
        if constexpr (cy(i) == -1) jy -= p;
        if constexpr (cz(i) == 1) jz += p;
        if constexpr (cz(i) == -1) jz -= p;
    });
    // Delta = sum c_i e_i + F / 2 and the velocity u* = (rho0 U0 + Delta) / rho
    const float Dx = FORCE ? fmaf(0.5f, Fx, jx) : jx, Dy = FORCE ? fmaf(0.5f, Fy, jy) : jy;
    const float Dz = FORCE ? fmaf(0.5f, Fz, jz) : jz;
    const float vx = (p.j0x + Dx) * inv_rho, vy = Dy * inv_rho, vz = Dz * inv_rho;
    const float s15 = 1.5f * inv_rho, s45 = 4.5f * inv_rho;
    const float usq15 = s15 * (fmaf(Dx, fmaf(2.0f, p.j0x, Dx), fmaf(Dy, Dy, Dz * Dz)) - drho * p.u0b);
    const float inv_tau = p.inv_tau;
    const float Frx = ax * rho, Fry = ay * rho, Frz = az * rho;
    const float vF = Frx * vx + Fry * vy + Frz * vz;
    const float fac3 = p.fac3;
    // BGK (+ Guo source) of the moving populations, pair (i, j) with c_j = -c_i, d = c_i.Delta:
    //   f_eq - s = w (drho + 4.5 (d (a + d) - drho b) / rho - usq15 +- 3 d),  a = 2 rho0 c.U0, b = rho0 (c.U0)^2
    //   S = 3 (1 - 1/2tau) w (3 (c.F)(c.u) - u.F +- c.F)
    sfor<0, 9>([&](auto M) {
        constexpr int i = 2 * decltype(M)::value + 1;
        constexpr float w = wgt<float>(i);
        const float cD = cdotp<i>(Dx, Dy, Dz);
        float q;  // (c.Delta) (2 rho0 c.U0 + c.Delta) - drho rho0 (c.U0)^2
        if constexpr (cx(i) == 0) q = cD * cD;
        else q = fmaf(cD, fmaf(cx(i) > 0 ? 2.0f : -2.0f, p.j0x, cD), -drho * p.u0b);
        const float sym = w * fmaf(s45, q, drho - usq15);
        const float asym = (3.0f * w) * cD;
        float ei = fmaf((sym + asym) - e[i], inv_tau, e[i]);
        float ej = fmaf((sym - asym) - e[i + 1], inv_tau, e[i + 1]);
        if constexpr (FORCE) {
            const float cu = cdotp<i>(vx, vy, vz);
            const float cF = cdotp<i>(Frx, Fry, Frz);
            const float P = fmaf(3.0f * cF, cu, -vF);
            ei = fmaf(fac3 * w, P + cF, ei);
            ej = fmaf(fac3 * w, P - cF, ej);
        }
        e[i] = ei;
        e[i + 1] = ej;
    });
    const float mod2 = gmx * gmx + gmy * gmy + gmz * gmz;
    const float mod = sqrtf(mod2);
    if constexpr (!FORCE) {
        // class P: f_i += A |g| (w_i (c_i.g)^2 / |g|^2 - B_i), the same for both of a pair
        const float A = p.A;
        if (!(mod2 <= 1.0e-30f || A == 0.0f)) {
            const float inv2 = 1.0f / mod2;
            const float amod = A * mod;
            const float B1 = p.B1, B2 = p.B2;
            sfor<0, 9>([&](auto M) {
                constexpr int i = 2 * decltype(M)::value + 1;
                constexpr float w = wgt<float>(i);
                const float cg = cdotp<i>(gmx, gmy, gmz);
                const float om = amod * fmaf(w * cg, cg * inv2, -(cc(i) == 1 ? B1 : B2));
                e[i] += om;
                e[i + 1] += om;
            });
        }
    }
    // Every site update conserves the mass (sum e_i = drho) exactly; in float arithmetic the weights
    // do not sum to 1 (1 + 1.5e-8), which would bias the sum every step.  The rest population e_0 is
    // therefore the complement.
    {
        float s0 = (e[1] + e[2]) + (e[3] + e[4]), s1 = (e[5] + e[6]) + (e[7] + e[8]);
        float s2 = (e[9] + e[10]) + (e[11] + e[12]), s3 = (e[13] + e[14]) + (e[15] + e[16]);
        e[0] = drho - (((s0 + s1) + (s2 + s3)) + (e[17] + e[18]));
    }
    const float fat2 = 0.5f * p.beta * (1.0f - phi * phi) * rho;
    const float inv_mod = mod > 0.0f ? 1.0f / mod : 0.0f;
    rc.phi = phi;
    rc.k1 = fat2 * wgt<float>(1) * inv_mod;
    rc.k2 = fat2 * wgt<float>(7) * 0.70710678118654752f * inv_mod;
    rc.gx = gmx;
    rc.gy = gmy;
    rc.gz = gmz;
}

// ---------------------------------------------------------------------------------------------
// FP32 fold: the nine in-plane classes of D3Q19 (see itlbm_internal.h), by opposite pairs
// (classes 2m - 1 and 2m, m = 1..4).  Every term of colisao_comum is linear in the populations of
// a class member or depends only on the moments, and members of a class share c . u, c . F and c . g
// (u_z = F_z = g_z = 0), so the class sums follow from class quantities:
//   sum w_i = W_K;  sum B_i = B0 + 2 B1 (K0), B1 + 2 B2 (axes), B2 (diagonals);
//   sum w_i / |c_i| (recolouring) = (1 + 1/sqrt 2) / 18 (axes), 1 / (36 sqrt 2) (diagonals).
// ---------------------------------------------------------------------------------------------
template <int K, class T>
__device__ __forceinline__ T kdot(T a, T b) {  // e_K . (a, b)
    if constexpr (kx(K) == 0) return ky(K) > 0 ? b : -b;
    else if constexpr (ky(K) == 0) return kx(K) > 0 ? a : -a;
    else {
        const T s = kx(K) > 0 ? a : -a;
        return ky(K) > 0 ? s + b : s - b;
    }
}

struct RecolourFold {
    float phi, k1, k2, gx, gy;
    bool skip;
};

// d_K and d_{K+1} of the class pair (K, K + 1), K odd, from the post-collision e_K, e_{K+1} and the
// class shifts s_K, s_{K+1}.
template <int K>
__device__ __forceinline__ void split_fold_pair(const RecolourFold &r, float eK, float eJ, float sK, float sJ,
                                                float &dK, float &dJ) {
    const float A = kdot<K>(r.gx, r.gy) * (kk(K) == 1 ? r.k1 : r.k2);
    dK = fmaf(r.phi, sK + eK, -A);
    dJ = fmaf(r.phi, sJ + eJ, A);
}

// e_K = F_K - s_K of the nine classes in (s_K the class sum of the shifts s_i), post-collision out;
// drho = sum e_K, D = sum d_K.  The equilibrium is formed from the deviations as in collide_f32.
template <bool FORCE>
__device__ __forceinline__ void collide_fold(float (&e)[NK], float drho, float D, float gmx, float gmy,
                                             float Fx, float Fy, const CaseDev::F32Par &p, RecolourFold &rc) {
    const float rho0 = p.rho0;
    const float rho = rho0 + drho;
    rc.skip = !(rho > 1.0e-30f);
    if (rc.skip) return;
    const float inv_rho = 1.0f / rho;
    const float phi = D * inv_rho;
    float ax = 0.f, ay = 0.f;
    if constexpr (FORCE) {
        ax = Fx * inv_rho;
        ay = Fy * inv_rho;
    }
    float jx = 0.f, jy = 0.f;
    sfor<0, 4>([&](auto M) {
        constexpr int K = 2 * decltype(M)::value + 1;
        const float p = e[K] - e[K + 1];
        if constexpr (kx(K) == 1) jx += p;
        if constexpr (kx(K) == -1) jx -= p;
        if constexpr (ky(K) == 1) jy += p;
        if constexpr (ky(K) == -1) jy -= p;
    });
    const float Dx = FORCE ? fmaf(0.5f, Fx, jx) : jx, Dy = FORCE ? fmaf(0.5f, Fy, jy) : jy;
    const float vx = (p.j0x + Dx) * inv_rho, vy = Dy * inv_rho;
    const float s15 = 1.5f * inv_rho, s45 = 4.5f * inv_rho;
    const float usq15 = s15 * (fmaf(Dx, fmaf(2.0f, p.j0x, Dx), Dy * Dy) - drho * p.u0b);
    const float inv_tau = p.inv_tau;
    const float Frx = ax * rho, Fry = ay * rho;
    const float vF = Frx * vx + Fry * vy;
    const float fac3 = p.fac3;
    sfor<0, 4>([&](auto M) {
        constexpr int K = 2 * decltype(M)::value + 1;
        constexpr float W = wk<float>(K);
        const float cD = kdot<K>(Dx, Dy);
        float q;
        if constexpr (kx(K) == 0) q = cD * cD;
        else q = fmaf(cD, fmaf(kx(K) > 0 ? 2.0f : -2.0f, p.j0x, cD), -drho * p.u0b);
        const float sym = W * fmaf(s45, q, drho - usq15);
        const float asym = (3.0f * W) * cD;
        float eK = fmaf((sym + asym) - e[K], inv_tau, e[K]);
        float eJ = fmaf((sym - asym) - e[K + 1], inv_tau, e[K + 1]);
        if constexpr (FORCE) {
            const float cu = kdot<K>(vx, vy);
            const float cF = kdot<K>(Frx, Fry);
            const float P = fmaf(3.0f * cF, cu, -vF);
            eK = fmaf(fac3 * W, P + cF, eK);
            eJ = fmaf(fac3 * W, P - cF, eJ);
        }
        e[K] = eK;
        e[K + 1] = eJ;
    });
    const float mod2 = gmx * gmx + gmy * gmy;
    const float mod = sqrtf(mod2);
    if constexpr (!FORCE) {
        const float A = p.A;
        if (!(mod2 <= 1.0e-30f || A == 0.0f)) {
            const float inv2 = 1.0f / mod2;
            const float amod = A * mod;
            const float Bax = p.Bax, Bdg = p.B2;
            sfor<0, 4>([&](auto M) {
                constexpr int K = 2 * decltype(M)::value + 1;
                constexpr float W = wk<float>(K);
                const float cg = kdot<K>(gmx, gmy);
                const float om = amod * fmaf(W * cg, cg * inv2, -(kk(K) == 1 ? Bax : Bdg));
                e[K] += om;
                e[K + 1] += om;
            });
        }
    }
    e[0] = drho - (((e[1] + e[2]) + (e[3] + e[4])) + ((e[5] + e[6]) + (e[7] + e[8])));
    const float fat2 = 0.5f * p.beta * (1.0f - phi * phi) * rho;
    const float inv_mod = mod > 0.0f ? 1.0f / mod : 0.0f;
    rc.phi = phi;
    rc.k1 = fat2 * ((1.0f + 0.70710678118654752f) / 18.0f) * inv_mod;
    rc.k2 = fat2 * (0.70710678118654752f / 36.0f) * inv_mod;
    rc.gx = gmx;
    rc.gy = gmy;
}

// Mediator momentum sum_K e_K W_K 3 phi(x - e_K) of the fold; the isotropic gradient is its negative.
template <class P>
__device__ __forceinline__ void mediator_grad_fold(P phi, float &gx, float &gy) {
    float ax = 0.f, ay = 0.f;
    sfor<0, 4>([&](auto M) {
        constexpr int K = 2 * decltype(M)::value + 1;
        constexpr float w3 = 3.0f * wk<float>(K);
        const float dphi = w3 * (phi(-kx(K), -ky(K)) - phi(kx(K), ky(K)));
        if constexpr (kx(K) == 1) ax += dphi;
        if constexpr (kx(K) == -1) ax -= dphi;
        if constexpr (ky(K) == 1) ay += dphi;
        if constexpr (ky(K) == -1) ay -= dphi;
    });
    gx = ax;
    gy = ay;
}
// FP32 F1 / F2 auxiliaries by class.  On the slab g_z = 0, so n_z = 0 and the stress has no xz, yz
// components, and the z-moving members of a class read the same in-plane node with opposite c_z: in
// curvature_at and stress_div_at they cancel in pairs, and what is left is the class sum.
//   F1: n = (n_x, n_y) in a[0..1];  kappa = -3 sum_K W_K (e_K . n(x + e_K))
//   F2: (T_xx, T_yy, T_xy) in a[0..2];  F_a = 3 sum_K W_K (T_ax e_Kx + T_ay e_Ky)(x + e_K), F_z = 0
__device__ __forceinline__ void aux_normal_plane(float gx, float gy, float *a) {
    const float m = sqrtf(gx * gx + gy * gy);
    const float inv = (m > 1.0e-12f) ? 1.0f / m : 0.0f;
    a[0] = gx * inv;
    a[1] = gy * inv;
}
__device__ __forceinline__ void aux_stress_plane(float gx, float gy, float sigma, float *a) {
    const float m = sqrtf(gx * gx + gy * gy);
    const float h = 0.5f * sigma;
    const float inv = (m > 1.0e-30f) ? 1.0f / m : 0.0f;
    a[0] = h * (m - gx * gx * inv);
    a[1] = h * (m - gy * gy * inv);
    a[2] = -h * gx * gy * inv;
}
template <class A>
__device__ __forceinline__ float curvature_plane(A aux) {
    float d1 = 0.f, d2 = 0.f;
    sfor<1, NK>([&](auto KC) {
        constexpr int K = decltype(KC)::value;
        const float *v = aux(kx(K), ky(K));
        const float s = kdot<K>(v[0], v[1]);
        if constexpr (kk(K) == 1) d1 += s;
        else d2 += s;
    });
    return -3.0f * (d1 * (1.0f / 9.0f) + d2 * (1.0f / 36.0f));
}
template <class A>
__device__ __forceinline__ void stress_div_plane(A aux, float &Fx, float &Fy) {
    float x1 = 0.f, y1 = 0.f, x2 = 0.f, y2 = 0.f;
    sfor<1, NK>([&](auto KC) {
        constexpr int K = decltype(KC)::value;
        const float *t = aux(kx(K), ky(K));
        const float fx = kdot<K>(t[0], t[2]), fy = kdot<K>(t[2], t[1]);
        if constexpr (kk(K) == 1) {
            x1 += fx;
            y1 += fy;
        } else {
            x2 += fx;
            y2 += fy;
        }
    });
    Fx = 3.0f * (x1 * (1.0f / 9.0f) + x2 * (1.0f / 36.0f));
    Fy = 3.0f * (y1 * (1.0f / 9.0f) + y2 * (1.0f / 36.0f));
}

// F3 chemical potential, lap = 6 sum_K W_K (phi(x + e_K) - phi)
template <class P>
__device__ __forceinline__ float chem_pot_fold(P phi, float kf, float bf) {
    const float ph = phi(0, 0);
    float l1 = 0.f, l2 = 0.f;
    sfor<0, 4>([&](auto M) {
        constexpr int K = 2 * decltype(M)::value + 1;
        const float s = phi(kx(K), ky(K)) + phi(-kx(K), -ky(K));
        if constexpr (kk(K) == 1) l1 += s;
        else l2 += s;
    });
    const float lap = 6.0f * (fmaf(-4.0f, ph, l1) * (1.0f / 9.0f) + fmaf(-4.0f, ph, l2) * (1.0f / 36.0f));
    return 4.0f * bf * ph * (ph * ph - 1.0f) - kf * lap;
}

// ---------------------------------------------------------------------------------------------
// Stencils on a staged phase tile, generic in the real type
// ---------------------------------------------------------------------------------------------

// The stencils below read the staged phase field through an accessor P(dx, dy) = rho^N at
// (x + dx, y + dy), so that every tile shape (a plain 2-D array of its own width) and the per-site
// seam evaluate them with the same arithmetic in the same order.

// Mediator momentum at the node: sum_i c_i * (w_i * (phi(x - c_i) * 3)), the momentum()
// (LBM_functions.cpp:1057-1087) of the mediators after emite_mediadores + propag_site_med
// (LBM_functions.cpp:1287-1337), accumulated in index order.
template <class T, class P>
__device__ __forceinline__ void mediator_grad_at(P phi, T &gx, T &gy, T &gz) {
    T ax = T(0), ay = T(0), az = T(0);
    sfor<0, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T M = wgt<T>(i) * (phi(-cx(i), -cy(i)) * T(3));
        if constexpr (cx(i) == 1) ax = ax + M;
        if constexpr (cx(i) == -1) ax = ax - M;
        if constexpr (cy(i) == 1) ay = ay + M;
        if constexpr (cy(i) == -1) ay = ay - M;
        if constexpr (cz(i) == 1) az = az + M;
        if constexpr (cz(i) == -1) az = az - M;
    });
    gx = ax;
    gy = ay;
    gz = az;
}

// Isotropic gradient 3 sum_{i>=1} w_i c_i phi(x + c_i) (Operadores_tensao.cpp:219-235).
template <class T, class P>
__device__ __forceinline__ void iso_grad_at(P phi, T &gx, T &gy, T &gz) {
    T ax = T(0), ay = T(0), az = T(0);
    sfor<1, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T ph = wgt<T>(i) * phi(cx(i), cy(i));
        if constexpr (cx(i) == 1) ax += ph;
        if constexpr (cx(i) == -1) ax -= ph;
        if constexpr (cy(i) == 1) ay += ph;
        if constexpr (cy(i) == -1) ay -= ph;
        if constexpr (cz(i) == 1) az += ph;
        if constexpr (cz(i) == -1) az -= ph;
    });
    gx = T(3) * ax;
    gy = T(3) * ay;
    gz = T(3) * az;
}

// F3 chemical potential mu = 4 b phi (phi^2 - 1) - k lap phi (Operadores_tensao.cpp:273-287).
template <class T, class P>
__device__ __forceinline__ T chem_pot_at(P phi, T kf, T bf) {
    const T ph = phi(0, 0);
    T lap = T(0);
    sfor<1, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        lap += wgt<T>(i) * (phi(cx(i), cy(i)) - ph);
    });
    lap *= T(6);
    return T(4) * bf * ph * (ph * ph - T(1)) - kf * lap;
}

// the same on a staged 2-D tile at position (px, py)
template <class T, int W_>
__device__ __forceinline__ void mediator_grad(const T (*phi)[W_], int px, int py, T &gx, T &gy,
                                              T &gz) {
    mediator_grad_at<T>([&](int dx, int dy) { return phi[py + dy][px + dx]; }, gx, gy, gz);
}
template <class T, int W_>
__device__ __forceinline__ void iso_grad(const T (*phi)[W_], int px, int py, T &gx, T &gy, T &gz) {
    iso_grad_at<T>([&](int dx, int dy) { return phi[py + dy][px + dx]; }, gx, gy, gz);
}
template <class T, int W_>
__device__ __forceinline__ T chem_pot(const T (*phi)[W_], int px, int py, T kf, T bf) {
    return chem_pot_at<T>([&](int dx, int dy) { return phi[py + dy][px + dx]; }, kf, bf);
}

// F1 unit normal (Operadores_tensao.cpp:251-258) and F2 stress (:259-272) from the gradient.
template <class T>
__device__ __forceinline__ void aux_normal(T gx, T gy, T gz, T *a) {
    const T m = sqrt(gx * gx + gy * gy + gz * gz);
    const T inv = (m > T(1.0e-12)) ? T(1) / m : T(0);
    a[0] = gx * inv;
    a[1] = gy * inv;
    a[2] = gz * inv;
}
template <class T>
__device__ __forceinline__ void aux_stress(T gx, T gy, T gz, T sigma, T *a) {
    const T m = sqrt(gx * gx + gy * gy + gz * gz);
    const T h = T(0.5) * sigma;
    const T inv = (m > T(1.0e-30)) ? T(1) / m : T(0);
    a[0] = h * (m - gx * gx * inv);
    a[1] = h * (m - gy * gy * inv);
    a[2] = h * (m - gz * gz * inv);
    a[3] = -h * gx * gy * inv;
    a[4] = -h * gx * gz * inv;
    a[5] = -h * gy * gz * inv;
}

// F1: kappa = -div_iso(n) (Operadores_tensao.cpp:187-200, :298-305).  A(dx, dy) points at the
// auxiliary components of node (x + dx, y + dy), the normal in components 0..2.
template <class T, class A>
__device__ __forceinline__ T curvature_at(A aux) {
    T d = T(0);
    sfor<1, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T *v = aux(cx(i), cy(i));
        T s = T(0);
        bool first = true;
        auto add = [&](int ci, T val) {
            if (ci == 0) return;
            const T t = ci > 0 ? val : -val;
            s = first ? t : s + t;
            first = false;
        };
        add(cx(i), v[0]);
        add(cy(i), v[1]);
        add(cz(i), v[2]);
        d += wgt<T>(i) * s;
    });
    return -(T(3) * d);
}

// F2: F_a = 3 sum_i w_i T_ab(x + c_i) c_ib (Operadores_tensao.cpp:306-324).
template <class T, class A>
__device__ __forceinline__ void stress_div_at(A aux, T &Fx, T &Fy, T &Fz) {
    T ax = T(0), ay = T(0), az = T(0);
    sfor<1, NV>([&](auto I) {
        constexpr int i = decltype(I)::value;
        const T *t = aux(cx(i), cy(i));
        auto dotc = [&](T a, T b, T c3) {
            T s = T(0);
            bool first = true;
            auto add = [&](int ci, T val) {
                if (ci == 0) return;
                const T u = ci > 0 ? val : -val;
                s = first ? u : s + u;
                first = false;
            };
            add(cx(i), a);
            add(cy(i), b);
            add(cz(i), c3);
            return s;
        };
        const T w = wgt<T>(i);
        ax += w * dotc(t[0], t[3], t[4]);
        ay += w * dotc(t[3], t[1], t[5]);
        az += w * dotc(t[4], t[5], t[2]);
    });
    Fx = T(3) * ax;
    Fy = T(3) * ay;
    Fz = T(3) * az;
}

template <class T, int AS, int W_>
__device__ __forceinline__ T curvature(const T (*aux)[W_][AS], int qx, int qy) {
    return curvature_at<T>([&](int dx, int dy) { return aux[qy + dy][qx + dx]; });
}
template <class T, int AS, int W_>
__device__ __forceinline__ void stress_div(const T (*aux)[W_][AS], int qx, int qy, T &Fx, T &Fy,
                                           T &Fz) {
    stress_div_at<T>([&](int dx, int dy) { return aux[qy + dy][qx + dx]; }, Fx, Fy, Fz);
}

}  // namespace itlbm
