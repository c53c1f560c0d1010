// imhd_physics_fast.cuh -- FP32 evaluation of the Riemann fluxes and of the
// characteristic PLM slope.
//
// Same mathematics as imhd_physics.cuh (which keeps the reference's
// operation order for the FP64 parity path), rearranged to issue fewer
// instructions:
//  * divisions by a density become one reciprocal and products, 1/sqrt
//    becomes rsqrtf;
//  * the +/- eigenvector pairs of the fast, slow and Alfven families share
//    their terms: L.d is formed as P +/- Q, R.dm from the sums and
//    differences of the paired amplitudes;
//  * the continuity sign flips of the Roe eigenvectors (K98 eq. 2.20) are
//    dropped: they multiply both a left and the matching right eigenvector,
//    so they cancel in the dissipation term.
//  * the eigenvector renormalisation constants come from forms without
//    cancellation: cs^2 = a^2 ca^2 / cf^2, the larger of cf^2 - ca^2 and
//    cf^2 - a^2 as a sum of positive terms and the smaller from their
//    product cf^2 bt^2.  Only near the triple point (cf^2 - cs^2 small) are
//    they evaluated in FP64 with the reference's limiting values.
#pragma once

#include "imhd_physics.cuh"

namespace imhd {

// Roe flux of one interface (vanleer_mod.f90:2264-2863), FP32.
__device__ __forceinline__ void flux_roe_fast(const float* uL, const float* uR, float cs, float asqr, float* Fo,
                                              float& smax) {
    float iL = 1.0f / uL[0], iR = 1.0f / uR[0];
    float vxL = uL[1] * iL, vyL = uL[2] * iL, vzL = uL[3] * iL;
    float vxR = uR[1] * iR, vyR = uR[2] * iR, vzR = uR[3] * iR;
    float rho2 = 0.5f * (uL[0] + uR[0]);
    float isrho = rsqrtf(rho2);
    float srho = rho2 * isrho;
    float vx2 = 0.5f * (vxL + vxR), vy2 = 0.5f * (vyL + vyR), vz2 = 0.5f * (vzL + vzR);
    float Bx = uL[4];
    float qa5 = Bx * isrho;
    float qa6 = 0.5f * (uL[5] + uR[5]) * isrho;
    float qa7 = 0.5f * (uL[6] + uR[6]) * isrho;
    float btsqr = qa6 * qa6 + qa7 * qa7;
    float ca2 = qa5 * qa5;
    float bsqr = ca2 + btsqr;
    float tmp1 = asqr + bsqr;
    float dac = asqr - ca2;
    float dd = dac - btsqr;
    float tmp2 = sqrtf(dd * dd + 4.0f * asqr * btsqr);     // cf^2 - cs^2
    float cf2 = 0.5f * (tmp1 + tmp2);
    float icf = rsqrtf(cf2);
    float ca = fabsf(qa5), cf = cf2 * icf;
    float css = cs * ca * icf;                             // cf^2 cs^2 = a^2 ca^2
    float ev0 = vx2 - cf, ev1 = vx2 - ca, ev2 = vx2 - css, ev3 = vx2 + css, ev4 = vx2 + ca, ev5 = vx2 + cf;
    smax = fmaxf(smax, fabsf(vx2) + cf);

    float af, as;
    if (tmp2 < 1.0e-2f * cf2) {
        double afd, asd;
        roe_alphas_fp64((double)qa5, (double)qa6, (double)qa7, (double)asqr, afd, asd);
        af = (float)afd;
        as = (float)asd;
    } else {
        // af = sqrt(cf^2 - ca^2) / sqrt(cf^2 - cs^2), as = sqrt(cf^2 - a^2) / sqrt(cf^2 - cs^2): the
        // larger radicand is big, the smaller cf^2 bt^2 / big
        float big = 0.5f * (fabsf(dac) + btsqr + tmp2);
        float q = rsqrtf(big * tmp2);
        float cfbt = cf * sqrtf(btsqr);
        af = (dac >= 0.0f ? big : cfbt) * q;
        as = (dac >= 0.0f ? cfbt : big) * q;
    }
    float gy, gz;
    if (btsqr < 1.0e-30f) {
        gy = 0.70710678118654752f;
        gz = 0.70710678118654752f;
    } else {
        float ib = rsqrtf(btsqr);
        gy = qa6 * ib;
        gz = qa7 * ib;
    }
    float signbx = copysignf(1.0f, qa5);

    // characteristic amplitudes (K98 eq. 2.16-2.19, 2.27)
    float dq0 = uR[0] - uL[0], dq1 = uR[1] - uL[1], dq2 = uR[2] - uL[2], dq3 = uR[3] - uL[3];
    float dq4 = uR[5] - uL[5], dq5 = uR[6] - uL[6];
    float af2 = af * af, as2 = as * as;
    float it1 = 0.5f / (af2 * asqr + as2 * cf2);
    float it2 = 0.5f / (af2 * cs * cf + as2 * css * ca);
    float vt = gy * vy2 + gz * vz2;
    float dqt = gy * dq2 + gz * dq3;    // transverse momentum jump along beta
    float dbt = gy * dq4 + gz * dq5;    // transverse field jump along beta
    // fast
    float t1 = it1 * af * asqr;
    float t2 = it2 * (as * css * signbx * vt - af * cs * vx2);
    float t3 = it2 * as * css * signbx;
    float t4 = it1 * as * cf * srho;
    float Pf = dq0 * t1 + t4 * dbt;
    float Qf = t3 * dqt - dq0 * t2 - dq1 * (it2 * af * cs);
    float ck0 = Pf + Qf, ck5 = Pf - Qf;
    // Alfven
    float Ua = 0.5f * signbx * ((gz * dq2 - gy * dq3) - dq0 * (gz * vy2 - gy * vz2));
    float Va = 0.5f * srho * (gz * dq4 - gy * dq5);
    float ck1 = Ua + Va, ck4 = Va - Ua;
    // slow
    float s1 = it1 * as * cf2;
    float s2 = it2 * (as * ca * vx2 + af * cf * signbx * vt);
    float s3 = it2 * af * cf * signbx;
    float s4 = it1 * af * cf * srho;
    float Ps = dq0 * s1 - s4 * dbt;
    float Qs = dq0 * s2 - dq1 * (it2 * as * ca) - s3 * dqt;
    float ck2 = Ps + Qs, ck3 = Ps - Qs;

    // Harten entropy fix, delta = 0.3 on the fast and slow families (vanleer_mod.f90:78, 2829-2833)
    auto harten = [](float ev, float c) {
        float a = fabsf(ev);
        return (a >= 0.3f ? a : (a + 0.09f) * (1.0f / 0.6f)) * c;
    };
    float b0 = harten(ev0, ck0), b5 = harten(ev5, ck5);
    float b2 = harten(ev2, ck2), b3 = harten(ev3, ck3);
    float b1 = fabsf(ev1) * ck1, b4 = fabsf(ev4) * ck4;

    // sum_k beta_k R_k with the right eigenvectors of K98 eq. 2.12
    float sF = b0 + b5, dF = b0 - b5;
    float sA = b1 + b4, dA = b1 - b4;
    float sS = b2 + b3, dS = b3 - b2;
    float t5f = as * cf * isrho;
    float t5s = af * asqr * isrho * icf;
    float dis0 = af * sF + as * sS;
    float dis1 = af * (b0 * ev0 + b5 * ev5) + as * (b2 * ev2 + b3 * ev3);
    float q2 = as * qa5 * dF + af * cs * signbx * dS;      // coefficient of beta in components 2, 3
    float dis2 = vy2 * (af * sF + as * sS) + gy * q2 + signbx * gz * dA;
    float dis3 = vz2 * (af * sF + as * sS) + gz * q2 - signbx * gy * dA;
    float c4 = t5f * sF - t5s * sS;
    float dis4 = gy * c4 + isrho * gz * sA;
    float dis5 = gz * c4 - isrho * gy * sA;

    // physical fluxes (vanleer_mod.f90:2765-2801)
    float hb = 0.5f * (uL[5] * uL[5] + uL[6] * uL[6] - Bx * Bx);
    float hbR = 0.5f * (uR[5] * uR[5] + uR[6] * uR[6] - Bx * Bx);
    float FL0 = uL[1], FR0 = uR[1];
    float FL1 = uL[1] * vxL + uL[0] * asqr + hb;
    float FR1 = uR[1] * vxR + uR[0] * asqr + hbR;
    float FL2 = uL[1] * vyL - Bx * uL[5], FR2 = uR[1] * vyR - Bx * uR[5];
    float FL3 = uL[1] * vzL - Bx * uL[6], FR3 = uR[1] * vzR - Bx * uR[6];
    float FL4 = vxL * uL[5] - vyL * Bx, FR4 = vxR * uR[5] - vyR * Bx;
    float FL5 = vxL * uL[6] - vzL * Bx, FR5 = vxR * uR[6] - vzR * Bx;
    Fo[0] = 0.5f * (FL0 + FR0 - dis0);
    Fo[1] = 0.5f * (FL1 + FR1 - dis1);
    Fo[2] = 0.5f * (FL2 + FR2 - dis2);
    Fo[3] = 0.5f * (FL3 + FR3 - dis3);
    Fo[4] = 0.0f;
    Fo[5] = 0.5f * (FL4 + FR4 - dis4);
    Fo[6] = 0.5f * (FL5 + FR5 - dis5);
}

// Fast magnetosonic speed of a conserved rotated state given 1/rho.
__device__ __forceinline__ float fast_speed_fast(const float* u, float irho, float asqr) {
    float btsqr = (u[5] * u[5] + u[6] * u[6]) * irho;
    float bsqr = u[4] * u[4] * irho + btsqr;
    float tmp1 = asqr + bsqr, dd = asqr - bsqr;
    float tmp2 = sqrtf(dd * dd + 4.0f * asqr * btsqr);
    return sqrtf(0.5f * (tmp1 + tmp2));
}

__device__ __forceinline__ void phys_flux_fast(const float* u, float vx, float vy, float vz, float asqr, float* F) {
    F[0] = u[1];
    F[1] = u[1] * vx + u[0] * asqr + 0.5f * (u[5] * u[5] + u[6] * u[6] - u[4] * u[4]);
    F[2] = u[1] * vy - u[4] * u[5];
    F[3] = u[1] * vz - u[4] * u[6];
    F[4] = 0.0f;
    F[5] = vx * u[5] - vy * u[4];
    F[6] = vx * u[6] - vz * u[4];
}

// HLLE flux (vanleer_mod.f90:2867-2981), FP32.
__device__ __forceinline__ void flux_hlle_fast(const float* uL, const float* uR, float asqr, float* Fo, float& smax) {
    float iL = 1.0f / uL[0], iR = 1.0f / uR[0];
    float vxL = uL[1] * iL, vyL = uL[2] * iL, vzL = uL[3] * iL;
    float vxR = uR[1] * iR, vyR = uR[2] * iR, vzR = uR[3] * iR;
    float ua[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) ua[m] = 0.5f * (uL[m] + uR[m]);
    float ia = 1.0f / ua[0];
    float FL[7], FR[7];
    phys_flux_fast(uL, vxL, vyL, vzL, asqr, FL);
    phys_flux_fast(uR, vxR, vyR, vzR, asqr, FR);
    float cfL = fast_speed_fast(uL, iL, asqr), cfR = fast_speed_fast(uR, iR, asqr), cfa = fast_speed_fast(ua, ia, asqr);
    float vxa = ua[1] * ia;
    float sL = fminf(fminf(vxL - cfL, vxa - cfa), 0.0f);
    float sR = fmaxf(fmaxf(vxR + cfR, vxa + cfa), 0.0f);
    smax = fmaxf(fmaxf(fmaxf(smax, fabsf(vxL) + cfL), fabsf(vxR) + cfR), fabsf(vxa) + cfa);
    float isRL = 1.0f / (sR - sL);
    float sRsL = sR * sL;
#pragma unroll
    for (int m = 0; m < 7; ++m) Fo[m] = (sR * FL[m] - sL * FR[m] + sRsL * (uR[m] - uL[m])) * isRL;
}

// Isothermal HLLD flux (Mignone 2007; vanleer_mod.f90:2986-3239), FP32.
__device__ __forceinline__ void flux_hlld_fast(const float* uL, const float* uR, float asqr, float* Fo, float& smax) {
    const float ZERO = 1.0e-20f;
    float iL = 1.0f / uL[0], iR = 1.0f / uR[0];
    float Bx = uL[4];
    float vxL = uL[1] * iL, vyL = uL[2] * iL, vzL = uL[3] * iL;
    float vxR = uR[1] * iR, vyR = uR[2] * iR, vzR = uR[3] * iR;
    float ua[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) ua[m] = 0.5f * (uL[m] + uR[m]);
    float ia = 1.0f / ua[0];
    float FL[7], FR[7];
    phys_flux_fast(uL, vxL, vyL, vzL, asqr, FL);
    phys_flux_fast(uR, vxR, vyR, vzR, asqr, FR);
    float cfL = fast_speed_fast(uL, iL, asqr), cfR = fast_speed_fast(uR, iR, asqr), cfa = fast_speed_fast(ua, ia, asqr);
    float vxa = ua[1] * ia;
    float sL = fminf(fminf(vxL - cfL, vxa - cfa), 0.0f);
    float sR = fmaxf(fmaxf(vxR + cfR, vxa + cfa), 0.0f);
    smax = fmaxf(fmaxf(fmaxf(smax, fabsf(vxL) + cfL), fabsf(vxR) + cfR), fabsf(vxa) + cfa);
    if (sL >= 0.0f) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FL[m];
        return;
    }
    if (sR <= 0.0f) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FR[m];
        return;
    }
    float isRL = 1.0f / (sR - sL);
    float sRsL = sR * sL;
    float rho_s = (sR * uR[0] - sL * uL[0] - FR[0] + FL[0]) * isRL;
    float momx_s = (sR * uR[1] - sL * uL[1] - FR[1] + FL[1]) * isRL;
    float FHLL0 = (sR * FL[0] - sL * FR[0] + sRsL * (uR[0] - uL[0])) * isRL;
    float FHLL1 = (sR * FL[1] - sL * FR[1] + sRsL * (uR[1] - uL[1])) * isRL;
    float irho_s = 1.0f / rho_s;
    float vx_s = FHLL0 * irho_s;
    float isrho_s = rsqrtf(rho_s);
    float abx = fabsf(Bx) * isrho_s;
    float sLs = vx_s - abx, sRs = vx_s + abx;
    float uLs[7], uRs[7];
    uLs[0] = rho_s; uLs[1] = momx_s;
    if ((fabsf(sL - sLs) < ZERO) || (fabsf(sL - sRs) < ZERO)) {
#pragma unroll
        for (int m = 2; m < 7; ++m) uLs[m] = uL[m];
    } else {
        float is = 1.0f / ((sL - sLs) * (sL - sRs));
        float t1 = Bx * (vx_s - vxL) * is;
        float dv = sL - vxL;
        float t2 = (uL[0] * dv * dv - Bx * Bx) * irho_s * is;
        uLs[2] = rho_s * vyL - t1 * uL[5];
        uLs[3] = rho_s * vzL - t1 * uL[6];
        uLs[4] = uL[4];
        uLs[5] = t2 * uL[5];
        uLs[6] = t2 * uL[6];
    }
    uRs[0] = rho_s; uRs[1] = momx_s;
    if ((fabsf(sR - sLs) < ZERO) || (fabsf(sR - sRs) < ZERO)) {
#pragma unroll
        for (int m = 2; m < 7; ++m) uRs[m] = uR[m];
    } else {
        float is = 1.0f / ((sR - sLs) * (sR - sRs));
        float t1 = Bx * (vx_s - vxR) * is;
        float dv = sR - vxR;
        float t2 = (uR[0] * dv * dv - Bx * Bx) * irho_s * is;
        uRs[2] = rho_s * vyR - t1 * uR[5];
        uRs[3] = rho_s * vzR - t1 * uR[6];
        uRs[4] = uR[4];
        uRs[5] = t2 * uR[5];
        uRs[6] = t2 * uR[6];
    }
    if (sLs >= 0.0f) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FL[m] + sL * (uLs[m] - uL[m]);
    } else if (sRs <= 0.0f) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FR[m] + sR * (uRs[m] - uR[m]);
    } else {
        float srs = rho_s * isrho_s;    // sqrt(rho_s)
        float X = copysignf(srs, Bx);
        float iX = copysignf(isrho_s, Bx);
        float uC2 = 0.5f * (uLs[2] + uRs[2] + X * (uRs[5] - uLs[5]));
        float uC3 = 0.5f * (uLs[3] + uRs[3] + X * (uRs[6] - uLs[6]));
        float uC5 = 0.5f * (uLs[5] + uRs[5] + iX * (uRs[2] - uLs[2]));
        float uC6 = 0.5f * (uLs[6] + uRs[6] + iX * (uRs[3] - uLs[3]));
        Fo[0] = FHLL0;
        Fo[1] = FHLL1;
        Fo[2] = uC2 * vx_s - Bx * uC5;
        Fo[3] = uC3 * vx_s - Bx * uC6;
        Fo[4] = 0.0f;
        Fo[5] = vx_s * uC5 - uC2 * Bx * irho_s;
        Fo[6] = vx_s * uC6 - uC3 * Bx * irho_s;
    }
}

// Limited characteristic slope of one cell (S08 A12/A22, vanleer_mod.f90:
// 941-1141, 1507-1546), FP32.  wm, w0, wp: rotated primitives of cells
// i-1, i, i+1; bn: face field at i+1/2.
template <bool PPM = false>
__device__ __forceinline__ void plm_char_slope_fast(const float* wm, const float* w0, const float* wp,
                                                    const float* wp2, float bn, float cs, float asqr, float* delw) {
    float rho = w0[0];
    float irho = 1.0f / rho;
    float irhos = rsqrtf(rho);
    float rhos = rho * irhos;
    float bx = irhos * bn, by = irhos * w0[4], bz = irhos * w0[5];
    float btsqr = by * by + bz * bz;
    float ca2 = bx * bx;
    float bsqr = ca2 + btsqr;
    float tmp1 = asqr + bsqr;
    float dac = asqr - ca2;
    float dd = dac - btsqr;
    float tmp2 = sqrtf(dd * dd + 4.0f * asqr * btsqr);     // cf^2 - cs^2
    float cf2 = 0.5f * (tmp1 + tmp2);
    float icf = rsqrtf(cf2);
    float cf = cf2 * icf;
    float css = cs * fabsf(bx) * icf;                      // cf^2 cs^2 = a^2 ca^2
    float af, as;
    if (tmp2 < 1.0e-2f * cf2) {
        double afd, asd;
        prim_alphas_fp64<float>((double)rho, (double)bn, (double)w0[4], (double)w0[5], (double)asqr, afd, asd);
        af = (float)afd;
        as = (float)asd;
    } else {
        // af^2 = (a^2 - cs^2) / tmp2 = a^2 (cf^2 - ca^2) / (cf^2 tmp2), as^2 = (cf^2 - a^2) / tmp2; the
        // larger of cf^2 - ca^2 and cf^2 - a^2 is big, the smaller cf^2 bt^2 / big
        float big = 0.5f * (fabsf(dac) + btsqr + tmp2);
        float bt = sqrtf(btsqr);
        if (dac >= 0.0f) {
            float q = rsqrtf(cf2 * tmp2 * big);
            af = cs * big * q;
            as = cf2 * bt * q;
        } else {
            float q = rsqrtf(tmp2 * big);
            af = cs * bt * q;
            as = big * q;
        }
    }
    float gy, gz;
    if (btsqr < 1.0e-30f) {
        gy = 0.70710678118654752f;
        gz = 0.70710678118654752f;
    } else {
        float ib = rsqrtf(btsqr);
        gy = by * ib;
        gz = bz * ib;
    }
    float S = copysignf(1.0f, bx);
    float Nf = 0.5f / asqr;
    // left-eigenvector coefficients (S08 A22)
    float f0 = 0.5f * af * irho, f1 = Nf * cf * af, fq = Nf * css * as * S, fa = Nf * cs * as * irhos;
    float s0 = 0.5f * as * irho, s1 = Nf * css * as, sq_ = Nf * cf * af * S, sa = Nf * cs * af * irhos;
    float hS = 0.5f * S * irhos;
    float dm[6];
    {
        constexpr int NS = PPM ? 3 : 2;   // projected differences: w0-wm, wp-w0 (, wp2-wp)
        float dD[NS][6];
#pragma unroll
        for (int m = 0; m < 6; ++m) {
            dD[0][m] = w0[m] - wm[m];
            dD[1][m] = wp[m] - w0[m];
            if constexpr (PPM) dD[2][m] = wp2[m] - wp[m];
        }
        float aD[NS][6];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const float* d = dD[s];
            float* a = aD[s];
            float dvt = gy * d[2] + gz * d[3];
            float dbt = gy * d[4] + gz * d[5];
            float P = f0 * d[0] + fa * dbt, Q = fq * dvt - f1 * d[1];
            a[0] = P + Q; a[5] = P - Q;
            float P2 = s0 * d[0] - sa * dbt, Q2 = -s1 * d[1] - sq_ * dvt;
            a[2] = P2 + Q2; a[3] = P2 - Q2;
            float U = 0.5f * (gy * d[3] - gz * d[2]), V = hS * (gy * d[5] - gz * d[4]);
            a[1] = U + V; a[4] = V - U;
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            float m1 = mc_limit(aD[0][k], aD[1][k], 0.5f * (aD[0][k] + aD[1][k]));
            if constexpr (PPM) dm[k] = mc_limit(aD[1][k], aD[2][k], 0.5f * (aD[1][k] + aD[2][k])) - m1;
            else dm[k] = m1;
        }
    }
    // right eigenvectors (S08 A12) applied to the limited amplitudes
    float sf = dm[0] + dm[5], df = dm[5] - dm[0];
    float ss = dm[2] + dm[3], ds = dm[3] - dm[2];
    float sA = dm[1] + dm[4], dA = dm[4] - dm[1];
    float Qs = css * as * S, Qf = cf * af * S, As = cs * as * rhos, Af = cs * af * rhos;
    float tq = Qf * ds - Qs * df;
    float ta = As * sf - Af * ss;
    float Srh = S * rhos;
    delw[0] = rho * (af * sf + as * ss);
    delw[1] = cf * af * df + css * as * ds;
    delw[2] = gy * tq + gz * dA;
    delw[3] = gz * tq - gy * dA;
    delw[4] = gy * ta - gz * Srh * sA;
    delw[5] = gz * ta + gy * Srh * sA;
}

}  // namespace imhd

namespace imhd {

// Precision dispatch: the FP64 path keeps the reference's operation order
// (bit parity with the oracle), the FP32 path uses the rearranged forms above.
template <int SOLVER, class T>
__device__ __forceinline__ void riemann_flux(const T* uL, const T* uR, T cs, T asqr, T* Fo, T& smax) {
    if constexpr (std::is_same<T, float>::value) {
        if (SOLVER == 1 || SOLVER == 4) flux_roe_fast(uL, uR, cs, asqr, Fo, smax);
        else if (SOLVER == 2) flux_hlld_fast(uL, uR, asqr, Fo, smax);
        else flux_hlle_fast(uL, uR, asqr, Fo, smax);
    } else {
        riemann<SOLVER>(uL, uR, cs, asqr, Fo, smax);
    }
}

template <class T, bool PPM = false>
__device__ __forceinline__ void char_slope(const T* wm, const T* w0, const T* wp, const T* wp2, T bn, T cs, T asqr,
                                           T* delw) {
    if constexpr (std::is_same<T, float>::value) plm_char_slope_fast<PPM>(wm, w0, wp, wp2, bn, cs, asqr, delw);
    else plm_char_slope<T, PPM>(wm, w0, wp, wp2, bn, cs, asqr, delw);
}

// Slope of a sweep's reconstruction (scheme_recon: bit 0 PPM, bit 1 primitive
// variables): the characteristic slope or the primitive-variable one.
template <class T, int RECON>
__device__ __forceinline__ void recon_slope(const T* wm, const T* w0, const T* wp, const T* wp2, T bn, T cs, T asqr,
                                           T* delw) {
    constexpr bool PPM = (RECON & 1) != 0;
    if constexpr ((RECON & 2) != 0) prim_slope<T, PPM>(wm, w0, wp, wp2, delw);
    else char_slope<T, PPM>(wm, w0, wp, wp2, bn, cs, asqr, delw);
}

}  // namespace imhd
