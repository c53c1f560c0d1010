// imhd_physics.cuh -- per-interface and per-cell device functions of the
// isothermal-MHD van Leer + CT step, templated on the arithmetic type.
//
// The arithmetic follows the reference's Fortran expressions operation for
// operation (left-to-right evaluation, x**2 as x*x, SIGN as copysign, MAX/MIN
// as `b > a ? b : a`), so that the FP64 instantiation, compiled with
// --fmad=false and IEEE div/sqrt, reproduces a faithful CPU restatement bit
// for bit.  The FP32 instantiation keeps the same formulas (with FMA
// contraction) and evaluates the Roe / primitive eigenvector normalisation in
// FP64 when the fast, slow and Alfven speeds are nearly degenerate.
//
// Rotated interface states use the reference's qint order
// (vanleer_mod.f90:443-461): 0 rho, 1 m_n, 2 m_t1, 3 m_t2, 4 B_n, 5 B_t1, 6 B_t2.
// Fluxes come back in Fs_2d order (0..6, component 4 is the normal-B flux = 0).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <type_traits>

namespace imhd {

constexpr double kZERO = 1.0e-20;      // vanleer_mod.f90:72
constexpr double kMIN_DENS = 1.0e-20;  // vanleer_mod.f90:73
constexpr double kMC_BETA = 1.01;      // vanleer_mod.f90:77

template <class T>
struct is_exact : std::integral_constant<bool, std::is_same<T, double>::value> {};

template <class T> __device__ __forceinline__ T vmax(T a, T b) { return (b > a) ? b : a; }
template <class T> __device__ __forceinline__ T vmin(T a, T b) { return (b < a) ? b : a; }
template <class T> __device__ __forceinline__ T sgn1(T b) { return copysign(T(1), b); }
template <class T> __device__ __forceinline__ T sq(T x) { return x * x; }

// ---------------------------------------------------------------------------
// FP64 evaluation of the Roe-eigenvector renormalisation (vanleer_mod.f90:
// 2392-2405) from the averaged state, used by the FP32 path near degeneracy.
__device__ __forceinline__ void roe_alphas_fp64(double qa5, double qa6, double qa7, double asqr,
                                                double& af, double& as) {
    double bsqr = qa5 * qa5 + qa6 * qa6 + qa7 * qa7;
    double btsqr = qa6 * qa6 + qa7 * qa7;
    double t1 = asqr + bsqr;
    double t2 = sqrt((asqr - bsqr) * (asqr - bsqr) + 4.0 * asqr * btsqr);
    double cs2 = vmax(0.0, 0.5 * (t1 - t2));
    double cf2 = 0.5 * (t1 + t2);
    double ca2 = qa5 * qa5;
    if (fabs(cf2 - cs2) < kZERO) { af = 1.0; as = 1.0; }
    else if (fabs(cf2 - ca2) < kZERO) { af = 0.0; as = 1.0; }
    else if (fabs(cf2 - asqr) < kZERO) { af = 1.0; as = 0.0; }
    else {
        double t = 1.0 / sqrt(vmax(0.0, cf2 - cs2));
        af = sqrt(vmax(0.0, cf2 - ca2)) * t;
        as = sqrt(vmax(0.0, cf2 - asqr)) * t;
    }
}

// ---------------------------------------------------------------------------
// Roe flux of one interface: compute_roe_avg_state_1d, _eigenvalues_1d,
// _eigenvectors_1d and compute_ROE_fluxes_1d (vanleer_mod.f90:2264-2863).
template <class T>
__device__ __forceinline__ void flux_roe(const T* uL, const T* uR, T cs, T asqr, T* Fo, T& smax) {
    const T ZERO = T(kZERO);
    // arithmetic average (vanleer_mod.f90:2273-2290)
    T rho2 = T(0.5) * (uL[0] + uR[0]);
    T srho = sqrt(rho2);
    T isrho = T(1) / srho;
    T vx2 = T(0.5) * (uL[1] / uL[0] + uR[1] / uR[0]);
    T vy2 = T(0.5) * (uL[2] / uL[0] + uR[2] / uR[0]);
    T vz2 = T(0.5) * (uL[3] / uL[0] + uR[3] / uR[0]);
    T Bx2 = uL[4];
    T By2 = T(0.5) * (uL[5] + uR[5]);
    T Bz2 = T(0.5) * (uL[6] + uR[6]);
    T qa5 = Bx2 * isrho, qa6 = By2 * isrho, qa7 = Bz2 * isrho;
    // eigenvalues and wave speeds (vanleer_mod.f90:2309-2341)
    T bsqr = sq(qa5) + sq(qa6) + sq(qa7);
    T btsqr = sq(qa6) + sq(qa7);
    T tmp1 = asqr + bsqr;
    T tmp2 = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    T css = sqrt(vmax(T(0), T(0.5) * (tmp1 - tmp2)));
    T ca = fabs(qa5);
    T cf = sqrt(T(0.5) * (tmp1 + tmp2));
    T ev[6];
    ev[0] = vx2 - cf; ev[1] = vx2 - ca; ev[2] = vx2 - css;
    ev[3] = vx2 + css; ev[4] = vx2 + ca; ev[5] = vx2 + cf;
    smax = vmax(smax, fabs(vx2) + cf);

    // renormalisation constants (vanleer_mod.f90:2371-2437)
    T bt = sqrt(sq(qa6) + sq(qa7));
    T af, as;
    bool done = false;
    if (!is_exact<T>::value) {
        T cf2 = cf * cf;
        T thr = T(1.0e-3) * cf2;
        if ((cf2 - css * css < thr) || (fabs(cf2 - ca * ca) < thr) || (fabs(cf2 - asqr) < thr)) {
            double afd, asd;
            roe_alphas_fp64((double)qa5, (double)qa6, (double)qa7, (double)asqr, afd, asd);
            af = (T)afd; as = (T)asd;
            done = true;
        }
    }
    if (!done) {
        if (fabs(sq(cf) - sq(css)) < ZERO) { af = T(1); as = T(1); }
        else if (fabs(sq(cf) - sq(ca)) < ZERO) { af = T(0); as = T(1); }
        else if (fabs(sq(cf) - asqr) < ZERO) { af = T(1); as = T(0); }
        else {
            T t = T(1) / sqrt(vmax(T(0), sq(cf) - sq(css)));
            af = sqrt(vmax(T(0), sq(cf) - sq(ca))) * t;
            as = sqrt(vmax(T(0), sq(cf) - asqr)) * t;
        }
    }
    T by, bz;
    if (bt < ZERO) { by = T(1) / sqrt(T(2)); bz = T(1) / sqrt(T(2)); }
    else { T t2 = T(1) / bt; by = qa6 * t2; bz = qa7 * t2; }

    T amc = sq(cs) - sq(ca);
    T signbx = sgn1(qa5);
    T signbt = (fabs(qa6) >= ZERO) ? sgn1(qa6) : sgn1(qa7);
    T sfast = (amc < ZERO) ? signbt : T(1);
    T sslow = (amc > ZERO) ? signbt : T(1);

    // characteristic amplitudes ck = L . dq (vanleer_mod.f90:2566-2742)
    T dq[6];
    dq[0] = uR[0] - uL[0]; dq[1] = uR[1] - uL[1]; dq[2] = uR[2] - uL[2]; dq[3] = uR[3] - uL[3];
    dq[4] = uR[5] - uL[5]; dq[5] = uR[6] - uL[6];
    T it1 = T(1) / (T(2) * (sq(af) * sq(cs) + sq(as) * sq(cf)));
    T it2 = T(1) / (T(2) * (sq(af) * cs * cf + sq(as) * css * ca));
    T ck[6];
    {   // fast waves
        T t1 = it1 * af * sq(cs);
        T t2 = it2 * (-(af * cs * vx2) + as * css * signbx * (by * vy2 + bz * vz2));
        T t3 = it2 * as * css * signbx;
        T t4 = it1 * as * cf * srho;
        T Lm[6], Lp[6];
        Lm[0] = t1 - t2; Lp[0] = t1 + t2;
        Lm[1] = -(it2 * af * cs); Lp[1] = -Lm[1];
        Lm[2] = t3 * by; Lp[2] = -Lm[2];
        Lm[3] = t3 * bz; Lp[3] = -Lm[3];
        Lm[4] = t4 * by; Lp[4] = Lm[4];
        Lm[5] = t4 * bz; Lp[5] = Lm[5];
        if (amc < ZERO) {
#pragma unroll
            for (int m = 0; m < 6; ++m) { Lm[m] = signbt * Lm[m]; Lp[m] = signbt * Lp[m]; }
        }
        ck[0] = dq[0] * Lm[0] + dq[1] * Lm[1] + dq[2] * Lm[2] + dq[3] * Lm[3] + dq[4] * Lm[4] + dq[5] * Lm[5];
        ck[5] = dq[0] * Lp[0] + dq[1] * Lp[1] + dq[2] * Lp[2] + dq[3] * Lp[3] + dq[4] * Lp[4] + dq[5] * Lp[5];
    }
    {   // Alfven waves
        T t1 = T(0.5) * (bz * vy2 - by * vz2) * signbx;
        T t2 = T(0.5) * signbx;
        T t3 = T(0.5) * srho;
        T Lm[6], Lp[6];
        Lm[0] = -t1; Lp[0] = t1;
        Lm[1] = T(0); Lp[1] = T(0);
        Lm[2] = t2 * bz; Lp[2] = -Lm[2];
        Lm[3] = -(t2 * by); Lp[3] = -Lm[3];
        Lm[4] = t3 * bz; Lp[4] = Lm[4];
        Lm[5] = -(t3 * by); Lp[5] = Lm[5];
        ck[1] = dq[0] * Lm[0] + dq[1] * Lm[1] + dq[2] * Lm[2] + dq[3] * Lm[3] + dq[4] * Lm[4] + dq[5] * Lm[5];
        ck[4] = dq[0] * Lp[0] + dq[1] * Lp[1] + dq[2] * Lp[2] + dq[3] * Lp[3] + dq[4] * Lp[4] + dq[5] * Lp[5];
    }
    {   // slow waves
        T t1 = it1 * as * sq(cf);
        T t2 = it2 * (as * ca * vx2 + af * cf * signbx * (by * vy2 + bz * vz2));
        T t3 = it2 * af * cf * signbx;
        T t4 = it1 * af * cf * srho;
        T Lm[6], Lp[6];
        Lm[0] = t1 + t2; Lp[0] = t1 - t2;
        Lm[1] = -(it2 * as * ca); Lp[1] = -Lm[1];
        Lm[2] = -(t3 * by); Lp[2] = -Lm[2];
        Lm[3] = -(t3 * bz); Lp[3] = -Lm[3];
        Lm[4] = -(t4 * by); Lp[4] = Lm[4];
        Lm[5] = -(t4 * bz); Lp[5] = Lm[5];
        if (amc > ZERO) {
#pragma unroll
            for (int m = 0; m < 6; ++m) { Lm[m] = signbt * Lm[m]; Lp[m] = signbt * Lp[m]; }
        }
        ck[2] = dq[0] * Lm[0] + dq[1] * Lm[1] + dq[2] * Lm[2] + dq[3] * Lm[3] + dq[4] * Lm[4] + dq[5] * Lm[5];
        ck[3] = dq[0] * Lp[0] + dq[1] * Lp[1] + dq[2] * Lp[2] + dq[3] * Lp[3] + dq[4] * Lp[4] + dq[5] * Lp[5];
    }

    // right eigenvectors (K98 eq. 2.12, vanleer_mod.f90:2446-2560) and the
    // dissipation sum with Harten's entropy fix (vanleer_mod.f90:2809-2845)
    T R[6][6];   // R[k][m]: component m of wave k
    {
        T t1 = af * vy2, t2 = as * by * qa5, t3 = af * vz2, t4 = as * bz * qa5, t5 = as * cf * isrho;
        R[0][0] = af; R[0][1] = af * ev[0]; R[0][2] = t1 + t2; R[0][3] = t3 + t4; R[0][4] = t5 * by; R[0][5] = t5 * bz;
        R[5][0] = af; R[5][1] = af * ev[5]; R[5][2] = t1 - t2; R[5][3] = t3 - t4; R[5][4] = t5 * by; R[5][5] = t5 * bz;
    }
    R[1][0] = T(0); R[1][1] = T(0); R[1][2] = signbx * bz; R[1][3] = -(signbx * by);
    R[1][4] = isrho * bz; R[1][5] = -(isrho * by);
    R[4][0] = T(0); R[4][1] = T(0); R[4][2] = -(signbx * bz); R[4][3] = signbx * by;
    R[4][4] = isrho * bz; R[4][5] = -(isrho * by);
    {
        T t1 = as * vy2, t2 = af * by * cs * signbx, t3 = as * vz2, t4 = af * bz * cs * signbx;
        T t5 = af * sq(cs) * isrho / cf;
        R[2][0] = as; R[2][1] = as * ev[2]; R[2][2] = t1 - t2; R[2][3] = t3 - t4; R[2][4] = -t5 * by; R[2][5] = -t5 * bz;
        R[3][0] = as; R[3][1] = as * ev[3]; R[3][2] = t1 + t2; R[3][3] = t3 + t4; R[3][4] = -t5 * by; R[3][5] = -t5 * bz;
    }
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        R[0][m] = sfast * R[0][m]; R[5][m] = sfast * R[5][m];
        R[2][m] = sslow * R[2][m]; R[3][m] = sslow * R[3][m];
    }
    T ftvd[6];
#pragma unroll
    for (int m = 0; m < 6; ++m) ftvd[m] = T(0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const bool fixed = (k != 1 && k != 4);      // delta_h = (0.3,0,0.3,0.3,0,0.3)
        T dh = fixed ? T(0.3) : T(0);
        T aev = fabs(ev[k]);
        T betak;
        if (aev >= dh) betak = aev * ck[k];
        else betak = ((aev + sq(dh)) / (T(2) * dh)) * ck[k];
#pragma unroll
        for (int m = 0; m < 6; ++m) ftvd[m] = ftvd[m] - betak * R[k][m];
    }

    // physical fluxes of the two states (vanleer_mod.f90:2765-2801)
    T FLR[2][6];
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        const T* u = s ? uR : uL;
        T rho = u[0];
        T vx = u[1] / rho, vy = u[2] / rho, vz = u[3] / rho;
        T Bx = u[4], By = u[5], Bz = u[6];
        FLR[s][0] = rho * vx;
        FLR[s][1] = rho * (sq(vx) + sq(cs)) + T(0.5) * (sq(By) + sq(Bz) - sq(Bx));
        FLR[s][2] = rho * vx * vy - Bx * By;
        FLR[s][3] = rho * vx * vz - Bx * Bz;
        FLR[s][4] = vx * By - vy * Bx;
        FLR[s][5] = vx * Bz - vz * Bx;
    }
    Fo[0] = T(0.5) * (ftvd[0] + FLR[0][0] + FLR[1][0]);
    Fo[1] = T(0.5) * (ftvd[1] + FLR[0][1] + FLR[1][1]);
    Fo[2] = T(0.5) * (ftvd[2] + FLR[0][2] + FLR[1][2]);
    Fo[3] = T(0.5) * (ftvd[3] + FLR[0][3] + FLR[1][3]);
    Fo[4] = T(0);
    Fo[5] = T(0.5) * (ftvd[4] + FLR[0][4] + FLR[1][4]);
    Fo[6] = T(0.5) * (ftvd[5] + FLR[0][5] + FLR[1][5]);
}

// ---------------------------------------------------------------------------
// Shared pieces of HLLE / HLLD (vanleer_mod.f90:2895-2962, 3020-3086).
template <class T>
__device__ __forceinline__ void phys_flux_cons(const T* u, T vx, T vy, T vz, T asqr, T* F) {
    F[0] = u[1];
    F[1] = u[0] * (sq(vx) + asqr) + T(0.5) * (sq(u[5]) + sq(u[6]) - sq(u[4]));
    F[2] = u[1] * vy - u[4] * u[5];
    F[3] = u[1] * vz - u[4] * u[6];
    F[4] = T(0);
    F[5] = vx * u[5] - vy * u[4];
    F[6] = vx * u[6] - vz * u[4];
}
template <class T>
__device__ __forceinline__ T fast_speed_cons(const T* u, T asqr) {
    T bsqr = (sq(u[4]) + sq(u[5]) + sq(u[6])) / u[0];
    T btsqr = (sq(u[5]) + sq(u[6])) / u[0];
    T tmp1 = asqr + bsqr;
    T tmp2 = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    return sqrt(T(0.5) * (tmp1 + tmp2));
}

// HLLE flux (vanleer_mod.f90:2867-2981)
template <class T>
__device__ __forceinline__ void flux_hlle(const T* uL, const T* uR, T asqr, T* Fo, T& smax) {
    T ua[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) ua[m] = T(0.5) * (uL[m] + uR[m]);
    T vxL = uL[1] / uL[0], vyL = uL[2] / uL[0], vzL = uL[3] / uL[0];
    T vxR = uR[1] / uR[0], vyR = uR[2] / uR[0], vzR = uR[3] / uR[0];
    T FL[7], FR[7];
    phys_flux_cons(uL, vxL, vyL, vzL, asqr, FL);
    phys_flux_cons(uR, vxR, vyR, vzR, asqr, FR);
    T cfL = fast_speed_cons(uL, asqr);
    T cfR = fast_speed_cons(uR, asqr);
    T cfa = fast_speed_cons(ua, asqr);
    T vxa = ua[1] / ua[0];
    T sL = vmin(vmin(vxL - cfL, vxa - cfa), T(0));
    T sR = vmax(vmax(vxR + cfR, vxa + cfa), T(0));
    smax = vmax(vmax(vmax(smax, fabs(vxL) + cfL), fabs(vxR) + cfR), fabs(vxa) + cfa);
    T isRL = T(1) / (sR - sL);
#pragma unroll
    for (int m = 0; m < 7; ++m) Fo[m] = (sR * FL[m] - sL * FR[m] + sR * sL * (uR[m] - uL[m])) * isRL;
}

// HLLD flux, isothermal (Mignone 2007), vanleer_mod.f90:2986-3239
template <class T>
__device__ __forceinline__ void flux_hlld(const T* uL, const T* uR, T asqr, T* Fo, T& smax) {
    const T ZERO = T(kZERO);
    T ua[7];
#pragma unroll
    for (int m = 0; m < 7; ++m) ua[m] = T(0.5) * (uL[m] + uR[m]);
    T Bx = uL[4];
    T vxL = uL[1] / uL[0], vyL = uL[2] / uL[0], vzL = uL[3] / uL[0];
    T vxR = uR[1] / uR[0], vyR = uR[2] / uR[0], vzR = uR[3] / uR[0];
    T FL[7], FR[7];
    phys_flux_cons(uL, vxL, vyL, vzL, asqr, FL);
    phys_flux_cons(uR, vxR, vyR, vzR, asqr, FR);
    T cfL = fast_speed_cons(uL, asqr);
    T cfR = fast_speed_cons(uR, asqr);
    T cfa = fast_speed_cons(ua, asqr);
    T vxa = ua[1] / ua[0];
    T sL = vmin(vmin(vxL - cfL, vxa - cfa), T(0));
    T sR = vmax(vmax(vxR + cfR, vxa + cfa), T(0));
    smax = vmax(vmax(vmax(smax, fabs(vxL) + cfL), fabs(vxR) + cfR), fabs(vxa) + cfa);
    if (sL >= T(0)) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FL[m];
        return;
    }
    if (sR <= T(0)) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FR[m];
        return;
    }
    T isRL = T(1) / (sR - sL);
    T uHLL0 = (sR * uR[0] - sL * uL[0] - FR[0] + FL[0]) * isRL;
    T uHLL1 = (sR * uR[1] - sL * uL[1] - FR[1] + FL[1]) * isRL;
    T FHLL0 = (sR * FL[0] - sL * FR[0] + sR * sL * (uR[0] - uL[0])) * isRL;
    T FHLL1 = (sR * FL[1] - sL * FR[1] + sR * sL * (uR[1] - uL[1])) * isRL;
    T rho_s = uHLL0;
    T momx_s = uHLL1;
    T vx_s = FHLL0 / rho_s;
    T irho_s = T(1) / rho_s;
    T isrho_s = sqrt(irho_s);
    T sLs = vx_s - fabs(Bx) * isrho_s;
    T sRs = vx_s + fabs(Bx) * isrho_s;
    T uLs[7], uRs[7];
    uLs[0] = rho_s; uLs[1] = momx_s;
    if ((fabs(sL - sLs) < ZERO) || (fabs(sL - sRs) < ZERO)) {
#pragma unroll
        for (int m = 2; m < 7; ++m) uLs[m] = uL[m];
    } else {
        T is = T(1) / ((sL - sLs) * (sL - sRs));
        T t1 = Bx * (vx_s - vxL) * is;
        T t2 = (uL[0] * sq(sL - vxL) - sq(Bx)) * irho_s * is;
        uLs[2] = rho_s * vyL - t1 * uL[5];
        uLs[3] = rho_s * vzL - t1 * uL[6];
        uLs[4] = uL[4];
        uLs[5] = t2 * uL[5];
        uLs[6] = t2 * uL[6];
    }
    uRs[0] = rho_s; uRs[1] = momx_s;
    if ((fabs(sR - sLs) < ZERO) || (fabs(sR - sRs) < ZERO)) {
#pragma unroll
        for (int m = 2; m < 7; ++m) uRs[m] = uR[m];
    } else {
        T is = T(1) / ((sR - sLs) * (sR - sRs));
        T t1 = Bx * (vx_s - vxR) * is;
        T t2 = (uR[0] * sq(sR - vxR) - sq(Bx)) * irho_s * is;
        uRs[2] = rho_s * vyR - t1 * uR[5];
        uRs[3] = rho_s * vzR - t1 * uR[6];
        uRs[4] = uR[4];
        uRs[5] = t2 * uR[5];
        uRs[6] = t2 * uR[6];
    }
    if (sLs >= T(0)) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FL[m] + sL * (uLs[m] - uL[m]);
    } else if (sRs <= T(0)) {
#pragma unroll
        for (int m = 0; m < 7; ++m) Fo[m] = FR[m] + sR * (uRs[m] - uR[m]);
    } else {
        T X = sqrt(rho_s) * sgn1(Bx);
        T iX = T(1) / X;
        T uC2 = T(0.5) * (uLs[2] + uRs[2] + X * (uRs[5] - uLs[5]));
        T uC3 = T(0.5) * (uLs[3] + uRs[3] + X * (uRs[6] - uLs[6]));
        T uC5 = T(0.5) * (uLs[5] + uRs[5] + iX * (uRs[2] - uLs[2]));
        T uC6 = T(0.5) * (uLs[6] + uRs[6] + iX * (uRs[3] - uLs[3]));
        Fo[0] = FHLL0;
        Fo[1] = FHLL1;
        Fo[2] = uC2 * vx_s - Bx * uC5;
        Fo[3] = uC3 * vx_s - Bx * uC6;
        Fo[4] = T(0);
        Fo[5] = vx_s * uC5 - (uC2 * Bx) / rho_s;
        Fo[6] = vx_s * uC6 - (uC3 * Bx) / rho_s;
    }
}

template <int SOLVER, class T>
__device__ __forceinline__ void riemann(const T* uL, const T* uR, T cs, T asqr, T* Fo, T& smax) {
    if (SOLVER == 1 || SOLVER == 4) flux_roe(uL, uR, cs, asqr, Fo, smax);   // 4: Roe with protection fluxes
    else if (SOLVER == 2) flux_hlld(uL, uR, asqr, Fo, smax);
    else flux_hlle(uL, uR, asqr, Fo, smax);
}

// ---------------------------------------------------------------------------
// Limited characteristic slope of one cell for PLM (compute_primitive_eigenvectors
// vanleer_mod.f90:941-1141 + the PLM branch of compute_interface_states_char
// :1507-1546).  wm, w0, wp are the rotated primitives (rho, v_n, v_t1, v_t2,
// B_t1, B_t2) of cells i-1, i, i+1; bn is the face field at i+1/2 (wb).
template <class T>
__device__ __forceinline__ T mc_limit(T dL, T dR, T dC) {
    if ((dL * dR) > T(0))
        return sgn1(dC) * vmin(vmin(T(kMC_BETA) * fabs(dL), T(kMC_BETA) * fabs(dR)), fabs(dC));
    return T(0);
}

template <class T>
__device__ __forceinline__ void prim_alphas_fp64(double rho, double bn, double w4, double w5, double asqr,
                                                 double& af, double& as) {
    double rhos = sqrt(rho), irhos = 1.0 / rhos;
    double bx = irhos * bn, by = irhos * w4, bz = irhos * w5;
    double bsqr = bx * bx + by * by + bz * bz;
    double btsqr = by * by + bz * bz;
    double t1 = asqr + bsqr;
    double t2 = sqrt((asqr - bsqr) * (asqr - bsqr) + 4.0 * asqr * btsqr);
    double cs2 = vmax(0.0, 0.5 * (t1 - t2));
    double cf2 = 0.5 * (t1 + t2);
    if (fabs(cf2 - cs2) < kZERO) { af = 1.0; as = 0.0; }
    else {
        af = sqrt(vmax((asqr - cs2) / (cf2 - cs2), 0.0));
        as = sqrt(vmax((cf2 - asqr) / (cf2 - cs2), 0.0));
    }
}

// With PPM the slope is the difference of the MC-limited characteristic
// slopes of cells i+1 and i, both projected on the eigenvectors of cell i
// (the PPM branch :1593-1627); wp2 is w(i+2) and is not read for PLM.
template <class T, bool PPM = false>
__device__ __forceinline__ void plm_char_slope(const T* wm, const T* w0, const T* wp, const T* wp2, T bn, T cs, T asqr,
                                               T* delw) {
    const T ZERO = T(kZERO);
    T rho = w0[0];
    T irho = T(1) / rho;
    T rhos = sqrt(rho);
    T irhos = T(1) / rhos;
    T bx = irhos * bn;
    T by = irhos * w0[4];
    T bz = irhos * w0[5];
    T bsqr = sq(bx) + sq(by) + sq(bz);
    T btsqr = sq(by) + sq(bz);
    T tmp1 = asqr + bsqr;
    T tmp2 = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    T css = sqrt(vmax(T(0), T(0.5) * (tmp1 - tmp2)));
    T cf = sqrt(T(0.5) * (tmp1 + tmp2));
    T af, as;
    bool done = false;
    if (!is_exact<T>::value) {
        T cf2 = cf * cf;
        if (cf2 - css * css < T(1.0e-3) * cf2) {
            double afd, asd;
            prim_alphas_fp64<T>((double)rho, (double)bn, (double)w0[4], (double)w0[5], (double)asqr, afd, asd);
            af = (T)afd; as = (T)asd;
            done = true;
        }
    }
    if (!done) {
        if (fabs(sq(cf) - sq(css)) < ZERO) { af = T(1); as = T(0); }
        else {
            af = sqrt(vmax((asqr - sq(css)) / (sq(cf) - sq(css)), T(0)));
            as = sqrt(vmax((sq(cf) - asqr) / (sq(cf) - sq(css)), T(0)));
        }
    }
    T betay, betaz;
    if (btsqr < ZERO) { betay = T(1) / sqrt(T(2)); betaz = T(1) / sqrt(T(2)); }
    else { betay = by / sqrt(btsqr); betaz = bz / sqrt(btsqr); }
    T S = sgn1(bx);
    T Cff = cf * af;
    T Css = css * as;
    T Qf = cf * af * S;
    T Qs = css * as * S;
    T Af = cs * af * rhos;
    T As = cs * as * rhos;
    T Nf = T(0.5) / asqr;
    T Ns = Nf;

    // left eigenvectors, rows (S08 A22)
    T L[6][6];
    L[0][0] = Nf * af * asqr * irho; L[0][1] = -(Nf * Cff); L[0][2] = Nf * Qs * betay; L[0][3] = Nf * Qs * betaz;
    L[0][4] = Nf * As * betay * irho; L[0][5] = Nf * As * betaz * irho;
    L[1][0] = T(0); L[1][1] = T(0); L[1][2] = -(T(0.5) * betaz); L[1][3] = T(0.5) * betay;
    L[1][4] = -(T(0.5) * betaz * S * irhos); L[1][5] = T(0.5) * betay * S * irhos;
    L[2][0] = Ns * as * asqr * irho; L[2][1] = -(Ns * Css); L[2][2] = -(Ns * Qf * betay); L[2][3] = -(Ns * Qf * betaz);
    L[2][4] = -(Ns * Af * betay * irho); L[2][5] = -(Ns * Af * betaz * irho);
    L[3][0] = Ns * as * asqr * irho; L[3][1] = Ns * Css; L[3][2] = Ns * Qf * betay; L[3][3] = Ns * Qf * betaz;
    L[3][4] = -(Ns * Af * betay * irho); L[3][5] = -(Ns * Af * betaz * irho);
    L[4][0] = T(0); L[4][1] = T(0); L[4][2] = T(0.5) * betaz; L[4][3] = -(T(0.5) * betay);
    L[4][4] = -(T(0.5) * betaz * S * irhos); L[4][5] = T(0.5) * betay * S * irhos;
    L[5][0] = Nf * af * asqr * irho; L[5][1] = Nf * Cff; L[5][2] = -(Nf * Qs * betay); L[5][3] = -(Nf * Qs * betaz);
    L[5][4] = Nf * As * betay * irho; L[5][5] = Nf * As * betaz * irho;

    // project, limit (MC beta) and project back (vanleer_mod.f90:1513-1546)
    T dm[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        T aL, aC, aR;
        if (is_exact<T>::value || (k != 1 && k != 4)) {
            aL = L[k][0] * wm[0] + L[k][1] * wm[1] + L[k][2] * wm[2] + L[k][3] * wm[3] + L[k][4] * wm[4] + L[k][5] * wm[5];
            aC = L[k][0] * w0[0] + L[k][1] * w0[1] + L[k][2] * w0[2] + L[k][3] * w0[3] + L[k][4] * w0[4] + L[k][5] * w0[5];
            aR = L[k][0] * wp[0] + L[k][1] * wp[1] + L[k][2] * wp[2] + L[k][3] * wp[3] + L[k][4] * wp[4] + L[k][5] * wp[5];
        } else {   // rows 2 and 5 have zero rho and v_n entries; skipped in FP32
            aL = L[k][2] * wm[2] + L[k][3] * wm[3] + L[k][4] * wm[4] + L[k][5] * wm[5];
            aC = L[k][2] * w0[2] + L[k][3] * w0[3] + L[k][4] * w0[4] + L[k][5] * w0[5];
            aR = L[k][2] * wp[2] + L[k][3] * wp[3] + L[k][4] * wp[4] + L[k][5] * wp[5];
        }
        if constexpr (PPM) {
            T aR2;
            if (is_exact<T>::value || (k != 1 && k != 4))
                aR2 = L[k][0] * wp2[0] + L[k][1] * wp2[1] + L[k][2] * wp2[2] + L[k][3] * wp2[3] + L[k][4] * wp2[4] +
                      L[k][5] * wp2[5];
            else
                aR2 = L[k][2] * wp2[2] + L[k][3] * wp2[3] + L[k][4] * wp2[4] + L[k][5] * wp2[5];
            T dL1 = aC - aL;
            T dR1 = aR - aC;
            T dC1 = T(0.5) * (dL1 + dR1);
            T dL2 = aR - aC;
            T dR2 = aR2 - aR;
            T dC2 = T(0.5) * (dL2 + dR2);
            T m1 = mc_limit(dL1, dR1, dC1);
            T m2 = mc_limit(dL2, dR2, dC2);
            dm[k] = m2 - m1;
        } else {
            T dL = aC - aL;
            T dR = aR - aC;
            T dC = T(0.5) * (dL + dR);
            dm[k] = mc_limit(dL, dR, dC);
        }
    }
    // right eigenvectors, columns (S08 A12): R(row r, column c)
    T R[6][6];
    R[0][0] = rho * af; R[1][0] = -Cff; R[2][0] = Qs * betay; R[3][0] = Qs * betaz; R[4][0] = As * betay; R[5][0] = As * betaz;
    R[0][1] = T(0); R[1][1] = T(0); R[2][1] = -betaz; R[3][1] = betay; R[4][1] = -betaz * S * rhos; R[5][1] = betay * S * rhos;
    R[0][2] = rho * as; R[1][2] = -Css; R[2][2] = -Qf * betay; R[3][2] = -Qf * betaz; R[4][2] = -Af * betay; R[5][2] = -Af * betaz;
    R[0][3] = rho * as; R[1][3] = Css; R[2][3] = Qf * betay; R[3][3] = Qf * betaz; R[4][3] = -Af * betay; R[5][3] = -Af * betaz;
    R[0][4] = T(0); R[1][4] = T(0); R[2][4] = betaz; R[3][4] = -betay; R[4][4] = -betaz * S * rhos; R[5][4] = betay * S * rhos;
    R[0][5] = rho * af; R[1][5] = Cff; R[2][5] = -Qs * betay; R[3][5] = -Qs * betaz; R[4][5] = As * betay; R[5][5] = As * betaz;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (is_exact<T>::value || k >= 2)
            delw[k] = dm[0] * R[k][0] + dm[1] * R[k][1] + dm[2] * R[k][2] + dm[3] * R[k][3] + dm[4] * R[k][4] + dm[5] * R[k][5];
        else   // rows rho and v_n have zero Alfven entries; skipped in FP32
            delw[k] = dm[0] * R[k][0] + dm[2] * R[k][2] + dm[3] * R[k][3] + dm[5] * R[k][5];
    }
}

// Primitive-variable slopes (compute_interface_states_prim, vanleer_mod.f90:
// 1144-1485), per primitive, no eigenvectors.  PLM (:1161-1179): the MC slope
// SIGN(1,dC) MIN(beta|dL|, beta|dR|, |dC|) with no same-sign test.  PPM
// (:1216-1245): the MC slope with the test (mc_limit; beta MIN(|dL|,|dR|) is
// MIN(beta|dL|, beta|dR|) exactly); what is returned is delw(i) - delw(i+1),
// the operand of the edge formula of :1253-1254, so that ppm_edges<T, true>
// adds sixth times it as the reference does.  wp2 = w(i+2) is read for PPM only.
template <class T>
__device__ __forceinline__ T prim_ppm_limit(T wm, T w0, T wp) {
    const T dL = w0 - wm;
    const T dR = wp - w0;
    const T dC = T(0.5) * (dL + dR);
    return mc_limit(dL, dR, dC);
}
template <class T, bool PPM>
__device__ __forceinline__ void prim_slope(const T* wm, const T* w0, const T* wp, const T* wp2, T* delw) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if constexpr (PPM) {
            delw[k] = prim_ppm_limit(wm[k], w0[k], wp[k]) - prim_ppm_limit(w0[k], wp[k], wp2[k]);
        } else {
            const T dL = w0[k] - wm[k];
            const T dR = wp[k] - w0[k];
            const T dC = T(0.5) * (dL + dR);
            delw[k] = sgn1(dC) * vmin(vmin(T(kMC_BETA) * fabs(dL), T(kMC_BETA) * fabs(dR)), fabs(dC));
        }
    }
}

// Interface states of face i+1/2 from the primitives and slopes of cells i
// and i+1 (vanleer_mod.f90:1552-1584 and the prim->cons step :1799-1814; the
// primitive-variable PLM states of :1183-1207 are the same formulas).
template <class T>
__device__ __forceinline__ void plm_left_state(const T* w, const T* d, T bn, T* q) {
    q[0] = w[0] + T(0.5) * d[0];
    q[1] = w[1] + T(0.5) * d[1];
    q[2] = w[2] + T(0.5) * d[2];
    q[3] = w[3] + T(0.5) * d[3];
    q[4] = bn;
    q[5] = w[4] + T(0.5) * d[4];
    q[6] = w[5] + T(0.5) * d[5];
    q[1] = q[1] * q[0];
    q[2] = q[2] * q[0];
    q[3] = q[3] * q[0];
}
template <class T>
__device__ __forceinline__ void plm_right_state(const T* w, const T* d, T bn, T* q) {
    q[0] = w[0] - T(0.5) * d[0];
    q[1] = w[1] - T(0.5) * d[1];
    q[2] = w[2] - T(0.5) * d[2];
    q[3] = w[3] - T(0.5) * d[3];
    q[4] = bn;
    q[5] = w[4] - T(0.5) * d[4];
    q[6] = w[5] - T(0.5) * d[5];
    q[1] = q[1] * q[0];
    q[2] = q[2] * q[0];
    q[3] = q[3] * q[0];
}

// PPM edge values of cell i (vanleer_mod.f90:1660-1743): the parabola's
// left and right values from the neighbour averages and the slope
// differences delw(i-1) (dm) and delw(i) (d0), then the monotonicity
// constraints (flatten at an extremum, steepen an overshooting edge).
// PRIM: the primitive-variable edges of :1251-1330, where dm and d0 are the
// slope operands of prim_slope<T, true> (added, not subtracted) and an
// extremum flattens to the linear profile w -/+ delw(i)/2 instead of w.
template <class T, bool PRIM = false>
__device__ __forceinline__ void ppm_edges(const T* wm, const T* w0, const T* wp, const T* dm, const T* d0, T* wl,
                                          T* wr) {
    const T sixth = T(1.0 / 6.0);
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        T l, r;
        if constexpr (PRIM) {
            l = T(0.5) * (wm[k] + w0[k]) + sixth * dm[k];
            r = T(0.5) * (w0[k] + wp[k]) + sixth * d0[k];
        } else {
            l = T(0.5) * (wm[k] + w0[k]) - sixth * dm[k];
            r = T(0.5) * (w0[k] + wp[k]) - sixth * d0[k];
        }
        T c = w0[k];
        T tmp1 = (r - c) * (c - l);
        T tmp2 = T(6) * (r - l) * (c - T(0.5) * (l + r));
        T tmp3 = sq(r - l);
        if (tmp1 <= T(0)) {
            if constexpr (PRIM) {
                const T s = prim_ppm_limit(wm[k], w0[k], wp[k]);
                l = c - T(0.5) * s;
                r = c + T(0.5) * s;
            } else {
                l = c;
                r = c;
            }
        } else if (tmp2 > tmp3) {
            l = T(3) * c - T(2) * r;
        } else if (tmp2 < -tmp3) {
            r = T(3) * c - T(2) * l;
        }
        wl[k] = l;
        wr[k] = r;
    }
}
// Conserved interface state of face i+1/2 from a PPM edge (right edge of
// cell i for the left state, left edge of cell i+1 for the right state) and
// the face field (:1750-1778, 1799-1814).
template <class T>
__device__ __forceinline__ void ppm_state(const T* e, T bn, T* q) {
    q[0] = e[0];
    q[1] = e[1];
    q[2] = e[2];
    q[3] = e[3];
    q[4] = bn;
    q[5] = e[4];
    q[6] = e[5];
    q[1] = q[1] * q[0];
    q[2] = q[2] * q[0];
    q[3] = q[3] * q[0];
}

// Fast speed along each axis plus |v| (get_max_speed_vanleer, vanleer_mod.f90:3281-3318).
template <class T>
__device__ __forceinline__ T cell_max_speed(T rho, T mx, T my, T mz, T bxc, T byc, T bzc, T asqr) {
    T isrho = T(1) / sqrt(rho);
    T bx = bxc * isrho, by = byc * isrho, bz = bzc * isrho;
    T btsqr = sq(by) + sq(bz);
    T bsqr = sq(bx) + btsqr;
    T tmp = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    T cfx = sqrt(T(0.5) * (asqr + bsqr + tmp));
    btsqr = sq(bx) + sq(bz);
    bsqr = sq(by) + btsqr;
    tmp = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    T cfy = sqrt(T(0.5) * (asqr + bsqr + tmp));
    btsqr = sq(bx) + sq(by);
    bsqr = sq(bz) + btsqr;
    tmp = sqrt(sq(asqr - bsqr) + T(4) * asqr * btsqr);
    T cfz = sqrt(T(0.5) * (asqr + bsqr + tmp));
    T vx = mx / rho, vy = my / rho, vz = mz / rho;
    T m = T(0);
    m = vmax(m, fabs(vx) + cfx);
    m = vmax(m, fabs(vy) + cfy);
    m = vmax(m, fabs(vz) + cfz);
    return m;
}

}  // namespace imhd
