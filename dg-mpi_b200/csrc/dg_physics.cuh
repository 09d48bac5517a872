// dg_physics.cuh -- pointwise 3D Euler physics shared by the host C++ side and
// the CUDA kernels: pressure, wave speed, interior flux, Lax-Friedrichs and
// HLLC numerical fluxes, initial conditions / exact solutions.  Operation
// order follows the reference's functions so that a face flux computed here
// rounds like the reference's; citations are relative to the reference root.
#pragma once
#include <cmath>
#include <math.h>

#ifdef __CUDACC__
#define DG_HD __host__ __device__ __forceinline__
#else
#define DG_HD inline
#endif

namespace dgp {

constexpr double kPi = 3.14159265358979323846;

// The flux functions are templates on the arithmetic type T: double on the
// FP64 path (operation order identical to the reference's), float on the
// mixed-precision path.  Literals are written as T(...) so that the float
// instantiation stays in FP32.

// EulerFcnType::get_pressure<3>, src/physics/euler/functions.cpp:10-23
template <typename T>
DG_HD T pressure(T gamma, const T* U)
{
    const T rKE = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
    return (gamma - T(1.0)) * (U[4] - T(0.5) * rKE);
}

// EulerFcnType::get_maxwavespeed<3>, functions.cpp:25-40
template <typename T>
DG_HD T max_wave_speed(T gamma, const T* U)
{
    const T rho1 = T(1.) / U[0];
    const T sqrtrKE = sqrt(U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) * rho1;
    return sqrtrKE + sqrt(gamma * pressure(gamma, U) * rho1);
}

// EulerFcnType::conv_flux_interior<3>, functions.cpp:64-91; F[j*5+s]
template <typename T>
DG_HD void interior_flux(T gamma, const T* U, T* F)
{
    const T r1 = T(1.) / U[0];
    const T ru = U[1], rv = U[2], rw = U[3], rE = U[4];
    const T P = pressure(gamma, U);
    F[0] = ru;
    F[1] = ru * ru * r1 + P;
    F[2] = ru * rv * r1;
    F[3] = ru * rw * r1;
    F[4] = (rE + P) * ru * r1;
    F[5] = rv;
    F[6] = rv * ru * r1;
    F[7] = rv * rv * r1 + P;
    F[8] = rv * rw * r1;
    F[9] = (rE + P) * rv * r1;
    F[10] = rw;
    F[11] = rw * ru * r1;
    F[12] = rw * rv * r1;
    F[13] = rw * rw * r1 + P;
    F[14] = (rE + P) * rw * r1;
}

// BaseConvNumFluxType::compute_flux_laxfriedrichs<3>, base/functions.cpp:33-89.
// N is the unnormalised normal of the left element (its length carries the
// surface Jacobian).
template <typename T>
DG_HD void flux_lax_friedrichs(T gamma, const T* UL, const T* UR, const T* N, T* F)
{
    T n_mag = T(0.0);
    for (int d = 0; d < 3; ++d) n_mag += N[d] * N[d];
    n_mag = sqrt(n_mag);
    T n_hat[3];
    for (int d = 0; d < 3; ++d) n_hat[d] = N[d] / n_mag;
    T Fq[15], FqL[5] = {T(0), T(0), T(0), T(0), T(0)}, FqR[5] = {T(0), T(0), T(0), T(0), T(0)};
    interior_flux(gamma, UL, Fq);
    for (int s = 0; s < 5; ++s)
        for (int d = 0; d < 3; ++d) FqL[s] += Fq[s + d * 5] * n_hat[d];
    interior_flux(gamma, UR, Fq);
    for (int s = 0; s < 5; ++s)
        for (int d = 0; d < 3; ++d) FqR[s] += Fq[s + d * 5] * n_hat[d];
    T a = max_wave_speed(gamma, UL);
    const T aR = max_wave_speed(gamma, UR);
    if (aR > a) a = aR;
    for (int s = 0; s < 5; ++s) F[s] = n_mag * (T(0.5) * (FqL[s] + FqR[s]) - T(0.5) * a * (UR[s] - UL[s]));
}

// The interior flux with one reciprocal of the density: P = (gamma-1)(rE -
// |m|^2 r1 / 2) instead of the reference's division of |m|^2 by rho (the same
// quantity, rounded differently); returns P for the positivity check.
//
// SHIFT: the state's energy is stored relative to a constant E_ref
// (U[4] = rE - E_ref, so that FP32 keeps its digits for the fluctuation when
// rE is large, as at low Mach).  P is then P - (gamma-1) E_ref: the constant
// part of the pressure is left out of the momentum fluxes -- a constant flux
// has zero weak divergence (the volume and face quadratures integrate it
// exactly, so the two terms cancel) -- and the energy flux adds it back,
// (rE + P) u = (U[4] + P + hr) u with hr = gamma E_ref.
template <typename T, bool SHIFT = false>
DG_HD T interior_flux_r1(T gamma, const T* U, T* F, T hr = T(0))
{
    const T r1 = T(1.) / U[0];
    const T ru = U[1], rv = U[2], rw = U[3], rE = U[4];
    const T P = (gamma - T(1.0)) * (rE - T(0.5) * ((ru * ru + rv * rv + rw * rw) * r1));
    const T u = ru * r1, v = rv * r1, w = rw * r1, H = SHIFT ? rE + P + hr : rE + P;
    F[0] = ru;
    F[1] = ru * u + P;
    F[2] = rv * u;
    F[3] = rw * u;
    F[4] = H * u;
    F[5] = rv;
    F[6] = ru * v;
    F[7] = rv * v + P;
    F[8] = rw * v;
    F[9] = H * v;
    F[10] = rw;
    F[11] = ru * w;
    F[12] = rv * w;
    F[13] = rw * w + P;
    F[14] = H * w;
    return P;
}

// One side of a face for the Lax-Friedrichs flux: the normal flux F(U).n_hat
// = m (m.n_hat)/rho + P n_hat, (rE + P)(m.n_hat)/rho, and the wave speed
// |m|/rho + sqrt(gamma P / rho) of get_maxwavespeed, with one reciprocal.
// SHIFT as for interior_flux_r1, with pref = (gamma-1) E_ref restoring the
// full pressure in the wave speed.
template <typename T, bool SHIFT = false>
DG_HD T lf_side(T gamma, const T* U, const T* n_hat, T* Fn, T hr = T(0), T pref = T(0))
{
    const T r1 = T(1.) / U[0];
    const T m2 = U[1] * U[1] + U[2] * U[2] + U[3] * U[3];
    const T P = (gamma - T(1.0)) * (U[4] - T(0.5) * (m2 * r1));
    const T mn = U[1] * n_hat[0] + U[2] * n_hat[1] + U[3] * n_hat[2];
    const T vn = mn * r1;
    Fn[0] = mn;
    Fn[1] = U[1] * vn + P * n_hat[0];
    Fn[2] = U[2] * vn + P * n_hat[1];
    Fn[3] = U[3] * vn + P * n_hat[2];
    Fn[4] = (SHIFT ? U[4] + P + hr : U[4] + P) * vn;
    return sqrt(m2) * r1 + sqrt(gamma * (SHIFT ? P + pref : P) * r1);
}

// Lax-Friedrichs of the stage kernel: compute_flux_laxfriedrichs with the
// face's |N| and N/|N| precomputed and lf_side for each state.
template <typename T, bool SHIFT = false>
DG_HD void flux_lax_friedrichs_fast(T gamma, const T* UL, const T* UR, const T* n_hat, T n_mag, T* F, T hr = T(0),
                                    T pref = T(0))
{
    T FnL[5], FnR[5];
    const T aL = lf_side<T, SHIFT>(gamma, UL, n_hat, FnL, hr, pref);
    const T aR = lf_side<T, SHIFT>(gamma, UR, n_hat, FnR, hr, pref);
    const T a = aR > aL ? aR : aL;
    for (int s = 0; s < 5; ++s) F[s] = n_mag * (T(0.5) * (FnL[s] + FnR[s]) - T(0.5) * a * (UR[s] - UL[s]));
}

// Lax-Friedrichs with the face's normal data precomputed (it is constant on a
// face of an affine element): n_mag = |N| and n_hat = N / n_mag, evaluated
// once on the host by the formulas of flux_lax_friedrichs.
template <typename T>
DG_HD void flux_lax_friedrichs_n(T gamma, const T* UL, const T* UR, const T* n_hat, T n_mag, T* F)
{
    T Fq[15], FqL[5] = {T(0), T(0), T(0), T(0), T(0)}, FqR[5] = {T(0), T(0), T(0), T(0), T(0)};
    interior_flux(gamma, UL, Fq);
    for (int s = 0; s < 5; ++s)
        for (int d = 0; d < 3; ++d) FqL[s] += Fq[s + d * 5] * n_hat[d];
    interior_flux(gamma, UR, Fq);
    for (int s = 0; s < 5; ++s)
        for (int d = 0; d < 3; ++d) FqR[s] += Fq[s + d * 5] * n_hat[d];
    T a = max_wave_speed(gamma, UL);
    const T aR = max_wave_speed(gamma, UR);
    if (aR > a) a = aR;
    for (int s = 0; s < 5; ++s) F[s] = n_mag * (T(0.5) * (FqL[s] + FqR[s]) - T(0.5) * a * (UR[s] - UL[s]));
}

// EulerConvNumFluxType::compute_flux_hllc<3>, functions.cpp:298-399.
// Returns false on the reference's assert branch (no valid wave ordering,
// e.g. NaN input); F is zeroed then.
template <typename T>
DG_HD bool flux_hllc_n(T gam, const T* UL, const T* UR, const T* n, T djac, T* F);

template <typename T>
DG_HD bool flux_hllc(T gam, const T* UL, const T* UR, const T* N, T* F)
{
    const T djac = sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
    const T djac1 = T(1.) / djac;
    const T n[3] = {N[0] * djac1, N[1] * djac1, N[2] * djac1};
    return flux_hllc_n(gam, UL, UR, n, djac, F);
}

// HLLC with the face's unit normal n = N * (1/|N|) and djac = |N| precomputed
// by the same operations as in flux_hllc.
template <typename T>
DG_HD bool flux_hllc_n(T gam, const T* UL, const T* UR, const T* n, T djac, T* F)
{
    const T rhoL = UL[0], rhoL1 = T(1.) / rhoL;
    const T unL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) * rhoL1;
    const T PL = pressure(gam, UL);
    const T aL = sqrt(gam * PL * rhoL1);
    const T rhoR = UR[0], rhoR1 = T(1.) / rhoR;
    const T unR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) * rhoR1;
    const T PR = pressure(gam, UR);
    const T aR = sqrt(gam * PR * rhoR1);
    const T rAvg = T(0.5) * (rhoL + rhoR);
    const T aAvg = T(0.5) * (aL + aR);
    const T pStar = fmax(T(0.), T(0.5) * (PL + PR - (unR - unL) * rAvg * aAvg));
    T qL = T(1.0), qR = T(1.0);
    if (pStar / PL > T(1.)) qL = sqrt(T(1.) + (gam + T(1.)) / (T(2.) * gam) * (pStar / PL - T(1.)));
    if (pStar / PR > T(1.)) qR = sqrt(T(1.) + (gam + T(1.)) / (T(2.) * gam) * (pStar / PR - T(1.)));
    const T sL = unL - aL * qL;
    const T sR = unR + aR * qR;
    const T sStar = (PR - PL + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR)) /
                    (rhoL * (sL - unL) - rhoR * (sR - unR));
    if (sL >= T(0.)) {
        F[0] = djac * rhoL * unL;
        for (int i = 0; i < 3; ++i) F[1 + i] = djac * (UL[1 + i] * unL + PL * n[i]);
        F[4] = djac * ((UL[4] + PL) * unL);
    } else if (sR <= T(0.)) {
        F[0] = djac * rhoR * unR;
        for (int i = 0; i < 3; ++i) F[1 + i] = djac * (UR[1 + i] * unR + PR * n[i]);
        F[4] = djac * (UR[4] + PR) * unR;
    } else if ((sL < T(0.)) && (sStar >= T(0.))) {
        const T c = (sL - unL) / (sL - sStar);
        const T f1 = sStar - unL;
        const T f2 = sStar + PL / (rhoL * (sL - unL));
        F[0] = djac * (rhoL * unL + rhoL * sL * (c - T(1.)));
        for (int i = 0; i < 3; ++i)
            F[1 + i] = djac * (UL[1 + i] * unL + PL * n[i] + sL * (UL[1 + i] * (c - T(1.)) + rhoL * c * f1 * n[i]));
        F[4] = djac * ((UL[4] + PL) * unL + sL * (UL[4] * (c - T(1.)) + rhoL * c * f1 * f2));
    } else if ((sStar < T(0.)) && (sR > T(0.))) {
        const T c = (sR - unR) / (sR - sStar);
        const T f1 = sStar - unR;
        const T f2 = sStar + PR / (rhoR * (sR - unR));
        F[0] = djac * (rhoR * unR + rhoR * sR * (c - T(1.)));
        for (int i = 0; i < 3; ++i)
            F[1 + i] = djac * (UR[1 + i] * unR + PR * n[i] + sR * (UR[1 + i] * (c - T(1.)) + rhoR * c * f1 * n[i]));
        F[4] = djac * ((UR[4] + PR) * unR + sR * (UR[4] * (c - T(1.)) + rhoR * c * f1 * f2));
    } else {
        for (int s = 0; s < 5; ++s) F[s] = T(0.0);
        return false;
    }
    return true;
}

// HLLC of flux_hllc_n on states whose energy is stored relative to a constant
// (U[4] = rE - eref), for the FP32 residual.  The pressure enters in its
// shifted form P' = P - pref, pref = (gamma-1) eref, wherever only differences
// of pressures or the momentum fluxes need it: the PVRS estimate and sStar use
// P'R - P'L, the compression test pStar > P_K becomes p'Star > P'_K, and the
// momentum fluxes carry P' n (the constant pref n is left out, as in
// interior_flux_r1: its volume and face terms cancel).  The full pressure
// P' + pref enters only the sound speeds, the shock factor's denominator and
// the energy fluxes, where FP32's relative rounding is harmless.  So the
// momenta never see the rounding of the large energy at low Mach.  In exact
// arithmetic this is flux_hllc_n with pref n subtracted from the momenta.
template <typename T>
DG_HD bool flux_hllc_shift(T gam, const T* UL, const T* UR, const T* n, T djac, T eref, T* F)
{
    const T pref = (gam - T(1.)) * eref;
    const T rhoL = UL[0], rhoL1 = T(1.) / rhoL;
    const T unL = (UL[1] * n[0] + UL[2] * n[1] + UL[3] * n[2]) * rhoL1;
    const T PsL = pressure(gam, UL);  // shifted
    const T PL = PsL + pref;
    const T aL = sqrt(gam * PL * rhoL1);
    const T rhoR = UR[0], rhoR1 = T(1.) / rhoR;
    const T unR = (UR[1] * n[0] + UR[2] * n[1] + UR[3] * n[2]) * rhoR1;
    const T PsR = pressure(gam, UR);
    const T PR = PsR + pref;
    const T aR = sqrt(gam * PR * rhoR1);
    const T rAvg = T(0.5) * (rhoL + rhoR);
    const T aAvg = T(0.5) * (aL + aR);
    // shifted PVRS estimate, clamped where the full estimate is negative
    T psStar = T(0.5) * (PsL + PsR - (unR - unL) * rAvg * aAvg);
    if (psStar + pref < T(0.)) psStar = -pref;
    const T dL = psStar - PsL, dR = psStar - PsR;  // pStar - P_K
    T qL = T(1.0), qR = T(1.0);
    if (dL > T(0.)) qL = sqrt(T(1.) + (gam + T(1.)) / (T(2.) * gam) * (dL / PL));
    if (dR > T(0.)) qR = sqrt(T(1.) + (gam + T(1.)) / (T(2.) * gam) * (dR / PR));
    const T sL = unL - aL * qL;
    const T sR = unR + aR * qR;
    const T sStar = (PsR - PsL + rhoL * unL * (sL - unL) - rhoR * unR * (sR - unR)) /
                    (rhoL * (sL - unL) - rhoR * (sR - unR));
    const T hr = gam * eref;  // rE + P = U[4] + P' + gamma eref
    if (sL >= T(0.)) {
        F[0] = djac * rhoL * unL;
        for (int i = 0; i < 3; ++i) F[1 + i] = djac * (UL[1 + i] * unL + PsL * n[i]);
        F[4] = djac * ((UL[4] + PsL + hr) * unL);
    } else if (sR <= T(0.)) {
        F[0] = djac * rhoR * unR;
        for (int i = 0; i < 3; ++i) F[1 + i] = djac * (UR[1 + i] * unR + PsR * n[i]);
        F[4] = djac * ((UR[4] + PsR + hr) * unR);
    } else if ((sL < T(0.)) && (sStar >= T(0.))) {
        const T f1 = sStar - unL;
        const T cm1 = f1 / (sL - sStar);  // c - 1, c = (sL - unL) / (sL - sStar)
        const T c = T(1.) + cm1;
        const T f2 = sStar + PL / (rhoL * (sL - unL));
        F[0] = djac * (rhoL * unL + rhoL * sL * cm1);
        for (int i = 0; i < 3; ++i)
            F[1 + i] = djac * (UL[1 + i] * unL + PsL * n[i] + sL * (UL[1 + i] * cm1 + rhoL * c * f1 * n[i]));
        F[4] = djac * ((UL[4] + PsL + hr) * unL + sL * ((UL[4] + eref) * cm1 + rhoL * c * f1 * f2));
    } else if ((sStar < T(0.)) && (sR > T(0.))) {
        const T f1 = sStar - unR;
        const T cm1 = f1 / (sR - sStar);
        const T c = T(1.) + cm1;
        const T f2 = sStar + PR / (rhoR * (sR - unR));
        F[0] = djac * (rhoR * unR + rhoR * sR * cm1);
        for (int i = 0; i < 3; ++i)
            F[1 + i] = djac * (UR[1 + i] * unR + PsR * n[i] + sR * (UR[1 + i] * cm1 + rhoR * c * f1 * n[i]));
        F[4] = djac * ((UR[4] + PsR + hr) * unR + sR * ((UR[4] + eref) * cm1 + rhoR * c * f1 * f2));
    } else {
        for (int s = 0; s < 5; ++s) F[s] = T(0.0);
        return false;
    }
    return true;
}

// Initial conditions / exact solutions, Physics<3>::call_IC and
// call_exact_solution (src/physics/base/base.cpp:90-137) plus the advected
// xy vortex and Taylor-Green families.  Type codes match DG_IC_* in dg_b200.h.
DG_HD void initial_state(int type, const double* data, double gamma, double R, const double* x,
                         double t, double* U)
{
    if (type == 0) {  // Uniform, base.cpp:150-158
        for (int s = 0; s < 5; ++s) U[s] = data[s];
    } else if (type == 1) {  // reference 3D isentropic vortex, functions.cpp:147-191
        const double rho0 = 1., sos0 = 1., L = 1., Mach = 1.0, radius = L / 10., sigma = 1;
        const double beta = Mach * 5. * sqrt(2.) / (4. * kPi) * exp(0.5);
        const double u0 = Mach * sos0;
        const double x1 = x[0] - 0.5, y1 = x[2] - 0.5;
        const double f = -0.5 / (sigma * sigma) * (x1 * x1 + y1 * y1) / (radius * radius);
        const double Omega = beta * exp(f);
        const double du = -y1 / radius * Omega, dv = x1 / radius * Omega;
        const double dT = -(gamma - 1.) / 2. * Omega * Omega;
        const double p = 1. / gamma * pow(1 + dT, gamma / (gamma - 1.));
        U[0] = pow(rho0 + dT, 1. / (gamma - 1.));
        U[1] = U[0] * (u0 + du);
        U[2] = 0.;
        U[3] = U[0] * dv;
        const double rKE = (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0];
        U[4] = p / (gamma - 1.0) + 0.5 * rKE;
    } else if (type == 2) {  // smooth sphere, base.cpp:177-194
        const double magR = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        for (int s = 0; s < 5; ++s) U[s] = 0.5 * (1. - 0.) * (tanh(kPi * (0.5 - magR) / 0.5) + 1.0) + 0.;
    } else if (type == 3) {  // 2D vortex of functions.cpp:94-145, extruded in z, advected, periodic
        const double rhob = data[0], ub = data[1], vb = data[2], pb = data[3], vs = data[4];
        const double xc = data[5], yc = data[6], Lx = data[7], Ly = data[8];
        const double Tb = pb / (rhob * R);
        const double s = pb / pow(rhob, gamma);
        double xr = x[0] - xc - ub * t;
        double yr = x[1] - yc - vb * t;
        xr -= Lx * floor(xr / Lx + 0.5);
        yr -= Ly * floor(yr / Ly + 0.5);
        const double r = sqrt(xr * xr + yr * yr);
        const double r2 = r * r;
        const double dUm = vs / (2.0 * kPi) * exp(0.5 * (1.0 - r2));
        const double du = dUm * -1.0 * yr, dv = dUm * xr;
        const double dT = -1.0 * (gamma - 1.0) * (vs * vs) / (8.0 * gamma * (kPi * kPi)) * exp(1.0 - r2);
        const double u = ub + du, v = vb + dv, T = Tb + dT;
        const double rho = pow(T / s, 1.0 / (gamma - 1.0));
        const double rhou = rho * u, rhov = rho * v;
        U[0] = rho;
        U[1] = rhou;
        U[2] = rhov;
        U[3] = 0.0;
        U[4] = rho * R / (gamma - 1.0) * T + 0.5 * (rhou * rhou + rhov * rhov) / rho;
    } else if (type == 4) {  // Taylor-Green vortex, data = {Mach}
        const double M = data[0];
        const double u = sin(x[0]) * cos(x[1]) * cos(x[2]);
        const double v = -cos(x[0]) * sin(x[1]) * cos(x[2]);
        const double p = 1.0 / (gamma * M * M) + (cos(2.0 * x[0]) + cos(2.0 * x[1])) * (cos(2.0 * x[2]) + 2.0) / 16.0;
        U[0] = 1.0;
        U[1] = u;
        U[2] = v;
        U[3] = 0.0;
        U[4] = p / (gamma - 1.0) + 0.5 * (u * u + v * v);
    } else {
        for (int s = 0; s < 5; ++s) U[s] = 0.0;
    }
}

}  // namespace dgp
