/*
 * cells.h -- per-cell Drude-Lorentz, four-level and three-level gain recursions of the
 * oracle restatement, shared by oracle.c and the reference harness (which
 * needs them because the reference has no 3-D Drude-Lorentz or gain class).
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#ifndef CPS_ORACLE_CELLS_H
#define CPS_ORACLE_CELLS_H

#include <math.h>
#include <stdint.h>
#include <string.h>

/* Physical constants, values as Constants.h:19-26 */
#ifndef K_PI
#define K_PI 3.1415926535897932384626433832795
#define K_C 2.99792458E8
#define K_HPLANCK 6.62607004081E-34
#define K_MU0 1.2566370614E-6
#define K_EPS0 8.8541878176E-12
#endif

#define MAXP 16

typedef struct {
    int on;
    int nD, nL;
    double kappa[MAXP], beta[MAXP], alpha[MAXP], xi[MAXP], gammaL[MAXP];
    double C1, C2, C3, C4[MAXP], C5[MAXP], C6[MAXP];
    int64_t ncell;
    int64_t *cell; /* linear [i][j][k] index */
    /* per cell, per component c (0..2): JD[nD], JL[nL], JL1[nL], E1 */
    double *state;
    int stride; /* words per component */
} dl_t;

typedef struct {
    int on;
    int gain_id;
    double CPa1, CPa2, CPa3, CPb1, CPb2, CPb3, CEP;
    double t30, t32, t21, t10;
    double t30t32dt, t30t32_2, t30dt, t32dt, dt_2, homega_bdt;
    double t10t21dt, t10t21_2, t10dt, t21dt, t21_2, homega_adt;
    double t32t21dt, t32t21_2, t32_2;
    double pump_dt;
    int64_t ncell;
    int64_t *cell;
    /* per cell: Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3], E1[3], N[4] */
    double *state;
} gain_t;

#define GAIN_WORDS 25

/* Coefficients: Drude_Lorentz.cpp:65-108 (frequencies in Hz, times 2*pi). */
static void dl_coeffs(dl_t *D, double dt, double sigma, double epsInf, int nD, const double *fD,
                      const double *gD, int nL, const double *fL, const double *dL,
                      const double *depsL, int literal)
{
    double temp1 = 0, temp2 = 0;
    D->nD = nD; D->nL = nL;
    for (int p = 0; p < nD; ++p) {
        const double omega = fD[p] * 2.0 * K_PI, gamma = gD[p] * 2.0 * K_PI;
        D->kappa[p] = (1.0 - gamma * dt / 2.0) / (1.0 + gamma * dt / 2.0);
        D->beta[p] = (omega * omega * K_EPS0 * dt / 2.0) / (1.0 + gamma * dt / 2.0);
        temp1 = temp1 + D->beta[p];
    }
    for (int p = 0; p < nL; ++p) {
        const double omega = fL[p] * 2.0 * K_PI, delta = dL[p] * 2.0 * K_PI;
        D->alpha[p] = (2.0 - omega * omega * dt * dt) / (1.0 + delta * dt);
        D->xi[p] = (delta * dt - 1.0) / (1.0 + delta * dt);
        D->gammaL[p] = (K_EPS0 * depsL[p] * omega * omega * dt * dt) / (1.0 + delta * dt);
        temp2 = temp2 + D->gammaL[p];
    }
    if (literal == 2 && nD == 1 && nL == 0) {
        /* the single-pole Drude class: Drude.cpp:56-60 in its own order
         * (C1Drude, C2Drude, C3Drude are the C1, C3, C4[0] of this recursion) */
        const double b = D->beta[0], kp = D->kappa[0];
        D->C1 = (2 * K_EPS0 * epsInf - dt * b - sigma * dt) / (2 * K_EPS0 * epsInf + dt * b + sigma * dt);
        D->C2 = 0.0;
        D->C3 = (2 * dt) / (2 * K_EPS0 * epsInf + dt * b + sigma * dt);
        D->C4[0] = ((1 + kp) * dt) / (2 * K_EPS0 * epsInf + dt * b + sigma * dt);
        return;
    }
    const double den = 2.0 * K_EPS0 * epsInf + sigma * dt + dt * temp1 + temp2 / 2.0;
    /* literal: C1 and C5 exactly as Drude_Lorentz.cpp:96,106.  Otherwise the
     * values the ADE discretisation gives: the E^n coefficient carries
     * -sigma dt - dt sum(beta) and the J_L^n coefficient carries dt; the literal
     * C5 makes any Lorentz pole unstable. */
    if (literal)
        D->C1 = (2.0 * K_EPS0 * epsInf + sigma * dt + dt * temp1) / den;
    else
        D->C1 = (2.0 * K_EPS0 * epsInf - sigma * dt - dt * temp1) / den;
    D->C2 = temp2 / 2.0 / den;
    D->C3 = 2.0 * dt / den;
    for (int p = 0; p < nD; ++p) D->C4[p] = (1.0 + D->kappa[p]) * dt / den;
    for (int p = 0; p < nL; ++p) {
        D->C5[p] = literal ? (1.0 + D->alpha[p]) / den : (1.0 + D->alpha[p]) * dt / den;
        D->C6[p] = D->xi[p] * dt / den;
    }
}

/* One component of the ADE update at one cell: Drude_Lorentz.cpp:163-184.
 * curl is the curl term already multiplied by C3.  st = JD[nD] JL[nL] JL1[nL] E1. */
static inline double dl_component(const dl_t *D, double dt, double E, double curl, double *st)
{
    double *JD = st, *JL = st + D->nD, *JL1 = st + D->nD + D->nL;
    double *E1 = st + D->nD + 2 * D->nL;
    const double temp = E;
    double t1 = 0.0, t2 = 0.0;
    for (int p = 0; p < D->nD; ++p) t1 = t1 + D->C4[p] * JD[p];
    for (int p = 0; p < D->nL; ++p) t2 = t2 + D->C5[p] * JL[p] + D->C6[p] * JL1[p];
    E = D->C1 * E + D->C2 * (*E1) + curl - t1 - t2;
    for (int p = 0; p < D->nD; ++p) JD[p] = D->kappa[p] * JD[p] + D->beta[p] * (E + temp);
    for (int p = 0; p < D->nL; ++p) {
        const double t0 = JL[p];
        JL[p] = D->alpha[p] * JL[p] + D->xi[p] * JL1[p] + D->gammaL[p] * (E - *E1) / 2.0 / dt;
        JL1[p] = t0;
    }
    *E1 = temp;
    return E;
}

/* Coefficients: FourLevelLaser.cpp:96-105, 202-206.  pump_rate is an added
 * incoherent pump N0 -> N3 (no reference counterpart; 0 reproduces it). */
static void gain_coeffs(gain_t *G, double dt, double dx, double dy, double lambda_a,
                        double lambda_b, double gamma_a, double gamma_b, double t30, double t32,
                        double t21, double t10, double N_0, double pump_rate)
{
    const double omega_a = 2.0 * K_PI * K_C / lambda_a;
    const double omega_b = 2.0 * K_PI * K_C / lambda_b;
    const double zeta_a = 6.0 * K_PI * K_EPS0 * K_C * K_C * K_C / (omega_a * omega_a * t21);
    const double zeta_b = 6.0 * K_PI * K_EPS0 * K_C * K_C * K_C / (omega_b * omega_b * t30);
    G->CPa1 = (2.0 - omega_a * omega_a * dt * dt) / (1.0 + gamma_a * dt / 2.0);
    G->CPa2 = (gamma_a * dt / 2.0 - 1.0) / (1.0 + gamma_a * dt / 2.0);
    G->CPa3 = dt * dt * zeta_a / (1.0 + gamma_a * dt / 2.0);
    G->CPb1 = (2.0 - omega_b * omega_b * dt * dt) / (1.0 + gamma_b * dt / 2.0);
    G->CPb2 = (gamma_b * dt / 2.0 - 1.0) / (1.0 + gamma_b * dt / 2.0);
    G->CPb3 = dt * dt * zeta_b / (1.0 + gamma_b * dt / 2.0);
    G->CEP = 2.0 * N_0 * dx * dy * dx / K_EPS0 / dt;
    G->t30 = t30; G->t32 = t32; G->t21 = t21; G->t10 = t10;
    G->t30t32dt = t30 * t32 * dt; G->t30t32_2 = 2.0 * t30 * t32; G->t30dt = t30 * dt;
    G->t32dt = t32 * dt; G->dt_2 = 2.0 / dt; G->homega_bdt = K_HPLANCK * omega_b * dt / 2.0 / K_PI;
    G->t10t21dt = t10 * t21 * dt; G->t10t21_2 = 2.0 * t10 * t21; G->t10dt = t10 * dt;
    G->t21dt = t21 * dt; G->t21_2 = t21 / 2.0; G->homega_adt = K_HPLANCK * omega_a * dt / 2.0 / K_PI;
    G->t32t21dt = t32 * t21 * dt; G->t32t21_2 = 2.0 * t32 * t21; G->t32_2 = t32 / 2.0;
    G->pump_dt = pump_rate * dt;
}

/* state layout per site */
#define GS_PA 0
#define GS_PA1 3
#define GS_PA2 6
#define GS_PB 9
#define GS_PB1 12
#define GS_PB2 15
#define GS_E1 18
#define GS_N 21

static void gain_site_init(double *st)
{
    memset(st, 0, sizeof(double) * GAIN_WORDS);
    st[GS_N + 0] = 1.0; /* N0, FourLevelLaser.cpp:194-197 */
    st[GS_N + 1] = 1.0; /* N1 */
}

/* UpdatePolarizationDensities at one site, FourLevelLaser.cpp:274-295; nc = 2 (TE) or 3 */
static inline void gain_site_p(const gain_t *G, double *st, const double *E, int nc)
{
    const double N0 = st[GS_N], N1 = st[GS_N + 1], N2 = st[GS_N + 2], N3 = st[GS_N + 3];
    for (int c = 0; c < nc; ++c) {
        st[GS_PA2 + c] = st[GS_PA1 + c];
        st[GS_PA1 + c] = st[GS_PA + c];
        st[GS_PA + c] = G->CPa1 * st[GS_PA + c] + G->CPa2 * st[GS_PA2 + c] + E[c] * G->CPa3 * (N2 - N1);
    }
    for (int c = 0; c < nc; ++c) {
        st[GS_PB2 + c] = st[GS_PB1 + c];
        st[GS_PB1 + c] = st[GS_PB + c];
        st[GS_PB + c] = G->CPb1 * st[GS_PB + c] + G->CPb2 * st[GS_PB2 + c] + E[c] * G->CPb3 * (N3 - N0);
    }
    for (int c = 0; c < nc; ++c) st[GS_E1 + c] = E[c];
}

/* UpdateElectricField at one site, FourLevelLaser.cpp:302-305 */
static inline void gain_site_e(const gain_t *G, const double *st, double *E, int nc)
{
    for (int c = 0; c < nc; ++c)
        E[c] = E[c] - G->CEP * (st[GS_PA + c] - st[GS_PA1 + c] + st[GS_PB + c] - st[GS_PB1 + c]);
}

/* UpdateStatesPopulations at one site, FourLevelLaser.cpp:313-324.  The N2
 * term for Ey uses Pay - Pay_1 as the reference does (:316); Ez follows the Ex
 * form.  The pump term is added to N3 after its update. */
static inline void gain_site_n(const gain_t *G, double *st, const double *E, int nc)
{
    const double *Pa = st + GS_PA, *Pa1 = st + GS_PA1, *Pa2 = st + GS_PA2;
    const double *Pb = st + GS_PB, *Pb2 = st + GS_PB2;
    const double *E1 = st + GS_E1;
    double *N = st + GS_N;
    const double N0old = N[0];
    double sb = E1[0] * (Pb[0] - Pb2[0]) + E1[1] * (Pb[1] - Pb2[1]);
    if (nc == 3) sb = sb + E1[2] * (Pb[2] - Pb2[2]);
    N[3] = G->t30t32dt / (G->t30t32_2 + G->t30dt * (1 - N[2]) + G->t32dt * (1 - N[0])) *
           (N[3] * ((N[0] - 1) / G->t30 + (N[2] - 1) / G->t32 + G->dt_2) + sb / G->homega_bdt);
    N[3] = N[3] + G->pump_dt * N0old;
    double sa = E1[0] * (Pa[0] - Pa2[0]) + E1[1] * (Pa[1] - Pa2[1]);
    if (nc == 3) sa = sa + E1[2] * (Pa[2] - Pa2[2]);
    N[1] = G->t10t21dt / (G->t10t21_2 + G->t10dt * N[2] + G->t21dt * (1 - N[0])) *
           (N[1] * ((N[0] - 1) / G->t10 - N[2] / G->t21 + G->dt_2) + N[2] / G->t21_2 - sa / G->homega_adt);
    double s2 = (E[0] + E1[0]) * (Pa[0] - Pa2[0]) + (E[1] + E1[1]) * (Pa[1] - Pa1[1]);
    if (nc == 3) s2 = s2 + (E[2] + E1[2]) * (Pa[2] - Pa2[2]);
    N[2] = G->t32t21dt / (G->t32t21_2 + G->t21dt * N[3] + G->t32dt * (1 - N[1])) *
           (N[2] * ((N[1] - 1) / G->t21 - N[3] / G->t32 + G->dt_2) + N[3] / G->t32_2 + s2 / G->homega_adt);
    N[0] = 2.0 - N[1] - N[2] - N[3];
}

/* ------------------------------------------------ three-level gain --- */

#ifndef K_QE
#define K_QE (-1.602176565E-19) /* electron charge, Constants.h:26 */
#define K_ME 9.10938215E-31     /* electron mass, Constants.h:25 */
#endif

typedef struct {
    int on;
    int gain_id;
    double CPa1, CPa2, CPa3, CPb1, CPb2, CPb3, CEP;
    double CN2N2, CN2E, CN1N1, CN1N2, CN1E, CN0N2, CN0N1, CN0Ea, CN0Eb, CN0Ebx;
    double N_0;
    int64_t ncell;
    int64_t *cell;
    /* per site: Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3], E1[3], N0 N1 N2 N1_1 N2_1 */
    double *state;
} three_t;

#define THREE_WORDS 26
#define TS_PA 0
#define TS_PA1 3
#define TS_PA2 6
#define TS_PB 9
#define TS_PB1 12
#define TS_PB2 15
#define TS_E1 18
#define TS_N0 21
#define TS_N1 22
#define TS_N2 23
#define TS_N1_1 24
#define TS_N2_1 25

/* Coefficients: ThreeLevel.cpp:96-119 and :208.  literal = 1 takes them as
 * the reference writes them: its oscillator coefficients CPa1 = 2/((dt^2 +
 * w^2)(1/dt^2 + g/2dt)) and CPa2 = (2/dt^2 + 1/2dt)/(...) make P double every
 * two steps, and the N0 update applies CN0Ea to the Pbx term.  literal = 0
 * uses the Lorentz-oscillator discretisation (2/dt^2 - w^2)/(1/dt^2 + g/2dt)
 * and (g/2dt - 1/dt^2)/(1/dt^2 + g/2dt), and CN0Eb on every b term. */
static void three_coeffs(three_t *T3, double dt, double lambda_a, double lambda_b, double gamma_a,
                         double gamma_b, double t20, double t21, double t10, double N_0, int literal)
{
    const double omega_a = 2.0 * K_PI * K_C / lambda_a;
    const double omega_b = 2.0 * K_PI * K_C / lambda_b;
    if (literal) {
        T3->CPa1 = 2 / ((dt * dt + omega_a * omega_a) * (1 / (dt * dt) + gamma_a / (2 * dt)));
        T3->CPa2 = (2 / (dt * dt) + 1 / (2 * dt)) / (1 / (dt * dt) + gamma_a / (2 * dt));
        T3->CPb1 = 2 / ((dt * dt + omega_b * omega_b) * (1 / (dt * dt) + gamma_b / (2 * dt)));
        T3->CPb2 = (2 / (dt * dt) + 1 / (2 * dt)) / (1 / (dt * dt) + gamma_b / (2 * dt));
    } else {
        T3->CPa1 = (2 / (dt * dt) - omega_a * omega_a) / (1 / (dt * dt) + gamma_a / (2 * dt));
        T3->CPa2 = (gamma_a / (2 * dt) - 1 / (dt * dt)) / (1 / (dt * dt) + gamma_a / (2 * dt));
        T3->CPb1 = (2 / (dt * dt) - omega_b * omega_b) / (1 / (dt * dt) + gamma_b / (2 * dt));
        T3->CPb2 = (gamma_b / (2 * dt) - 1 / (dt * dt)) / (1 / (dt * dt) + gamma_b / (2 * dt));
    }
    T3->CPa3 = (K_QE * K_QE / K_ME) / (1 / (dt * dt) + gamma_a / (2 * dt)) / N_0;
    T3->CPb3 = (K_QE * K_QE / K_ME) / (1 / (dt * dt) + gamma_b / (2 * dt)) / N_0;
    T3->CN2N2 = (1.0 / dt - 1.0 / (2.0 * t20) - 1.0 / (2.0 * t21)) / (1.0 / dt + 1.0 / (2.0 * t20) + 1.0 / (2.0 * t21));
    T3->CN2E = (1.0 / (2.0 * dt * K_HPLANCK * omega_a / 2.0 / K_PI)) / (1.0 / dt + 1.0 / (2.0 * t20) + 1.0 / (2.0 * t21));
    T3->CN1N1 = (1.0 / dt - 1.0 / (2.0 * t10)) / (1.0 / dt + 1.0 / (2.0 * t10));
    T3->CN1N2 = (1.0 / (2.0 * t21)) / (1.0 / dt + 1.0 / (2.0 * t10));
    T3->CN1E = (1.0 / (2.0 * dt * K_HPLANCK * omega_b / 2.0 / K_PI)) / (1.0 / dt + 1.0 / (2.0 * t10));
    T3->CN0N1 = dt / (2.0 * t10);
    T3->CN0N2 = dt / (2.0 * t20);
    T3->CN0Ea = 1.0 / (2.0 * K_HPLANCK * omega_a / 2.0 / K_PI);
    T3->CN0Eb = 1.0 / (2.0 * K_HPLANCK * omega_b / 2.0 / K_PI);
    T3->CN0Ebx = literal ? T3->CN0Ea : T3->CN0Eb;
    T3->CEP = 1.0 / dt / K_EPS0;
    T3->N_0 = N_0;
}

/* ThreeLevel.cpp:200-206: P, E1, N1, N2 zero, N0 = N_0 */
static void three_site_init(double *st, double N_0)
{
    memset(st, 0, sizeof(double) * THREE_WORDS);
    st[TS_N0] = N_0;
}

/* UpdatePolarizationDensities at one site, ThreeLevel.cpp:216-245; nc = 2 (TE) or 3 */
static inline void three_site_p(const three_t *T3, double *st, const double *E, int nc)
{
    const double N0 = st[TS_N0], N1 = st[TS_N1], N2 = st[TS_N2];
    for (int c = 0; c < nc; ++c) {
        st[TS_PA2 + c] = st[TS_PA1 + c];
        st[TS_PA1 + c] = st[TS_PA + c];
        st[TS_PA + c] = T3->CPa1 * st[TS_PA + c] + T3->CPa2 * st[TS_PA2 + c] + E[c] * T3->CPa3 * (N2 - N0);
    }
    for (int c = 0; c < nc; ++c) {
        st[TS_PB2 + c] = st[TS_PB1 + c];
        st[TS_PB1 + c] = st[TS_PB + c];
        st[TS_PB + c] = T3->CPb1 * st[TS_PB + c] + T3->CPb2 * st[TS_PB2 + c] + E[c] * T3->CPb3 * (N1 - N0);
    }
    for (int c = 0; c < nc; ++c) st[TS_E1 + c] = E[c];
}

/* UpdateElectricField at one site, ThreeLevel.cpp:248-255 */
static inline void three_site_e(const three_t *T3, const double *st, double *E, int nc)
{
    for (int c = 0; c < nc; ++c)
        E[c] = E[c] - T3->CEP * (st[TS_PA + c] - st[TS_PA1 + c] + st[TS_PB + c] - st[TS_PB1 + c]);
}

/* UpdateStatesPopulations at one site, ThreeLevel.cpp:258-266 (the Ez terms,
 * absent in the reference's 2-D class, follow the Ex and Ey forms) */
static inline void three_site_n(const three_t *T3, double *st, const double *E, int nc)
{
    const double *Pa = st + TS_PA, *Pa1 = st + TS_PA1, *Pb = st + TS_PB, *Pb1 = st + TS_PB1;
    const double *E1 = st + TS_E1;
    st[TS_N2_1] = st[TS_N2];
    double n2 = T3->CN2N2 * st[TS_N2] + T3->CN2E * (E[0] + E1[0]) * (Pa[0] - Pa1[0]) +
                T3->CN2E * (E[1] + E1[1]) * (Pa[1] - Pa1[1]);
    if (nc == 3) n2 = n2 + T3->CN2E * (E[2] + E1[2]) * (Pa[2] - Pa1[2]);
    st[TS_N2] = n2;
    st[TS_N1_1] = st[TS_N1];
    double n1 = T3->CN1N1 * st[TS_N1] + T3->CN1N2 * (st[TS_N2] + st[TS_N2_1]) +
                T3->CN1E * (E[0] + E1[0]) * (Pb[0] - Pb1[0]) + T3->CN1E * (E[1] + E1[1]) * (Pb[1] - Pb1[1]);
    if (nc == 3) n1 = n1 + T3->CN1E * (E[2] + E1[2]) * (Pb[2] - Pb1[2]);
    st[TS_N1] = n1;
    double n0 = st[TS_N0] + T3->CN0N2 * (st[TS_N2] + st[TS_N2_1]) + T3->CN0N1 * (st[TS_N1] + st[TS_N1_1]) -
                T3->CN0Ea * (E[0] + E1[0]) * (Pa[0] - Pa1[0]) - T3->CN0Ea * (E[1] + E1[1]) * (Pa[1] - Pa1[1]) -
                T3->CN0Ebx * (E[0] + E1[0]) * (Pb[0] - Pb1[0]) - T3->CN0Eb * (E[1] + E1[1]) * (Pb[1] - Pb1[1]);
    if (nc == 3)
        n0 = n0 - T3->CN0Ea * (E[2] + E1[2]) * (Pa[2] - Pa1[2]) - T3->CN0Eb * (E[2] + E1[2]) * (Pb[2] - Pb1[2]);
    st[TS_N0] = n0;
}

#endif
