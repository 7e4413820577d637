// cells.cuh -- per-cell recursions shared by the plain and fused kernels.
//
// Each function is the device form of one reference update at one cell; the
// arithmetic keeps the reference's operation order term by term.
#pragma once

#include "cps_internal.h"

namespace cps {

template <typename T>
__device__ __forceinline__ T ld(const T *p) { return __ldg(p); }

// Coefficient of a cell's psi term.  By default the cell's own curl
// coefficient: bE of its medium, the Drude-Lorentz C3 on ID-2 cells (p.ce_disp),
// bH of its medium on the H side -- the CFS-PML update for any medium, and
// equal to the reference's values wherever the CPML holds eps_r = mu_r = 1
// media.  With p.literal the reference's single coefficients dt/eps0 and
// bH[0] (CPML.cpp:524-525), which make the CPML grow without bound when its
// medium has eps_r != 1.
template <typename T>
__device__ __forceinline__ T pml_ce_cell(const PmlView<T> &p, const T *bE_table, int id)
{
    if (p.literal) return p.cpmlE;
    return id == CPS_ID_DISPERSIVE ? p.ce_disp : __ldg(&bE_table[id]);
}
template <typename T>
__device__ __forceinline__ T pml_ch_cell(const PmlView<T> &p, const T *bH_table, int id)
{
    return p.literal ? p.cpmlH : __ldg(&bH_table[id]);
}

// One component of the Drude-Lorentz ADE at one cell: Drude_Lorentz.cpp:163-184.
// curl is the curl term already multiplied by C3; the state words of this
// component are st[w * stride_cells], w = JD[nD] JL[nL] JL1[nL] E1.
template <typename T>
__device__ __forceinline__ T dl_component(const DlCoef<T> &D, T E, T curl, T *st, int64_t sc)
{
    const T temp = E;
    T t1 = T(0), t2 = T(0);
#pragma unroll 1
    for (int p = 0; p < D.nD; ++p) t1 = t1 + D.C4[p] * st[p * sc];
#pragma unroll 1
    for (int p = 0; p < D.nL; ++p) t2 = t2 + D.C5[p] * st[(D.nD + p) * sc] + D.C6[p] * st[(D.nD + D.nL + p) * sc];
    T *E1 = st + (D.nD + 2 * D.nL) * sc;
    const T e1 = *E1;
    E = D.C1 * E + D.C2 * e1 + curl - t1 - t2;
#pragma unroll 1
    for (int p = 0; p < D.nD; ++p) st[p * sc] = D.kappa[p] * st[p * sc] + D.beta[p] * (E + temp);
#pragma unroll 1
    for (int p = 0; p < D.nL; ++p) {
        const T t0 = st[(D.nD + p) * sc];
        st[(D.nD + p) * sc] = D.alpha[p] * t0 + D.xi[p] * st[(D.nD + D.nL + p) * sc] + D.gammaL[p] * (E - e1) / T(2.0) / D.dt;
        st[(D.nD + D.nL + p) * sc] = t0;
    }
    *E1 = temp;
    return E;
}

// The same update for compile-time pole counts, from state words already in
// registers (w[0 .. ND+2NL], the component's words in order); the arithmetic
// is dl_component's, operation for operation.
template <typename T, int ND, int NL>
__device__ __forceinline__ T dl_component_regs(const DlCoef<T> &D, T E, T curl, const T *w, T *st, int64_t sc)
{
    const T temp = E;
    T t1 = T(0), t2 = T(0);
#pragma unroll
    for (int p = 0; p < ND; ++p) t1 = t1 + D.C4[p] * w[p];
#pragma unroll
    for (int p = 0; p < NL; ++p) t2 = t2 + D.C5[p] * w[ND + p] + D.C6[p] * w[ND + NL + p];
    const T e1 = w[ND + 2 * NL];
    E = D.C1 * E + D.C2 * e1 + curl - t1 - t2;
#pragma unroll
    for (int p = 0; p < ND; ++p) st[p * sc] = D.kappa[p] * w[p] + D.beta[p] * (E + temp);
#pragma unroll
    for (int p = 0; p < NL; ++p) {
        const T t0 = w[ND + p];
        st[(ND + p) * sc] = D.alpha[p] * t0 + D.xi[p] * w[ND + NL + p] + D.gammaL[p] * (E - e1) / T(2.0) / D.dt;
        st[(ND + NL + p) * sc] = t0;
    }
    st[(ND + 2 * NL) * sc] = temp;
    return E;
}

// ---------------------------------------------------------------- gain
// FP64 layout (reference state, unscaled): words
//   0..2 Pa, 3..5 Pa1, 6..8 Pa2, 9..11 Pb, 12..14 Pb1, 15..17 Pb2, 18..20 E1, 21..24 N0..N3
// FP32 layout (P scaled by CEP, populations as offsets): words
//   0..2 Pa, 3..5 Pa1, 6..8 Pb, 9..11 Pb1, 12 N1-1, 13 N2, 14 N3, 15..17 Pa2, 18..20 Pb2, 21..23 E1
struct GainSite64 {
    static constexpr int PA = 0, PA1 = 3, PA2 = 6, PB = 9, PB1 = 12, PB2 = 15, E1 = 18, N = 21;
};
struct GainSite32 {
    static constexpr int PA = 0, PA1 = 3, PB = 6, PB1 = 9, DN1 = 12, N2 = 13, N3 = 14, PA2 = 15, PB2 = 18, E1 = 21;
};

// Populations of a site.  FP64 grids keep N0..N3 as the reference does.
// FP32 grids keep the offsets from the initial state, n1 = N1 - 1, n2 = N2,
// n3 = N3, and m0 = N0 - 1 = -(n1 + n2 + n3) from conservation (the sum in
// FP64, FourLevelLaser.cpp:324), so no update subtracts numbers near 1.
template <typename T>
struct Pops {
    double N[4];
};
template <>
struct Pops<float> {
    float n1, n2, n3, m0;
};

__device__ __forceinline__ float conserve_m0(float n1, float n2, float n3)
{
    return (float)(-((double)n1 + (double)n2 + (double)n3));
}

template <typename T>
__device__ __forceinline__ void gain_load_n(const T *st, int64_t sc, Pops<T> &P);
template <>
__device__ __forceinline__ void gain_load_n<double>(const double *st, int64_t sc, Pops<double> &P)
{
    for (int q = 0; q < 4; ++q) P.N[q] = st[(GainSite64::N + q) * sc];
}
template <>
__device__ __forceinline__ void gain_load_n<float>(const float *st, int64_t sc, Pops<float> &P)
{
    P.n1 = st[GainSite32::DN1 * sc];
    P.n2 = st[GainSite32::N2 * sc];
    P.n3 = st[GainSite32::N3 * sc];
    P.m0 = conserve_m0(P.n1, P.n2, P.n3);
}

// P update (FourLevelLaser.cpp:274-295) with explicit P, P1 in/out and the
// shifted-out P2 returned; P values are in the grid's storage scale.
template <typename T>
__device__ __forceinline__ void gain_p_update(const GainCoef &G, const Pops<T> &P, const T E[3], T Pa[3],
                                              T Pa1[3], T Pa2[3], T Pb[3], T Pb1[3], T Pb2[3])
{
    const T ca1 = (T)G.CPa1, ca2 = (T)G.CPa2, ca3 = (T)(G.CPa3 * G.scaleP);
    const T cb1 = (T)G.CPb1, cb2 = (T)G.CPb2, cb3 = (T)(G.CPb3 * G.scaleP);
    const T dNa = (T)(P.N[2] - P.N[1]), dNb = (T)(P.N[3] - P.N[0]);
    for (int c = 0; c < 3; ++c) {
        Pa2[c] = Pa1[c];
        Pa1[c] = Pa[c];
        Pa[c] = ca1 * Pa[c] + ca2 * Pa2[c] + E[c] * ca3 * dNa;
    }
    for (int c = 0; c < 3; ++c) {
        Pb2[c] = Pb1[c];
        Pb1[c] = Pb[c];
        Pb[c] = cb1 * Pb[c] + cb2 * Pb2[c] + E[c] * cb3 * dNb;
    }
}

// FP32 grids: the same recursion with the float coefficients prepared on the
// host; N2 - N1 = (n2 - n1) - 1 and N3 - N0 = (n3 - m0) - 1
template <>
__device__ __forceinline__ void gain_p_update<float>(const GainCoef &G, const Pops<float> &P, const float E[3],
                                                     float Pa[3], float Pa1[3], float Pa2[3], float Pb[3],
                                                     float Pb1[3], float Pb2[3])
{
    const float dNa = (P.n2 - P.n1) - 1.0f, dNb = (P.n3 - P.m0) - 1.0f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        Pa2[c] = Pa1[c];
        Pa1[c] = Pa[c];
        Pa[c] = G.fa1 * Pa[c] + G.fa2 * Pa2[c] + E[c] * G.fa3 * dNa;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        Pb2[c] = Pb1[c];
        Pb1[c] = Pb[c];
        Pb[c] = G.fb1 * Pb[c] + G.fb2 * Pb2[c] + E[c] * G.fb3 * dNb;
    }
}

// E correction (FourLevelLaser.cpp:302-305): E -= CEP (dPa + dPb)
template <typename T>
__device__ __forceinline__ T gain_e_corr(const GainCoef &G, T E, T pa, T pa1, T pb, T pb1)
{
    if (G.scaleP == 1.0) return E - (T)G.CEP * (pa - pa1 + pb - pb1);
    return E - (pa - pa1 + pb - pb1);  // P already carries the factor CEP
}

// Population update (FourLevelLaser.cpp:313-324) in FP64; the N2 term for Ey
// uses Pay - Pay_1 as the reference does (:316), Ez follows the Ex form; the
// pump moves pump_rate*dt*N0 from N0 to N3.
template <typename T>
__device__ __forceinline__ void gain_n_update(const GainCoef &G, Pops<T> &P, const T E[3], const T E1[3],
                                              const T Pa[3], const T Pa1[3], const T Pa2[3], const T Pb[3],
                                              const T Pb2[3])
{
    double *N = P.N;
    const double inv = 1.0 / G.scaleP;
    // on FP64 grids (scaleP == 1) the sums keep the reference's exact roundings
    double sb = (double)E1[0] * ((double)Pb[0] - (double)Pb2[0]) + (double)E1[1] * ((double)Pb[1] - (double)Pb2[1]);
    sb = sb + (double)E1[2] * ((double)Pb[2] - (double)Pb2[2]);
    if (G.scaleP != 1.0) sb = sb * inv;
    const double N0old = N[0];
    N[3] = G.t30t32dt / (G.t30t32_2 + G.t30dt * (1 - N[2]) + G.t32dt * (1 - N[0])) *
           (N[3] * ((N[0] - 1) / G.t30 + (N[2] - 1) / G.t32 + G.dt_2) + sb / G.homega_bdt);
    N[3] = N[3] + G.pump_dt * N0old;
    double sa = (double)E1[0] * ((double)Pa[0] - (double)Pa2[0]) + (double)E1[1] * ((double)Pa[1] - (double)Pa2[1]);
    sa = sa + (double)E1[2] * ((double)Pa[2] - (double)Pa2[2]);
    double s2 = ((double)E[0] + (double)E1[0]) * ((double)Pa[0] - (double)Pa2[0]) + ((double)E[1] + (double)E1[1]) * ((double)Pa[1] - (double)Pa1[1]);
    s2 = s2 + ((double)E[2] + (double)E1[2]) * ((double)Pa[2] - (double)Pa2[2]);
    if (G.scaleP != 1.0) { sa = sa * inv; s2 = s2 * inv; }
    N[1] = G.t10t21dt / (G.t10t21_2 + G.t10dt * N[2] + G.t21dt * (1 - N[0])) *
           (N[1] * ((N[0] - 1) / G.t10 - N[2] / G.t21 + G.dt_2) + N[2] / G.t21_2 - sa / G.homega_adt);
    N[2] = G.t32t21dt / (G.t32t21_2 + G.t21dt * N[3] + G.t32dt * (1 - N[1])) *
           (N[2] * ((N[1] - 1) / G.t21 - N[3] / G.t32 + G.dt_2) + N[3] / G.t32_2 + s2 / G.homega_adt);
    N[0] = 2.0 - N[1] - N[2] - N[3];
}

// FP32 grids: the same semi-implicit update in FP32 on the offsets.  Dividing
// numerator and denominator of each update by its lifetime product (2 t30 t32,
// 2 t10 t21, 2 t32 t21) and writing N1 = 1 + n1, N0 = 1 + m0 gives, with
// k1a = dt/2t21, k1b = dt/2t10, k3a = dt/2t32, k3b = dt/2t30, ha = dt/2hwa,
// hb = dt/2hwb (hw* = homega_*dt; ha, hb also undo P's storage scale):
//   n3' = [n3 (1 + k3b m0 - k3a (1 - n2)) + hb sb] / [1 + k3a (1 - n2) - k3b m0]
//         + pump dt (1 + m0)
//   n1' = [n1 (1 + k1b m0 - k1a n2) + 2 k1b m0 - ha sa] / [1 + k1a n2 - k1b m0]
//   n2' = [n2 (1 + k1a n1' - k3a n3') + 2 k3a n3' + ha s2] / [1 + k3a n3' - k1a n1']
// (algebraically the reference's expressions; every term is an offset or a
// small multiple of one, so FP32 keeps the offsets to a few ulps), then
// m0' = -(n1' + n2' + n3') in FP64.  The energy-exchange sums E.(P - P'') are
// formed in float.
template <>
__device__ __forceinline__ void gain_n_update<float>(const GainCoef &G, Pops<float> &P, const float E[3],
                                                     const float E1[3], const float Pa[3], const float Pa1[3],
                                                     const float Pa2[3], const float Pb[3], const float Pb2[3])
{
    const float sb = E1[0] * (Pb[0] - Pb2[0]) + E1[1] * (Pb[1] - Pb2[1]) + E1[2] * (Pb[2] - Pb2[2]);
    const float sa = E1[0] * (Pa[0] - Pa2[0]) + E1[1] * (Pa[1] - Pa2[1]) + E1[2] * (Pa[2] - Pa2[2]);
    const float s2 = (E[0] + E1[0]) * (Pa[0] - Pa2[0]) + (E[1] + E1[1]) * (Pa[1] - Pa1[1]) +
                     (E[2] + E1[2]) * (Pa[2] - Pa2[2]);
    const float n1 = P.n1, n2 = P.n2, n3 = P.n3, m0 = P.m0;
    const float q3 = G.k3a * (1.0f - n2) - G.k3b * m0;
    const float n3n = __fdividef(n3 * (1.0f - q3) + G.hb * sb, 1.0f + q3) + G.fpump * (1.0f + m0);
    const float q1 = G.k1a * n2 - G.k1b * m0;
    const float n1n = __fdividef(n1 * (1.0f - q1) + 2.0f * G.k1b * m0 - G.ha * sa, 1.0f + q1);
    const float q2 = G.k3a * n3n - G.k1a * n1n;
    const float n2n = __fdividef(n2 * (1.0f - q2) + 2.0f * G.k3a * n3n + G.ha * s2, 1.0f + q2);
    P.n1 = n1n;
    P.n2 = n2n;
    P.n3 = n3n;
    P.m0 = conserve_m0(n1n, n2n, n3n);
}

template <typename T>
__device__ __forceinline__ void gain_store_n(T *st, int64_t sc, const Pops<T> &P);
template <>
__device__ __forceinline__ void gain_store_n<double>(double *st, int64_t sc, const Pops<double> &P)
{
    for (int q = 0; q < 4; ++q) st[(GainSite64::N + q) * sc] = P.N[q];
}
template <>
__device__ __forceinline__ void gain_store_n<float>(float *st, int64_t sc, const Pops<float> &P)
{
    st[GainSite32::DN1 * sc] = P.n1;
    st[GainSite32::N2 * sc] = P.n2;
    st[GainSite32::N3 * sc] = P.n3;
}

// TF/SF incident-table lookup, TF_SF.cpp:966-986; indices past the table read 0
template <typename T>
__device__ __forceinline__ double inc_lookup(const T *tab, int Nt, double retarded)
{
    if (retarded <= 0) return 0.0;
    const double fl = floor(retarded);
    const double resid = retarded - fl;
    const long long m = (long long)fl;
    const double a = m <= Nt ? (double)tab[m] : 0.0;
    const double b = m + 1 <= Nt ? (double)tab[m + 1] : 0.0;
    return ((1.0 - resid) * a + resid * b);
}

}  // namespace cps
