// kernels_three.cu -- the three-level gain class (ThreeLevel.cpp) on the
// compacted list of its sites, one thread per site.  Built without FMA
// contraction: the FP64 state follows the oracle's roundings.  The three
// routines are separate launches on the per-routine path; the fused and
// one-pass steps run them as one launch after their E sweep (the values of
// E between the routines are the grid's, rounded to its precision, on both).
#include "cps_internal.h"

namespace cps {

namespace {

enum { TPA = 0, TPA1 = 3, TPA2 = 6, TPB = 9, TPB1 = 12, TPB2 = 15, TE1 = 18, TN0 = 21, TN1 = 22, TN2 = 23,
       TN1_1 = 24, TN2_1 = 25 };

// one site's words in the [word][site] arrays
struct Site {
    double *s;
    int64_t n;
    __device__ double &operator[](int w) const { return s[(int64_t)w * n]; }
};

// UpdatePolarizationDensities, ThreeLevel.cpp:216-245 (Ez as Ex and Ey)
__device__ __forceinline__ void site_p(const ThreeCoef &K, const Site &st, const double E[3])
{
    const double N0 = st[TN0], N1 = st[TN1], N2 = st[TN2];
    for (int c = 0; c < 3; ++c) {
        st[TPA2 + c] = st[TPA1 + c];
        st[TPA1 + c] = st[TPA + c];
        st[TPA + c] = K.CPa1 * st[TPA + c] + K.CPa2 * st[TPA2 + c] + E[c] * K.CPa3 * (N2 - N0);
    }
    for (int c = 0; c < 3; ++c) {
        st[TPB2 + c] = st[TPB1 + c];
        st[TPB1 + c] = st[TPB + c];
        st[TPB + c] = K.CPb1 * st[TPB + c] + K.CPb2 * st[TPB2 + c] + E[c] * K.CPb3 * (N1 - N0);
    }
    for (int c = 0; c < 3; ++c) st[TE1 + c] = E[c];
}

// UpdateElectricField, ThreeLevel.cpp:248-255
__device__ __forceinline__ void site_e(const ThreeCoef &K, const Site &st, double E[3])
{
    for (int c = 0; c < 3; ++c) E[c] = E[c] - K.CEP * (st[TPA + c] - st[TPA1 + c] + st[TPB + c] - st[TPB1 + c]);
}

// UpdateStatesPopulations, ThreeLevel.cpp:258-266 (Ez terms after the Ex and Ey ones)
__device__ __forceinline__ void site_n(const ThreeCoef &K, const Site &st, const double E[3])
{
    double Pa[3], Pa1[3], Pb[3], Pb1[3], E1[3];
    for (int c = 0; c < 3; ++c) {
        Pa[c] = st[TPA + c]; Pa1[c] = st[TPA1 + c]; Pb[c] = st[TPB + c]; Pb1[c] = st[TPB1 + c]; E1[c] = st[TE1 + c];
    }
    const double N2old = st[TN2], N1old = st[TN1];
    double n2 = K.CN2N2 * N2old + K.CN2E * (E[0] + E1[0]) * (Pa[0] - Pa1[0]) + K.CN2E * (E[1] + E1[1]) * (Pa[1] - Pa1[1]);
    n2 = n2 + K.CN2E * (E[2] + E1[2]) * (Pa[2] - Pa1[2]);
    double n1 = K.CN1N1 * N1old + K.CN1N2 * (n2 + N2old) + K.CN1E * (E[0] + E1[0]) * (Pb[0] - Pb1[0]) +
                K.CN1E * (E[1] + E1[1]) * (Pb[1] - Pb1[1]);
    n1 = n1 + K.CN1E * (E[2] + E1[2]) * (Pb[2] - Pb1[2]);
    double n0 = st[TN0] + K.CN0N2 * (n2 + N2old) + K.CN0N1 * (n1 + N1old) -
                K.CN0Ea * (E[0] + E1[0]) * (Pa[0] - Pa1[0]) - K.CN0Ea * (E[1] + E1[1]) * (Pa[1] - Pa1[1]) -
                K.CN0Ebx * (E[0] + E1[0]) * (Pb[0] - Pb1[0]) - K.CN0Eb * (E[1] + E1[1]) * (Pb[1] - Pb1[1]);
    n0 = n0 - K.CN0Ea * (E[2] + E1[2]) * (Pa[2] - Pa1[2]) - K.CN0Eb * (E[2] + E1[2]) * (Pb[2] - Pb1[2]);
    st[TN2_1] = N2old;
    st[TN2] = n2;
    st[TN1_1] = N1old;
    st[TN1] = n1;
    st[TN0] = n0;
}

template <typename T>
__global__ void __launch_bounds__(128) k_three(FieldView<T> f, ThreeView tv, int which)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= tv.ncell) return;
    const int64_t g = tv.cell[c];
    const Site st{tv.state + c, tv.ncell};
    double E[3] = {(double)f.Ex[g], (double)f.Ey[g], (double)f.Ez[g]};
    if (which == 0 || which == 3) site_p(tv.c, st, E);
    if (which == 1 || which == 3) {
        site_e(tv.c, st, E);
        const T ex = (T)E[0], ey = (T)E[1], ez = (T)E[2];
        f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
        E[0] = (double)ex; E[1] = (double)ey; E[2] = (double)ez;
    }
    if (which == 2 || which == 3) site_n(tv.c, st, E);
}

__global__ void k_three_init(double *state, int64_t n, double N_0)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c < n) state[(int64_t)TN0 * n + c] = N_0;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

template <typename T>
void launch_three(const FieldView<T> &f, const ThreeView &t, int which, cudaStream_t s)
{
    if (!t.on || t.ncell <= 0) return;
    k_three<T><<<cdiv(t.ncell, 128), 128, 0, s>>>(f, t, which);
}

void launch_three_init(const ThreeView &t, double N_0, cudaStream_t s)
{
    if (t.ncell <= 0) return;
    cudaMemsetAsync(t.state, 0, (size_t)t.ncell * kThreeWords * sizeof(double), s);
    k_three_init<<<cdiv(t.ncell, 256), 256, 0, s>>>(t.state, t.ncell, N_0);
}

template void launch_three<float>(const FieldView<float> &, const ThreeView &, int, cudaStream_t);
template void launch_three<double>(const FieldView<double> &, const ThreeView &, int, cudaStream_t);

}  // namespace cps
