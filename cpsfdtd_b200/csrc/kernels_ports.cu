// kernels_ports.cu -- port sampling, the blocked FP64 port DFT, flux
// reduction, a non-finite watchdog and host<->device layout conversion.
//
// Port samples of every step are gathered into a ring of T slots
// ([slot][component][point], float on FP32 grids).  Every T steps (and before
// a read-out) one contraction folds the ring into FP64 accumulators:
//   acc[c][f][p] += sum_t s[t][c][p] * exp(-i w_f t_c(n_t))
// with t_c = n dt for E and (n - 1/2) dt for H, i.e. a [P x T] by [T x F]
// complex product per component, accumulated in FP64.  The phasors of the
// block are tabulated once per flush into a small scratch table.
#include "cells.cuh"

namespace cps {

namespace {

template <typename T>
__global__ void k_gather(FieldView<T> f, const int64_t *idx, int npts, T *slot)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    const int64_t g = idx[p];
    slot[p] = f.Ex[g];
    slot[npts + p] = f.Ey[g];
    slot[2 * (int64_t)npts + p] = f.Ez[g];
    slot[3 * (int64_t)npts + p] = f.Hx[g];
    slot[4 * (int64_t)npts + p] = f.Hy[g];
    slot[5 * (int64_t)npts + p] = f.Hz[g];
}

// phasor table [t][f] = (cos, sin)(w_f * n_t * dt), FP64
__global__ void k_phasors(const double *omega, int nfreq, int nslots, int64_t n_first, double dt, double *tab)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nslots * nfreq) return;
    const int t = q / nfreq, fi = q - t * nfreq;
    double s, c;
    sincos(omega[fi] * ((double)(n_first + t) * dt), &s, &c);
    tab[2 * q] = c;
    tab[2 * q + 1] = s;
}

constexpr int kFch = 16;  // frequencies per thread

// one thread = one (point, component, 16-frequency chunk); blockIdx.y = component
template <typename T>
__global__ void __launch_bounds__(128) k_dft(const T *ring, int npts, int nslots, const double *tab,
                                             const double *omega, int nfreq, double dt,
                                             const int32_t *comps, double *acc)
{
    extern __shared__ double sh[];  // [nslots][kFch][2]
    const int ci = blockIdx.y, f0 = blockIdx.z * kFch;
    const int nf = min(kFch, nfreq - f0);
    for (int q = threadIdx.x; q < nslots * kFch; q += blockDim.x) {
        const int t = q / kFch, fi = q - t * kFch;
        const bool ok = fi < nf;
        sh[2 * q] = ok ? tab[2 * (t * nfreq + f0 + fi)] : 0.0;
        sh[2 * q + 1] = ok ? tab[2 * (t * nfreq + f0 + fi) + 1] : 0.0;
    }
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npts) return;
    const int comp = comps[ci];
    double re[kFch], im[kFch];
#pragma unroll
    for (int fi = 0; fi < kFch; ++fi) { re[fi] = 0.0; im[fi] = 0.0; }
    for (int t = 0; t < nslots; ++t) {
        const double v = (double)ring[((int64_t)t * 6 + comp) * npts + p];
        const double *ph = sh + 2 * t * kFch;
#pragma unroll
        for (int fi = 0; fi < kFch; ++fi) {
            re[fi] = fma(v, ph[2 * fi], re[fi]);
            im[fi] = fma(-v, ph[2 * fi + 1], im[fi]);
        }
    }
    for (int fi = 0; fi < nf; ++fi) {
        double r = re[fi], m = im[fi];
        if (comp >= 3) {  // H sits half a step earlier: multiply by exp(+i w dt/2)
            double sn, cs;
            sincos(omega[f0 + fi] * (0.5 * dt), &sn, &cs);
            const double r2 = r * cs - m * sn, m2 = r * sn + m * cs;
            r = r2; m = m2;
        }
        double *a = acc + ((int64_t)(ci * nfreq + f0 + fi) * 2) * npts + p;
        a[0] += r;
        a[npts] += m;
    }
}

// flux[f] = 0.5 * Re sum_p (A_p conj(B_p) - C_p conj(D_p)) * dA over the
// accumulators of four components (indices in sel), block per frequency,
// warp-shuffle reduction
__global__ void k_flux(const double *acc, int npts, int nfreq, int4 sel, double dA, double *out)
{
    const int f = blockIdx.x;
    double s = 0.0;
    auto re = [&](int c, int p) { return acc[((int64_t)(c * nfreq + f) * 2) * npts + p]; };
    auto im = [&](int c, int p) { return acc[((int64_t)(c * nfreq + f) * 2 + 1) * npts + p]; };
    for (int p = threadIdx.x; p < npts; p += blockDim.x) {
        // Re(a conj(b)) = ar br + ai bi
        s += re(sel.x, p) * re(sel.y, p) + im(sel.x, p) * im(sel.y, p);
        s -= re(sel.z, p) * re(sel.w, p) + im(sel.z, p) * im(sel.w, p);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double ws[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) ws[w] = s;
    __syncthreads();
    if (w == 0) {
        s = lane < (blockDim.x >> 5) ? ws[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[f] = 0.5 * s * dA;
    }
}

template <typename T>
__global__ void k_nonfinite(FieldView<T> f, int64_t n, unsigned long long *out)
{
    unsigned long long c = 0;
    const T *F[6] = {f.Ex, f.Ey, f.Ez, f.Hx, f.Hy, f.Hz};
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        for (int a = 0; a < 6; ++a) c += !isfinite((double)F[a][q]);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// reference order [i][j][k] (k fastest) <-> device order
template <typename T>
__global__ void k_to_dev(const double *src, T *dst, Dims d)
{
    const int64_t NZ = d.nz + 1, NY = d.ny + 1, n = (int64_t)(d.nx + 1) * NY * NZ;
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int k = (int)(q % NZ), j = (int)((q / NZ) % NY), i = (int)(q / (NZ * NY));
    dst[d.idx(i, j, k)] = (T)src[q];
}

template <typename T>
__global__ void k_from_dev(const T *src, double *dst, Dims d)
{
    const int64_t NZ = d.nz + 1, NY = d.ny + 1, n = (int64_t)(d.nx + 1) * NY * NZ;
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int k = (int)(q % NZ), j = (int)((q / NZ) % NY), i = (int)(q / (NZ * NY));
    dst[q] = (double)src[d.idx(i, j, k)];
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

template <typename T>
void launch_port_gather(const FieldView<T> &f, const int64_t *idx, int npts, T *slot, cudaStream_t s)
{
    if (npts <= 0) return;
    k_gather<T><<<cdiv(npts, 256), 256, 0, s>>>(f, idx, npts, slot);
}

template <typename T>
void launch_port_dft(const T *ring, int npts, int nslots, int64_t n_first, double dt, const double *omega,
                     int nfreq, const int32_t *comps, int ncomp, double *acc, double *scratch_phasor,
                     cudaStream_t s)
{
    if (npts <= 0 || nslots <= 0 || nfreq <= 0 || ncomp <= 0) return;
    k_phasors<<<cdiv((int64_t)nslots * nfreq, 256), 256, 0, s>>>(omega, nfreq, nslots, n_first, dt, scratch_phasor);
    dim3 grid(cdiv(npts, 128), ncomp, cdiv(nfreq, kFch));
    const size_t smem = sizeof(double) * 2 * kFch * nslots;
    k_dft<T><<<grid, 128, smem, s>>>(ring, npts, nslots, scratch_phasor, omega, nfreq, dt, comps, acc);
}

void launch_port_flux(const double *acc, int npts, int nfreq, int ncomp, const int32_t *sel, double dA,
                      double *out, cudaStream_t s)
{
    (void)ncomp;
    k_flux<<<nfreq, 256, 0, s>>>(acc, npts, nfreq, make_int4(sel[0], sel[1], sel[2], sel[3]), dA, out);
}

template <typename T>
void launch_count_nonfinite(const FieldView<T> &f, unsigned long long *out, cudaStream_t s)
{
    const int64_t n = f.d.pxy * (f.d.nz + 1);
    k_nonfinite<T><<<1184, 256, 0, s>>>(f, n, out);
}

template <typename T>
void launch_to_device_layout(const double *src, T *dst, Dims d, cudaStream_t s)
{
    const int64_t n = (int64_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
    k_to_dev<T><<<cdiv(n, 256), 256, 0, s>>>(src, dst, d);
}

template <typename T>
void launch_from_device_layout(const T *src, double *dst, Dims d, cudaStream_t s)
{
    const int64_t n = (int64_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
    k_from_dev<T><<<cdiv(n, 256), 256, 0, s>>>(src, dst, d);
}

#define CPS_INST(T)                                                                                        \
    template void launch_port_gather<T>(const FieldView<T> &, const int64_t *, int, T *, cudaStream_t);    \
    template void launch_port_dft<T>(const T *, int, int, int64_t, double, const double *, int,            \
                                     const int32_t *, int, double *, double *, cudaStream_t);              \
    template void launch_count_nonfinite<T>(const FieldView<T> &, unsigned long long *, cudaStream_t);     \
    template void launch_to_device_layout<T>(const double *, T *, Dims, cudaStream_t);                     \
    template void launch_from_device_layout<T>(const T *, double *, Dims, cudaStream_t);
CPS_INST(double)
CPS_INST(float)

}  // namespace cps
