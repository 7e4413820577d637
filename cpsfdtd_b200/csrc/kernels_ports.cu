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

// all ports of a grid in one launch: blockIdx.y selects the port
template <typename T>
__global__ void k_gather(FieldView<T> f, GatherBatch b)
{
    const GatherDesc &q = b.p[blockIdx.y];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int npts = q.npts;
    if (p >= npts) return;
    T *slot = (T *)q.slot;
    const int64_t g = q.idx[p];
    slot[p] = f.Ex[g];
    slot[npts + p] = f.Ey[g];
    slot[2 * (int64_t)npts + p] = f.Ez[g];
    slot[3 * (int64_t)npts + p] = f.Hx[g];
    slot[4 * (int64_t)npts + p] = f.Hy[g];
    slot[5 * (int64_t)npts + p] = f.Hz[g];
}

template <typename R> struct Vec2;
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<double> { using type = double2; };

// phasor table [t][f] = (cos, sin)(w_f * n_t * dt), phases in FP64, stored in
// the contraction precision R
template <typename R>
__global__ void k_phasors(const double *omega, int nfreq, int nslots, int64_t n_first, double dt,
                          typename Vec2<R>::type *tab)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nslots * nfreq) return;
    const int t = q / nfreq, fi = q - t * nfreq;
    double s, c;
    sincos(omega[fi] * ((double)(n_first + t) * dt), &s, &c);
    tab[q].x = (R)c;
    tab[q].y = (R)s;
}

// Register-tiled contraction: a block of 256 threads covers 64 points x 64
// frequencies of one component; thread (tp, tf) accumulates points
// p0 + 16a + tp (a = 0..3) at frequencies f0 + 4tf + b (b = 0..3), so
// neighbouring lanes touch neighbouring points in shared memory and in the
// FP64 accumulators.  The block's samples [slots][64] and phasors
// [slots][64] are staged in shared memory.  Products and the sum over the
// (at most 64) slots of one flush run in the sample precision T; the block
// sums are then added to the FP64 accumulators, H components rotated by
// exp(+i w dt/2) (they sit half a step earlier).
constexpr int kPT = 64, kFT = 64, kMaxSlots = 64;

template <typename T>
__global__ void __launch_bounds__(256) k_dft(const T *ring, int npts, int nslots,
                                             const typename Vec2<T>::type *tab, const double *omega,
                                             int nfreq, double dt, const int32_t *comps, double *acc)
{
    using V = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char sh_raw[];
    T *ss = reinterpret_cast<T *>(sh_raw);                                // [nslots][kPT]
    V *sp = reinterpret_cast<V *>(sh_raw + sizeof(T) * kMaxSlots * kPT);  // [nslots][kFT]
    const int ci = blockIdx.y, p0 = blockIdx.x * kPT, f0 = blockIdx.z * kFT;
    const int comp = comps[ci];
    const int tid = threadIdx.x, tp = tid & 15, tf = tid >> 4;
    for (int q = tid; q < nslots * kPT; q += blockDim.x) {
        const int t = q / kPT, pl = q - t * kPT, p = p0 + pl;
        ss[q] = p < npts ? ring[((int64_t)t * 6 + comp) * npts + p] : T(0);
    }
    for (int q = tid; q < nslots * kFT; q += blockDim.x) {
        const int t = q / kFT, fl = q - t * kFT, f = f0 + fl;
        V z;
        z.x = T(0); z.y = T(0);
        sp[q] = f < nfreq ? tab[(int64_t)t * nfreq + f] : z;
    }
    __syncthreads();
    T re[4][4], im[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) { re[a][b] = T(0); im[a][b] = T(0); }
    for (int t = 0; t < nslots; ++t) {
        T sv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) sv[a] = ss[t * kPT + a * 16 + tp];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const V w = sp[t * kFT + tf * 4 + b];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                re[a][b] = fma(sv[a], w.x, re[a][b]);
                im[a][b] = fma(-sv[a], w.y, im[a][b]);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int f = f0 + tf * 4 + b;
        if (f >= nfreq) continue;
        double cs = 1.0, sn = 0.0;
        if (comp >= 3) sincos(omega[f] * (0.5 * dt), &sn, &cs);
        double *ar = acc + ((int64_t)(ci * nfreq + f) * 2) * npts;
        double *ai = ar + npts;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int p = p0 + a * 16 + tp;
            if (p >= npts) continue;
            const double r = (double)re[a][b], m = (double)im[a][b];
            ar[p] += r * cs - m * sn;
            ai[p] += r * sn + m * cs;
        }
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
void launch_port_gather(const FieldView<T> &f, const GatherBatch &b, cudaStream_t s)
{
    if (b.n <= 0 || b.max_npts <= 0) return;
    k_gather<T><<<dim3(cdiv(b.max_npts, 256), b.n), 256, 0, s>>>(f, b);
}

template <typename T>
void launch_port_dft(const T *ring, int npts, int nslots, int64_t n_first, double dt, const double *omega,
                     int nfreq, const int32_t *comps, int ncomp, double *acc, double *scratch_phasor,
                     cudaStream_t s)
{
    if (npts <= 0 || nslots <= 0 || nfreq <= 0 || ncomp <= 0) return;
    using V = typename Vec2<T>::type;
    V *tab = reinterpret_cast<V *>(scratch_phasor);
    k_phasors<T><<<cdiv((int64_t)nslots * nfreq, 256), 256, 0, s>>>(omega, nfreq, nslots, n_first, dt, tab);
    dim3 grid(cdiv(npts, kPT), ncomp, cdiv(nfreq, kFT));
    const size_t smem = (sizeof(T) * kPT + sizeof(V) * kFT) * kMaxSlots;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_dft<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_dft<T><<<grid, 256, smem, s>>>(ring, npts, nslots, tab, omega, nfreq, dt, comps, acc);
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
    template void launch_port_gather<T>(const FieldView<T> &, const GatherBatch &, cudaStream_t);          \
    template void launch_port_dft<T>(const T *, int, int, int64_t, double, const double *, int,            \
                                     const int32_t *, int, double *, double *, cudaStream_t);              \
    template void launch_count_nonfinite<T>(const FieldView<T> &, unsigned long long *, cudaStream_t);     \
    template void launch_to_device_layout<T>(const double *, T *, Dims, cudaStream_t);                     \
    template void launch_from_device_layout<T>(const T *, double *, Dims, cudaStream_t);
CPS_INST(double)
CPS_INST(float)

}  // namespace cps
