// kernels_ports.cu -- port sampling, the blocked FP64 port DFT, flux
// reduction, a non-finite watchdog and host<->device layout conversion.
//
// Port samples of every step are gathered into a ring of slots
// ([slot][component][point], float on FP32 grids).  Every 64 steps (and
// before a read-out) one contraction folds the ring into FP64 accumulators,
//   acc[c][f][p] += s[t][c][p] * exp(-i w_f t_c(n_t))   for t in slot order,
// with t_c = n dt for E and (n - 1/2) dt for H: a [P x T] by [T x F] complex
// product per component in which every sample is added to the accumulators
// on its own, in FP64, so the sums do not depend on how samples are grouped
// into flushes.  The FP64 phasors of a flush are tabulated once into a
// scratch table [2][slots][nfreq] (E time, then H time).
#include "batch.h"
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

// phasor table of a flush: tab[0][t][f] = (cos, sin)(w_f n_t dt) and
// tab[1][t][f] = (cos, sin)(w_f (n_t - 1/2) dt), n_t = n_first + t, phases
// formed as w * (n dt) the way the FP64 oracle forms them; cap = slots of
// each half
__device__ __forceinline__ void phasor_entry(const double *omega, int nfreq, int cap, int64_t n_first, double dt,
                                             int q, double2 *tab)
{
    const int t = q / nfreq, fi = q - t * nfreq;
    const double n = (double)(n_first + t);
    double s, c;
    sincos(omega[fi] * (n * dt), &s, &c);
    tab[q] = make_double2(c, s);
    sincos(omega[fi] * ((n - 0.5) * dt), &s, &c);
    tab[(int64_t)cap * nfreq + q] = make_double2(c, s);
}

__global__ void k_phasors(const double *omega, int nfreq, int nslots, int64_t n_first, double dt, double2 *tab)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nslots * nfreq) return;
    phasor_entry(omega, nfreq, nslots, n_first, dt, q, tab);
}

// Contraction of one flush: a block of 256 threads covers PT points x FT
// frequencies of one component (64 x 64, or 128 x 32 for ports with at most
// 32 frequencies); thread (tp, tf), tp < PT/4, tf < FT/4, owns points
// p0 + (PT/4)a + tp (a = 0..3) at frequencies f0 + 4tf + b (b = 0..3), so
// neighbouring lanes touch neighbouring points in shared memory and in the
// accumulators.  The block's samples [slots][PT] and phasors [slots][FT] are
// staged in shared memory; each thread loads its 16 FP64 accumulator pairs,
// adds the samples one slot at a time (acc_re += s cos, acc_im -= s sin,
// FP64 fused multiply-adds) and stores them back.  Every accumulator sees
// the same operations in the same order whatever the tile.
constexpr int kMaxSlots = 64;
// shared memory of either tile: samples [slots][PT] + phasors [slots][FT]
constexpr size_t kDftSmem(size_t esz)
{
    return (esz * 64 + sizeof(double2) * 64) * kMaxSlots > (esz * 128 + sizeof(double2) * 32) * kMaxSlots
               ? (esz * 64 + sizeof(double2) * 64) * kMaxSlots
               : (esz * 128 + sizeof(double2) * 32) * kMaxSlots;
}

template <typename T, int FT>
__device__ __forceinline__ void dft_tile(const T *ring, int npts, int nslots, const double2 *tab, int nfreq,
                                         int comp, int ci, int p0, int f0, double *acc, unsigned char *sh_raw)
{
    constexpr int TF = FT / 4, TP = 256 / TF, PT = 4 * TP;
    T *ss = reinterpret_cast<T *>(sh_raw);                                          // [nslots][PT]
    double2 *sp = reinterpret_cast<double2 *>(sh_raw + sizeof(T) * kMaxSlots * PT);  // [nslots][FT]
    const int tid = threadIdx.x, tp = tid % TP, tf = tid / TP;
    for (int q = tid; q < nslots * PT; q += blockDim.x) {
        const int t = q / PT, pl = q - t * PT, p = p0 + pl;
        ss[q] = p < npts ? ring[((int64_t)t * 6 + comp) * npts + p] : T(0);
    }
    for (int q = tid; q < nslots * FT; q += blockDim.x) {
        const int t = q / FT, fl = q - t * FT, f = f0 + fl;
        sp[q] = f < nfreq ? tab[(int64_t)t * nfreq + f] : make_double2(0.0, 0.0);
    }
    double re[4][4], im[4][4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int f = f0 + tf * 4 + b;
        const double *ar = acc + ((int64_t)(ci * nfreq + min(f, nfreq - 1)) * 2) * npts;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int p = p0 + a * TP + tp;
            const bool ok = f < nfreq && p < npts;
            re[a][b] = ok ? ar[p] : 0.0;
            im[a][b] = ok ? ar[npts + p] : 0.0;
        }
    }
    __syncthreads();
    for (int t = 0; t < nslots; ++t) {
        double sv[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) sv[a] = (double)ss[t * PT + a * TP + tp];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const double2 w = sp[t * FT + tf * 4 + b];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                re[a][b] = __fma_rn(sv[a], w.x, re[a][b]);
                im[a][b] = __fma_rn(-sv[a], w.y, im[a][b]);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        const int f = f0 + tf * 4 + b;
        if (f >= nfreq) continue;
        double *ar = acc + ((int64_t)(ci * nfreq + f) * 2) * npts;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int p = p0 + a * TP + tp;
            if (p >= npts) continue;
            ar[p] = re[a][b];
            ar[npts + p] = im[a][b];
        }
    }
}

// block (pb, fb) of a port's contraction, with the port's tile
template <typename T>
__device__ __forceinline__ void dft_block(const T *ring, int npts, int nslots, const double2 *tab, int nfreq,
                                          int comp, int ci, int pb, int fb, double *acc, unsigned char *sh_raw)
{
    if (dft_freq_tile(nfreq) == 32)
        dft_tile<T, 32>(ring, npts, nslots, tab, nfreq, comp, ci, pb * 128, fb * 32, acc, sh_raw);
    else
        dft_tile<T, 64>(ring, npts, nslots, tab, nfreq, comp, ci, pb * 64, fb * 64, acc, sh_raw);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_dft(const T *ring, int npts, int nslots, const double2 *tab, int nfreq,
                                             const int32_t *comps, double *acc)
{
    extern __shared__ __align__(16) unsigned char sh_raw[];
    const int ci = blockIdx.y, comp = comps[ci];
    dft_block<T>(ring, npts, nslots, tab + (comp >= 3 ? (int64_t)nslots * nfreq : 0), nfreq, comp, ci,
                 blockIdx.x, blockIdx.z, acc, sh_raw);
}

// batched forms over the ports of many grids
// A chunk's rings are read only by its DFT contraction (the components the
// port transforms) and by the last-sample read-out (the slot of the chunk's
// last step, all six components).  So the last step (last_off) samples all
// six components, earlier steps only the transformed ones, and a port without
// a DFT (one slot, overwritten every step) only the last step.
template <typename T>
__global__ void k_gather_batch(const BatchGrid<T> *__restrict__ grids, const BatchPort<T> *__restrict__ ports,
                               const int2 *__restrict__ blocks, int step_off, int last_off)
{
    const int2 e = blocks[blockIdx.x];
    const BatchPort<T> &P = ports[e.x];
    const bool last = step_off == last_off;
    if (!last && P.slots == 1) return;
    const int p = e.y + (int)threadIdx.x;
    const int npts = P.npts;
    if (p >= npts) return;
    const FieldView<T> &f = grids[P.grid].f;
    T *slot = P.ring + (int64_t)(P.slots == 1 ? 0 : step_off) * 6 * npts;
    const int64_t g = P.idx[p];
    if (last) {
        slot[p] = f.Ex[g];
        slot[npts + p] = f.Ey[g];
        slot[2 * (int64_t)npts + p] = f.Ez[g];
        slot[3 * (int64_t)npts + p] = f.Hx[g];
        slot[4 * (int64_t)npts + p] = f.Hy[g];
        slot[5 * (int64_t)npts + p] = f.Hz[g];
        return;
    }
    const int nc = P.ncomp;
    T v[6];
#pragma unroll
    for (int ci = 0; ci < 6; ++ci)  // every load before the first store
        if (ci < nc) v[ci] = field_comp(f, __ldg(&P.comps[ci]))[g];
#pragma unroll
    for (int ci = 0; ci < 6; ++ci)
        if (ci < nc) slot[(int64_t)__ldg(&P.comps[ci]) * npts + p] = v[ci];
}

template <typename T>
__global__ void k_phasors_batch(const BatchGrid<T> *__restrict__ grids, const BatchPort<T> *__restrict__ ports,
                                const int2 *__restrict__ blocks, int nslots)
{
    const int2 e = blocks[blockIdx.x];
    const BatchPort<T> &P = ports[e.x];
    const int q = e.y + (int)threadIdx.x;
    if (q >= nslots * P.nfreq) return;
    const BatchGrid<T> &B = grids[P.grid];
    phasor_entry(P.omega, P.nfreq, kMaxRing, B.n0, B.dt, q, P.tab);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_dft_batch(const BatchPort<T> *__restrict__ ports,
                                                   const int4 *__restrict__ blocks, int nslots)
{
    extern __shared__ __align__(16) unsigned char sh_raw[];
    const int4 e = blocks[blockIdx.x];
    const BatchPort<T> &P = ports[e.x];
    const int comp = P.comps[e.z];
    dft_block<T>(P.ring, P.npts, nslots, P.tab + (comp >= 3 ? (int64_t)kMaxRing * P.nfreq : 0), P.nfreq, comp, e.z,
                 e.y, e.w, P.acc, sh_raw);
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
    double2 *tab = reinterpret_cast<double2 *>(scratch_phasor);
    k_phasors<<<cdiv((int64_t)nslots * nfreq, 256), 256, 0, s>>>(omega, nfreq, nslots, n_first, dt, tab);
    dim3 grid(cdiv(npts, dft_point_tile(nfreq)), ncomp, cdiv(nfreq, dft_freq_tile(nfreq)));
    if (!kernel_smem<k_dft<T>>((int)kDftSmem(sizeof(T)))) return;
    k_dft<T><<<grid, 256, kDftSmem(sizeof(T)), s>>>(ring, npts, nslots, tab, nfreq, comps, acc);
}

template <typename T>
void launch_gather_batch(const BatchGrid<T> *grids, const BatchPort<T> *ports, const int2 *blocks, int nblocks,
                         int step_off, int last_off, cudaStream_t s)
{
    if (nblocks <= 0) return;
    k_gather_batch<T><<<nblocks, 256, 0, s>>>(grids, ports, blocks, step_off, last_off);
}

template <typename T>
bool dft_batch_attributes()
{
    return kernel_smem<k_dft_batch<T>>((int)kDftSmem(sizeof(T)));
}

template <typename T>
void launch_dft_batch(const BatchGrid<T> *grids, const BatchPort<T> *ports, const int2 *ph_blocks, int nph,
                      const int4 *blocks, int nblocks, int nslots, cudaStream_t s)
{
    if (nph <= 0 || nblocks <= 0 || nslots <= 0) return;
    k_phasors_batch<T><<<nph, 256, 0, s>>>(grids, ports, ph_blocks, nslots);
    if (!dft_batch_attributes<T>()) return;
    k_dft_batch<T><<<nblocks, 256, kDftSmem(sizeof(T)), s>>>(ports, blocks, nslots);
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
    template void launch_from_device_layout<T>(const T *, double *, Dims, cudaStream_t);                   \
    template void launch_gather_batch<T>(const BatchGrid<T> *, const BatchPort<T> *, const int2 *, int, int, \
                                         int, cudaStream_t);                                               \
    template void launch_dft_batch<T>(const BatchGrid<T> *, const BatchPort<T> *, const int2 *, int,       \
                                      const int4 *, int, int, cudaStream_t);                             \
    template bool dft_batch_attributes<T>();
CPS_INST(double)
CPS_INST(float)

}  // namespace cps
