// kernels_plain.cu -- one kernel per reference routine ("plain" path).
//
// Compiled with --fmad=false: every multiply and add rounds on its own, in
// the reference's order, so the FP64 instantiation reproduces the reference
// arithmetic of BasicFDTD.cpp, CPML.cpp, TF_SF.cpp and the oracle's
// Drude-Lorentz/gain recursions operation by operation.
#include "batch.h"
#include "cells.cuh"

namespace cps {

namespace {

constexpr int kBY = 8;

// BasicHFieldUpdate, BasicFDTD.cpp:67-84: i,j,k in [0, N-1]
template <typename T>
__global__ void __launch_bounds__(32 * kBY) k_h_bulk(FieldView<T> f)
{
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * kBY + threadIdx.y, k = blockIdx.z;
    if (i >= f.d.nx || j >= f.d.ny) return;
    const int64_t g = f.d.idx(i, j, k), sy = f.d.px, sz = f.d.pxy;
    const int id = f.id[g];
    const T aH = f.aH[id], bH = f.bH[id];
    const StretchView<T> &s = f.s;
    f.Hx[g] = aH * f.Hx[g] - bH * (f.Ez[g + sy] - f.Ez[g]) * s.cHxz[j] + bH * (f.Ey[g + sz] - f.Ey[g]) * s.cHxy[k];
    f.Hy[g] = aH * f.Hy[g] - bH * (f.Ex[g + sz] - f.Ex[g]) * s.cHyx[k] + bH * (f.Ez[g + 1] - f.Ez[g]) * s.cHyz[i];
    f.Hz[g] = aH * f.Hz[g] + bH * (f.Ex[g + sy] - f.Ex[g]) * s.cHzx[j] - bH * (f.Ey[g + 1] - f.Ey[g]) * s.cHzy[i];
}

// BasicEFieldUpdate, BasicFDTD.cpp:25-47: i,j,k in [1, N-1]; ID 4 zeroes E,
// ID 2 is left to the Drude-Lorentz routine
template <typename T>
__global__ void __launch_bounds__(32 * kBY) k_e_bulk(FieldView<T> f)
{
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * kBY + threadIdx.y, k = blockIdx.z + 1;
    if (i < 1 || i >= f.d.nx || j < 1 || j >= f.d.ny) return;
    const int64_t g = f.d.idx(i, j, k), sy = f.d.px, sz = f.d.pxy;
    const int id = f.id[g];
    if (id == CPS_ID_PEC) {
        f.Ex[g] = T(0); f.Ey[g] = T(0); f.Ez[g] = T(0);
    } else if (id != CPS_ID_DISPERSIVE) {
        const T aE = f.aE[id], bE = f.bE[id];
        const StretchView<T> &s = f.s;
        f.Ex[g] = aE * f.Ex[g] + bE * (f.Hz[g] - f.Hz[g - sy]) * s.cExz[j] - bE * (f.Hy[g] - f.Hy[g - sz]) * s.cExy[k];
        f.Ey[g] = aE * f.Ey[g] + bE * (f.Hx[g] - f.Hx[g - sz]) * s.cEyx[k] - bE * (f.Hz[g] - f.Hz[g - 1]) * s.cEyz[i];
        f.Ez[g] = aE * f.Ez[g] + bE * (f.Hy[g] - f.Hy[g - 1]) * s.cEzy[i] - bE * (f.Hx[g] - f.Hx[g - sy]) * s.cEzx[j];
    }
}

// psi index of slab-local s at (i,j,k) for axis a (x: [k][j][s], y: [k][s][i], z: [s][j][i])
__device__ __forceinline__ int64_t psi_index(const Dims &d, int axis, int np, int s, int i, int j, int k)
{
    if (axis == 0) return ((int64_t)k * (d.ny + 1) + j) * psi_xw(np) + s;
    if (axis == 1) return ((int64_t)k * (np + 1) + s) * d.px + i;
    return ((int64_t)s * (d.ny + 1) + j) * d.px + i;
}

// CPML::UpdateCPMLEFields, one face: CPML.cpp:529-607.  Threads cover
// (u, v, w) = slab-local index plus the two transverse ranges [1, N-1].
template <typename T>
__global__ void k_e_pml_face(FieldView<T> f, PmlView<T> p, int face)
{
    const int axis = face >> 1, end = face & 1, np = p.np[face];
    const Dims &d = f.d;
    int i, j, k, s;
    if (axis == 0) {
        s = blockIdx.x * 32 + threadIdx.x; j = blockIdx.y * kBY + threadIdx.y + 1; k = blockIdx.z + 1;
        if (s >= np || j >= d.ny) return;
        i = end == 0 ? s + 1 : d.nx - np + s;
    } else if (axis == 1) {
        i = blockIdx.x * 32 + threadIdx.x + 1; s = blockIdx.y * kBY + threadIdx.y; k = blockIdx.z + 1;
        if (i >= d.nx || s >= np) return;
        j = end == 0 ? s + 1 : d.ny - np + s;
    } else {
        i = blockIdx.x * 32 + threadIdx.x + 1; j = blockIdx.y * kBY + threadIdx.y + 1; s = blockIdx.z;
        if (i >= d.nx || j >= d.ny) return;
        k = end == 0 ? s + 1 : d.nz - np + s;
    }
    const int cs = end == 0 ? s + 1 : s;  // coefficient index (CPML.cpp:534, 546)
    const int64_t g = d.idx(i, j, k), q = psi_index(d, axis, np, cs, i, j, k);
    const T b = p.bE[face][cs], c = p.cE[face][cs], ce = pml_ce_cell(p, f.bE, (int)f.id[g]);
    T *q0 = p.qe[face][0], *q1 = p.qe[face][1];
    if (axis == 0) {
        q0[q] = b * q0[q] + c * (f.Hz[g] - f.Hz[g - 1]);
        f.Ey[g] = f.Ey[g] - q0[q] * ce;
        q1[q] = b * q1[q] + c * (f.Hy[g] - f.Hy[g - 1]);
        f.Ez[g] = f.Ez[g] + q1[q] * ce;
    } else if (axis == 1) {
        q0[q] = b * q0[q] + c * (f.Hx[g] - f.Hx[g - d.px]);
        f.Ez[g] = f.Ez[g] - q0[q] * ce;
        q1[q] = b * q1[q] + c * (f.Hz[g] - f.Hz[g - d.px]);
        f.Ex[g] = f.Ex[g] + q1[q] * ce;
    } else {
        q0[q] = b * q0[q] + c * (f.Hy[g] - f.Hy[g - d.pxy]);
        f.Ex[g] = f.Ex[g] - q0[q] * ce;
        q1[q] = b * q1[q] + c * (f.Hx[g] - f.Hx[g - d.pxy]);
        f.Ey[g] = f.Ey[g] + q1[q] * ce;
    }
}

// CPML::UpdateCPMLHFields, one face: CPML.cpp:609-689; transverse ranges [0, N-1]
template <typename T>
__global__ void k_h_pml_face(FieldView<T> f, PmlView<T> p, int face)
{
    const int axis = face >> 1, end = face & 1, np = p.np[face];
    const Dims &d = f.d;
    int i, j, k, s;
    if (axis == 0) {
        s = blockIdx.x * 32 + threadIdx.x; j = blockIdx.y * kBY + threadIdx.y; k = blockIdx.z;
        if (s >= np || j >= d.ny) return;
        i = end == 0 ? s : d.nx - np + s;
    } else if (axis == 1) {
        i = blockIdx.x * 32 + threadIdx.x; s = blockIdx.y * kBY + threadIdx.y; k = blockIdx.z;
        if (i >= d.nx || s >= np) return;
        j = end == 0 ? s : d.ny - np + s;
    } else {
        i = blockIdx.x * 32 + threadIdx.x; j = blockIdx.y * kBY + threadIdx.y; s = blockIdx.z;
        if (i >= d.nx || j >= d.ny) return;
        k = end == 0 ? s : d.nz - np + s;
    }
    const int64_t g = d.idx(i, j, k), q = psi_index(d, axis, np, s, i, j, k);
    const T b = p.bH[face][s], c = p.cH[face][s], ch = pml_ch_cell(p, f.bH, (int)f.id[g]);
    T *q0 = p.qh[face][0], *q1 = p.qh[face][1];
    if (axis == 0) {
        q0[q] = b * q0[q] + c * (f.Ez[g + 1] - f.Ez[g]);
        f.Hy[g] = f.Hy[g] + q0[q] * ch;
        q1[q] = b * q1[q] + c * (f.Ey[g + 1] - f.Ey[g]);
        f.Hz[g] = f.Hz[g] - q1[q] * ch;
    } else if (axis == 1) {
        q0[q] = b * q0[q] + c * (f.Ex[g + d.px] - f.Ex[g]);
        f.Hz[g] = f.Hz[g] - q0[q] * ch;
        q1[q] = b * q1[q] + c * (f.Ez[g + d.px] - f.Ez[g]);
        f.Hx[g] = f.Hx[g] + q1[q] * ch;
    } else {
        q0[q] = b * q0[q] + c * (f.Ey[g + d.pxy] - f.Ey[g]);
        f.Hx[g] = f.Hx[g] - q0[q] * ch;
        q1[q] = b * q1[q] + c * (f.Ex[g + d.pxy] - f.Ex[g]);
        f.Hy[g] = f.Hy[g] + q1[q] * ch;
    }
}

__device__ __forceinline__ void decode(const Dims &d, int64_t g, int &i, int &j, int &k)
{
    k = (int)(g / d.pxy);
    const int64_t r = g - (int64_t)k * d.pxy;
    j = (int)(r / d.px);
    i = (int)(r - (int64_t)j * d.px);
}

// 3-D Drude-Lorentz ADE on the ID==2 cell list (Drude_Lorentz.cpp:153-227
// with the curl terms of BasicFDTD.cpp:39-41 and bE replaced by C3)
template <typename T>
__global__ void k_dl(FieldView<T> f, DlView<T> D)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= D.ncell) return;
    const int64_t g = D.cell[c];
    int i, j, k;
    decode(f.d, g, i, j, k);
    const int64_t sy = f.d.px, sz = f.d.pxy;
    const StretchView<T> &s = f.s;
    const T C3 = D.c.C3;
    const T cx = C3 * (f.Hz[g] - f.Hz[g - sy]) * s.cExz[j] - C3 * (f.Hy[g] - f.Hy[g - sz]) * s.cExy[k];
    const T cy = C3 * (f.Hx[g] - f.Hx[g - sz]) * s.cEyx[k] - C3 * (f.Hz[g] - f.Hz[g - 1]) * s.cEyz[i];
    const T cz = C3 * (f.Hy[g] - f.Hy[g - 1]) * s.cEzy[i] - C3 * (f.Hx[g] - f.Hx[g - sy]) * s.cEzx[j];
    const int64_t sc = D.ncell;
    T *st = D.state + c;
    f.Ex[g] = dl_component(D.c, f.Ex[g], cx, st, sc);
    f.Ey[g] = dl_component(D.c, f.Ey[g], cy, st + (int64_t)D.c.stride * sc, sc);
    f.Ez[g] = dl_component(D.c, f.Ez[g], cz, st + (int64_t)2 * D.c.stride * sc, sc);
}

// FourLevelLaser routines on the gain cell list: which 0 = polarization
// (:270-298), 1 = E correction (:300-308), 2 = populations (:310-325)
template <typename T, typename L>
__global__ void k_gain(FieldView<T> f, GainView<T> G, int which)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= G.ncell) return;
    const int64_t g = G.cell[c], sc = kGainGroup;
    // persistent words (stride 32 in both layouts) and the transient words
    // Pa2 Pb2 E1 (FP32: their own list-layout array)
    T *st, *tr;
    if (sizeof(T) == 4) {
        st = G.state + gain_dense_index(g);
        tr = G.trans + gain_base_index(c, kGainTrans);
    } else {
        st = G.state + gain_base_index(c, kG64Words);
        tr = st;
    }
    auto tw = [&](int w) -> T & { return sizeof(T) == 4 ? tr[(w - kGainPersist) * sc] : st[w * sc]; };
    T *F[3] = {f.Ex, f.Ey, f.Ez};
    T E[3] = {F[0][g], F[1][g], F[2][g]};
    T Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3];
    for (int q = 0; q < 3; ++q) {
        Pa[q] = st[(L::PA + q) * sc]; Pa1[q] = st[(L::PA1 + q) * sc];
        Pb[q] = st[(L::PB + q) * sc]; Pb1[q] = st[(L::PB1 + q) * sc];
    }
    if (which == 0) {
        Pops<T> N;
        gain_load_n<T>(st, sc, N);
        gain_p_update<T>(G.c, N, E, Pa, Pa1, Pa2, Pb, Pb1, Pb2);
        for (int q = 0; q < 3; ++q) {
            st[(L::PA + q) * sc] = Pa[q]; st[(L::PA1 + q) * sc] = Pa1[q]; tw(L::PA2 + q) = Pa2[q];
            st[(L::PB + q) * sc] = Pb[q]; st[(L::PB1 + q) * sc] = Pb1[q]; tw(L::PB2 + q) = Pb2[q];
            tw(L::E1 + q) = E[q];
        }
    } else if (which == 1) {
        for (int q = 0; q < 3; ++q) F[q][g] = gain_e_corr<T>(G.c, E[q], Pa[q], Pa1[q], Pb[q], Pb1[q]);
    } else {
        Pops<T> N;
        T E1[3];
        gain_load_n<T>(st, sc, N);
        for (int q = 0; q < 3; ++q) {
            Pa2[q] = tw(L::PA2 + q); Pb2[q] = tw(L::PB2 + q); E1[q] = tw(L::E1 + q);
        }
        gain_n_update<T>(G.c, N, E, E1, Pa, Pa1, Pa2, Pb, Pb2);
        gain_store_n<T>(st, sc, N);
    }
}

// FP32 population offsets of each list cell for the host read-out
__global__ void k_gain_pops32(const float *state, const int64_t *cell, int64_t ncell, float *out)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    const float *st = state + gain_dense_index(cell[c]);
    for (int q = 0; q < 3; ++q) out[c * 3 + q] = st[(GainSite32::DN1 + q) * kGainGroup];
}

// FP64 initial populations N0 = N1 = 1 (words 21, 22 of each cell)
__global__ void k_gain_init64(double *state, int64_t ncell)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncell) return;
    double *st = state + gain_base_index(c, kG64Words);
    st[GainSite64::N * kGainGroup] = 1.0;
    st[(GainSite64::N + 1) * kGainGroup] = 1.0;
}

// TF/SF (and any other table-driven) injection in CSR form: each thread owns
// one (cell, component) target and adds its contributions in order,
// F += coef * inc(n - delay) * profile (TF_SF.cpp:992-1087, 1206-1299)
// one TF/SF target: its contributions in the reference's face order
template <typename T>
__device__ __forceinline__ T inject_add(T v, const InjContrib &a, const T *table, int Nt, double n)
{
    const T inc = (T)inc_lookup<T>(table, Nt, n - a.delay);
    return v + (T)a.coef * inc * (T)a.profile;
}

template <typename T>
__device__ __forceinline__ void inject_target(const FieldView<T> &f, const InjTarget &q, const InjContrib *ct,
                                              const T *table, int Nt, double n, uint32_t face_mask)
{
    T *F = field_comp(f, q.comp) + q.idx;
    T v = *F;
    for (int c = q.start; c < q.start + q.count; ++c) {
        const InjContrib a = ct[c];
        if (!(face_mask & (1u << a.face))) continue;
        v = inject_add(v, a, table, Nt, n);
    }
    *F = v;
}

template <typename T>
__global__ void k_inject(FieldView<T> f, const InjTarget *tg, int ntarget, const InjContrib *ct,
                         const T *table, int Nt, double n, uint32_t face_mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntarget) return;
    inject_target<T>(f, tg[t], ct, table, Nt, n, face_mask);
}

// batched forms: the step number is the grid's chunk start plus step_off.
// A block entry covers kInjPerBlock targets; each thread takes two of them,
// kInjThreads apart, and requests both targets' records, field values and
// first contributions before using any (the kernel is bound by the latency
// of these dependent loads).  Each target's contributions are added in its
// own order, as in inject_target; the two targets are distinct (cell,
// component) pairs, so their updates are independent.
template <typename T>
__global__ void __launch_bounds__(kInjThreads) k_inject_batch(const BatchGrid<T> *__restrict__ grids,
                                                              const int4 *__restrict__ blocks, int side,
                                                              int step_off)
{
    const int4 e = blocks[blockIdx.x];
    const int t0 = e.y + (int)threadIdx.x, t1 = t0 + kInjThreads;
    if (t0 >= e.z) return;
    const bool two = t1 < e.z;
    const BatchGrid<T> &B = grids[e.x];
    const InjTarget *tg = B.tg[side];
    const InjContrib *ct = B.ct[side];
    const T *table = B.inc[side];
    const int Nt = B.Nt;
    const double n = (double)(B.n0 + step_off);
    const InjTarget q0 = tg[t0];
    const InjTarget q1 = two ? tg[t1] : q0;
    T *F0 = field_comp(B.f, q0.comp) + q0.idx;
    T *F1 = field_comp(B.f, q1.comp) + q1.idx;
    T v0 = *F0;
    T v1 = two ? *F1 : T(0);
    const InjContrib a0 = ct[q0.start];  // every target has at least one contribution
    const InjContrib a1 = ct[q1.start];
    v0 = inject_add(v0, a0, table, Nt, n);
    for (int c = q0.start + 1; c < q0.start + q0.count; ++c) v0 = inject_add(v0, ct[c], table, Nt, n);
    *F0 = v0;
    if (!two) return;
    v1 = inject_add(v1, a1, table, Nt, n);
    for (int c = q1.start + 1; c < q1.start + q1.count; ++c) v1 = inject_add(v1, ct[c], table, Nt, n);
    *F1 = v1;
}

template <typename T>
__global__ void k_sources_batch(const BatchGrid<T> *__restrict__ grids, const int2 *__restrict__ ents, int n,
                                int step_off)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const int2 e = ents[q];
    const BatchGrid<T> &B = grids[e.x];
    const int s = e.y;
    const int64_t nn = B.n0 + step_off;
    if (nn < 0 || nn >= B.src_len[s]) return;
    const FieldView<T> &f = B.f;
    T *F[6] = {f.Ex, f.Ey, f.Ez, f.Hx, f.Hy, f.Hz};
    const int64_t g = B.src_idx[s];
    T *dst = F[B.src_comp[s]];
    dst[g] = dst[g] + (T)B.src_wave[B.src_off[s] + nn];
}

template <typename T>
__global__ void k_sources(FieldView<T> f, int nsrc, const int64_t *idx, const int32_t *comp,
                          const double *waves, const int32_t *off, const int32_t *len, int n)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nsrc || n < 0 || n >= len[s]) return;
    T *F[6] = {f.Ex, f.Ey, f.Ez, f.Hx, f.Hy, f.Hz};
    F[comp[s]][idx[s]] = F[comp[s]][idx[s]] + (T)waves[off[s] + n];
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

}  // namespace

template <typename T>
void launch_h_bulk(const FieldView<T> &f, cudaStream_t s)
{
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, kBY), f.d.nz);
    k_h_bulk<T><<<grid, dim3(32, kBY), 0, s>>>(f);
}

template <typename T>
void launch_e_bulk(const FieldView<T> &f, cudaStream_t s)
{
    if (f.d.nz < 2) return;
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, kBY), f.d.nz - 1);
    k_e_bulk<T><<<grid, dim3(32, kBY), 0, s>>>(f);
}

template <typename T>
void launch_e_pml(const FieldView<T> &f, const PmlView<T> &p, cudaStream_t s)
{
    const Dims &d = f.d;
    for (int face = 0; face < 6; ++face) {  // reference order x1 x2 y1 y2 z1 z2
        const int np = p.np[face];
        if (np <= 0) continue;
        dim3 grid;
        if (face < 2) grid = dim3(cdiv(np, 32), cdiv(d.ny - 1, kBY), d.nz - 1);
        else if (face < 4) grid = dim3(cdiv(d.nx - 1, 32), cdiv(np, kBY), d.nz - 1);
        else grid = dim3(cdiv(d.nx - 1, 32), cdiv(d.ny - 1, kBY), np);
        k_e_pml_face<T><<<grid, dim3(32, kBY), 0, s>>>(f, p, face);
    }
}

template <typename T>
void launch_h_pml(const FieldView<T> &f, const PmlView<T> &p, cudaStream_t s)
{
    const Dims &d = f.d;
    for (int face = 0; face < 6; ++face) {
        const int np = p.np[face];
        if (np <= 0) continue;
        dim3 grid;
        if (face < 2) grid = dim3(cdiv(np, 32), cdiv(d.ny, kBY), d.nz);
        else if (face < 4) grid = dim3(cdiv(d.nx, 32), cdiv(np, kBY), d.nz);
        else grid = dim3(cdiv(d.nx, 32), cdiv(d.ny, kBY), np);
        k_h_pml_face<T><<<grid, dim3(32, kBY), 0, s>>>(f, p, face);
    }
}

template <typename T>
void launch_dl(const FieldView<T> &f, const DlView<T> &d, cudaStream_t s)
{
    if (d.ncell <= 0) return;
    k_dl<T><<<cdiv(d.ncell, 128), 128, 0, s>>>(f, d);
}

template <typename T>
void launch_gain(const FieldView<T> &f, const GainView<T> &g, int which, cudaStream_t s)
{
    if (g.ncell <= 0) return;
    if (sizeof(T) == 8)
        k_gain<T, GainSite64><<<cdiv(g.ncell, 128), 128, 0, s>>>(f, g, which);
    else
        k_gain<T, GainSite32><<<cdiv(g.ncell, 128), 128, 0, s>>>(f, g, which);
}

void launch_gain_pops32(const float *state, const int64_t *cell, int64_t ncell, float *out, cudaStream_t s)
{
    if (ncell <= 0) return;
    k_gain_pops32<<<cdiv(ncell, 256), 256, 0, s>>>(state, cell, ncell, out);
}

void launch_gain_init64(double *state, int64_t ncell, cudaStream_t s)
{
    if (ncell <= 0) return;
    k_gain_init64<<<cdiv(ncell, 256), 256, 0, s>>>(state, ncell);
}

template <typename T>
void launch_inject(const FieldView<T> &f, const InjTarget *tg, int ntarget, const InjContrib *ct,
                   const T *table, int Nt, double n, uint32_t face_mask, cudaStream_t s)
{
    if (ntarget <= 0) return;
    k_inject<T><<<cdiv(ntarget, 128), 128, 0, s>>>(f, tg, ntarget, ct, table, Nt, n, face_mask);
}

template <typename T>
void launch_sources(const FieldView<T> &f, int nsrc, const int64_t *idx, const int32_t *comp,
                    const double *waves, const int32_t *wave_off, const int32_t *wave_len, int n,
                    cudaStream_t s)
{
    if (nsrc <= 0) return;
    k_sources<T><<<cdiv(nsrc, 64), 64, 0, s>>>(f, nsrc, idx, comp, waves, wave_off, wave_len, n);
}

template <typename T>
void launch_inject_batch(const BatchGrid<T> *grids, const int4 *blocks, int nblocks, int side, int step_off,
                         cudaStream_t s)
{
    if (nblocks <= 0) return;
    k_inject_batch<T><<<nblocks, kInjThreads, 0, s>>>(grids, blocks, side, step_off);
}

template <typename T>
void launch_sources_batch(const BatchGrid<T> *grids, const int2 *ents, int n, int step_off, cudaStream_t s)
{
    if (n <= 0) return;
    k_sources_batch<T><<<cdiv(n, 64), 64, 0, s>>>(grids, ents, n, step_off);
}

#define CPS_INSTANTIATE(T)                                                                              \
    template void launch_h_bulk<T>(const FieldView<T> &, cudaStream_t);                                 \
    template void launch_e_bulk<T>(const FieldView<T> &, cudaStream_t);                                 \
    template void launch_h_pml<T>(const FieldView<T> &, const PmlView<T> &, cudaStream_t);              \
    template void launch_e_pml<T>(const FieldView<T> &, const PmlView<T> &, cudaStream_t);              \
    template void launch_dl<T>(const FieldView<T> &, const DlView<T> &, cudaStream_t);                  \
    template void launch_gain<T>(const FieldView<T> &, const GainView<T> &, int, cudaStream_t);         \
    template void launch_inject<T>(const FieldView<T> &, const InjTarget *, int, const InjContrib *,    \
                                   const T *, int, double, uint32_t, cudaStream_t);                     \
    template void launch_sources<T>(const FieldView<T> &, int, const int64_t *, const int32_t *,        \
                                    const double *, const int32_t *, const int32_t *, int, cudaStream_t); \
    template void launch_inject_batch<T>(const BatchGrid<T> *, const int4 *, int, int, int, cudaStream_t); \
    template void launch_sources_batch<T>(const BatchGrid<T> *, const int2 *, int, int, cudaStream_t);
CPS_INSTANTIATE(double)
CPS_INSTANTIATE(float)

}  // namespace cps
