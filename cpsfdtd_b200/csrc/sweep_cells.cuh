// sweep_cells.cuh -- per-cell pieces of the fused sweeps that do not depend
// on how the field values reached the thread (registers or a TMA-staged
// shared-memory tile): CPML psi corrections and the Drude-Lorentz / gain
// updates looked up on their compacted lists.
#pragma once

#include "cells.cuh"

namespace cps {

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// CPML slab membership of a column, fixed along the k march
template <typename T>
struct ColPml {
    int fx, sxl, fy, syl;
    T bx, cx, by, cy;
};

// E side: x slabs cover i in [1, np] and [nx-np, nx-1] (CPML.cpp:534-556)
template <typename T>
__device__ __forceinline__ ColPml<T> col_pml_e(const PmlView<T> &p, const Dims &d, int i, int j, bool act)
{
    ColPml<T> c{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
    if (act && i <= p.np[kFX1]) { c.fx = kFX1; c.sxl = i; }
    else if (act && i >= d.nx - p.np[kFX2]) { c.fx = kFX2; c.sxl = i - (d.nx - p.np[kFX2]); }
    if (j <= p.np[kFY1]) { c.fy = kFY1; c.syl = j; }
    else if (j >= d.ny - p.np[kFY2]) { c.fy = kFY2; c.syl = j - (d.ny - p.np[kFY2]); }
    if (c.fx >= 0) { c.bx = p.bE[c.fx][c.sxl]; c.cx = p.cE[c.fx][c.sxl]; }
    if (c.fy >= 0) { c.by = p.bE[c.fy][c.syl]; c.cy = p.cE[c.fy][c.syl]; }
    return c;
}

// H side: x slabs cover i in [0, np-1] and [nx-np, nx-1] (CPML.cpp:614-636)
template <typename T>
__device__ __forceinline__ ColPml<T> col_pml_h(const PmlView<T> &p, const Dims &d, int i, int j, bool act)
{
    ColPml<T> c{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
    if (act && i < p.np[kFX1]) { c.fx = kFX1; c.sxl = i; }
    else if (act && i >= d.nx - p.np[kFX2]) { c.fx = kFX2; c.sxl = i - (d.nx - p.np[kFX2]); }
    if (j < p.np[kFY1]) { c.fy = kFY1; c.syl = j; }
    else if (j >= d.ny - p.np[kFY2]) { c.fy = kFY2; c.syl = j - (d.ny - p.np[kFY2]); }
    if (c.fx >= 0) { c.bx = p.bH[c.fx][c.sxl]; c.cx = p.cH[c.fx][c.sxl]; }
    if (c.fy >= 0) { c.by = p.bH[c.fy][c.syl]; c.cy = p.cH[c.fy][c.syl]; }
    return c;
}

// CPML H corrections at one cell (CPML.cpp:617-682), x then y then z slabs
template <typename T>
__device__ __forceinline__ void pml_h_cell(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, T ch, int i,
                                           int j, int k, T dEz_i, T dEy_i, T dEx_j, T dEz_j, T dEy_k, T dEx_k, T &hx,
                                           T &hy, T &hz)
{
    if (c.fx >= 0) {
        const int np = p.np[c.fx];
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(np) + c.sxl;
        T *q0 = p.qh[c.fx][0], *q1 = p.qh[c.fx][1];
        const T a0 = c.bx * q0[q] + c.cx * dEz_i, a1 = c.bx * q1[q] + c.cx * dEy_i;
        q0[q] = a0; q1[q] = a1;
        hy = hy + a0 * ch;
        hz = hz - a1 * ch;
    }
    if (c.fy >= 0) {
        const int np = p.np[c.fy];
        const int64_t q = ((int64_t)k * (np + 1) + c.syl) * d.px + i;
        T *q0 = p.qh[c.fy][0], *q1 = p.qh[c.fy][1];
        const T a0 = c.by * q0[q] + c.cy * dEx_j, a1 = c.by * q1[q] + c.cy * dEz_j;
        q0[q] = a0; q1[q] = a1;
        hz = hz - a0 * ch;
        hx = hx + a1 * ch;
    }
    int fz = -1, szl = 0;
    if (k < p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        T *q0 = p.qh[fz][0], *q1 = p.qh[fz][1];
        const T b = p.bH[fz][szl], cc = p.cH[fz][szl];
        const T a0 = b * q0[q] + cc * dEy_k, a1 = b * q1[q] + cc * dEx_k;
        q0[q] = a0; q1[q] = a1;
        hx = hx - a0 * ch;
        hy = hy + a1 * ch;
    }
}

// CPML E corrections at one cell (CPML.cpp:537-602), x then y then z slabs
template <typename T>
__device__ __forceinline__ void pml_e_cell(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, T ce, int i,
                                           int j, int k, T dHz_i, T dHy_i, T dHx_j, T dHz_j, T dHy_k, T dHx_k, T &ex,
                                           T &ey, T &ez)
{
    if (c.fx >= 0) {
        const int np = p.np[c.fx];
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(np) + c.sxl;
        T *q0 = p.qe[c.fx][0], *q1 = p.qe[c.fx][1];
        const T a0 = c.bx * q0[q] + c.cx * dHz_i, a1 = c.bx * q1[q] + c.cx * dHy_i;
        q0[q] = a0; q1[q] = a1;
        ey = ey - a0 * ce;
        ez = ez + a1 * ce;
    }
    if (c.fy >= 0) {
        const int np = p.np[c.fy];
        const int64_t q = ((int64_t)k * (np + 1) + c.syl) * d.px + i;
        T *q0 = p.qe[c.fy][0], *q1 = p.qe[c.fy][1];
        const T a0 = c.by * q0[q] + c.cy * dHx_j, a1 = c.by * q1[q] + c.cy * dHz_j;
        q0[q] = a0; q1[q] = a1;
        ez = ez - a0 * ce;
        ex = ex + a1 * ce;
    }
    int fz = -1, szl = 0;
    if (k <= p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        T *q0 = p.qe[fz][0], *q1 = p.qe[fz][1];
        const T b = p.bE[fz][szl], cc = p.cE[fz][szl];
        const T a0 = b * q0[q] + cc * dHy_k, a1 = b * q1[q] + cc * dHx_k;
        q0[q] = a0; q1[q] = a1;
        ex = ex - a0 * ce;
        ey = ey + a1 * ce;
    }
}

// psi words of one cell, loaded a plane ahead of their use
template <typename T>
struct PsiRegs {
    T x0, x1, y0, y1, z0, z1;
};

// E-side psi of plane k for a column (slab membership as in pml_e_cell)
template <typename T>
__device__ __forceinline__ void psi_load_e(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, int i, int j, int k,
                                           PsiRegs<T> &r)
{
    if (c.fx >= 0) {
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(p.np[c.fx]) + c.sxl;
        r.x0 = __ldg(p.qe[c.fx][0] + q); r.x1 = __ldg(p.qe[c.fx][1] + q);
    }
    if (c.fy >= 0) {
        const int64_t q = ((int64_t)k * (p.np[c.fy] + 1) + c.syl) * d.px + i;
        r.y0 = __ldg(p.qe[c.fy][0] + q); r.y1 = __ldg(p.qe[c.fy][1] + q);
    }
    int fz = -1, szl = 0;
    if (k <= p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        r.z0 = __ldg(p.qe[fz][0] + q); r.z1 = __ldg(p.qe[fz][1] + q);
    }
}

// H-side psi of plane k for a column (slab membership as in pml_h_cell)
template <typename T>
__device__ __forceinline__ void psi_load_h(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, int i, int j, int k,
                                           PsiRegs<T> &r)
{
    if (c.fx >= 0) {
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(p.np[c.fx]) + c.sxl;
        r.x0 = __ldg(p.qh[c.fx][0] + q); r.x1 = __ldg(p.qh[c.fx][1] + q);
    }
    if (c.fy >= 0) {
        const int64_t q = ((int64_t)k * (p.np[c.fy] + 1) + c.syl) * d.px + i;
        r.y0 = __ldg(p.qh[c.fy][0] + q); r.y1 = __ldg(p.qh[c.fy][1] + q);
    }
    int fz = -1, szl = 0;
    if (k < p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        r.z0 = __ldg(p.qh[fz][0] + q); r.z1 = __ldg(p.qh[fz][1] + q);
    }
}

// CPML E corrections with psi already in registers (same arithmetic as pml_e_cell)
template <typename T>
__device__ __forceinline__ void pml_e_cell_pre(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, T ce, int i,
                                               int j, int k, const PsiRegs<T> &r, T dHz_i, T dHy_i, T dHx_j, T dHz_j,
                                               T dHy_k, T dHx_k, T &ex, T &ey, T &ez)
{
    if (c.fx >= 0) {
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(p.np[c.fx]) + c.sxl;
        const T a0 = c.bx * r.x0 + c.cx * dHz_i, a1 = c.bx * r.x1 + c.cx * dHy_i;
        p.qe[c.fx][0][q] = a0; p.qe[c.fx][1][q] = a1;
        ey = ey - a0 * ce;
        ez = ez + a1 * ce;
    }
    if (c.fy >= 0) {
        const int64_t q = ((int64_t)k * (p.np[c.fy] + 1) + c.syl) * d.px + i;
        const T a0 = c.by * r.y0 + c.cy * dHx_j, a1 = c.by * r.y1 + c.cy * dHz_j;
        p.qe[c.fy][0][q] = a0; p.qe[c.fy][1][q] = a1;
        ez = ez - a0 * ce;
        ex = ex + a1 * ce;
    }
    int fz = -1, szl = 0;
    if (k <= p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        const T b = p.bE[fz][szl], cc = p.cE[fz][szl];
        const T a0 = b * r.z0 + cc * dHy_k, a1 = b * r.z1 + cc * dHx_k;
        p.qe[fz][0][q] = a0; p.qe[fz][1][q] = a1;
        ex = ex - a0 * ce;
        ey = ey + a1 * ce;
    }
}

// CPML H corrections with psi already in registers (same arithmetic as
// pml_h_cell); STORE = false computes the corrected H without writing psi
template <typename T, bool STORE = true>
__device__ __forceinline__ void pml_h_cell_pre(const PmlView<T> &p, const Dims &d, const ColPml<T> &c, T ch, int i,
                                               int j, int k, const PsiRegs<T> &r, T dEz_i, T dEy_i, T dEx_j, T dEz_j,
                                               T dEy_k, T dEx_k, T &hx, T &hy, T &hz, bool store = true)
{
    if (c.fx >= 0) {
        const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(p.np[c.fx]) + c.sxl;
        const T a0 = c.bx * r.x0 + c.cx * dEz_i, a1 = c.bx * r.x1 + c.cx * dEy_i;
        if (STORE && store) { p.qh[c.fx][0][q] = a0; p.qh[c.fx][1][q] = a1; }
        hy = hy + a0 * ch;
        hz = hz - a1 * ch;
    }
    if (c.fy >= 0) {
        const int64_t q = ((int64_t)k * (p.np[c.fy] + 1) + c.syl) * d.px + i;
        const T a0 = c.by * r.y0 + c.cy * dEx_j, a1 = c.by * r.y1 + c.cy * dEz_j;
        if (STORE && store) { p.qh[c.fy][0][q] = a0; p.qh[c.fy][1][q] = a1; }
        hz = hz - a0 * ch;
        hx = hx + a1 * ch;
    }
    int fz = -1, szl = 0;
    if (k < p.np[kFZ1]) { fz = kFZ1; szl = k; }
    else if (k >= d.nz - p.np[kFZ2]) { fz = kFZ2; szl = k - (d.nz - p.np[kFZ2]); }
    if (fz >= 0) {
        const int64_t q = ((int64_t)szl * (d.ny + 1) + j) * d.px + i;
        const T b = p.bH[fz][szl], cc = p.cH[fz][szl];
        const T a0 = b * r.z0 + cc * dEy_k, a1 = b * r.z1 + cc * dEx_k;
        if (STORE && store) { p.qh[fz][0][q] = a0; p.qh[fz][1][q] = a1; }
        hx = hx - a0 * ch;
        hy = hy + a1 * ch;
    }
}

// Drude-Lorentz update of the ID-2 cells of a warp row (ballot-ranked lookup
// into the compacted list); the whole warp must call it
template <typename T>
__device__ __forceinline__ void dl_warp(const DlView<T> &D, const Dims &d, int j, int k, int seg, bool act, int id,
                                        T dHz_j, T dHy_k, T dHx_k, T dHz_i, T dHy_i, T dHx_j, T cExy, T cEyx,
                                        T cExz, T cEyz, T cEzy, T cEzx, T &ex, T &ey, T &ez)
{
    const bool mine = act && id == CPS_ID_DISPERSIVE;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (!m) return;
    const int nseg = d.px >> 5;
    const int64_t base = D.seg[((int64_t)k * (d.ny + 1) + j) * nseg + seg];
    if (!mine) return;
    const int64_t c = base + __popc(m & lanemask_lt()), sc = D.ncell;
    const T C3 = D.c.C3;
    const T cxx = C3 * dHz_j * cExz - C3 * dHy_k * cExy;
    const T cyy = C3 * dHx_k * cEyx - C3 * dHz_i * cEyz;
    const T czz = C3 * dHy_i * cEzy - C3 * dHx_j * cEzx;
    T *st = D.state + c;
    ex = dl_component(D.c, ex, cxx, st, sc);
    ey = dl_component(D.c, ey, cyy, st + (int64_t)D.c.stride * sc, sc);
    ez = dl_component(D.c, ez, czz, st + (int64_t)2 * D.c.stride * sc, sc);
}

// four-level gain P -> E -> N at the gain cells of a warp row; the whole warp
// must call it
template <typename T>
__device__ __forceinline__ void gain_warp(const GainView<T> &G, const Dims &d, int j, int k, int seg, bool act,
                                          int id, T &ex, T &ey, T &ez)
{
    const bool mine = act && id == G.gain_id;
    const unsigned m = __ballot_sync(0xffffffffu, mine);
    if (!m) return;
    const int nseg = d.px >> 5;
    const int64_t base = G.seg[((int64_t)k * (d.ny + 1) + j) * nseg + seg];
    if (!mine) return;
    const int64_t c = base + __popc(m & lanemask_lt()), sc = kGainGroup;
    T *st = G.state + (sizeof(T) == 4 ? gain_dense_index(d.idx(seg * 32 + (int)(threadIdx.x & 31u), j, k))
                                      : gain_base_index(c, kG64Words));
    T E[3] = {ex, ey, ez}, E1[3] = {ex, ey, ez};
    T Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3];
    Pops<T> N;
    if (sizeof(T) == 8) {
        using L = GainSite64;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            Pa[q] = st[(L::PA + q) * sc]; Pa1[q] = st[(L::PA1 + q) * sc];
            Pb[q] = st[(L::PB + q) * sc]; Pb1[q] = st[(L::PB1 + q) * sc];
        }
    } else {
        using L = GainSite32;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            Pa[q] = st[(L::PA + q) * sc]; Pa1[q] = st[(L::PA1 + q) * sc];
            Pb[q] = st[(L::PB + q) * sc]; Pb1[q] = st[(L::PB1 + q) * sc];
        }
    }
    gain_load_n<T>(st, sc, N);
    gain_p_update<T>(G.c, N, E, Pa, Pa1, Pa2, Pb, Pb1, Pb2);
#pragma unroll
    for (int q = 0; q < 3; ++q) E[q] = gain_e_corr<T>(G.c, E[q], Pa[q], Pa1[q], Pb[q], Pb1[q]);
    gain_n_update<T>(G.c, N, E, E1, Pa, Pa1, Pa2, Pb, Pb2);
    // the transient words (Pa2 Pb2 E1) are not stored: only the plain path's
    // separate routines read them, after its own polarisation routine wrote them
    if (sizeof(T) == 8) {
        using L = GainSite64;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            st[(L::PA + q) * sc] = Pa[q]; st[(L::PA1 + q) * sc] = Pa1[q];
            st[(L::PB + q) * sc] = Pb[q]; st[(L::PB1 + q) * sc] = Pb1[q];
        }
    } else {
        using L = GainSite32;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            st[(L::PA + q) * sc] = Pa[q]; st[(L::PA1 + q) * sc] = Pa1[q];
            st[(L::PB + q) * sc] = Pb[q]; st[(L::PB1 + q) * sc] = Pb1[q];
        }
    }
    gain_store_n<T>(st, sc, N);
    ex = E[0]; ey = E[1]; ez = E[2];
}


// ---- FP32 gain on the segment-dense layout: the 15 persistent words of the
// cell at device index g are at gain_dense_index(g) + 32 w, for every cell of
// the grid, so a plane's words can be requested (or staged by TMA) before its
// fields and IDs arrive.  The arithmetic is gain_warp's.
struct GainRegs32 {
    float pa[3], pa1[3], pb[3], pb1[3];
    float n[3];  // the population offsets N1 - 1, N2, N3
};

// the words of the cell at device index g from global memory
__device__ __forceinline__ void gain_fetch32(const GainView<float> &G, int64_t g, GainRegs32 &r)
{
    using L = GainSite32;
    const float *st = G.state + gain_dense_index(g);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        r.pa[q] = __ldg(st + (L::PA + q) * kGainGroup);
        r.pa1[q] = __ldg(st + (L::PA1 + q) * kGainGroup);
        r.pb[q] = __ldg(st + (L::PB + q) * kGainGroup);
        r.pb1[q] = __ldg(st + (L::PB1 + q) * kGainGroup);
    }
    r.n[0] = __ldg(st + L::DN1 * kGainGroup);
    r.n[1] = __ldg(st + L::N2 * kGainGroup);
    r.n[2] = __ldg(st + L::N3 * kGainGroup);
}

// the words of a cell from a staged tile: word w at ws[32 w]
__device__ __forceinline__ void gain_staged32(const float *ws, GainRegs32 &r)
{
    using L = GainSite32;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        r.pa[q] = ws[(L::PA + q) * 32];
        r.pa1[q] = ws[(L::PA1 + q) * 32];
        r.pb[q] = ws[(L::PB + q) * 32];
        r.pb1[q] = ws[(L::PB1 + q) * 32];
    }
    r.n[0] = ws[L::DN1 * 32];
    r.n[1] = ws[L::N2 * 32];
    r.n[2] = ws[L::N3 * 32];
}

// P -> E -> N at a gain cell (device index g) from its words r; the new words
// go to the dense state
__device__ __forceinline__ void gain_apply32(const GainView<float> &G, int64_t g, const GainRegs32 &r, float &ex,
                                             float &ey, float &ez)
{
    using L = GainSite32;
    float *st = G.state + gain_dense_index(g);
    const int64_t sc = kGainGroup;
    float E[3] = {ex, ey, ez}, E1[3] = {ex, ey, ez};
    float Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) { Pa[q] = r.pa[q]; Pa1[q] = r.pa1[q]; Pb[q] = r.pb[q]; Pb1[q] = r.pb1[q]; }
    Pops<float> N;
    N.n1 = r.n[0];
    N.n2 = r.n[1];
    N.n3 = r.n[2];
    N.m0 = conserve_m0(N.n1, N.n2, N.n3);  // FP64 conservation, FourLevelLaser.cpp:324
    gain_p_update<float>(G.c, N, E, Pa, Pa1, Pa2, Pb, Pb1, Pb2);
#pragma unroll
    for (int q = 0; q < 3; ++q) E[q] = gain_e_corr<float>(G.c, E[q], Pa[q], Pa1[q], Pb[q], Pb1[q]);
    gain_n_update<float>(G.c, N, E, E1, Pa, Pa1, Pa2, Pb, Pb2);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        st[(L::PA + q) * sc] = Pa[q]; st[(L::PA1 + q) * sc] = Pa1[q];
        st[(L::PB + q) * sc] = Pb[q]; st[(L::PB1 + q) * sc] = Pb1[q];
    }
    gain_store_n<float>(st, sc, N);
    ex = E[0]; ey = E[1]; ez = E[2];
}

}  // namespace cps
