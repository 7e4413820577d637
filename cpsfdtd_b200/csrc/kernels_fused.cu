// kernels_fused.cu -- the fused sweeps of one time step.
//
// Each block covers a 32 x BY patch of (i, j) columns and marches KC planes
// in k.  A thread keeps the k-neighbour of its own column in registers (E at
// k+1 for H, H at k-1 for E), so every field word crosses HBM once per sweep;
// the x/y neighbours come from the L1 lines the neighbouring threads of the
// same block load.  Per cell the sweep applies, in the reference order:
//   H: bulk (BasicFDTD.cpp:67-84) then CPML psi corrections (CPML.cpp:609-689)
//   E: bulk (BasicFDTD.cpp:25-47), Drude-Lorentz (ID 2), four-level gain
//      (P, E, N), then CPML (CPML.cpp:529-607).
// TF/SF corrections, point sources and port sampling run as small separate
// launches between/after the sweeps (they touch surfaces only).
// Coefficients come from the per-medium tables (uint8 ID per cell) and the
// 1-D stretched-coordinate arrays; psi lives only on the boundary slabs and
// Drude-Lorentz/gain state only on the compacted cell lists.
#include "cells.cuh"

namespace cps {

namespace {

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename T, int BY, bool PML>
__global__ void __launch_bounds__(32 * BY) k_h_fused(FieldView<T> f, PmlView<T> p, int kc)
{
    const Dims d = f.d;
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int k0 = blockIdx.z * kc, k1 = min(k0 + kc, d.nz);
    if (i >= d.nx || j >= d.ny) return;
    const StretchView<T> &s = f.s;
    const T cHyz = s.cHyz[i], cHzy = s.cHzy[i], cHxz = s.cHxz[j], cHzx = s.cHzx[j];
    // CPML slabs this column belongs to (x and y are fixed along the march)
    int fx = -1, sxl = 0, fy = -1, syl = 0;
    T bx = 0, cx = 0, by = 0, cy = 0;
    if (PML) {
        if (i < p.np[kFX1]) { fx = kFX1; sxl = i; }
        else if (i >= d.nx - p.np[kFX2]) { fx = kFX2; sxl = i - (d.nx - p.np[kFX2]); }
        if (j < p.np[kFY1]) { fy = kFY1; syl = j; }
        else if (j >= d.ny - p.np[kFY2]) { fy = kFY2; syl = j - (d.ny - p.np[kFY2]); }
        if (fx >= 0) { bx = p.bH[fx][sxl]; cx = p.cH[fx][sxl]; }
        if (fy >= 0) { by = p.bH[fy][syl]; cy = p.cH[fy][syl]; }
    }
    int64_t g = d.idx(i, j, k0);
    T ex = f.Ex[g], ey = f.Ey[g];
    for (int k = k0; k < k1; ++k, g += d.pxy) {
        const T exk = f.Ex[g + d.pxy], eyk = f.Ey[g + d.pxy];
        const T ez = f.Ez[g];
        const T dEz_i = ld(&f.Ez[g + 1]) - ez, dEz_j = ld(&f.Ez[g + d.px]) - ez;
        const T dEx_j = ld(&f.Ex[g + d.px]) - ex, dEy_i = ld(&f.Ey[g + 1]) - ey;
        const T dEx_k = exk - ex, dEy_k = eyk - ey;
        const int id = f.id[g];
        const T aH = ld(&f.aH[id]), bH = ld(&f.bH[id]);
        T hx = f.Hx[g], hy = f.Hy[g], hz = f.Hz[g];
        hx = aH * hx - bH * dEz_j * cHxz + bH * dEy_k * s.cHxy[k];
        hy = aH * hy - bH * dEx_k * s.cHyx[k] + bH * dEz_i * cHyz;
        hz = aH * hz + bH * dEx_j * cHzx - bH * dEy_i * cHzy;
        if (PML) {
            const T ch = p.cpmlH;
            if (fx >= 0) {
                const int np = p.np[fx];
                const int64_t q = ((int64_t)k * (d.ny + 1) + j) * (np + 1) + sxl;
                T *q0 = p.qh[fx][0], *q1 = p.qh[fx][1];
                const T a0 = bx * q0[q] + cx * dEz_i, a1 = bx * q1[q] + cx * dEy_i;
                q0[q] = a0; q1[q] = a1;
                hy = hy + a0 * ch;
                hz = hz - a1 * ch;
            }
            if (fy >= 0) {
                const int np = p.np[fy];
                const int64_t q = ((int64_t)k * (np + 1) + syl) * d.px + i;
                T *q0 = p.qh[fy][0], *q1 = p.qh[fy][1];
                const T a0 = by * q0[q] + cy * dEx_j, a1 = by * q1[q] + cy * dEz_j;
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
                const T b = p.bH[fz][szl], c = p.cH[fz][szl];
                const T a0 = b * q0[q] + c * dEy_k, a1 = b * q1[q] + c * dEx_k;
                q0[q] = a0; q1[q] = a1;
                hx = hx - a0 * ch;
                hy = hy + a1 * ch;
            }
        }
        f.Hx[g] = hx; f.Hy[g] = hy; f.Hz[g] = hz;
        ex = exk; ey = eyk;
    }
}

template <typename T, int BY, bool PML, bool DL, bool GAIN>
__global__ void __launch_bounds__(32 * BY) k_e_fused(FieldView<T> f, PmlView<T> p, DlView<T> D,
                                                     GainView<T> G, int kc)
{
    const Dims d = f.d;
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * BY + threadIdx.y;
    const int k0 = max(1, blockIdx.z * kc), k1 = min(blockIdx.z * kc + kc, d.nz);
    // a warp is one row j; rows outside [1, ny-1] leave whole, lanes outside
    // [1, nx-1] stay for the ballots but touch no memory
    if (j < 1 || j >= d.ny || k0 >= k1) return;
    const bool act = i >= 1 && i < d.nx;
    const int ic = act ? i : 1;
    const StretchView<T> &s = f.s;
    const T cEyz = s.cEyz[ic], cEzy = s.cEzy[ic], cExz = s.cExz[j], cEzx = s.cEzx[j];
    int fx = -1, sxl = 0, fy = -1, syl = 0;
    T bx = 0, cx = 0, by = 0, cy = 0;
    if (PML) {
        if (ic <= p.np[kFX1]) { fx = kFX1; sxl = ic; }
        else if (ic >= d.nx - p.np[kFX2]) { fx = kFX2; sxl = ic - (d.nx - p.np[kFX2]); }
        if (j <= p.np[kFY1]) { fy = kFY1; syl = j; }
        else if (j >= d.ny - p.np[kFY2]) { fy = kFY2; syl = j - (d.ny - p.np[kFY2]); }
        if (fx >= 0) { bx = p.bE[fx][sxl]; cx = p.cE[fx][sxl]; }
        if (fy >= 0) { by = p.bE[fy][syl]; cy = p.cE[fy][syl]; }
    }
    const int nseg = d.px >> 5;
    int64_t g = d.idx(ic, j, k0);
    T hxm = act ? f.Hx[g - d.pxy] : T(0), hym = act ? f.Hy[g - d.pxy] : T(0);
    for (int k = k0; k < k1; ++k, g += d.pxy) {
        T hx = 0, hy = 0, hz = 0, ex = 0, ey = 0, ez = 0;
        T dHz_j = 0, dHy_k = 0, dHx_k = 0, dHz_i = 0, dHy_i = 0, dHx_j = 0;
        int id = 0;
        if (act) {
            hx = f.Hx[g]; hy = f.Hy[g]; hz = f.Hz[g];
            dHz_j = hz - ld(&f.Hz[g - d.px]);
            dHz_i = hz - ld(&f.Hz[g - 1]);
            dHy_i = hy - ld(&f.Hy[g - 1]);
            dHx_j = hx - ld(&f.Hx[g - d.px]);
            dHy_k = hy - hym;
            dHx_k = hx - hxm;
            ex = f.Ex[g]; ey = f.Ey[g]; ez = f.Ez[g];
            id = f.id[g];
            if (id == CPS_ID_PEC) {
                ex = T(0); ey = T(0); ez = T(0);
            } else if (id != CPS_ID_DISPERSIVE) {
                const T aE = ld(&f.aE[id]), bE = ld(&f.bE[id]);
                ex = aE * ex + bE * dHz_j * cExz - bE * dHy_k * s.cExy[k];
                ey = aE * ey + bE * dHx_k * s.cEyx[k] - bE * dHz_i * cEyz;
                ez = aE * ez + bE * dHy_i * cEzy - bE * dHx_j * cEzx;
            }
        }
        if (DL) {
            const unsigned m = __ballot_sync(0xffffffffu, act && id == CPS_ID_DISPERSIVE);
            if (m) {
                const int64_t base = D.seg[((int64_t)k * (d.ny + 1) + j) * nseg + blockIdx.x];
                if (act && id == CPS_ID_DISPERSIVE) {
                    const int64_t c = base + __popc(m & lanemask_lt()), sc = D.ncell;
                    const T C3 = D.c.C3;
                    const T cxx = C3 * dHz_j * cExz - C3 * dHy_k * s.cExy[k];
                    const T cyy = C3 * dHx_k * s.cEyx[k] - C3 * dHz_i * cEyz;
                    const T czz = C3 * dHy_i * cEzy - C3 * dHx_j * cEzx;
                    T *st = D.state + c;
                    ex = dl_component(D.c, ex, cxx, st, sc);
                    ey = dl_component(D.c, ey, cyy, st + (int64_t)D.c.stride * sc, sc);
                    ez = dl_component(D.c, ez, czz, st + (int64_t)2 * D.c.stride * sc, sc);
                }
            }
        }
        if (GAIN) {
            const bool mine = act && id == G.gain_id;
            const unsigned m = __ballot_sync(0xffffffffu, mine);
            if (m) {
                const int64_t base = G.seg[((int64_t)k * (d.ny + 1) + j) * nseg + blockIdx.x];
                if (mine) {
                    using L = GainSite32;
                    const int64_t c = base + __popc(m & lanemask_lt()), sc = G.ncell;
                    T *st = G.state + c;
                    T E[3] = {ex, ey, ez}, E1[3] = {ex, ey, ez};
                    T Pa[3], Pa1[3], Pa2[3], Pb[3], Pb1[3], Pb2[3];
                    double N[4];
                    if (sizeof(T) == 8) {
                        using L64 = GainSite64;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            Pa[q] = st[(L64::PA + q) * sc]; Pa1[q] = st[(L64::PA1 + q) * sc];
                            Pb[q] = st[(L64::PB + q) * sc]; Pb1[q] = st[(L64::PB1 + q) * sc];
                        }
                    } else {
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
                    if (sizeof(T) == 8) {
                        using L64 = GainSite64;
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            st[(L64::PA + q) * sc] = Pa[q]; st[(L64::PA1 + q) * sc] = Pa1[q]; st[(L64::PA2 + q) * sc] = Pa2[q];
                            st[(L64::PB + q) * sc] = Pb[q]; st[(L64::PB1 + q) * sc] = Pb1[q]; st[(L64::PB2 + q) * sc] = Pb2[q];
                            st[(L64::E1 + q) * sc] = E1[q];
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < 3; ++q) {
                            st[(L::PA + q) * sc] = Pa[q]; st[(L::PA1 + q) * sc] = Pa1[q];
                            st[(L::PB + q) * sc] = Pb[q]; st[(L::PB1 + q) * sc] = Pb1[q];
                        }
                    }
                    gain_store_n<T>(st, sc, N);
                    ex = E[0]; ey = E[1]; ez = E[2];
                }
            }
        }
        if (act) {
            if (PML) {
                const T ce = p.cpmlE;
                if (fx >= 0) {
                    const int np = p.np[fx];
                    const int64_t q = ((int64_t)k * (d.ny + 1) + j) * (np + 1) + sxl;
                    T *q0 = p.qe[fx][0], *q1 = p.qe[fx][1];
                    const T a0 = bx * q0[q] + cx * dHz_i, a1 = bx * q1[q] + cx * dHy_i;
                    q0[q] = a0; q1[q] = a1;
                    ey = ey - a0 * ce;
                    ez = ez + a1 * ce;
                }
                if (fy >= 0) {
                    const int np = p.np[fy];
                    const int64_t q = ((int64_t)k * (np + 1) + syl) * d.px + i;
                    T *q0 = p.qe[fy][0], *q1 = p.qe[fy][1];
                    const T a0 = by * q0[q] + cy * dHx_j, a1 = by * q1[q] + cy * dHz_j;
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
                    const T b = p.bE[fz][szl], c = p.cE[fz][szl];
                    const T a0 = b * q0[q] + c * dHy_k, a1 = b * q1[q] + c * dHx_k;
                    q0[q] = a0; q1[q] = a1;
                    ex = ex - a0 * ce;
                    ey = ey + a1 * ce;
                }
            }
            f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
        }
        hxm = hx; hym = hy;
    }
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

template <typename T, int BY>
void h_fused_by(const FieldView<T> &f, const PmlView<T> &p, int kc, cudaStream_t s)
{
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    if (p.on) k_h_fused<T, BY, true><<<grid, dim3(32, BY), 0, s>>>(f, p, kc);
    else k_h_fused<T, BY, false><<<grid, dim3(32, BY), 0, s>>>(f, p, kc);
}

template <typename T, int BY, bool PML>
void e_fused_pml(const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D, const GainView<T> &G,
                 int kc, cudaStream_t s)
{
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    const bool dl = D.on && D.ncell > 0, gn = G.on && G.ncell > 0;
    if (dl && gn) k_e_fused<T, BY, PML, true, true><<<grid, dim3(32, BY), 0, s>>>(f, p, D, G, kc);
    else if (dl) k_e_fused<T, BY, PML, true, false><<<grid, dim3(32, BY), 0, s>>>(f, p, D, G, kc);
    else if (gn) k_e_fused<T, BY, PML, false, true><<<grid, dim3(32, BY), 0, s>>>(f, p, D, G, kc);
    else k_e_fused<T, BY, PML, false, false><<<grid, dim3(32, BY), 0, s>>>(f, p, D, G, kc);
}

template <typename T, int BY>
void e_fused_by(const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D, const GainView<T> &G,
                int kc, cudaStream_t s)
{
    if (p.on) e_fused_pml<T, BY, true>(f, p, D, G, kc, s);
    else e_fused_pml<T, BY, false>(f, p, D, G, kc, s);
}

}  // namespace

template <typename T>
void launch_h_fused(const FieldView<T> &f, const PmlView<T> &p, FusedShape sh, cudaStream_t s)
{
    switch (sh.by) {
    case 2: h_fused_by<T, 2>(f, p, sh.kc, s); break;
    case 4: h_fused_by<T, 4>(f, p, sh.kc, s); break;
    case 16: h_fused_by<T, 16>(f, p, sh.kc, s); break;
    default: h_fused_by<T, 8>(f, p, sh.kc, s); break;
    }
}

template <typename T>
void launch_e_fused(const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &d, const GainView<T> &g,
                    FusedShape sh, cudaStream_t s)
{
    switch (sh.by) {
    case 2: e_fused_by<T, 2>(f, p, d, g, sh.kc, s); break;
    case 4: e_fused_by<T, 4>(f, p, d, g, sh.kc, s); break;
    case 16: e_fused_by<T, 16>(f, p, d, g, sh.kc, s); break;
    default: e_fused_by<T, 8>(f, p, d, g, sh.kc, s); break;
    }
}

template void launch_h_fused<double>(const FieldView<double> &, const PmlView<double> &, FusedShape, cudaStream_t);
template void launch_h_fused<float>(const FieldView<float> &, const PmlView<float> &, FusedShape, cudaStream_t);
template void launch_e_fused<double>(const FieldView<double> &, const PmlView<double> &, const DlView<double> &,
                                     const GainView<double> &, FusedShape, cudaStream_t);
template void launch_e_fused<float>(const FieldView<float> &, const PmlView<float> &, const DlView<float> &,
                                    const GainView<float> &, FusedShape, cudaStream_t);

}  // namespace cps
