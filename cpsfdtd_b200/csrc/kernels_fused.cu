// kernels_fused.cu -- the fused sweeps of one time step.
//
// Each block covers a 32 x BY patch of (i, j) columns and marches KC planes
// in k.  A thread keeps the k-neighbour of its own column in registers (E at
// k+1 for H, H at k-1 for E), takes its x-neighbour from the adjacent lane by
// a warp shuffle, and reads the y-neighbour through L1, so every field word
// crosses HBM once per sweep.  All loads of plane k+1 are issued (read-only,
// non-coherent path) before plane k is computed and stored, which keeps two
// planes of loads in flight per thread.
// Per cell the sweep applies, in the reference order:
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

template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// values of one plane that the H sweep of a column needs
template <typename T>
struct HPlane {
    T exk, eyk;        // E at k+1 of the own column
    T ez, ezj, exj;    // Ez own, Ez(j+1), Ex(j+1)
    T ezi, eyi;        // Ez(i+1), Ey(i+1): only lane 31 loads them
    T hx, hy, hz;
    int id;
};

template <typename T>
__device__ __forceinline__ void h_load(HPlane<T> &q, const FieldView<T> &f, int64_t g, bool last_lane, bool ok)
{
    const Dims &d = f.d;
    q.exk = ldg(&f.Ex[g + d.pxy]);
    q.eyk = ldg(&f.Ey[g + d.pxy]);
    q.ez = ldg(&f.Ez[g]);
    q.ezj = ldg(&f.Ez[g + d.px]);
    q.exj = ldg(&f.Ex[g + d.px]);
    q.ezi = (last_lane && ok) ? ldg(&f.Ez[g + 1]) : T(0);
    q.eyi = (last_lane && ok) ? ldg(&f.Ey[g + 1]) : T(0);
    q.hx = ldg(&f.Hx[g]);
    q.hy = ldg(&f.Hy[g]);
    q.hz = ldg(&f.Hz[g]);
    q.id = ldg(&f.id[g]);
}

template <typename T, int BY, bool PML>
__global__ void __launch_bounds__(32 * BY, (768 / (32 * BY)) > 0 ? 768 / (32 * BY) : 1)
k_h_fused(FieldView<T> f, PmlView<T> p, int kc)
{
    const Dims d = f.d;
    const int lane = threadIdx.x;
    const int i = blockIdx.x * 32 + lane, j = blockIdx.y * BY + threadIdx.y;
    const int k0 = blockIdx.z * kc, k1 = min(k0 + kc, d.nz);
    // a warp is one row; rows outside [0, ny-1] leave whole, lanes past nx-1
    // load their (padded, in-bounds) cell for the shuffles but store nothing
    if (j >= d.ny || k0 >= k1) return;
    const bool act = i < d.nx;
    const StretchView<T> &s = f.s;
    const int ic = act ? i : d.nx - 1;
    const T cHyz = s.cHyz[ic], cHzy = s.cHzy[ic], cHxz = s.cHxz[j], cHzx = s.cHzx[j];
    int fx = -1, sxl = 0, fy = -1, syl = 0;
    T bx = 0, cx = 0, by = 0, cy = 0;
    if (PML) {
        if (i < p.np[kFX1]) { fx = kFX1; sxl = i; }
        else if (act && i >= d.nx - p.np[kFX2]) { fx = kFX2; sxl = i - (d.nx - p.np[kFX2]); }
        if (j < p.np[kFY1]) { fy = kFY1; syl = j; }
        else if (j >= d.ny - p.np[kFY2]) { fy = kFY2; syl = j - (d.ny - p.np[kFY2]); }
        if (fx >= 0) { bx = p.bH[fx][sxl]; cx = p.cH[fx][sxl]; }
        if (fy >= 0) { by = p.bH[fy][syl]; cy = p.cH[fy][syl]; }
    }
    const bool last = lane == 31;
    int64_t g = d.idx(i, j, k0);
    T ex = ldg(&f.Ex[g]), ey = ldg(&f.Ey[g]);
    HPlane<T> cur, nxt;
    h_load(cur, f, g, last, act);
    for (int k = k0; k < k1; ++k, g += d.pxy) {
        if (k + 1 < k1) h_load(nxt, f, g + d.pxy, last, act);
        // x-neighbours from lane + 1
        T ezi = __shfl_down_sync(0xffffffffu, cur.ez, 1);
        T eyi = __shfl_down_sync(0xffffffffu, ey, 1);
        if (last) { ezi = cur.ezi; eyi = cur.eyi; }
        const T dEz_i = ezi - cur.ez, dEz_j = cur.ezj - cur.ez;
        const T dEx_j = cur.exj - ex, dEy_i = eyi - ey;
        const T dEx_k = cur.exk - ex, dEy_k = cur.eyk - ey;
        const T aH = ldg(&f.aH[cur.id]), bH = ldg(&f.bH[cur.id]);
        T hx = aH * cur.hx - bH * dEz_j * cHxz + bH * dEy_k * ldg(&s.cHxy[k]);
        T hy = aH * cur.hy - bH * dEx_k * ldg(&s.cHyx[k]) + bH * dEz_i * cHyz;
        T hz = aH * cur.hz + bH * dEx_j * cHzx - bH * dEy_i * cHzy;
        if (PML && act) {
            const T ch = pml_ch_cell(p, f.bH, (int)cur.id);
            if (fx >= 0) {
                const int np = p.np[fx];
                const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(np) + sxl;
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
        if (act) { f.Hx[g] = hx; f.Hy[g] = hy; f.Hz[g] = hz; }
        ex = cur.exk; ey = cur.eyk;
        cur = nxt;
    }
}

// values of one plane that the E sweep of a column needs
template <typename T>
struct EPlane {
    T hx, hy, hz;      // own H
    T hzj, hxj;        // Hz(j-1), Hx(j-1)
    T hzi, hyi;        // Hz(i-1), Hy(i-1): only lane 0 loads them
    T ex, ey, ez;
    int id;
};

template <typename T>
__device__ __forceinline__ void e_load(EPlane<T> &q, const FieldView<T> &f, int64_t g, bool first_lane, bool has_left)
{
    const Dims &d = f.d;
    q.hx = ldg(&f.Hx[g]);
    q.hy = ldg(&f.Hy[g]);
    q.hz = ldg(&f.Hz[g]);
    q.hzj = ldg(&f.Hz[g - d.px]);
    q.hxj = ldg(&f.Hx[g - d.px]);
    q.hzi = (first_lane && has_left) ? ldg(&f.Hz[g - 1]) : T(0);
    q.hyi = (first_lane && has_left) ? ldg(&f.Hy[g - 1]) : T(0);
    q.ex = ldg(&f.Ex[g]);
    q.ey = ldg(&f.Ey[g]);
    q.ez = ldg(&f.Ez[g]);
    q.id = ldg(&f.id[g]);
}

template <typename T, int BY, bool PML, bool DL, bool GAIN>
__global__ void __launch_bounds__(32 * BY, (768 / (32 * BY)) > 0 ? 768 / (32 * BY) : 1)
k_e_fused(FieldView<T> f, PmlView<T> p, DlView<T> D, GainView<T> G, int kc)
{
    const Dims d = f.d;
    const int lane = threadIdx.x;
    const int i = blockIdx.x * 32 + lane, j = blockIdx.y * BY + threadIdx.y;
    const int k0 = max(1, blockIdx.z * kc), k1 = min(blockIdx.z * kc + kc, d.nz);
    // a warp is one row j; rows outside [1, ny-1] leave whole, lanes outside
    // [1, nx-1] load their (in-bounds) cell for the shuffles but store nothing
    if (j < 1 || j >= d.ny || k0 >= k1) return;
    const bool act = i >= 1 && i < d.nx;
    const int ic = act ? i : 1;
    const StretchView<T> &s = f.s;
    const T cEyz = s.cEyz[ic], cEzy = s.cEzy[ic], cExz = s.cExz[j], cEzx = s.cEzx[j];
    int fx = -1, sxl = 0, fy = -1, syl = 0;
    T bx = 0, cx = 0, by = 0, cy = 0;
    if (PML) {
        if (act && i <= p.np[kFX1]) { fx = kFX1; sxl = i; }
        else if (act && i >= d.nx - p.np[kFX2]) { fx = kFX2; sxl = i - (d.nx - p.np[kFX2]); }
        if (j <= p.np[kFY1]) { fy = kFY1; syl = j; }
        else if (j >= d.ny - p.np[kFY2]) { fy = kFY2; syl = j - (d.ny - p.np[kFY2]); }
        if (fx >= 0) { bx = p.bE[fx][sxl]; cx = p.cE[fx][sxl]; }
        if (fy >= 0) { by = p.bE[fy][syl]; cy = p.cE[fy][syl]; }
    }
    const int nseg = d.px >> 5;
    const bool first = lane == 0, has_left = i > 0;
    int64_t g = d.idx(i, j, k0);
    T hxm = ldg(&f.Hx[g - d.pxy]), hym = ldg(&f.Hy[g - d.pxy]);
    EPlane<T> cur, nxt;
    e_load(cur, f, g, first, has_left);
    for (int k = k0; k < k1; ++k, g += d.pxy) {
        if (k + 1 < k1) e_load(nxt, f, g + d.pxy, first, has_left);
        T hzi = __shfl_up_sync(0xffffffffu, cur.hz, 1);
        T hyi = __shfl_up_sync(0xffffffffu, cur.hy, 1);
        if (first) { hzi = cur.hzi; hyi = cur.hyi; }
        const T dHz_j = cur.hz - cur.hzj, dHz_i = cur.hz - hzi, dHy_i = cur.hy - hyi;
        const T dHx_j = cur.hx - cur.hxj, dHy_k = cur.hy - hym, dHx_k = cur.hx - hxm;
        const T cExy = ldg(&s.cExy[k]), cEyx = ldg(&s.cEyx[k]);
        T ex = cur.ex, ey = cur.ey, ez = cur.ez;
        const int id = cur.id;
        if (id == CPS_ID_PEC) {
            ex = T(0); ey = T(0); ez = T(0);
        } else if (id != CPS_ID_DISPERSIVE) {
            const T aE = ldg(&f.aE[id]), bE = ldg(&f.bE[id]);
            ex = aE * ex + bE * dHz_j * cExz - bE * dHy_k * cExy;
            ey = aE * ey + bE * dHx_k * cEyx - bE * dHz_i * cEyz;
            ez = aE * ez + bE * dHy_i * cEzy - bE * dHx_j * cEzx;
        }
        if (DL) {
            const unsigned m = __ballot_sync(0xffffffffu, act && id == CPS_ID_DISPERSIVE);
            if (m) {
                const int64_t base = D.seg[((int64_t)k * (d.ny + 1) + j) * nseg + blockIdx.x];
                if (act && id == CPS_ID_DISPERSIVE) {
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
            }
        }
        if (GAIN) {
            const bool mine = act && id == G.gain_id;
            const unsigned m = __ballot_sync(0xffffffffu, mine);
            if (m) {
                const int64_t base = G.seg[((int64_t)k * (d.ny + 1) + j) * nseg + blockIdx.x];
                if (mine) {
                    const int64_t c = base + __popc(m & lanemask_lt()), sc = kGainGroup;
                    T *st = G.state + (sizeof(T) == 4 ? gain_dense_index(d.idx(i, j, k))
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
                    if (sizeof(T) == 8) {  // the plain path's transient words are not stored
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
            }
        }
        if (act) {
            if (PML) {
                const T ce = pml_ce_cell(p, f.bE, id);
                if (fx >= 0) {
                    const int np = p.np[fx];
                    const int64_t q = ((int64_t)k * (d.ny + 1) + j) * psi_xw(np) + sxl;
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
        hxm = cur.hx; hym = cur.hy;
        cur = nxt;
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
