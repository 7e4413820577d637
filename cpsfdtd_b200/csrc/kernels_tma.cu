// kernels_tma.cu -- fused H and E sweeps fed by TMA (sm_100a).
//
// A block owns a 32 x BY tile of (i, j) columns and marches kc planes in k.
// Thread 0 keeps S = 4 planes of x-y tiles in flight: for each plane one
// mbarrier, and cp.async.bulk.tensor loads of
//   E sweep: H with a one-cell low halo (box 36 x (BY+1) from (x0-4, y0-1)),
//            E and the uint8 ID of the tile (box 32 x BY from (x0, y0));
//   H sweep: E with a one-cell high halo (box 36 x (BY+1) from (x0, y0)),
//            H and the ID of the tile.
// The x origin of every box is a multiple of 4 elements (16 bytes); boxes
// that reach outside the arrays read zeros.  No multicast is used.
// Threads take their cell and its x/y neighbours from the staged tile and the
// k-neighbour from registers, update, and store with plain coalesced stores;
// when all threads are done with a stage (__syncthreads) thread 0 refills it
// with the plane S ahead.  CPML psi, Drude-Lorentz and gain state go through
// the same per-cell code as the register sweeps (sweep_cells.cuh).
// Every mbarrier wait is bounded; on expiry the block records an error code
// for the host and leaves.
#include <cuda.h>

#include "sweep_cells.cuh"
#include "tma.cuh"

namespace cps {

namespace {

constexpr int kStages = 4;
constexpr int kWaitLimit = 1 << 18;

__host__ __device__ constexpr int a128(int b) { return (b + 127) / 128 * 128; }

template <typename T, int BY>
struct StageLayout {
    static constexpr int HW = 36, HH = BY + 1, OW = 32, OH = BY;
    static constexpr int HALO_B = a128(HW * HH * (int)sizeof(T));
    static constexpr int OWN_B = a128(OW * OH * (int)sizeof(T));
    static constexpr int ID_B = a128(OW * OH);
    static constexpr int STAGE_B = 3 * HALO_B + 3 * OWN_B + ID_B;
    static constexpr uint32_t TX = 3 * HW * HH * sizeof(T) + 3 * OW * OH * sizeof(T) + OW * OH;
    static constexpr int SMEM = kStages * STAGE_B + 128;
};

__device__ __forceinline__ bool wait_stage(uint64_t *bar, uint32_t phase)
{
    for (int it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

template <typename T, int BY, bool PML, bool DL, bool GAIN>
__device__ __forceinline__ void e_tma_body(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p,
                                           const DlView<T> &D, const GainView<T> &G, int kc, int *err,
                                           unsigned char *sm, uint64_t *full)
{
    using L = StageLayout<T, BY>;
    const Dims d = f.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * BY;
    const int i = x0 + tx, j = y0 + ty;
    const int k0 = max(1, (int)blockIdx.z * kc), k1 = min((int)blockIdx.z * kc + kc, d.nz);
    if (k0 >= k1) return;  // whole block
    const bool rowok = j >= 1 && j < d.ny;
    const bool act = rowok && i >= 1 && i < d.nx;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int s, int k) {
        unsigned char *b = sm + s * L::STAGE_B;
        fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
        mbar_expect_tx(&full[s], L::TX);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + c * L::HALO_B, &M.halo[3 + c], &full[s], x0 - 4, y0 - 1, k);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + 3 * L::HALO_B + c * L::OWN_B, &M.own[c], &full[s], x0, y0, k);
        tma_load_3d(b + 3 * L::HALO_B + 3 * L::OWN_B, &M.id, &full[s], x0, y0, k);
    };
    if (tid == 0)
        for (int s = 0; s < kStages && k0 + s < k1; ++s) issue(s, k0 + s);
    const int ic = act ? i : 1, jc = rowok ? j : 1;
    const StretchView<T> &sv = f.s;
    const T cEyz = sv.cEyz[ic], cEzy = sv.cEzy[ic], cExz = sv.cExz[jc], cEzx = sv.cEzx[jc];
    ColPml<T> pc{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
    if (PML && rowok) pc = col_pml_e(p, d, i, j, act);
    T hxm = 0, hym = 0;
    if (rowok) {
        const int64_t gm = d.idx(i, j, k0 - 1);
        hxm = __ldg(&f.Hx[gm]);
        hym = __ldg(&f.Hy[gm]);
    }
    // psi two planes ahead: qc (plane k), qn (k+1), loads for k+2 issued at plane k
    PsiRegs<T> qc{}, qn{}, qnn{};
    if (PML && act) {
        psi_load_e(p, d, pc, i, j, k0, qc);
        if (k0 + 1 < k1) psi_load_e(p, d, pc, i, j, k0 + 1, qn);
    }
    const int hr = (ty + 1) * L::HW + tx + 4, orow = ty * L::OW + tx;
    for (int k = k0, it = 0; k < k1; ++k, ++it) {
        if (PML && act && k + 2 < k1) psi_load_e(p, d, pc, i, j, k + 2, qnn);
        const int s = it % kStages;
        const bool ok = wait_stage(&full[s], (uint32_t)(it / kStages) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 1);
            return;
        }
        const unsigned char *b = sm + s * L::STAGE_B;
        const T *hxt = (const T *)b, *hyt = (const T *)(b + L::HALO_B), *hzt = (const T *)(b + 2 * L::HALO_B);
        const T *ext = (const T *)(b + 3 * L::HALO_B), *eyt = (const T *)(b + 3 * L::HALO_B + L::OWN_B);
        const T *ezt = (const T *)(b + 3 * L::HALO_B + 2 * L::OWN_B);
        const uint8_t *idt = b + 3 * L::HALO_B + 3 * L::OWN_B;
        const T hx = hxt[hr], hy = hyt[hr], hz = hzt[hr];
        const T dHz_j = hz - hzt[hr - L::HW], dHx_j = hx - hxt[hr - L::HW];
        const T dHz_i = hz - hzt[hr - 1], dHy_i = hy - hyt[hr - 1];
        const T dHy_k = hy - hym, dHx_k = hx - hxm;
        T ex = ext[orow], ey = eyt[orow], ez = ezt[orow];
        const int id = idt[orow];
        const T cExy = sv.cExy[k], cEyx = sv.cEyx[k];
        if (id == CPS_ID_PEC) {
            ex = T(0); ey = T(0); ez = T(0);
        } else if (id != CPS_ID_DISPERSIVE) {
            const T aE = __ldg(&f.aE[id]), bE = __ldg(&f.bE[id]);
            ex = aE * ex + bE * dHz_j * cExz - bE * dHy_k * cExy;
            ey = aE * ey + bE * dHx_k * cEyx - bE * dHz_i * cEyz;
            ez = aE * ez + bE * dHy_i * cEzy - bE * dHx_j * cEzx;
        }
        if (GAIN && rowok) gain_warp(G, d, j, k, blockIdx.x, act, id, ex, ey, ez);
        // ID-2 cells are left untouched here: k_dl_cells updates them (ADE,
        // then CPML) after the sweep, in the reference order
        if (act && !(DL && id == CPS_ID_DISPERSIVE)) {
            if (PML) pml_e_cell_pre(p, d, pc, i, j, k, qc, dHz_i, dHy_i, dHx_j, dHz_j, dHy_k, dHx_k, ex, ey, ez);
            const int64_t g = d.idx(i, j, k);
            f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
        }
        hxm = hx; hym = hy;
        qc = qn;
        qn = qnn;
        __syncthreads();
        if (tid == 0 && k + kStages < k1) issue(s, k + kStages);
    }
}

template <typename T, int BY, bool PML>
__device__ __forceinline__ void h_tma_body(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc,
                                           int *err, unsigned char *sm, uint64_t *full)
{
    using L = StageLayout<T, BY>;
    const Dims d = f.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * BY;
    const int i = x0 + tx, j = y0 + ty;
    const int k0 = (int)blockIdx.z * kc, k1 = min(k0 + kc, d.nz);
    if (k0 >= k1) return;
    const bool rowok = j < d.ny;
    const bool act = rowok && i < d.nx;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    // stages hold planes k0 .. k1 (E is needed one plane past the last H plane)
    auto issue = [&](int s, int k) {
        unsigned char *b = sm + s * L::STAGE_B;
        fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
        mbar_expect_tx(&full[s], L::TX);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + c * L::HALO_B, &M.halo[c], &full[s], x0, y0, k);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + 3 * L::HALO_B + c * L::OWN_B, &M.own[3 + c], &full[s], x0, y0, k);
        tma_load_3d(b + 3 * L::HALO_B + 3 * L::OWN_B, &M.id, &full[s], x0, y0, k);
    };
    if (tid == 0)
        for (int s = 0; s < kStages && k0 + s <= k1; ++s) issue(s, k0 + s);
    const int ic = act ? i : 0, jc = rowok ? j : 0;
    const StretchView<T> &sv = f.s;
    const T cHyz = sv.cHyz[ic], cHzy = sv.cHzy[ic], cHxz = sv.cHxz[jc], cHzx = sv.cHzx[jc];
    ColPml<T> pc{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
    if (PML && rowok) pc = col_pml_h(p, d, i, j, act);
    const int er = ty * L::HW + tx, orow = ty * L::OW + tx;
    {
        const bool ok = wait_stage(&full[0], 0u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 2);
            return;
        }
    }
    T ex = ((const T *)sm)[er], ey = ((const T *)(sm + L::HALO_B))[er];
    PsiRegs<T> qc{}, qn{}, qnn{};
    if (PML && act) {
        psi_load_h(p, d, pc, i, j, k0, qc);
        if (k0 + 1 < k1) psi_load_h(p, d, pc, i, j, k0 + 1, qn);
    }
    for (int k = k0, it = 0; k < k1; ++k, ++it) {
        if (PML && act && k + 2 < k1) psi_load_h(p, d, pc, i, j, k + 2, qnn);  // psi two planes ahead
        const int s = it % kStages, sn = (it + 1) % kStages;
        const bool ok = wait_stage(&full[sn], (uint32_t)((it + 1) / kStages) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(err, 2);
            return;
        }
        const unsigned char *b = sm + s * L::STAGE_B, *bn = sm + sn * L::STAGE_B;
        const T *ext = (const T *)b, *eyt = (const T *)(b + L::HALO_B), *ezt = (const T *)(b + 2 * L::HALO_B);
        const T *hxt = (const T *)(b + 3 * L::HALO_B), *hyt = (const T *)(b + 3 * L::HALO_B + L::OWN_B);
        const T *hzt = (const T *)(b + 3 * L::HALO_B + 2 * L::OWN_B);
        const uint8_t *idt = b + 3 * L::HALO_B + 3 * L::OWN_B;
        const T exk = ((const T *)bn)[er], eyk = ((const T *)(bn + L::HALO_B))[er];
        const T ez = ezt[er];
        const T dEz_i = ezt[er + 1] - ez, dEz_j = ezt[er + L::HW] - ez;
        const T dEx_j = ext[er + L::HW] - ex, dEy_i = eyt[er + 1] - ey;
        const T dEx_k = exk - ex, dEy_k = eyk - ey;
        const int id = idt[orow];
        const T aH = __ldg(&f.aH[id]), bH = __ldg(&f.bH[id]);
        T hx = aH * hxt[orow] - bH * dEz_j * cHxz + bH * dEy_k * sv.cHxy[k];
        T hy = aH * hyt[orow] - bH * dEx_k * sv.cHyx[k] + bH * dEz_i * cHyz;
        T hz = aH * hzt[orow] + bH * dEx_j * cHzx - bH * dEy_i * cHzy;
        if (act) {
            if (PML) pml_h_cell_pre(p, d, pc, i, j, k, qc, dEz_i, dEy_i, dEx_j, dEz_j, dEy_k, dEx_k, hx, hy, hz);
            const int64_t g = d.idx(i, j, k);
            f.Hx[g] = hx; f.Hy[g] = hy; f.Hz[g] = hz;
        }
        ex = exk; ey = eyk;
        qc = qn;
        qn = qnn;
        __syncthreads();
        if (tid == 0 && k + kStages <= k1) issue(s, k + kStages);
    }
}


// Does a block's tile (32 columns from x0, BY rows from y0, planes [k0, k1))
// meet a CPML slab?  E side: slabs [1, np] and [n-np, n-1]; H side: [0, np-1]
// and [n-np, n-1] on each axis.  Blocks that do not run the CPML-free body.
__device__ __forceinline__ bool tile_in_pml(const int np[6], const Dims &d, int x0, int y0, int by, int k0, int k1,
                                            bool eside)
{
    const int lo = eside ? 0 : 1;  // first-end slab reaches index np (E) or np-1 (H)
    const bool x = x0 <= np[kFX1] - lo || x0 + 31 >= d.nx - np[kFX2];
    const bool y = y0 <= np[kFY1] - lo || y0 + by - 1 >= d.ny - np[kFY2];
    const bool z = k0 <= np[kFZ1] - lo || k1 - 1 >= d.nz - np[kFZ2];
    return x || y || z;
}

template <typename T, int BY, bool PML, bool DL, bool GAIN>
__global__ void __launch_bounds__(32 * BY) k_e_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p,
                                                    DlView<T> D, GainView<T> G, int kc, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    // TMA destinations 128-byte aligned in the shared window (SMEM holds 128 spare bytes)
    unsigned char *sm = sm_raw + (((smem_u32(sm_raw) + 127u) & ~127u) - smem_u32(sm_raw));
    const int k0 = max(1, (int)blockIdx.z * kc), k1 = min((int)blockIdx.z * kc + kc, f.d.nz);
    if (PML && tile_in_pml(p.np, f.d, blockIdx.x * 32, blockIdx.y * BY, BY, k0, k1, true))
        e_tma_body<T, BY, true, DL, GAIN>(M, f, p, D, G, kc, err, sm, full);
    else
        e_tma_body<T, BY, false, DL, GAIN>(M, f, p, D, G, kc, err, sm, full);
}

template <typename T, int BY, bool PML>
__global__ void __launch_bounds__(32 * BY) k_h_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p,
                                                    int kc, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = sm_raw + (((smem_u32(sm_raw) + 127u) & ~127u) - smem_u32(sm_raw));
    const int k0 = (int)blockIdx.z * kc, k1 = min(k0 + kc, f.d.nz);
    if (PML && tile_in_pml(p.np, f.d, blockIdx.x * 32, blockIdx.y * BY, BY, k0, k1, false))
        h_tma_body<T, BY, true>(M, f, p, kc, err, sm, full);
    else
        h_tma_body<T, BY, false>(M, f, p, kc, err, sm, full);
}

// The ID-2 cells the TMA E sweep leaves alone: Drude-Lorentz ADE update
// (Drude_Lorentz.cpp:153-227 in 3-D form, curl of the updated H) followed by
// their CPML correction, one thread per cell of the compacted list.
template <typename T, bool PML>
__global__ void __launch_bounds__(128) k_dl_cells(FieldView<T> f, PmlView<T> p, DlView<T> D)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= D.ncell) return;
    const Dims &d = f.d;
    const int64_t g = D.cell[c];
    int i, j, k;
    if (d.pxy * (d.nz + 1) < (int64_t)UINT32_MAX) {  // 32-bit division when the grid allows
        const uint32_t g32 = (uint32_t)g, pxy = (uint32_t)d.pxy, px = (uint32_t)d.px;
        k = (int)(g32 / pxy);
        const uint32_t r = g32 - (uint32_t)k * pxy;
        j = (int)(r / px);
        i = (int)(r - (uint32_t)j * px);
    } else {
        k = (int)(g / d.pxy);
        const int64_t r = g - (int64_t)k * d.pxy;
        j = (int)(r / d.px);
        i = (int)(r - (int64_t)j * d.px);
    }
    const T hx = f.Hx[g], hy = f.Hy[g], hz = f.Hz[g];
    const T dHz_j = hz - f.Hz[g - d.px], dHx_j = hx - f.Hx[g - d.px];
    const T dHz_i = hz - f.Hz[g - 1], dHy_i = hy - f.Hy[g - 1];
    const T dHy_k = hy - f.Hy[g - d.pxy], dHx_k = hx - f.Hx[g - d.pxy];
    const StretchView<T> &s = f.s;
    const T cExz = s.cExz[j], cEzx = s.cEzx[j], cEyz = s.cEyz[i], cEzy = s.cEzy[i], cExy = s.cExy[k], cEyx = s.cEyx[k];
    const T C3 = D.c.C3;
    const T cxx = C3 * dHz_j * cExz - C3 * dHy_k * cExy;
    const T cyy = C3 * dHx_k * cEyx - C3 * dHz_i * cEyz;
    const T czz = C3 * dHy_i * cEzy - C3 * dHx_j * cEzx;
    const int64_t sc = D.ncell;
    T *st = D.state + c;
    T ex = dl_component(D.c, f.Ex[g], cxx, st, sc);
    T ey = dl_component(D.c, f.Ey[g], cyy, st + (int64_t)D.c.stride * sc, sc);
    T ez = dl_component(D.c, f.Ez[g], czz, st + (int64_t)2 * D.c.stride * sc, sc);
    if (PML) {
        const ColPml<T> pc = col_pml_e(p, d, i, j, true);
        pml_e_cell(p, d, pc, i, j, k, dHz_i, dHy_i, dHx_j, dHz_j, dHy_k, dHx_k, ex, ey, ez);
    }
    f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

template <typename T, int BY, bool PML, bool DL, bool GAIN>
void e_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                  const GainView<T> &G, int kc, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_e_tma<T, BY, PML, DL, GAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
        attr = true;
    }
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    k_e_tma<T, BY, PML, DL, GAIN><<<grid, dim3(32, BY), L::SMEM, s>>>(M, f, p, D, G, kc, err);
}

template <typename T, int BY, bool PML>
void h_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_h_tma<T, BY, PML>, cudaFuncAttributeMaxDynamicSharedMemorySize, L::SMEM);
        attr = true;
    }
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    k_h_tma<T, BY, PML><<<grid, dim3(32, BY), L::SMEM, s>>>(M, f, p, kc, err);
}

template <typename T, int BY>
void e_tma_by(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
              const GainView<T> &G, int kc, int *err, cudaStream_t s)
{
    const bool dl = D.on && D.ncell > 0, gn = G.on && G.ncell > 0;
    if (p.on) {
        if (dl && gn) e_tma_launch<T, BY, true, true, true>(M, f, p, D, G, kc, err, s);
        else if (dl) e_tma_launch<T, BY, true, true, false>(M, f, p, D, G, kc, err, s);
        else if (gn) e_tma_launch<T, BY, true, false, true>(M, f, p, D, G, kc, err, s);
        else e_tma_launch<T, BY, true, false, false>(M, f, p, D, G, kc, err, s);
    } else {
        if (dl && gn) e_tma_launch<T, BY, false, true, true>(M, f, p, D, G, kc, err, s);
        else if (dl) e_tma_launch<T, BY, false, true, false>(M, f, p, D, G, kc, err, s);
        else if (gn) e_tma_launch<T, BY, false, false, true>(M, f, p, D, G, kc, err, s);
        else e_tma_launch<T, BY, false, false, false>(M, f, p, D, G, kc, err, s);
    }
}

}  // namespace

template <typename T>
void launch_h_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, FusedShape sh, int *err,
                  cudaStream_t s)
{
    if (sh.by == 4) {
        if (p.on) h_tma_launch<T, 4, true>(M, f, p, sh.kc, err, s);
        else h_tma_launch<T, 4, false>(M, f, p, sh.kc, err, s);
    } else {
        if (p.on) h_tma_launch<T, 8, true>(M, f, p, sh.kc, err, s);
        else h_tma_launch<T, 8, false>(M, f, p, sh.kc, err, s);
    }
}

template <typename T>
void launch_e_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                  const GainView<T> &G, FusedShape sh, int *err, cudaStream_t s)
{
    if (sh.by == 4) e_tma_by<T, 4>(M, f, p, D, G, sh.kc, err, s);
    else e_tma_by<T, 8>(M, f, p, D, G, sh.kc, err, s);
    if (D.on && D.ncell > 0) {
        if (p.on) k_dl_cells<T, true><<<cdiv(D.ncell, 128), 128, 0, s>>>(f, p, D);
        else k_dl_cells<T, false><<<cdiv(D.ncell, 128), 128, 0, s>>>(f, p, D);
    }
}

template void launch_h_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &, FusedShape, int *,
                                  cudaStream_t);
template void launch_h_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &, FusedShape,
                                   int *, cudaStream_t);
template void launch_e_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &,
                                  const DlView<float> &, const GainView<float> &, FusedShape, int *, cudaStream_t);
template void launch_e_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &,
                                   const DlView<double> &, const GainView<double> &, FusedShape, int *, cudaStream_t);

}  // namespace cps
