// tma_bodies.cuh -- the per-tile bodies of the TMA-fed fused H and E sweeps,
// shared by the one-grid kernels (kernels_tma.cu) and the batched kernels
// over many grids (kernels_batch.cu).
//
// A tile is a 32 x BY block of (i, j) columns marching planes [k0, k1) in k.
// Thread 0 keeps kStages planes of x-y tiles in flight: for each plane one
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
// with the plane kStages ahead.
//
// Stage bookkeeping runs on a block-uniform counter `ctr` of planes that went
// through the ring, so a block may run several tiles in a row (persistent
// launches): plane q of the block's life uses stage q % kStages and waits for
// mbarrier phase parity (q / kStages) & 1.  The mbarriers are initialised once
// per block by the caller (init_stages).
//
// Every wait is bounded (kWaitLimit polls and kWaitNs of wall-clock time,
// whichever ends first).  When a wait gives up, the body records an error
// code in err[0] for the host, thread 0 waits (bounded again) for the loads
// of the other planes still in flight so that no copy into the block's shared
// memory outlives it, and the body returns false.  err[1] is a test setting
// (0 in normal use): the first plane of every tile then expects err[1] more
// bytes than its loads bring, so its wait runs out and the sweep reports the
// timeout without any fault (cps_grid_set_wait_skew).
#pragma once

#include "sweep_cells.cuh"
#include "tma.cuh"

namespace cps {

constexpr int kStages = 4;
constexpr int kWaitLimit = 1 << 18;
constexpr uint64_t kWaitNs = 1000000000ull;  // 1 s

__host__ __device__ constexpr int a128(int b) { return (b + 127) / 128 * 128; }

// One stage: three halo tiles, three own tiles, the IDs and, for an FP32 E
// sweep with gain (G), the tile's segment-dense gain words [row][word][32].
template <typename T, int BY, bool G = false>
struct StageLayout {
    static constexpr int HW = 36, HH = BY + 1, OW = 32, OH = BY;
    static constexpr int HALO_B = a128(HW * HH * (int)sizeof(T));
    static constexpr int OWN_B = a128(OW * OH * (int)sizeof(T));
    static constexpr int ID_B = a128(OW * OH);
    static constexpr int GAIN_OFF = 3 * HALO_B + 3 * OWN_B + ID_B;
    static constexpr int GAIN_RAW = G ? 32 * kGainPersist * BY * 4 : 0;
    static constexpr int STAGE_B = GAIN_OFF + a128(GAIN_RAW);
    static constexpr uint32_t TX = 3 * HW * HH * sizeof(T) + 3 * OW * OH * sizeof(T) + OW * OH + GAIN_RAW;
    // planes in flight: three when the stage carries gain words (more blocks
    // per SM fit), kStages otherwise
    static constexpr int NS = G ? 3 : kStages;
    static constexpr int SMEM = NS * STAGE_B + 128;
};

// the stage layout of an E sweep (FP32 with gain stages the gain words)
template <typename T, int BY, bool GAIN>
using ELayout = StageLayout<T, BY, GAIN && sizeof(T) == 4>;

struct TileXYZ {
    int bx, by, bz;  // tile index along x (32 columns), y (BY rows), z (kc planes)
};

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool wait_stage(uint64_t *bar, uint32_t phase)
{
    if (mbar_try_wait(bar, phase)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (int it = 1; it < kWaitLimit; ++it) {
        if (mbar_try_wait(bar, phase)) return true;
        if ((it & 255) == 0 && globaltimer_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// After a wait gave up: thread 0 waits (bounded) for the planes [pl0, pl1]
// of the tile whose loads may still be in flight (the plane that gave up has
// had its whole limit already)
template <int NS = kStages>
__device__ __forceinline__ void drain_stages(uint64_t *full, uint32_t c0, int pl0, int pl1)
{
    for (int pl = pl0; pl <= pl1; ++pl) {
        const uint32_t q = c0 + (uint32_t)pl;
        wait_stage(&full[q % NS], (q / NS) & 1u);
    }
}

// the test setting err[1] (extra bytes the first plane of a tile expects)
__device__ __forceinline__ uint32_t wait_skew(const int *err)
{
    return (uint32_t)*(const volatile int *)(err + 1);
}

// 128-byte aligned start of the dynamic shared window (SMEM holds 128 spare bytes)
__device__ __forceinline__ unsigned char *align_smem(unsigned char *raw)
{
    return raw + (((smem_u32(raw) + 127u) & ~127u) - smem_u32(raw));
}

__device__ __forceinline__ void init_stages(uint64_t *full)
{
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&full[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
}

// Does a tile (32 columns from x0, BY rows from y0, planes [k0, k1)) meet a
// CPML slab?  E side: slabs [1, np] and [n-np, n-1]; H side: [0, np-1] and
// [n-np, n-1] on each axis.  Tiles that do not run the CPML-free body.
__device__ __forceinline__ bool tile_in_pml(const int np[6], const Dims &d, int x0, int y0, int by, int k0, int k1,
                                            bool eside)
{
    const int lo = eside ? 0 : 1;  // first-end slab reaches index np (E) or np-1 (H)
    const bool x = x0 <= np[kFX1] - lo || x0 + 31 >= d.nx - np[kFX2];
    const bool y = y0 <= np[kFY1] - lo || y0 + by - 1 >= d.ny - np[kFY2];
    const bool z = k0 <= np[kFZ1] - lo || k1 - 1 >= d.nz - np[kFZ2];
    return x || y || z;
}

// Up to six boxes of tiles (in tile coordinates) covered by one launch, one
// block per tile: a sweep launches its interior tiles (one box, the CPML-free
// body) and its CPML tiles (the rest of the grid, up to six boxes) separately,
// so the interior blocks are not held to the CPML body's register count.
struct TileBoxes {
    int n;         // boxes in use
    int start[7];  // first block of each box; start[n] = blocks in the launch
    int bx0[6], by0[6], bz0[6];
    int nbx[6], nby[6];
};

__device__ __forceinline__ TileXYZ box_tile(const TileBoxes &b, int q)
{
    int k = 0;
    while (k + 1 < b.n && q >= b.start[k + 1]) ++k;
    const int r = q - b.start[k];
    const int nxy = b.nbx[k] * b.nby[k];
    const int z = r / nxy, rem = r - z * nxy;
    const int y = rem / b.nbx[k];
    return TileXYZ{b.bx0[k] + rem - y * b.nbx[k], b.by0[k] + y, b.bz0[k] + z};
}

// E sweep of one tile: planes max(1, bz*kc) .. min(bz*kc+kc, nz)-1.
template <typename T, int BY, bool PML, bool DL, bool GAIN>
__device__ __forceinline__ bool e_tma_body(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p,
                                           const DlView<T> &D, const GainView<T> &G, int kc, TileXYZ t,
                                           uint32_t &ctr, int *err, unsigned char *sm, uint64_t *full)
{
    // FP32 gain: the tile's gain words travel with its fields in every stage
    constexpr bool GST = GAIN && sizeof(T) == 4;
    using L = StageLayout<T, BY, GST>;
    const Dims d = f.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int x0 = t.bx * 32, y0 = t.by * BY;
    const int i = x0 + tx, j = y0 + ty;
    const int k0 = max(1, t.bz * kc), k1 = min(t.bz * kc + kc, d.nz);
    if (k0 >= k1) return true;  // whole block
    const bool rowok = j >= 1 && j < d.ny;
    const bool act = rowok && i >= 1 && i < d.nx;
    const uint32_t c0 = ctr;
    const int npl = k1 - k0;
    const uint32_t skew = tid == 0 ? wait_skew(err) : 0u;
    auto issue = [&](int pl, int k) {
        const int s = (int)((c0 + (uint32_t)pl) % L::NS);
        unsigned char *b = sm + s * L::STAGE_B;
        fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
        mbar_expect_tx(&full[s], L::TX + (pl == 0 ? skew : 0u));
        for (int c = 0; c < 3; ++c) tma_load_3d(b + c * L::HALO_B, &M.halo[3 + c], &full[s], x0 - 4, y0 - 1, k);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + 3 * L::HALO_B + c * L::OWN_B, &M.own[c], &full[s], x0, y0, k);
        tma_load_3d(b + 3 * L::HALO_B + 3 * L::OWN_B, &M.id, &full[s], x0, y0, k);
        if (GST) tma_load_5d(b + L::GAIN_OFF, &M.gain, &full[s], 0, 0, t.bx, y0, k);
    };
    if (tid == 0)
        for (int pl = 0; pl < L::NS && k0 + pl < k1; ++pl) issue(pl, k0 + pl);
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
        const uint32_t q = c0 + (uint32_t)it;
        const int s = (int)(q % L::NS);
        const bool ok = wait_stage(&full[s], (q / L::NS) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(err, 1);
                drain_stages<L::NS>(full, c0, it + 1, min(it + L::NS - 1, npl - 1));
            }
            return false;
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
        if constexpr (GST) {
            // the gain list holds interior cells only (act), with the gain ID
            if (act && id == G.gain_id) {
                GainRegs32 r;
                gain_staged32((const float *)(b + L::GAIN_OFF) + ty * kGainPersist * 32 + tx, r);
                gain_apply32(G, d.idx(i, j, k), r, ex, ey, ez);
            }
        } else if (GAIN && rowok) {
            gain_warp(G, d, j, k, t.bx, act, id, ex, ey, ez);
        }
        // ID-2 cells are left untouched here: the Drude-Lorentz cell kernel
        // updates them (ADE, then CPML, the reference order) beside the sweep
        if (act && !(DL && id == CPS_ID_DISPERSIVE)) {
            if (PML) pml_e_cell_pre(p, d, pc, pml_ce_cell(p, f.bE, id), i, j, k, qc, dHz_i, dHy_i, dHx_j, dHz_j, dHy_k, dHx_k, ex, ey, ez);
            const int64_t g = d.idx(i, j, k);
            f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
        }
        hxm = hx; hym = hy;
        qc = qn;
        qn = qnn;
        __syncthreads();
        if (tid == 0 && k + L::NS < k1) issue(it + L::NS, k + L::NS);
    }
    ctr = c0 + (uint32_t)(k1 - k0);
    return true;
}

// H sweep of one tile: planes bz*kc .. min(bz*kc+kc, nz)-1 (E is staged one
// plane past the last H plane).
template <typename T, int BY, bool PML>
__device__ __forceinline__ bool h_tma_body(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc,
                                           TileXYZ t, uint32_t &ctr, int *err, unsigned char *sm, uint64_t *full)
{
    using L = StageLayout<T, BY>;
    const Dims d = f.d;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int x0 = t.bx * 32, y0 = t.by * BY;
    const int i = x0 + tx, j = y0 + ty;
    const int k0 = t.bz * kc, k1 = min(k0 + kc, d.nz);
    if (k0 >= k1) return true;
    const bool rowok = j < d.ny;
    const bool act = rowok && i < d.nx;
    const uint32_t c0 = ctr;
    const int npl = k1 - k0;  // planes k0..k1 go through the ring (E one past the last H plane)
    const uint32_t skew = tid == 0 ? wait_skew(err) : 0u;
    auto issue = [&](int pl, int k) {
        const int s = (int)((c0 + (uint32_t)pl) % kStages);
        unsigned char *b = sm + s * L::STAGE_B;
        fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
        mbar_expect_tx(&full[s], L::TX + (pl == 0 ? skew : 0u));
        for (int c = 0; c < 3; ++c) tma_load_3d(b + c * L::HALO_B, &M.halo[c], &full[s], x0, y0, k);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + 3 * L::HALO_B + c * L::OWN_B, &M.own[3 + c], &full[s], x0, y0, k);
        tma_load_3d(b + 3 * L::HALO_B + 3 * L::OWN_B, &M.id, &full[s], x0, y0, k);
    };
    if (tid == 0)
        for (int pl = 0; pl < kStages && k0 + pl <= k1; ++pl) issue(pl, k0 + pl);
    const int ic = act ? i : 0, jc = rowok ? j : 0;
    const StretchView<T> &sv = f.s;
    const T cHyz = sv.cHyz[ic], cHzy = sv.cHzy[ic], cHxz = sv.cHxz[jc], cHzx = sv.cHzx[jc];
    ColPml<T> pc{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
    if (PML && rowok) pc = col_pml_h(p, d, i, j, act);
    const int er = ty * L::HW + tx, orow = ty * L::OW + tx;
    const int s0 = (int)(c0 % kStages);
    {
        const bool ok = wait_stage(&full[s0], (c0 / kStages) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(err, 2);
                drain_stages(full, c0, 1, min(kStages - 1, npl));
            }
            return false;
        }
    }
    T ex = ((const T *)(sm + s0 * L::STAGE_B))[er], ey = ((const T *)(sm + s0 * L::STAGE_B + L::HALO_B))[er];
    // psi of plane k+1 requested at the top of plane k into the other of two
    // register slots (the loop is unrolled by two, so the slots are never copied)
    PsiRegs<T> qA{}, qB{};
    if (PML && act) psi_load_h(p, d, pc, i, j, k0, qA);
    for (int kb = k0, itb = 0; kb < k1; kb += 2, itb += 2) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int k = kb + u, it = itb + u;
            if (k >= k1) break;
            PsiRegs<T> &qc = u == 0 ? qA : qB, &qn = u == 0 ? qB : qA;
            if (PML && act && k + 1 < k1) psi_load_h(p, d, pc, i, j, k + 1, qn);
            const uint32_t q = c0 + (uint32_t)it, qn1 = q + 1u;
            const int s = (int)(q % kStages), sn = (int)(qn1 % kStages);
            const bool ok = wait_stage(&full[sn], (qn1 / kStages) & 1u);
            if (__syncthreads_or(!ok)) {
                if (tid == 0) {
                    atomicExch(err, 2);
                    drain_stages(full, c0, it + 2, min(it + kStages - 1, npl));
                }
                return false;
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
                if (PML)
                    pml_h_cell_pre(p, d, pc, pml_ch_cell(p, f.bH, id), i, j, k, qc, dEz_i, dEy_i, dEx_j, dEz_j, dEy_k,
                                   dEx_k, hx, hy, hz);
                const int64_t g = d.idx(i, j, k);
                f.Hx[g] = hx; f.Hy[g] = hy; f.Hz[g] = hz;
            }
            ex = exk; ey = eyk;
            __syncthreads();
            if (tid == 0 && k + kStages <= k1) issue(it + kStages, k + kStages);
        }
    }
    ctr = c0 + (uint32_t)(k1 - k0 + 1);
    return true;
}

// Drude-Lorentz cell c of a grid's compacted list (Drude_Lorentz.cpp:153-227
// in 3-D form, curl of the updated H), followed by its CPML correction.  The
// cell's old E is read from fo (the same view as f in place; the other field
// buffer after a one-pass step), H and the new E from/to f.
// ND < 0: pole counts taken at run time from D.c (any count); ND >= 0: the
// cell's ND Drude and NL Lorentz poles fixed at compile time, state loaded first.
template <typename T, bool PML, int ND = -1, int NL = 0>
__device__ __forceinline__ void dl_cell(const FieldView<T> &f, const FieldView<T> &fo, const PmlView<T> &p,
                                        const DlView<T> &D, int64_t c)
{
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
    T ex = fo.Ex[g], ey = fo.Ey[g], ez = fo.Ez[g];
    if (ND >= 0) {
        // every state word of the cell is requested before any is used
        constexpr int W = (ND < 0 ? 0 : ND) + 2 * NL + 1;
        constexpr int NDV = ND < 0 ? 0 : ND;
        T w[3][W];
#pragma unroll
        for (int cpt = 0; cpt < 3; ++cpt)
#pragma unroll
            for (int q = 0; q < W; ++q) w[cpt][q] = st[((int64_t)cpt * W + q) * sc];
        ex = dl_component_regs<T, NDV, NL>(D.c, ex, cxx, w[0], st, sc);
        ey = dl_component_regs<T, NDV, NL>(D.c, ey, cyy, w[1], st + (int64_t)W * sc, sc);
        ez = dl_component_regs<T, NDV, NL>(D.c, ez, czz, w[2], st + (int64_t)2 * W * sc, sc);
    } else {
        ex = dl_component(D.c, ex, cxx, st, sc);
        ey = dl_component(D.c, ey, cyy, st + (int64_t)D.c.stride * sc, sc);
        ez = dl_component(D.c, ez, czz, st + (int64_t)2 * D.c.stride * sc, sc);
    }
    if (PML) {
        const ColPml<T> pc = col_pml_e(p, d, i, j, true);
        pml_e_cell(p, d, pc, pml_ce_cell(p, f.bE, CPS_ID_DISPERSIVE), i, j, k, dHz_i, dHy_i, dHx_j, dHz_j, dHy_k, dHx_k, ex, ey, ez);
    }
    f.Ex[g] = ex; f.Ey[g] = ey; f.Ez[g] = ez;
}

// dl_cell with the pole counts of the grid's material dispatched to a
// compile-time form where one exists
template <typename T, bool PML>
__device__ __forceinline__ void dl_cell_any(const FieldView<T> &f, const FieldView<T> &fo, const PmlView<T> &p,
                                            const DlView<T> &D, int64_t c)
{
    const int nd = D.c.nD, nl = D.c.nL;
    if (nd == 1 && nl == 2) dl_cell<T, PML, 1, 2>(f, fo, p, D, c);
    else if (nd == 1 && nl == 1) dl_cell<T, PML, 1, 1>(f, fo, p, D, c);
    else if (nd == 1 && nl == 0) dl_cell<T, PML, 1, 0>(f, fo, p, D, c);
    else if (nd == 0 && nl == 1) dl_cell<T, PML, 0, 1>(f, fo, p, D, c);
    else if (nd == 0 && nl == 2) dl_cell<T, PML, 0, 2>(f, fo, p, D, c);
    else dl_cell<T, PML>(f, fo, p, D, c);
}

}  // namespace cps
