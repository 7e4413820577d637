// kernels_step.cu -- the one-pass step (sm_100a): H and E of one time step in
// a single z-march over the fields, so each field word crosses HBM once read
// and once written per step instead of twice each in separate H and E sweeps.
//
// The step reads the current buffers (E, H, the H-side CPML psi) and writes
// the other set, which then becomes current: blocks never see a neighbour's
// new values, so a tile computes the new H of its own cells plus a one-cell
// low halo (column x0-1, row y0-1) itself, from staged old values, and the
// new E of its own cells from that tile of new H.  A tile of 32 x BY columns
// marches planes [kb, ke); it first recomputes plane kb-1's new H (its own
// columns only) for the k-difference of plane kb's E.
//
// Per plane, thread 0 keeps kStages planes of staged tiles in flight
// (cp.async.bulk.tensor, one mbarrier each, bounded waits):
//   E: box 40 x (BY+2) from (x0-4, y0-1)   H: box 36 x (BY+1) from (x0-4, y0-1)
//   IDs: box 48 x (BY+1) from (x0-16, y0-1)
// (x origins are multiples of 16 bytes; loads outside the arrays read zeros;
// no multicast).  Plane k's H update uses the staged E of planes k and k+1.
//
// The H-side TF/SF correction (TF_SF::UpdateHField, TF_SF.cpp:1201-1300) is
// added to each new H value as it is computed, halo cells included: a small
// kernel first writes every correction term of the step into dense arrays,
// one per face of the targets' bounding box (the targets lie on its surface),
// and a cell on that surface sums the terms of the faces it lies on, loaded
// at the top of the plane.
// Cells outside the update ranges (boundary planes, ID-2 cells without the
// Drude-Lorentz module) are copied through, so every cell of the new buffers
// is written; ID-2 cells with the module on are left to the Drude-Lorentz
// cell kernel, which runs after the sweep with the old E of the other buffer.
#include <cuda.h>

#include "tma_bodies.cuh"

namespace cps {

namespace {

template <typename T, int BY>
struct StepLayout {
    static constexpr int EW = 40, EH = BY + 2, HW = 36, HH = BY + 1, IW = 48, IH = BY + 1;
    static constexpr int E_B = a128(EW * EH * (int)sizeof(T));
    static constexpr int H_B = a128(HW * HH * (int)sizeof(T));
    static constexpr int I_B = a128(IW * IH);
    static constexpr int STAGE_B = 3 * E_B + 3 * H_B + I_B;
    static constexpr uint32_t TX = 3 * EW * EH * sizeof(T) + 3 * HW * HH * sizeof(T) + IW * IH;
    static constexpr int HN_B = 3 * H_B;  // one new-H tile: 3 components of HW x HH
    static constexpr int SMEM = kStages * STAGE_B + 2 * HN_B + 128;  // + two new-H tiles (plane parity)
};

// Sum of the H-side TF/SF terms at cell (i, j, k): zero off the targets'
// bounding-box surface; a cell on an edge or corner sums its faces in order.
template <typename T>
struct HSum {
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ HSum<T> h_corr_sum(const HCorr<T> &q, int i, int j, int k)
{
    HSum<T> r{T(0), T(0), T(0)};
    if (i < q.box[0] || i > q.box[1] || j < q.box[2] || j > q.box[3] || k < q.box[4] || k > q.box[5]) return r;
    const int c[3] = {i, j, k};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int ax = f >> 1;
        if (c[ax] != q.box[f]) continue;
        const int ua = ax == 0 ? 1 : 0, va = ax == 2 ? 1 : 2;  // the face's (u, v) axes
        const int o = q.base[f] + (c[va] - q.box[2 * va]) * q.nu[f] + (c[ua] - q.box[2 * ua]);
        r.x += __ldg(&q.corr[o]);
        r.y += __ldg(&q.corr[o + q.area[f]]);
        r.z += __ldg(&q.corr[o + 2 * q.area[f]]);
    }
    return r;
}

// stretch coefficients of a column's H update, fixed along the k march
template <typename T>
struct HCol {
    T cHxz, cHzx, cHyz, cHzy;
};

template <typename T>
__device__ __forceinline__ HCol<T> h_col(const StretchView<T> &sv, int i, int j)
{
    return HCol<T>{sv.cHxz[j], sv.cHzx[j], sv.cHyz[i], sv.cHzy[i]};
}

// New H of the cell at tile-local column lx (-1..31), row ly (-1..BY-1) of
// plane k, from stage b (plane k) and bn (plane k+1); the arithmetic of
// h_tma_body.  STORE: write the cell's new psi to pout.
template <typename T, int BY, bool PML, bool TFSF, bool STORE>
__device__ __forceinline__ void h_cell(const FieldView<T> &f, const PmlView<T> &pout, const HSum<T> &hs,
                                       const unsigned char *b, const unsigned char *bn, int lx, int ly, int i, int j,
                                       int k, const HCol<T> &hc, const ColPml<T> &pc, const PsiRegs<T> &r, T &hx,
                                       T &hy, T &hz, bool store = true)
{
    using L = StepLayout<T, BY>;
    const Dims &d = f.d;
    const T *ext = (const T *)b, *eyt = (const T *)(b + L::E_B), *ezt = (const T *)(b + 2 * L::E_B);
    const T *hxt = (const T *)(b + 3 * L::E_B), *hyt = (const T *)(b + 3 * L::E_B + L::H_B);
    const T *hzt = (const T *)(b + 3 * L::E_B + 2 * L::H_B);
    const uint8_t *idt = b + 3 * L::E_B + 3 * L::H_B;
    const int er = (ly + 1) * L::EW + lx + 4, hr = (ly + 1) * L::HW + lx + 4, ir = (ly + 1) * L::IW + lx + 16;
    const T ex = ext[er], ey = eyt[er], ez = ezt[er];
    const T exk = ((const T *)bn)[er], eyk = ((const T *)(bn + L::E_B))[er];
    const T dEz_i = ezt[er + 1] - ez, dEz_j = ezt[er + L::EW] - ez;
    const T dEx_j = ext[er + L::EW] - ex, dEy_i = eyt[er + 1] - ey;
    const T dEx_k = exk - ex, dEy_k = eyk - ey;
    const int id = idt[ir];
    const T aH = __ldg(&f.aH[id]), bH = __ldg(&f.bH[id]);
    const StretchView<T> &sv = f.s;
    hx = aH * hxt[hr] - bH * dEz_j * hc.cHxz + bH * dEy_k * sv.cHxy[k];
    hy = aH * hyt[hr] - bH * dEx_k * sv.cHyx[k] + bH * dEz_i * hc.cHyz;
    hz = aH * hzt[hr] + bH * dEx_j * hc.cHzx - bH * dEy_i * hc.cHzy;
    if (PML)
        pml_h_cell_pre<T, STORE>(pout, d, pc, pml_ch_cell(pout, f.bH, id), i, j, k, r, dEz_i, dEy_i, dEx_j, dEz_j, dEy_k, dEx_k, hx, hy, hz, store);
    if (TFSF) {
        hx = hx + hs.x;
        hy = hy + hs.y;
        hz = hz + hs.z;
    }
}

// Does the tile (H cells x in [x0-1, x0+31], y in [y0-1, y0+BY-1], planes
// [ks, ke); E cells its own columns) meet a CPML slab of either side?
__device__ __forceinline__ bool step_tile_in_pml(const int np[6], const Dims &d, int x0, int y0, int by, int ks, int ke)
{
    return x0 <= np[kFX1] || x0 + 31 >= d.nx - np[kFX2] || y0 <= np[kFY1] || y0 + by - 1 >= d.ny - np[kFY2] ||
           ks <= np[kFZ1] || ke - 1 >= d.nz - np[kFZ2];
}

// Per plane: every thread waits (bounded) for the next plane's stage; warps
// 0..BY-1 compute the new H of their own row, warp BY the halo row y0-1 and
// warp BY+1 (lanes < BY) the halo column x0-1, into the new-H tile of this
// plane's parity; one block barrier (after which the stage of plane k-1 is
// free and is refilled); then warps 0..BY-1 update E.
template <typename T, int BY, bool PML, bool DL, bool GAIN, bool TFSF>
__device__ __forceinline__ void step_body(const StepMaps &M, const FieldView<T> &fo, const FieldView<T> &fn,
                                          const PmlView<T> &pin, const PmlView<T> &pout, const DlView<T> &D,
                                          const GainView<T> &G, const HCorr<T> &hc, int kb, int ke, int *err,
                                          unsigned char *sm, uint64_t *full)
{
    using L = StepLayout<T, BY>;
    constexpr int HS = L::H_B / (int)sizeof(T), ES = L::E_B / (int)sizeof(T);
    const Dims d = fo.d;
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int bx = blockIdx.x, x0 = bx * 32, y0 = blockIdx.y * BY;
    const int ks = max(kb - 1, 0);
    const bool issuer = ty == BY + 1 && tx == 31;  // a lane of the halo-column warp that has no cell
    auto issue = [&](int k) {
        const int s = (k - ks) % kStages;
        unsigned char *b = sm + s * L::STAGE_B;
        fence_proxy_async_smem();  // the stage's previous contents were read through the generic proxy
        mbar_expect_tx(&full[s], L::TX);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + c * L::E_B, &M.e[c], &full[s], x0 - 4, y0 - 1, k);
        for (int c = 0; c < 3; ++c) tma_load_3d(b + 3 * L::E_B + c * L::H_B, &M.h[c], &full[s], x0 - 4, y0 - 1, k);
        tma_load_3d(b + 3 * L::E_B + 3 * L::H_B, &M.id, &full[s], x0 - 16, y0 - 1, k);
    };
    if (issuer)
        for (int k = ks; k < ks + kStages && k <= ke; ++k) issue(k);
    auto wait_plane = [&](int k) {  // bounded; a timeout is reported and the sweep runs on
        const int q = k - ks;
        if (!wait_stage(&full[q % kStages], (uint32_t)(q / kStages) & 1u)) atomicExch(err, 3);
    };
    unsigned char *hn_base = sm + kStages * L::STAGE_B;
    const StretchView<T> &sv = fo.s;

    if (ty >= BY) {
        // ---- halo warps: new H of row y0-1 (warp BY) or column x0-1 (warp BY+1)
        const bool hrow = ty == BY;
        const int hi_ = hrow ? x0 + tx : x0 - 1, hj = hrow ? y0 - 1 : y0 + tx;
        const bool hact = (hrow || tx < BY) && hi_ >= 0 && hj >= 0 && hi_ < d.nx && hj < d.ny;
        const int hlx = hrow ? tx : -1, hly = hrow ? -1 : tx;
        const bool hcell = hrow || tx < BY;
        const int hrh = (hly + 1) * L::HW + hlx + 4;
        const HCol<T> hch = h_col(sv, hact ? hi_ : 0, hact ? hj : 0);
        ColPml<T> pc{-1, 0, -1, 0, T(0), T(0), T(0), T(0)};
        if (PML && hact) pc = col_pml_h(pin, d, hi_, hj, true);
        wait_plane(ks);
        for (int k = ks; k < ke; ++k) {
            const bool store = k >= kb;
            PsiRegs<T> r{};
            if (PML && hact && store) psi_load_h(pin, d, pc, hi_, hj, k, r);
            HSum<T> hs{T(0), T(0), T(0)};
            if (TFSF && hact && store) hs = h_corr_sum(hc, hi_, hj, k);
            wait_plane(k + 1);
            const int q = k - ks;
            const unsigned char *b = sm + (q % kStages) * L::STAGE_B, *bn = sm + ((q + 1) % kStages) * L::STAGE_B;
            if (store && hcell) {
                T *hn = (T *)(hn_base + (k & 1) * L::HN_B);
                T ax = T(0), ay = T(0), az = T(0);
                if (hact) h_cell<T, BY, PML, TFSF, false>(fo, pout, hs, b, bn, hlx, hly, hi_, hj, k, hch, pc, r, ax, ay, az);
                hn[hrh] = ax; hn[HS + hrh] = ay; hn[2 * HS + hrh] = az;
            }
            __syncthreads();
            // every thread is past plane k-1: its stage takes the plane kStages ahead
            if (issuer && k > ks && k - 1 + kStages <= ke) issue(k - 1 + kStages);
        }
        return;
    }

    // ---- own rows
    const int i = x0 + tx, j = y0 + ty;
    const bool inarr = i <= d.nx && j <= d.ny;  // a cell of the arrays (not x padding, not past row ny)
    const bool act_h = i < d.nx && j < d.ny;
    const bool rowok = j >= 1 && j < d.ny;
    const bool act_e_col = rowok && i >= 1 && i < d.nx;
    const int ic = act_e_col ? i : 1, jc = rowok ? j : 1;
    const T cEyz = sv.cEyz[ic], cEzy = sv.cEzy[ic], cExz = sv.cExz[jc], cEzx = sv.cEzx[jc];
    const HCol<T> hco = h_col(sv, act_h ? i : 0, act_h ? j : 0);
    ColPml<T> pce{-1, 0, -1, 0, T(0), T(0), T(0), T(0)}, pch = pce;
    if (PML) {
        if (rowok) pce = col_pml_e(pin, d, i, j, act_e_col);
        if (act_h) pch = col_pml_h(pin, d, i, j, true);
    }
    const int ke0 = max(kb, 1);  // first plane of E updates
    constexpr bool GPRE = GAIN && sizeof(T) == 4;
    // FP32 gain: the segment-dense words of plane k+1 requested during plane k
    GainRegs32 gcur{}, gnext{};
    if constexpr (GPRE) {
        if (ke0 < ke && rowok) gain_fetch32(G, d.idx(i, j, ke0), gcur);
    }
    const int hr = (ty + 1) * L::HW + tx + 4, er = (ty + 1) * L::EW + tx + 4, ir = (ty + 1) * L::IW + tx + 16;
    T hxm = 0, hym = 0;
    wait_plane(ks);
    for (int k = ks; k < ke; ++k) {
        const bool store = k >= kb;
        const bool eplane = store && k >= 1;
        const bool act = act_e_col && eplane;
        PsiRegs<T> qho{}, qe{};
        if (PML) {  // psi of this plane, requested before the wait
            if (act_h) psi_load_h(pin, d, pch, i, j, k, qho);
            if (act) psi_load_e(pin, d, pce, i, j, k, qe);
        }
        HSum<T> hs{T(0), T(0), T(0)};
        if (TFSF && act_h) hs = h_corr_sum(hc, i, j, k);
        if constexpr (GPRE) {
            if (eplane && rowok && k + 1 < ke) gain_fetch32(G, d.idx(i, j, k + 1), gnext);
        }
        wait_plane(k + 1);
        const int q = k - ks;
        const unsigned char *b = sm + (q % kStages) * L::STAGE_B, *bn = sm + ((q + 1) % kStages) * L::STAGE_B;
        T *hn = (T *)(hn_base + (k & 1) * L::HN_B);
        T hx = T(0), hy = T(0), hz = T(0);
        if (act_h)  // psi is written from the chunk's own planes only
            h_cell<T, BY, PML, TFSF, true>(fo, pout, hs, b, bn, tx, ty, i, j, k, hco, pch, qho, hx, hy, hz, store);
        const int64_t g = d.idx(i, j, k);
        if (store) {
            if (act_h) {
                fn.Hx[g] = hx; fn.Hy[g] = hy; fn.Hz[g] = hz;
            } else if (inarr) {
                const T *ht = (const T *)(b + 3 * L::E_B);
                fn.Hx[g] = ht[hr]; fn.Hy[g] = ht[HS + hr]; fn.Hz[g] = ht[2 * HS + hr];
            }
            hn[hr] = hx; hn[HS + hr] = hy; hn[2 * HS + hr] = hz;
        }
        __syncthreads();
        if (store) {
            // E of plane k from the new H tile (the arithmetic of e_tma_body)
            const T *ext = (const T *)b, *eyt = (const T *)(b + L::E_B), *ezt = (const T *)(b + 2 * L::E_B);
            const uint8_t *idt = b + 3 * L::E_B + 3 * L::H_B;
            T ex = ext[er], ey = eyt[er], ez = ezt[er];
            if (eplane) {
                const T dHz_j = hz - hn[2 * HS + hr - L::HW], dHx_j = hx - hn[hr - L::HW];
                const T dHz_i = hz - hn[2 * HS + hr - 1], dHy_i = hy - hn[HS + hr - 1];
                const T dHy_k = hy - hym, dHx_k = hx - hxm;
                const int id = idt[ir];
                const T cExy = sv.cExy[k], cEyx = sv.cEyx[k];
                if (act) {
                    if (id == CPS_ID_PEC) {
                        ex = T(0); ey = T(0); ez = T(0);
                    } else if (id != CPS_ID_DISPERSIVE) {
                        const T aE = __ldg(&fo.aE[id]), bE = __ldg(&fo.bE[id]);
                        ex = aE * ex + bE * dHz_j * cExz - bE * dHy_k * cExy;
                        ey = aE * ey + bE * dHx_k * cEyx - bE * dHz_i * cEyz;
                        ez = aE * ez + bE * dHy_i * cEzy - bE * dHx_j * cEzx;
                    }
                }
                if constexpr (GPRE) {
                    if (act && id == G.gain_id) gain_apply32(G, g, gcur, ex, ey, ez);
                    gcur = gnext;
                } else if (GAIN && rowok) {
                    gain_warp(G, d, j, k, bx, act, id, ex, ey, ez);
                }
                if (act && !(DL && id == CPS_ID_DISPERSIVE)) {
                    if (PML) pml_e_cell_pre(pin, d, pce, pml_ce_cell(pin, fo.bE, id), i, j, k, qe, dHz_i, dHy_i, dHx_j, dHz_j, dHy_k, dHx_k, ex, ey, ez);
                    fn.Ex[g] = ex; fn.Ey[g] = ey; fn.Ez[g] = ez;
                } else if (!act && inarr) {
                    fn.Ex[g] = ex; fn.Ey[g] = ey; fn.Ez[g] = ez;
                }
            } else if (inarr) {  // plane 0: E is not updated
                fn.Ex[g] = ex; fn.Ey[g] = ey; fn.Ez[g] = ez;
            }
        }
        hxm = hx; hym = hy;
    }
    if (ke == d.nz && inarr) {  // plane nz is never updated: copy it through
        const unsigned char *b = sm + ((ke - ks) % kStages) * L::STAGE_B;
        const T *et = (const T *)b, *ht = (const T *)(b + 3 * L::E_B);
        const int64_t g = d.idx(i, j, ke);
        fn.Ex[g] = et[er]; fn.Ey[g] = et[ES + er]; fn.Ez[g] = et[2 * ES + er];
        fn.Hx[g] = ht[hr]; fn.Hy[g] = ht[HS + hr]; fn.Hz[g] = ht[2 * HS + hr];
    }
}

template <typename T, int BY, bool PML, bool DL, bool GAIN, bool TFSF>
__global__ void __launch_bounds__(32 * (BY + 2), (GAIN || sizeof(T) == 8) ? 2 : 3) k_step_tma(const __grid_constant__ StepMaps M, FieldView<T> fo,
                                                      FieldView<T> fn, PmlView<T> pin, PmlView<T> pout, DlView<T> D,
                                                      GainView<T> G, HCorr<T> hc, int kc, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    const Dims &d = fo.d;
    const int kb = blockIdx.z * kc;
    if (kb >= d.nz) return;
    const int ke = min(kb + kc, d.nz);
    init_stages(full);
    if (PML && step_tile_in_pml(pin.np, d, blockIdx.x * 32, blockIdx.y * BY, BY, max(kb - 1, 0), ke))
        step_body<T, BY, true, DL, GAIN, TFSF>(M, fo, fn, pin, pout, D, G, hc, kb, ke, err, sm, full);
    else
        step_body<T, BY, false, DL, GAIN, TFSF>(M, fo, fn, pin, pout, D, G, hc, kb, ke, err, sm, full);
}

// the Drude-Lorentz cells after a one-pass sweep: old E from fo, H and new E in fn
template <typename T, bool PML>
__global__ void __launch_bounds__(128) k_dl_cells_step(FieldView<T> fn, FieldView<T> fo, PmlView<T> p, DlView<T> D)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= D.ncell) return;
    dl_cell_any<T, PML>(fn, fo, p, D, c);
}

// one thread per H-side contribution: its term at step n (the arithmetic of
// inject_target) into its face-array slot
template <typename T>
__global__ void __launch_bounds__(256) k_h_corrections(const InjContrib *__restrict__ ct,
                                                       const int32_t *__restrict__ slot, int n_ct,
                                                       const T *__restrict__ table, int Nt, double n, T *corr)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_ct) return;
    const InjContrib b = ct[c];
    const T inc = (T)inc_lookup<T>(table, Nt, n - b.delay);
    corr[slot[c]] = (T)b.coef * inc * (T)b.profile;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// dynamic shared memory and the largest shared-memory carveout, set once per
// kernel and device
template <auto K>
bool set_smem(int bytes)
{
    return kernel_smem<K>(bytes, 100);
}

template <typename T, int BY, bool PML, bool DL, bool GAIN, bool TFSF>
void step_launch(const StepMaps &M, const FieldView<T> &fo, const FieldView<T> &fn, const PmlView<T> &pin,
                 const PmlView<T> &pout, const DlView<T> &D, const GainView<T> &G, const HCorr<T> &hc, int kc,
                 int *err, cudaStream_t s)
{
    using L = StepLayout<T, BY>;
    if (!set_smem<k_step_tma<T, BY, PML, DL, GAIN, TFSF>>(L::SMEM)) return;
    const Dims &d = fo.d;
    dim3 grid(cdiv(d.nx + 1, 32), cdiv(d.ny + 1, BY), cdiv(d.nz, kc));
    k_step_tma<T, BY, PML, DL, GAIN, TFSF><<<grid, dim3(32, BY + 2), L::SMEM, s>>>(M, fo, fn, pin, pout, D, G, hc, kc,
                                                                                  err);
}

template <typename T, int BY, bool PML>
void step_by_flags(const StepMaps &M, const FieldView<T> &fo, const FieldView<T> &fn, const PmlView<T> &pin,
                   const PmlView<T> &pout, const DlView<T> &D, const GainView<T> &G, const HCorr<T> &hc, int kc,
                   int *err, cudaStream_t s)
{
    const bool dl = D.on && D.ncell > 0, gn = G.on && G.ncell > 0, tf = hc.corr != nullptr;
    const int key = (dl ? 1 : 0) | (gn ? 2 : 0) | (tf ? 4 : 0);
    switch (key) {
    case 0: step_launch<T, BY, PML, false, false, false>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 1: step_launch<T, BY, PML, true, false, false>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 2: step_launch<T, BY, PML, false, true, false>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 3: step_launch<T, BY, PML, true, true, false>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 4: step_launch<T, BY, PML, false, false, true>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 5: step_launch<T, BY, PML, true, false, true>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    case 6: step_launch<T, BY, PML, false, true, true>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    default: step_launch<T, BY, PML, true, true, true>(M, fo, fn, pin, pout, D, G, hc, kc, err, s); break;
    }
}

}  // namespace

template <typename T>
void launch_step_tma(const StepMaps &M, const FieldView<T> &fo, const FieldView<T> &fn, const PmlView<T> &pin,
                     const PmlView<T> &pout, const DlView<T> &D, const GainView<T> &G, const HCorr<T> &hc,
                     FusedShape sh, int *err, cudaStream_t s)
{
    if (sh.by == 4) {
        if (pin.on) step_by_flags<T, 4, true>(M, fo, fn, pin, pout, D, G, hc, sh.kc, err, s);
        else step_by_flags<T, 4, false>(M, fo, fn, pin, pout, D, G, hc, sh.kc, err, s);
    } else {
        if (pin.on) step_by_flags<T, 8, true>(M, fo, fn, pin, pout, D, G, hc, sh.kc, err, s);
        else step_by_flags<T, 8, false>(M, fo, fn, pin, pout, D, G, hc, sh.kc, err, s);
    }
}

template <typename T>
void launch_dl_cells_step(const FieldView<T> &fn, const FieldView<T> &fo, const PmlView<T> &p, const DlView<T> &D,
                          cudaStream_t s)
{
    if (!D.on || D.ncell <= 0) return;
    if (p.on) k_dl_cells_step<T, true><<<cdiv(D.ncell, 128), 128, 0, s>>>(fn, fo, p, D);
    else k_dl_cells_step<T, false><<<cdiv(D.ncell, 128), 128, 0, s>>>(fn, fo, p, D);
}

template <typename T>
void launch_h_corrections(const InjContrib *ct, const int32_t *slot, int ncontrib, const T *table, int Nt, double n,
                          T *corr, cudaStream_t s)
{
    if (ncontrib <= 0) return;
    k_h_corrections<T><<<cdiv(ncontrib, 256), 256, 0, s>>>(ct, slot, ncontrib, table, Nt, n, corr);
}

template void launch_h_corrections<float>(const InjContrib *, const int32_t *, int, const float *, int, double,
                                          float *, cudaStream_t);
template void launch_h_corrections<double>(const InjContrib *, const int32_t *, int, const double *, int, double,
                                           double *, cudaStream_t);
template void launch_step_tma<float>(const StepMaps &, const FieldView<float> &, const FieldView<float> &,
                                     const PmlView<float> &, const PmlView<float> &, const DlView<float> &,
                                     const GainView<float> &, const HCorr<float> &, FusedShape, int *, cudaStream_t);
template void launch_step_tma<double>(const StepMaps &, const FieldView<double> &, const FieldView<double> &,
                                      const PmlView<double> &, const PmlView<double> &, const DlView<double> &,
                                      const GainView<double> &, const HCorr<double> &, FusedShape, int *,
                                      cudaStream_t);
template void launch_dl_cells_step<float>(const FieldView<float> &, const FieldView<float> &, const PmlView<float> &,
                                          const DlView<float> &, cudaStream_t);
template void launch_dl_cells_step<double>(const FieldView<double> &, const FieldView<double> &,
                                           const PmlView<double> &, const DlView<double> &, cudaStream_t);

}  // namespace cps
