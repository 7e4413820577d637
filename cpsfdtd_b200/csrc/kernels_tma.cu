// kernels_tma.cu -- one-grid launches of the TMA-fed fused H and E sweeps
// (sm_100a): one block per 32 x BY x kc tile, bodies in tma_bodies.cuh.
#include <cuda.h>
#include <string.h>

#include <algorithm>

#include "tma_bodies.cuh"

namespace cps {

namespace {

// One block per tile of the launch's boxes.  PM selects the body: 0 the
// CPML-free body for every tile, 1 the CPML body for every tile, 2 the body
// each tile needs (tile_in_pml).  Sweeps without gain run one launch (PM 2).
// An FP32 sweep with gain (its gain words staged with the fields) runs every
// tile on the CPML body in one launch (PM 1; the body leaves cells outside
// the slabs as the CPML-free body would, bit for bit): measured faster than
// CPML and interior tiles as two launches at every grid size tried, 128^3 to
// 384^3, since a second launch's partial last wave costs more than the
// interior blocks gain from the CPML-free body's lower register count.  An
// FP64 sweep with gain (gain words read on the cell list) keeps the two
// launches, so its interior blocks are not held to the CPML body's registers.
template <typename T, int BY, int PM, bool DL, bool GAIN>
__global__ void __launch_bounds__(32 * BY, GAIN ? 512 / (32 * BY) : 1024 / (32 * BY))
    k_e_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p, DlView<T> D, GainView<T> G, int kc,
            const __grid_constant__ TileBoxes tb, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    const TileXYZ t = box_tile(tb, (int)blockIdx.x);
    const int k0 = max(1, t.bz * kc), k1 = min(t.bz * kc + kc, f.d.nz);
    if (k0 >= k1) return;
    init_stages(full);
    uint32_t ctr = 0;
    if (PM == 1 || (PM == 2 && tile_in_pml(p.np, f.d, t.bx * 32, t.by * BY, BY, k0, k1, true)))
        e_tma_body<T, BY, PM != 0, DL, GAIN>(M, f, p, D, G, kc, t, ctr, err, sm, full);
    else
        e_tma_body<T, BY, false, DL, GAIN>(M, f, p, D, G, kc, t, ctr, err, sm, full);
}

template <typename T, int BY, int PM>
__global__ void __launch_bounds__(32 * BY) k_h_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p,
                                                    int kc, const __grid_constant__ TileBoxes tb, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    const TileXYZ t = box_tile(tb, (int)blockIdx.x);
    const int k0 = t.bz * kc, k1 = min(k0 + kc, f.d.nz);
    if (k0 >= k1) return;
    init_stages(full);
    uint32_t ctr = 0;
    if (PM == 1 || (PM == 2 && tile_in_pml(p.np, f.d, t.bx * 32, t.by * BY, BY, k0, k1, false)))
        h_tma_body<T, BY, PM != 0>(M, f, p, kc, t, ctr, err, sm, full);
    else
        h_tma_body<T, BY, false>(M, f, p, kc, t, ctr, err, sm, full);
}

// The ID-2 cells the TMA E sweep leaves alone, one thread per cell of the
// compacted list.
template <typename T, bool PML>
__global__ void __launch_bounds__(128) k_dl_cells(FieldView<T> f, PmlView<T> p, DlView<T> D)
{
    const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= D.ncell) return;
    dl_cell_any<T, PML>(f, f, p, D, c);
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// the shared-memory attribute of each kernel, set once per device (outside
// any capture when tma_attributes runs first)
template <auto K>
bool set_smem(int bytes)
{
    return kernel_smem<K>(bytes);
}

// Interior and CPML tiles of a sweep as tile boxes.  A tile meets a CPML slab
// when its x, y or z range does (tile_in_pml in tma_bodies.cuh, per axis), so
// the interior tiles form one box [a0, a1) per axis and the CPML tiles the
// rest: below and above the interior in z (whole planes of tiles), then in y,
// then in x.
struct SweepTiles {
    TileBoxes interior, pml;
};

inline void add_box(TileBoxes &b, int x0, int x1, int y0, int y1, int z0, int z1)
{
    if (x1 <= x0 || y1 <= y0 || z1 <= z0) return;
    const int k = b.n++;
    b.bx0[k] = x0; b.by0[k] = y0; b.bz0[k] = z0;
    b.nbx[k] = x1 - x0; b.nby[k] = y1 - y0;
    b.start[k + 1] = b.start[k] + (x1 - x0) * (y1 - y0) * (z1 - z0);
}

// every tile of the grid as one box
inline TileBoxes whole_grid(const Dims &d, int by, int kc)
{
    TileBoxes b;
    memset(&b, 0, sizeof(b));
    add_box(b, 0, (int)cdiv(d.nx, 32), 0, (int)cdiv(d.ny, by), 0, (int)cdiv(d.nz, kc));
    return b;
}

inline SweepTiles sweep_tiles(const int np[6], bool pml_on, const Dims &d, int by, int kc, bool eside)
{
    const int tx = (int)cdiv(d.nx, 32), ty = (int)cdiv(d.ny, by), tz = (int)cdiv(d.nz, kc);
    SweepTiles t;
    memset(&t, 0, sizeof(t));
    if (!pml_on) {
        add_box(t.interior, 0, tx, 0, ty, 0, tz);
        return t;
    }
    const int lo = eside ? 0 : 1;
    // per axis: the first and one-past-last tile index that meets no slab
    auto interval = [](int n, auto in_slab, int &a0, int &a1) {
        a0 = 0;
        while (a0 < n && in_slab(a0)) ++a0;
        a1 = a0;
        while (a1 < n && !in_slab(a1)) ++a1;
        for (int q = a1; q < n; ++q)
            if (!in_slab(q)) { a0 = a1 = 0; return; }  // not one interval: every tile takes the CPML body
    };
    int ax0, ax1, ay0, ay1, az0, az1;
    interval(tx, [&](int b) { const int x0 = 32 * b; return x0 <= np[kFX1] - lo || x0 + 31 >= d.nx - np[kFX2]; },
             ax0, ax1);
    interval(ty, [&](int b) { const int y0 = by * b; return y0 <= np[kFY1] - lo || y0 + by - 1 >= d.ny - np[kFY2]; },
             ay0, ay1);
    interval(tz, [&](int b) {
        const int k0 = eside ? std::max(1, b * kc) : b * kc, k1 = std::min(b * kc + kc, d.nz);
        return k0 <= np[kFZ1] - lo || k1 - 1 >= d.nz - np[kFZ2];
    }, az0, az1);
    if (ax1 <= ax0 || ay1 <= ay0 || az1 <= az0) {
        add_box(t.pml, 0, tx, 0, ty, 0, tz);
        return t;
    }
    add_box(t.interior, ax0, ax1, ay0, ay1, az0, az1);
    add_box(t.pml, 0, tx, 0, ty, 0, az0);
    add_box(t.pml, 0, tx, 0, ty, az1, tz);
    add_box(t.pml, 0, tx, 0, ay0, az0, az1);
    add_box(t.pml, 0, tx, ay1, ty, az0, az1);
    add_box(t.pml, 0, ax0, ay0, ay1, az0, az1);
    add_box(t.pml, ax1, tx, ay0, ay1, az0, az1);
    return t;
}

template <typename T, int BY, int PM, bool DL, bool GAIN>
int e_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                 const GainView<T> &G, int kc, const TileBoxes &tb, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY, GAIN && sizeof(T) == 4>;
    const int blocks = tb.start[tb.n];
    if (blocks <= 0) return 0;
    if (!set_smem<k_e_tma<T, BY, PM, DL, GAIN>>(L::SMEM)) return 0;
    k_e_tma<T, BY, PM, DL, GAIN><<<blocks, dim3(32, BY), L::SMEM, s>>>(M, f, p, D, G, kc, tb, err);
    return 1;
}

template <typename T, int BY, int PM>
int h_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc, const TileBoxes &tb,
                 int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    const int blocks = tb.start[tb.n];
    if (blocks <= 0) return 0;
    if (!set_smem<k_h_tma<T, BY, PM>>(L::SMEM)) return 0;
    k_h_tma<T, BY, PM><<<blocks, dim3(32, BY), L::SMEM, s>>>(M, f, p, kc, tb, err);
    return 1;
}

// the kernels the launchers below use (CPML-free, per-tile, and for gain the
// two halves of the split)
template <typename T, int BY>
void attrs_by()
{
    constexpr int S = StageLayout<T, BY>::SMEM, SG = StageLayout<T, BY, sizeof(T) == 4>::SMEM;
    set_smem<k_h_tma<T, BY, 0>>(S);
    set_smem<k_h_tma<T, BY, 2>>(S);
    set_smem<k_e_tma<T, BY, 0, false, false>>(S);
    set_smem<k_e_tma<T, BY, 0, false, true>>(SG);
    set_smem<k_e_tma<T, BY, 0, true, false>>(S);
    set_smem<k_e_tma<T, BY, 0, true, true>>(SG);
    set_smem<k_e_tma<T, BY, 2, false, false>>(S);
    set_smem<k_e_tma<T, BY, 2, true, false>>(S);
    set_smem<k_e_tma<T, BY, 1, false, true>>(SG);
    set_smem<k_e_tma<T, BY, 1, true, true>>(SG);
}

template <typename T, int BY>
int e_tma_by(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
             const GainView<T> &G, int kc, int *err, cudaStream_t s)
{
    const bool dl = D.on && D.ncell > 0, gn = G.on && G.ncell > 0;
    const SweepTiles t = sweep_tiles(p.np, p.on, f.d, BY, kc, true);
    if (gn && sizeof(T) == 4 && p.on) {  // every tile on the CPML body, one launch
        const TileBoxes all = whole_grid(f.d, BY, kc);
        return dl ? e_tma_launch<T, BY, 1, true, true>(M, f, p, D, G, kc, all, err, s)
                  : e_tma_launch<T, BY, 1, false, true>(M, f, p, D, G, kc, all, err, s);
    }
    if (gn) {  // CPML tiles (if any) and interior tiles as two launches
        return (dl ? e_tma_launch<T, BY, 1, true, true>(M, f, p, D, G, kc, t.pml, err, s)
                   : e_tma_launch<T, BY, 1, false, true>(M, f, p, D, G, kc, t.pml, err, s)) +
               (dl ? e_tma_launch<T, BY, 0, true, true>(M, f, p, D, G, kc, t.interior, err, s)
                   : e_tma_launch<T, BY, 0, false, true>(M, f, p, D, G, kc, t.interior, err, s));
    }
    const TileBoxes all = whole_grid(f.d, BY, kc);
    if (p.on)
        return dl ? e_tma_launch<T, BY, 2, true, false>(M, f, p, D, G, kc, all, err, s)
                  : e_tma_launch<T, BY, 2, false, false>(M, f, p, D, G, kc, all, err, s);
    return dl ? e_tma_launch<T, BY, 0, true, false>(M, f, p, D, G, kc, all, err, s)
              : e_tma_launch<T, BY, 0, false, false>(M, f, p, D, G, kc, all, err, s);
}

template <typename T, int BY>
int h_tma_by(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc, int *err, cudaStream_t s)
{
    const TileBoxes all = whole_grid(f.d, BY, kc);
    return p.on ? h_tma_launch<T, BY, 2>(M, f, p, kc, all, err, s) : h_tma_launch<T, BY, 0>(M, f, p, kc, all, err, s);
}

}  // namespace

template <typename T>
int launch_h_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, FusedShape sh, int *err,
                 cudaStream_t s)
{
    const int kc = sh.kch > 0 ? sh.kch : sh.kc;
    return sh.by == 4 ? h_tma_by<T, 4>(M, f, p, kc, err, s) : h_tma_by<T, 8>(M, f, p, kc, err, s);
}

template <typename T>
int launch_e_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                 const GainView<T> &G, FusedShape sh, int *err, cudaStream_t s, const SideLane *lane)
{
    const bool dl = D.on && D.ncell > 0;
    const bool beside = dl && lane && lane->s;
    cudaStream_t ds = s;
    if (beside) {
        cudaEventRecord(lane->fork, s);
        cudaStreamWaitEvent(lane->s, lane->fork, 0);
        ds = lane->s;
    }
    if (dl) {  // launched first, so its blocks start beside the sweep's first wave
        if (p.on) k_dl_cells<T, true><<<cdiv(D.ncell, 128), 128, 0, ds>>>(f, p, D);
        else k_dl_cells<T, false><<<cdiv(D.ncell, 128), 128, 0, ds>>>(f, p, D);
    }
    // an FP32 sweep with gain takes its own plane count (4 by default: with
    // its three-stage ring of large stages it ran 1.9 % faster on 4-plane
    // tiles than on 8 on the 384^3 laser deck, while the E sweep without gain
    // ran 9 % slower on 4 than on 8 on the 256^3 dispersive deck)
    const int kc = G.on && G.ncell > 0 && sizeof(T) == 4 && sh.kcg > 0 ? sh.kcg : sh.kc;
    const int n = sh.by == 4 ? e_tma_by<T, 4>(M, f, p, D, G, kc, err, s) : e_tma_by<T, 8>(M, f, p, D, G, kc, err, s);
    if (beside) {
        cudaEventRecord(lane->join, lane->s);
        cudaStreamWaitEvent(s, lane->join, 0);
    }
    return n + (dl ? 1 : 0);
}

template <typename T>
void tma_attributes()
{
    attrs_by<T, 4>();
    attrs_by<T, 8>();
}

template void tma_attributes<float>();
template void tma_attributes<double>();
template int launch_h_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &, FusedShape, int *,
                                  cudaStream_t);
template int launch_h_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &, FusedShape,
                                   int *, cudaStream_t);
template int launch_e_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &,
                                  const DlView<float> &, const GainView<float> &, FusedShape, int *, cudaStream_t,
                                  const SideLane *);
template int launch_e_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &,
                                   const DlView<double> &, const GainView<double> &, FusedShape, int *, cudaStream_t,
                                   const SideLane *);

}  // namespace cps
