// kernels_tma.cu -- one-grid launches of the TMA-fed fused H and E sweeps
// (sm_100a): one block per 32 x BY x kc tile, bodies in tma_bodies.cuh.
#include <cuda.h>

#include "tma_bodies.cuh"

namespace cps {

namespace {

template <typename T, int BY, bool PML, bool DL, bool GAIN>
__global__ void __launch_bounds__(32 * BY, GAIN ? 512 / (32 * BY) : 1024 / (32 * BY)) k_e_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p,
                                                    DlView<T> D, GainView<T> G, int kc, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    const TileXYZ t{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z};
    const int k0 = max(1, t.bz * kc), k1 = min(t.bz * kc + kc, f.d.nz);
    if (k0 >= k1) return;
    init_stages(full);
    uint32_t ctr = 0;
    if (PML && tile_in_pml(p.np, f.d, t.bx * 32, t.by * BY, BY, k0, k1, true))
        e_tma_body<T, BY, true, DL, GAIN>(M, f, p, D, G, kc, t, ctr, err, sm, full);
    else
        e_tma_body<T, BY, false, DL, GAIN>(M, f, p, D, G, kc, t, ctr, err, sm, full);
}

template <typename T, int BY, bool PML>
__global__ void __launch_bounds__(32 * BY) k_h_tma(const __grid_constant__ TmaMaps M, FieldView<T> f, PmlView<T> p,
                                                    int kc, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    const TileXYZ t{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z};
    const int k0 = t.bz * kc, k1 = min(k0 + kc, f.d.nz);
    if (k0 >= k1) return;
    init_stages(full);
    uint32_t ctr = 0;
    if (PML && tile_in_pml(p.np, f.d, t.bx * 32, t.by * BY, BY, k0, k1, false))
        h_tma_body<T, BY, true>(M, f, p, kc, t, ctr, err, sm, full);
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

template <typename T, int BY, bool PML, bool DL, bool GAIN>
void e_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                  const GainView<T> &G, int kc, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    if (!set_smem<k_e_tma<T, BY, PML, DL, GAIN>>(L::SMEM)) return;
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    k_e_tma<T, BY, PML, DL, GAIN><<<grid, dim3(32, BY), L::SMEM, s>>>(M, f, p, D, G, kc, err);
}

template <typename T, int BY, bool PML>
void h_tma_launch(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, int kc, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    if (!set_smem<k_h_tma<T, BY, PML>>(L::SMEM)) return;
    dim3 grid(cdiv(f.d.nx, 32), cdiv(f.d.ny, BY), cdiv(f.d.nz, kc));
    k_h_tma<T, BY, PML><<<grid, dim3(32, BY), L::SMEM, s>>>(M, f, p, kc, err);
}

template <typename T, int BY>
void attrs_by()
{
    constexpr int S = StageLayout<T, BY>::SMEM;
    set_smem<k_h_tma<T, BY, false>>(S);
    set_smem<k_h_tma<T, BY, true>>(S);
    set_smem<k_e_tma<T, BY, false, false, false>>(S);
    set_smem<k_e_tma<T, BY, false, false, true>>(S);
    set_smem<k_e_tma<T, BY, false, true, false>>(S);
    set_smem<k_e_tma<T, BY, false, true, true>>(S);
    set_smem<k_e_tma<T, BY, true, false, false>>(S);
    set_smem<k_e_tma<T, BY, true, false, true>>(S);
    set_smem<k_e_tma<T, BY, true, true, false>>(S);
    set_smem<k_e_tma<T, BY, true, true, true>>(S);
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

template <typename T>
void tma_attributes()
{
    attrs_by<T, 4>();
    attrs_by<T, 8>();
}

template void tma_attributes<float>();
template void tma_attributes<double>();
template void launch_h_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &, FusedShape, int *,
                                  cudaStream_t);
template void launch_h_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &, FusedShape,
                                   int *, cudaStream_t);
template void launch_e_tma<float>(const TmaMaps &, const FieldView<float> &, const PmlView<float> &,
                                  const DlView<float> &, const GainView<float> &, FusedShape, int *, cudaStream_t);
template void launch_e_tma<double>(const TmaMaps &, const FieldView<double> &, const PmlView<double> &,
                                   const DlView<double> &, const GainView<double> &, FusedShape, int *, cudaStream_t);

}  // namespace cps
