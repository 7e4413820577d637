// kernels_batch.cu -- sweeps and Drude-Lorentz cells of many grids in one
// launch (sm_100a).  A block takes tiles from a flat table, each naming its
// grid, and runs the same per-tile bodies as the one-grid kernels
// (tma_bodies.cuh), so a cell's arithmetic does not depend on which launch,
// tile shape or co-resident grids processed it.  With fewer blocks than
// tiles a block walks the table with a stride of the grid size (persistent
// launch); its stage ring and mbarriers carry over from tile to tile.
//
// The tensor maps live in the descriptor table in device memory, written by
// the host before the launch; the issuing thread orders its TMA reads after
// those writes with fence.proxy.tensormap::generic.acquire whenever it moves
// to another grid's maps.  No multicast is used.
#include <cuda.h>

#include "batch.h"
#include "tma_bodies.cuh"

namespace cps {

namespace {

__device__ __forceinline__ void tensormap_acquire(const CUtensorMap *map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
}

// the seven maps one sweep side reads: E sweep H halos + E tiles + IDs, H
// sweep E halos + H tiles + IDs
__device__ __forceinline__ void acquire_maps(const TmaMaps &M, bool eside)
{
    for (int c = 0; c < 3; ++c) {
        tensormap_acquire(&M.halo[eside ? 3 + c : c]);
        tensormap_acquire(&M.own[eside ? c : 3 + c]);
    }
    tensormap_acquire(&M.id);
}

// The views of a tile's grid are copied into shared memory when a block
// moves to another grid: the sweep bodies then read pointers and CPML
// coefficients with shared loads that no global field store can alias,
// instead of reloading them from the descriptor table after every store.
template <typename V>
__device__ __forceinline__ void stage_view(V &dst, const V &src)
{
    static_assert(sizeof(V) % 8 == 0, "views are whole 8-byte words");
    const int n = (int)(sizeof(V) / 8), nt = (int)(blockDim.x * blockDim.y);
    const uint64_t *s = reinterpret_cast<const uint64_t *>(&src);
    uint64_t *d = reinterpret_cast<uint64_t *>(&dst);
    for (int w = (int)(threadIdx.y * blockDim.x + threadIdx.x); w < n; w += nt) d[w] = s[w];
}

template <typename T, int BY, bool PML>
__global__ void __launch_bounds__(32 * BY) k_h_batch(const BatchGrid<T> *__restrict__ grids,
                                                      const int4 *__restrict__ tiles, int ntiles, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    init_stages(full);
    const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
    __shared__ FieldView<T> sf;
    __shared__ PmlView<T> sp;
    uint32_t ctr = 0;
    int last = -1;
    for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
        const int4 e = tiles[q];
        const BatchGrid<T> &B = grids[e.x];
        if (e.x != last) {  // uniform over the block: every thread reads the same entry
            __syncthreads();  // the previous grid's views are no longer read
            stage_view(sf, B.f);
            if (PML) stage_view(sp, B.p);
            if (lead) acquire_maps(B.M, false);
            __syncthreads();
            last = e.x;
        }
        if (!h_tma_body<T, BY, PML>(B.M, sf, sp, B.kc, TileXYZ{e.y, e.z, e.w}, ctr, err, sm, full)) return;
    }
}

template <typename T, int BY, bool PML, bool GAIN, bool DL>
__global__ void __launch_bounds__(32 * BY) k_e_batch(const BatchGrid<T> *__restrict__ grids,
                                                      const int4 *__restrict__ tiles, int ntiles, int *err)
{
    extern __shared__ __align__(128) unsigned char sm_raw[];
    __shared__ __align__(8) uint64_t full[kStages];
    unsigned char *sm = align_smem(sm_raw);
    init_stages(full);
    const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
    __shared__ FieldView<T> sf;
    __shared__ PmlView<T> sp;
    __shared__ DlView<T> sD;
    __shared__ GainView<T> sG;
    uint32_t ctr = 0;
    int last = -1;
    for (int q = blockIdx.x; q < ntiles; q += gridDim.x) {
        const int4 e = tiles[q];
        const BatchGrid<T> &B = grids[e.x];
        if (e.x != last) {  // uniform over the block
            __syncthreads();
            stage_view(sf, B.f);
            if (PML) stage_view(sp, B.p);
            if (DL) stage_view(sD, B.D);
            if (GAIN) stage_view(sG, B.G);
            if (lead) {
                acquire_maps(B.M, true);
                if (GAIN && sizeof(T) == 4) tensormap_acquire(&B.M.gain);
            }
            __syncthreads();
            last = e.x;
        }
        if (!e_tma_body<T, BY, PML, DL, GAIN>(B.M, sf, sp, sD, sG, B.kc, TileXYZ{e.y, e.z, e.w}, ctr, err, sm,
                                               full))
            return;
    }
}

template <typename T>
__global__ void __launch_bounds__(128) k_dl_batch(const BatchGrid<T> *__restrict__ grids,
                                                  const int4 *__restrict__ blocks)
{
    const int4 e = blocks[blockIdx.x];
    const int64_t c = (int64_t)e.y + threadIdx.x;
    if (c >= e.z) return;
    const BatchGrid<T> &B = grids[e.x];
    if (B.p.on) dl_cell_any<T, true>(B.f, B.f, B.p, B.D, c);
    else dl_cell_any<T, false>(B.f, B.f, B.p, B.D, c);
}

template <typename T>
__global__ void k_advance(BatchGrid<T> *grids, int ngrids, int nsteps)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ngrids) grids[g].n0 += nsteps;
}

inline unsigned cdiv(int64_t a, int64_t b) { return (unsigned)((a + b - 1) / b); }

// set once per kernel and device; false when the attribute could not be set
template <auto K>
bool smem_attr(int bytes)
{
    return kernel_smem<K>(bytes);
}

template <typename T, int BY, bool PML>
void h_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int *err, cudaStream_t s)
{
    using L = StageLayout<T, BY>;
    if (!smem_attr<k_h_batch<T, BY, PML>>(L::SMEM)) return;
    k_h_batch<T, BY, PML><<<nblocks, dim3(32, BY), L::SMEM, s>>>(grids, tiles, ntiles, err);
}

template <typename K>
int occupancy(K kernel, int threads, int smem)
{
    int n = 0;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, threads, smem) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    return n > 0 ? n : 1;
}

template <typename T, int BY, bool PML, bool GAIN, bool DL>
void e_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int *err, cudaStream_t s)
{
    using L = ELayout<T, BY, GAIN>;
    if (!smem_attr<k_e_batch<T, BY, PML, GAIN, DL>>(L::SMEM)) return;
    k_e_batch<T, BY, PML, GAIN, DL><<<nblocks, dim3(32, BY), L::SMEM, s>>>(grids, tiles, ntiles, err);
}

template <typename T, int BY>
void e_batch_by(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int cls, int *err,
                cudaStream_t s)
{
    switch (cls & 7) {
    case 0: e_batch<T, BY, false, false, false>(grids, tiles, ntiles, nblocks, err, s); break;
    case 1: e_batch<T, BY, true, false, false>(grids, tiles, ntiles, nblocks, err, s); break;
    case 2: e_batch<T, BY, false, false, true>(grids, tiles, ntiles, nblocks, err, s); break;
    case 3: e_batch<T, BY, true, false, true>(grids, tiles, ntiles, nblocks, err, s); break;
    case 4: e_batch<T, BY, false, true, false>(grids, tiles, ntiles, nblocks, err, s); break;
    case 5: e_batch<T, BY, true, true, false>(grids, tiles, ntiles, nblocks, err, s); break;
    case 6: e_batch<T, BY, false, true, true>(grids, tiles, ntiles, nblocks, err, s); break;
    default: e_batch<T, BY, true, true, true>(grids, tiles, ntiles, nblocks, err, s); break;
    }
}

template <typename T, int BY>
void e_batch_attrs()
{
    constexpr int S = StageLayout<T, BY>::SMEM, SG = ELayout<T, BY, true>::SMEM;
    smem_attr<k_e_batch<T, BY, false, false, false>>(S);
    smem_attr<k_e_batch<T, BY, true, false, false>>(S);
    smem_attr<k_e_batch<T, BY, false, false, true>>(S);
    smem_attr<k_e_batch<T, BY, true, false, true>>(S);
    smem_attr<k_e_batch<T, BY, false, true, false>>(SG);
    smem_attr<k_e_batch<T, BY, true, true, false>>(SG);
    smem_attr<k_e_batch<T, BY, false, true, true>>(SG);
    smem_attr<k_e_batch<T, BY, true, true, true>>(SG);
}

template <typename T, int BY>
int e_batch_occupancy(int cls)
{
    constexpr int S = StageLayout<T, BY>::SMEM, SG = ELayout<T, BY, true>::SMEM;
    switch (cls & 7) {
    case 0: return occupancy(k_e_batch<T, BY, false, false, false>, 32 * BY, S);
    case 1: return occupancy(k_e_batch<T, BY, true, false, false>, 32 * BY, S);
    case 2: return occupancy(k_e_batch<T, BY, false, false, true>, 32 * BY, S);
    case 3: return occupancy(k_e_batch<T, BY, true, false, true>, 32 * BY, S);
    case 4: return occupancy(k_e_batch<T, BY, false, true, false>, 32 * BY, SG);
    case 5: return occupancy(k_e_batch<T, BY, true, true, false>, 32 * BY, SG);
    case 6: return occupancy(k_e_batch<T, BY, false, true, true>, 32 * BY, SG);
    default: return occupancy(k_e_batch<T, BY, true, true, true>, 32 * BY, SG);
    }
}

}  // namespace

template <typename T>
void launch_h_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int by, bool pml,
                    int *err, cudaStream_t s)
{
    if (ntiles <= 0) return;
    if (nblocks <= 0 || nblocks > ntiles) nblocks = ntiles;
    if (by == 4) {
        if (pml) h_batch<T, 4, true>(grids, tiles, ntiles, nblocks, err, s);
        else h_batch<T, 4, false>(grids, tiles, ntiles, nblocks, err, s);
    } else {
        if (pml) h_batch<T, 8, true>(grids, tiles, ntiles, nblocks, err, s);
        else h_batch<T, 8, false>(grids, tiles, ntiles, nblocks, err, s);
    }
}

template <typename T>
void launch_e_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int by, int cls, int *err,
                    cudaStream_t s)
{
    if (ntiles <= 0) return;
    if (nblocks <= 0 || nblocks > ntiles) nblocks = ntiles;
    if (by == 4) e_batch_by<T, 4>(grids, tiles, ntiles, nblocks, cls, err, s);
    else e_batch_by<T, 8>(grids, tiles, ntiles, nblocks, cls, err, s);
}

template <typename T>
void launch_dl_batch(const BatchGrid<T> *grids, const int4 *blocks, int nblocks, cudaStream_t s)
{
    if (nblocks <= 0) return;
    k_dl_batch<T><<<nblocks, 128, 0, s>>>(grids, blocks);
}

template <typename T>
void launch_advance_batch(BatchGrid<T> *grids, int ngrids, int nsteps, cudaStream_t s)
{
    if (ngrids <= 0) return;
    k_advance<T><<<cdiv(ngrids, 128), 128, 0, s>>>(grids, ngrids, nsteps);
}

template <typename T>
int batch_blocks_per_sm(int by, bool eside, int cls)
{
    if (by == 4) {
        using L = StageLayout<T, 4>;
        if (!eside) return (cls & 1) ? occupancy(k_h_batch<T, 4, true>, 128, L::SMEM)
                                     : occupancy(k_h_batch<T, 4, false>, 128, L::SMEM);
        return e_batch_occupancy<T, 4>(cls);
    }
    using L = StageLayout<T, 8>;
    if (!eside) return (cls & 1) ? occupancy(k_h_batch<T, 8, true>, 256, L::SMEM)
                                 : occupancy(k_h_batch<T, 8, false>, 256, L::SMEM);
    return e_batch_occupancy<T, 8>(cls);
}

template <typename T>
void batch_kernel_attributes()
{
    smem_attr<k_h_batch<T, 4, false>>(StageLayout<T, 4>::SMEM);
    smem_attr<k_h_batch<T, 4, true>>(StageLayout<T, 4>::SMEM);
    smem_attr<k_h_batch<T, 8, false>>(StageLayout<T, 8>::SMEM);
    smem_attr<k_h_batch<T, 8, true>>(StageLayout<T, 8>::SMEM);
    e_batch_attrs<T, 4>();
    e_batch_attrs<T, 8>();
    dft_batch_attributes<T>();
}

#define CPS_BATCH_INSTANTIATE(T)                                                                             \
    template void launch_h_batch<T>(const BatchGrid<T> *, const int4 *, int, int, int, bool, int *,          \
                                    cudaStream_t);                                                           \
    template void launch_e_batch<T>(const BatchGrid<T> *, const int4 *, int, int, int, int, int *,          \
                                    cudaStream_t);                                                           \
    template void launch_dl_batch<T>(const BatchGrid<T> *, const int4 *, int, cudaStream_t);                 \
    template void launch_advance_batch<T>(BatchGrid<T> *, int, int, cudaStream_t);                           \
    template int batch_blocks_per_sm<T>(int, bool, int);                                              \
    template void batch_kernel_attributes<T>();
CPS_BATCH_INSTANTIATE(float)
CPS_BATCH_INSTANTIATE(double)

}  // namespace cps
