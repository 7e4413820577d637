// batch.h -- device descriptors and launchers of the batched engine: many
// independent grids of uneven size advanced together, one launch per sweep
// class over a flat table of work items that name their grid.
//
// Every per-step value a kernel needs (the step number, a ring slot) comes
// from the descriptors in device memory or from the step's offset inside a
// chunk of steps, so one chunk is captured once into a CUDA graph and
// replayed while the set of grids stays the same.
#pragma once

#include "cps_internal.h"

namespace cps {

// One grid of a batch.  The tensor maps come first so that they sit on the
// 64-byte boundary TMA requires (the array is allocated 256-byte aligned and
// the struct size is a multiple of 64).
template <typename T>
struct alignas(64) BatchGrid {
    TmaMaps M;
    FieldView<T> f;
    PmlView<T> p;
    DlView<T> D;
    GainView<T> G;
    const InjTarget *tg[2];   // TF/SF targets: [0] E side, [1] H side
    const InjContrib *ct[2];
    const T *inc[2];          // incident tables: [0] Hinc (E side), [1] Einc (H side)
    int ntg[2];
    int Nt;
    int nsrc;
    const int64_t *src_idx;
    const int32_t *src_comp, *src_off, *src_len;
    const double *src_wave;
    int64_t n0;               // step number at the start of the current chunk
    double dt;
    int kc;                   // planes per tile along z
    int pad;
};

// One port of a batch: ring [slots][6][npts] of T; FP64 phasor scratch
// [2][kMaxRing][nfreq] of (cos, sin) (E time, H time); FP64 accumulators
// [ncomp][nfreq][2][npts].
template <typename T>
struct BatchPort {
    const int64_t *idx;
    T *ring;
    double2 *tab;
    const double *omega;
    const int32_t *comps;
    double *acc;
    int grid, npts, slots, nfreq, ncomp, pad;
};

constexpr int kMaxRing = 64;  // samples per port ring = longest chunk

// DFT contraction tile of a port: 64 frequencies x 64 points per block, or
// 32 frequencies x 128 points when the port transforms at most 32 (no block
// then spends half its threads on frequencies the port does not have)
__host__ __device__ constexpr int dft_freq_tile(int nfreq) { return nfreq <= 32 ? 32 : 64; }
__host__ __device__ constexpr int dft_point_tile(int nfreq) { return nfreq <= 32 ? 128 : 64; }
constexpr int kInjThreads = 128;                // threads of a batched injection block
constexpr int kInjPerBlock = 2 * kInjThreads;   // TF/SF targets per injection block entry

// Work tables (device arrays):
//   tiles      int4 {grid, bx, by, bz}      sweeps
//   dl blocks  int4 {grid, c0, c1, -}       Drude-Lorentz cells [c0, c1)
//   inj blocks int4 {grid, t0, t1, -}       TF/SF targets [t0, t1) of one side
//   sources    int2 {grid, s}
//   gather     int2 {port, p0}              points [p0, p0+256)
//   phasors    int2 {port, q0}              table entries [q0, q0+256)
//   dft        int4 {port, p-block, component index, f-block}
template <typename T>
void launch_h_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int by, bool pml,
                    int *err, cudaStream_t s);
// cls bits: 1 CPML tiles, 2 Drude-Lorentz grids, 4 gain grids
template <typename T>
void launch_e_batch(const BatchGrid<T> *grids, const int4 *tiles, int ntiles, int nblocks, int by, int cls, int *err,
                    cudaStream_t s);
template <typename T>
void launch_dl_batch(const BatchGrid<T> *grids, const int4 *blocks, int nblocks, cudaStream_t s);
template <typename T>
void launch_advance_batch(BatchGrid<T> *grids, int ngrids, int nsteps, cudaStream_t s);
template <typename T>
void launch_inject_batch(const BatchGrid<T> *grids, const int4 *blocks, int nblocks, int side, int step_off,
                         cudaStream_t s);
template <typename T>
void launch_sources_batch(const BatchGrid<T> *grids, const int2 *ents, int n, int step_off, cudaStream_t s);
template <typename T>
void launch_gather_batch(const BatchGrid<T> *grids, const BatchPort<T> *ports, const int2 *blocks, int nblocks,
                         int step_off, int last_off, cudaStream_t s);
template <typename T>
void launch_dft_batch(const BatchGrid<T> *grids, const BatchPort<T> *ports, const int2 *ph_blocks, int nph,
                      const int4 *blocks, int nblocks, int nslots, cudaStream_t s);
// set the shared-memory attributes of every batched kernel (outside captures)
template <typename T>
void batch_kernel_attributes();
template <typename T>
bool dft_batch_attributes();
// sweep blocks of one SM that fit at once (for persistent launches)
template <typename T>
int batch_blocks_per_sm(int by, bool eside, int cls);

}  // namespace cps
