// cps_internal.h -- device layout and kernel interfaces of the engine.
//
// Device layout of a grid with nx*ny*nz cells (reference arrays span 0..N):
//   every field and the uint8 material-ID array is NX*NY*NZ values with
//   NX = nx+1 padded to `px` (a multiple of 32), NY = ny+1, NZ = nz+1,
//   linear index i + px*(j + NY*k): x fastest, so a warp reads 32
//   consecutive cells of one row and a thread marching in k walks a column.
//   CPML psi lives only on the six boundary slabs; Drude-Lorentz and gain
//   state only on compacted cell lists sorted by linear index (SoA, one array
//   per state word), found from a thread's cell by a per-warp-segment start
//   offset and a ballot rank.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/cps_capi.h"
#include "attr_once.h"

namespace cps {

constexpr int kXPad = 32;
constexpr int kMaxPoles = CPS_MAX_POLES;
constexpr int kFX1 = 0, kFX2 = 1, kFY1 = 2, kFY2 = 3, kFZ1 = 4, kFZ2 = 5;

// Physical constants, values as Constants.h:19-26
constexpr double kPi = 3.1415926535897932384626433832795;
constexpr double kC = 2.99792458E8;
constexpr double kHPlanck = 6.62607004081E-34;
constexpr double kMu0 = 1.2566370614E-6;
constexpr double kEps0 = 8.8541878176E-12;
constexpr double kQe = -1.602176565E-19;  // electron charge
constexpr double kMe = 9.10938215E-31;    // electron mass

// row width of an x-slab psi array ([k][j][s], s = 0..np): np+1 rounded up to
// 32 words so every row starts on a 128-byte line
__host__ __device__ inline int psi_xw(int np) { return (np + 32) / 32 * 32; }

struct Dims {
    int nx, ny, nz;   // cells
    int px;           // x pitch in elements
    int64_t pxy;      // px * (ny+1): plane stride
    __host__ __device__ int64_t idx(int i, int j, int k) const
    {
        return (int64_t)i + (int64_t)px * j + pxy * k;
    }
};

// --- Drude-Lorentz coefficients (host FP64, converted to T for the device)
template <typename T>
struct DlCoef {
    int nD, nL, stride;  // stride = words per component = nD + 2 nL + 1
    T C1, C2, C3, dt, inv2dt;
    T kappa[kMaxPoles], beta[kMaxPoles], C4[kMaxPoles];
    T alpha[kMaxPoles], xi[kMaxPoles], gammaL[kMaxPoles], C5[kMaxPoles], C6[kMaxPoles];
};

// --- gain coefficients.  FP64 grids hold P unscaled (scaleP = 1); FP32 grids
// hold P multiplied by CEP so that it stays in the normal float range, and
// populations as offsets from their initial values (N1-1, N2, N3).
struct GainCoef {
    double CPa1, CPa2, CPa3, CPb1, CPb2, CPb3, CEP;
    double t30, t32, t21, t10;
    double t30t32dt, t30t32_2, t30dt, t32dt, dt_2, homega_bdt;
    double t10t21dt, t10t21_2, t10dt, t21dt, t21_2, homega_adt;
    double t32t21dt, t32t21_2, t32_2;
    double pump_dt;
    double scaleP;  // P stored = scaleP * P
    // FP32 grids: P coefficients in float (CP3 carrying scaleP) and the
    // constant divisors of the population update as FP64 reciprocals
    float fa1, fa2, fa3, fb1, fb2, fb3;
    double r_t30, r_t32, r_t21, r_t10, r_t21_2, r_t32_2, r_hwb, r_hwa, inv_scale;
    // FP32 grids: the population update on offsets (cells.cuh gain_n_update<float>):
    // k1a = dt/2t21, k1b = dt/2t10, k3a = dt/2t32, k3b = dt/2t30,
    // ha = dt/(2 homega_adt)/scaleP, hb = dt/(2 homega_bdt)/scaleP, fpump = pump_rate dt
    float k1a, k1b, k3a, k3b, ha, hb, fpump;
};

// per-cell gain state words
constexpr int kG64Words = 25;  // Pa Pa1 Pa2 Pb Pb1 Pb2 (x3 each) E1 (x3) N0..N3
constexpr int kG32Words = 24;  // Pa Pa1 Pb Pb1 (x3, scaled) dN1 N2 N3 | Pa2 Pb2 E1 (x3, per-routine transients)
template <typename T>
__host__ __device__ constexpr int gain_words()
{
    return sizeof(T) == 4 ? kG32Words : kG64Words;
}
// FP32 gain state, segment-dense: the 15 persistent words (Pa Pa1 Pb Pb1 x3,
// n1 n2 n3) of every cell of the grid, [k][j][x-segment][word][32], so word w
// of the cell at device index g is at gain_dense_index(g) + 32 w (g >> 5 is
// the cell's (k, j, segment) row, g & 31 its lane).  A tile's gain words for a
// plane are one box of a tensor map, staged with its fields.  The plain
// path's transient words (Pa2 Pb2 E1) are kept apart, [group][9][32] by list
// index.  FP64 grids keep all 25 words in the list layout below.
constexpr int kGainPersist = 15;
constexpr int kGainTrans = 9;
__host__ __device__ inline int64_t gain_dense_index(int64_t g)
{
    return (g >> 5) * (int64_t)(kGainPersist * 32) + (g & 31);
}
// Gain state storage: the list cells in groups of 32, group q holding word w
// of its cells at [q][w][32].  Word w of list cell c is then
// state[gain_base_index(c, words) + w * kGainGroup]: one base per cell and a
// compile-time offset per word, and a warp's consecutive cells read whole
// 128-byte lines of every word.
constexpr int kGainGroup = 32;
__host__ __device__ inline int64_t gain_base_index(int64_t c, int words)
{
    return (c >> 5) * (int64_t)words * kGainGroup + (c & 31);
}
__host__ __device__ inline int64_t gain_state_elems(int64_t ncell, int words)
{
    return ((ncell + kGainGroup - 1) / kGainGroup) * (int64_t)words * kGainGroup;
}

// --- TF/SF / source injection in CSR form: each target (cell, component)
// owns a run of contributions applied in the reference's face order.
struct InjTarget {
    int64_t idx;
    int32_t comp;
    int32_t start;
    int32_t count;
    int32_t face;  // face of the first contribution (for face-mask calls)
};
struct InjContrib {
    double delay;    // retarded-time offset in steps (k.r/c - l0)/dt
    double profile;  // Gaussian transverse profile
    double coef;     // signed C * E0/H0 component
    int32_t face;
    int32_t pad;
};

template <typename T>
struct PmlView {
    int on;
    int np[6];
    const T *bE[6], *cE[6], *bH[6], *cH[6];
    T *qe[6][2], *qh[6][2];  // x slabs [k][j][s], y slabs [k][s][i], z slabs [s][j][i]
    T cpmlE, cpmlH;  // the reference's single psi coefficients (literal mode)
    T ce_disp;       // psi coefficient of ID-2 cells: the Drude-Lorentz C3 (bE[2] without Drude-Lorentz)
    int literal;     // 1: cpmlE/cpmlH for every cell; 0: each cell's own curl coefficient
};

template <typename T>
struct StretchView {
    // names as Structure.h:82-83
    const T *cExy, *cEyx, *cEzx, *cExz, *cEzy, *cEyz;
    const T *cHxy, *cHyx, *cHzx, *cHxz, *cHzy, *cHyz;
};

template <typename T>
struct FieldView {
    Dims d;
    T *Ex, *Ey, *Ez, *Hx, *Hy, *Hz;
    const uint8_t *id;
    const T *aE, *bE, *aH, *bH;  // 256 entries each
    StretchView<T> s;
};

// a field component's array by index (Ex Ey Ez Hx Hy Hz), without an indexed
// local array of pointers
template <typename T>
__host__ __device__ __forceinline__ T *field_comp(const FieldView<T> &f, int c)
{
    switch (c) {
    case 0: return f.Ex;
    case 1: return f.Ey;
    case 2: return f.Ez;
    case 3: return f.Hx;
    case 4: return f.Hy;
    default: return f.Hz;
    }
}

template <typename T>
struct DlView {
    int on;
    int64_t ncell;
    const int64_t *cell;     // sorted linear indices
    const int32_t *seg;      // start offset per (k, j, 32-wide x segment)
    T *state;                // [word][ncell]
    DlCoef<T> c;
};

template <typename T>
struct GainView {
    int on;
    int gain_id;
    int64_t ncell;
    const int64_t *cell;
    const int32_t *seg;
    const uint2 *segm;       // per (k, j, 32-wide x segment): list offset and the segment's gain-cell bit mask
    T *state;                // FP64: list layout [group][word][32]; FP32: segment-dense persistent words
    T *trans;                // FP32: the plain path's transient words, list layout [group][9][32]
    GainCoef c;
};

// --- three-level gain (ThreeLevel.cpp): FP64 state on both precisions (its
// polarisation is of order 1e-40 of E), SoA [word][site]: Pa[3] Pa1[3] Pa2[3]
// Pb[3] Pb1[3] Pb2[3] E1[3] N0 N1 N2 N1_1 N2_1
constexpr int kThreeWords = 26;
struct ThreeCoef {
    double CPa1, CPa2, CPa3, CPb1, CPb2, CPb3, CEP;
    double CN2N2, CN2E, CN1N1, CN1N2, CN1E, CN0N2, CN0N1, CN0Ea, CN0Eb, CN0Ebx;
};
struct ThreeView {
    int on;
    int64_t ncell;
    const int64_t *cell;  // sorted linear indices
    double *state;        // [word][ncell]
    ThreeCoef c;
};

// Dynamic shared memory of kernel `func` (and, carveout >= 0, its preferred
// shared-memory carveout), set once per device through `done` (one flag word
// per kernel).  Returns the attribute call's error; the runtime also keeps it
// as the thread's last error, so the launch check that follows reports it.
inline cudaError_t smem_attr_once(std::atomic<uint64_t> &done, const void *func, int bytes, int carveout = -1)
{
    return (cudaError_t)attr_once_per_device(
        done, [](int *dev) { return (int)cudaGetDevice(dev); },
        [&]() {
            cudaError_t e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
            if (e == cudaSuccess && carveout >= 0)
                e = cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, carveout);
            return (int)e;
        });
}

// the same for a kernel given as a template argument, one flag per kernel;
// true when the kernel may be launched
template <auto K>
bool kernel_smem(int bytes, int carveout = -1)
{
    static std::atomic<uint64_t> done{0};
    return smem_attr_once(done, reinterpret_cast<const void *>(K), bytes, carveout) == cudaSuccess;
}

// ------------------------------------------------------------ launchers
// Plain path: one kernel per reference routine (kernels_plain.cu, built
// without FMA contraction so FP64 results follow the reference roundings).
template <typename T> void launch_h_bulk(const FieldView<T> &f, cudaStream_t s);
template <typename T> void launch_e_bulk(const FieldView<T> &f, cudaStream_t s);
template <typename T> void launch_h_pml(const FieldView<T> &f, const PmlView<T> &p, cudaStream_t s);
template <typename T> void launch_e_pml(const FieldView<T> &f, const PmlView<T> &p, cudaStream_t s);
template <typename T> void launch_dl(const FieldView<T> &f, const DlView<T> &d, cudaStream_t s);
template <typename T> void launch_gain(const FieldView<T> &f, const GainView<T> &g, int which, cudaStream_t s);
// initial gain state: FP64 N0 = N1 = 1 in every group (the rest zeroed by the caller)
void launch_gain_init64(double *state, int64_t ncell, cudaStream_t s);
// FP32 population offsets n1 n2 n3 of every list cell, [ncell][3]
void launch_gain_pops32(const float *state, const int64_t *cell, int64_t ncell, float *out, cudaStream_t s);
// three-level gain sites: which 0 polarisation, 1 E field, 2 populations, 3 all
// three in order (kernels_three.cu, no FMA contraction); init: zero state, N0 = N_0
template <typename T> void launch_three(const FieldView<T> &f, const ThreeView &t, int which, cudaStream_t s);
void launch_three_init(const ThreeView &t, double N_0, cudaStream_t s);
template <typename T>
void launch_inject(const FieldView<T> &f, const InjTarget *tg, int ntarget, const InjContrib *ct,
                   const T *table, int Nt, double n, uint32_t face_mask, cudaStream_t s);
template <typename T>
void launch_sources(const FieldView<T> &f, int nsrc, const int64_t *idx, const int32_t *comp,
                    const double *waves, const int32_t *wave_off, const int32_t *wave_len, int n,
                    cudaStream_t s);

// Fused path (kernels_fused.cu): 2.5D z-marching sweeps.
struct FusedShape {
    int by;       // rows per block (block = 32 x by threads)
    int kc;       // planes per block along z (E sweep; H sweep too when kch is 0)
    int kch = 0;  // planes per block of the TMA H sweep (0: kc)
    int kcg = 0;  // planes per block of an FP32 TMA E sweep with gain (0: kc)
};
// A second stream of a grid with a fork and a join event: work that does not
// depend on a sweep (the Drude-Lorentz cell pass beside the E sweep) runs on
// it between the fork and the join, which a stream capture records as graph
// edges.  Created with the grid, outside any capture.
struct SideLane {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};
template <typename T>
void launch_h_fused(const FieldView<T> &f, const PmlView<T> &p, FusedShape sh, cudaStream_t s);
template <typename T>
void launch_e_fused(const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &d,
                    const GainView<T> &g, FusedShape sh, cudaStream_t s);

// TMA-fed fused sweeps (kernels_tma.cu); rows per block 4 or 8
}  // namespace cps
#include "tma.cuh"
namespace cps {
// (each sweep launches its CPML tiles and its interior tiles separately;
// the return value is the number of kernels launched)
template <typename T>
int launch_h_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, FusedShape sh, int *err,
                 cudaStream_t s);
// With a side lane, the Drude-Lorentz cell pass runs on it beside the E sweep
// (the sweep leaves the ID-2 cells, their E and their psi alone, and both
// read only H and the cells' own old E); the call returns after the join.
template <typename T>
int launch_e_tma(const TmaMaps &M, const FieldView<T> &f, const PmlView<T> &p, const DlView<T> &D,
                 const GainView<T> &G, FusedShape sh, int *err, cudaStream_t s, const SideLane *lane = nullptr);
// set the shared-memory attributes of every TMA sweep kernel (call outside captures)
template <typename T>
void tma_attributes();

// One-pass step (kernels_step.cu): H and E of a step in one sweep from the
// buffers of fo (and pin's H-side psi) into those of fn (pout's H-side psi).
// The H-side TF/SF corrections of the step come from dense per-face arrays
// (launch_h_corrections fills them first); corr == nullptr: none.
template <typename T>
struct HCorr {
    const T *corr;  // per face f: 3 components x nv x nu, from base[f]
    int box[6];     // bounding box of the H targets: i0 i1 j0 j1 k0 k1
    int base[6], nu[6], area[6];
};
template <typename T>
void launch_step_tma(const StepMaps &M, const FieldView<T> &fo, const FieldView<T> &fn, const PmlView<T> &pin,
                     const PmlView<T> &pout, const DlView<T> &D, const GainView<T> &G, const HCorr<T> &hc,
                     FusedShape sh, int *err, cudaStream_t s);
// the H-side TF/SF correction of every contribution at step n into its slot
// of the per-face arrays (TF_SF::UpdateHField's terms, TF_SF.cpp:1201-1300)
template <typename T>
void launch_h_corrections(const InjContrib *ct, const int32_t *slot, int ncontrib, const T *table, int Nt, double n,
                          T *corr, cudaStream_t s);
// the Drude-Lorentz cells after a one-pass sweep (old E from fo, H and new E in fn)
template <typename T>
void launch_dl_cells_step(const FieldView<T> &fn, const FieldView<T> &fo, const PmlView<T> &p, const DlView<T> &D,
                          cudaStream_t s);

// Ports (kernels_ports.cu)
constexpr int kMaxGather = 16;
struct GatherDesc {
    const int64_t *idx;
    void *slot;  // ring slot [6][npts] of T
    int npts;
    int pad;
};
struct GatherBatch {
    GatherDesc p[kMaxGather];
    int n;
    int max_npts;
};
template <typename T>
void launch_port_gather(const FieldView<T> &f, const GatherBatch &b, cudaStream_t s);
template <typename T>
void launch_port_dft(const T *ring, int npts, int nslots, int64_t n_first, double dt,
                     const double *omega, int nfreq, const int32_t *comps, int ncomp,
                     double *acc, double *scratch_phasor, cudaStream_t s);
void launch_port_flux(const double *acc, int npts, int nfreq, int ncomp, const int32_t *sign_pair,
                      double dA, double *out, cudaStream_t s);
template <typename T>
void launch_count_nonfinite(const FieldView<T> &f, unsigned long long *out, cudaStream_t s);
template <typename T>
void launch_to_device_layout(const double *src, T *dst, Dims d, cudaStream_t s);
template <typename T>
void launch_from_device_layout(const T *src, double *dst, Dims d, cudaStream_t s);

}  // namespace cps
