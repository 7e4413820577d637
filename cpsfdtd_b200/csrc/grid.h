// grid.h -- the host-side grid object behind the cps_grid handle, shared by
// the C ABI (capi.cpp) and the batched engine (batch.cpp).
#pragma once

#include <string.h>

#include <string>
#include <utility>
#include <vector>

#include "cps_internal.h"

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                         \
            return e_ == cudaErrorMemoryAllocation ? CPS_E_NOMEM : CPS_E_CUDA;                     \
        }                                                                                          \
    } while (0)

#define REQUIRE(cond, code, msg)                                                                   \
    do {                                                                                           \
        if (!(cond)) {                                                                             \
            set_error(msg);                                                                        \
            return code;                                                                           \
        }                                                                                          \
    } while (0)

namespace cps {

struct PortState {
    int npts = 0;
    std::vector<int32_t> ijk;
    int64_t *d_idx = nullptr;
    void *d_ring = nullptr;  // [slots][6][npts] of T
    int slots = 1;
    int fill = 0;            // samples in the ring not yet folded into the DFT
    int64_t ring_n0 = 0;     // step of ring slot 0
    int last_slot = -1;
    int nfreq = 0;
    uint32_t mask = 0;
    int ncomp = 0;
    int comps[6] = {0, 0, 0, 0, 0, 0};
    int32_t *d_comps = nullptr;
    double *d_omega = nullptr;
    double *d_acc = nullptr;  // [ncomp][nfreq][2][npts]
    double *d_flux = nullptr; // [nfreq]: cps_port_flux's result, allocated with the accumulators
};

// one recorded per-routine call (cps_op_*), kept until the recorder flushes
enum RecKind { kOpHBulk, kOpEBulk, kOpHPml, kOpEPml, kOpDl, kOpGainP, kOpGainE, kOpGainN, kOpTfsfH, kOpTfsfE,
               kOpSrc, kOpPort, kOpThreeP, kOpThreeE, kOpThreeN };
struct RecOp {
    int kind;
    int32_t n;      // step index (TF/SF, sources, ports)
    int32_t port;   // port id
    uint32_t mask;  // TF/SF face mask
};

struct Src {
    int comp;
    int64_t idx;
    std::vector<double> wave;
};

}  // namespace cps

struct cps_grid {
    using PortState = cps::PortState;
    using Src = cps::Src;
    using Dims = cps::Dims;
    using GainCoef = cps::GainCoef;
    using InjTarget = cps::InjTarget;
    using InjContrib = cps::InjContrib;
    using FusedShape = cps::FusedShape;
    using TmaMaps = cps::TmaMaps;
    using StepMaps = cps::StepMaps;
    template <typename T> using DlCoef = cps::DlCoef<T>;
    cps_grid_desc desc{};
    bool fp32 = false;
    size_t esz = 8;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cps::SideLane lane;  // the Drude-Lorentz cell pass beside the E sweep
    Dims d{};
    int64_t elems = 0;  // device elements per field array
    void *F[6] = {};
    uint8_t *d_id = nullptr;
    std::vector<uint8_t> ids_dev;  // host copy in device order
    bool ids_set = false;
    int nmedia = 0;
    double eps_r[256] = {}, mu_r[256] = {};  // relative permittivity and permeability per medium
    double aE[256] = {}, bE[256] = {}, aH[256] = {}, bH[256] = {};
    void *d_media = nullptr;  // aE bE aH bH, 256 each, of T
    std::vector<double> st[12];
    void *d_st = nullptr;
    // CPML
    bool pml_on = false;
    cps_pml_params pml{};
    std::vector<double> pbE[6], pcE[6], pbH[6], pcH[6];
    void *d_pcoef = nullptr;
    void *d_q[6][4] = {};
    double cpmlE = 0, cpmlH = 0;
    // Drude-Lorentz
    bool dl_on = false;
    DlCoef<double> dlc{};
    int64_t dl_n = 0;
    int64_t *d_dl_cell = nullptr;
    int32_t *d_dl_seg = nullptr;
    void *d_dl_state = nullptr;
    // gain
    bool gain_on = false;
    GainCoef gc{};
    int gain_id = 5;
    int64_t g_n = 0;
    int64_t *d_g_cell = nullptr;
    int32_t *d_g_seg = nullptr;
    uint2 *d_g_segm = nullptr;
    void *d_g_state = nullptr;  // FP32: segment-dense persistent words; FP64: all words, list layout
    void *d_g_trans = nullptr;  // FP32: transient words of the plain path, list layout
    // three-level gain (FP64 state on both precisions)
    int ids_max = 0;              // largest material ID set
    bool three_on = false;
    cps::ThreeCoef tc{};
    int three_id = 5;
    double three_N0 = 0.0;
    int64_t t_n = 0;
    int64_t *d_t_cell = nullptr;
    int32_t *d_t_seg = nullptr;
    double *d_t_state = nullptr;
    // TF/SF
    bool tfsf_on = false;
    cps_tfsf_params tp{};
    std::vector<double> einc, hinc;
    void *d_einc = nullptr, *d_hinc = nullptr;
    InjTarget *d_tg[2] = {nullptr, nullptr};   // 0: E targets, 1: H targets
    InjContrib *d_ct[2] = {nullptr, nullptr};
    int ntg[2] = {0, 0};
    // sources
    std::vector<Src> src;
    int64_t *d_src_idx = nullptr;
    int32_t *d_src_comp = nullptr, *d_src_off = nullptr, *d_src_len = nullptr;
    double *d_src_wave = nullptr;
    bool src_dirty = false;
    // ports
    std::vector<PortState> ports;
    double *d_phasor = nullptr;
    size_t phasor_cap = 0;
    // misc
    int64_t step = 1;
    int64_t launches = 0;
    // the E sweep's tiles march 8 planes, the H sweep's 16 and an FP32 E
    // sweep with gain 4 (measured fastest on the laser and dispersive decks);
    // cps_grid_set_tile sets all three
    FusedShape shape{4, 8, 16, 4};
    double *d_conv = nullptr;
    unsigned long long *d_counter = nullptr;
    // TMA tensor maps of the fused sweeps (built for tile rows tma_by)
    TmaMaps tma{};
    int tma_by = 0;
    int sweep_mode = 0;  // 0: TMA-fed sweeps, 1: register sweeps
    // one-pass step (CPS_PATH_ONEPASS): a second field buffer and H-side psi
    // set; a step reads F / d_q[f][2..3] and writes F2 / d_q2, then the two swap
    void *F2[6] = {};
    void *d_q2[6][2] = {};
    StepMaps om{}, om2{};          // tensor maps over F and over F2
    int om_by = 0;                 // tile rows the maps were built for
    // H-side TF/SF corrections of the one-pass step: per-face arrays over the
    // targets' bounding box and each contribution's slot in them
    void *d_hcorr = nullptr;
    int32_t *d_hslot = nullptr;
    int hc_n = 0;                 // contributions
    int hc_box[6] = {}, hc_base[6] = {}, hc_nu[6] = {}, hc_area[6] = {};
    bool hc_ok = true;            // every target lies on the box's surface (else no one-pass)
    bool onepass_ready = false;
    int *d_err = nullptr;  // set by a device wait that gave up
    // sweep timing samples: events (start, after H sweep, after E sweep)
    int timing_stride = 0;
    std::vector<cudaEvent_t> ev;
    int ev_used = 0;
    std::vector<std::pair<void *, size_t>> owned;  // every device allocation and its size
    // cps_step on the fused path as graph-replayed chunks of a one-grid batch
    bool chunked = true;
    cps_batch *solo = nullptr;
    // op recorder (cps_grid_set_record)
    bool record = false;
    std::vector<cps::RecOp> pending;
    int64_t fused_steps = 0, replayed_ops = 0;
};


namespace cps {

void set_error(const std::string &msg);
cps_status dalloc(cps_grid *g, void **p, size_t bytes);
void dfree(cps_grid *g, void *p);
cps_status upload_raw(cps_grid *g, void *dst, const void *src, size_t bytes);
cps_status ensure_sources(cps_grid *g);
cps_status ensure_tma(cps_grid *g);
// second buffer set, tensor maps and TF/SF target table of the one-pass step
cps_status ensure_onepass(cps_grid *g);
// make the buffers the last one-pass step wrote current
void swap_step_buffers(cps_grid *g);
cps_status flush_dft(cps_grid *g, PortState &P);
cps_status check_device_error(cps_grid *g);
// run the recorded calls of the grid (fused into one step when they form one)
cps_status flush_recorded(cps_grid *g);

inline int kStretchLen(const cps_grid *g, int w)
{
    const int n[12] = {g->d.nz, g->d.nz, g->d.ny, g->d.ny, g->d.nx, g->d.nx,
                       g->d.nz, g->d.nz, g->d.ny, g->d.ny, g->d.nx, g->d.nx};
    return n[w];
}

template <typename T>
inline StretchView<T> stretch_view(const cps_grid *g)
{
    StretchView<T> v;
    const T *base = (const T *)g->d_st;
    const T *a[12];
    size_t off = 0;
    for (int w = 0; w < 12; ++w) {
        a[w] = base + off;
        off += (size_t)(kStretchLen(g, w) + 7) / 8 * 8;
    }
    v.cExy = a[0]; v.cEyx = a[1]; v.cEzx = a[2]; v.cExz = a[3]; v.cEzy = a[4]; v.cEyz = a[5];
    v.cHxy = a[6]; v.cHyx = a[7]; v.cHzx = a[8]; v.cHxz = a[9]; v.cHzy = a[10]; v.cHyz = a[11];
    return v;
}

template <typename T>
inline FieldView<T> field_view(const cps_grid *g)
{
    FieldView<T> f;
    f.d = g->d;
    f.Ex = (T *)g->F[0]; f.Ey = (T *)g->F[1]; f.Ez = (T *)g->F[2];
    f.Hx = (T *)g->F[3]; f.Hy = (T *)g->F[4]; f.Hz = (T *)g->F[5];
    f.id = g->d_id;
    const T *m = (const T *)g->d_media;
    f.aE = m; f.bE = m + 256; f.aH = m + 512; f.bH = m + 768;
    f.s = stretch_view<T>(g);
    return f;
}

// the second field buffer set of the one-pass step (written by the next step)
template <typename T>
inline FieldView<T> field_view_alt(const cps_grid *g)
{
    FieldView<T> f = field_view<T>(g);
    f.Ex = (T *)g->F2[0]; f.Ey = (T *)g->F2[1]; f.Ez = (T *)g->F2[2];
    f.Hx = (T *)g->F2[3]; f.Hy = (T *)g->F2[4]; f.Hz = (T *)g->F2[5];
    return f;
}

template <typename T>
inline PmlView<T> pml_view(const cps_grid *g)
{
    PmlView<T> p;
    memset(&p, 0, sizeof(p));
    p.on = g->pml_on;
    if (!g->pml_on) return p;
    const T *c = (const T *)g->d_pcoef;
    size_t off = 0;
    for (int f = 0; f < 6; ++f) {
        p.np[f] = g->pml.npml[f];
        const size_t n = (size_t)p.np[f] + 1;
        p.bE[f] = c + off; off += n;
        p.cE[f] = c + off; off += n;
        p.bH[f] = c + off; off += n;
        p.cH[f] = c + off; off += n;
        p.qe[f][0] = (T *)g->d_q[f][0]; p.qe[f][1] = (T *)g->d_q[f][1];
        p.qh[f][0] = (T *)g->d_q[f][2]; p.qh[f][1] = (T *)g->d_q[f][3];
    }
    p.cpmlE = (T)g->cpmlE;
    p.cpmlH = (T)g->cpmlH;
    p.ce_disp = g->dl_on ? (T)g->dlc.C3 : (T)g->bE[CPS_ID_DISPERSIVE];
    p.literal = g->pml.literal ? 1 : 0;
    return p;
}

// pml_view with the H-side psi of the second buffer set
template <typename T>
inline PmlView<T> pml_view_alt(const cps_grid *g)
{
    PmlView<T> p = pml_view<T>(g);
    if (p.on)
        for (int f = 0; f < 6; ++f) {
            p.qh[f][0] = (T *)g->d_q2[f][0];
            p.qh[f][1] = (T *)g->d_q2[f][1];
        }
    return p;
}

// words of one psi array of CPML face f: x slabs [k][j][s], y slabs [k][s][i], z slabs [s][j][i]
inline size_t psi_words(const cps_grid *g, int f)
{
    const Dims &d = g->d;
    const int np = g->pml.npml[f];
    if (f < 2) return (size_t)(d.nz + 1) * (d.ny + 1) * psi_xw(np);
    if (f < 4) return (size_t)(d.nz + 1) * (np + 1) * d.px;
    return (size_t)(np + 1) * (d.ny + 1) * d.px;
}

template <typename T>
inline DlView<T> dl_view(const cps_grid *g)
{
    DlView<T> v;
    memset(&v, 0, sizeof(v));
    v.on = g->dl_on;
    if (!g->dl_on) return v;
    v.ncell = g->dl_n; v.cell = g->d_dl_cell; v.seg = g->d_dl_seg; v.state = (T *)g->d_dl_state;
    const DlCoef<double> &c = g->dlc;
    v.c.nD = c.nD; v.c.nL = c.nL; v.c.stride = c.stride;
    v.c.C1 = (T)c.C1; v.c.C2 = (T)c.C2; v.c.C3 = (T)c.C3; v.c.dt = (T)c.dt; v.c.inv2dt = (T)c.inv2dt;
    for (int p = 0; p < kMaxPoles; ++p) {
        v.c.kappa[p] = (T)c.kappa[p]; v.c.beta[p] = (T)c.beta[p]; v.c.C4[p] = (T)c.C4[p];
        v.c.alpha[p] = (T)c.alpha[p]; v.c.xi[p] = (T)c.xi[p]; v.c.gammaL[p] = (T)c.gammaL[p];
        v.c.C5[p] = (T)c.C5[p]; v.c.C6[p] = (T)c.C6[p];
    }
    return v;
}

template <typename T>
inline GainView<T> gain_view(const cps_grid *g)
{
    GainView<T> v;
    memset(&v, 0, sizeof(v));
    v.on = g->gain_on;
    if (!g->gain_on) return v;
    v.gain_id = g->gain_id; v.ncell = g->g_n; v.cell = g->d_g_cell; v.seg = g->d_g_seg; v.segm = g->d_g_segm;
    v.state = (T *)g->d_g_state; v.trans = (T *)g->d_g_trans; v.c = g->gc;
    return v;
}

inline ThreeView three_view(const cps_grid *g)
{
    ThreeView v;
    memset(&v, 0, sizeof(v));
    v.on = g->three_on;
    if (!g->three_on) return v;
    v.ncell = g->t_n; v.cell = g->d_t_cell; v.state = g->d_t_state; v.c = g->tc;
    return v;
}

// clears the device error word of a batch (batch.cpp)
cps_status batch_clear_error(cps_batch *b);
// planes per tile of the H sweeps and of the FP32 E sweeps with gain that a
// batch launches per member (0: its kc)
void batch_set_h_planes(cps_batch *b, int kch, int kcg = 0);

}  // namespace cps
