// capi.cpp -- the C ABI of include/cps_capi.h: grid objects, host FP64
// coefficient builders (restating Structure.cpp:309-359, CPML.cpp:139-527,
// Drude_Lorentz.cpp:65-108, FourLevelLaser.cpp:96-105/202-209,
// TF_SF.cpp:98-955), device allocation, and the step driver.
//
// Built without FMA contraction (host code), so coefficient values equal the
// oracle's bit for bit.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "grid.h"
#include "tfsf_csr.h"

namespace cps {

static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }

}  // namespace cps

using namespace cps;

namespace {
// f(begin, end) over [0, n) split across up to 16 host threads (the calling one included)
template <typename F>
void parallel_for(int n, F f)
{
    const int nt = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), 16));
    const int parts = std::min(nt, n);
    if (parts <= 1) {
        f(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (int t = 1; t < parts; ++t)
        th.emplace_back([&f, n, t, parts] { f((int)((int64_t)n * t / parts), (int)((int64_t)n * (t + 1) / parts)); });
    f(0, (int)((int64_t)n / parts));
    for (std::thread &x : th) x.join();
}
}  // namespace

// calls recorded on the grid run before anything that reads or changes its state
#define FLUSH_RECORDED(g)                                  \
    do {                                                   \
        cps_status fs_ = cps::flush_recorded(g);           \
        if (fs_) return fs_;                               \
    } while (0)

extern "C" const char *cps_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *cps_version(void) { return "cpsfdtd-b200 0.1 (sm_100a)"; }


namespace cps {

cps_status dalloc(cps_grid *g, void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    // stream-ordered pool allocation: freeing a finished job's arrays returns
    // them to the device pool without a device-wide synchronisation
    cudaError_t e = cudaMallocAsync(p, bytes, g->stream);
    if (e != cudaSuccess) {
        set_error(std::string("device allocation of ") + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
        cudaGetLastError();
        return CPS_E_NOMEM;
    }
    g->owned.push_back({*p, bytes});
    e = cudaMemsetAsync(*p, 0, bytes, g->stream);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return CPS_E_CUDA; }
    return CPS_OK;
}

void dfree(cps_grid *g, void *p)
{
    if (!p) return;
    for (auto it = g->owned.begin(); it != g->owned.end(); ++it)
        if (it->first == p) { g->owned.erase(it); break; }
    cudaFreeAsync(p, g->stream);
}

template <typename T>
cps_status upload_T(cps_grid *g, void *dst, const double *src, size_t n)
{
    std::vector<T> tmp(n);
    for (size_t q = 0; q < n; ++q) tmp[q] = (T)src[q];
    CK(cudaMemcpyAsync(dst, tmp.data(), n * sizeof(T), cudaMemcpyHostToDevice, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

cps_status upload_real(cps_grid *g, void *dst, const double *src, size_t n)
{
    return g->fp32 ? upload_T<float>(g, dst, src, n) : upload_T<double>(g, dst, src, n);
}

cps_status upload_raw(cps_grid *g, void *dst, const void *src, size_t bytes)
{
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

// stretch arrays on the device: 12 arrays packed, each padded to 8 entries
cps_status push_stretch(cps_grid *g)
{
    std::vector<double> all;
    for (int w = 0; w < 12; ++w) {
        all.insert(all.end(), g->st[w].begin(), g->st[w].end());
        all.resize((all.size() + 7) / 8 * 8, 0.0);
    }
    if (!g->d_st) {
        cps_status s = dalloc(g, &g->d_st, all.size() * g->esz);
        if (s) return s;
    }
    return upload_real(g, g->d_st, all.data(), all.size());
}

// ------------------------------------------------------------ CPML coefs

// E-side grading, CPML.cpp:139-183
void grade_e(std::vector<double> &kappa, std::vector<double> &b, std::vector<double> &c, bool first, int np,
             double dt, double del, double m, double ma, double sigmax, double kapmax, double alpmax)
{
    std::vector<double> sigma(np + 1), alpha(np + 1);
    kappa.assign(np + 1, 0); b.assign(np + 1, 0); c.assign(np + 1, 0);
    for (int i = 1; i <= np + 1; ++i) {
        double ps, pa;
        if (first) {
            ps = pow(((double)np + 1.0 - i) / ((double)np), m);
            pa = pow(((double)i - 1.0) / ((double)np), ma);
        } else {
            ps = pow(((double)i - 1.0) / np, m);
            pa = pow(((double)np + 1.0 - i) / np, ma);
        }
        sigma[i - 1] = sigmax * ps;
        kappa[i - 1] = 1.0 + (kapmax - 1.0) * ps;
        alpha[i - 1] = alpmax * pa;
    }
    for (int i = 0; i <= np; ++i) {
        b[i] = exp(-(sigma[i] / kappa[i] + alpha[i]) * dt / kEps0);
        if ((sigma[i] == 0.0) && (alpha[i] == 0.0)) c[i] = 0.0;
        else c[i] = sigma[i] * (b[i] - 1.0) / (sigma[i] + kappa[i] * alpha[i]) / kappa[i] / del;
    }
}

// H-side grading, CPML.cpp:185-229, every entry including np-1
void grade_h(std::vector<double> &kappa, std::vector<double> &b, std::vector<double> &c, bool first, int np,
             double dt, double del, double m, double ma, double sigmax, double kapmax, double alpmax)
{
    std::vector<double> sigma(np), alpha(np);
    kappa.assign(np, 0); b.assign(np + 1, 0); c.assign(np + 1, 0);
    for (int i = 1; i <= np; ++i) {
        double ps, pa;
        if (first) { ps = pow(((np - i + 0.5) / np), m); pa = pow(((i - 0.5) / np), ma); }
        else { ps = pow(((i - 0.5) / np), m); pa = pow(((np - i + 0.5) / np), ma); }
        sigma[i - 1] = sigmax * ps;
        kappa[i - 1] = 1.0 + (kapmax - 1.0) * ps;
        alpha[i - 1] = alpmax * pa;
    }
    for (int i = 0; i < np; ++i) {
        b[i] = exp(-(sigma[i] / kappa[i] + alpha[i]) * dt / kEps0);
        if ((sigma[i] == 0.0) && (alpha[i] == 0.0)) c[i] = 0.0;
        else c[i] = sigma[i] * (b[i] - 1.0) / (sigma[i] + kappa[i] * alpha[i]) / kappa[i] / del;
    }
}

// sorted cell list (device linear index) of cells with a given ID inside the
// E-update range, plus per (k, j, 32-wide x segment) start offsets
cps_status build_list(cps_grid *g, int id_match, int64_t *count, int64_t **d_cell, int32_t **d_seg,
                      uint2 **d_segm = nullptr)
{
    const Dims &d = g->d;
    const int nseg = d.px / 32;
    std::vector<int32_t> seg((size_t)(d.nz + 1) * (d.ny + 1) * nseg, 0);
    std::vector<uint2> segm(d_segm ? seg.size() : 0);
    // planes split across threads: each lists its cells with plane-local offsets,
    // then the parts are joined in plane order and the offsets rebased
    const int nz1 = d.nz + 1;
    std::vector<std::vector<int64_t>> part(nz1);
    parallel_for(nz1, [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k) {
            std::vector<int64_t> &cells = part[k];
            for (int j = 0; j <= d.ny; ++j)
                for (int s = 0; s < nseg; ++s) {
                    const size_t w = ((size_t)k * (d.ny + 1) + j) * nseg + s;
                    seg[w] = (int32_t)cells.size();
                    uint32_t bits = 0;
                    if (k >= 1 && k < d.nz && j >= 1 && j < d.ny)
                        for (int i = s * 32; i < s * 32 + 32 && i < d.nx; ++i) {
                            if (i < 1) continue;
                            const int64_t q = d.idx(i, j, k);
                            if (g->ids_dev[q] == id_match) {
                                cells.push_back(q);
                                bits |= 1u << (i - s * 32);
                            }
                        }
                    if (d_segm) segm[w] = make_uint2(0u, bits);
                }
        }
    });
    std::vector<int64_t> base(nz1 + 1, 0);
    for (int k = 0; k < nz1; ++k) base[k + 1] = base[k] + (int64_t)part[k].size();
    REQUIRE(base[nz1] < (int64_t)INT32_MAX, CPS_E_INVALID, "too many cells in one compacted list");
    std::vector<int64_t> cells((size_t)base[nz1]);
    parallel_for(nz1, [&](int k0, int k1) {
        for (int k = k0; k < k1; ++k) {
            std::copy(part[k].begin(), part[k].end(), cells.begin() + base[k]);
            const size_t w0 = (size_t)k * (d.ny + 1) * nseg, w1 = w0 + (size_t)(d.ny + 1) * nseg;
            for (size_t w = w0; w < w1; ++w) {
                seg[w] += (int32_t)base[k];
                if (d_segm) segm[w].x = (unsigned)seg[w];
            }
        }
    });
    REQUIRE(cells.size() < (size_t)INT32_MAX, CPS_E_INVALID, "too many cells in one compacted list");
    *count = (int64_t)cells.size();
    cps_status s = dalloc(g, (void **)d_cell, cells.size() * sizeof(int64_t));
    if (s) return s;
    s = dalloc(g, (void **)d_seg, seg.size() * sizeof(int32_t));
    if (s) return s;
    if (!cells.empty()) { s = upload_raw(g, *d_cell, cells.data(), cells.size() * sizeof(int64_t)); if (s) return s; }
    if (d_segm) {
        if ((s = dalloc(g, (void **)d_segm, segm.size() * sizeof(uint2)))) return s;
        if ((s = upload_raw(g, *d_segm, segm.data(), segm.size() * sizeof(uint2)))) return s;
    }
    return upload_raw(g, *d_seg, seg.data(), seg.size() * sizeof(int32_t));
}

// initial gain state: all zero (FP32 keeps population offsets) except FP64
// N0 = N1 = 1 (FourLevelLaser.cpp:194-197)
cps_status gain_state_init(cps_grid *g)
{
    if (g->fp32) {
        CK(cudaMemsetAsync(g->d_g_state, 0, (size_t)g->elems * kGainPersist * sizeof(float), g->stream));
        CK(cudaMemsetAsync(g->d_g_trans, 0, (size_t)gain_state_elems(g->g_n, kGainTrans) * sizeof(float), g->stream));
    } else {
        CK(cudaMemsetAsync(g->d_g_state, 0, (size_t)gain_state_elems(g->g_n, kG64Words) * sizeof(double), g->stream));
    }
    if (!g->fp32 && g->g_n > 0) {
        launch_gain_init64((double *)g->d_g_state, g->g_n, g->stream);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

cps_status flush_dft(cps_grid *g, PortState &P);

cps_status ensure_sources(cps_grid *g)
{
    if (!g->src_dirty) return CPS_OK;
    for (void *p : {(void *)g->d_src_idx, (void *)g->d_src_comp, (void *)g->d_src_off, (void *)g->d_src_len,
                    (void *)g->d_src_wave})
        dfree(g, p);
    const size_t ns = g->src.size();
    std::vector<int64_t> idx(ns);
    std::vector<int32_t> comp(ns), off(ns), len(ns);
    std::vector<double> wave;
    for (size_t s = 0; s < ns; ++s) {
        idx[s] = g->src[s].idx; comp[s] = g->src[s].comp;
        off[s] = (int32_t)wave.size(); len[s] = (int32_t)g->src[s].wave.size();
        wave.insert(wave.end(), g->src[s].wave.begin(), g->src[s].wave.end());
    }
    cps_status s;
    if ((s = dalloc(g, (void **)&g->d_src_idx, ns * 8)) || (s = dalloc(g, (void **)&g->d_src_comp, ns * 4)) ||
        (s = dalloc(g, (void **)&g->d_src_off, ns * 4)) || (s = dalloc(g, (void **)&g->d_src_len, ns * 4)) ||
        (s = dalloc(g, (void **)&g->d_src_wave, wave.size() * 8)))
        return s;
    if ((s = upload_raw(g, g->d_src_idx, idx.data(), ns * 8)) || (s = upload_raw(g, g->d_src_comp, comp.data(), ns * 4)) ||
        (s = upload_raw(g, g->d_src_off, off.data(), ns * 4)) || (s = upload_raw(g, g->d_src_len, len.data(), ns * 4)) ||
        (s = upload_raw(g, g->d_src_wave, wave.data(), wave.size() * 8)))
        return s;
    g->src_dirty = false;
    return CPS_OK;
}

// ---------------------------------------------------------- step pieces

template <typename T>
void op_inject(cps_grid *g, int isH, double n, uint32_t mask)
{
    if (!g->tfsf_on || g->ntg[isH] == 0) return;
    const FieldView<T> f = field_view<T>(g);
    launch_inject<T>(f, g->d_tg[isH], g->ntg[isH], g->d_ct[isH], (const T *)(isH ? g->d_einc : g->d_hinc),
                     g->tp.Nt, n, mask, g->stream);
    g->launches++;
}

template <typename T>
void op_sources(cps_grid *g, int n)
{
    if (g->src.empty()) return;
    launch_sources<T>(field_view<T>(g), (int)g->src.size(), g->d_src_idx, g->d_src_comp, g->d_src_wave,
                      g->d_src_off, g->d_src_len, n, g->stream);
    g->launches++;
}

// Sample ports into their rings (Update_Fields_on_Port), all ports of the
// list in one launch; a full ring is first folded into the DFT accumulators.
template <typename T>
cps_status op_ports(cps_grid *g, PortState *const *ports, int nports, int64_t n, const int64_t *port_n = nullptr)
{
    for (int b0 = 0; b0 < nports; b0 += kMaxGather) {
        GatherBatch B;
        memset(&B, 0, sizeof(B));
        for (int q = b0; q < nports && q < b0 + kMaxGather; ++q) {
            PortState &P = *ports[q];
            if (P.fill == P.slots) {
                cps_status s = flush_dft(g, P);
                if (s) return s;
            }
            if (P.fill == 0) P.ring_n0 = port_n ? port_n[q] : n;
            GatherDesc &D = B.p[B.n++];
            D.idx = P.d_idx;
            D.slot = (T *)P.d_ring + (int64_t)P.fill * 6 * P.npts;
            D.npts = P.npts;
            B.max_npts = std::max(B.max_npts, P.npts);
            P.last_slot = P.fill;
            P.fill++;
            if (P.nfreq == 0) P.fill = 0;  // no DFT: the ring holds the last sample only
        }
        launch_port_gather<T>(field_view<T>(g), B, g->stream);
        g->launches++;
    }
    return CPS_OK;
}

template <typename T>
cps_status op_port(cps_grid *g, PortState &P, int64_t n)
{
    PortState *one = &P;
    return op_ports<T>(g, &one, 1, n);
}

template <typename T>
cps_status flush_dft_T(cps_grid *g, PortState &P)
{
    if (P.nfreq == 0 || P.fill == 0) return CPS_OK;
    const size_t need = (size_t)2 * P.slots * P.nfreq * 2 * sizeof(double);  // [2][slots][nfreq] of (cos, sin)
    if (g->phasor_cap < need) {
        dfree(g, g->d_phasor);
        cps_status s = dalloc(g, (void **)&g->d_phasor, need);
        if (s) return s;
        g->phasor_cap = need;
    }
    launch_port_dft<T>((const T *)P.d_ring, P.npts, P.fill, P.ring_n0, g->desc.dt, P.d_omega, P.nfreq, P.d_comps,
                       P.ncomp, P.d_acc, g->d_phasor, g->stream);
    // a failed launch leaves the ring as it was, so a later flush folds its samples
    const cudaError_t e = cudaGetLastError();
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("port DFT launch failed: ") + cudaGetErrorString(e));
    g->launches += 2;
    // keep the last sample readable: move it to slot 0
    if (P.last_slot > 0) {
        CK(cudaMemcpyAsync(P.d_ring, (T *)P.d_ring + (int64_t)P.last_slot * 6 * P.npts, sizeof(T) * 6 * P.npts,
                           cudaMemcpyDeviceToDevice, g->stream));
        P.last_slot = 0;
    }
    P.fill = 0;
    return CPS_OK;
}

cps_status flush_dft(cps_grid *g, PortState &P)
{
    return g->fp32 ? flush_dft_T<float>(g, P) : flush_dft_T<double>(g, P);
}

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiled)p;
    });
    return fn;
}

// tensor maps of the six fields and the IDs for tiles of `by` rows
cps_status ensure_tma(cps_grid *g)
{
    const int by = g->shape.by;
    if (g->tma_by == by) return CPS_OK;
    EncodeTiled enc = encode_fn();
    REQUIRE(enc, CPS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const Dims &d = g->d;
    const cuuint64_t dims[3] = {(cuuint64_t)d.px, (cuuint64_t)(d.ny + 1), (cuuint64_t)(d.nz + 1)};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUtensorMapDataType dt = g->fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t st[2] = {(cuuint64_t)d.px * g->esz, (cuuint64_t)d.pxy * g->esz};
    const cuuint32_t halo[3] = {36, (cuuint32_t)by + 1, 1}, own[3] = {32, (cuuint32_t)by, 1};
    for (int c = 0; c < 6; ++c) {
        CUresult r1 = enc(&g->tma.halo[c], dt, 3, g->F[c], dims, st, halo, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        CUresult r2 = enc(&g->tma.own[c], dt, 3, g->F[c], dims, st, own, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        REQUIRE(r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS, CPS_E_CUDA, "cuTensorMapEncodeTiled failed for a field");
    }
    const cuuint64_t sid[2] = {(cuuint64_t)d.px, (cuuint64_t)d.pxy};
    CUresult r = enc(&g->tma.id, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, g->d_id, dims, sid, own, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    REQUIRE(r == CUDA_SUCCESS, CPS_E_CUDA, "cuTensorMapEncodeTiled failed for the IDs");
    if (g->gain_on && g->fp32) {
        // segment-dense gain words: {32 lanes, 15 words, segments, rows, planes}
        const cuuint64_t nseg = (cuuint64_t)d.px / 32;
        const cuuint64_t gdims[5] = {32, (cuuint64_t)kGainPersist, nseg, (cuuint64_t)(d.ny + 1), (cuuint64_t)(d.nz + 1)};
        const cuuint64_t seg_b = (cuuint64_t)kGainPersist * 32 * sizeof(float);
        const cuuint64_t gst[4] = {32 * sizeof(float), seg_b, nseg * seg_b, nseg * seg_b * (cuuint64_t)(d.ny + 1)};
        const cuuint32_t gbox[5] = {32, (cuuint32_t)kGainPersist, 1, (cuuint32_t)by, 1};
        const cuuint32_t ges[5] = {1, 1, 1, 1, 1};
        r = enc(&g->tma.gain, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, g->d_g_state, gdims, gst, gbox, ges,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        REQUIRE(r == CUDA_SUCCESS, CPS_E_CUDA, "cuTensorMapEncodeTiled failed for the gain words");
    }
    g->tma_by = by;
    return CPS_OK;
}

// tensor maps of the one-pass sweep over one buffer set (E boxes 40 x (by+2),
// H boxes 36 x (by+1), ID box 48 x (by+1))
cps_status encode_step_maps(cps_grid *g, void *const F[6], StepMaps *m, int by)
{
    EncodeTiled enc = encode_fn();
    REQUIRE(enc, CPS_E_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    const Dims &d = g->d;
    const cuuint64_t dims[3] = {(cuuint64_t)d.px, (cuuint64_t)(d.ny + 1), (cuuint64_t)(d.nz + 1)};
    const cuuint32_t es[3] = {1, 1, 1};
    const CUtensorMapDataType dt = g->fp32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    const cuuint64_t st[2] = {(cuuint64_t)d.px * g->esz, (cuuint64_t)d.pxy * g->esz};
    const cuuint32_t ebox[3] = {40, (cuuint32_t)by + 2, 1}, hbox[3] = {36, (cuuint32_t)by + 1, 1};
    const cuuint32_t ibox[3] = {48, (cuuint32_t)by + 1, 1};
    for (int c = 0; c < 3; ++c) {
        CUresult r1 = enc(&m->e[c], dt, 3, F[c], dims, st, ebox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        CUresult r2 = enc(&m->h[c], dt, 3, F[3 + c], dims, st, hbox, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        REQUIRE(r1 == CUDA_SUCCESS && r2 == CUDA_SUCCESS, CPS_E_CUDA, "cuTensorMapEncodeTiled failed for a field");
    }
    const cuuint64_t sid[2] = {(cuuint64_t)d.px, (cuuint64_t)d.pxy};
    CUresult r = enc(&m->id, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, g->d_id, dims, sid, ibox, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    REQUIRE(r == CUDA_SUCCESS, CPS_E_CUDA, "cuTensorMapEncodeTiled failed for the IDs");
    return CPS_OK;
}

cps_status ensure_onepass(cps_grid *g)
{
    cps_status s;
    if (!g->F2[0]) {
        // zeroed once: the sweep writes every cell of the arrays, never the x padding
        for (int c = 0; c < 6; ++c) {
            if ((s = dalloc(g, &g->F2[c], (size_t)g->elems * g->esz))) return s;
            CK(cudaMemsetAsync(g->F2[c], 0, (size_t)g->elems * g->esz, g->stream));
        }
    }
    if (g->pml_on && !g->d_q2[0][0]) {
        for (int f = 0; f < 6; ++f)
            for (int q = 0; q < 2; ++q) {
                const size_t n = psi_words(g, f) * g->esz;
                if ((s = dalloc(g, &g->d_q2[f][q], n))) return s;
                CK(cudaMemsetAsync(g->d_q2[f][q], 0, n, g->stream));
            }
    }
    if (g->tfsf_on && g->ntg[1] > 0 && !g->d_hslot && g->hc_ok) {
        // each H-side contribution's slot in the per-face arrays of the targets' bounding box
        const Dims &d = g->d;
        std::vector<InjTarget> tg(g->ntg[1]);
        CK(cudaMemcpyAsync(tg.data(), g->d_tg[1], tg.size() * sizeof(InjTarget), cudaMemcpyDeviceToHost, g->stream));
        CK(cudaStreamSynchronize(g->stream));
        int nct = 0;
        for (const InjTarget &t : tg) nct = std::max(nct, t.start + t.count);
        std::vector<InjContrib> ct(nct);
        CK(cudaMemcpyAsync(ct.data(), g->d_ct[1], ct.size() * sizeof(InjContrib), cudaMemcpyDeviceToHost, g->stream));
        CK(cudaStreamSynchronize(g->stream));
        std::vector<int> ijk(3 * tg.size());
        int box[6] = {INT32_MAX, -1, INT32_MAX, -1, INT32_MAX, -1};
        for (size_t t = 0; t < tg.size(); ++t) {
            const int64_t q = tg[t].idx;
            const int k = (int)(q / d.pxy), j = (int)((q - k * d.pxy) / d.px), i = (int)(q - k * d.pxy - (int64_t)j * d.px);
            const int v[3] = {i, j, k};
            for (int a = 0; a < 3; ++a) {
                ijk[3 * t + a] = v[a];
                box[2 * a] = std::min(box[2 * a], v[a]);
                box[2 * a + 1] = std::max(box[2 * a + 1], v[a]);
            }
        }
        int base = 0;
        for (int f = 0; f < 6; ++f) {
            const int ax = f >> 1, ua = ax == 0 ? 1 : 0, va = ax == 2 ? 1 : 2;
            g->hc_nu[f] = box[2 * ua + 1] - box[2 * ua] + 1;
            g->hc_area[f] = g->hc_nu[f] * (box[2 * va + 1] - box[2 * va] + 1);
            g->hc_base[f] = base;
            base += 3 * g->hc_area[f];
        }
        std::vector<int32_t> slot(nct, -1);
        bool ok = true;
        for (size_t t = 0; t < tg.size() && ok; ++t)
            for (int c = tg[t].start; c < tg[t].start + tg[t].count && ok; ++c) {
                const int f = ct[c].face, ax = f >> 1, ua = ax == 0 ? 1 : 0, va = ax == 2 ? 1 : 2;
                const int *v = &ijk[3 * t];
                ok = f >= 0 && f < 6 && v[ax] == box[f] && tg[t].comp >= CPS_HX && tg[t].comp <= CPS_HZ;
                if (ok)
                    slot[c] = g->hc_base[f] + (tg[t].comp - CPS_HX) * g->hc_area[f] +
                              (v[va] - box[2 * va]) * g->hc_nu[f] + (v[ua] - box[2 * ua]);
            }
        // a cell on two faces sums both, so each face takes its own contributions only once
        for (int c = 0; c < nct && ok; ++c) ok = slot[c] >= 0;
        if (ok) {
            std::vector<int32_t> seen(base, 0);
            for (int c = 0; c < nct && ok; ++c) ok = seen[slot[c]]++ == 0;
        }
        g->hc_ok = ok;
        if (ok) {
            for (int a = 0; a < 6; ++a) g->hc_box[a] = box[a];
            g->hc_n = nct;
            if ((s = dalloc(g, &g->d_hcorr, (size_t)base * g->esz))) return s;
            CK(cudaMemsetAsync(g->d_hcorr, 0, (size_t)base * g->esz, g->stream));
            if ((s = dalloc(g, (void **)&g->d_hslot, slot.size() * sizeof(int32_t)))) return s;
            if ((s = upload_raw(g, g->d_hslot, slot.data(), slot.size() * sizeof(int32_t)))) return s;
        }
    }
    const int by = g->shape.by;
    if (g->om_by != by) {
        if ((s = encode_step_maps(g, g->F, &g->om, by)) || (s = encode_step_maps(g, g->F2, &g->om2, by))) return s;
        g->om_by = by;
    }
    g->onepass_ready = true;
    return CPS_OK;
}

void swap_step_buffers(cps_grid *g)
{
    for (int c = 0; c < 6; ++c) std::swap(g->F[c], g->F2[c]);
    if (g->pml_on)
        for (int f = 0; f < 6; ++f) {
            std::swap(g->d_q[f][2], g->d_q2[f][0]);
            std::swap(g->d_q[f][3], g->d_q2[f][1]);
        }
    std::swap(g->om, g->om2);
    g->tma_by = 0;  // the two-sweep maps were built over the other buffers
}

template <typename T>
HCorr<T> h_corrections(const cps_grid *g)
{
    HCorr<T> q;
    memset(&q, 0, sizeof(q));
    if (g->tfsf_on && g->ntg[1] > 0) {
        q.corr = (const T *)g->d_hcorr;
        for (int a = 0; a < 6; ++a) {
            q.box[a] = g->hc_box[a]; q.base[a] = g->hc_base[a]; q.nu[a] = g->hc_nu[a]; q.area[a] = g->hc_area[a];
        }
    }
    return q;
}

cps_status check_device_error(cps_grid *g)
{
    int e = 0;
    CK(cudaMemcpyAsync(&e, g->d_err, sizeof(int), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    REQUIRE(e == 0, CPS_E_TIMEOUT, "a device-side wait of a sweep gave up (TMA data did not arrive)");
    return CPS_OK;
}

template <typename T>
cps_status step_T(cps_grid *g, int nsteps, int path)
{
    cps_status s = ensure_sources(g);
    if (s) return s;
    // TMA boxes are 36 x (rows+1): grids narrower than that use the register sweeps
    const bool use_tma = path != CPS_PATH_PLAIN && g->sweep_mode == 0 && (g->shape.by == 4 || g->shape.by == 8) &&
                         g->d.px >= 64 && g->d.ny + 1 >= g->shape.by + 1;
    bool onepass = use_tma && path == CPS_PATH_ONEPASS;
    if (onepass && (s = ensure_onepass(g))) return s;
    onepass = onepass && g->hc_ok;  // TF/SF targets off their box's surface: two sweeps instead
    if (use_tma && !onepass && (s = ensure_tma(g))) return s;
    const FieldView<T> f = field_view<T>(g);
    const PmlView<T> p = pml_view<T>(g);
    const DlView<T> D = dl_view<T>(g);
    const GainView<T> G = gain_view<T>(g);
    for (int it = 0; it < nsteps; ++it) {
        const int64_t n = g->step;
        if (path == CPS_PATH_PLAIN) {
            launch_h_bulk<T>(f, g->stream);
            op_inject<T>(g, 1, (double)n, CPS_FACE_ALL);
            if (g->pml_on) launch_h_pml<T>(f, p, g->stream);
            launch_e_bulk<T>(f, g->stream);
            if (g->dl_on) launch_dl<T>(f, D, g->stream);
            if (g->gain_on) {
                launch_gain<T>(f, G, 0, g->stream);
                launch_gain<T>(f, G, 1, g->stream);
                launch_gain<T>(f, G, 2, g->stream);
            }
            if (g->three_on) {
                const ThreeView tv = three_view(g);
                launch_three<T>(f, tv, 0, g->stream);
                launch_three<T>(f, tv, 1, g->stream);
                launch_three<T>(f, tv, 2, g->stream);
                g->launches += 3;
            }
            op_inject<T>(g, 0, (double)n, CPS_FACE_ALL);
            op_sources<T>(g, (int)n);
            if (g->pml_on) launch_e_pml<T>(f, p, g->stream);
            g->launches += 2 + (g->pml_on ? 12 : 0) + (g->dl_on ? 1 : 0) + (g->gain_on ? 3 : 0);
        } else if (onepass) {
            // one sweep into the other buffers, which become current; then the
            // Drude-Lorentz cells (old E from the previous buffers), TF/SF E, sources
            const bool timed = g->timing_stride > 0 && n % g->timing_stride == 0 &&
                               g->ev_used + 4 <= (int)g->ev.size();
            if (timed) cudaEventRecord(g->ev[g->ev_used], g->stream);
            if (g->tfsf_on && g->ntg[1] > 0) {
                launch_h_corrections<T>(g->d_ct[1], g->d_hslot, g->hc_n, (const T *)g->d_einc, g->tp.Nt, (double)n,
                                        (T *)g->d_hcorr, g->stream);
                g->launches++;
            }
            launch_step_tma<T>(g->om, field_view<T>(g), field_view_alt<T>(g), pml_view<T>(g), pml_view_alt<T>(g), D,
                               G, h_corrections<T>(g), g->shape, g->d_err, g->stream);
            g->launches++;
            swap_step_buffers(g);
            if (timed) {
                cudaEventRecord(g->ev[g->ev_used + 1], g->stream);
                cudaEventRecord(g->ev[g->ev_used + 2], g->stream);
            }
            if (D.on && D.ncell > 0) {
                launch_dl_cells_step<T>(field_view<T>(g), field_view_alt<T>(g), pml_view<T>(g), D, g->stream);
                g->launches++;
            }
            if (g->three_on) {
                launch_three<T>(field_view<T>(g), three_view(g), 3, g->stream);
                g->launches++;
            }
            if (timed) {
                cudaEventRecord(g->ev[g->ev_used + 3], g->stream);
                g->ev_used += 4;
            }
            op_inject<T>(g, 0, (double)n, CPS_FACE_ALL);
            op_sources<T>(g, (int)n);
        } else {
            const bool timed = g->timing_stride > 0 && n % g->timing_stride == 0 &&
                               g->ev_used + 4 <= (int)g->ev.size();
            if (timed) cudaEventRecord(g->ev[g->ev_used], g->stream);
            if (use_tma) g->launches += launch_h_tma<T>(g->tma, f, p, g->shape, g->d_err, g->stream);
            else launch_h_fused<T>(f, p, g->shape, g->stream), g->launches++;
            if (timed) cudaEventRecord(g->ev[g->ev_used + 1], g->stream);
            op_inject<T>(g, 1, (double)n, CPS_FACE_ALL);
            if (timed) cudaEventRecord(g->ev[g->ev_used + 2], g->stream);
            if (use_tma) g->launches += launch_e_tma<T>(g->tma, f, p, D, G, g->shape, g->d_err, g->stream, &g->lane);
            else launch_e_fused<T>(f, p, D, G, g->shape, g->stream), g->launches++;
            if (g->three_on) {
                launch_three<T>(f, three_view(g), 3, g->stream);
                g->launches++;
            }
            if (timed) {
                cudaEventRecord(g->ev[g->ev_used + 3], g->stream);
                g->ev_used += 4;
            }
            op_inject<T>(g, 0, (double)n, CPS_FACE_ALL);
            op_sources<T>(g, (int)n);
        }
        if (!g->ports.empty()) {
            std::vector<PortState *> all;
            for (PortState &P : g->ports) all.push_back(&P);
            s = op_ports<T>(g, all.data(), (int)all.size(), n);
            if (s) return s;
        }
        g->step++;
    }
    cudaError_t e = cudaGetLastError();
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return CPS_OK;
}

cps_status need_setup(const cps_grid *g)
{
    REQUIRE(g, CPS_E_INVALID, "grid handle is NULL");
    REQUIRE(g->nmedia > 0, CPS_E_STATE, "media are not set (cps_grid_set_media)");
    REQUIRE(g->ids_set, CPS_E_STATE, "material IDs are not uploaded (cps_grid_upload_ids)");
    return CPS_OK;
}

}  // namespace cps

// ================================================================ lifetime

extern "C" cps_status cps_grid_create(const cps_grid_desc *desc, cps_grid **out)
{
    REQUIRE(desc && out, CPS_E_INVALID, "cps_grid_create: NULL argument");
    *out = nullptr;
    REQUIRE(desc->nx >= 4 && desc->ny >= 4 && desc->nz >= 4, CPS_E_INVALID, "grid needs at least 4 cells per axis");
    REQUIRE(desc->nx < 16384 && desc->ny < 16384 && desc->nz < 16384, CPS_E_INVALID, "grid edge too large");
    REQUIRE(desc->dx > 0 && desc->dy > 0 && desc->dz > 0, CPS_E_INVALID, "cell sizes must be positive");
    REQUIRE(desc->precision == CPS_FP64 || desc->precision == CPS_FP32, CPS_E_INVALID, "precision must be CPS_FP64 or CPS_FP32");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    REQUIRE(desc->device >= 0 && desc->device < ndev, CPS_E_INVALID, "no such CUDA device");
    CK(cudaSetDevice(desc->device));
    {
        // this process's default pool on the device keeps freed memory for the
        // next grid instead of handing it back to the driver
        static std::mutex pool_mu;
        static std::vector<int> pooled;
        std::lock_guard<std::mutex> lk(pool_mu);
        if (std::find(pooled.begin(), pooled.end(), desc->device) == pooled.end()) {
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, desc->device) == cudaSuccess) {
                uint64_t keep = UINT64_MAX;
                cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
            }
            cudaGetLastError();
            pooled.push_back(desc->device);
        }
    }
    cps_grid *g = new cps_grid();
    g->desc = *desc;
    if (!(g->desc.dt > 0)) g->desc.dt = cps_courant_dt(desc->dx, desc->dy, desc->dz);
    g->fp32 = desc->precision == CPS_FP32;
    g->esz = g->fp32 ? 4 : 8;
    g->d.nx = desc->nx; g->d.ny = desc->ny; g->d.nz = desc->nz;
    g->d.px = (desc->nx + 1 + kXPad - 1) / kXPad * kXPad;
    g->d.pxy = (int64_t)g->d.px * (desc->ny + 1);
    g->elems = g->d.pxy * (desc->nz + 1);
    cudaError_t e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); delete g; return CPS_E_CUDA; }
    g->own_stream = true;
    e = cudaStreamCreateWithFlags(&g->lane.s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->lane.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g->lane.join, cudaEventDisableTiming);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); cps_grid_destroy(g); return CPS_E_CUDA; }
    cps_status s = CPS_OK;
    for (int c = 0; c < 6 && !s; ++c) s = dalloc(g, &g->F[c], (size_t)g->elems * g->esz);
    if (!s) s = dalloc(g, (void **)&g->d_id, (size_t)g->elems);
    if (!s) s = dalloc(g, &g->d_media, 4 * 256 * g->esz);
    if (!s) s = dalloc(g, (void **)&g->d_counter, sizeof(unsigned long long));
    if (!s) s = dalloc(g, (void **)&g->d_err, 2 * sizeof(int));  // error code, wait test setting
    if (s) { cps_grid_destroy(g); return s; }
    g->ids_dev.assign((size_t)g->elems, 0);
    // stretched coordinates start at 1/delta (Structure.cpp:425-445)
    for (int w = 0; w < 12; ++w) {
        const int axis = (w % 6) < 2 ? 2 : ((w % 6) < 4 ? 1 : 0);
        const double del = axis == 0 ? desc->dx : axis == 1 ? desc->dy : desc->dz;
        g->st[w].assign(kStretchLen(g, w), 1.0 / del);
    }
    s = push_stretch(g);
    if (s) { cps_grid_destroy(g); return s; }
    e = cudaStreamSynchronize(g->stream);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); cps_grid_destroy(g); return CPS_E_CUDA; }
    *out = g;
    return CPS_OK;
}

extern "C" cps_status cps_grid_destroy(cps_grid *g)
{
    if (!g) return CPS_OK;
    cudaSetDevice(g->desc.device);
    if (g->solo) cps_batch_destroy(g->solo);
    for (auto &a : g->owned) cudaFreeAsync(a.first, g->stream);
    g->owned.clear();
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (auto &e : g->ev) cudaEventDestroy(e);
    if (g->lane.s) cudaStreamSynchronize(g->lane.s);
    if (g->lane.fork) cudaEventDestroy(g->lane.fork);
    if (g->lane.join) cudaEventDestroy(g->lane.join);
    if (g->lane.s) cudaStreamDestroy(g->lane.s);
    if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
    delete g;
    return CPS_OK;
}

extern "C" cps_status cps_grid_info(const cps_grid *g, cps_grid_desc *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "NULL argument");
    *out = g->desc;
    return CPS_OK;
}

extern "C" cps_status cps_grid_coefficients(const cps_grid *g, double *aE, double *bE, double *aH, double *bH)
{
    REQUIRE(g, CPS_E_INVALID, "cps_grid_coefficients: NULL grid");
    REQUIRE(g->nmedia > 0, CPS_E_STATE, "cps_grid_coefficients: media are not set");
    for (int m = 0; m < g->nmedia; ++m) {
        if (aE) aE[m] = g->aE[m];
        if (bE) bE[m] = g->bE[m];
        if (aH) aH[m] = g->aH[m];
        if (bH) bH[m] = g->bH[m];
    }
    return CPS_OK;
}

extern "C" cps_status cps_grid_stretch(const cps_grid *g, int32_t which, double *out, int32_t *len)
{
    REQUIRE(g, CPS_E_INVALID, "cps_grid_stretch: NULL grid");
    REQUIRE(which >= 0 && which < 12, CPS_E_INVALID, "cps_grid_stretch: which is 0..11");
    const int n = kStretchLen(g, which);
    if (len) *len = n;
    if (out)
        for (int q = 0; q < n; ++q) out[q] = q < (int)g->st[which].size() ? g->st[which][q] : 0.0;
    return CPS_OK;
}

extern "C" cps_status cps_grid_bytes(const cps_grid *g, int64_t *bytes)
{
    REQUIRE(g && bytes, CPS_E_INVALID, "NULL argument");
    size_t total = 0;
    for (const auto &a : g->owned) total += a.second;
    *bytes = (int64_t)total;
    return CPS_OK;
}

extern "C" cps_status cps_grid_set_stream(cps_grid *g, void *stream)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    FLUSH_RECORDED(g);
    CK(cudaStreamSynchronize(g->stream));
    if (g->own_stream && stream) { cudaStreamDestroy(g->stream); g->own_stream = false; }
    if (stream) g->stream = (cudaStream_t)stream;
    return CPS_OK;
}

extern "C" cps_status cps_grid_get_stream(const cps_grid *g, void **stream)
{
    REQUIRE(g && stream, CPS_E_INVALID, "NULL argument");
    *stream = (void *)g->stream;
    return CPS_OK;
}

extern "C" cps_status cps_synchronize(cps_grid *g)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    FLUSH_RECORDED(g);
    if (g->solo) {
        cps_status s = cps_batch_synchronize(g->solo);
        if (s) return s;
    }
    CK(cudaStreamSynchronize(g->stream));
    return check_device_error(g);
}

// ================================================================ geometry

extern "C" cps_status cps_grid_set_media(cps_grid *g, int32_t n, const double *epsR, const double *muR,
                                         const double *sig, const double *sigM)
{
    REQUIRE(g && epsR && muR && sig && sigM, CPS_E_INVALID, "cps_grid_set_media: NULL argument");
    FLUSH_RECORDED(g);
    REQUIRE(n >= 1 && n <= 256, CPS_E_INVALID, "cps_grid_set_media: 1..256 media");
    const double dt = g->desc.dt;
    for (int i = 0; i < n; ++i) {
        REQUIRE(epsR[i] > 0 && muR[i] > 0, CPS_E_INVALID, "cps_grid_set_media: epsR and muR must be positive");
        // Structure.cpp:446-451
        g->aE[i] = (2.0 * kEps0 * epsR[i] - sig[i] * dt) / (2.0 * kEps0 * epsR[i] + sig[i] * dt);
        g->bE[i] = (2.0 * dt) / (2.0 * kEps0 * epsR[i] + sig[i] * dt);
        g->aH[i] = (2.0 * kMu0 * muR[i] - sigM[i] * dt) / (2.0 * kMu0 * muR[i] + sigM[i] * dt);
        g->bH[i] = (2.0 * dt) / (2.0 * kMu0 * muR[i] + sigM[i] * dt);
        g->eps_r[i] = epsR[i];
        g->mu_r[i] = muR[i];
    }
    g->nmedia = n;
    std::vector<double> t(1024, 0.0);
    for (int i = 0; i < 256; ++i) { t[i] = g->aE[i]; t[256 + i] = g->bE[i]; t[512 + i] = g->aH[i]; t[768 + i] = g->bH[i]; }
    return upload_real(g, g->d_media, t.data(), t.size());
}

extern "C" cps_status cps_grid_upload_ids(cps_grid *g, const uint8_t *ids)
{
    REQUIRE(g && ids, CPS_E_INVALID, "cps_grid_upload_ids: NULL argument");
    FLUSH_RECORDED(g);
    REQUIRE(!g->dl_on && !g->gain_on && !g->pml_on, CPS_E_STATE,
            "cps_grid_upload_ids: IDs must be set before the physics modules are initialised");
    const Dims &d = g->d;
    std::fill(g->ids_dev.begin(), g->ids_dev.end(), 0);
    // [i][j][k] to the device layout in 64 x 64 (i, k) blocks per row j, rows split across threads
    std::mutex mu;
    int maxid = 0;
    uint8_t *dst = g->ids_dev.data();
    parallel_for(d.ny + 1, [&](int j0, int j1) {
        int mx = 0;
        for (int j = j0; j < j1; ++j)
            for (int ib = 0; ib <= d.nx; ib += 64)
                for (int kb = 0; kb <= d.nz; kb += 64) {
                    const int ie = std::min(ib + 64, d.nx + 1), kend = std::min(kb + 64, d.nz + 1);
                    for (int i = ib; i < ie; ++i) {
                        const uint8_t *src = ids + ((size_t)i * (d.ny + 1) + j) * (d.nz + 1);
                        for (int k = kb; k < kend; ++k) {
                            const uint8_t v = src[k];
                            mx = std::max<int>(mx, v);
                            dst[d.idx(i, j, k)] = v;
                        }
                    }
                }
        std::lock_guard<std::mutex> lk(mu);
        maxid = std::max(maxid, mx);
    });
    REQUIRE(g->nmedia == 0 || maxid < g->nmedia, CPS_E_INVALID,
            "cps_grid_upload_ids: an ID has no medium (set the media first or extend them)");
    g->ids_max = maxid;
    cps_status s = upload_raw(g, g->d_id, g->ids_dev.data(), g->ids_dev.size());
    if (s) return s;
    g->ids_set = true;
    return CPS_OK;
}

extern "C" cps_status cps_grid_download_ids(const cps_grid *g, uint8_t *ids)
{
    REQUIRE(g && ids, CPS_E_INVALID, "NULL argument");
    const Dims &d = g->d;
    size_t q = 0;
    for (int i = 0; i <= d.nx; ++i)
        for (int j = 0; j <= d.ny; ++j)
            for (int k = 0; k <= d.nz; ++k) ids[q++] = g->ids_dev[d.idx(i, j, k)];
    return CPS_OK;
}

// ================================================================ modules

extern "C" cps_status cps_pml_init(cps_grid *g, const cps_pml_params *pp)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(pp, CPS_E_INVALID, "cps_pml_init: NULL params");
    REQUIRE(!g->pml_on, CPS_E_STATE, "cps_pml_init: CPML already initialised");
    const int nax[3] = {g->d.nx, g->d.ny, g->d.nz};
    for (int a = 0; a < 3; ++a) {
        const int n1 = pp->npml[2 * a], n2 = pp->npml[2 * a + 1];
        REQUIRE(n1 == n2, CPS_E_INVALID,
                "cps_pml_init: both ends of an axis need the same thickness (the reference folds the second-end "
                "kappa with the first-end count, CPML.cpp:374)");
        REQUIRE(n1 >= 1 && 2 * n1 < nax[a] - 1, CPS_E_INVALID, "cps_pml_init: thickness must be >= 1 and leave an interior");
    }
    REQUIRE(pp->m >= 0 && pp->kapmax >= 1.0 && pp->alpmax >= 0, CPS_E_INVALID, "cps_pml_init: bad grading parameters");
    REQUIRE(pp->literal == 0 || pp->literal == 1, CPS_E_INVALID, "cps_pml_init: literal must be 0 or 1");
    g->pml = *pp;
    const double eta0 = sqrt(kMu0 / kEps0);
    const double del[3] = {g->desc.dx, g->desc.dy, g->desc.dz};
    // stretch arrays: E side (cEzy,cEyz | cEzx,cExz | cExy,cEyx), H side likewise
    const int wE[3][2] = {{4, 5}, {2, 3}, {0, 1}};
    const int wH[3][2] = {{10, 11}, {8, 9}, {6, 7}};
    for (int a = 0; a < 3; ++a) {
        const double sigmax = pp->sig_ratio * (0.8 * (pp->m + 1) / (del[a] * eta0));
        for (int end = 0; end < 2; ++end) {
            const int f = 2 * a + end, np = pp->npml[f];
            std::vector<double> kap, kapH, bh, ch;
            grade_e(kap, g->pbE[f], g->pcE[f], end == 0, np, g->desc.dt, del[a], pp->m, pp->malp, sigmax, pp->kapmax, pp->alpmax);
            grade_h(kapH, g->pbH[f], g->pcH[f], end == 0, np, g->desc.dt, del[a], pp->m, pp->malp, sigmax, pp->kapmax, pp->alpmax);
            // kappa folding, CPML.cpp:361-365, 374-378, 446-450, 459-463
            for (int q = 0; q < 2; ++q) {
                std::vector<double> &se = g->st[wE[a][q]], &sh = g->st[wH[a][q]];
                if (end == 0) {
                    for (int i = 0; i <= np; ++i) se[i] = se[i] / kap[i];
                    for (int i = 0; i < np; ++i) sh[i] = sh[i] / kapH[i];
                } else {
                    const int base = nax[a] - np;
                    for (int i = 0; i < np; ++i) se[base + i] = se[base + i] / kap[i];
                    for (int i = 0; i < np; ++i) sh[base + i] = sh[base + i] / kapH[i];
                }
            }
        }
    }
    g->cpmlE = g->desc.dt / kEps0;  // CPML.cpp:524
    g->cpmlH = g->bH[0];            // CPML.cpp:525
    // coefficient tables: per face bE cE bH cH, each np+1
    std::vector<double> coef;
    for (int f = 0; f < 6; ++f) {
        const int np = pp->npml[f];
        for (std::vector<double> *v : {&g->pbE[f], &g->pcE[f], &g->pbH[f], &g->pcH[f]}) {
            std::vector<double> t = *v;
            t.resize(np + 1, 0.0);
            coef.insert(coef.end(), t.begin(), t.end());
        }
    }
    if ((s = dalloc(g, &g->d_pcoef, coef.size() * g->esz))) return s;
    if ((s = upload_real(g, g->d_pcoef, coef.data(), coef.size()))) return s;
    const Dims &d = g->d;
    for (int f = 0; f < 6; ++f) {
        const int np = pp->npml[f];
        size_t n;
        if (f < 2) n = (size_t)(d.nz + 1) * (d.ny + 1) * psi_xw(np);
        else if (f < 4) n = (size_t)(d.nz + 1) * (np + 1) * d.px;
        else n = (size_t)(np + 1) * (d.ny + 1) * d.px;
        for (int q = 0; q < 4; ++q)
            if ((s = dalloc(g, &g->d_q[f][q], n * g->esz))) return s;
    }
    if ((s = push_stretch(g))) return s;
    g->pml_on = true;
    return CPS_OK;
}

extern "C" cps_status cps_dl_init(cps_grid *g, const cps_dl_params *p)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(p, CPS_E_INVALID, "cps_dl_init: NULL params");
    REQUIRE(!g->dl_on, CPS_E_STATE, "cps_dl_init: already initialised");
    REQUIRE(p->nD >= 0 && p->nL >= 0 && p->nD <= kMaxPoles && p->nL <= kMaxPoles && p->nD + p->nL > 0,
            CPS_E_INVALID, "cps_dl_init: 0..8 Drude and 0..8 Lorentz poles, at least one");
    REQUIRE(p->epsInf > 0, CPS_E_INVALID, "cps_dl_init: epsInf must be positive");
    REQUIRE(p->literal >= 0 && p->literal <= 2, CPS_E_INVALID, "cps_dl_init: literal must be 0, 1 or 2");
    REQUIRE(p->literal != 2 || (p->nD == 1 && p->nL == 0), CPS_E_INVALID,
            "cps_dl_init: the single-pole Drude form (literal 2) takes one Drude pole and no Lorentz pole");
    const double dt = g->desc.dt;
    DlCoef<double> &D = g->dlc;
    memset(&D, 0, sizeof(D));
    D.nD = p->nD; D.nL = p->nL; D.stride = p->nD + 2 * p->nL + 1; D.dt = dt; D.inv2dt = 1.0 / (2.0 * dt);
    // Drude_Lorentz.cpp:65-108
    double temp1 = 0, temp2 = 0;
    for (int q = 0; q < p->nD; ++q) {
        const double omega = p->fD[q] * 2.0 * kPi, gamma = p->gD[q] * 2.0 * kPi;
        D.kappa[q] = (1.0 - gamma * dt / 2.0) / (1.0 + gamma * dt / 2.0);
        D.beta[q] = (omega * omega * kEps0 * dt / 2.0) / (1.0 + gamma * dt / 2.0);
        temp1 = temp1 + D.beta[q];
    }
    for (int q = 0; q < p->nL; ++q) {
        const double omega = p->fL[q] * 2.0 * kPi, delta = p->dL[q] * 2.0 * kPi;
        D.alpha[q] = (2.0 - omega * omega * dt * dt) / (1.0 + delta * dt);
        D.xi[q] = (delta * dt - 1.0) / (1.0 + delta * dt);
        D.gammaL[q] = (kEps0 * p->depsL[q] * omega * omega * dt * dt) / (1.0 + delta * dt);
        temp2 = temp2 + D.gammaL[q];
    }
    if (p->literal == 2) {
        // the single-pole Drude class: Drude.cpp:56-60 in its own order; its
        // C1Drude, C2Drude, C3Drude are this recursion's C1, C3 and C4[0]
        const double b = D.beta[0], kp = D.kappa[0], e = p->epsInf, sg = p->sigma;
        D.C1 = (2 * kEps0 * e - dt * b - sg * dt) / (2 * kEps0 * e + dt * b + sg * dt);
        D.C2 = 0.0;
        D.C3 = (2 * dt) / (2 * kEps0 * e + dt * b + sg * dt);
        D.C4[0] = ((1 + kp) * dt) / (2 * kEps0 * e + dt * b + sg * dt);
    }
    const double den = 2.0 * kEps0 * p->epsInf + p->sigma * dt + dt * temp1 + temp2 / 2.0;
    // literal: C1 and C5 as Drude_Lorentz.cpp:96,106; else the values of the
    // ADE discretisation (E^n coefficient with -sigma dt - dt sum(beta), J_L
    // coefficient with the factor dt)
    if (p->literal != 2) {
        if (p->literal) D.C1 = (2.0 * kEps0 * p->epsInf + p->sigma * dt + dt * temp1) / den;
        else D.C1 = (2.0 * kEps0 * p->epsInf - p->sigma * dt - dt * temp1) / den;
        D.C2 = temp2 / 2.0 / den;
        D.C3 = 2.0 * dt / den;
        for (int q = 0; q < p->nD; ++q) D.C4[q] = (1.0 + D.kappa[q]) * dt / den;
        for (int q = 0; q < p->nL; ++q) {
            D.C5[q] = p->literal ? (1.0 + D.alpha[q]) / den : (1.0 + D.alpha[q]) * dt / den;
            D.C6[q] = D.xi[q] * dt / den;
        }
    }
    if ((s = build_list(g, CPS_ID_DISPERSIVE, &g->dl_n, &g->d_dl_cell, &g->d_dl_seg))) return s;
    if ((s = dalloc(g, &g->d_dl_state, (size_t)g->dl_n * 3 * D.stride * g->esz))) return s;
    g->dl_on = true;
    return CPS_OK;
}

extern "C" cps_status cps_drude_init(cps_grid *g, const cps_drude_params *p)
{
    REQUIRE(p, CPS_E_INVALID, "cps_drude_init: NULL params");
    cps_dl_params q;
    memset(&q, 0, sizeof(q));
    q.sigma = p->sigma; q.epsInf = p->epsInf;
    q.nD = 1; q.nL = 0;
    q.fD[0] = p->omegaP_hz; q.gD[0] = p->gamma_hz;
    q.literal = 2;
    return cps_dl_init(g, &q);
}

extern "C" cps_status cps_three_init(cps_grid *g, const cps_three_params *p)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(p, CPS_E_INVALID, "cps_three_init: NULL params");
    REQUIRE(!g->three_on, CPS_E_STATE, "cps_three_init: already initialised");
    REQUIRE(!g->gain_on, CPS_E_STATE, "cps_three_init: the grid already has the four-level gain");
    REQUIRE(p->gain_id >= 0 && p->gain_id <= 255 && p->gain_id != CPS_ID_DISPERSIVE && p->gain_id != CPS_ID_PEC,
            CPS_E_INVALID, "cps_three_init: gain_id must be a plain medium");
    REQUIRE(p->lambda_a > 0 && p->lambda_b > 0 && p->t20 > 0 && p->t21 > 0 && p->t10 > 0 && p->N_0 > 0,
            CPS_E_INVALID, "cps_three_init: wavelengths, lifetimes and N_0 must be positive");
    REQUIRE(p->literal == 0 || p->literal == 1, CPS_E_INVALID, "cps_three_init: literal must be 0 or 1");
    const double dt = g->desc.dt;
    ThreeCoef &K = g->tc;
    // ThreeLevel.cpp:96-119, :208
    const double omega_a = 2.0 * kPi * kC / p->lambda_a, omega_b = 2.0 * kPi * kC / p->lambda_b;
    const double ga = p->gamma_a, gb = p->gamma_b, t20 = p->t20, t21 = p->t21, t10 = p->t10;
    if (p->literal) {
        K.CPa1 = 2 / ((dt * dt + omega_a * omega_a) * (1 / (dt * dt) + ga / (2 * dt)));
        K.CPa2 = (2 / (dt * dt) + 1 / (2 * dt)) / (1 / (dt * dt) + ga / (2 * dt));
        K.CPb1 = 2 / ((dt * dt + omega_b * omega_b) * (1 / (dt * dt) + gb / (2 * dt)));
        K.CPb2 = (2 / (dt * dt) + 1 / (2 * dt)) / (1 / (dt * dt) + gb / (2 * dt));
    } else {
        K.CPa1 = (2 / (dt * dt) - omega_a * omega_a) / (1 / (dt * dt) + ga / (2 * dt));
        K.CPa2 = (ga / (2 * dt) - 1 / (dt * dt)) / (1 / (dt * dt) + ga / (2 * dt));
        K.CPb1 = (2 / (dt * dt) - omega_b * omega_b) / (1 / (dt * dt) + gb / (2 * dt));
        K.CPb2 = (gb / (2 * dt) - 1 / (dt * dt)) / (1 / (dt * dt) + gb / (2 * dt));
    }
    K.CPa3 = (kQe * kQe / kMe) / (1 / (dt * dt) + ga / (2 * dt)) / p->N_0;
    K.CPb3 = (kQe * kQe / kMe) / (1 / (dt * dt) + gb / (2 * dt)) / p->N_0;
    K.CN2N2 = (1.0 / dt - 1.0 / (2.0 * t20) - 1.0 / (2.0 * t21)) / (1.0 / dt + 1.0 / (2.0 * t20) + 1.0 / (2.0 * t21));
    K.CN2E = (1.0 / (2.0 * dt * kHPlanck * omega_a / 2.0 / kPi)) / (1.0 / dt + 1.0 / (2.0 * t20) + 1.0 / (2.0 * t21));
    K.CN1N1 = (1.0 / dt - 1.0 / (2.0 * t10)) / (1.0 / dt + 1.0 / (2.0 * t10));
    K.CN1N2 = (1.0 / (2.0 * t21)) / (1.0 / dt + 1.0 / (2.0 * t10));
    K.CN1E = (1.0 / (2.0 * dt * kHPlanck * omega_b / 2.0 / kPi)) / (1.0 / dt + 1.0 / (2.0 * t10));
    K.CN0N1 = dt / (2.0 * t10);
    K.CN0N2 = dt / (2.0 * t20);
    K.CN0Ea = 1.0 / (2.0 * kHPlanck * omega_a / 2.0 / kPi);
    K.CN0Eb = 1.0 / (2.0 * kHPlanck * omega_b / 2.0 / kPi);
    K.CN0Ebx = p->literal ? K.CN0Ea : K.CN0Eb;
    K.CEP = 1.0 / dt / kEps0;
    g->three_id = p->gain_id;
    g->three_N0 = p->N_0;
    if ((s = build_list(g, p->gain_id, &g->t_n, &g->d_t_cell, &g->d_t_seg))) return s;
    if ((s = dalloc(g, (void **)&g->d_t_state, (size_t)g->t_n * kThreeWords * sizeof(double)))) return s;
    g->three_on = true;
    launch_three_init(three_view(g), p->N_0, g->stream);
    g->launches++;
    CK(cudaGetLastError());
    return CPS_OK;
}

extern "C" cps_status cps_gain_init(cps_grid *g, const cps_gain_params *p)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(p, CPS_E_INVALID, "cps_gain_init: NULL params");
    REQUIRE(!g->gain_on, CPS_E_STATE, "cps_gain_init: already initialised");
    REQUIRE(!g->three_on, CPS_E_STATE, "cps_gain_init: the grid already has the three-level gain");
    REQUIRE(p->gain_id >= 0 && p->gain_id < 256 && p->gain_id != CPS_ID_DISPERSIVE && p->gain_id != CPS_ID_PEC,
            CPS_E_INVALID, "cps_gain_init: gain_id must be a plain medium (not 2 or 4)");
    REQUIRE(p->lambda_a > 0 && p->lambda_b > 0 && p->t30 > 0 && p->t32 > 0 && p->t21 > 0 && p->t10 > 0 && p->N_0 > 0,
            CPS_E_INVALID, "cps_gain_init: wavelengths, lifetimes and N_0 must be positive");
    const double dt = g->desc.dt, dx = g->desc.dx, dy = g->desc.dy;
    GainCoef &G = g->gc;
    // FourLevelLaser.cpp:96-105, 202-209
    const double omega_a = 2.0 * kPi * kC / p->lambda_a, omega_b = 2.0 * kPi * kC / p->lambda_b;
    const double zeta_a = 6.0 * kPi * kEps0 * kC * kC * kC / (omega_a * omega_a * p->t21);
    const double zeta_b = 6.0 * kPi * kEps0 * kC * kC * kC / (omega_b * omega_b * p->t30);
    G.CPa1 = (2.0 - omega_a * omega_a * dt * dt) / (1.0 + p->gamma_a * dt / 2.0);
    G.CPa2 = (p->gamma_a * dt / 2.0 - 1.0) / (1.0 + p->gamma_a * dt / 2.0);
    G.CPa3 = dt * dt * zeta_a / (1.0 + p->gamma_a * dt / 2.0);
    G.CPb1 = (2.0 - omega_b * omega_b * dt * dt) / (1.0 + p->gamma_b * dt / 2.0);
    G.CPb2 = (p->gamma_b * dt / 2.0 - 1.0) / (1.0 + p->gamma_b * dt / 2.0);
    G.CPb3 = dt * dt * zeta_b / (1.0 + p->gamma_b * dt / 2.0);
    G.CEP = 2.0 * p->N_0 * dx * dy * dx / kEps0 / dt;
    G.t30 = p->t30; G.t32 = p->t32; G.t21 = p->t21; G.t10 = p->t10;
    G.t30t32dt = p->t30 * p->t32 * dt; G.t30t32_2 = 2.0 * p->t30 * p->t32; G.t30dt = p->t30 * dt;
    G.t32dt = p->t32 * dt; G.dt_2 = 2.0 / dt; G.homega_bdt = kHPlanck * omega_b * dt / 2.0 / kPi;
    G.t10t21dt = p->t10 * p->t21 * dt; G.t10t21_2 = 2.0 * p->t10 * p->t21; G.t10dt = p->t10 * dt;
    G.t21dt = p->t21 * dt; G.t21_2 = p->t21 / 2.0; G.homega_adt = kHPlanck * omega_a * dt / 2.0 / kPi;
    G.t32t21dt = p->t32 * p->t21 * dt; G.t32t21_2 = 2.0 * p->t32 * p->t21; G.t32_2 = p->t32 / 2.0;
    G.pump_dt = p->pump_rate * dt;
    G.scaleP = g->fp32 ? G.CEP : 1.0;
    G.fa1 = (float)G.CPa1; G.fa2 = (float)G.CPa2; G.fa3 = (float)(G.CPa3 * G.scaleP);
    G.fb1 = (float)G.CPb1; G.fb2 = (float)G.CPb2; G.fb3 = (float)(G.CPb3 * G.scaleP);
    G.r_t30 = 1.0 / G.t30; G.r_t32 = 1.0 / G.t32; G.r_t21 = 1.0 / G.t21; G.r_t10 = 1.0 / G.t10;
    G.r_t21_2 = 1.0 / G.t21_2; G.r_t32_2 = 1.0 / G.t32_2;
    G.r_hwb = 1.0 / G.homega_bdt; G.r_hwa = 1.0 / G.homega_adt;
    G.inv_scale = 1.0 / G.scaleP;
    G.k1a = (float)(dt / (2.0 * p->t21)); G.k1b = (float)(dt / (2.0 * p->t10));
    G.k3a = (float)(dt / (2.0 * p->t32)); G.k3b = (float)(dt / (2.0 * p->t30));
    G.ha = (float)(dt / (2.0 * G.homega_adt) * G.inv_scale); G.hb = (float)(dt / (2.0 * G.homega_bdt) * G.inv_scale);
    G.fpump = (float)G.pump_dt;
    g->gain_id = p->gain_id;
    if ((s = build_list(g, p->gain_id, &g->g_n, &g->d_g_cell, &g->d_g_seg, &g->d_g_segm))) return s;
    if (g->fp32) {
        if ((s = dalloc(g, &g->d_g_state, (size_t)g->elems * kGainPersist * sizeof(float)))) return s;
        if ((s = dalloc(g, &g->d_g_trans, (size_t)gain_state_elems(g->g_n, kGainTrans) * sizeof(float)))) return s;
    } else if ((s = dalloc(g, &g->d_g_state, (size_t)gain_state_elems(g->g_n, kG64Words) * sizeof(double)))) {
        return s;
    }
    if ((s = gain_state_init(g))) return s;
    g->gain_on = true;
    g->tma_by = 0;  // the sweeps' tensor maps now include the gain words
    return CPS_OK;
}

namespace {

// Gaussian-beam profile and delay of one boundary point (TF_SF.cpp:156-166, repeated per face)
void tfsf_point(double x, double y, double z, double kx, double ky, double kz, double kabs, double w0, double z0,
                double zR, double l0, double dt, double *delay, double *profile)
{
    const double r2 = x * x + y * y + z * z;
    double r_dot_k = (x * kx + y * ky + z * kz) / kabs;
    const double rho2 = r2 - r_dot_k * r_dot_k;
    r_dot_k = r_dot_k - z0;
    const double wz = w0 * sqrt(1 + r_dot_k * r_dot_k / (zR * zR));
    *profile = exp(-rho2 / wz / wz);
    *delay = ((x * kx + y * ky + z * kz) / kC - l0) / dt;
}

}  // namespace

extern "C" cps_status cps_tfsf_init(cps_grid *g, const cps_tfsf_params *p)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(p, CPS_E_INVALID, "cps_tfsf_init: NULL params");
    REQUIRE(!g->tfsf_on, CPS_E_STATE, "cps_tfsf_init: already initialised");
    const Dims &d = g->d;
    const double dx = g->desc.dx, dy = g->desc.dy, dz = g->desc.dz, dt = g->desc.dt;
    const int i1 = p->n[0], i2 = d.nx - p->n[1], j1 = p->n[2], j2 = d.ny - p->n[3], k1 = p->n[4], k2 = d.nz - p->n[5];
    REQUIRE(i1 >= 1 && j1 >= 1 && k1 >= 1 && i2 + 1 <= d.nx - 1 && j2 + 1 <= d.ny - 1 && k2 + 1 <= d.nz - 1 &&
                i2 > i1 && j2 > j1 && k2 > k1,
            CPS_E_INVALID, "cps_tfsf_init: TF/SF box must lie inside the grid with one cell to spare");
    REQUIRE(p->Nt >= 1 && p->lambda > 0 && p->w0 > 0, CPS_E_INVALID, "cps_tfsf_init: bad Nt, lambda or w0");
    g->tp = *p;
    const double theta = p->theta_deg * kPi / 180.0, phi = p->phi_deg * kPi / 180.0, psi = p->psi_deg * kPi / 180.0;
    const double E0 = p->E0, eta0 = sqrt(kMu0 / kEps0);
    // Taflove polarisation and direction, TF_SF.cpp:112-122
    const double E0x = E0 * (cos(psi) * sin(phi) - sin(psi) * cos(theta) * cos(phi));
    const double E0y = E0 * (-cos(psi) * cos(phi) - sin(psi) * cos(theta) * sin(phi));
    const double E0z = E0 * sin(psi) * sin(theta);
    const double H0x = E0 / eta0 * (sin(psi) * sin(phi) + cos(psi) * cos(theta) * cos(phi));
    const double H0y = E0 / eta0 * (-sin(psi) * cos(phi) + cos(psi) * cos(theta) * sin(phi));
    const double H0z = -E0 / eta0 * cos(psi) * sin(theta);
    const double kx = sin(theta) * cos(phi), ky = sin(theta) * sin(phi), kz = cos(theta);
    const double kabs = sqrt(kx * kx + ky * ky + kz * kz);
    const int ci[2] = {i1, i2}, cj[2] = {j1, j2}, ck[2] = {k1, k2};
    double l0 = 0;  // earliest corner, TF_SF.cpp:124-138
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                const double v = (kx * (ci[a] - p->i0) * dx + ky * (cj[b] - p->j0) * dy + kz * (ck[c] - p->k0) * dz) / kC;
                if ((a | b | c) == 0 || l0 > v) l0 = v;
            }
    const double zR = kPi * p->w0 * p->w0 / p->lambda;
    const double CE[3] = {dt / (kEps0 * dx), dt / (kEps0 * dy), dt / (kEps0 * dz)};
    const double CH[3] = {dt / (kMu0 * dx), dt / (kMu0 * dy), dt / (kMu0 * dz)};
    // signed coefficients per face and correction (TF_SF.cpp:988-1089, 1201-1300)
    double cE[6][2], cH[6][2];
    cE[kFX1][0] = CE[0] * H0z; cE[kFX1][1] = -(CE[0] * H0y);
    cE[kFX2][0] = -(CE[0] * H0z); cE[kFX2][1] = CE[0] * H0y;
    cE[kFY1][0] = -(CE[1] * H0z); cE[kFY1][1] = CE[1] * H0x;
    cE[kFY2][0] = CE[1] * H0z; cE[kFY2][1] = -(CE[1] * H0x);
    cE[kFZ1][0] = CE[2] * H0y; cE[kFZ1][1] = -(CE[2] * H0x);
    cE[kFZ2][0] = -(CE[2] * H0y); cE[kFZ2][1] = CE[2] * H0x;
    cH[kFX1][0] = CH[0] * E0y; cH[kFX1][1] = -(CH[0] * E0z);
    cH[kFX2][0] = -(CH[0] * E0y); cH[kFX2][1] = CH[0] * E0z;
    cH[kFY1][0] = -(CH[1] * E0x); cH[kFY1][1] = CH[1] * E0z;
    cH[kFY2][0] = CH[1] * E0x; cH[kFY2][1] = -(CH[1] * E0z);
    cH[kFZ1][0] = CH[2] * E0x; cH[kFZ1][1] = -(CH[2] * E0y);
    cH[kFZ2][0] = -(CH[2] * E0x); cH[kFZ2][1] = CH[2] * E0y;
    // components of correction 1/2: x faces (Ey|Hz, Ez|Hy), y faces (Ex|Hz, Ez|Hx), z faces (Ex|Hy, Ey|Hx)
    const int compE[3][2] = {{CPS_EY, CPS_EZ}, {CPS_EX, CPS_EZ}, {CPS_EX, CPS_EY}};
    const int compH[3][2] = {{CPS_HZ, CPS_HY}, {CPS_HZ, CPS_HX}, {CPS_HY, CPS_HX}};
    const int order[6] = {kFY1, kFY2, kFX1, kFX2, kFZ1, kFZ2};
    struct Item {
        int64_t key;  // idx * 8 + comp
        InjContrib c;
    };
    for (int isH = 0; isH < 2; ++isH) {
        // the twelve (face, component) strips are generated in parallel and
        // joined in the reference's face order
        std::vector<std::vector<Item>> strips(12);
        parallel_for(12, [&](int t0, int t1) {
            for (int t = t0; t < t1; ++t) {
                const int oi = t / 2, which = t % 2;
                std::vector<Item> &items = strips[t];
                const int f = order[oi], ax = f / 2, far = f & 1;
                int u1, u2, v1, v2;
                if (ax == 0) { u1 = j1; u2 = j2; v1 = k1; v2 = k2; }
                else if (ax == 1) { u1 = i1; u2 = i2; v1 = k1; v2 = k2; }
                else { u1 = i1; u2 = i2; v1 = j1; v2 = j2; }
                {
                    // E1 covers [u1,u2) x [v1,v2], E2 [u1,u2] x [v1,v2); the x-face H
                    // strips add nothing in the reference (TF_SF.cpp:1244-1251,
                    // 1260-1267 read unset point members), so x-face H covers [u1,u2) x [v1,v2)
                    int ue = which == 0 ? u2 - 1 : u2, ve = which == 0 ? v2 : v2 - 1;
                    if (isH && ax == 0) { ue = u2 - 1; ve = v2 - 1; }
                    const int comp = isH ? compH[ax][which] : compE[ax][which];
                    const double coef = isH ? cH[f][which] : cE[f][which];
                    for (int u = u1; u <= ue; ++u)
                        for (int v = v1; v <= ve; ++v) {
                            int i, j, k;
                            double x, y, z;
                            if (ax == 0) {
                                i = far ? i2 : i1; j = u; k = v;
                                x = isH ? dx * (i - p->i0) : dx * (far ? (i - p->i0 + 0.5) : (i - p->i0 - 0.5));
                                y = dy * (j - p->j0); z = dz * (k - p->k0);
                                if (isH) i += far ? 1 : -1;
                            } else if (ax == 1) {
                                i = u; j = far ? j2 : j1; k = v;
                                x = dx * (i - p->i0);
                                y = isH ? dy * (j - p->j0) : dy * (far ? (j - p->j0 + 0.5) : (j - p->j0 - 0.5));
                                z = dz * (k - p->k0);
                                if (isH) j += far ? 1 : -1;
                            } else {
                                i = u; j = v; k = far ? k2 : k1;
                                x = dx * (i - p->i0); y = dy * (j - p->j0);
                                z = isH ? dz * (k - p->k0) : dz * (far ? (k - p->k0 + 0.5) : (k - p->k0 - 0.5));
                                if (isH) k += far ? 1 : -1;
                            }
                            InjContrib c;
                            tfsf_point(x, y, z, kx, ky, kz, kabs, p->w0, p->z0, zR, l0, dt, &c.delay, &c.profile);
                            c.coef = coef;
                            c.face = f;
                            c.pad = 0;
                            items.push_back({d.idx(i, j, k) * 8 + comp, c});
                        }
                }
            }
        });
        // targets in device order, so neighbouring threads touch neighbouring
        // cells, each with its contributions in the reference's face order
        std::vector<InjTarget> tg;
        std::vector<InjContrib> ct;
        tfsf_assemble(strips, d.nz + 1, d.pxy, [](int n, auto f) { parallel_for(n, f); }, tg, ct);
        const int side = isH;  // d_tg[0] = E targets, d_tg[1] = H targets
        g->ntg[side] = (int)tg.size();
        if ((s = dalloc(g, (void **)&g->d_tg[side], tg.size() * sizeof(InjTarget)))) return s;
        if ((s = dalloc(g, (void **)&g->d_ct[side], ct.size() * sizeof(InjContrib)))) return s;
        if ((s = upload_raw(g, g->d_tg[side], tg.data(), tg.size() * sizeof(InjTarget)))) return s;
        if ((s = upload_raw(g, g->d_ct[side], ct.data(), ct.size() * sizeof(InjContrib)))) return s;
    }
    // incident tables, TF_SF.cpp:898-955
    const int Nt = p->Nt;
    g->einc.assign(Nt + 1, 0.0);
    g->hinc.assign(Nt + 1, 0.0);
    const double nu = kC / p->lambda, T = 1.0 / nu;
    const int nT = (int)(T / dt);
    const double dnu = kC / (p->lambda - p->dlambda / 2.0) - kC / (p->lambda + p->dlambda / 2.0);
    const double domega = 2.0 * kPi * dnu;
    const double sig = domega * domega / (16 * log(2));
    if (p->cwmode) {
        const int nd = 5 * nT;
        for (int n = 0; n < nd && n <= Nt; ++n) {
            g->einc[n] = exp(-((n * dt) - 5.0 * T) * ((n * dt) - 5 * T) / (4.0 * T * T)) * sin(2.0 * kPi * nu * (n * dt));
            g->hinc[n] = exp(-((n * dt + dt / 2.0) - 5.0 * T) * ((n * dt + dt / 2.0) - 5 * T) / (4.0 * T * T)) * sin(2.0 * kPi * nu * (n * dt + dt / 2.0));
        }
        for (int n = nd; n <= Nt; ++n) {
            g->einc[n] = sin(2.0 * kPi * nu * (n * dt));
            g->hinc[n] = sin(2.0 * kPi * nu * (n * dt + dt / 2.0));
        }
    } else {
        const double t0 = 5 * T;
        for (int n = 0; n <= Nt; ++n) {
            g->einc[n] = exp(-sig * ((double)n * dt - t0) * ((double)n * dt - t0)) * sin(2.0 * kPi * nu * ((double)n * dt - t0));
            g->hinc[n] = exp(-sig * ((double)n * dt + dt / 2.0 - t0) * ((double)n * dt + dt / 2.0 - t0)) * sin(2.0 * kPi * nu * ((double)n * dt + dt / 2.0 - t0));
        }
    }
    if ((s = dalloc(g, &g->d_einc, (Nt + 2) * g->esz)) || (s = dalloc(g, &g->d_hinc, (Nt + 2) * g->esz))) return s;
    if ((s = upload_real(g, g->d_einc, g->einc.data(), Nt + 1)) || (s = upload_real(g, g->d_hinc, g->hinc.data(), Nt + 1)))
        return s;
    g->tfsf_on = true;
    return CPS_OK;
}

extern "C" cps_status cps_tfsf_set_tables(cps_grid *g, int32_t n, const double *einc, const double *hinc)
{
    REQUIRE(g && einc && hinc, CPS_E_INVALID, "NULL argument");
    FLUSH_RECORDED(g);
    REQUIRE(g->tfsf_on, CPS_E_STATE, "TF/SF is not initialised");
    REQUIRE(n == g->tp.Nt + 1, CPS_E_INVALID, "tables must hold Nt + 1 values");
    g->einc.assign(einc, einc + n);
    g->hinc.assign(hinc, hinc + n);
    cps_status s = upload_real(g, g->d_einc, einc, n);
    return s ? s : upload_real(g, g->d_hinc, hinc, n);
}

extern "C" cps_status cps_tfsf_get_tables(const cps_grid *g, int32_t n, double *einc, double *hinc)
{
    REQUIRE(g && einc && hinc, CPS_E_INVALID, "NULL argument");
    REQUIRE(g->tfsf_on && n == g->tp.Nt + 1, CPS_E_INVALID, "TF/SF not initialised or wrong length");
    memcpy(einc, g->einc.data(), n * sizeof(double));
    memcpy(hinc, g->hinc.data(), n * sizeof(double));
    return CPS_OK;
}

extern "C" cps_status cps_source_add(cps_grid *g, int32_t comp, int32_t i, int32_t j, int32_t k, const double *wave,
                                     int32_t nwave)
{
    REQUIRE(g && wave, CPS_E_INVALID, "cps_source_add: NULL argument");
    FLUSH_RECORDED(g);
    REQUIRE(comp >= 0 && comp < 6 && nwave >= 1, CPS_E_INVALID, "cps_source_add: bad component or wave length");
    REQUIRE(i >= 0 && j >= 0 && k >= 0 && i <= g->d.nx && j <= g->d.ny && k <= g->d.nz, CPS_E_INVALID,
            "cps_source_add: point outside the grid");
    Src s;
    s.comp = comp; s.idx = g->d.idx(i, j, k); s.wave.assign(wave, wave + nwave);
    g->src.push_back(s);
    g->src_dirty = true;
    return CPS_OK;
}

// ================================================================== ports

extern "C" cps_status cps_port_add(cps_grid *g, int32_t npoints, const int32_t *ijk, int32_t *port_id)
{
    REQUIRE(g && ijk && port_id, CPS_E_INVALID, "cps_port_add: NULL argument");
    REQUIRE(npoints >= 1, CPS_E_INVALID, "cps_port_add: a port needs at least one point");
    PortState P;
    P.npts = npoints;
    P.ijk.assign(ijk, ijk + 3 * (size_t)npoints);
    std::vector<int64_t> idx(npoints);
    for (int q = 0; q < npoints; ++q) {
        const int i = ijk[3 * q], j = ijk[3 * q + 1], k = ijk[3 * q + 2];
        REQUIRE(i >= 0 && j >= 0 && k >= 0 && i <= g->d.nx && j <= g->d.ny && k <= g->d.nz, CPS_E_INVALID,
                "cps_port_add: point outside the grid");
        idx[q] = g->d.idx(i, j, k);
    }
    cps_status s;
    if ((s = dalloc(g, (void **)&P.d_idx, npoints * sizeof(int64_t)))) return s;
    if ((s = upload_raw(g, P.d_idx, idx.data(), npoints * sizeof(int64_t)))) return s;
    P.slots = 1;
    if ((s = dalloc(g, &P.d_ring, (size_t)P.slots * 6 * npoints * g->esz))) return s;
    g->ports.push_back(P);
    *port_id = (int32_t)g->ports.size() - 1;
    return CPS_OK;
}

extern "C" cps_status cps_port_set_dft(cps_grid *g, int32_t port_id, int32_t nfreq, const double *freq_hz,
                                       uint32_t comp_mask)
{
    REQUIRE(g && freq_hz, CPS_E_INVALID, "cps_port_set_dft: NULL argument");
    REQUIRE(port_id >= 0 && port_id < (int)g->ports.size(), CPS_E_NOTFOUND, "cps_port_set_dft: no such port");
    FLUSH_RECORDED(g);
    REQUIRE(nfreq >= 1 && nfreq <= 4096 && (comp_mask & 63u), CPS_E_INVALID, "cps_port_set_dft: 1..4096 frequencies and a component");
    PortState &P = g->ports[port_id];
    REQUIRE(P.nfreq == 0, CPS_E_STATE, "cps_port_set_dft: DFT already configured");
    P.nfreq = nfreq;
    P.mask = comp_mask & 63u;
    P.ncomp = 0;
    for (int c = 0; c < 6; ++c)
        if (P.mask & (1u << c)) P.comps[P.ncomp++] = c;
    std::vector<double> om(nfreq);
    for (int f = 0; f < nfreq; ++f) om[f] = 2.0 * kPi * freq_hz[f];
    cps_status s;
    if ((s = dalloc(g, (void **)&P.d_omega, nfreq * sizeof(double)))) return s;
    if ((s = upload_raw(g, P.d_omega, om.data(), nfreq * sizeof(double)))) return s;
    if ((s = dalloc(g, (void **)&P.d_comps, 6 * sizeof(int32_t)))) return s;
    if ((s = upload_raw(g, P.d_comps, P.comps, 6 * sizeof(int32_t)))) return s;
    if ((s = dalloc(g, (void **)&P.d_acc, (size_t)P.ncomp * nfreq * 2 * P.npts * sizeof(double)))) return s;
    if ((s = dalloc(g, (void **)&P.d_flux, nfreq * sizeof(double)))) return s;
    // a ring of 64 samples between contractions
    dfree(g, P.d_ring);
    P.slots = 64;
    P.fill = 0;
    P.last_slot = -1;
    if ((s = dalloc(g, &P.d_ring, (size_t)P.slots * 6 * P.npts * g->esz))) return s;
    return CPS_OK;
}

namespace {
template <typename T>
cps_status port_read_T(cps_grid *g, PortState &P, double *out)
{
    std::vector<T> tmp((size_t)6 * P.npts, T(0));
    if (P.last_slot >= 0)
        CK(cudaMemcpyAsync(tmp.data(), (T *)P.d_ring + (int64_t)P.last_slot * 6 * P.npts, tmp.size() * sizeof(T),
                           cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    for (int p = 0; p < P.npts; ++p)
        for (int c = 0; c < 6; ++c) out[p * 6 + c] = (double)tmp[(size_t)c * P.npts + p];
    return CPS_OK;
}
}  // namespace

extern "C" cps_status cps_port_read(cps_grid *g, int32_t port_id, double *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "cps_port_read: NULL argument");
    REQUIRE(port_id >= 0 && port_id < (int)g->ports.size(), CPS_E_NOTFOUND, "cps_port_read: no such port");
    FLUSH_RECORDED(g);
    PortState &P = g->ports[port_id];
    return g->fp32 ? port_read_T<float>(g, P, out) : port_read_T<double>(g, P, out);
}

extern "C" cps_status cps_port_dft_read(cps_grid *g, int32_t port_id, double *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "cps_port_dft_read: NULL argument");
    REQUIRE(port_id >= 0 && port_id < (int)g->ports.size(), CPS_E_NOTFOUND, "cps_port_dft_read: no such port");
    FLUSH_RECORDED(g);
    PortState &P = g->ports[port_id];
    REQUIRE(P.nfreq > 0, CPS_E_STATE, "cps_port_dft_read: no DFT configured on this port");
    cps_status s = flush_dft(g, P);
    if (s) return s;
    CK(cudaMemcpyAsync(out, P.d_acc, (size_t)P.ncomp * P.nfreq * 2 * P.npts * sizeof(double), cudaMemcpyDeviceToHost,
                       g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

extern "C" cps_status cps_port_flux(cps_grid *g, int32_t port_id, char normal, double *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "cps_port_flux: NULL argument");
    REQUIRE(port_id >= 0 && port_id < (int)g->ports.size(), CPS_E_NOTFOUND, "cps_port_flux: no such port");
    FLUSH_RECORDED(g);
    PortState &P = g->ports[port_id];
    REQUIRE(P.nfreq > 0, CPS_E_STATE, "cps_port_flux: no DFT configured on this port");
    int a, b, c, e;  // flux = Re(E_a H_b* - E_c H_e*)
    double dA;
    if (normal == 'x') { a = CPS_EY; b = CPS_HZ; c = CPS_EZ; e = CPS_HY; dA = g->desc.dy * g->desc.dz; }
    else if (normal == 'y') { a = CPS_EZ; b = CPS_HX; c = CPS_EX; e = CPS_HZ; dA = g->desc.dx * g->desc.dz; }
    else if (normal == 'z') { a = CPS_EX; b = CPS_HY; c = CPS_EY; e = CPS_HX; dA = g->desc.dx * g->desc.dy; }
    else REQUIRE(false, CPS_E_INVALID, "cps_port_flux: normal must be 'x', 'y' or 'z'");
    int sel[4], want[4] = {a, b, c, e};
    for (int q = 0; q < 4; ++q) {
        sel[q] = -1;
        for (int ci = 0; ci < P.ncomp; ++ci)
            if (P.comps[ci] == want[q]) sel[q] = ci;
        REQUIRE(sel[q] >= 0, CPS_E_STATE, "cps_port_flux: the DFT lacks a tangential component");
    }
    cps_status s = flush_dft(g, P);
    if (s) return s;
    // the port's own result buffer, allocated with its accumulators
    launch_port_flux(P.d_acc, P.npts, P.nfreq, P.ncomp, sel, dA, P.d_flux, g->stream);
    const cudaError_t e0 = cudaGetLastError();
    REQUIRE(e0 == cudaSuccess, CPS_E_CUDA, std::string("cps_port_flux: launch failed: ") + cudaGetErrorString(e0));
    g->launches++;
    cudaError_t e1 = cudaMemcpyAsync(out, P.d_flux, P.nfreq * sizeof(double), cudaMemcpyDeviceToHost, g->stream);
    cudaError_t e2 = cudaStreamSynchronize(g->stream);
    REQUIRE(e1 == cudaSuccess && e2 == cudaSuccess, CPS_E_CUDA, "cps_port_flux: copy failed");
    return CPS_OK;
}

// ================================================================== steps

extern "C" cps_status cps_grid_set_step(cps_grid *g, int64_t n)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    g->step = n;
    return CPS_OK;
}

extern "C" cps_status cps_grid_get_step(const cps_grid *g, int64_t *n)
{
    REQUIRE(g && n, CPS_E_INVALID, "NULL argument");
    *n = g->step;
    return CPS_OK;
}

namespace {
// grids at or above this size step the fused path as chunks of a one-grid
// batch: the batch launches their sweeps per grid inside CUDA-graph-replayed
// chunks and the rest of the step in batched launches, with results equal to
// the direct launches
constexpr int64_t kSoloMinCells = 4 << 20;

bool solo_eligible(const cps_grid *g)
{
    return g->chunked && g->timing_stride == 0 && g->sweep_mode == 0 && !g->three_on &&
           (g->shape.by == 4 || g->shape.by == 8) && g->d.px >= 64 && g->d.ny >= 8 && g->d.nz >= 2 &&
           (int64_t)g->d.nx * g->d.ny * g->d.nz >= kSoloMinCells;
}

cps_status solo_step(cps_grid *g, int32_t nsteps)
{
    cps_status s;
    if (!g->solo) {
        if ((s = cps_batch_create(g->desc.precision, &g->solo))) return s;
        if ((s = cps_batch_add(g->solo, g))) {
            cps_batch_destroy(g->solo);
            g->solo = nullptr;
            return s;
        }
    }
    int32_t rows = 0, planes = 0, pers = 0;
    if ((s = cps_batch_get_tile(g->solo, &rows, &planes, &pers))) return s;
    if ((rows != g->shape.by || planes != g->shape.kc || pers != 0) &&
        (s = cps_batch_set_tile(g->solo, g->shape.by, g->shape.kc, 0)))
        return s;
    batch_set_h_planes(g->solo, g->shape.kch, g->shape.kcg);
    int64_t l0 = 0, l1 = 0;
    cps_batch_launch_count(g->solo, &l0);
    s = cps_batch_step(g->solo, nsteps);
    cps_batch_launch_count(g->solo, &l1);
    g->launches += l1 - l0;
    return s;
}
}  // namespace

extern "C" cps_status cps_grid_set_chunked(cps_grid *g, int32_t on)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    g->chunked = on != 0;
    return CPS_OK;
}

extern "C" cps_status cps_step(cps_grid *g, int32_t nsteps, int32_t path)
{
    cps_status s = need_setup(g);
    if (s) return s;
    FLUSH_RECORDED(g);
    REQUIRE(nsteps >= 0, CPS_E_INVALID, "cps_step: negative step count");
    REQUIRE(path == CPS_PATH_PLAIN || path == CPS_PATH_FUSED || path == CPS_PATH_ONEPASS, CPS_E_INVALID,
            "cps_step: unknown path");
    CK(cudaSetDevice(g->desc.device));
    if (path == CPS_PATH_FUSED && nsteps > 0 && solo_eligible(g)) return solo_step(g, nsteps);
    return g->fp32 ? step_T<float>(g, nsteps, path) : step_T<double>(g, nsteps, path);
}

// ============================================================ op recorder
//
// The reference's main loop calls one routine per physics term each step
// (main.cpp:264-330).  Each cps_op_* entry point runs that routine alone; with
// recording on (cps_grid_set_record) the calls are queued instead, and a queue
// that forms one whole step in an order the fused sweeps reproduce runs as one
// fused H sweep and one fused E sweep.  The order rules: H_BULK first; TF/SF-H
// and H_PML (additive to H) in any order before E_BULK; DL, then gain P, E, N,
// after E_BULK; TF/SF-E, sources and E_PML (additive to E) in any order after
// the dispersive terms; port samples last, each port once.  The terms the
// sweeps absorb (PML, DL, gain) appear exactly once when initialised; TF/SF and
// sources run as recorded, with their own step index, face mask and count.
// Anything else is replayed call by call, in order.

namespace cps {
namespace {

bool absorbed_kind(int k)
{
    return k == kOpHPml || k == kOpEPml || k == kOpDl || (k >= kOpGainP && k <= kOpGainN) ||
           (k >= kOpThreeP && k <= kOpThreeN);
}

// Whether `ops` is a prefix (full = false) or a whole step (full = true) that
// the fused sweeps reproduce.
bool fusable(const cps_grid *g, const std::vector<RecOp> &ops, bool full)
{
    int phase = 0;  // 0 start, 1 H terms, 2 dispersive E terms, 3 additive E terms, 4 ports
    int hpml = 0, epml = 0, dl = 0, gain = 0, three = 0;
    std::vector<char> seen(g->ports.size(), 0);
    const int want_dl = g->dl_on ? 1 : 0, want_gain = g->gain_on ? 3 : 0, want_three = g->three_on ? 3 : 0;
    for (const RecOp &o : ops) {
        switch (o.kind) {
        case kOpHBulk:
            if (phase != 0) return false;
            phase = 1;
            break;
        case kOpHPml:
            if (phase != 1 || hpml++) return false;
            break;
        case kOpTfsfH:
            if (phase != 1) return false;
            break;
        case kOpEBulk:
            if (phase != 1) return false;
            phase = 2;
            break;
        case kOpDl:
            if (phase != 2 || dl++ || gain) return false;
            break;
        case kOpGainP:
        case kOpGainE:
        case kOpGainN:
            if (phase != 2 || gain != o.kind - kOpGainP) return false;
            ++gain;
            break;
        case kOpThreeP:
        case kOpThreeE:
        case kOpThreeN:
            if (phase != 2 || three != o.kind - kOpThreeP) return false;
            ++three;
            break;
        case kOpTfsfE:
        case kOpSrc:
        case kOpEPml:
            if (phase == 2) {
                if (dl != want_dl || gain != want_gain || three != want_three) return false;
                phase = 3;
            }
            if (phase != 3) return false;
            if (o.kind == kOpEPml && epml++) return false;
            break;
        case kOpPort:
            if (phase < 2) return false;
            if (phase == 2 && (dl != want_dl || gain != want_gain || three != want_three)) return false;
            phase = 4;
            if (seen[o.port]++) return false;
            break;
        default:
            return false;
        }
    }
    if (!full) return true;
    const int want_pml = g->pml_on ? 1 : 0;
    return phase >= 2 && hpml == want_pml && epml == want_pml && dl == want_dl && gain == want_gain &&
           three == want_three;
}

// one routine alone on the grid's stream
template <typename T>
cps_status run_op_T(cps_grid *g, const RecOp &o)
{
    const FieldView<T> f = field_view<T>(g);
    switch (o.kind) {
    case kOpHBulk: launch_h_bulk<T>(f, g->stream); g->launches++; break;
    case kOpEBulk: launch_e_bulk<T>(f, g->stream); g->launches++; break;
    case kOpHPml: launch_h_pml<T>(f, pml_view<T>(g), g->stream); g->launches++; break;
    case kOpEPml: launch_e_pml<T>(f, pml_view<T>(g), g->stream); g->launches++; break;
    case kOpDl: launch_dl<T>(f, dl_view<T>(g), g->stream); g->launches++; break;
    case kOpGainP:
    case kOpGainE:
    case kOpGainN: launch_gain<T>(f, gain_view<T>(g), o.kind - kOpGainP, g->stream); g->launches++; break;
    case kOpThreeP:
    case kOpThreeE:
    case kOpThreeN: launch_three<T>(f, three_view(g), o.kind - kOpThreeP, g->stream); g->launches++; break;
    case kOpTfsfH: op_inject<T>(g, 1, (double)o.n, o.mask); break;
    case kOpTfsfE: op_inject<T>(g, 0, (double)o.n, o.mask); break;
    case kOpSrc: {
        cps_status s = ensure_sources(g);
        if (s) return s;
        op_sources<T>(g, o.n);
        break;
    }
    case kOpPort: {
        cps_status s = op_port<T>(g, g->ports[o.port], o.n);
        if (s) return s;
        break;
    }
    default: break;
    }
    cudaError_t e = cudaGetLastError();
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return CPS_OK;
}

// one whole recorded step as the fused H and E sweeps (the step of step_T's
// fused path, with the recorded TF/SF, source and port calls)
template <typename T>
cps_status run_fused_T(cps_grid *g, const std::vector<RecOp> &ops)
{
    cps_status s = ensure_sources(g);
    if (s) return s;
    const bool use_tma = g->sweep_mode == 0 && (g->shape.by == 4 || g->shape.by == 8) && g->d.px >= 64 &&
                         g->d.ny + 1 >= g->shape.by + 1;
    if (use_tma && (s = ensure_tma(g))) return s;
    const FieldView<T> f = field_view<T>(g);
    const PmlView<T> p = pml_view<T>(g);
    std::vector<PortState *> ports;
    std::vector<int64_t> port_n;
    for (const RecOp &o : ops) {
        switch (o.kind) {
        case kOpHBulk:
            if (use_tma) g->launches += launch_h_tma<T>(g->tma, f, p, g->shape, g->d_err, g->stream);
            else launch_h_fused<T>(f, p, g->shape, g->stream), g->launches++;
            break;
        case kOpEBulk:
            if (use_tma)
                g->launches += launch_e_tma<T>(g->tma, f, p, dl_view<T>(g), gain_view<T>(g), g->shape, g->d_err, g->stream,
                                             &g->lane);
            else launch_e_fused<T>(f, p, dl_view<T>(g), gain_view<T>(g), g->shape, g->stream), g->launches++;
            if (g->three_on) {
                launch_three<T>(f, three_view(g), 3, g->stream);
                g->launches++;
            }
            break;
        case kOpTfsfH: op_inject<T>(g, 1, (double)o.n, o.mask); break;
        case kOpTfsfE: op_inject<T>(g, 0, (double)o.n, o.mask); break;
        case kOpSrc: op_sources<T>(g, o.n); break;
        case kOpPort:
            ports.push_back(&g->ports[o.port]);
            port_n.push_back(o.n);
            break;
        default: break;  // absorbed by the sweeps
        }
    }
    if (!ports.empty() && (s = op_ports<T>(g, ports.data(), (int)ports.size(), 0, port_n.data()))) return s;
    cudaError_t e = cudaGetLastError();
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
    return CPS_OK;
}

// queue one call; a call that cannot continue a fusable step flushes the queue
cps_status record_op(cps_grid *g, const RecOp &o)
{
    if (o.kind == kOpHBulk && !g->pending.empty()) {
        cps_status s = flush_recorded(g);
        if (s) return s;
    }
    g->pending.push_back(o);
    return fusable(g, g->pending, false) ? CPS_OK : flush_recorded(g);
}

cps_status submit_op(cps_grid *g, const RecOp &o)
{
    cps_status s = need_setup(g);
    if (s) return s;
    if (g->record) return record_op(g, o);
    return g->fp32 ? run_op_T<float>(g, o) : run_op_T<double>(g, o);
}

}  // namespace

cps_status flush_recorded(cps_grid *g)
{
    if (g->pending.empty()) return CPS_OK;
    std::vector<RecOp> ops;
    ops.swap(g->pending);
    if (fusable(g, ops, true)) {
        g->fused_steps++;
        return g->fp32 ? run_fused_T<float>(g, ops) : run_fused_T<double>(g, ops);
    }
    for (const RecOp &o : ops) {
        g->replayed_ops++;
        cps_status s = g->fp32 ? run_op_T<float>(g, o) : run_op_T<double>(g, o);
        if (s) return s;
    }
    return CPS_OK;
}

}  // namespace cps

extern "C" cps_status cps_grid_set_record(cps_grid *g, int32_t on)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    if (!on) {
        cps_status s = flush_recorded(g);
        g->record = false;
        return s;
    }
    g->record = true;
    return CPS_OK;
}

extern "C" cps_status cps_grid_record_stats(const cps_grid *g, int64_t *fused_steps, int64_t *replayed_calls,
                                            int32_t *pending)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    if (fused_steps) *fused_steps = g->fused_steps;
    if (replayed_calls) *replayed_calls = g->replayed_ops;
    if (pending) *pending = (int32_t)g->pending.size();
    return CPS_OK;
}

extern "C" cps_status cps_op_h_bulk(cps_grid *g) { return submit_op(g, {kOpHBulk, 0, 0, 0}); }
extern "C" cps_status cps_op_e_bulk(cps_grid *g) { return submit_op(g, {kOpEBulk, 0, 0, 0}); }
extern "C" cps_status cps_op_h_pml(cps_grid *g)
{
    if (g && !g->pml_on) { set_error("CPML not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpHPml, 0, 0, 0});
}
extern "C" cps_status cps_op_e_pml(cps_grid *g)
{
    if (g && !g->pml_on) { set_error("CPML not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpEPml, 0, 0, 0});
}
extern "C" cps_status cps_op_dl(cps_grid *g)
{
    if (g && !g->dl_on) { set_error("Drude-Lorentz not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpDl, 0, 0, 0});
}
extern "C" cps_status cps_op_gain_polarization(cps_grid *g)
{
    if (g && !g->gain_on) { set_error("gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpGainP, 0, 0, 0});
}
extern "C" cps_status cps_op_gain_efield(cps_grid *g)
{
    if (g && !g->gain_on) { set_error("gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpGainE, 0, 0, 0});
}
extern "C" cps_status cps_op_gain_populations(cps_grid *g)
{
    if (g && !g->gain_on) { set_error("gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpGainN, 0, 0, 0});
}
extern "C" cps_status cps_op_tfsf_h(cps_grid *g, int32_t n, uint32_t face_mask)
{
    if (g && !g->tfsf_on) { set_error("TF/SF not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpTfsfH, n, 0, face_mask});
}
extern "C" cps_status cps_op_tfsf_e(cps_grid *g, int32_t n, uint32_t face_mask)
{
    if (g && !g->tfsf_on) { set_error("TF/SF not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpTfsfE, n, 0, face_mask});
}
extern "C" cps_status cps_op_sources(cps_grid *g, int32_t n) { return submit_op(g, {kOpSrc, n, 0, 0}); }
extern "C" cps_status cps_op_three_polarization(cps_grid *g)
{
    if (g && !g->three_on) { set_error("three-level gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpThreeP, 0, 0, 0});
}
extern "C" cps_status cps_op_three_efield(cps_grid *g)
{
    if (g && !g->three_on) { set_error("three-level gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpThreeE, 0, 0, 0});
}
extern "C" cps_status cps_op_three_populations(cps_grid *g)
{
    if (g && !g->three_on) { set_error("three-level gain not initialised"); return CPS_E_STATE; }
    return submit_op(g, {kOpThreeN, 0, 0, 0});
}
extern "C" cps_status cps_op_port_sample(cps_grid *g, int32_t port_id, int32_t n)
{
    if (g && (port_id < 0 || port_id >= (int)g->ports.size())) { set_error("no such port"); return CPS_E_NOTFOUND; }
    return submit_op(g, {kOpPort, n, port_id, 0});
}

// ============================================================ field access

namespace {
template <typename T>
cps_status download_T(cps_grid *g, int comp, double *out)
{
    const size_t n = (size_t)(g->d.nx + 1) * (g->d.ny + 1) * (g->d.nz + 1);
    if (!g->d_conv) {
        cps_status s = dalloc(g, (void **)&g->d_conv, n * sizeof(double));
        if (s) return s;
    }
    launch_from_device_layout<T>((const T *)g->F[comp], g->d_conv, g->d, g->stream);
    CK(cudaMemcpyAsync(out, g->d_conv, n * sizeof(double), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}
template <typename T>
cps_status upload_field_T(cps_grid *g, int comp, const double *in)
{
    const size_t n = (size_t)(g->d.nx + 1) * (g->d.ny + 1) * (g->d.nz + 1);
    if (!g->d_conv) {
        cps_status s = dalloc(g, (void **)&g->d_conv, n * sizeof(double));
        if (s) return s;
    }
    CK(cudaMemcpyAsync(g->d_conv, in, n * sizeof(double), cudaMemcpyHostToDevice, g->stream));
    launch_to_device_layout<T>(g->d_conv, (T *)g->F[comp], g->d, g->stream);
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}
}  // namespace

extern "C" cps_status cps_field_download(cps_grid *g, int32_t comp, double *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "cps_field_download: NULL argument");
    REQUIRE(comp >= 0 && comp < 6, CPS_E_INVALID, "cps_field_download: component 0..5");
    FLUSH_RECORDED(g);
    return g->fp32 ? download_T<float>(g, comp, out) : download_T<double>(g, comp, out);
}

extern "C" cps_status cps_field_upload(cps_grid *g, int32_t comp, const double *in)
{
    REQUIRE(g && in, CPS_E_INVALID, "cps_field_upload: NULL argument");
    REQUIRE(comp >= 0 && comp < 6, CPS_E_INVALID, "cps_field_upload: component 0..5");
    FLUSH_RECORDED(g);
    return g->fp32 ? upload_field_T<float>(g, comp, in) : upload_field_T<double>(g, comp, in);
}

extern "C" cps_status cps_field_download_f32(cps_grid *g, int32_t comp, float *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "NULL argument");
    REQUIRE(comp >= 0 && comp < 6, CPS_E_INVALID, "component 0..5");
    const size_t n = (size_t)(g->d.nx + 1) * (g->d.ny + 1) * (g->d.nz + 1);
    std::vector<double> tmp(n);
    cps_status s = cps_field_download(g, comp, tmp.data());
    if (s) return s;
    for (size_t q = 0; q < n; ++q) out[q] = (float)tmp[q];
    return CPS_OK;
}

extern "C" cps_status cps_grid_reset(cps_grid *g, int64_t n0)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    FLUSH_RECORDED(g);
    for (int c = 0; c < 6; ++c) CK(cudaMemsetAsync(g->F[c], 0, (size_t)g->elems * g->esz, g->stream));
    if (g->pml_on) {
        const Dims &d = g->d;
        for (int f = 0; f < 6; ++f) {
            const int np = g->pml.npml[f];
            size_t n;
            if (f < 2) n = (size_t)(d.nz + 1) * (d.ny + 1) * psi_xw(np);
            else if (f < 4) n = (size_t)(d.nz + 1) * (np + 1) * d.px;
            else n = (size_t)(np + 1) * (d.ny + 1) * d.px;
            for (int q = 0; q < 4; ++q) CK(cudaMemsetAsync(g->d_q[f][q], 0, n * g->esz, g->stream));
        }
    }
    if (g->dl_on) CK(cudaMemsetAsync(g->d_dl_state, 0, (size_t)g->dl_n * 3 * g->dlc.stride * g->esz, g->stream));
    if (g->gain_on) {
        cps_status s = gain_state_init(g);
        if (s) return s;
    }
    if (g->three_on) launch_three_init(three_view(g), g->three_N0, g->stream);
    for (PortState &P : g->ports) {
        P.fill = 0;
        P.last_slot = -1;
        CK(cudaMemsetAsync(P.d_ring, 0, (size_t)P.slots * 6 * P.npts * g->esz, g->stream));
        if (P.d_acc) CK(cudaMemsetAsync(P.d_acc, 0, (size_t)P.ncomp * P.nfreq * 2 * P.npts * sizeof(double), g->stream));
    }
    // a sweep that gave up left the state incomplete; the reset state is whole again
    CK(cudaMemsetAsync(g->d_err, 0, sizeof(int), g->stream));
    if (g->solo) {
        cps_status s = batch_clear_error(g->solo);
        if (s) return s;
    }
    g->step = n0;
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

extern "C" cps_status cps_grid_set_wait_skew(cps_grid *g, int32_t extra_bytes)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    REQUIRE(extra_bytes >= 0 && extra_bytes <= 4096, CPS_E_INVALID, "cps_grid_set_wait_skew: 0..4096 bytes");
    FLUSH_RECORDED(g);
    CK(cudaSetDevice(g->desc.device));
    CK(cudaMemcpyAsync(g->d_err + 1, &extra_bytes, sizeof(int), cudaMemcpyHostToDevice, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    return CPS_OK;
}

extern "C" cps_status cps_grid_check_finite(cps_grid *g, int64_t *nonfinite)
{
    REQUIRE(g && nonfinite, CPS_E_INVALID, "NULL argument");
    FLUSH_RECORDED(g);
    CK(cudaMemsetAsync(g->d_counter, 0, sizeof(unsigned long long), g->stream));
    if (g->fp32) launch_count_nonfinite<float>(field_view<float>(g), g->d_counter, g->stream);
    else launch_count_nonfinite<double>(field_view<double>(g), g->d_counter, g->stream);
    g->launches++;
    unsigned long long h = 0;
    CK(cudaMemcpyAsync(&h, g->d_counter, sizeof(h), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    *nonfinite = (int64_t)h;
    return CPS_OK;
}

extern "C" cps_status cps_gain_populations(cps_grid *g, double *out, int64_t *ncells)
{
    REQUIRE(g && ncells, CPS_E_INVALID, "NULL argument");
    REQUIRE(g->gain_on, CPS_E_STATE, "gain not initialised");
    FLUSH_RECORDED(g);
    *ncells = g->g_n;
    if (!out) return CPS_OK;
    // FP32: the offsets n1 n2 n3 of each list cell gathered on the device;
    // FP64: the list-layout state as it is
    std::vector<double> st;
    if (g->fp32) {
        std::vector<float> t((size_t)g->g_n * 3);
        float *d_out = nullptr;
        cps_status s = dalloc(g, (void **)&d_out, t.size() * sizeof(float) + 16);
        if (s) return s;
        launch_gain_pops32((const float *)g->d_g_state, g->d_g_cell, g->g_n, d_out, g->stream);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(t.data(), d_out, t.size() * sizeof(float), cudaMemcpyDeviceToHost, g->stream));
        CK(cudaStreamSynchronize(g->stream));
        dfree(g, d_out);
        st.assign(t.begin(), t.end());
    } else {
        st.resize((size_t)gain_state_elems(g->g_n, kG64Words));
        CK(cudaMemcpyAsync(st.data(), g->d_g_state, st.size() * 8, cudaMemcpyDeviceToHost, g->stream));
        CK(cudaStreamSynchronize(g->stream));
    }
    // device list is in device order (k, j, i); report in (i, j, k) order
    std::vector<int64_t> cells(g->g_n);
    CK(cudaMemcpy(cells.data(), g->d_g_cell, g->g_n * sizeof(int64_t), cudaMemcpyDeviceToHost));
    std::vector<std::pair<int64_t, int64_t>> ord(g->g_n);
    const Dims &d = g->d;
    for (int64_t c = 0; c < g->g_n; ++c) {
        const int64_t q = cells[c];
        const int k = (int)(q / d.pxy), j = (int)((q - k * d.pxy) / d.px), i = (int)(q - k * d.pxy - (int64_t)j * d.px);
        ord[c] = {((int64_t)i * (d.ny + 1) + j) * (d.nz + 1) + k, c};
    }
    std::sort(ord.begin(), ord.end());
    const int64_t sc = kGainGroup;
    for (int64_t r = 0; r < g->g_n; ++r) {
        double N[4];
        if (g->fp32) {
            const int64_t c = ord[r].second * 3;
            N[1] = 1.0 + st[c]; N[2] = st[c + 1]; N[3] = st[c + 2];
            N[0] = 2.0 - N[1] - N[2] - N[3];
        } else {
            const int64_t c = gain_base_index(ord[r].second, kG64Words);
            for (int q = 0; q < 4; ++q) N[q] = st[(21 + q) * sc + c];
        }
        for (int q = 0; q < 4; ++q) out[r * 4 + q] = N[q];
    }
    return CPS_OK;
}

extern "C" cps_status cps_three_populations(cps_grid *g, double *out, int64_t *ncells)
{
    REQUIRE(g && ncells, CPS_E_INVALID, "NULL argument");
    REQUIRE(g->three_on, CPS_E_STATE, "three-level gain not initialised");
    FLUSH_RECORDED(g);
    *ncells = g->t_n;
    if (!out) return CPS_OK;
    const int64_t n = g->t_n;
    std::vector<double> st((size_t)n * 3);
    std::vector<int64_t> cells(n);
    CK(cudaMemcpyAsync(st.data(), g->d_t_state + (size_t)21 * n, (size_t)n * 3 * sizeof(double),
                       cudaMemcpyDeviceToHost, g->stream));
    CK(cudaMemcpyAsync(cells.data(), g->d_t_cell, n * sizeof(int64_t), cudaMemcpyDeviceToHost, g->stream));
    CK(cudaStreamSynchronize(g->stream));
    // device list is in device order (k, j, i); report in (i, j, k) order
    std::vector<std::pair<int64_t, int64_t>> ord(n);
    const Dims &d = g->d;
    for (int64_t c = 0; c < n; ++c) {
        const int64_t q = cells[c];
        const int k = (int)(q / d.pxy), j = (int)((q - k * d.pxy) / d.px), i = (int)(q - k * d.pxy - (int64_t)j * d.px);
        ord[c] = {((int64_t)i * (d.ny + 1) + j) * (d.nz + 1) + k, c};
    }
    std::sort(ord.begin(), ord.end());
    for (int64_t r = 0; r < n; ++r)
        for (int q = 0; q < 3; ++q) out[r * 3 + q] = st[(size_t)q * n + ord[r].second];
    return CPS_OK;
}

extern "C" cps_status cps_grid_launch_count(const cps_grid *g, int64_t *launches)
{
    REQUIRE(g && launches, CPS_E_INVALID, "NULL argument");
    *launches = g->launches;
    return CPS_OK;
}

extern "C" cps_status cps_ports_flush(cps_grid *g)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    FLUSH_RECORDED(g);
    for (PortState &P : g->ports) {
        cps_status s = flush_dft(g, P);
        if (s) return s;
    }
    return CPS_OK;
}

extern "C" cps_status cps_grid_set_timing(cps_grid *g, int32_t stride)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    REQUIRE(stride >= 0, CPS_E_INVALID, "cps_grid_set_timing: negative stride");
    CK(cudaStreamSynchronize(g->stream));
    if (g->ev.empty() && stride > 0) {
        g->ev.resize(4 * 4096);
        for (auto &e : g->ev) CK(cudaEventCreate(&e));
    }
    g->timing_stride = stride;
    g->ev_used = 0;
    return CPS_OK;
}

extern "C" cps_status cps_grid_timing(cps_grid *g, double *h_ms, double *e_ms, int64_t *samples)
{
    REQUIRE(g && h_ms && e_ms && samples, CPS_E_INVALID, "NULL argument");
    CK(cudaStreamSynchronize(g->stream));
    double h = 0, e = 0;
    const int n = g->ev_used / 4;
    for (int s = 0; s < n; ++s) {
        float a = 0, b = 0;
        CK(cudaEventElapsedTime(&a, g->ev[4 * s], g->ev[4 * s + 1]));
        CK(cudaEventElapsedTime(&b, g->ev[4 * s + 2], g->ev[4 * s + 3]));
        h += a;
        e += b;
    }
    *h_ms = n ? h / n : 0.0;
    *e_ms = n ? e / n : 0.0;
    *samples = n;
    return CPS_OK;
}

extern "C" cps_status cps_grid_set_tile(cps_grid *g, int32_t rows, int32_t planes)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    REQUIRE((rows == 4 || rows == 8 || rows == 16) && planes >= 1, CPS_E_INVALID,
            "cps_grid_set_tile: rows must be 4, 8 or 16 and planes >= 1");
    g->shape.by = rows;
    g->shape.kc = planes;
    g->shape.kch = planes;
    g->shape.kcg = planes;
    return CPS_OK;
}

extern "C" cps_status cps_grid_get_tile(const cps_grid *g, int32_t *rows, int32_t *planes)
{
    REQUIRE(g && rows && planes, CPS_E_INVALID, "NULL argument");
    *rows = g->shape.by;
    *planes = g->shape.kc;
    return CPS_OK;
}

extern "C" cps_status cps_grid_set_sweep(cps_grid *g, int32_t mode)
{
    REQUIRE(g, CPS_E_INVALID, "NULL grid");
    REQUIRE(mode == 0 || mode == 1, CPS_E_INVALID, "cps_grid_set_sweep: 0 (TMA-fed) or 1 (register)");
    g->sweep_mode = mode;
    return CPS_OK;
}
