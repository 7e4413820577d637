// batch.cpp -- the batched engine behind cps_batch_*: many independent grids
// of uneven size advanced together.  There is no counterpart in the reference,
// which runs one grid per process (main.cpp's time loop); every member grid
// is built with the one-grid C ABI and keeps its own state, step counter and
// results, which the one-grid calls read as usual.
//
// A step of the batch is one launch per sweep class (H interior / H CPML
// tiles; E interior / E CPML tiles, each with and without gain) over flat
// tables of tiles that name their grid, then the Drude-Lorentz cells, TF/SF
// injection, sources and port sampling of all grids, each one launch.  Steps
// run in chunks of at most kMaxRing; a chunk ends with one port-DFT
// contraction over every port and a kernel that advances every grid's step
// counter, and is captured once into a CUDA graph per chunk length and
// replayed while the membership and tiling stay the same.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "batch.h"
#include "grid.h"

using namespace cps;

namespace {

struct GridSig {
    int64_t step;
    const void *f0, *dl, *gain, *st, *q, *tg0, *tg1, *srcw, *ring0;
    int64_t dl_n, g_n;
    int nports, nsrc, ntg0, ntg1, pml, by;
    int64_t nfreq_sum;
    bool operator==(const GridSig &o) const { return memcmp(this, &o, sizeof(GridSig)) == 0; }
};

GridSig signature(const cps_grid *g)
{
    GridSig s;
    memset(&s, 0, sizeof(s));
    s.step = g->step;
    s.f0 = g->F[0]; s.dl = g->d_dl_cell; s.gain = g->d_g_cell; s.st = g->d_st; s.q = g->d_q[0][0];
    s.tg0 = g->d_tg[0]; s.tg1 = g->d_tg[1]; s.srcw = g->d_src_wave;
    s.ring0 = g->ports.empty() ? nullptr : g->ports[0].d_ring;
    s.dl_n = g->dl_on ? g->dl_n : -1; s.g_n = g->gain_on ? g->g_n : -1;
    s.nports = (int)g->ports.size(); s.nsrc = (int)g->src.size();
    s.ntg0 = g->tfsf_on ? g->ntg[0] : -1; s.ntg1 = g->tfsf_on ? g->ntg[1] : -1;
    s.pml = g->pml_on; s.by = g->tma_by;
    for (const PortState &P : g->ports) s.nfreq_sum += P.nfreq * 7 + P.npts;
    return s;
}

inline int cdiv_i(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// host copy of the device-side tile classification in tma_bodies.cuh
bool tile_in_pml_host(const int np[6], const Dims &d, int x0, int y0, int by, int k0, int k1, bool eside)
{
    const int lo = eside ? 0 : 1;
    const bool x = x0 <= np[kFX1] - lo || x0 + 31 >= d.nx - np[kFX2];
    const bool y = y0 <= np[kFY1] - lo || y0 + by - 1 >= d.ny - np[kFY2];
    const bool z = k0 <= np[kFZ1] - lo || k1 - 1 >= d.nz - np[kFZ2];
    return x || y || z;
}

// sweep classes: H interior / H CPML tiles, then E tiles by class bits
// (1 CPML tile, 2 Drude-Lorentz grid, 4 gain grid)
enum { kHInt, kHPml, kE0, kNumSweep = kE0 + 8 };

// members of at least this many cells fill the device by themselves: their
// sweeps are launched per grid with the one-grid kernels, whose tensor maps
// and views are kernel parameters (faster than the shared tile tables)
constexpr int64_t kBigCells = 4 << 20;

}  // namespace

struct cps_batch {
    bool fp32 = true;
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<cps_grid *> grids;
    std::vector<GridSig> sigs;
    bool dirty = true;
    // configuration
    int by = 4, kc = 16, persistent = 2, graph = 1;  // per-member launches: fastest on the measured mixes
    int kch = 0;  // planes per tile of the per-member H sweeps (0: kc)
    int kcg = 0;  // planes per tile of the per-member FP32 E sweeps with gain (0: kc)
    // device tables (owned)
    std::vector<void *> owned;
    void *d_grids = nullptr;
    void *d_ports = nullptr;
    int *d_err = nullptr;
    int4 *d_tiles[kNumSweep] = {};
    int ntiles[kNumSweep] = {};
    int nblocks[kNumSweep] = {};
    int4 *d_dl = nullptr; int ndl = 0;
    int4 *d_inj[2] = {nullptr, nullptr}; int ninj[2] = {0, 0};
    int2 *d_src = nullptr; int nsrc = 0;
    int2 *d_gather = nullptr; int ngather = 0;
    int2 *d_phasor = nullptr; int nphasor = 0;
    int4 *d_dft = nullptr; int ndft = 0;
    int nports = 0;
    int64_t cells = 0;
    std::vector<int> big;  // members stepped with their own sweep launches
    // side streams the per-member sweep launches fan out over (member q on
    // side[q % side.size()]), so that several members' sweeps run at once
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> side_done;
    cudaEvent_t fork = nullptr;
    // graphs per chunk length
    std::map<int, std::pair<cudaGraphExec_t, int64_t>> graphs;  // executable and its kernel count
    std::map<int, int> direct;  // chunk lengths launched directly since the last rebuild
    std::vector<cudaEvent_t> ev;  // one per member grid (ordering with the grid streams)
    cudaEvent_t done = nullptr;
    int64_t launches = 0;
};

namespace {

cps_status bmalloc(cps_batch *b, void **p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, b->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("batch table allocation of ") + std::to_string(bytes) + " bytes failed");
        return CPS_E_NOMEM;
    }
    b->owned.push_back(*p);
    return CPS_OK;
}

template <typename V>
cps_status upload_vec(cps_batch *b, V **dst, const std::vector<V> &v)
{
    cps_status s = bmalloc(b, (void **)dst, v.size() * sizeof(V));
    if (s) return s;
    if (!v.empty()) CK(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice, b->stream));
    return CPS_OK;
}

void drop_graphs(cps_batch *b)
{
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second.first);
    b->graphs.clear();
    b->direct.clear();
}

void free_tables(cps_batch *b)
{
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    for (void *p : b->owned) cudaFreeAsync(p, b->stream);
    b->owned.clear();
    b->d_grids = b->d_ports = nullptr;
    b->d_err = nullptr;
    for (int c = 0; c < kNumSweep; ++c) { b->d_tiles[c] = nullptr; b->ntiles[c] = b->nblocks[c] = 0; }
    b->d_dl = nullptr; b->ndl = 0;
    b->d_inj[0] = b->d_inj[1] = nullptr; b->ninj[0] = b->ninj[1] = 0;
    b->d_src = nullptr; b->nsrc = 0;
    b->d_gather = nullptr; b->ngather = 0;
    b->d_phasor = nullptr; b->nphasor = 0;
    b->d_dft = nullptr; b->ndft = 0;
    b->nports = 0;
    b->big.clear();
}

cps_status sync_grid_streams_in(cps_batch *b)
{
    // the batch stream waits for work already queued on each member's stream
    for (size_t q = 0; q < b->grids.size(); ++q) {
        CK(cudaEventRecord(b->ev[q], b->grids[q]->stream));
        CK(cudaStreamWaitEvent(b->stream, b->ev[q], 0));
    }
    return CPS_OK;
}

cps_status sync_grid_streams_out(cps_batch *b)
{
    CK(cudaEventRecord(b->done, b->stream));
    for (cps_grid *g : b->grids) CK(cudaStreamWaitEvent(g->stream, b->done, 0));
    return CPS_OK;
}

// Side streams for the per-member sweep launches: up to kSideStreams, made
// outside any capture when the tables are rebuilt.
constexpr size_t kSideStreams = 8;

cps_status ensure_side_streams(cps_batch *b)
{
    const size_t want = b->big.size() > 1 ? std::min(kSideStreams, b->big.size()) : 0;
    if (want && !b->fork) CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    while (b->side.size() < want) {
        cudaStream_t st = nullptr;
        cudaEvent_t ev = nullptr;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            cudaStreamDestroy(st);
            CK(e);
        }
        b->side.push_back(st);
        b->side_done.push_back(ev);
    }
    return CPS_OK;
}

// The per-member sweeps of one phase: on the batch stream one after another,
// or fanned out over the side streams between an event fork and join (which a
// capture records as graph edges).
template <typename F>
void per_member(cps_batch *b, F &&launch)
{
    if (b->big.empty()) return;
    const size_t ns = b->big.size() > 1 ? std::min(b->side.size(), b->big.size()) : 0;
    if (ns == 0) {
        for (int gi : b->big) launch(gi, b->stream);
        return;
    }
    cudaEventRecord(b->fork, b->stream);
    for (size_t k = 0; k < ns; ++k) cudaStreamWaitEvent(b->side[k], b->fork, 0);
    for (size_t q = 0; q < b->big.size(); ++q) launch(b->big[q], b->side[q % ns]);
    for (size_t k = 0; k < ns; ++k) {
        cudaEventRecord(b->side_done[k], b->side[k]);
        cudaStreamWaitEvent(b->stream, b->side_done[k], 0);
    }
}

template <typename T>
cps_status rebuild_T(cps_batch *b)
{
    free_tables(b);
    const int by = b->by, kc = b->kc;
    std::vector<BatchGrid<T>> hg(b->grids.size());
    std::vector<BatchPort<T>> hp;
    std::vector<int4> tiles[kNumSweep], dl, inj[2], dft;
    std::vector<int2> src, gather, phasor;
    std::vector<std::pair<int, size_t>> tab_size;  // (port, bytes) of phasor scratch
    b->cells = 0;
    for (size_t gi = 0; gi < b->grids.size(); ++gi) {
        cps_grid *g = b->grids[gi];
        cps_status s;
        if ((s = ensure_sources(g))) return s;
        if (g->shape.by != by) g->shape.by = by;
        if ((s = ensure_tma(g))) return s;
        // fold samples left in the rings by one-grid stepping
        for (PortState &P : g->ports)
            if (P.fill > 0 && P.nfreq > 0 && (s = flush_dft(g, P))) return s;
        CK(cudaStreamSynchronize(g->stream));
        BatchGrid<T> &B = hg[gi];
        memset((void *)&B, 0, sizeof(B));
        B.M = g->tma;
        B.f = field_view<T>(g);
        B.p = pml_view<T>(g);
        B.D = dl_view<T>(g);
        B.G = gain_view<T>(g);
        if (g->tfsf_on) {
            for (int side = 0; side < 2; ++side) {
                B.tg[side] = g->d_tg[side];
                B.ct[side] = g->d_ct[side];
                B.ntg[side] = g->ntg[side];
            }
            B.inc[0] = (const T *)g->d_hinc;
            B.inc[1] = (const T *)g->d_einc;
            B.Nt = g->tp.Nt;
        }
        B.nsrc = (int)g->src.size();
        B.src_idx = g->d_src_idx; B.src_comp = g->d_src_comp; B.src_off = g->d_src_off;
        B.src_len = g->d_src_len; B.src_wave = g->d_src_wave;
        B.n0 = g->step;
        B.dt = g->desc.dt;
        B.kc = kc;
        const Dims &d = g->d;
        b->cells += (int64_t)d.nx * d.ny * d.nz;
        // sweep tiles, z outermost so that neighbouring blocks share halos
        const bool gain = B.G.on && B.G.ncell > 0, dlg = B.D.on && B.D.ncell > 0;
        const int nbx = cdiv_i(d.nx, 32), nby = cdiv_i(d.ny, by), nbz = cdiv_i(d.nz, kc);
        // a grid that fills the device alone gets its own sweep launches (tensor
        // maps as kernel parameters); the rest of its step stays batched
        const bool is_big = b->persistent == 2 || (int64_t)d.nx * d.ny * d.nz >= kBigCells;
        if (is_big) b->big.push_back((int)gi);
        for (int bz = 0; bz < nbz && !is_big; ++bz)
            for (int yb = 0; yb < nby; ++yb)
                for (int xb = 0; xb < nbx; ++xb) {
                    const int4 t = make_int4((int)gi, xb, yb, bz);
                    {   // H: planes [bz*kc, min(bz*kc+kc, nz))
                        const int k0 = bz * kc, k1 = std::min(k0 + kc, d.nz);
                        if (k0 < k1) {
                            const bool pml = B.p.on && tile_in_pml_host(B.p.np, d, xb * 32, yb * by, by, k0, k1, false);
                            tiles[pml ? kHPml : kHInt].push_back(t);
                        }
                    }
                    {   // E: planes [max(1, bz*kc), min(bz*kc+kc, nz))
                        const int k0 = std::max(1, bz * kc), k1 = std::min(bz * kc + kc, d.nz);
                        if (k0 < k1) {
                            const bool pml = B.p.on && tile_in_pml_host(B.p.np, d, xb * 32, yb * by, by, k0, k1, true);
                            tiles[kE0 + (pml ? 1 : 0) + (dlg ? 2 : 0) + (gain ? 4 : 0)].push_back(t);
                        }
                    }
                }
        if (B.D.on && B.D.ncell > 0 && !is_big) {
            REQUIRE(B.D.ncell < INT32_MAX, CPS_E_INVALID, "batch: Drude-Lorentz list too long");
            for (int64_t c0 = 0; c0 < B.D.ncell; c0 += 128)
                dl.push_back(make_int4((int)gi, (int)c0, (int)std::min<int64_t>(c0 + 128, B.D.ncell), 0));
        }
        for (int side = 0; side < 2; ++side)
            for (int t0 = 0; t0 < B.ntg[side]; t0 += kInjPerBlock)
                inj[side].push_back(make_int4((int)gi, t0, std::min(t0 + kInjPerBlock, B.ntg[side]), 0));
        for (int q = 0; q < B.nsrc; ++q) src.push_back(make_int2((int)gi, q));
        for (PortState &P : g->ports) {
            BatchPort<T> bp;
            memset(&bp, 0, sizeof(bp));
            bp.idx = P.d_idx; bp.ring = (T *)P.d_ring; bp.omega = P.d_omega; bp.comps = P.d_comps;
            bp.acc = P.d_acc; bp.grid = (int)gi; bp.npts = P.npts; bp.slots = P.slots;
            bp.nfreq = P.nfreq; bp.ncomp = P.ncomp;
            const int pi = (int)hp.size();
            for (int p0 = 0; p0 < P.npts; p0 += 256) gather.push_back(make_int2(pi, p0));
            if (P.nfreq > 0 && P.npts > 0) {
                tab_size.push_back({pi, (size_t)2 * kMaxRing * P.nfreq * sizeof(double2)});
                for (int q0 = 0; q0 < kMaxRing * P.nfreq; q0 += 256) phasor.push_back(make_int2(pi, q0));
                const int ft = dft_freq_tile(P.nfreq), pt = dft_point_tile(P.nfreq);
                for (int fb = 0; fb < cdiv_i(P.nfreq, ft); ++fb)
                    for (int ci = 0; ci < P.ncomp; ++ci)
                        for (int pb = 0; pb < cdiv_i(P.npts, pt); ++pb) dft.push_back(make_int4(pi, pb, ci, fb));
            }
            hp.push_back(bp);
        }
    }
    // phasor scratch, one slice per port with a DFT
    size_t tab_total = 0;
    for (auto &ts : tab_size) tab_total += (ts.second + 255) / 256 * 256;
    if (tab_total) {
        void *tab = nullptr;
        cps_status s = bmalloc(b, &tab, tab_total);
        if (s) return s;
        size_t off = 0;
        for (auto &ts : tab_size) {
            hp[ts.first].tab = (double2 *)((char *)tab + off);
            off += (ts.second + 255) / 256 * 256;
        }
    }
    cps_status s;
    if ((s = upload_vec(b, (BatchGrid<T> **)&b->d_grids, hg))) return s;
    if ((s = upload_vec(b, (BatchPort<T> **)&b->d_ports, hp))) return s;
    if ((s = bmalloc(b, (void **)&b->d_err, 2 * sizeof(int)))) return s;  // error code, wait test setting (0)
    CK(cudaMemsetAsync(b->d_err, 0, 2 * sizeof(int), b->stream));
    // kernel attributes are set here, outside any stream capture
    batch_kernel_attributes<T>();
    tma_attributes<T>();
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    for (int c = 0; c < kNumSweep; ++c) {
        if ((s = upload_vec(b, &b->d_tiles[c], tiles[c]))) return s;
        b->ntiles[c] = (int)tiles[c].size();
        b->nblocks[c] = b->ntiles[c];
        if (b->persistent == 1 && b->ntiles[c] > 0) {
            const bool eside = c >= kE0;
            const int cls = eside ? c - kE0 : (c == kHPml ? 1 : 0);
            const int per_sm = batch_blocks_per_sm<T>(by, eside, cls);
            b->nblocks[c] = std::min(b->ntiles[c], per_sm * nsm);
        }
    }
    if ((s = ensure_side_streams(b))) return s;
    if ((s = upload_vec(b, &b->d_dl, dl))) return s;
    b->ndl = (int)dl.size();
    for (int side = 0; side < 2; ++side) {
        if ((s = upload_vec(b, &b->d_inj[side], inj[side]))) return s;
        b->ninj[side] = (int)inj[side].size();
    }
    if ((s = upload_vec(b, &b->d_src, src))) return s;
    b->nsrc = (int)src.size();
    if ((s = upload_vec(b, &b->d_gather, gather))) return s;
    b->ngather = (int)gather.size();
    if ((s = upload_vec(b, &b->d_phasor, phasor))) return s;
    b->nphasor = (int)phasor.size();
    if ((s = upload_vec(b, &b->d_dft, dft))) return s;
    b->ndft = (int)dft.size();
    b->nports = (int)hp.size();
    CK(cudaStreamSynchronize(b->stream));
    b->sigs.clear();
    for (cps_grid *g : b->grids) b->sigs.push_back(signature(g));
    b->dirty = false;
    return CPS_OK;
}

// Enqueue one chunk of S steps on the batch stream; returns the launch count.
template <typename T>
int64_t enqueue_chunk(cps_batch *b, int S)
{
    const BatchGrid<T> *G = (const BatchGrid<T> *)b->d_grids;
    const BatchPort<T> *P = (const BatchPort<T> *)b->d_ports;
    cudaStream_t st = b->stream;
    int64_t n = 0;
    for (int s = 0; s < S; ++s) {
        launch_h_batch<T>(G, b->d_tiles[kHInt], b->ntiles[kHInt], b->nblocks[kHInt], b->by, false, b->d_err, st);
        launch_h_batch<T>(G, b->d_tiles[kHPml], b->ntiles[kHPml], b->nblocks[kHPml], b->by, true, b->d_err, st);
        per_member(b, [&](int gi, cudaStream_t ms) {
            const cps_grid *g = b->grids[gi];
            n += launch_h_tma<T>(g->tma, field_view<T>(g), pml_view<T>(g), FusedShape{b->by, b->kc, b->kch}, b->d_err,
                                 ms);
        });
        launch_inject_batch<T>(G, b->d_inj[1], b->ninj[1], 1, s, st);
        for (int c = 0; c < 8; ++c)
            launch_e_batch<T>(G, b->d_tiles[kE0 + c], b->ntiles[kE0 + c], b->nblocks[kE0 + c], b->by, c, b->d_err, st);
        launch_dl_batch<T>(G, b->d_dl, b->ndl, st);
        per_member(b, [&](int gi, cudaStream_t ms) {
            const cps_grid *g = b->grids[gi];
            n += launch_e_tma<T>(g->tma, field_view<T>(g), pml_view<T>(g), dl_view<T>(g), gain_view<T>(g),
                            FusedShape{b->by, b->kc, 0, b->kcg}, b->d_err, ms, &g->lane);
        });
        launch_inject_batch<T>(G, b->d_inj[0], b->ninj[0], 0, s, st);
        launch_sources_batch<T>(G, b->d_src, b->nsrc, s, st);
        launch_gather_batch<T>(G, P, b->d_gather, b->ngather, s, S - 1, st);
        for (int c = 0; c < kNumSweep; ++c) n += b->ntiles[c] > 0;
        n += (b->ndl > 0) + (b->ninj[0] > 0) + (b->ninj[1] > 0) + (b->nsrc > 0) + (b->ngather > 0);
    }
    launch_dft_batch<T>(G, P, b->d_phasor, b->nphasor, b->d_dft, b->ndft, S, st);
    n += b->ndft > 0 ? 2 : 0;
    launch_advance_batch<T>((BatchGrid<T> *)b->d_grids, (int)b->grids.size(), S, st);
    return n + 1;
}

// A chunk length is launched directly the first time after a rebuild and
// captured into a graph when it comes again, so membership that changes every
// chunk (serving) does not pay for captures it never replays.
template <typename T>
cps_status run_chunk(cps_batch *b, int S)
{
    if (!b->graph || (b->graphs.find(S) == b->graphs.end() && b->direct[S]++ == 0)) {
        b->launches += enqueue_chunk<T>(b, S);
        cudaError_t e = cudaGetLastError();
        REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("batch launch failed: ") + cudaGetErrorString(e));
        return CPS_OK;
    }
    auto it = b->graphs.find(S);
    if (it == b->graphs.end()) {
        cudaGraph_t graph = nullptr;
        CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int64_t n = enqueue_chunk<T>(b, S);
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(std::string("batch graph capture failed: ") + cudaGetErrorString(e));
            return CPS_E_CUDA;
        }
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error(std::string("batch graph instantiation failed: ") + cudaGetErrorString(e));
            return CPS_E_CUDA;
        }
        it = b->graphs.insert({S, {exec, n}}).first;
    }
    CK(cudaGraphLaunch(it->second.first, b->stream));
    b->launches += it->second.second;  // kernels inside the graph
    return CPS_OK;
}

template <typename T>
cps_status step_batch_T(cps_batch *b, int nsteps)
{
    // rebuild when a member changed since the tables were made
    if (!b->dirty)
        for (size_t q = 0; q < b->grids.size(); ++q)
            if (!(signature(b->grids[q]) == b->sigs[q])) { b->dirty = true; break; }
    cps_status s;
    if (b->dirty && (s = rebuild_T<T>(b))) return s;
    if ((s = sync_grid_streams_in(b))) return s;
    while (nsteps > 0) {
        const int S = std::min(nsteps, kMaxRing);
        if (b->graph && S != kMaxRing && b->graphs.find(S) == b->graphs.end() && b->graphs.size() > 8) drop_graphs(b);
        if ((s = run_chunk<T>(b, S))) return s;
        for (cps_grid *g : b->grids) {
            g->step += S;
            for (PortState &P : g->ports) {
                P.fill = 0;
                P.last_slot = P.slots == 1 ? 0 : S - 1;
            }
        }
        nsteps -= S;
    }
    for (size_t q = 0; q < b->grids.size(); ++q) b->sigs[q].step = b->grids[q]->step;
    return sync_grid_streams_out(b);
}

cps_status check_batch_error(cps_batch *b)
{
    if (!b->d_err) return CPS_OK;
    int e = 0;
    CK(cudaMemcpyAsync(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    REQUIRE(e == 0, CPS_E_TIMEOUT, "a device-side wait of a batched sweep gave up (TMA data did not arrive)");
    return CPS_OK;
}

// ------------------------------------------------------------ autotuner

std::string bucket_key(const cps_batch *b)
{
    // shape bucket (log2 of mean cells, mean aspect) and material mix
    double cells = 0, aspect = 0;
    int ngain = 0, ndl = 0, ntfsf = 0, nports = 0;
    for (const cps_grid *g : b->grids) {
        const double c = (double)g->d.nx * g->d.ny * g->d.nz;
        cells += c;
        aspect += (double)g->d.nx / std::max(1, std::max(g->d.ny, g->d.nz));
        ngain += g->gain_on && g->g_n > 0;
        ndl += g->dl_on && g->dl_n > 0;
        ntfsf += g->tfsf_on;
        nports += (int)g->ports.size();
    }
    const int n = std::max<int>(1, (int)b->grids.size());
    char buf[256];
    snprintf(buf, sizeof(buf), "%s:g%d:c%d:a%d:gain%d:dl%d:tfsf%d:ports%d", b->fp32 ? "f32" : "f64",
             (int)lround(log2((double)n)), (int)lround(log2(std::max(1.0, cells / n))),
             (int)lround(4.0 * aspect / n), (int)lround(10.0 * ngain / n), (int)lround(10.0 * ndl / n),
             (int)lround(10.0 * ntfsf / n), nports > 0);
    return buf;
}

bool cache_lookup(const char *path, const std::string &key, int *by, int *kc, int *pers)
{
    if (!path || !*path) return false;
    std::ifstream in(path);
    std::string line;
    bool found = false;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string k;
        int a, c, p;
        double ms;
        if (ss >> k >> a >> c >> p >> ms && k == key && (a == 4 || a == 8) && c >= 1 && p >= 0 && p <= 2) {
            *by = a; *kc = c; *pers = p;
            found = true;  // the last entry for a key wins
        }
    }
    return found;
}

}  // namespace

void cps::batch_set_h_planes(cps_batch *b, int kch, int kcg)
{
    if (b->kch != kch || b->kcg != kcg) {
        b->kch = kch;
        b->kcg = kcg;
        b->dirty = true;  // captured chunks launch the per-member sweeps with them
    }
}

// clears a batch's device error word (the grid reset of a grid stepped
// through its internal one-grid batch)
cps_status cps::batch_clear_error(cps_batch *b)
{
    if (b->d_err) CK(cudaMemsetAsync(b->d_err, 0, sizeof(int), b->stream));
    return CPS_OK;
}

// ================================================================ C ABI

extern "C" cps_status cps_batch_create(int32_t precision, cps_batch **out)
{
    REQUIRE(out, CPS_E_INVALID, "cps_batch_create: NULL output");
    REQUIRE(precision == CPS_FP32 || precision == CPS_FP64, CPS_E_INVALID, "cps_batch_create: bad precision");
    *out = nullptr;
    cps_batch *b = new cps_batch();
    b->fp32 = precision == CPS_FP32;
    cudaGetDevice(&b->device);
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        set_error(std::string("cps_batch_create: ") + cudaGetErrorString(e));
        return CPS_E_CUDA;
    }
    *out = b;
    return CPS_OK;
}

extern "C" cps_status cps_batch_destroy(cps_batch *b)
{
    if (!b) return CPS_OK;
    free_tables(b);
    for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
    if (b->done) cudaEventDestroy(b->done);
    for (cudaStream_t st : b->side) cudaStreamDestroy(st);
    for (cudaEvent_t e : b->side_done) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return CPS_OK;
}

extern "C" cps_status cps_batch_add(cps_batch *b, cps_grid *g)
{
    REQUIRE(b && g, CPS_E_INVALID, "cps_batch_add: NULL argument");
    REQUIRE(g->fp32 == b->fp32, CPS_E_INVALID, "cps_batch_add: grid precision differs from the batch's");
    REQUIRE(g->nmedia > 0 && g->ids_set, CPS_E_STATE, "cps_batch_add: grid media and IDs must be set first");
    REQUIRE(!g->three_on, CPS_E_INVALID, "cps_batch_add: grids with the three-level gain are stepped one at a time");
    REQUIRE(std::find(b->grids.begin(), b->grids.end(), g) == b->grids.end(), CPS_E_INVALID,
            "cps_batch_add: grid is already in the batch");
    REQUIRE(g->d.px >= 64 && g->d.ny + 1 >= 9 && g->d.nz >= 2, CPS_E_INVALID,
            "cps_batch_add: grid too small for the batched sweeps (needs nx >= 32, ny >= 8, nz >= 2)");
    cudaEvent_t e = nullptr;
    CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->grids.push_back(g);
    b->ev.push_back(e);
    b->dirty = true;
    return CPS_OK;
}

extern "C" cps_status cps_batch_remove(cps_batch *b, cps_grid *g)
{
    REQUIRE(b && g, CPS_E_INVALID, "cps_batch_remove: NULL argument");
    auto it = std::find(b->grids.begin(), b->grids.end(), g);
    REQUIRE(it != b->grids.end(), CPS_E_NOTFOUND, "cps_batch_remove: grid is not in the batch");
    CK(cudaStreamSynchronize(b->stream));
    const size_t q = it - b->grids.begin();
    cudaEventDestroy(b->ev[q]);
    b->ev.erase(b->ev.begin() + q);
    b->grids.erase(it);
    b->dirty = true;
    return CPS_OK;
}

extern "C" cps_status cps_batch_info(const cps_batch *b, int32_t *ngrids, int64_t *cells)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_info: NULL batch");
    int64_t c = 0;
    for (const cps_grid *g : b->grids) c += (int64_t)g->d.nx * g->d.ny * g->d.nz;
    if (ngrids) *ngrids = (int32_t)b->grids.size();
    if (cells) *cells = c;
    return CPS_OK;
}

extern "C" cps_status cps_batch_set_tile(cps_batch *b, int32_t rows, int32_t planes, int32_t persistent)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_set_tile: NULL batch");
    REQUIRE(rows == 4 || rows == 8, CPS_E_INVALID, "cps_batch_set_tile: rows must be 4 or 8");
    REQUIRE(planes >= 1 && planes <= 4096, CPS_E_INVALID, "cps_batch_set_tile: planes out of range");
    REQUIRE(persistent >= 0 && persistent <= 2, CPS_E_INVALID, "cps_batch_set_tile: persistent is 0, 1 or 2");
    if (b->by != rows || b->kc != planes || b->persistent != persistent) {
        b->by = rows; b->kc = planes; b->persistent = persistent;
        b->dirty = true;
    }
    return CPS_OK;
}

extern "C" cps_status cps_batch_get_tile(const cps_batch *b, int32_t *rows, int32_t *planes, int32_t *persistent)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_get_tile: NULL batch");
    if (rows) *rows = b->by;
    if (planes) *planes = b->kc;
    if (persistent) *persistent = b->persistent;
    return CPS_OK;
}

extern "C" cps_status cps_batch_set_graph(cps_batch *b, int32_t on)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_set_graph: NULL batch");
    b->graph = on ? 1 : 0;
    return CPS_OK;
}

extern "C" cps_status cps_batch_get_stream(const cps_batch *b, void **stream)
{
    REQUIRE(b && stream, CPS_E_INVALID, "cps_batch_get_stream: NULL argument");
    *stream = (void *)b->stream;
    return CPS_OK;
}

extern "C" cps_status cps_batch_step(cps_batch *b, int32_t nsteps)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_step: NULL batch");
    REQUIRE(nsteps >= 0, CPS_E_INVALID, "cps_batch_step: negative step count");
    if (nsteps == 0 || b->grids.empty()) return CPS_OK;
    for (cps_grid *g : b->grids) {  // calls recorded on a member run first, on its own stream
        cps_status s = flush_recorded(g);
        if (s) return s;
    }
    return b->fp32 ? step_batch_T<float>(b, nsteps) : step_batch_T<double>(b, nsteps);
}

extern "C" cps_status cps_batch_synchronize(cps_batch *b)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_synchronize: NULL batch");
    CK(cudaStreamSynchronize(b->stream));
    return check_batch_error(b);
}

extern "C" cps_status cps_batch_launch_count(const cps_batch *b, int64_t *launches)
{
    REQUIRE(b && launches, CPS_E_INVALID, "cps_batch_launch_count: NULL argument");
    *launches = b->launches;
    return CPS_OK;
}

extern "C" cps_status cps_batch_tune_key(const cps_batch *b, char *buf, int32_t len)
{
    REQUIRE(b && buf && len > 0, CPS_E_INVALID, "cps_batch_tune_key: bad argument");
    const std::string k = bucket_key(b);
    snprintf(buf, (size_t)len, "%s", k.c_str());
    return CPS_OK;
}

// Pick rows, planes and persistence for this batch: from the cache file when
// it holds the batch's key, else by timing every candidate for trial_steps
// steps of the live batch (the tiling does not change results, so the trial
// steps are real steps: every member advances by the steps the trials ran,
// reported in *steps_run) and appending the winner to the cache.
extern "C" cps_status cps_batch_autotune(cps_batch *b, const char *cache_path, int32_t trial_steps,
                                         int32_t *steps_run)
{
    REQUIRE(b, CPS_E_INVALID, "cps_batch_autotune: NULL batch");
    REQUIRE(trial_steps >= 1 && trial_steps <= 4096, CPS_E_INVALID, "cps_batch_autotune: trial_steps out of range");
    if (steps_run) *steps_run = 0;
    if (b->grids.empty()) return CPS_OK;
    const std::string key = bucket_key(b);
    int by, kc, pers;
    if (cache_lookup(cache_path, key, &by, &kc, &pers)) return cps_batch_set_tile(b, by, kc, pers);
    static const int rows[] = {4, 8}, planes[] = {8, 16, 32, 64}, perss[] = {0, 1, 2};
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best = 1e300;
    int bb = b->by, bk = b->kc, bp = b->persistent, ran = 0;
    cps_status s = CPS_OK;
    for (int r : rows)
        for (int k : planes)
            for (int p : perss) {
                if ((s = cps_batch_set_tile(b, r, k, p))) break;
                // one untimed step builds the tables (and the graph of that length)
                if ((s = cps_batch_step(b, 1))) break;
                cudaEventRecord(e0, b->stream);
                if ((s = cps_batch_step(b, trial_steps))) break;
                cudaEventRecord(e1, b->stream);
                if ((s = cps_batch_synchronize(b))) break;
                float ms = 0;
                cudaEventElapsedTime(&ms, e0, e1);
                ran += 1 + trial_steps;
                if (ms < best) { best = ms; bb = r; bk = k; bp = p; }
            }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (steps_run) *steps_run = ran;
    if (s) return s;
    if (cache_path && *cache_path) {
        FILE *f = fopen(cache_path, "a");
        if (f) {
            fprintf(f, "%s %d %d %d %.6f\n", key.c_str(), bb, bk, bp, best / trial_steps);
            fclose(f);
        }
    }
    return cps_batch_set_tile(b, bb, bk, bp);
}
