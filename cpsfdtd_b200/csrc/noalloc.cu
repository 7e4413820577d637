// noalloc.cu -- cps_ports_flush_static: the port-DFT flush (fold the samples
// waiting in every port ring into the FP64 accumulators) without any device
// allocation.  cps_ports_flush may allocate the phasor scratch of the
// contraction on first use or when a port needs more; this form uses a
// file-scope device array instead.  It is for callers that cannot allocate:
// a serving process that admitted the job against a fixed memory budget and
// may not grow its footprint, and latency-bounded loops that must not enter
// the driver's allocator (cudaMalloc/cudaFree may synchronise the device).
//
// Limits: ports of at most kStaticMaxFreq frequencies (rings hold at most 64
// samples); larger ports are rejected with CPS_E_INVALID before anything is
// launched.  The scratch need not start at zero: the phasor kernel of a call
// writes every entry its contraction reads.  The scratch is shared by every
// grid on a device, so calls on one device must not overlap (issue them from
// one stream, or order them): overlapping calls race on the table.
//
// Set-up: the first call on a device looks up the array's device address
// (cudaGetSymbolAddress, with that device current) and caches it; make one
// call on each device before any stream capture that includes this call.
#include <mutex>

#include "grid.h"

namespace cps {

namespace {

constexpr int kStaticMaxFreq = 256;
constexpr int kStaticMaxSlots = 64;
// [2][slots][nfreq] of (cos, sin) in FP64: 512 KiB
constexpr size_t kStaticScratchDoubles = (size_t)2 * kStaticMaxSlots * kStaticMaxFreq * 2;
static __device__ __align__(256) double g_flush_scratch[kStaticScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
double *g_scratch_ptr[kMaxDevices] = {};

cps_status static_scratch(int device, double **out)
{
    REQUIRE(device >= 0 && device < kMaxDevices, CPS_E_INVALID, "cps_ports_flush_static: device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        int cur = -1;
        CK(cudaGetDevice(&cur));
        CK(cudaSetDevice(device));
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_flush_scratch);
        if (cur >= 0) cudaSetDevice(cur);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error(std::string("cps_ports_flush_static: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return CPS_E_CUDA;
        }
        g_scratch_ptr[device] = (double *)p;
    }
    *out = g_scratch_ptr[device];
    return CPS_OK;
}

template <typename T>
cps_status flush_static_T(cps_grid *g, double *scratch)
{
    for (PortState &P : g->ports) {
        if (P.nfreq == 0 || P.fill == 0) continue;
        launch_port_dft<T>((const T *)P.d_ring, P.npts, P.fill, P.ring_n0, g->desc.dt, P.d_omega, P.nfreq, P.d_comps,
                           P.ncomp, P.d_acc, scratch, g->stream);
        // a failed launch leaves the ring as it was, so a later flush folds its samples
        const cudaError_t e = cudaGetLastError();
        REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("cps_ports_flush_static: ") + cudaGetErrorString(e));
        g->launches += 2;
        // keep the last sample readable: move it to slot 0
        if (P.last_slot > 0) {
            CK(cudaMemcpyAsync(P.d_ring, (T *)P.d_ring + (int64_t)P.last_slot * 6 * P.npts, sizeof(T) * 6 * P.npts,
                               cudaMemcpyDeviceToDevice, g->stream));
            P.last_slot = 0;
        }
        P.fill = 0;
    }
    return CPS_OK;
}

}  // namespace

}  // namespace cps

using namespace cps;

extern "C" cps_status cps_ports_flush_static(cps_grid *g)
{
    REQUIRE(g, CPS_E_INVALID, "cps_ports_flush_static: NULL grid");
    // running recorded calls may allocate (a full ring's fold, first source upload)
    REQUIRE(g->pending.empty(), CPS_E_STATE,
            "cps_ports_flush_static: the grid holds recorded calls not yet run (cps_synchronize first)");
    for (const PortState &P : g->ports)
        REQUIRE(P.nfreq <= kStaticMaxFreq && P.slots <= kStaticMaxSlots, CPS_E_INVALID,
                "cps_ports_flush_static: a port has more than 256 DFT frequencies (use cps_ports_flush)");
    double *scratch = nullptr;
    cps_status s = static_scratch(g->desc.device, &scratch);
    if (s) return s;
    CK(cudaSetDevice(g->desc.device));
    return g->fp32 ? flush_static_T<float>(g, scratch) : flush_static_T<double>(g, scratch);
}
