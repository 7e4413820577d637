// raster.cu -- device-side mesh rasterisation (Structure::generate_mesh,
// Structure.cpp:159-307) straight into a grid's uint8 ID array in the device
// layout.  The decisions equal cps_mesh_rasterize's bit for bit: the host
// expands multi shapes and truncates corners exactly as the host rasteriser
// does, the in/out predicates run in FP64 without FMA contraction, and the
// sample coordinates of rotated cuboids are the host loop's accumulated
// values, uploaded.  Shapes are applied in order, one launch each, so a later
// shape overwrites an earlier one as in the reference.
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "grid.h"

namespace cps {

namespace {

struct RasterOp {
    int kind;  // 0 axis-aligned cuboid, 1 rotated cuboid, 2 ellipsoid, 3 cylinder
    int mat;
    int i0, j0, k0, ni, nj, nk;  // iteration box (cells, or sample counts for kind 1)
    double x0, y0, z0, a2, b2, c2;
    double ct, st, cp, sp, cs, ss;
    int off_x, off_y, off_z;     // kind 1: offsets of the sample coordinates
};

__global__ void k_raster(RasterOp op, const double *__restrict__ samples, uint8_t *ids, Dims d, double dx, double dy,
                         double dz)
{
    const int64_t n = (int64_t)op.ni * op.nj * op.nk;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int a = (int)(q % op.ni), b = (int)((q / op.ni) % op.nj), c = (int)(q / ((int64_t)op.ni * op.nj));
        int i, j, k;
        if (op.kind == 0) {  // cuboid(), axis-aligned branch
            i = op.i0 + a; j = op.j0 + b; k = op.k0 + c;
        } else if (op.kind == 1) {  // cuboid(), rotations about x (theta), y (phi), z (psi)
            const double x = samples[op.off_x + a], y = samples[op.off_y + b], z = samples[op.off_z + c];
            const double x1 = x;
            const double y1 = op.ct * (y) - op.st * (z);
            const double z1 = op.st * (y) + op.ct * (z);
            const double x2 = op.cp * (x1) + op.sp * (z1);
            const double y2 = y1;
            const double z2 = -op.sp * (x1) + op.cp * (z1);
            const double x3 = op.cs * (x2) - op.ss * (y2);
            const double y3 = op.ss * (x2) + op.cs * (y2);
            const double z3 = z2;
            i = (int)((x3 + op.x0) / dx);
            j = (int)((y3 + op.y0) / dy);
            k = (int)((z3 + op.z0) / dz);
        } else if (op.kind == 2) {  // ellipsoid()
            i = op.i0 + a; j = op.j0 + b; k = op.k0 + c;
            const double X = (double)i * dx - op.x0, Y = (double)j * dy - op.y0, Z = (double)k * dz - op.z0;
            const double temp = X * X / op.a2 + Y * Y / op.b2 + Z * Z / op.c2;
            if (!(temp <= 1.0)) continue;
        } else {  // cylinder()
            i = a; j = b; k = c + op.k0;
            const double X = (double)i * dx - op.x0, Y = (double)j * dy - op.y0;
            const double temp = X * X / op.a2 + Y * Y / op.b2;
            if (!(temp <= 1.0)) continue;
        }
        if (i < 0 || j < 0 || k < 0 || i > d.nx || j > d.ny || k > d.nz) continue;
        ids[d.idx(i, j, k)] = (uint8_t)op.mat;
    }
}

// a shape after Structure.cpp:100-106 parsing: integer corners by truncation
struct ShapeT {
    int mat;
    double theta, phi, psi, x0, y0, z0, a, b, c;
    int ix0, jy0, kz0, ia, jb, kc;
};

ShapeT make_shape(const cps_shape &s, double dx, double dy, double dz)
{
    ShapeT h;
    h.mat = s.material_index;
    h.theta = s.theta; h.phi = s.phi; h.psi = s.psi;
    h.x0 = s.x0; h.y0 = s.y0; h.z0 = s.z0;
    h.a = s.a; h.b = s.b; h.c = s.c;
    h.ix0 = (int)(h.x0 / dx); h.jy0 = (int)(h.y0 / dy); h.kz0 = (int)(h.z0 / dz);
    h.ia = (int)(h.a / dx); h.jb = (int)(h.b / dy); h.kc = (int)(h.c / dz);
    return h;
}

// the launches of one shape (host_setup.cpp's loops as iteration boxes)
void plan_shape(const ShapeT &s, int type, const Dims &d, double dx, double dy, double dz, std::vector<RasterOp> &ops,
                std::vector<double> &samples)
{
    RasterOp op;
    memset(&op, 0, sizeof(op));
    op.mat = s.mat;
    if (type == CPS_SHAPE_CUBOID) {
        if ((s.theta == 0) && (s.phi == 0) && (s.psi == 0)) {
            op.kind = 0;
            op.i0 = s.ix0; op.j0 = s.jy0; op.k0 = s.kz0;
            op.ni = s.ia; op.nj = s.jb; op.nk = s.kc;
        } else {
            op.kind = 1;
            op.x0 = s.x0; op.y0 = s.y0; op.z0 = s.z0;
            op.ct = cos(s.theta); op.st = sin(s.theta); op.cp = cos(s.phi); op.sp = sin(s.phi);
            op.cs = cos(s.psi); op.ss = sin(s.psi);
            // the host loop's sample coordinates, accumulated the same way
            op.off_x = (int)samples.size();
            for (double x = 0; x < s.a; x = x + (dx / 2.0)) samples.push_back(x);
            op.ni = (int)samples.size() - op.off_x;
            op.off_y = (int)samples.size();
            for (double y = 0; y < s.b; y = y + (dy / 2.0)) samples.push_back(y);
            op.nj = (int)samples.size() - op.off_y;
            op.off_z = (int)samples.size();
            for (double z = 0; z < s.c; z = z + (dz / 2.0)) samples.push_back(z);
            op.nk = (int)samples.size() - op.off_z;
        }
    } else if (type == CPS_SHAPE_ELLIPSOID) {
        op.kind = 2;
        op.x0 = s.x0; op.y0 = s.y0; op.z0 = s.z0;
        op.a2 = s.a * s.a; op.b2 = s.b * s.b; op.c2 = s.c * s.c;
        auto lo = [](double c, double h, double del) { return (int)floor((c - fabs(h)) / del) - 2; };
        auto hi = [](double c, double h, double del) { return (int)ceil((c + fabs(h)) / del) + 2; };
        const int i0 = std::max(0, lo(s.x0, s.a, dx)), j0 = std::max(0, lo(s.y0, s.b, dy)), k0 = std::max(0, lo(s.z0, s.c, dz));
        const int i1 = std::min(d.nx, hi(s.x0, s.a, dx)), j1 = std::min(d.ny, hi(s.y0, s.b, dy)),
                  k1 = std::min(d.nz, hi(s.z0, s.c, dz));
        op.i0 = i0; op.j0 = j0; op.k0 = k0;
        op.ni = std::max(0, i1 - i0); op.nj = std::max(0, j1 - j0); op.nk = std::max(0, k1 - k0);
    } else {
        op.kind = 3;
        op.x0 = s.x0; op.y0 = s.y0;
        op.a2 = s.a * s.a; op.b2 = s.b * s.b;
        op.k0 = s.kz0;
        op.ni = d.nx; op.nj = d.ny; op.nk = std::max(0, s.kc);
    }
    if (op.ni > 0 && op.nj > 0 && op.nk > 0) ops.push_back(op);
}

}  // namespace

}  // namespace cps

using namespace cps;

extern "C" cps_status cps_grid_rasterize(cps_grid *g, int32_t nshapes, const cps_shape *shapes, int32_t keep)
{
    REQUIRE(g, CPS_E_INVALID, "cps_grid_rasterize: NULL grid");
    REQUIRE(nshapes >= 0 && (nshapes == 0 || shapes), CPS_E_INVALID, "cps_grid_rasterize: bad shape list");
    REQUIRE(!g->dl_on && !g->gain_on && !g->three_on && !g->pml_on, CPS_E_STATE,
            "cps_grid_rasterize: IDs must be set before the physics modules are initialised");
    cps_status s = flush_recorded(g);
    if (s) return s;
    const Dims &d = g->d;
    const double dx = g->desc.dx, dy = g->desc.dy, dz = g->desc.dz;
    std::vector<RasterOp> ops;
    std::vector<double> samples;
    int maxid = keep ? g->ids_max : 0;
    for (int q = 0; q < nshapes; ++q) {
        const cps_shape &sh = shapes[q];
        REQUIRE(sh.material_index >= 0 && sh.material_index <= 255, CPS_E_INVALID,
                "cps_grid_rasterize: material index outside 0..255");
        if (sh.type == CPS_SHAPE_MULTI) {  // Structure.cpp:238-307: counts in theta/phi/psi, pitch in a/b/c
            const int t = sh.material_index;
            REQUIRE(t >= 0 && t < nshapes && shapes[t].type != CPS_SHAPE_MULTI, CPS_E_INVALID,
                    "cps_grid_rasterize: multi shape refers to an invalid template");
            const ShapeT multi = make_shape(sh, dx, dy, dz);
            ShapeT m = make_shape(shapes[t], dx, dy, dz);
            maxid = std::max(maxid, m.mat);
            for (int i = 0; i < multi.theta; ++i) {
                m.x0 = multi.x0 + i * multi.a;
                m.ix0 = (int)(m.x0 / dx);
                for (int j = 0; j < multi.phi; ++j) {
                    m.y0 = multi.y0 + j * multi.b;
                    m.jy0 = (int)(m.y0 / dy);
                    for (int k = 0; k < multi.psi; ++k) {
                        m.z0 = multi.z0 + k * multi.c;
                        m.kz0 = (int)(m.z0 / dz);
                        plan_shape(m, shapes[t].type, d, dx, dy, dz, ops, samples);
                    }
                }
            }
        } else {
            REQUIRE(sh.type >= CPS_SHAPE_CUBOID && sh.type <= CPS_SHAPE_CYLINDER, CPS_E_INVALID,
                    "cps_grid_rasterize: unknown shape type");
            plan_shape(make_shape(sh, dx, dy, dz), sh.type, d, dx, dy, dz, ops, samples);
            maxid = std::max(maxid, sh.material_index);
        }
    }
    REQUIRE(g->nmedia == 0 || maxid < g->nmedia, CPS_E_INVALID,
            "cps_grid_rasterize: an ID has no medium (set the media first or extend them)");
    CK(cudaSetDevice(g->desc.device));
    if (!keep) CK(cudaMemsetAsync(g->d_id, 0, (size_t)g->elems, g->stream));
    double *d_samples = nullptr;
    if (!samples.empty()) {
        if ((s = dalloc(g, (void **)&d_samples, samples.size() * sizeof(double)))) return s;
        if ((s = upload_raw(g, d_samples, samples.data(), samples.size() * sizeof(double)))) return s;
    }
    for (const RasterOp &op : ops) {
        const int64_t n = (int64_t)op.ni * op.nj * op.nk;
        const unsigned blocks = (unsigned)std::min<int64_t>((n + 255) / 256, 148 * 16);
        k_raster<<<blocks, 256, 0, g->stream>>>(op, d_samples, g->d_id, d, dx, dy, dz);
        g->launches++;
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess)  // the host copy the compacted-list builders read
        e = cudaMemcpyAsync(g->ids_dev.data(), g->d_id, (size_t)g->elems, cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    if (d_samples) dfree(g, d_samples);
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("cps_grid_rasterize: ") + cudaGetErrorString(e));
    g->ids_max = maxid;
    g->ids_set = true;
    return CPS_OK;
}
