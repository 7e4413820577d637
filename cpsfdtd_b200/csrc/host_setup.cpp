// host_setup.cpp -- host-side geometry builders of the C ABI: mesh
// rasterisation (Structure.cpp:159-307), port point sets (Ports.cpp:28-86,
// 201-306) and the Courant step (Structure.cpp:124).  Built without FMA
// contraction so that every in/out decision and index truncation matches the
// reference bit for bit.
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "cps_internal.h"

namespace cps {
void set_error(const std::string &msg);
}

using namespace cps;

extern "C" double cps_courant_dt(double dx, double dy, double dz)
{
    return 0.99 / (kC * sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)));
}

namespace {

struct Raster {
    int nx, ny, nz;
    double dx, dy, dz;
    uint8_t *ids;
    int64_t at(int i, int j, int k) const { return ((int64_t)i * (ny + 1) + j) * (nz + 1) + k; }
    bool inside(int i, int j, int k) const { return i >= 0 && j >= 0 && k >= 0 && i <= nx && j <= ny && k <= nz; }
    void put(int i, int j, int k, int m)
    {
        if (inside(i, j, k)) ids[at(i, j, k)] = (uint8_t)m;
    }
};

// Shape after Structure.cpp:100-106 parsing: integer corners by truncation
struct Sh {
    int mat;
    double theta, phi, psi, x0, y0, z0, a, b, c;
    int ix0, jy0, kz0, ia, jb, kc;
};

Sh make_shape(const cps_shape &s, const Raster &r)
{
    Sh h;
    h.mat = s.material_index;
    h.theta = s.theta; h.phi = s.phi; h.psi = s.psi;
    h.x0 = s.x0; h.y0 = s.y0; h.z0 = s.z0;
    h.a = s.a; h.b = s.b; h.c = s.c;
    h.ix0 = (int)(h.x0 / r.dx); h.jy0 = (int)(h.y0 / r.dy); h.kz0 = (int)(h.z0 / r.dz);
    h.ia = (int)(h.a / r.dx); h.jb = (int)(h.b / r.dy); h.kc = (int)(h.c / r.dz);
    return h;
}

// cuboid(), Structure.cpp:159-203; the axis-aligned branch writes only cells
// inside the grid (the reference writes past the array when a box overhangs)
void cuboid(Raster &r, const Sh &s)
{
    if ((s.theta == 0) && (s.phi == 0) && (s.psi == 0)) {
        for (int i = 0; i < s.ia; ++i)
            for (int j = 0; j < s.jb; ++j)
                for (int k = 0; k < s.kc; ++k) r.put(i + s.ix0, j + s.jy0, k + s.kz0, s.mat);
        return;
    }
    const double ct = cos(s.theta), st = sin(s.theta), cp = cos(s.phi), sp = sin(s.phi);
    const double cs = cos(s.psi), ss = sin(s.psi);
    for (double x = 0; x < s.a; x = x + (r.dx / 2.0))
        for (double y = 0; y < s.b; y = y + (r.dy / 2.0))
            for (double z = 0; z < s.c; z = z + (r.dz / 2.0)) {
                // rotations about x (theta), y (phi), z (psi)
                const double x1 = x;
                const double y1 = ct * (y) - st * (z);
                const double z1 = st * (y) + ct * (z);
                const double x2 = cp * (x1) + sp * (z1);
                const double y2 = y1;
                const double z2 = -sp * (x1) + cp * (z1);
                const double x3 = cs * (x2) - ss * (y2);
                const double y3 = ss * (x2) + cs * (y2);
                const double z3 = z2;
                const int i3 = (int)((x3 + s.x0) / r.dx);
                const int j3 = (int)((y3 + s.y0) / r.dy);
                const int k3 = (int)((z3 + s.z0) / r.dz);
                if ((i3 >= 0) && (i3 <= r.nx) && (j3 >= 0) && (j3 <= r.ny) && (k3 >= 0) && (k3 <= r.nz))
                    r.ids[r.at(i3, j3, k3)] = (uint8_t)s.mat;
            }
}

// ellipsoid(), Structure.cpp:205-221 (cells i<Nx, j<Ny, k<Nz); the scan is
// limited to the shape's bounding box widened by two cells, which leaves the
// predicate and its result unchanged
void ellipsoid(Raster &r, const Sh &s)
{
    const double a2 = s.a * s.a, b2 = s.b * s.b, c2 = s.c * s.c;
    auto lo = [](double c, double h, double d) { return (int)floor((c - fabs(h)) / d) - 2; };
    auto hi = [](double c, double h, double d) { return (int)ceil((c + fabs(h)) / d) + 2; };
    const int i0 = lo(s.x0, s.a, r.dx) < 0 ? 0 : lo(s.x0, s.a, r.dx);
    const int j0 = lo(s.y0, s.b, r.dy) < 0 ? 0 : lo(s.y0, s.b, r.dy);
    const int k0 = lo(s.z0, s.c, r.dz) < 0 ? 0 : lo(s.z0, s.c, r.dz);
    const int i1 = hi(s.x0, s.a, r.dx) > r.nx ? r.nx : hi(s.x0, s.a, r.dx);
    const int j1 = hi(s.y0, s.b, r.dy) > r.ny ? r.ny : hi(s.y0, s.b, r.dy);
    const int k1 = hi(s.z0, s.c, r.dz) > r.nz ? r.nz : hi(s.z0, s.c, r.dz);
    for (int i = i0; i < i1; ++i)
        for (int j = j0; j < j1; ++j)
            for (int k = k0; k < k1; ++k) {
                const double X = (double)i * r.dx - s.x0, Y = (double)j * r.dy - s.y0, Z = (double)k * r.dz - s.z0;
                const double temp = X * X / a2 + Y * Y / b2 + Z * Z / c2;
                if (temp <= 1.0) r.ids[r.at(i, j, k)] = (uint8_t)s.mat;
            }
}

// cylinder(), Structure.cpp:223-236: kc planes from kz0, disc test over i<Nx, j<Ny
void cylinder(Raster &r, const Sh &s)
{
    const double a2 = s.a * s.a, b2 = s.b * s.b;
    for (int k = 0; k < s.kc; ++k)
        for (int i = 0; i < r.nx; ++i)
            for (int j = 0; j < r.ny; ++j) {
                const double X = (double)i * r.dx - s.x0, Y = (double)j * r.dy - s.y0;
                const double temp = X * X / a2 + Y * Y / b2;
                if (temp <= 1.0) r.put(i, j, k + s.kz0, s.mat);
            }
}

// multishape(), Structure.cpp:238-307: counts in theta/phi/psi, pitch in a/b/c
void multishape(Raster &r, const Sh &multi, const Sh &single, int type)
{
    Sh m = single;
    for (int i = 0; i < multi.theta; ++i) {
        m.x0 = multi.x0 + i * multi.a;
        m.ix0 = (int)(m.x0 / r.dx);
        for (int j = 0; j < multi.phi; ++j) {
            m.y0 = multi.y0 + j * multi.b;
            m.jy0 = (int)(m.y0 / r.dy);
            for (int k = 0; k < multi.psi; ++k) {
                m.z0 = multi.z0 + k * multi.c;
                m.kz0 = (int)(m.z0 / r.dz);
                if (type == CPS_SHAPE_CUBOID) cuboid(r, m);
                else if (type == CPS_SHAPE_ELLIPSOID) ellipsoid(r, m);
                else if (type == CPS_SHAPE_CYLINDER) cylinder(r, m);
            }
        }
    }
}

}  // namespace

extern "C" cps_status cps_mesh_rasterize(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                         int32_t nshapes, const cps_shape *shapes, uint8_t *ids, int32_t keep)
{
    if (nx < 2 || ny < 2 || nz < 2 || !(dx > 0) || !(dy > 0) || !(dz > 0) || !ids || nshapes < 0 ||
        (nshapes > 0 && !shapes)) {
        set_error("cps_mesh_rasterize: invalid grid, spacing or shape list");
        return CPS_E_INVALID;
    }
    Raster r{nx, ny, nz, dx, dy, dz, ids};
    if (!keep) memset(ids, 0, (size_t)(nx + 1) * (ny + 1) * (nz + 1));
    for (int s = 0; s < nshapes; ++s) {
        const cps_shape &sh = shapes[s];
        if (sh.material_index < 0 || sh.material_index > 255) {
            set_error("cps_mesh_rasterize: material index outside 0..255");
            return CPS_E_INVALID;
        }
        const Sh h = make_shape(sh, r);
        switch (sh.type) {
        case CPS_SHAPE_CUBOID: cuboid(r, h); break;
        case CPS_SHAPE_ELLIPSOID: ellipsoid(r, h); break;
        case CPS_SHAPE_CYLINDER: cylinder(r, h); break;
        case CPS_SHAPE_MULTI: {
            const int t = sh.material_index;  // template shape index (Structure.cpp:150-152)
            if (t < 0 || t >= nshapes || shapes[t].type == CPS_SHAPE_MULTI) {
                set_error("cps_mesh_rasterize: multi shape refers to an invalid template");
                return CPS_E_INVALID;
            }
            multishape(r, h, make_shape(shapes[t], r), shapes[t].type);
            break;
        }
        default:
            set_error("cps_mesh_rasterize: unknown shape type");
            return CPS_E_INVALID;
        }
    }
    return CPS_OK;
}

extern "C" cps_status cps_port_points_plain(int32_t nx, int32_t ny, int32_t nz, double dx, double dy, double dz,
                                            char normal, double position, double w1, double w2, double h1,
                                            double h2, int32_t *count, int32_t *ijk)
{
    if (!count) { set_error("cps_port_points_plain: count is NULL"); return CPS_E_INVALID; }
    int i1, i2, j1, j2, k1, k2;
    if (normal == 'x') {
        i1 = i2 = (int)(position / dx); j1 = (int)(w1 / dy); j2 = (int)(w2 / dy); k1 = (int)(h1 / dz); k2 = (int)(h2 / dz);
    } else if (normal == 'y') {
        j1 = j2 = (int)(position / dy); i1 = (int)(w1 / dx); i2 = (int)(w2 / dx); k1 = (int)(h1 / dz); k2 = (int)(h2 / dz);
    } else if (normal == 'z') {
        k1 = k2 = (int)(position / dz); i1 = (int)(w1 / dx); i2 = (int)(w2 / dx); j1 = (int)(h1 / dy); j2 = (int)(h2 / dy);
    } else {
        set_error("cps_port_points_plain: normal must be 'x', 'y' or 'z'");
        return CPS_E_INVALID;
    }
    if (i2 < i1 || j2 < j1 || k2 < k1 || i1 < 0 || j1 < 0 || k1 < 0 || i2 > nx || j2 > ny || k2 > nz) {
        set_error("cps_port_points_plain: port rectangle outside the grid");
        return CPS_E_INVALID;
    }
    const int64_t n = (int64_t)(i2 - i1 + 1) * (j2 - j1 + 1) * (k2 - k1 + 1);
    if (!ijk) { *count = (int32_t)n; return CPS_OK; }
    if (*count < n) { set_error("cps_port_points_plain: output too small"); return CPS_E_INVALID; }
    int64_t q = 0;
    // loop orders of Ports.cpp:242-293: the first in-plane axis varies fastest
    if (normal == 'x') {
        for (int k = k1; k <= k2; k++) for (int j = j1; j <= j2; j++) { ijk[3 * q] = i1; ijk[3 * q + 1] = j; ijk[3 * q + 2] = k; ++q; }
    } else if (normal == 'y') {
        for (int k = k1; k <= k2; k++) for (int i = i1; i <= i2; i++) { ijk[3 * q] = i; ijk[3 * q + 1] = j1; ijk[3 * q + 2] = k; ++q; }
    } else {
        for (int j = j1; j <= j2; j++) for (int i = i1; i <= i2; i++) { ijk[3 * q] = i; ijk[3 * q + 1] = j; ijk[3 * q + 2] = k1; ++q; }
    }
    *count = (int32_t)n;
    return CPS_OK;
}

extern "C" cps_status cps_port_points_spherical(int32_t nx, int32_t ny, int32_t nz, double dx, double dy,
                                                double dz, double r, double xc, double yc, double zc,
                                                double theta1_deg, double theta2_deg, double phi1_deg,
                                                double phi2_deg, int32_t *count, int32_t *ijk)
{
    if (!count || !(r > 0)) { set_error("cps_port_points_spherical: bad radius or count"); return CPS_E_INVALID; }
    const double theta1 = theta1_deg * kPi / 180.0, theta2 = theta2_deg * kPi / 180.0;
    const double phi1 = phi1_deg * kPi / 180.0, phi2 = phi2_deg * kPi / 180.0;
    const double dphi = dx / r, dtheta = dz / r;  // Ports.cpp:66-67
    int64_t n = 0;
    for (double phi = phi1; phi <= phi2; phi = phi + dphi)
        for (double theta = theta1; theta <= theta2; theta = theta + dtheta) {
            if (ijk) {
                if (n >= *count) { set_error("cps_port_points_spherical: output too small"); return CPS_E_INVALID; }
                const int i = (int)((xc + r * sin(theta) * cos(phi)) / dx);
                const int j = (int)((yc + r * sin(theta) * sin(phi)) / dy);
                const int k = (int)((zc + r * cos(theta)) / dz);
                if (i < 0 || j < 0 || k < 0 || i > nx || j > ny || k > nz) {
                    set_error("cps_port_points_spherical: sphere leaves the grid");
                    return CPS_E_INVALID;
                }
                ijk[3 * n] = i; ijk[3 * n + 1] = j; ijk[3 * n + 2] = k;
            }
            ++n;
        }
    *count = (int32_t)n;
    return CPS_OK;
}
