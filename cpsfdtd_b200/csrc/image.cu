// image.cu -- headless field images: a plane of one field component (or of
// |E|^2) cut on the device, and PNG files with the colour map of the
// reference's OutImage (OutImage.cpp:140-216) written without any display or
// image library.  The PNG is RGB, 8 bits, one IDAT holding a zlib stream of
// stored (uncompressed) deflate blocks; CRC-32 and Adler-32 as the PNG and
// zlib specifications define them.
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "grid.h"

namespace cps {

namespace {

// out[u][v]: (u, v) = (j, k) for a plane of x, (i, k) of y, (i, j) of z
template <typename T>
__global__ void k_slice(FieldView<T> f, int what, int axis, int index, int nu, int nv, double *out)
{
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= (int64_t)nu * nv) return;
    const int u = (int)(q / nv), v = (int)(q % nv);
    int i, j, k;
    if (axis == 0) { i = index; j = u; k = v; }
    else if (axis == 1) { i = u; j = index; k = v; }
    else { i = u; j = v; k = index; }
    const int64_t g = f.d.idx(i, j, k);
    double r;
    if (what == 6) {
        const double ex = (double)f.Ex[g], ey = (double)f.Ey[g], ez = (double)f.Ez[g];
        r = ex * ex + ey * ey + ez * ez;
    } else {
        const T *F[6] = {f.Ex, f.Ey, f.Ez, f.Hx, f.Hy, f.Hz};
        r = (double)F[what][g];
    }
    out[q] = r;
}

struct MediaTable {
    double eps[256], mu[256];  // eps0 epsR and mu0 muR per medium
};

// electric and magnetic energy sums, FP64, one atomic pair per block
template <typename T>
__global__ void __launch_bounds__(256) k_energy(FieldView<T> f, MediaTable m, double *out)
{
    const Dims &d = f.d;
    const int64_t n = (int64_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
    double we = 0.0, wh = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(q % (d.nx + 1)), j = (int)((q / (d.nx + 1)) % (d.ny + 1)),
                  k = (int)(q / ((int64_t)(d.nx + 1) * (d.ny + 1)));
        const int64_t g = d.idx(i, j, k);
        const int id = f.id[g];
        const double ex = (double)f.Ex[g], ey = (double)f.Ey[g], ez = (double)f.Ez[g];
        const double hx = (double)f.Hx[g], hy = (double)f.Hy[g], hz = (double)f.Hz[g];
        we += m.eps[id] * (ex * ex + ey * ey + ez * ez);
        wh += m.mu[id] * (hx * hx + hy * hy + hz * hz);
    }
    __shared__ double se[8], sh[8];
    for (int o = 16; o > 0; o >>= 1) {
        we += __shfl_down_sync(0xffffffffu, we, o);
        wh += __shfl_down_sync(0xffffffffu, wh, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { se[w] = we; sh[w] = wh; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += se[q]; b += sh[q]; }
        atomicAdd(&out[0], a);
        atomicAdd(&out[1], b);
    }
}

struct CrcTable {
    uint32_t t[256];
    CrcTable()
    {
        for (uint32_t b = 0; b < 256; ++b) {
            uint32_t c = b;
            for (int s = 0; s < 8; ++s) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            t[b] = c;
        }
    }
};

uint32_t crc32_update(uint32_t crc, const unsigned char *p, size_t n)
{
    static const CrcTable table;  // built once, thread-safe
    for (size_t q = 0; q < n; ++q) crc = table.t[(crc ^ p[q]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<unsigned char> &v, uint32_t x)
{
    v.push_back((unsigned char)(x >> 24)); v.push_back((unsigned char)(x >> 16));
    v.push_back((unsigned char)(x >> 8)); v.push_back((unsigned char)x);
}

void chunk(std::vector<unsigned char> &png, const char *type, const std::vector<unsigned char> &data)
{
    put_be32(png, (uint32_t)data.size());
    const size_t at = png.size();
    png.insert(png.end(), type, type + 4);
    png.insert(png.end(), data.begin(), data.end());
    const uint32_t crc = crc32_update(0xFFFFFFFFu, png.data() + at, png.size() - at) ^ 0xFFFFFFFFu;
    put_be32(png, crc);
}

}  // namespace

}  // namespace cps

using namespace cps;

extern "C" cps_status cps_field_slice(cps_grid *g, int32_t what, int32_t axis, int32_t index, double *out)
{
    REQUIRE(g && out, CPS_E_INVALID, "cps_field_slice: NULL argument");
    REQUIRE(what >= 0 && what <= 6, CPS_E_INVALID, "cps_field_slice: what is a component 0..5 or 6 (|E|^2)");
    REQUIRE(axis >= 0 && axis <= 2, CPS_E_INVALID, "cps_field_slice: axis 0 (x), 1 (y) or 2 (z)");
    const Dims &d = g->d;
    const int n[3] = {d.nx, d.ny, d.nz};
    REQUIRE(index >= 0 && index <= n[axis], CPS_E_INVALID, "cps_field_slice: plane index outside the grid");
    cps_status s = flush_recorded(g);
    if (s) return s;
    const int nu = (axis == 0 ? d.ny : d.nx) + 1, nv = (axis == 2 ? d.ny : d.nz) + 1;
    const size_t bytes = (size_t)nu * nv * sizeof(double);
    double *d_out = nullptr;
    if ((s = dalloc(g, (void **)&d_out, bytes))) return s;
    const unsigned blocks = (unsigned)(((int64_t)nu * nv + 255) / 256);
    if (g->fp32) k_slice<float><<<blocks, 256, 0, g->stream>>>(field_view<float>(g), what, axis, index, nu, nv, d_out);
    else k_slice<double><<<blocks, 256, 0, g->stream>>>(field_view<double>(g), what, axis, index, nu, nv, d_out);
    g->launches++;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    dfree(g, d_out);
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("cps_field_slice: ") + cudaGetErrorString(e));
    return CPS_OK;
}

extern "C" cps_status cps_png_rgb(const char *path, int32_t nx, int32_t ny, const uint8_t *rgb)
{
    REQUIRE(path && rgb, CPS_E_INVALID, "cps_png_rgb: NULL argument");
    REQUIRE(nx >= 1 && ny >= 1 && nx <= 1 << 15 && ny <= 1 << 15, CPS_E_INVALID, "cps_png_rgb: bad image size");
    std::vector<unsigned char> raw((size_t)ny * (1 + 3 * (size_t)nx));
    for (int y = 0; y < ny; ++y) {
        unsigned char *row = raw.data() + (size_t)y * (1 + 3 * (size_t)nx);
        row[0] = 0;  // filter: none
        memcpy(row + 1, rgb + (size_t)y * 3 * nx, 3 * (size_t)nx);
    }
    // zlib stream of stored deflate blocks (at most 65535 bytes each)
    std::vector<unsigned char> z = {0x78, 0x01};
    uint32_t a = 1, b = 0;
    for (size_t q = 0; q < raw.size(); ++q) {
        a = (a + raw[q]) % 65521u;
        b = (b + a) % 65521u;
    }
    for (size_t off = 0;;) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((unsigned char)(len & 0xFF)); z.push_back((unsigned char)(len >> 8));
        z.push_back((unsigned char)(~len & 0xFF)); z.push_back((unsigned char)((~len >> 8) & 0xFF));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        off += len;
        if (last) break;
    }
    put_be32(z, (b << 16) | a);
    std::vector<unsigned char> png = {0x89, 'P', 'N', 'G', 0x0D, 0x0A, 0x1A, 0x0A};
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, (uint32_t)nx);
    put_be32(ihdr, (uint32_t)ny);
    ihdr.push_back(8);  // bit depth
    ihdr.push_back(2);  // colour type: RGB
    ihdr.push_back(0); ihdr.push_back(0); ihdr.push_back(0);
    chunk(png, "IHDR", ihdr);
    chunk(png, "IDAT", z);
    chunk(png, "IEND", {});
    FILE *f = fopen(path, "wb");
    REQUIRE(f, CPS_E_INVALID, std::string("cps_png_rgb: cannot write ") + path);
    const size_t w = fwrite(png.data(), 1, png.size(), f);
    const int c = fclose(f);
    REQUIRE(w == png.size() && c == 0, CPS_E_INVALID, std::string("cps_png_rgb: write failed for ") + path);
    return CPS_OK;
}

extern "C" cps_status cps_image_png(const char *path, int32_t nx, int32_t ny, const double *values, double cmin,
                                    double cmax)
{
    REQUIRE(path && values, CPS_E_INVALID, "cps_image_png: NULL argument");
    REQUIRE(nx >= 1 && ny >= 1 && nx <= 1 << 15 && ny <= 1 << 15, CPS_E_INVALID, "cps_image_png: bad image size");
    REQUIRE(cmax > cmin, CPS_E_INVALID, "cps_image_png: cmax must exceed cmin");
    // OutImage's colour map (OutImage.cpp:21-32, 146-172): black below cmin,
    // (254,254,254) above cmax, between them red, then yellow, then white ramps;
    // pixel (x, y) is values[x][y] (the reference's img(i, j) of dD[i][j])
    const double cthird = (cmax + cmin) / 3.0, c2third = (cmax + cthird) / 2.0;
    std::vector<uint8_t> rgb((size_t)ny * nx * 3);
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const double v = values[(size_t)x * ny + y];
            const int temp = (int)((v - cmin) * 254.0 / (cmax - cmin));
            uint8_t *px = rgb.data() + ((size_t)y * nx + x) * 3;
            if (v <= cmin) { px[0] = 0; px[1] = 0; px[2] = 0; }
            else if (v >= cmax) { px[0] = 254; px[1] = 254; px[2] = 254; }
            else if (v <= cthird) { px[0] = (uint8_t)temp; px[1] = 0; px[2] = 0; }
            else if (v > cthird && v <= c2third) { px[0] = 254; px[1] = (uint8_t)temp; px[2] = 0; }
            else { px[0] = 254; px[1] = 254; px[2] = (uint8_t)temp; }
        }
    return cps_png_rgb(path, nx, ny, rgb.data());
}

extern "C" cps_status cps_grid_energy(cps_grid *g, double *electric, double *magnetic)
{
    REQUIRE(g && electric && magnetic, CPS_E_INVALID, "cps_grid_energy: NULL argument");
    REQUIRE(g->nmedia > 0 && g->ids_set, CPS_E_STATE, "cps_grid_energy: media and IDs are not set");
    cps_status s = flush_recorded(g);
    if (s) return s;
    MediaTable m;
    for (int q = 0; q < 256; ++q) {
        m.eps[q] = kEps0 * (q < g->nmedia ? g->eps_r[q] : 1.0);
        m.mu[q] = kMu0 * (q < g->nmedia ? g->mu_r[q] : 1.0);
    }
    double *d_out = nullptr;
    if ((s = dalloc(g, (void **)&d_out, 2 * sizeof(double)))) return s;
    double h[2] = {0.0, 0.0};
    cudaError_t e = cudaMemsetAsync(d_out, 0, 2 * sizeof(double), g->stream);
    if (e == cudaSuccess) {
        if (g->fp32) k_energy<float><<<148 * 8, 256, 0, g->stream>>>(field_view<float>(g), m, d_out);
        else k_energy<double><<<148 * 8, 256, 0, g->stream>>>(field_view<double>(g), m, d_out);
        g->launches++;
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, g->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(g->stream);
    dfree(g, d_out);
    REQUIRE(e == cudaSuccess, CPS_E_CUDA, std::string("cps_grid_energy: ") + cudaGetErrorString(e));
    const double dV = g->desc.dx * g->desc.dy * g->desc.dz;
    *electric = 0.5 * h[0] * dV;
    *magnetic = 0.5 * h[1] * dV;
    return CPS_OK;
}
