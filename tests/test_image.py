"""Headless images (OutImage without a display): the PNG writer and the
reference's colour map, checked by decoding the files; the drop-in OutImage
class; on the GPU, the device plane cut against the downloaded field."""
import os
import struct
import subprocess
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def read_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        kind, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(kind + body) & 0xFFFFFFFF
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype = hdr[:4]
    assert depth == 8 and ctype == 2
    raw = zlib.decompress(idat)
    rows = np.frombuffer(raw, np.uint8).reshape(h, 1 + 3 * w)
    assert (rows[:, 0] == 0).all()
    return rows[:, 1:].reshape(h, w, 3)


def colour_map(v, cmin, cmax):
    """OutImage.cpp:146-172 restated with numpy."""
    third = (cmax + cmin) / 3.0
    two = (cmax + third) / 2.0
    temp = np.trunc((v - cmin) * 254.0 / (cmax - cmin)).astype(np.int64)
    rgb = np.zeros(v.shape + (3,), np.int64)
    mid = (v > cmin) & (v < cmax)
    b1 = mid & (v <= third)
    b2 = mid & (v > third) & (v <= two)
    b3 = mid & (v > two)
    rgb[v >= cmax] = 254
    rgb[b1, 0] = temp[b1]
    rgb[b2, 0] = 254
    rgb[b2, 1] = temp[b2]
    rgb[b3, 0] = 254
    rgb[b3, 1] = 254
    rgb[b3, 2] = temp[b3]
    return rgb.astype(np.uint8)


def test_png_colour_map_round_trip(tmp_path):
    import cpsfdtd_b200 as cps
    rng = np.random.default_rng(3)
    v = rng.uniform(-0.2, 1.3, size=(97, 301))  # 97 wide, 301 high: several deflate blocks
    path = str(tmp_path / "f.png")
    cps.image_png(path, v, 0.0, 1.0)
    img = read_png(path)
    assert img.shape == (301, 97, 3)
    assert np.array_equal(img, colour_map(v, 0.0, 1.0).transpose(1, 0, 2))
    with pytest.raises(cps.CpsError):
        cps.image_png(path, v, 1.0, 1.0)


def test_dropin_outimage_writes_the_reference_files(tmp_path):
    import cpsfdtd_b200 as cps
    cps.lib()
    src = tmp_path / "oi.cpp"
    src.write_text(r'''
#include "cpsfdtd_classes.hpp"
int main(int, char **argv)
{
    const int nx = 40, ny = 30;
    double **d = new double *[nx];
    short **s = new short *[nx];
    for (int i = 0; i < nx; ++i) {
        d[i] = new double[ny];
        s[i] = new short[ny];
        for (int j = 0; j < ny; ++j) { d[i][j] = (i + j) / 70.0; s[i][j] = (short)((i / 4 + j / 5) % 10); }
    }
    OutImage img(nx, ny, 5, 0.0, 1.0, argv[1]);
    img.plot_save(d, 10);
    img.plot_save(d, 11);  // not a multiple of the save modulus: nothing written
    img.structure_plot_save(s);
    return 0;
}
''')
    exe = str(tmp_path / "oi")
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                        "-L", os.path.join(ROOT, "cpsfdtd_b200"), "-lcpsfdtd",
                        "-Wl,-rpath," + os.path.join(ROOT, "cpsfdtd_b200"), "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    base = str(tmp_path / "Ez")
    r = subprocess.run([exe, base], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert sorted(os.listdir(tmp_path)) == ["Ez000002.png", "Ez_structure.png", "oi", "oi.cpp"]
    d = np.add.outer(np.arange(40), np.arange(30)) / 70.0
    assert np.array_equal(read_png(base + "000002.png"), colour_map(d, 0.0, 1.0).transpose(1, 0, 2))
    table = np.array([[254, 254, 254], [254, 0, 0], [0, 0, 254], [0, 254, 0], [0, 0, 0], [254, 254, 0],
                      [0, 254, 254], [254, 0, 254], [127, 0, 254], [0, 127, 254]], np.uint8)
    ids = (np.arange(40)[:, None] // 4 + np.arange(30)[None, :] // 5) % 10
    assert np.array_equal(read_png(base + "_structure.png"), table[ids].transpose(1, 0, 2))


@pytest.mark.gpu
def test_field_slice_equals_download():
    import cpsfdtd_b200 as cps
    from cpsfdtd_b200 import decks
    dk = decks.config2(n=40, steps=1, nfreq=1)
    for prec in (cps.FP32, cps.FP64):
        g = cps.Grid.from_deck(dk, prec)
        g.step(25, cps.FUSED)
        f = [g.field(c) for c in range(6)]
        inten = f[0] ** 2 + f[1] ** 2 + f[2] ** 2
        for axis, index in ((0, 7), (1, 20), (2, 33)):
            for what in range(7):
                want = (inten if what == 6 else f[what]).take(index, axis=axis)
                got = g.slice(what, axis, index)
                assert np.allclose(got, want, rtol=1e-12, atol=0) if what == 6 else np.array_equal(got, want)
        g.close()


@pytest.mark.gpu
def test_grid_energy_equals_host_sum():
    import cpsfdtd_b200 as cps
    from cpsfdtd_b200 import decks
    dk = decks.config1(n=40, steps=1)
    eps0, mu0 = 8.8541878176e-12, 1.2566370614e-6
    for prec in (cps.FP32, cps.FP64):
        g = cps.Grid.from_deck(dk, prec)
        g.step(30, cps.FUSED)
        ids = g.download_ids()
        epsr = np.array([m[0] for m in dk.media])[ids]
        mur = np.array([m[1] for m in dk.media])[ids]
        f = [g.field(c) for c in range(6)]
        dv = dk.dx * dk.dy * dk.dz
        want_e = 0.5 * dv * eps0 * np.sum(epsr * (f[0] ** 2 + f[1] ** 2 + f[2] ** 2))
        want_h = 0.5 * dv * mu0 * np.sum(mur * (f[3] ** 2 + f[4] ** 2 + f[5] ** 2))
        got_e, got_h = g.energy()
        assert want_e > 0 and want_h > 0
        assert abs(got_e - want_e) <= 1e-12 * want_e and abs(got_h - want_h) <= 1e-12 * want_h
        g.close()
