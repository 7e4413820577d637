"""The single-routine entry points (the drop-in classes' calls) in orders
other than cps_step's, against the same oracle routines."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _pair(dk, oracle_mod, prec):
    import cpsfdtd_b200 as cps
    ids = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    return cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts), oracle_mod.Oracle.from_deck(dk, ids, pts)


def test_face_masked_tfsf_and_reordered_calls(oracle_mod):
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    g, o = _pair(dk, oracle_mod, cps.FP64)
    L = o.L
    for n in range(1, 31):
        g.op("h_bulk"); L.orc_op_h_bulk(o.h)
        g.op("h_pml"); L.orc_op_h_pml(o.h)
        g.op("tfsf_h", n, 0x3F); L.orc_op_tfsf_h(o.h, n)   # TF/SF after CPML: additive, same result
        g.op("e_bulk"); L.orc_op_e_bulk(o.h)
        g.op("dl"); L.orc_op_dl(o.h)
        g.op("tfsf_e", n, 0x3F); L.orc_op_tfsf_e(o.h, n)
        g.op("e_pml"); L.orc_op_e_pml(o.h)
    for c in range(6):
        assert rel_l2(g.field(c), o.field(c)) < 1e-10


def test_single_face_variant_only_touches_that_face(oracle_mod):
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    g, _ = _pair(dk, oracle_mod, cps.FP64)
    for n in range(1, 60):
        g.op("tfsf_e", n, 4)  # y1 face only (TF_SF::y1UpdateEField)
    ey = g.field(1)
    assert np.abs(ey).max() == 0  # the y1 face corrects Ex and Ez only
    ex = g.field(0)
    j1 = dk.tfsf["n6"][2]
    nz = np.argwhere(ex != 0)
    assert len(nz) and (nz[:, 1] == j1).all()


def test_gain_routines_called_separately(oracle_mod):
    import cpsfdtd_b200 as cps
    dk = decks.config3(n=32, steps=1, port=False)
    for prec, tol in ((cps.FP64, 1e-10), (cps.FP32, 1e-4)):
        g, o = _pair(dk, oracle_mod, prec)
        L = o.L
        for n in range(1, 41):
            g.op("h_bulk"); L.orc_op_h_bulk(o.h)
            g.op("h_pml"); L.orc_op_h_pml(o.h)
            g.op("e_bulk"); L.orc_op_e_bulk(o.h)
            g.op("gain_polarization"); L.orc_op_gain_p(o.h)
            g.op("gain_efield"); L.orc_op_gain_e(o.h)
            g.op("gain_populations"); L.orc_op_gain_n(o.h)
            g.op("sources", n); L.orc_op_sources(o.h, n)
            g.op("e_pml"); L.orc_op_e_pml(o.h)
        for c in range(6):
            assert rel_l2(g.field(c), o.field(c)) < tol


def test_reset_and_rerun_is_identical():
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=60, nfreq=4)
    g = cps.Grid.from_deck(dk, cps.FP32)
    g.step(60, cps.FUSED)
    a = [g.field(c) for c in range(6)] + [g.port_dft(0)]
    g.reset(dk.n0)
    g.step(60, cps.FUSED)
    b = [g.field(c) for c in range(6)] + [g.port_dft(0)]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_watchdog_counts_nonfinite():
    import cpsfdtd_b200 as cps
    dk = decks.config1(n=24, steps=1)
    g = cps.Grid.from_deck(dk, cps.FP32)
    assert g.nonfinite() == 0
    f = g.field(0)
    f[3, 4, 5] = np.nan
    f[6, 7, 8] = np.inf
    g.set_field(0, f)
    assert g.nonfinite() == 2


def test_errors_are_reported():
    import cpsfdtd_b200 as cps
    g = cps.Grid(16, 16, 16, 1e-8, 1e-8, 1e-8, precision=cps.FP32)
    with pytest.raises(cps.CpsError, match="media"):
        g.step(1)
    g.set_media([(1, 1, 0, 0)])
    with pytest.raises(cps.CpsError):
        g.upload_ids(np.full(g.shape3, 3, np.uint8))  # ID without a medium
    g.upload_ids(np.zeros(g.shape3, np.uint8))
    with pytest.raises(cps.CpsError, match="thickness"):
        g.pml_init(dict(npml=[4, 5, 4, 4, 4, 4], m=3, malp=1, kapmax=5, sig_ratio=1, alpmax=0.05))
    with pytest.raises(cps.CpsError):
        g.port_add(np.array([[0, 0, 17]]))


@pytest.mark.parametrize("name", ["shapes_pec", "c2", "c1"])
def test_device_rasterisation_equals_host(name):
    """cps_grid_rasterize gives every cell the ID cps_mesh_rasterize gives it:
    axis-aligned and rotated cuboids, cylinders, ellipsoids, multi shapes."""
    import cpsfdtd_b200 as cps
    import golden.golden_cases as gc
    dk = {"shapes_pec": gc.shapes_pec, "c2": lambda: decks.config2(n=96, steps=1, nfreq=1),
          "c1": lambda: decks.config1(n=64, steps=1)}[name]()
    host = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    g = cps.Grid(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.dt, cps.FP32)
    g.set_media(dk.media)
    g.rasterize(dk.shapes)
    assert np.array_equal(g.download_ids(), host)
    g.rasterize(dk.shapes[:1], keep=True)  # keep: the first shape painted again on top
    again = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, list(dk.shapes) + list(dk.shapes[:1]))
    assert np.array_equal(g.download_ids(), again)
    bad = decks.Shape(len(dk.media), "cuboid", 0, 0, 0, dk.dx, dk.dx, dk.dx)
    with pytest.raises(cps.CpsError):
        g.rasterize([bad])
