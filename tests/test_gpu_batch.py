"""Batched engine (cps_batch_*): grids of uneven size and different material
mixes stepped together give exactly the results of each grid stepped alone
on the fused path, whatever the tiling, persistence, graph replay, chunking
or co-tenants."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _members(steps):
    """Four grids covering the sweep classes: gain + CPML + spherical port DFT
    (anisotropic box), Drude-Lorentz + TF/SF + six planar port DFTs,
    dielectric + CPML + line port without DFT, and one without CPML."""
    m = [decks.config4_member(40, 48, 36, seed=1, steps=steps, nfreq=4),
         decks.config2(n=40, steps=steps, nfreq=3),
         decks.config1(n=36, steps=steps)]
    bare = decks.config1(n=34, steps=steps)
    bare.pml = None
    bare.ports = []
    m.append(bare)
    return m


def _grid(dk, prec):
    import cpsfdtd_b200 as cps
    return cps.Grid.from_deck(dk, prec)


def _state(g):
    out = {"fields": g.fields()}
    out["dft"] = [g.port_dft(p, raw=True).copy() for p in range(len(g.ports)) if g.ports[p][2] > 0]
    out["last"] = [g.port_last(p) for p in range(len(g.ports))]
    out["step"] = g.get_step()
    return out


def _alone(dk, prec, nsteps):
    import cpsfdtd_b200 as cps
    g = _grid(dk, prec)
    g.step(nsteps, cps.FUSED)
    s = _state(g)
    g.close()
    return s


def _same(a, b, what=""):
    assert a["step"] == b["step"], what
    for c in range(6):
        assert np.array_equal(a["fields"][c], b["fields"][c]), f"{what} field {c}: rel {rel_l2(a['fields'][c], b['fields'][c])}"
    for x, y in zip(a["dft"], b["dft"]):
        assert np.array_equal(x, y), f"{what} port DFT: rel {rel_l2(x, y)}"
    for x, y in zip(a["last"], b["last"]):
        assert np.array_equal(x, y), f"{what} port sample"


@pytest.mark.parametrize("tile", [(4, 8, 0, True), (8, 16, 1, True), (4, 32, 1, False), (8, 8, 0, False),
                                  (4, 8, 2, True), (8, 64, 2, False)])
def test_batch_equals_alone(tile):
    import cpsfdtd_b200 as cps
    steps = 70  # alone, port rings fold at 64 samples; in the batch, at every chunk
    dks = _members(steps)
    ref = [_alone(dk, cps.FP32, steps) for dk in dks]
    b = cps.Batch(cps.FP32)
    rows, planes, pers, graph = tile
    b.set_tile(rows, planes, pers)
    b.set_graph(graph)
    gs = [_grid(dk, cps.FP32) for dk in dks]
    for g in gs:
        b.add(g)
    assert b.info()[0] == len(gs)
    b.step(20)   # launched directly
    b.step(20)   # the same chunk again: captured into a graph and replayed
    b.step(30)
    b.sync()
    assert b.launches() > 0
    for n, g in enumerate(gs):
        _same(ref[n], _state(g), f"member {n} tile {tile}")
    b.close()


def test_batch_membership_changes_and_interleaved_alone_steps():
    import cpsfdtd_b200 as cps
    dks = _members(120)
    ref_a = _alone(dks[0], cps.FP32, 90)
    ref_b = _alone(dks[1], cps.FP32, 30)
    ref_c = _alone(dks[2], cps.FP32, 60)
    b = cps.Batch(cps.FP32)
    ga, gb, gc = (_grid(dk, cps.FP32) for dk in dks[:3])
    b.add(ga)
    b.add(gb)
    b.step(30)
    b.remove(gb)
    b.add(gc)
    b.step(20)
    ga.step(10, cps.FUSED)   # a member stepped on its own between batch steps
    gc.step(10, cps.FUSED)
    b.step(30)
    b.sync()
    _same(ref_a, _state(ga), "a")
    _same(ref_b, _state(gb), "b")
    _same(ref_c, _state(gc), "c")


@pytest.mark.parametrize("tile", [(4, 16, 2), (4, 8, 0)])
def test_batch_fp64_equals_alone_and_oracle(oracle_mod, tile):
    """FP64 through both sweep forms: the member's own launches (the default)
    and the class launches over the shared tile table."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=36, steps=50, nfreq=2)
    ref = _alone(dk, cps.FP64, 50)
    b = cps.Batch(cps.FP64)
    b.set_tile(*tile)
    g = _grid(dk, cps.FP64)
    b.add(g)
    b.step(50)
    b.sync()
    got = _state(g)
    _same(ref, got, "fp64")
    ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    o = oracle_mod.Oracle.from_deck(dk, ids, [cps.port_points(dk, p) for p in dk.ports])
    o.step(50)
    for c in range(6):
        assert rel_l2(got["fields"][c], o.field(c)) < 1e-10


def test_batch_rejects_bad_members():
    import cpsfdtd_b200 as cps
    b = cps.Batch(cps.FP32)
    g64 = _grid(decks.config1(n=36, steps=5), cps.FP64)
    with pytest.raises(cps.CpsError):
        b.add(g64)
    small = _grid(decks.config1(n=24, steps=5), cps.FP32)
    with pytest.raises(cps.CpsError):
        b.add(small)
    g = _grid(decks.config1(n=36, steps=5), cps.FP32)
    b.add(g)
    with pytest.raises(cps.CpsError):
        b.add(g)
    with pytest.raises(cps.CpsError):
        b.set_tile(5, 8, 0)
    with pytest.raises(cps.CpsError):
        b.set_tile(4, 8, 3)


def test_batch_autotune_cache(tmp_path):
    import cpsfdtd_b200 as cps
    dks = _members(200)
    b = cps.Batch(cps.FP32)
    gs = [_grid(dk, cps.FP32) for dk in dks]
    for g in gs:
        b.add(g)
    cache = str(tmp_path / "tune.txt")
    ran = b.autotune(cache, trial_steps=2)
    assert ran == 24 * 3  # rows {4, 8} x planes {8, 16, 32, 64} x launch modes {0, 1, 2}, 1 + 2 steps each
    key = b.tune_key()
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and lines[0].split()[0] == key
    chosen = b.get_tile()
    # a second batch with the same key reads the cache and runs nothing
    b2 = cps.Batch(cps.FP32)
    gs2 = [_grid(dk, cps.FP32) for dk in dks]
    for g in gs2:
        b2.add(g)
    assert b2.autotune(cache, trial_steps=2) == 0
    assert b2.get_tile() == chosen
    # the tuning steps were real steps: members match grids stepped alone
    for dk, g in zip(dks, gs):
        _same(_alone(dk, cps.FP32, ran), _state(g), "autotuned")


def test_batch_with_a_large_member_equals_alone():
    """A member of more than 4 M cells is swept by its own launches inside the
    batch's chunk; it and a small co-member still match their alone runs."""
    import cpsfdtd_b200 as cps
    steps = 70
    big = decks.config2(n=164, steps=steps, nfreq=2)
    small = decks.config4_member(40, 48, 36, seed=2, steps=steps, nfreq=3)
    ref = [_alone(dk, cps.FP32, steps) for dk in (big, small)]
    b = cps.Batch(cps.FP32)
    gs = [_grid(dk, cps.FP32) for dk in (big, small)]
    for g in gs:
        b.add(g)
    b.step(30)
    b.step(30)
    b.step(10)
    b.sync()
    for n, g in enumerate(gs):
        _same(ref[n], _state(g), f"member {n}")


def test_chunked_fused_steps_equal_direct_launches():
    """A grid of 4 Mi cells or more steps the fused path as one-grid batch
    chunks (graph replay); results equal the direct launches bit for bit,
    across chunk boundaries, a reset and the port DFTs."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=164, steps=1, nfreq=3)
    a, b = _grid(dk, cps.FP32), _grid(dk, cps.FP32)
    b.set_chunked(False)
    for g in (a, b):
        g.step(70, cps.FUSED)
        g.step(64, cps.FUSED)
        g.step(3, cps.FUSED)
    ra, rb = _state(a), _state(b)
    _same(rb, ra, "chunked")
    for g in (a, b):
        g.reset(1)
        g.step(65, cps.FUSED)
    _same(_state(b), _state(a), "after reset")
    assert a.launches() > 0
