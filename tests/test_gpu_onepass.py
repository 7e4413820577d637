"""The one-pass step (CPS_PATH_ONEPASS): H and E of a step in one sweep into a
second buffer set.  Against the two-sweep fused path on the same grid, across
tile shapes, grid edges that are not tile multiples, mixed paths and batches;
parity with the oracle is in test_gpu_parity.py."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _state(g):
    out = [g.field(c) for c in range(6)]
    out += [g.port_last(p) for p in range(len(g.ports))]
    out += [g.port_dft(p) for p in range(len(g.ports)) if g.ports[p][2] > 0]
    return out


def _run(dk, prec, path, steps, tile=None, ids=None):
    import cpsfdtd_b200 as cps
    g = cps.Grid.from_deck(dk, prec, ids=ids)
    if tile:
        g.set_tile(*tile)
    g.step(steps, path)
    return g


DECKS = {
    "dispersive": lambda: decks.config2(n=56, steps=1, nfreq=4),
    "dielectric_sources": lambda: decks.config1(n=44, steps=1),
    "laser": lambda: decks.config4_member(72, 40, 36, seed=5, steps=1, nfreq=3),
}


@pytest.mark.parametrize("name", sorted(DECKS))
@pytest.mark.parametrize("tile", [(8, 8), (4, 16), (8, 64)])
def test_onepass_equals_two_sweeps(name, tile):
    """FP32: the one-pass step and the two fused sweeps do the same arithmetic
    per cell except the order of TF/SF terms at box edges; they agree to FP32
    rounding."""
    import cpsfdtd_b200 as cps
    dk = DECKS[name]()
    steps = 70
    a = _state(_run(dk, cps.FP32, cps.FUSED, steps, tile))
    b = _state(_run(dk, cps.FP32, cps.ONEPASS, steps, tile))
    for x, y in zip(a, b):
        assert rel_l2(x, y) < 1e-5


def test_onepass_fp64_ragged_grid_against_two_sweeps():
    """Edges that are not multiples of the tile (x 61, y 45, z 23 cells) and
    chunks of 5 planes: every boundary cell is carried through."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    dk.nx, dk.ny, dk.nz = 61, 45, 23
    dk.pml["npml"] = [4] * 6
    dk.tfsf["n6"] = [8, 8, 8, 8, 5, 5]
    dk.shapes = [s for s in dk.shapes][:3]
    dk.ports = []
    a = _state(_run(dk, cps.FP64, cps.FUSED, 60, (8, 5)))
    b = _state(_run(dk, cps.FP64, cps.ONEPASS, 60, (8, 5)))
    for x, y in zip(a, b):
        assert rel_l2(x, y) < 1e-13


def test_paths_mix_and_state_reads():
    """One-pass, fused and plain steps in any order on one grid, with reads,
    uploads and a reset between them, follow the FP64 fused run."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=48, steps=1, nfreq=3)
    ref = _run(dk, cps.FP64, cps.FUSED, 40)
    g = cps.Grid.from_deck(dk, cps.FP64)
    g.step(7, cps.ONEPASS)
    g.step(5, cps.FUSED)
    ex = g.field(0)
    g.set_field(0, ex)  # an upload between one-pass steps lands in the current buffer
    g.step(9, cps.ONEPASS)
    g.step(3, cps.PLAIN)
    g.step(16, cps.ONEPASS)
    assert g.nonfinite() == 0
    for x, y in zip(_state(ref), _state(g)):
        assert rel_l2(x, y) < 1e-11
    g.reset(1)
    g.step(40, cps.ONEPASS)
    for x, y in zip(_state(ref), _state(g)):
        assert rel_l2(x, y) < 1e-11


def test_batch_after_onepass_steps():
    """A grid stepped one-pass (its buffers swapped) then stepped in a batch
    matches a grid stepped fused throughout."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    ref = _run(dk, cps.FP32, cps.FUSED, 50)
    g = cps.Grid.from_deck(dk, cps.FP32)
    b = cps.Batch(cps.FP32)
    b.add(g)
    b.step(10)
    b.sync()
    g.step(11, cps.ONEPASS)  # odd: the second buffer set is current
    b.step(20)
    b.sync()
    g.step(9, cps.ONEPASS)
    for x, y in zip(_state(ref), _state(g)):
        assert rel_l2(x, y) < 1e-5
    b.close()


def test_dispersive_ids_without_the_module_are_held():
    """ID-2 cells keep their E when no Drude-Lorentz module is set (the
    reference's BasicEFieldUpdate skips them), on both paths."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    dk.dl = None
    a = _state(_run(dk, cps.FP32, cps.FUSED, 30))
    b = _state(_run(dk, cps.FP32, cps.ONEPASS, 30))
    for x, y in zip(a, b):
        assert rel_l2(x, y) < 1e-5
