"""Parity at the workloads' stated sizes, through the C ABI.

  C1, 96^3 x 1000 steps (sphere scatterer, CPML 10, dipole, line port): the
      FP64 plain path equals the oracle bit for bit; the FP64 fused and
      one-pass paths are within 1e-10 and the FP32 paths within 1e-4
      relative L2 on all six fields and the port samples.  The oracle is
      pinned to the reference's own code (BasicFDTD.cpp:25-84,
      CPML.cpp:529-689, Ports.cpp:201-353) by the golden fixtures.
  C2, 256^3 x 4000 steps (Drude-Lorentz spheres, TF/SF beam, six ports with
      64-frequency DFTs): the oracle needs minutes here, so the FP64 fused
      path stands for it after matching the FP64 plain path (<= 1e-10, the
      form the oracle pins); FP32 fused against FP64: fields, port DFT,
      spectrum and resonance shift within 1e-4.
  C3, 384^3, the first 2000 of its 20000 steps (four-level gain crystal,
      CPML 16, spherical port r = 150 with a 32-frequency DFT): as C2, plus
      the gain populations of the FP32 path.
  C4, the largest ensemble member (128^3, CPML 8, gain) for its full 5000
      steps inside a batch of three: FP32 batched against FP64 alone."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import accuracy, decks

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-4


def _fields(g):
    return [g.field(c) for c in range(6)]


def _run(dk, prec, path, ids=None, pts=None):
    import cpsfdtd_b200 as cps
    g = cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts)
    g.step(dk.nsteps, path)
    g.sync()
    return g


def _report(a, b, dk):
    """accuracy of grid a against grid b (fields, every DFT port)"""
    ports = []
    for n, p in enumerate(dk.ports):
        if p.dft_freqs is not None:
            ports.append(accuracy.port_errors(p.dft_freqs, a.port_dft(n, raw=True), b.port_dft(n, raw=True)))
    return accuracy.summarize(accuracy.field_errors(_fields(a), _fields(b)), ports)


def _assert_within(rep, tol, tag):
    assert rep["field_rel_l2"] <= tol, f"{tag} fields {rep['field_rel_l2_per_component']}"
    for key in ("port_dft_rel_l2", "port_spectrum_rel_err"):
        if key in rep:
            assert rep[key] <= tol, f"{tag} {key} {rep[key]:.3e}"
    if "resonance_shift_rel" in rep:
        assert abs(rep["resonance_shift_rel"]) <= tol, f"{tag} shift {rep['resonance_shift_rel']:.3e}"


@pytest.fixture(scope="module")
def c1_oracle(oracle_mod):
    import cpsfdtd_b200 as cps
    dk = decks.config1(n=96, steps=1000)
    ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    o = oracle_mod.Oracle.from_deck(dk, ids, pts)
    o.step(dk.nsteps)
    return dk, ids, pts, o


def test_c1_full_size_fp64_plain_is_bit_exact(c1_oracle):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = c1_oracle
    g = _run(dk, cps.FP64, cps.PLAIN, ids, pts)
    for c in range(6):
        assert np.array_equal(g.field(c), o.field(c)), accuracy.NAMES[c]
    assert np.array_equal(g.port_last(0), o.port_last(0))
    g.close()


@pytest.mark.parametrize("prec,path", [(0, 1), (0, 2), (1, 1), (1, 2)],
                         ids=["fp64-fused", "fp64-onepass", "fp32-fused", "fp32-onepass"])
def test_c1_full_size_paths_match_oracle(prec, path, c1_oracle):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = c1_oracle
    tol = FP64_TOL if prec == cps.FP64 else FP32_TOL
    g = _run(dk, prec, path, ids, pts)
    for c in range(6):
        err = rel_l2(g.field(c), o.field(c))
        assert err <= tol, f"{accuracy.NAMES[c]} rel L2 {err:.3e}"
    err = rel_l2(g.port_last(0), o.port_last(0))
    assert err <= tol, f"port samples rel L2 {err:.3e}"
    g.close()


def _fp64_pair_and_fp32(dk):
    """FP64 plain, FP64 fused and FP32 fused runs of one deck"""
    import cpsfdtd_b200 as cps
    ids = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    plain = _run(dk, cps.FP64, cps.PLAIN, ids, pts)
    fused = _run(dk, cps.FP64, cps.FUSED, ids, pts)
    rep64 = _report(fused, plain, dk)
    plain.close()
    f32 = _run(dk, cps.FP32, cps.FUSED, ids, pts)
    rep32 = _report(f32, fused, dk)
    return fused, f32, rep64, rep32


def test_c2_full_size_fp32_within_bar():
    dk = decks.config2(n=256, steps=4000, nfreq=64)
    fused, f32, rep64, rep32 = _fp64_pair_and_fp32(dk)
    _assert_within(rep64, FP64_TOL, "C2 fp64 fused vs plain")
    _assert_within(rep32, FP32_TOL, "C2 fp32 vs fp64")
    fused.close()
    f32.close()


def test_c3_full_grid_fp32_within_bar():
    dk = decks.config3(n=384, steps=2000, seed=0, nfreq=32)
    fused, f32, rep64, rep32 = _fp64_pair_and_fp32(dk)
    _assert_within(rep64, FP64_TOL, "C3 fp64 fused vs plain")
    _assert_within(rep32, FP32_TOL, "C3 fp32 vs fp64")
    n64, n32 = fused.populations(), f32.populations()
    assert np.abs(n32 - n64).max() <= 1e-6
    assert np.abs(n32.sum(axis=1) - 2.0).max() < 1e-12  # conservation, FourLevelLaser.cpp:324
    fused.close()
    f32.close()


def test_c4_largest_member_batched_fp32_within_bar():
    import cpsfdtd_b200 as cps
    dks = [decks.config4_member(128, 128, 128, seed=7, steps=5000, nfreq=32),
           decks.config4_member(64, 96, 80, seed=8, steps=5000, nfreq=32),
           decks.config4_member(112, 64, 128, seed=9, steps=5000, nfreq=32)]
    b = cps.Batch(cps.FP32)
    gs = [cps.Grid.from_deck(d, cps.FP32) for d in dks]
    for g in gs:
        b.add(g)
    b.step(5000)
    b.sync()
    ref = _run(dks[0], cps.FP64, cps.FUSED)
    rep = _report(gs[0], ref, dks[0])
    _assert_within(rep, FP32_TOL, "C4 member fp32 batched vs fp64 alone")
    b.close()
    for g in gs:
        g.close()
    ref.close()
