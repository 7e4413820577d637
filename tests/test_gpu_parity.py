"""CUDA engine against the FP64 oracle, through the C ABI.

Bars (per field component, relative L2 after N steps):
  FP64 grids, plain and fused paths: <= 1e-10
  FP32 grids, fused path:           <= 1e-4
Port samples and port DFT accumulators use the same bars."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks
import golden.golden_cases as gc

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32_TOL = 1e-4
NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def _setup(dk, oracle_mod):
    import cpsfdtd_b200 as cps
    ids = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    o = oracle_mod.Oracle.from_deck(dk, ids, pts)
    o.step(dk.nsteps)
    return ids, pts, o


def _c2_drude():
    """The dispersive deck with the single-pole Drude class (Drude.cpp) on its spheres."""
    dk = decks.config2(n=40, steps=100, nfreq=4)
    dk.dl = decks.drude_as_dl(decks.drude_params_metal())
    return dk


def _c3_three():
    """The laser deck with the three-level gain class (ThreeLevel.cpp, Lorentz
    oscillators) on its gain cells instead of the four-level one."""
    dk = decks.config3(n=40, steps=100, nfreq=4)
    dk.gain = None
    dk.three = decks.three_params_laser()
    return dk


CASES = {"c1": lambda: decks.config1(n=32, steps=120),
         # the reference's own CPML coefficients (literal) in an eps 2.25 CPML,
         # before that form starts to diverge
         "c3_literal_pml": lambda: gc.literal_pml(decks.config3(n=40, steps=100, nfreq=4)),
         "c2_drude": _c2_drude,
         "c3_three": _c3_three,
         "c2": lambda: decks.config2(n=48, steps=100, nfreq=8),
         # more frequencies than one 64-wide DFT tile holds (a ragged second tile)
         "c2_70freq": lambda: decks.config2(n=40, steps=60, nfreq=70),
         "c2_cw": gc.c2_cw,
         "c3": lambda: decks.config3(n=40, steps=100, nfreq=4),
         "shapes": gc.shapes_pec}


@pytest.fixture(scope="module")
def oracle_runs(oracle_mod):
    return {k: (f(), ) + _setup(f(), oracle_mod) for k, f in CASES.items()}


def _check(g, dk, pts, o, tol, tag):
    for c in range(6):
        want = o.field(c)
        if np.linalg.norm(want) == 0:
            assert np.abs(g.field(c)).max() == 0, f"{tag} {NAMES[c]} should stay zero"
            continue
        err = rel_l2(g.field(c), want)
        assert err <= tol, f"{tag} {NAMES[c]} rel L2 {err:.3e} > {tol:.0e}"
    for n, p in enumerate(dk.ports):
        err = rel_l2(g.port_last(n), o.port_last(n))
        assert err <= tol, f"{tag} port {n} samples rel L2 {err:.3e}"
        if p.dft_freqs is not None:
            ncomp = bin(p.dft_mask).count("1")
            want = o.port_dft(n, ncomp, len(p.dft_freqs))
            err = rel_l2(g.port_dft(n), want)
            assert err <= tol, f"{tag} port {n} DFT rel L2 {err:.3e}"


PATHS = {0: "plain", 1: "fused", 2: "onepass"}


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("path", [0, 1, 2], ids=["plain", "fused", "onepass"])
def test_fp64_matches_oracle(case, path, oracle_runs):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs[case]
    g = cps.Grid.from_deck(dk, cps.FP64, ids=ids, port_points_list=pts)
    g.step(dk.nsteps, path)
    _check(g, dk, pts, o, FP64_TOL, f"{case}/fp64/{PATHS[path]}")


@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("path", [1, 2], ids=["fused", "onepass"])
def test_fp32_matches_oracle(case, path, oracle_runs):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs[case]
    g = cps.Grid.from_deck(dk, cps.FP32, ids=ids, port_points_list=pts)
    g.step(dk.nsteps, path)
    _check(g, dk, pts, o, FP32_TOL, f"{case}/fp32/{PATHS[path]}")


def test_fp64_plain_is_bit_exact_on_dielectric_cpml(oracle_runs):
    """Without FMA contraction the plain FP64 kernels follow the reference's
    roundings: C1 (dielectric + CPML + source + port) agrees bit for bit."""
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs["c1"]
    g = cps.Grid.from_deck(dk, cps.FP64, ids=ids, port_points_list=pts)
    g.step(dk.nsteps, cps.PLAIN)
    for c in range(6):
        assert np.array_equal(g.field(c), o.field(c)), NAMES[c]


def test_gain_populations_match_oracle(oracle_mod, oracle_runs):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs["c3"]
    want = o.populations()
    for prec, tol, path in ((cps.FP64, 1e-12, cps.FUSED), (cps.FP32, 1e-6, cps.FUSED),
                            (cps.FP64, 1e-12, cps.ONEPASS), (cps.FP32, 1e-6, cps.ONEPASS)):
        g = cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts)
        g.step(dk.nsteps, path)
        got = g.populations()
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= tol
        assert np.abs(got.sum(axis=1) - 2.0).max() < 1e-12  # conservation, FourLevelLaser.cpp:324


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_tma_and_register_sweeps_agree(prec):
    """The TMA-fed sweeps (default) and the register sweeps compute the same
    update; on a grid wide enough for the TMA boxes they agree to rounding."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=72, steps=80, nfreq=4)
    ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    out = []
    for mode, rows in ((0, 8), (0, 4), (1, 8)):
        g = cps.Grid.from_deck(dk, prec, ids=ids)
        g.set_sweep(mode)
        g.set_tile(rows, 16)
        g.step(dk.nsteps, cps.FUSED)
        g.sync()
        out.append([g.field(c) for c in range(6)] + [g.port_dft(0)])
    tol = 1e-12 if prec == 0 else 1e-5
    for other in out[1:]:
        for a, b in zip(out[0], other):
            assert rel_l2(a, b) < tol


def test_drude_entry_point_equals_dl_form():
    """cps_drude_init (the Drude class's constructor) sets up exactly the
    Drude-Lorentz module in its single-pole Drude form."""
    import cpsfdtd_b200 as cps
    dk = _c2_drude()
    a = cps.Grid.from_deck(dk, cps.FP64)
    dl = dk.dl
    dk.dl = None
    b = cps.Grid.from_deck(dk, cps.FP64)
    dr = decks.drude_params_metal()
    with pytest.raises(cps.CpsError):
        b.drude_init(dict(dr, epsInf=-1.0))
    b.drude_init(dr)
    dk.dl = dl
    a.step(30, cps.FUSED)
    b.step(30, cps.FUSED)
    for c in range(6):
        assert np.array_equal(a.field(c), b.field(c))


def test_three_level_populations_match_oracle(oracle_runs):
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs["c3_three"]
    want = o.three_populations()
    assert want.shape[0] > 0 and np.abs(want[:, 1:]).max() > 0  # the field moved population
    for prec, tol, path in ((cps.FP64, 1e-12, cps.FUSED), (cps.FP64, 1e-12, cps.PLAIN), (cps.FP32, 1e-6, cps.FUSED)):
        g = cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts)
        g.step(dk.nsteps, path)
        got = g.three_populations()
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_three_level_rejects_a_second_gain_and_batches():
    import cpsfdtd_b200 as cps
    dk = _c3_three()
    g = cps.Grid.from_deck(dk, cps.FP32)
    with pytest.raises(cps.CpsError):
        g.gain_init(decks.gain_params_laser())
    b = cps.Batch(cps.FP32)
    with pytest.raises(cps.CpsError):
        b.add(g)
    b.close()


# tangential pairs of the net Poynting flux along a port's normal:
# S_n = Re(E_a conj(H_b) - E_c conj(H_e)) / 2
FLUX_PAIRS = {"x": (1, 5, 2, 4), "y": (2, 3, 0, 5), "z": (0, 4, 1, 3)}


def _oracle_flux(dft, mask, normal, dA):
    """The flux from the oracle's FP64 port DFT ([npts][ncomp][nfreq][2])."""
    comps = [c for c in range(6) if mask & (1 << c)]
    a, b, c, e = (comps.index(x) for x in FLUX_PAIRS[normal])
    z = dft[..., 0] + 1j * dft[..., 1]
    s = (z[:, a] * np.conj(z[:, b]) - z[:, c] * np.conj(z[:, e])).real.sum(axis=0)
    return 0.5 * s * dA


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_port_flux_matches_oracle(prec, oracle_runs):
    """cps_port_flux on the six planar ports of the dispersive deck against
    the flux formed from the oracle's FP64 DFT of the same samples (the port
    samples themselves follow Ports.cpp:201-353 and are pinned to the
    reference's series); two calls in a row give the same result."""
    import cpsfdtd_b200 as cps
    dk, ids, pts, o = oracle_runs["c2"]
    g = cps.Grid.from_deck(dk, prec, ids=ids, port_points_list=pts)
    g.step(dk.nsteps, cps.FUSED)
    # FP32: the flux is a product of two DFTs each within the 1e-4 bar
    tol = FP64_TOL if prec == 0 else 2 * FP32_TOL
    area = {"x": dk.dy * dk.dz, "y": dk.dx * dk.dz, "z": dk.dx * dk.dy}
    for n, p in enumerate(dk.ports):
        normal = p.params["dir"]
        want = _oracle_flux(o.port_dft(n, bin(p.dft_mask).count("1"), len(p.dft_freqs)), p.dft_mask, normal,
                            area[normal])
        got = g.port_flux(n, normal)
        assert np.abs(want).max() > 0
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err <= tol, f"port {n} ({normal}) flux error {err:.3e}"
        assert np.array_equal(g.port_flux(n, normal), got)
    g.close()


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_dft_tiles_agree_bit_for_bit(prec):
    """Ports with at most 32 frequencies are contracted in 128-point x
    32-frequency tiles, others in 64 x 64 tiles; every accumulator sees the
    same operations either way.  The same ports with 32 frequencies and with
    those 32 plus one more give identical accumulators for the 32."""
    import cpsfdtd_b200 as cps
    base = decks.config2(n=40, steps=70, nfreq=32)
    out = []
    for extra in (False, True):
        dk = decks.config2(n=40, steps=70, nfreq=32)
        for p, q in zip(dk.ports, base.ports):
            f = np.asarray(q.dft_freqs, dtype=np.float64)
            p.dft_freqs = np.concatenate([f, [f[-1] * 1.01]]) if extra else f.copy()
        g = cps.Grid.from_deck(dk, prec, device=0)
        g.step(dk.nsteps, cps.FUSED)
        out.append([np.array(g.port_dft(n)[:, :, :32, :]) for n, p in enumerate(dk.ports) if p.dft_freqs is not None])
        g.close()
    assert len(out[0]) == len(out[1]) > 0
    for a, b in zip(*out):
        assert np.array_equal(a, b)
