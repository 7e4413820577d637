"""The oracle restatement against the golden fixtures made from the
reference's own code (tests/golden/make_golden.py): every field, stretch
array, incident table and port sample series must match bit for bit."""
import hashlib
import json
import os

import numpy as np
import pytest

import golden.golden_cases as gc

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _ids_and_ports(dk):
    import cpsfdtd_b200 as cps
    ids = dk.ids if dk.ids is not None else cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    return ids, pts


@pytest.mark.parametrize("name", sorted(gc.CASES_3D))
def test_oracle_matches_reference_3d(name, oracle_mod):
    g = GOLDEN["cases3d"][name]
    dk = gc.literal_pml(gc.CASES_3D[name]())
    ids, pts = _ids_and_ports(dk)
    assert sha(ids) == g["ids"]["sha256"], "rasteriser differs from Structure::generate_mesh"
    for p, gp in zip(pts, g["ports"]):
        assert sha(p) == gp["points"]["sha256"], "port point set differs from the reference constructor"
    o = oracle_mod.Oracle.from_deck(dk, ids, pts)
    series = [[] for _ in pts]
    for _ in range(dk.nsteps):
        o.step(1)
        for n in range(len(pts)):
            series[n].append(o.port_last(n))
    for c, name_c in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        f = o.field(c)
        assert sha(f) == g[name_c]["sha256"], f"{name_c}: l2 {np.linalg.norm(f)} vs reference {g[name_c]['l2']}"
    for w, gs in enumerate(g["stretch"]):
        assert sha(o.stretch(w, gs["shape"][0])) == gs["sha256"], f"stretch array {w}"
    if "einc" in g:
        e, h = o.tfsf_tables(dk.tfsf["Nt"])
        assert sha(e) == g["einc"]["sha256"] and sha(h) == g["hinc"]["sha256"]
    for n, gp in enumerate(g["ports"]):
        assert sha(np.array(series[n])) == gp["series"]["sha256"], f"port {n} sample series"


@pytest.mark.parametrize("name", sorted(gc.CASES_2D))
def test_oracle_recursions_match_reference_2d(name, oracle_mod):
    g = GOLDEN["cases2d"][name]
    p, media, ids, wave, kw = gc.CASES_2D[name]()
    Ex, Ey, Hz = oracle_mod.run_orc2d(p, media, ids, wave, **kw)
    for arr, key in ((Ex, "Ex"), (Ey, "Ey"), (Hz, "Hz")):
        assert sha(arr) == g[key]["sha256"], f"{key}: l2 {np.linalg.norm(arr)} vs {g[key]['l2']}"


def test_gain_kat_exercises_the_gain_path(oracle_mod):
    """The gain KAT must differ from the same run without gain sites."""
    p, media, ids, wave, kw = gc.CASES_2D["gain"]()
    with_gain = oracle_mod.run_orc2d(p, media, ids, wave, **kw)
    without = oracle_mod.run_orc2d(p, media, ids, wave)
    assert np.abs(with_gain[0] - without[0]).max() > 0


def test_dl_kat_is_stable_and_dispersive(oracle_mod):
    p, media, ids, wave, kw = gc.CASES_2D["dl"]()
    Ex, Ey, Hz = oracle_mod.run_orc2d(p, media, ids, wave, **kw)
    assert np.isfinite(Ex).all() and np.abs(Ex).max() < 10
    plain = oracle_mod.run_orc2d(p, media, ids, wave, dl=None)
    assert np.abs(Ex - plain[0]).max() > 1e-3 * np.abs(plain[0]).max()


def test_drude_kat_is_dispersive_and_lossy(oracle_mod):
    """The single-pole Drude KAT (the reference's Drude class) differs from the
    free-space run and from the same pole without the Drude class's C1."""
    p, media, ids, wave, kw = gc.CASES_2D["drude"]()
    Ex, Ey, Hz = oracle_mod.run_orc2d(p, media, ids, wave, **kw)
    assert np.isfinite(Ex).all()
    plain = oracle_mod.run_orc2d(p, media, ids, wave)
    assert np.abs(Ex - plain[0]).max() > 1e-3 * np.abs(plain[0]).max()
    literal_dl = dict(oracle_mod.drude_as_dl(kw["drude"]), literal=1)
    other = oracle_mod.run_orc2d(p, media, ids, wave, dl=literal_dl)
    assert np.abs(Ex - other[0]).max() > 0


def test_three_level_kat_and_repaired_form(oracle_mod):
    """The three-level KAT (the reference's ThreeLevel class as written) is
    finite and moved by the gain sites; the repaired oscillators stay bounded
    over 20 times as many steps, where the literal ones diverge."""
    p, media, ids, wave, kw = gc.CASES_2D["three_literal"]()
    lit = oracle_mod.run_orc2d(p, media, ids, wave, **kw)
    assert all(np.isfinite(a).all() for a in lit)
    plain = oracle_mod.run_orc2d(p, media, ids, wave)
    assert np.abs(lit[0] - plain[0]).max() > 0
    long_p = dict(p, nsteps=1200)
    long_wave = np.concatenate([wave, np.zeros(1140)])
    rep = dict(kw["three"], literal=0)
    fixed = oracle_mod.run_orc2d(long_p, media, ids, long_wave, three=rep)
    free = oracle_mod.run_orc2d(long_p, media, ids, long_wave)
    assert all(np.isfinite(a).all() for a in fixed)
    assert np.abs(fixed[0]).max() < 10 * np.abs(free[0]).max() + 1e-30
    with np.errstate(all="ignore"):
        wild = oracle_mod.run_orc2d(long_p, media, ids, long_wave, **kw)
    assert not np.isfinite(wild[0]).all() or np.abs(wild[0]).max() > 1e6 * np.abs(free[0]).max()
