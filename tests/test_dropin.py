"""The C++ drop-in classes (include/cpsfdtd_classes.hpp): a main.cpp in the
reference's style builds against them and the library, reads the reference's
deck formats, and on the GPU gives the oracle's results for the same decks in
the same call order."""
import os
import subprocess

import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cpsfdtd_b200")


def _build(tmp_path):
    import cpsfdtd_b200 as cps
    cps.lib()  # the library must exist
    exe = str(tmp_path / "dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "dropin", "main.cpp"), "-L", LIBDIR, "-lcpsfdtd",
           "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_main_builds_and_fails_loudly(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe, str(tmp_path / "no_such_deck"), "3", str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open deck" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("record", ["1", "0"])
@pytest.mark.parametrize("case", ["dispersive", "dielectric", "drude", "three"])
def test_dropin_matches_oracle(tmp_path, oracle_mod, case, record):
    """record "1": the classes' calls run as fused steps (the default);
    "0": routine by routine."""
    import cpsfdtd_b200 as cps
    exe = _build(tmp_path)
    if case == "dispersive":
        dk = decks.config2(n=32, steps=40, nfreq=2)
    elif case == "drude":  # the single-pole Drude class (Drude.txt deck)
        dk = decks.config2(n=32, steps=40, nfreq=2)
        dk.dl = decks.drude_as_dl(decks.drude_params_metal())
    elif case == "three":  # the three-level gain class (ThreeLevel.txt deck) under a TF/SF beam
        dk = decks.config3(n=32, steps=40, nfreq=0, port=False)
        dk.gain = None
        dk.three = decks.three_params_laser()
        dk.sources = []
        dk.tfsf = decks.config2(n=32, steps=40, nfreq=1).tfsf
    else:
        dk = decks.config1(n=28, steps=40)
        dk.sources = []  # point sources are main.cpp code, not a class: drive it with a TF/SF beam instead
        dk.tfsf = decks.config2(n=28, steps=40, nfreq=1).tfsf
    deck = tmp_path / "deck"
    out = tmp_path / "out"
    os.makedirs(out)
    dk.write(str(deck))
    nsteps = 40
    env = dict(os.environ, CPSFDTD_RECORD=record)
    r = subprocess.run([exe, str(deck), str(nsteps), str(out)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.startswith("dropin ok")

    ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
    pts = [cps.port_points(dk, p) for p in dk.ports]
    o = oracle_mod.Oracle.from_deck(dk, ids, pts)
    L = o.L
    for n in range(1, nsteps + 1):  # the call order of tests/dropin/main.cpp
        L.orc_op_h_bulk(o.h)
        L.orc_op_tfsf_h(o.h, n)
        L.orc_op_h_pml(o.h)
        L.orc_op_e_bulk(o.h)
        if dk.dl:
            L.orc_op_dl(o.h)
        if dk.three:
            L.orc_op_three_p(o.h)
            L.orc_op_three_e(o.h)
            L.orc_op_three_n(o.h)
        L.orc_op_tfsf_e(o.h, n)
        L.orc_op_e_pml(o.h)
        L.orc_op_ports(o.h, n)
    shape = (dk.nx + 1, dk.ny + 1, dk.nz + 1)
    for c in range(6):
        got = np.fromfile(str(out / f"field{c}.bin"), dtype=np.float64).reshape(shape)
        assert rel_l2(got, o.field(c)) < 1e-10, c
    for q, p in enumerate(pts):
        got = np.loadtxt(str(out / f"portE{q}.txt")).reshape(-1, 3)
        ref = o.port_last(q)[:, :3]
        assert got.shape == ref.shape
        assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max() + 1e-300
        ijk = np.loadtxt(str(out / f"portP{q}.txt"), dtype=np.int64).reshape(-1, 3)
        assert np.array_equal(ijk, p)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["dispersive", "drude", "laser", "three"])
def test_deck_load_equals_grid_from_deck(tmp_path, case):
    """cps_deck_load (the drop-in classes' parsing, as one C call) builds the grid
    Grid.from_deck builds from the same deck: equal fields after 30 steps."""
    import cpsfdtd_b200 as cps
    if case in ("dispersive", "drude"):
        dk = decks.config2(n=36, steps=30, nfreq=0)
        if case == "drude":
            dk.dl = decks.drude_as_dl(decks.drude_params_metal())
    else:
        dk = decks.config3(n=36, steps=30, nfreq=0, port=False)
        if case == "three":
            dk.gain = None
            dk.three = decks.three_params_laser()
    dk.sources = []  # main.cpp code in the reference, not a deck
    for p in dk.ports:
        p.dft_freqs = None
    deck = tmp_path / "deck"
    dk.write(str(deck))
    a = cps.Grid.from_deck_dir(str(deck), cps.FP64)
    b = cps.Grid.from_deck(dk, cps.FP64)
    assert a.shape3 == b.shape3 and a.dt == b.dt
    a.set_step(1)
    b.set_step(1)
    a.step(30, cps.FUSED)
    b.step(30, cps.FUSED)
    for c in range(6):
        assert np.array_equal(a.field(c), b.field(c)), c
    a.close()
    b.close()


def test_deck_load_reports_bad_decks(tmp_path):
    import cpsfdtd_b200 as cps
    with pytest.raises(cps.CpsError) as e:
        cps.Grid.from_deck_dir(str(tmp_path / "nothing"), cps.FP32)
    assert "material.txt" in str(e.value)
