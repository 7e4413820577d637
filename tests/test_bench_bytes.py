"""The byte models behind bench.py's roofline (`sweep_bytes`), on CPU: a grid
without auxiliary state moves the survey's 50 B per cell-update per step in
FP32 (each sweep reads and writes its own three components once, 1 B ID), 74 B
when the other side's three components read by separate sweeps are counted;
CPML adds 2 psi words read and written per slab cell of each side, Drude-
Lorentz 3 x (nD + 2 nL + 1) words per ID-2 cell and gain 15 words per gain
cell, both read and written on the E side."""
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def deck(n, npml=0, dl=None):
    return SimpleNamespace(nx=n, ny=n, nz=n, pml={"npml": [npml] * 6} if npml else None, dl=dl)


def test_bare_grid_is_50_bytes_per_cell_update_in_fp32():
    n = 100
    (h, e), (h2, e2) = bench.sweep_bytes(deck(n), 0)
    assert h == n ** 3 * 25
    assert e == (n - 1) ** 3 * 25
    assert h2 - h == n ** 3 * 12 and e2 - e == (n - 1) ** 3 * 12
    # per cell-update of the whole step, large-grid limit: 50 and 74 B
    assert abs((h + e) / n ** 3 - 50) < 1.0
    assert abs((h2 + e2) / n ** 3 - 74) < 1.5


def test_fp64_doubles_the_field_words():
    n = 64
    (h, _), _ = bench.sweep_bytes(deck(n), 0, prec_bytes=8)
    assert h == n ** 3 * (6 * 8 + 1)


def test_cpml_adds_two_psi_words_read_and_written_per_slab_cell():
    n, np_ = 80, 10
    (h0, e0), _ = bench.sweep_bytes(deck(n), 0)
    (h, e), _ = bench.sweep_bytes(deck(n, npml=np_), 0)
    h_slab = 2 * np_ * 3 * n * n
    e_slab = 2 * np_ * 3 * (n - 1) * (n - 1)
    assert h - h0 == h_slab * 16
    assert e - e0 == e_slab * 16


def test_drude_lorentz_and_gain_state_on_the_e_side():
    n = 48
    dl = {"fD": [1.0], "fL": [1.0, 2.0]}  # one Drude and two Lorentz poles: 6 words per component
    (h0, e0), _ = bench.sweep_bytes(deck(n, dl=dl), 0)
    (h1, e1), _ = bench.sweep_bytes(deck(n, dl=dl), 1000)
    assert h1 == h0 and e1 - e0 == 1000 * 3 * 6 * 2 * 4
    (h2, e2), _ = bench.sweep_bytes(deck(n), 0, ngain=500)
    (_, e3), _ = bench.sweep_bytes(deck(n), 0)
    assert e2 - e3 == 500 * 15 * 2 * 4
