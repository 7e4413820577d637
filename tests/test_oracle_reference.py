"""Live checks of the oracle against the reference harness (need oracle/_ref,
built from the reference tree in this container): the port DFT against an
FP64 DFT of the reference's own sampled series, and a larger deck."""
import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks
import golden.golden_cases as gc


def test_port_dft_matches_dft_of_reference_series(oracle_mod, have_ref):
    dk = gc.literal_pml(gc.c2_small())
    ref = oracle_mod.run_ref_harness(dk, record_ports=True)
    pts = [p["points"] for p in ref["ports"]]
    o = oracle_mod.Oracle.from_deck(dk, ref["ids"], pts)
    o.step(dk.nsteps)
    for n, port in enumerate(dk.ports):
        series = ref["ports"][n]["series"]  # [steps][points][6]
        comps = [c for c in range(6) if port.dft_mask & (1 << c)]
        steps = np.arange(dk.n0, dk.n0 + dk.nsteps)
        w = 2 * np.pi * port.dft_freqs
        got = o.port_dft(n, len(comps), len(w))
        for ci, c in enumerate(comps):
            t = (steps - (0.5 if c >= 3 else 0.0)) * dk.dt
            ph = np.exp(-1j * np.outer(t, w))               # [steps][freq]
            want = np.einsum("sp,sf->pf", series[:, :, c], ph)
            assert rel_l2(got[:, ci, :, 0], want.real) < 1e-11
            assert rel_l2(got[:, ci, :, 1], want.imag) < 1e-11


def test_oracle_matches_reference_midsize(oracle_mod, have_ref):
    dk = gc.literal_pml(decks.config2(n=56, steps=40, nfreq=2))
    ref = oracle_mod.run_ref_harness(dk)
    o = oracle_mod.Oracle.from_deck(dk, ref["ids"], [p["points"] for p in ref["ports"]])
    o.step(dk.nsteps)
    for c, name in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        assert np.array_equal(o.field(c), ref[name]), name
