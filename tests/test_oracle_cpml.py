"""The CPML psi coefficient (CPML.cpp:524-525).  The reference applies one
coefficient, dt/eps0, to every cell's psi term; in a CPML filled with an
eps_r != 1 medium (the photonic-crystal laser decks keep their eps 2.25
background up to the boundary) that makes the fields grow without bound.
The default form takes each cell's own curl coefficient (bE of its medium),
the CFS-PML update for any medium: equal to the reference in vacuum CPMLs
(the golden decks with vacuum CPML pass in both forms) and stable here."""
import numpy as np

from cpsfdtd_b200 import decks
import golden.golden_cases as gc


def _max_e(o):
    return max(float(np.abs(o.field(c)).max()) for c in range(3))


def _laser(literal, steps):
    dk = decks.config3(n=48, steps=steps, seed=0, nfreq=0, port=False)
    dk.pml = dict(dk.pml, literal=literal)
    return dk


def test_literal_coefficient_grows_where_the_medium_form_is_stable(oracle_mod):
    """The seed pulse peaks near step 790; after it has passed, the default
    form's fields stay bounded, while the literal form has long diverged."""
    oracle_mod.Oracle.threads(4)
    dk = _laser(0, 2400)
    o = oracle_mod.Oracle.from_deck(dk, dk.ids)
    o.step(1200)
    mid = _max_e(o)
    o.step(1200)
    late = _max_e(o)
    assert np.isfinite(late) and 0 < late < 2 * mid, (mid, late)
    dk = _laser(1, 600)
    o = oracle_mod.Oracle.from_deck(dk, dk.ids)
    o.step(600)
    lit = _max_e(o)
    assert not np.isfinite(lit) or lit > 1e6 * mid, (mid, lit)


def test_both_forms_agree_in_a_vacuum_cpml(oracle_mod):
    out = []
    for literal in (0, 1):
        dk = gc.c2_small()
        dk.pml = dict(dk.pml, literal=literal)
        import cpsfdtd_b200 as cps
        ids = cps.rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
        o = oracle_mod.Oracle.from_deck(dk, ids)
        o.step(dk.nsteps)
        out.append([o.field(c) for c in range(6)])
    for a, b in zip(*out):
        assert np.array_equal(a, b)
