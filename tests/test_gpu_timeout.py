"""Bounded device waits of the TMA sweeps.

A sweep whose staged plane never completes gives up after its limit and the
grid reports CPS_E_TIMEOUT at the next synchronisation instead of hanging;
the CUDA context stays usable and, after cps_grid_reset, the grid steps
exactly as a fresh grid does.  The wait is made to run out by the test
setting cps_grid_set_wait_skew (the first plane of every tile expects more
bytes than its loads bring): no fault, no bad address, no trap, and every
copy the blocks issued still lands.  The reference has no failure handling
(main.cpp:68-85); this is the engine's own safety behaviour."""
import time

import numpy as np
import pytest

from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1], ids=["fp64", "fp32"])
def test_sweep_wait_runs_out_and_grid_recovers(prec):
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=64, steps=30, nfreq=2)
    g = cps.Grid.from_deck(dk, prec)
    ref = cps.Grid.from_deck(dk, prec)
    g.set_wait_skew(256)
    t0 = time.perf_counter()
    g.step(1, cps.FUSED)
    with pytest.raises(cps.CpsError) as ex:
        g.sync()
    elapsed = time.perf_counter() - t0
    assert ex.value.code == cps.CPS_E_TIMEOUT
    assert elapsed < 30.0, f"the timed-out step took {elapsed:.1f} s"
    # the error stays until the grid is reset
    with pytest.raises(cps.CpsError):
        g.sync()
    g.set_wait_skew(0)
    g.reset(dk.n0)
    g.step(dk.nsteps, cps.FUSED)
    g.sync()
    ref.step(dk.nsteps, cps.FUSED)
    ref.sync()
    for c in range(6):
        assert np.array_equal(g.field(c), ref.field(c))
    g.close()
    ref.close()


def test_wait_skew_is_validated():
    import cpsfdtd_b200 as cps
    g = cps.Grid.from_deck(decks.config1(n=32, steps=4), cps.FP32)
    for bad in (-1, 4097):
        with pytest.raises(cps.CpsError) as ex:
            g.set_wait_skew(bad)
        assert ex.value.code == cps.CPS_E_INVALID
    g.close()
