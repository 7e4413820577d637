"""Record-and-fuse (cps_grid_set_record): single-routine calls made in the
reference main loop's order (main.cpp:264-330) run as the fused step and give
exactly what cps_step's fused path gives; calls in any other order, or cut by
a read-back, replay one by one and give exactly what the unrecorded calls
give."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_l2
from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _grid(dk, prec):
    import cpsfdtd_b200 as cps
    return cps.Grid.from_deck(dk, prec)


def _reference_calls(g, dk, n):
    """One step of main.cpp's loop body as single-routine calls."""
    g.op("h_bulk")
    if dk.tfsf:
        g.op("tfsf_h", n, 0x3F)
    if dk.pml:
        g.op("h_pml")
    g.op("e_bulk")
    if dk.dl:
        g.op("dl")
    if dk.gain:
        g.op("gain_polarization")
        g.op("gain_efield")
        g.op("gain_populations")
    if dk.three:
        g.op("three_polarization")
        g.op("three_efield")
        g.op("three_populations")
    if dk.tfsf:
        g.op("tfsf_e", n, 0x3F)
    if dk.sources:
        g.op("sources", n)
    if dk.pml:
        g.op("e_pml")
    for p in range(len(g.ports)):
        g.op("port_sample", p, n)


def _state(g):
    return ([g.field(c) for c in range(6)],
            [g.port_last(p) for p in range(len(g.ports))],
            [g.port_dft(p, raw=True).copy() for p in range(len(g.ports)) if g.ports[p][2] > 0])


def _same(a, b):
    for x, y in zip(a[0], b[0]):
        assert np.array_equal(x, y), rel_l2(x, y)
    for x, y in zip(a[1], b[1]):
        assert np.array_equal(x, y)
    for x, y in zip(a[2], b[2]):
        assert np.array_equal(x, y), rel_l2(x, y)


_DECKS = {
    "dispersive": lambda: decks.config2(n=40, steps=1, nfreq=3),
    "dielectric_sources": lambda: decks.config1(n=36, steps=1),
    "laser": lambda: decks.config4_member(40, 48, 36, seed=3, steps=1, nfreq=2),
    "three_level": lambda: _three(),
}


def _three():
    dk = decks.config4_member(40, 48, 36, seed=6, steps=1, nfreq=2)
    dk.gain = None
    dk.three = decks.three_params_laser()
    return dk


@pytest.mark.parametrize("name", sorted(_DECKS))
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_recorded_reference_order_equals_fused_step(name, precision):
    import cpsfdtd_b200 as cps
    prec = cps.FP32 if precision == "fp32" else cps.FP64
    dk = _DECKS[name]()
    steps = 70  # port rings fold at 64 samples
    ref = _grid(dk, prec)
    ref.step(steps, cps.FUSED)
    g = _grid(dk, prec)
    g.set_record(True)
    n0 = g.get_step()
    for n in range(n0, n0 + steps):
        _reference_calls(g, dk, n)
    fused, replayed, pending = g.record_stats()
    assert (fused, replayed) == (steps - 1, 0) and pending > 0  # the last step waits for a read or the next step
    _same(_state(ref), _state(g))
    assert g.record_stats() == (steps, 0, 0)


def test_other_orders_replay_call_by_call():
    """E_PML before the Drude-Lorentz term, and a TF/SF-E call before E_BULK,
    are outside the fused step's order: replayed as made."""
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    ga, gb = _grid(dk, cps.FP64), _grid(dk, cps.FP64)
    gb.set_record(True)

    def calls(g, n):
        g.op("h_bulk"); g.op("h_pml"); g.op("tfsf_h", n, 0x3F)
        g.op("e_bulk"); g.op("e_pml"); g.op("dl"); g.op("tfsf_e", n, 0x3F)
        g.op("port_sample", 0, n)
        g.op("tfsf_e", n, 0x01)  # a stray face call outside any step

    for n in range(1, 21):
        calls(ga, n)
        calls(gb, n)
    _same(_state(ga), _state(gb))
    fused, replayed, pending = gb.record_stats()
    assert fused == 0 and replayed == 20 * 9 and pending == 0


def test_read_back_mid_step_flushes_in_order():
    import cpsfdtd_b200 as cps
    dk = decks.config4_member(40, 48, 36, seed=4, steps=1, nfreq=2)
    ga, gb = _grid(dk, cps.FP32), _grid(dk, cps.FP32)
    gb.set_record(True)
    for n in range(1, 13):
        for g in (ga, gb):
            g.op("h_bulk"); g.op("h_pml")
        # reading H between the H and E halves runs the queued H calls first
        assert np.array_equal(ga.field(3), gb.field(3))
        for g in (ga, gb):
            g.op("e_bulk"); g.op("gain_polarization"); g.op("gain_efield"); g.op("gain_populations")
            g.op("e_pml")
            for p in range(len(g.ports)):
                g.op("port_sample", p, n)
    _same(_state(ga), _state(gb))
    assert gb.record_stats()[0] == 0


def test_recording_switched_off_and_static_flush_refused():
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    g = _grid(dk, cps.FP32)
    g.set_record(True)
    _reference_calls(g, dk, 1)
    L = g.L
    L.cps_ports_flush_static.argtypes = [C.c_void_p]
    L.cps_ports_flush_static.restype = C.c_int32
    assert L.cps_ports_flush_static(g.h) == cps.CPS_E_STATE
    assert g.record_stats()[2] > 0
    g.set_record(False)  # runs the queued step
    assert g.record_stats()[:3] == (1, 0, 0)
    assert L.cps_ports_flush_static(g.h) == 0
    ref = _grid(dk, cps.FP32)
    ref.step(1, cps.FUSED)
    a, b = _state(ref), _state(g)
    _same(a[:2] + ([],), b[:2] + ([],))
    for x, y in zip(a[2], b[2]):  # the static flush's phasors agree to rounding
        assert np.abs(x - y).max() <= 1e-12 * np.abs(x).max()


def test_batch_step_runs_a_members_queue_first():
    import cpsfdtd_b200 as cps
    dk = decks.config2(n=40, steps=1, nfreq=2)
    ref = _grid(dk, cps.FP32)
    ref.step(11, cps.FUSED)
    g = _grid(dk, cps.FP32)
    g.set_record(True)
    _reference_calls(g, dk, 1)
    g.set_step(2)
    b = cps.Batch(cps.FP32)
    b.add(g)
    b.step(10)
    b.sync()
    _same(_state(ref), _state(g))
    b.close()
