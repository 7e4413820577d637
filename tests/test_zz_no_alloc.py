"""cps_ports_flush_static (the port-DFT flush that allocates nothing) against
cps_ports_flush on identical grids, through the C ABI: two flush cycles in a
row agree within the DFT tolerance, and the static form leaves the grid's
device allocations unchanged.  Collected last; passes alone too."""
import ctypes as C

import numpy as np
import pytest

from cpsfdtd_b200 import decks

pytestmark = pytest.mark.gpu


def _grid():
    import cpsfdtd_b200 as cps
    return cps.Grid.from_deck(decks.config2(n=32, steps=200, nfreq=5), cps.FP32)


def _bytes(L, g):
    b = C.c_int64()
    assert L.cps_grid_bytes(g.h, C.byref(b)) == 0
    return b.value


def _dft(L, g):
    out = []
    for p, (npts, ncomp, nfreq) in enumerate(g.ports):
        a = np.empty((ncomp, nfreq, 2, npts))
        assert L.cps_port_dft_read(g.h, p, a.ctypes.data_as(C.POINTER(C.c_double))) == 0
        out.append(a)
    return out


def test_static_flush_matches_allocating_flush():
    import cpsfdtd_b200 as cps
    L = cps.lib()
    L.cps_ports_flush_static.argtypes = [C.c_void_p]
    L.cps_ports_flush_static.restype = C.c_int32
    a, b = _grid(), _grid()
    before = _bytes(L, b)
    for steps in (37, 50):  # two flush cycles in a row, ring part-filled each time
        a.step(steps, cps.FUSED)
        b.step(steps, cps.FUSED)
        assert L.cps_ports_flush(a.h) == 0
        assert L.cps_ports_flush_static(b.h) == 0, L.cps_last_error().decode()
        assert L.cps_ports_flush_static(b.h) == 0  # nothing left: a no-op
        for x, y in zip(_dft(L, a), _dft(L, b)):
            scale = np.abs(x).max()
            assert scale > 0
            assert np.abs(x - y).max() <= 1e-12 * scale
        for p in range(len(a.ports)):
            assert np.array_equal(a.port_last(p), b.port_last(p))
    assert _bytes(L, b) == before  # no device allocation on the static path
    a.close()
    b.close()


def test_static_flush_rejects_large_ports():
    import cpsfdtd_b200 as cps
    L = cps.lib()
    L.cps_ports_flush_static.argtypes = [C.c_void_p]
    L.cps_ports_flush_static.restype = C.c_int32
    g = cps.Grid.from_deck(decks.config2(n=32, steps=20, nfreq=300), cps.FP32)
    g.step(3, cps.FUSED)
    assert L.cps_ports_flush_static(g.h) == cps.CPS_E_INVALID
    assert "256" in L.cps_last_error().decode()
    g.close()
