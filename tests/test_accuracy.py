"""The error-report helpers (cpsfdtd_b200/accuracy.py) on synthetic inputs:
the parabolic peak is exact on a parabola (uniform and non-uniform
frequency grids), the power spectrum reads the engine's raw DFT layout
[ncomp][nfreq][2][npts], and the field errors are per-component relative L2."""
import numpy as np

from cpsfdtd_b200 import accuracy as acc


def test_peak_is_exact_on_a_parabola():
    for f in (np.linspace(4.0e14, 6.0e14, 33), np.sort(np.random.default_rng(0).uniform(4e14, 6e14, 40))):
        f0 = 5.123456e14
        s = 7.0 - ((f - f0) / 1e14) ** 2
        assert abs(acc.peak_frequency(f, s) - f0) < 1e-6 * f0


def test_peak_at_the_ends_is_the_end_sample():
    f = np.linspace(1.0, 2.0, 11)
    assert acc.peak_frequency(f, f) == 2.0
    assert acc.peak_frequency(f, -f) == 1.0


def test_power_spectrum_layout():
    rng = np.random.default_rng(1)
    d = rng.normal(size=(4, 7, 2, 13))
    s = acc.power_spectrum(d)
    want = np.array([sum(d[c, f, 0, p] ** 2 + d[c, f, 1, p] ** 2 for c in range(4) for p in range(13))
                     for f in range(7)])
    assert np.allclose(s, want, rtol=1e-14)


def test_field_and_port_errors():
    rng = np.random.default_rng(2)
    b = [rng.normal(size=(5, 6, 7)) for _ in range(6)]
    a = [x * (1 + 1e-5) for x in b]
    e = acc.field_errors(a, b)
    assert abs(e["max"] - 1e-5) < 1e-12
    assert set(e["per_component"]) == set(acc.NAMES)
    f = np.linspace(1.0, 2.0, 9)
    dft = rng.normal(size=(2, 9, 2, 5))
    p = acc.port_errors(f, dft, dft)
    assert p["dft_rel_l2"] == 0 and p["spectrum_rel_err"] == 0 and p["peak_shift_rel"] == 0
    r = acc.summarize(e, [p])
    assert r["field_rel_l2"] == e["max"] and r["resonance_shift_rel"] == 0
