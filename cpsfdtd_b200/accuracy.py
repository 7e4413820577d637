"""Error report of a chosen form (FP32 fields, batched or served) against an
FP64 result of the same deck: field relative L2, port-spectrum relative error
and resonance-frequency shift.  Host-side numpy only.

The FP64 side is the plain form (the FP64 one-grid path, which matches the
oracle to 1e-10 relative L2) or the oracle itself; the quantities are the ones
the reference's port output feeds (Ports.cpp:88-99, 342-353: the six field
components sampled at the port points every step), reduced here to the
running DFT the engine keeps.

  field_errors(a, b)        per component |a - b|_2 / |b|_2 and the max
  power_spectrum(dft)       S(f) = sum over points and components of |A(f)|^2
  peak_frequency(f, S)      the |DFT| peak by parabolic interpolation
  port_errors(freqs, a, b)  port-DFT rel L2, spectrum rel error, peak shift
"""
from __future__ import annotations

import numpy as np

NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    n = float(np.linalg.norm(b))
    return float(np.linalg.norm(a - b)) / (n if n > 0 else 1.0)


def field_errors(a, b) -> dict:
    """a, b: sequences of the six field arrays (same shapes).  Components that
    are zero in b are compared in absolute terms (reported as 0 when a is zero
    there too)."""
    per = {}
    for name, x, y in zip(NAMES, a, b):
        per[name] = rel_l2(x, y) if np.any(np.asarray(y) != 0) else float(np.abs(np.asarray(x)).max())
    return {"max": max(per.values()), "per_component": per}


def power_spectrum(dft) -> np.ndarray:
    """dft in the engine's raw layout [ncomp][nfreq][2][npts] (re, im):
    S(f) = sum over points and components of re^2 + im^2."""
    d = np.asarray(dft, dtype=np.float64)
    return (d[:, :, 0, :] ** 2 + d[:, :, 1, :] ** 2).sum(axis=(0, 2))


def peak_frequency(freqs, s) -> float:
    """Frequency of the maximum of s(f): the sample maximum refined by the
    vertex of the parabola through it and its two neighbours (uniform or
    non-uniform spacing); an end sample is returned as it is."""
    f = np.asarray(freqs, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    m = int(np.argmax(s))
    if m == 0 or m == len(s) - 1:
        return float(f[m])
    x0, x1, x2 = f[m - 1], f[m], f[m + 1]
    y0, y1, y2 = s[m - 1], s[m], s[m + 1]
    den = (x0 - x1) * (x0 - x2) * (x1 - x2)
    a = (x2 * (y1 - y0) + x1 * (y0 - y2) + x0 * (y2 - y1)) / den
    b = (x2 * x2 * (y0 - y1) + x1 * x1 * (y2 - y0) + x0 * x0 * (y1 - y2)) / den
    if a >= 0:
        return float(x1)
    return float(-b / (2 * a))


def port_errors(freqs, a, b) -> dict:
    """a, b: the raw DFT accumulators of one port from the two runs."""
    sa, sb = power_spectrum(a), power_spectrum(b)
    fa, fb = peak_frequency(freqs, sa), peak_frequency(freqs, sb)
    return {"dft_rel_l2": rel_l2(a, b), "spectrum_rel_err": rel_l2(sa, sb),
            "peak_hz": fb, "peak_shift_rel": (fa - fb) / fb if fb else 0.0}


def summarize(field: dict, ports: list) -> dict:
    """One config's report: the largest field error, the largest port errors
    and shift over its ports."""
    out = {"field_rel_l2": field["max"], "field_rel_l2_per_component": field["per_component"]}
    if ports:
        out["port_dft_rel_l2"] = max(p["dft_rel_l2"] for p in ports)
        out["port_spectrum_rel_err"] = max(p["spectrum_rel_err"] for p in ports)
        out["resonance_shift_rel"] = max((p["peak_shift_rel"] for p in ports), key=abs)
        out["resonance_hz"] = ports[0]["peak_hz"]
    return out
