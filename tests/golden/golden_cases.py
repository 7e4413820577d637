"""Decks of the golden fixtures (tests/golden/golden.json) and of the
reference-pinned oracle tests.  Small sizes: each runs in well under a second."""
import numpy as np

from cpsfdtd_b200 import decks

S = decks.Shape


def literal_pml(dk):
    """The deck with the reference's own CPML coefficients (CPML.cpp:524-525):
    the form the reference's code computes, which the golden fixtures pin."""
    if dk.pml:
        dk.pml = dict(dk.pml, literal=1)
    return dk


def c1_small():
    return decks.config1(n=24, steps=40)


def c2_small():
    return decks.config2(n=32, steps=30, nfreq=4)


def c2_cw():
    dk = decks.config2(n=32, steps=24, nfreq=2)
    dk.tfsf["cwmode"] = 1
    # the reference fills 5 periods of ramp regardless of Nt (TF_SF.cpp:918-922): keep Nt past it
    dk.tfsf["Nt"] = 1100
    dk.tfsf["theta"], dk.tfsf["phi"], dk.tfsf["psi"] = 50.0, 20.0, 35.0
    dk.tfsf["k0"] = 10
    return dk


def c3_small():
    return decks.config3(n=32, steps=30)


def shapes_pec():
    d = 10e-9
    dk = decks.Deck(30, 26, 34, d, d, d, name="shapes")
    dk.media = [(1, 1, 0, 0), (2.0, 1, 0, 0), (1, 1, 0, 0), (3.0, 1, 0, 0), (1, 1, 0, 0), (1.5, 1, 2e3, 0)]
    dk.shapes = [S(1, "cuboid", 5 * d, 6 * d, 7 * d, 10 * d, 8 * d, 9 * d),
                 S(3, "cuboid", 14.3 * d, 11.2 * d, 10.7 * d, 6.1 * d, 5.3 * d, 7.9 * d, theta=0.3, phi=0.2, psi=0.5),
                 S(5, "cylinder", 15 * d, 14 * d, 4 * d, 6 * d, 4 * d, 10 * d),
                 S(4, "ellipsoid", 20 * d, 16 * d, 24 * d, 3 * d, 2 * d, 3 * d),
                 S(3, "cuboid", 1 * d, 1 * d, 1 * d, 2 * d, 2 * d, 2 * d),
                 S(4, "multi", 3 * d, 19 * d, 22 * d, 8 * d, 0, 0, theta=3, phi=1, psi=1)]
    dk.pml = decks.pml_params(5, m=3.0, malp=1.0, kapmax=7.0, sig_ratio=0.8, alpmax=0.1)
    wave = decks.gaussian_sine(60, dk.dt, 500e-9, 3e-15, 9e-15)
    dk.sources = [(decks.COMP["Ey"], 12, 13, 17, wave), (decks.COMP["Hz"], 18, 9, 20, 0.002 * wave)]
    dk.ports = [decks.Port("plain", dict(dir="y", position=13.5 * d, w1=2.5 * d, w2=27.5 * d, h1=3.5 * d, h2=30.5 * d)),
                decks.Port("spherical", dict(r=8 * d, xc=15.5 * d, yc=13.5 * d, zc=17.5 * d,
                                             theta1=10.0, theta2=170.0, phi1=0.0, phi2=360.0))]
    dk.nsteps = 45
    return dk


CASES_3D = {"c1_small": c1_small, "c2_small": c2_small, "c2_cw": c2_cw, "c3_small": c3_small,
            "shapes_pec": shapes_pec}


def _grid2d(kind):
    nx = ny = 48
    d = 5e-9
    dt = 0.99 / (decks.C0 * np.sqrt(2.0) / d)
    ii, jj = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), indexing="ij")
    ids = np.zeros((nx + 1, ny + 1), np.uint8)
    p = dict(nx=nx, ny=ny, dx=d, dy=d, dt=dt, nsteps=240, si=10, sj=24)
    wave = decks.gaussian_sine(240, dt, 550e-9, 4e-15, 12e-15)
    if kind == "three_literal":
        # the reference's ThreeLevel class as written: its polarisation doubles
        # every two steps, so the case stops after 60 steps, before it blows up
        ids[16:34, 14:36] = 5
        media = [(1, 1, 0, 0)] * 5 + [(2.25, 1, 0, 0)]
        p = dict(p, nsteps=60)
        return p, media, ids, 1e3 * wave[:60], {"three": decks.three_params_laser(literal=1)}
    if kind == "gain":
        ids[16:34, 14:36] = 5
        media = [(1, 1, 0, 0)] * 5 + [(2.25, 1, 0, 0)]
        return p, media, ids, 1e3 * wave, {"gain": decks.gain_params_laser(pump=0.0)}
    ids[(ii - 26) ** 2 + (jj - 24) ** 2 <= 64] = 2
    ids[40:44, 8:12] = 4
    media = [(1, 1, 0, 0), (1, 1, 0, 0), (1, 1, 0, 0), (1, 1, 0, 0), (1, 1, 0, 0)]
    if kind == "drude":  # the single-pole Drude class (Drude.cpp), with conductivity
        return p, media, ids, wave, {"drude": decks.drude_params_metal()}
    dl = decks.dl_params_metal()
    if kind == "dl_literal":
        dl = dict(dl, fL=[], dL=[], depsL=[], literal=1, sigma=1e4)
    return p, media, ids, wave, {"dl": dl}


CASES_2D = {"dl": lambda: _grid2d("dl"), "dl_literal": lambda: _grid2d("dl_literal"),
            "gain": lambda: _grid2d("gain"), "drude": lambda: _grid2d("drude"),
            "three_literal": lambda: _grid2d("three_literal")}
