"""Synthetic input decks for the cpsFDTD time-stepping workloads.

A :class:`Deck` holds one simulation: grid, media, shapes (or a precomputed
material-ID grid), CPML, Drude-Lorentz, four-level gain, TF/SF beam, point
sources and ports.  It can write itself as the reference's ``resourses/*.txt``
deck files (formats of Structure.cpp:26-52,68-157, CPML.cpp:29-68,
TF_SF.cpp:35-97,898-907, Drude_Lorentz.cpp:37-94, FourLevelLaser.cpp:37-93,
Ports.cpp:38-59,211-231) and hands the same parameters to the C-ABI.

The ``config*`` builders make the five benchmark workloads with seeded
synthetic geometry (numpy PCG64); no external dataset is involved.

Parameter translations from physical values to the reference's deck units:
  * Drude and Lorentz frequencies are written in Hz (the reference multiplies
    them by 2*pi, Drude_Lorentz.cpp:69,72,83,86).
  * The Lorentz damping enters as J'' + 2*delta*J' + w^2 J
    (Drude_Lorentz.cpp:90-92), so delta = gamma/2 for a pole of full width gamma.
  * Grid lengths are written as (N + 0.5)*delta because the reference truncates
    L/delta (Structure.cpp:121); port and source positions likewise sit at
    (n + 0.5)*delta.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

C0 = 2.99792458e8
EPS0 = 8.8541878176e-12
MU0 = 1.2566370614e-6
PI = 3.1415926535897932384626433832795

COMP = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}

ID_DISPERSIVE = 2
ID_PEC = 4
ID_GAIN = 5


def courant_dt(dx: float, dy: float, dz: float) -> float:
    """Time step of Structure.cpp:124: 0.99 of the 3-D Courant limit."""
    return 0.99 / (C0 * math.sqrt(1.0 / (dx * dx) + 1.0 / (dy * dy) + 1.0 / (dz * dz)))


def _f(x: float) -> str:
    return repr(float(x))


@dataclass
class Shape:
    """One line of structure.txt: index mat type theta phi psi x0 y0 z0 a b c."""
    mat: int
    type: str
    x0: float
    y0: float
    z0: float
    a: float
    b: float
    c: float
    theta: float = 0.0
    phi: float = 0.0
    psi: float = 0.0


@dataclass
class Port:
    kind: str                      # "plain" or "spherical"
    params: dict
    dft_freqs: Optional[np.ndarray] = None
    dft_mask: int = 0x3F


@dataclass
class Deck:
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    media: list = field(default_factory=lambda: [(1.0, 1.0, 0.0, 0.0)])
    shapes: list = field(default_factory=list)
    ids: Optional[np.ndarray] = None     # uint8 [(nx+1),(ny+1),(nz+1)] overrides shapes
    pml: Optional[dict] = None
    dl: Optional[dict] = None
    gain: Optional[dict] = None
    three: Optional[dict] = None       # three-level gain (ThreeLevel.cpp), one of gain/three
    tfsf: Optional[dict] = None
    sources: list = field(default_factory=list)
    ports: list = field(default_factory=list)
    n0: int = 1
    nsteps: int = 10
    name: str = "deck"

    @property
    def dt(self) -> float:
        return courant_dt(self.dx, self.dy, self.dz)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape3(self):
        return (self.nx + 1, self.ny + 1, self.nz + 1)

    # ------------------------------------------------------------ TF/SF
    def tfsf_abi(self) -> dict:
        """TF/SF parameters as the C-ABI takes them (TF_SF.cpp:35-97 semantics:
        i0 = xs/dx, j0 = ys/dy truncated; z0 = zs/dz as the reference sets it)."""
        t = self.tfsf
        return dict(lambda_=t["lambda"], dlambda=t["dlambda"], w0=t["w0"],
                    z0=t["zs"] / self.dz, i0=int(t["xs"] / self.dx), j0=int(t["ys"] / self.dy),
                    k0=int(t["k0"]), theta=t["theta"], phi=t["phi"], E0=t["E0"], psi=t["psi"],
                    n6=list(t["n6"]), Nt=int(t["Nt"]), cwmode=int(t["cwmode"]))

    # ------------------------------------------------------- deck files
    def write(self, path: str, harness: bool = True, record_ports: bool = False,
              bench: Optional[tuple] = None, threads: int = 0) -> None:
        os.makedirs(path, exist_ok=True)
        with open(os.path.join(path, "material.txt"), "w") as f:
            f.write(f"{len(self.media)}\n")
            for m in self.media:
                f.write("\t".join(_f(v) for v in m) + "\n")
        with open(os.path.join(path, "structure.txt"), "w") as f:
            f.write(f"{_f((self.nx + 0.5) * self.dx)}\t{_f((self.ny + 0.5) * self.dy)}\t{_f((self.nz + 0.5) * self.dz)}\n")
            f.write(f"{_f(self.dx)}\t{_f(self.dy)}\t{_f(self.dz)}\n")
            shapes = [] if self.ids is not None else self.shapes
            f.write(f"{1 if not shapes else 0}\n{len(shapes)}\n")
            for n, s in enumerate(shapes):
                f.write("\t".join([str(n), str(s.mat), s.type] + [_f(v) for v in (
                    s.theta, s.phi, s.psi, s.x0, s.y0, s.z0, s.a, s.b, s.c)]) + "\n")
        lines = [f"nsteps {self.nsteps}", f"n0 {self.n0}"]
        if self.ids is not None:
            np.ascontiguousarray(self.ids, dtype=np.uint8).tofile(os.path.join(path, "ids.bin"))
            lines.append("ids ids.bin")
        if self.pml:
            p = self.pml
            n = p["npml"]
            with open(os.path.join(path, "CFS_PML.txt"), "w") as f:
                f.write(f"{n[0]}\t{n[1]}\n{n[2]}\t{n[3]}\n{n[4]}\t{n[5]}\n")
                f.write(f"{_f(p['m'])}\t{_f(p['malp'])}\n{_f(p['kapmax'])}\t{_f(p['sig_ratio'])}\n{_f(p['alpmax'])}\n")
            lines.append("pml CFS_PML.txt")
        if self.tfsf:
            t = self.tfsf
            with open(os.path.join(path, "TF_SF.txt"), "w") as f:
                f.write(f"{_f(t['lambda'])}\n{_f(t['dlambda'])}\n{_f(t['w0'])}\t{_f(t.get('z0_deck', 0.0))}\n")
                f.write(f"{_f(t['xs'])}\t{_f(t['ys'])}\t{_f(t['zs'])}\t{int(t['k0'])}\n")
                f.write(f"{_f(t['theta'])}\t{_f(t['phi'])}\n{_f(t['E0'])}\t{_f(t['psi'])}\n")
                n = t["n6"]
                f.write(f"{n[0]}\t{n[1]}\n{n[2]}\t{n[3]}\n{n[4]}\t{n[5]}\n{int(t['Nt'])}\n{int(t['cwmode'])}\n")
            lines.append(f"tfsf TF_SF.txt {int(t['k0'])}")
        if self.dl and int(self.dl.get("literal", 0)) == 2:
            d = self.dl  # the single-pole Drude class's deck (Drude.cpp:29-52)
            with open(os.path.join(path, "Drude.txt"), "w") as f:
                f.write(f"{_f(d['epsInf'])}\tepsilon_infinity\n{_f(d['fD'][0])}\tomega_P (Hz)\n")
                f.write(f"{_f(d['sigma'])}\tsigma\n{_f(d['gD'][0])}\tgamma (Hz)\n")
            lines.append("drude Drude.txt")
        elif self.dl:
            d = self.dl
            with open(os.path.join(path, "DrudeLorentz.txt"), "w") as f:
                f.write(f"{len(d['fD'])}\tnum_of_D_poles\n{len(d['fL'])}\tnum_of_L_poles\n")
                f.write(f"{_f(d['sigma'])}\tsigma\n{_f(d['epsInf'])}\tepsilon_infinity\n")
                for a, b in zip(d["fD"], d["gD"]):
                    f.write(f"{_f(a)}\t{_f(b)}\n")
                for a, b, c in zip(d["fL"], d["dL"], d["depsL"]):
                    f.write(f"{_f(a)}\t{_f(b)}\t{_f(c)}\n")
            lines.append(f"dl DrudeLorentz.txt {int(d.get('literal', 0))}")
        if self.gain:
            g = self.gain
            with open(os.path.join(path, "FourLevelLaser.txt"), "w") as f:
                f.write("cells\tdistribution\n0\tnum of sources\n0\t0\n0\t0\n")
                for key in ("lambda_b", "lambda_a", "gamma_a", "gamma_b", "t30", "t32", "t21", "t10", "N_0"):
                    f.write(f"{_f(g[key])}\t{key}\n")
                f.write("0\tN_1\n")
                f.write(f"{_f(g.get('pump', 0.0))}\tpump rate (1/s)\n")
            lines.append("gain FourLevelLaser.txt")
        if self.three:
            t3 = self.three  # ThreeLevel.cpp:37-84, "cells" placement
            with open(os.path.join(path, "ThreeLevel.txt"), "w") as f:
                f.write("cells\tdistribution\n0\tnum of sources\n0\t0\n0\t0\n")
                for key in ("lambda_a", "lambda_b", "gamma_a", "gamma_b", "t20", "t21", "t10", "N_0"):
                    f.write(f"{_f(t3[key])}\t{key}\n")
                f.write("0\tN_1\n")
            lines.append(f"three ThreeLevel.txt {int(t3.get('literal', 0))}")
        for n, (comp, i, j, k, wave) in enumerate(self.sources):
            wf = f"source{n}.bin"
            np.ascontiguousarray(wave, dtype=np.float64).tofile(os.path.join(path, wf))
            lines.append(f"source {comp} {i} {j} {k} {wf} {len(wave)}")
        for n, p in enumerate(self.ports):
            fn = f"port{n}.txt"
            q = p.params
            with open(os.path.join(path, fn), "w") as f:
                if p.kind == "plain":
                    f.write(f"{q['dir']}\n{_f(q['position'])}\n{_f(q['w1'])}\t{_f(q['w2'])}\n{_f(q['h1'])}\t{_f(q['h2'])}\n")
                else:
                    f.write(f"{_f(q['r'])}\n{_f(q['xc'])}\t{_f(q['yc'])}\t{_f(q['zc'])}\n")
                    f.write(f"{_f(q['theta1'])}\t{_f(q['theta2'])}\n{_f(q['phi1'])}\t{_f(q['phi2'])}\n")
            lines.append(("plainport " if p.kind == "plain" else "sphericalport ") + fn)
        if record_ports:
            lines.append("record_ports 1")
        if bench:
            lines.append(f"bench {bench[0]} {bench[1]}")
        if threads:
            lines.append(f"threads {threads}")
        if harness:
            with open(os.path.join(path, "harness.txt"), "w") as f:
                f.write("\n".join(lines) + "\n")


# ------------------------------------------------------------ waveforms

def gaussian_sine(n: int, dt: float, lam: float, tau: float, t0: float, amp: float = 1.0) -> np.ndarray:
    """s(t) = amp * exp(-((t - t0)/tau)^2) * sin(2 pi c/lam (t - t0)), t = n dt."""
    t = np.arange(n, dtype=np.float64) * dt
    return amp * np.exp(-((t - t0) / tau) ** 2) * np.sin(2.0 * PI * C0 / lam * (t - t0))


def dlambda_for_tau(lam: float, tau: float) -> float:
    """dlambda that makes TF_SF's pulse envelope exp(-sig (t-t0)^2) have
    sig = 1/tau^2 (TF_SF.cpp:912-914: sig = (2 pi dnu)^2 / (16 ln 2))."""
    dnu = 4.0 * math.sqrt(math.log(2.0)) / (2.0 * PI * tau)
    # dnu = c/(lam - dl/2) - c/(lam + dl/2)  ->  solve for dl
    a = dnu / C0
    # a (lam^2 - dl^2/4) = dl  ->  (a/4) dl^2 + dl - a lam^2 = 0
    return (-1.0 + math.sqrt(1.0 + a * a * lam * lam)) / (a / 2.0)


def pml_params(n: int, m: float = 3.0, malp: float = 1.0, kapmax: float = 5.0,
               sig_ratio: float = 1.0, alpmax: float = 0.05, literal: int = 0) -> dict:
    """CPML deck values; literal = 1 keeps the reference's single psi
    coefficients (CPML.cpp:524-525), 0 each cell's own curl coefficient."""
    return dict(npml=[n] * 6, m=m, malp=malp, kapmax=kapmax, sig_ratio=sig_ratio, alpmax=alpmax, literal=literal)


def dl_params_metal() -> dict:
    """Config-2 metal: eps_inf 1, omega_D 1.37e16 rad/s, gamma_D 1e14 1/s, Lorentz
    (1.0, 4e15, 1e15), (0.5, 6e15, 2e15) in (d_eps, omega rad/s, gamma 1/s)."""
    two_pi = 2.0 * PI
    return dict(sigma=0.0, epsInf=1.0,
                fD=[1.37e16 / two_pi], gD=[1.0e14 / two_pi],
                fL=[4.0e15 / two_pi, 6.0e15 / two_pi],
                dL=[1.0e15 / 2.0 / two_pi, 2.0e15 / 2.0 / two_pi],
                depsL=[1.0, 0.5])


def three_params_laser(literal: int = 0) -> dict:
    """Three-level gain on the ID-5 cells (ThreeLevel.cpp deck values):
    transitions at 600 nm (a, 2->0) and 450 nm (b, 1->0), linewidths 2e13 Hz,
    lifetimes t20 1 ps, t21 100 fs, t10 300 ps, density 5e23 m^-3.  literal = 1
    takes the reference's coefficients as written (unstable oscillators)."""
    return dict(gain_id=5, lambda_a=600e-9, lambda_b=450e-9, gamma_a=2e13, gamma_b=2e13,
                t20=1e-12, t21=100e-15, t10=300e-12, N_0=5e23, literal=literal)


def drude_params_metal() -> dict:
    """A single-pole Drude metal for the reference's Drude class (Drude.cpp):
    eps_inf 1, omega_P 1.37e16 rad/s, gamma 1e14 1/s (as Hz on the deck, the
    class multiplies by 2 pi), conductivity 1e4 S/m."""
    two_pi = 2.0 * PI
    return dict(epsInf=1.0, fP=1.37e16 / two_pi, sigma=1.0e4, gamma=1.0e14 / two_pi)


def drude_as_dl(drude: dict) -> dict:
    """The Drude class as the engine's Drude-Lorentz module: one Drude pole, no
    Lorentz pole, the coefficients of Drude.cpp (literal = 2)."""
    return dict(sigma=drude["sigma"], epsInf=drude["epsInf"], fD=[drude["fP"]], gD=[drude["gamma"]],
                fL=[], dL=[], depsL=[], literal=2)


def gain_params_laser(pump: float = 1.0e9) -> dict:
    """Config-3 gain.  tau30, lambda_b and gamma_b are not given by the
    workload; they are chosen here as 100 fs, 450 nm and 2e13 1/s."""
    return dict(lambda_a=600e-9, lambda_b=450e-9, gamma_a=2.0e13, gamma_b=2.0e13,
                t30=100e-15, t32=100e-15, t21=300e-12, t10=100e-15, N_0=5.0e23, pump=pump)


# ---------------------------------------------------------------- configs

def config1(n: int = 96, steps: int = 1000) -> Deck:
    """Plain FP64 96^3 scatterer: vacuum, sphere eps 2.25 r = 20 cells at the
    centre, CPML 10, Ez point source at (30,48,48) (scaled with n), line port
    along x through the centre."""
    d = 10e-9
    dk = Deck(n, n, n, d, d, d, name="c1")
    dk.media = [(1.0, 1.0, 0.0, 0.0), (2.25, 1.0, 0.0, 0.0)]
    c = n // 2
    r = 20 * n / 96.0
    dk.shapes = [Shape(1, "ellipsoid", c * d, c * d, c * d, r * d, r * d, r * d)]
    dk.pml = pml_params(max(4, round(10 * n / 96)))
    tau = 5e-15
    wave = gaussian_sine(steps + dk.n0 + 1, dk.dt, 600e-9, tau, 3 * tau)
    dk.sources = [(COMP["Ez"], round(30 * n / 96), c, c, wave)]
    dk.ports = [Port("plain", dict(dir="z", position=(c + 0.5) * d, w1=0.5 * d, w2=(n - 1 + 0.5) * d,
                                   h1=(c + 0.5) * d, h2=(c + 0.5) * d))]
    dk.nsteps = steps
    return dk


def config2(n: int = 256, steps: int = 4000, nfreq: int = 64, ports: bool = True) -> Deck:
    """Dispersive scattering: CPML 12, TF/SF inset 20, Gaussian beam
    (w0 400 nm, 550 nm, theta 30, phi 45, psi 0 chosen), 4x4x4 Drude-Lorentz
    spheres r 15 pitch 40 centred, six planar ports 2 cells outside the TF/SF
    faces with DFT at nfreq frequencies over lambda0 +- FWHM.  Sizes scale with
    n/256 for parity-sized decks."""
    d = 5e-9
    s = n / 256.0
    dk = Deck(n, n, n, d, d, d, name="c2")
    dk.media = [(1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0)]
    r = 15 * s
    pitch = 40 * s
    first = n / 2.0 - 1.5 * pitch
    dk.shapes = [
        Shape(2, "ellipsoid", first * d, first * d, first * d, r * d, r * d, r * d),
        Shape(0, "multi", first * d, first * d, first * d, pitch * d, pitch * d, pitch * d,
              theta=4, phi=4, psi=4),
    ]
    npml = max(4, round(12 * s))
    inset = max(npml + 3, round(20 * s))
    dk.pml = pml_params(npml)
    lam = 550e-9
    tau = 4e-15
    dk.tfsf = dict(lam=lam, dlambda=dlambda_for_tau(lam, tau), w0=400e-9 * s, z0_deck=0.0,
                   xs=(n / 2 + 0.5) * d, ys=(n / 2 + 0.5) * d, zs=0.0, k0=n // 2,
                   theta=30.0, phi=45.0, E0=1.0, psi=0.0, n6=[inset] * 6,
                   Nt=steps + dk.n0 + 1, cwmode=0)
    dk.tfsf["lambda"] = dk.tfsf.pop("lam")
    if ports:
        fwhm = 2.0 * math.sqrt(math.log(2.0)) * tau       # intensity FWHM of the envelope
        nu0 = C0 / lam
        dnu = 2.0 * math.log(2.0) / (PI * fwhm) * 2.0
        freqs = np.linspace(nu0 - dnu, nu0 + dnu, nfreq)
        lo, hi = inset - 2, n - inset + 2
        for axis in "xyz":
            for pos in (lo, hi):
                dk.ports.append(Port("plain", dict(dir=axis, position=(pos + 0.5) * d,
                                                   w1=(lo + 0.5) * d, w2=(hi + 0.5) * d,
                                                   h1=(lo + 0.5) * d, h2=(hi + 0.5) * d),
                                     dft_freqs=freqs, dft_mask=_tangential_mask(axis)))
    dk.dl = dl_params_metal()
    dk.nsteps = steps
    return dk


def _tangential_mask(axis: str) -> int:
    t = {"x": ("Ey", "Ez", "Hy", "Hz"), "y": ("Ex", "Ez", "Hx", "Hz"), "z": ("Ex", "Ey", "Hx", "Hy")}[axis]
    m = 0
    for c in t:
        m |= 1 << COMP[c]
    return m


def jittered_lattice(n, pitch: float, jitter: float, seed: int):
    """Centres (cells) of a simple-cubic lattice filling [0,n)^3 (or a box
    n = (nx, ny, nz)), jittered by U[-jitter, jitter] per axis from a PCG64
    stream."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dims = (n, n, n) if np.isscalar(n) else tuple(n)
    axes = []
    for m_ in dims:
        m = max(1, int(m_ // pitch))
        off = (m_ - (m - 1) * pitch) / 2.0
        axes.append(off + pitch * np.arange(m))
    cx, cy, cz = np.meshgrid(*axes, indexing="ij")
    cen = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    return cen + rng.uniform(-jitter, jitter, size=cen.shape)


def config3(n: int = 384, steps: int = 20000, seed: int = 0, nfreq: int = 0,
            npml: Optional[int] = None, pitch: Optional[float] = None,
            radius: Optional[float] = None, port: bool = True) -> Deck:
    """Disordered photonic-crystal laser: background eps 2.25 doped with
    four-level gain (ID 5), SC lattice of eps 11.9 spheres (ID 3) r 8 pitch 30
    jittered +-4 cells, CPML 16, Gaussian seed pulse (Ez dipole at the centre),
    spherical port r 150 cells.  Sizes scale with n/384."""
    d = 10e-9
    s = n / 384.0
    dk = Deck(n, n, n, d, d, d, name="c3")
    dk.media = [(1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0),
                (11.9, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0), (2.25, 1.0, 0.0, 0.0)]
    pitch = pitch if pitch is not None else 30 * s
    radius = radius if radius is not None else 8 * s
    cen = jittered_lattice(n, pitch, 4 * s, seed)
    dk.ids = rasterize_spheres(dk.shape3, dk.dx, cen, radius, 3, background=ID_GAIN)
    dk.pml = pml_params(npml if npml is not None else max(4, round(16 * s)))
    dk.gain = gain_params_laser()
    c = n // 2
    wave = gaussian_sine(steps + dk.n0 + 1, dk.dt, 600e-9, 5e-15, 15e-15)
    dk.sources = [(COMP["Ez"], c, c, c, wave)]
    if port:
        r = 150 * s
        dk.ports.append(Port("spherical", dict(r=r * d, xc=(c + 0.5) * d, yc=(c + 0.5) * d, zc=(c + 0.5) * d,
                                               theta1=0.0, theta2=180.0, phi1=0.0, phi2=360.0),
                             dft_freqs=(np.linspace(0.9, 1.1, nfreq) * C0 / 600e-9) if nfreq else None))
    dk.nsteps = steps
    return dk


def config4_member(nx: int, ny: int, nz: int, seed: int, steps: int = 5000, nfreq: int = 32,
                   npml: int = 8, port: bool = True) -> Deck:
    """One realization of the disordered-crystal ensemble: the materials and
    gain of config3 (spheres eps 11.9 r 8 pitch 30 jittered +-4 from `seed` in
    a gain-doped eps 2.25 background) in an nx x ny x nz box, CPML npml, Ez
    seed pulse at the centre, spherical port of radius min(n)/2 - npml - 3
    cells with an FP64 DFT at nfreq frequencies around 600 nm."""
    d = 10e-9
    dk = Deck(nx, ny, nz, d, d, d, name=f"c4_{seed}")
    dk.media = [(1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0),
                (11.9, 1.0, 0.0, 0.0), (1.0, 1.0, 0.0, 0.0), (2.25, 1.0, 0.0, 0.0)]
    cen = jittered_lattice((nx, ny, nz), 30.0, 4.0, seed)
    dk.ids = rasterize_spheres(dk.shape3, dk.dx, cen, 8.0, 3, background=ID_GAIN)
    dk.pml = pml_params(npml)
    dk.gain = gain_params_laser()
    c = (nx // 2, ny // 2, nz // 2)
    wave = gaussian_sine(steps + dk.n0 + 1, dk.dt, 600e-9, 5e-15, 15e-15)
    dk.sources = [(COMP["Ez"], c[0], c[1], c[2], wave)]
    r = min(nx, ny, nz) / 2.0 - npml - 3
    if port and r >= 3:
        dk.ports.append(Port("spherical", dict(r=r * d, xc=(c[0] + 0.5) * d, yc=(c[1] + 0.5) * d,
                                               zc=(c[2] + 0.5) * d, theta1=0.0, theta2=180.0, phi1=0.0,
                                               phi2=360.0),
                             dft_freqs=(np.linspace(0.9, 1.1, nfreq) * C0 / 600e-9) if nfreq else None))
    dk.nsteps = steps
    return dk


def config4_shapes(count: int = 256, seed: int = 0, edges=(64, 80, 96, 112, 128)):
    """Box shapes of the ensemble: each axis drawn uniformly from `edges`
    (PCG64 stream from `seed`), so anisotropic mixes such as 128x64x96 occur."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [tuple(int(v) for v in rng.choice(edges, size=3)) for _ in range(count)]


def rasterize_spheres(shape3, d: float, centres, radius: float, mat: int, background: int = 0) -> np.ndarray:
    """ID grid with spheres drawn over a background value.  A cell (i,j,k) is
    inside when ((i d - x0)^2 + (j d - y0)^2 + (k d - z0)^2)/r^2 <= 1 with
    centres and radius in metres, the predicate of Structure.cpp:205-221, over
    i < Nx, j < Ny, k < Nz as the reference loops."""
    nx1, ny1, nz1 = shape3
    ids = np.full(shape3, background, dtype=np.uint8)
    r = radius * d
    for c in centres:
        x0, y0, z0 = (float(v) * d for v in c)
        lo = [max(0, int(math.floor(v - radius)) - 1) for v in c]
        hi = [min(m - 1, int(math.ceil(v + radius)) + 2) for v, m in zip(c, (nx1, ny1, nz1))]
        ii = np.arange(lo[0], hi[0]).astype(np.float64)
        jj = np.arange(lo[1], hi[1]).astype(np.float64)
        kk = np.arange(lo[2], hi[2]).astype(np.float64)
        tx = (ii * d - x0) * (ii * d - x0) / (r * r)
        ty = (jj * d - y0) * (jj * d - y0) / (r * r)
        tz = (kk * d - z0) * (kk * d - z0) / (r * r)
        inside = (tx[:, None, None] + ty[None, :, None]) + tz[None, None, :] <= 1.0
        ids[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]][inside] = mat
    return ids
