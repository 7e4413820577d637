"""ctypes binding of liboracle.so and runners for the reference harnesses.

TEST INFRASTRUCTURE ONLY.  Importable from tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg; the product never imports it.

``Oracle.from_deck(deck, ids)`` builds the FP64 CPU restatement for a
``cpsfdtd_b200.decks.Deck``; ``run_ref_harness`` runs the reference's own code
(oracle/_ref/ref_harness) on the same deck and returns its dumps.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")
REF_BENCH = os.path.join(HERE, "_ref", "ref_bench")
REF2D = os.path.join(HERE, "_ref", "ref2d_harness")

_lib = None


class TfsfParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("dlambda", C.c_double), ("w0", C.c_double), ("z0", C.c_double),
                ("i0", C.c_int32), ("j0", C.c_int32), ("k0", C.c_int32),
                ("theta_deg", C.c_double), ("phi_deg", C.c_double), ("E0", C.c_double), ("psi_deg", C.c_double),
                ("n_x1", C.c_int32), ("n_x2", C.c_int32), ("n_y1", C.c_int32), ("n_y2", C.c_int32),
                ("n_z1", C.c_int32), ("n_z2", C.c_int32), ("Nt", C.c_int32), ("cwmode", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, capture_output=True)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        dp = C.POINTER(C.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_destroy.argtypes = [P]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_media.argtypes = [P, C.c_int, dp, dp, dp, dp]
        L.orc_set_ids.argtypes = [P, C.c_void_p]
        L.orc_pml_init.argtypes = [P, C.POINTER(C.c_int32), C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int]
        L.orc_dl_init.argtypes = [P, C.c_double, C.c_double, C.c_int, dp, dp, C.c_int, dp, dp, dp, C.c_int]
        L.orc_gain_init.argtypes = [P, C.c_int] + [C.c_double] * 10
        L.orc_tfsf_init.argtypes = [P, C.POINTER(TfsfParams)]
        L.orc_tfsf_tables.argtypes = [P, dp, dp]
        L.orc_source_add.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int, dp, C.c_int]
        L.orc_port_add.argtypes = [P, C.c_int, C.POINTER(C.c_int32)]
        L.orc_port_set_dft.argtypes = [P, C.c_int, C.c_int, dp, C.c_uint32]
        L.orc_set_step.argtypes = [P, C.c_int64]
        L.orc_get_step.restype = C.c_int64
        L.orc_get_step.argtypes = [P]
        L.orc_step.argtypes = [P, C.c_int]
        L.orc_get_field.argtypes = [P, C.c_int, dp]
        L.orc_set_field.argtypes = [P, C.c_int, dp]
        L.orc_get_stretch.argtypes = [P, C.c_int, dp]
        L.orc_port_read.argtypes = [P, C.c_int, dp]
        L.orc_port_dft_read.argtypes = [P, C.c_int, dp]
        L.orc_gain_populations.argtypes = [P, dp]
        L.orc_three_init.argtypes = [P, C.c_int] + [C.c_double] * 8 + [C.c_int]
        L.orc_three_populations.argtypes = [P, dp]
        L.orc_count_cells.restype = C.c_int64
        L.orc_count_cells.argtypes = [P, C.c_int]
        for name in ("orc_op_h_bulk", "orc_op_h_pml", "orc_op_e_bulk", "orc_op_e_pml", "orc_op_dl",
                     "orc_op_gain_p", "orc_op_gain_e", "orc_op_gain_n",
                     "orc_op_three_p", "orc_op_three_e", "orc_op_three_n"):
            getattr(L, name).argtypes = [P]
        for name in ("orc_op_tfsf_h", "orc_op_tfsf_e", "orc_op_sources", "orc_op_ports"):
            getattr(L, name).argtypes = [P, C.c_int]
        L.orc2d_run.argtypes = ([C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_void_p, C.c_int,
                                 dp, dp, dp, dp, C.c_int, C.c_double, C.c_double, C.c_int, dp, dp, C.c_int,
                                 dp, dp, dp, C.c_int, C.c_int, dp, C.c_int, C.c_int, dp, C.c_int, dp, dp, dp])
        _lib = L
    return _lib


def _dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """FP64 CPU restatement of one grid."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt):
        self.L = lib()
        self.h = self.L.orc_create(nx, ny, nz, dx, dy, dz, dt)
        if not self.h:
            raise ValueError("orc_create failed")
        self.shape3 = (nx + 1, ny + 1, nz + 1)
        self.nports = []

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    @staticmethod
    def threads(n=0):
        return lib().orc_set_threads(n)

    @classmethod
    def from_deck(cls, dk, ids, port_points=None):
        o = cls(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.dt)
        m = np.array(dk.media, dtype=np.float64).reshape(-1, 4)
        keep = [_dp(m[:, c]) for c in range(4)]
        assert o.L.orc_set_media(o.h, len(m), *[k[1] for k in keep]) == 0
        ids = np.ascontiguousarray(ids, dtype=np.uint8)
        assert ids.shape == o.shape3
        o.L.orc_set_ids(o.h, ids.ctypes.data)
        if dk.pml:
            p = dk.pml
            n = (C.c_int32 * 6)(*p["npml"])
            assert o.L.orc_pml_init(o.h, n, p["m"], p["malp"], p["kapmax"], p["sig_ratio"], p["alpmax"],
                                    int(p.get("literal", 0))) == 0
        if dk.dl:
            d = dk.dl
            a = [_dp(d[k]) for k in ("fD", "gD", "fL", "dL", "depsL")]
            assert o.L.orc_dl_init(o.h, d["sigma"], d["epsInf"], len(d["fD"]), a[0][1], a[1][1],
                                   len(d["fL"]), a[2][1], a[3][1], a[4][1], int(d.get("literal", 0))) == 0
        if dk.gain:
            g = dk.gain
            assert o.L.orc_gain_init(o.h, 5, g["lambda_a"], g["lambda_b"], g["gamma_a"], g["gamma_b"],
                                     g["t30"], g["t32"], g["t21"], g["t10"], g["N_0"], g.get("pump", 0.0)) == 0
        if getattr(dk, "three", None):
            t3 = dk.three
            assert o.L.orc_three_init(o.h, int(t3.get("gain_id", 5)), t3["lambda_a"], t3["lambda_b"], t3["gamma_a"],
                                      t3["gamma_b"], t3["t20"], t3["t21"], t3["t10"], t3["N_0"],
                                      int(t3.get("literal", 0))) == 0
        if dk.tfsf:
            t = dk.tfsf_abi()
            tp = TfsfParams(t["lambda_"], t["dlambda"], t["w0"], t["z0"], t["i0"], t["j0"], t["k0"],
                            t["theta"], t["phi"], t["E0"], t["psi"], *t["n6"], t["Nt"], t["cwmode"])
            assert o.L.orc_tfsf_init(o.h, C.byref(tp)) == 0
        for comp, i, j, k, wave in dk.sources:
            w = _dp(wave)
            assert o.L.orc_source_add(o.h, comp, i, j, k, w[1], len(w[0])) == 0
        if port_points is not None:
            for p, pts in zip(dk.ports, port_points):
                pid = o.add_port(pts)
                if p.dft_freqs is not None:
                    f = _dp(p.dft_freqs)
                    assert o.L.orc_port_set_dft(o.h, pid, len(f[0]), f[1], p.dft_mask) == 0
        o.L.orc_set_step(o.h, dk.n0)
        return o

    def add_port(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.int32).reshape(-1, 3)
        pid = self.L.orc_port_add(self.h, len(pts), pts.ctypes.data_as(C.POINTER(C.c_int32)))
        if pid < 0:
            raise ValueError("orc_port_add failed")
        self.nports.append(len(pts))
        return pid

    def step(self, n=1):
        self.L.orc_step(self.h, n)

    def field(self, comp):
        out = np.empty(self.shape3, dtype=np.float64)
        self.L.orc_get_field(self.h, comp, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def fields(self):
        return [self.field(c) for c in range(6)]

    def set_field(self, comp, a):
        a, p = _dp(a)
        self.L.orc_set_field(self.h, comp, p)

    def stretch(self, which, n):
        out = np.empty(n)
        self.L.orc_get_stretch(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def port_last(self, p):
        out = np.empty((self.nports[p], 6))
        self.L.orc_port_read(self.h, p, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def port_dft(self, p, ncomp, nfreq):
        out = np.empty((self.nports[p], ncomp, nfreq, 2))
        assert self.L.orc_port_dft_read(self.h, p, out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        return out

    def tfsf_tables(self, Nt):
        e = np.empty(Nt + 1)
        h = np.empty(Nt + 1)
        self.L.orc_tfsf_tables(self.h, e.ctypes.data_as(C.POINTER(C.c_double)), h.ctypes.data_as(C.POINTER(C.c_double)))
        return e, h

    def populations(self):
        n = self.L.orc_count_cells(self.h, 1)
        out = np.empty((n, 4))
        self.L.orc_gain_populations(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def three_populations(self):
        """N0 N1 N2 per three-level site, sites in [i][j][k] order"""
        n = self.L.orc_count_cells(self.h, 2)
        out = np.empty((n, 3))
        self.L.orc_three_populations(self.h, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out


def have_reference_build() -> bool:
    return os.path.exists(REF_HARNESS) and os.path.exists(REF2D)


def run_ref_harness(dk, workdir=None, record_ports=False, exe=None, timeout=600):
    """Run the reference's own code on a deck; returns a dict of numpy arrays:
    ids, Ex..Hz, stretch (12 arrays), tfsf (Einc, Hinc), port points/last/series."""
    own = workdir is None
    workdir = workdir or tempfile.mkdtemp(prefix="cps_ref_")
    deck_dir = os.path.join(workdir, "deck")
    out_dir = os.path.join(workdir, "out")
    os.makedirs(out_dir, exist_ok=True)
    dk.write(deck_dir, record_ports=record_ports)
    # cwd: the reference's CW-mode TF/SF writes Pout.txt into the working directory
    r = subprocess.run([exe or REF_HARNESS, deck_dir, out_dir], capture_output=True, text=True, timeout=timeout,
                       cwd=out_dir)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
    info = {}
    for line in open(os.path.join(out_dir, "info.txt")):
        k, v = line.split()
        info[k] = float(v) if "." in v or "e" in v else int(v)
    nx, ny, nz = info["Nx"], info["Ny"], info["Nz"]
    shp = (nx + 1, ny + 1, nz + 1)
    res = {"info": info, "ids": np.fromfile(os.path.join(out_dir, "ids.bin"), dtype=np.uint8).reshape(shp)}
    for c, name in enumerate(("Ex", "Ey", "Ez", "Hx", "Hy", "Hz")):
        res[name] = np.fromfile(os.path.join(out_dir, name + ".bin")).reshape(shp)
    st = np.fromfile(os.path.join(out_dir, "stretch.bin"))
    lens = [nz, nz, ny, ny, nx, nx, nz, nz, ny, ny, nx, nx]
    res["stretch"] = np.split(st, np.cumsum(lens)[:-1])
    tf = os.path.join(out_dir, "tfsf_inc.bin")
    if os.path.exists(tf):
        t = np.fromfile(tf)
        res["tfsf"] = (t[: len(t) // 2], t[len(t) // 2:])
    res["ports"] = []
    for p in range(info["nports"]):
        pts = np.fromfile(os.path.join(out_dir, f"port{p}_points.bin"), dtype=np.int32).reshape(-1, 3)
        last = np.fromfile(os.path.join(out_dir, f"port{p}_last.bin")).reshape(-1, 6)
        entry = {"points": pts, "last": last}
        sf = os.path.join(out_dir, f"port{p}_series.bin")
        if os.path.exists(sf):
            entry["series"] = np.fromfile(sf).reshape(-1, len(pts), 6)
        res["ports"].append(entry)
    if own:
        import shutil
        shutil.rmtree(workdir, ignore_errors=True)
    return res


def ref_bench(dk, warm, timed, threads=0, exe=None, timeout=900):
    """Time `timed` steps of the reference's code (ref_bench build) after
    `warm` warm-up steps; returns the parsed REF_BENCH record."""
    import json
    workdir = tempfile.mkdtemp(prefix="cps_refb_")
    try:
        deck_dir = os.path.join(workdir, "deck")
        dk.write(deck_dir, bench=(warm, timed), threads=threads)
        r = subprocess.run([exe or REF_BENCH, deck_dir, workdir], capture_output=True, text=True, timeout=timeout,
                           cwd=workdir)
        if r.returncode != 0:
            raise RuntimeError(f"ref_bench failed ({r.returncode}): {r.stderr[-2000:]}")
        for line in r.stdout.splitlines():
            if line.startswith("REF_BENCH "):
                return json.loads(line[len("REF_BENCH "):])
        raise RuntimeError("ref_bench printed no record")
    finally:
        import shutil
        shutil.rmtree(workdir, ignore_errors=True)


def write_three_deck(path, three):
    """ThreeLevel.txt in the reference's format (ThreeLevel.cpp:37-84), "cells" placement."""
    with open(path, "w") as f:
        f.write("cells\n0\n0 0\n0 0\n")
        for key in ("lambda_a", "lambda_b", "gamma_a", "gamma_b", "t20", "t21", "t10", "N_0"):
            f.write(f"{float(three[key])!r}\n")
        f.write("0\n")


def run_ref2d(params, media, ids2d, wave, dl=None, gain=None, drude=None, three=None, timeout=120):
    """Run the reference's 2-D Drude_Lorentz / FourLevelLaser / Drude classes.
    params: dict nx ny dx dy dt nsteps si sj; drude: dict epsInf fP sigma gamma
    (Hz) for the single-pole Drude class.  Returns (Ex, Ey, Hz)."""
    workdir = tempfile.mkdtemp(prefix="cps_ref2d_")
    try:
        p = params
        with open(os.path.join(workdir, "params2d.txt"), "w") as f:
            f.write(f"{p['nx']} {p['ny']} {float(p['dx'])!r} {float(p['dy'])!r} {float(p['dt'])!r} {p['nsteps']} {p['si']} {p['sj']} "
                    f"{1 if dl else 0} {1 if gain else 0} {int((dl or {}).get('literal', 0))} {1 if drude else 0} "
                    f"{1 if three else 0}\n")
        with open(os.path.join(workdir, "media2d.txt"), "w") as f:
            f.write(f"{len(media)}\n")
            for m in media:
                f.write(" ".join(repr(float(v)) for v in m) + "\n")
        np.ascontiguousarray(ids2d, dtype=np.uint8).tofile(os.path.join(workdir, "ids2d.bin"))
        np.ascontiguousarray(wave, dtype=np.float64).tofile(os.path.join(workdir, "wave.bin"))
        if dl:
            with open(os.path.join(workdir, "DrudeLorentz.txt"), "w") as f:
                f.write(f"{len(dl['fD'])}\n{len(dl['fL'])}\n{float(dl['sigma'])!r}\n{float(dl['epsInf'])!r}\n")
                for a, b in zip(dl["fD"], dl["gD"]):
                    f.write(f"{float(a)!r}\t{float(b)!r}\n")
                for a, b, c in zip(dl["fL"], dl["dL"], dl["depsL"]):
                    f.write(f"{float(a)!r}\t{float(b)!r}\t{float(c)!r}\n")
        if three:
            write_three_deck(os.path.join(workdir, "ThreeLevel.txt"), three)
        if drude:
            with open(os.path.join(workdir, "Drude.txt"), "w") as f:
                for key in ("epsInf", "fP", "sigma", "gamma"):
                    f.write(f"{float(drude[key])!r}\n")
        if gain:
            g = gain
            with open(os.path.join(workdir, "FourLevelLaser.txt"), "w") as f:
                f.write("cells\n0\n0 0\n0 0\n")
                for key in ("lambda_b", "lambda_a", "gamma_a", "gamma_b", "t30", "t32", "t21", "t10", "N_0"):
                    f.write(f"{float(g[key])!r}\n")
                f.write("0\n")
        r = subprocess.run([REF2D, workdir, workdir], capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref2d_harness failed: {r.stderr[-2000:]}")
        shp = (p["nx"] + 1, p["ny"] + 1)
        return tuple(np.fromfile(os.path.join(workdir, n)).reshape(shp) for n in ("Ex2d.bin", "Ey2d.bin", "Hz2d.bin"))
    finally:
        import shutil
        shutil.rmtree(workdir, ignore_errors=True)


def drude_as_dl(drude):
    """The single-pole Drude class as the oracle's Drude-Lorentz recursion with
    one Drude pole and the coefficients of Drude.cpp (literal = 2)."""
    return dict(sigma=drude["sigma"], epsInf=drude["epsInf"], fD=[drude["fP"]], gD=[drude["gamma"]],
                fL=[], dL=[], depsL=[], literal=2)


def run_orc2d(params, media, ids2d, wave, dl=None, gain=None, drude=None, three=None):
    """The oracle's 2-D TE driver on the same problem as run_ref2d; three: the
    three-level gain with literal = 1 reproducing the reference's class."""
    L = lib()
    if drude:
        dl = drude_as_dl(drude)
    p = params
    m = np.array(media, dtype=np.float64).reshape(-1, 4)
    cols = [_dp(m[:, c]) for c in range(4)]
    ids2d = np.ascontiguousarray(ids2d, dtype=np.uint8)
    shp = (p["nx"] + 1, p["ny"] + 1)
    Ex, Ey, Hz = (np.zeros(shp) for _ in range(3))
    empty = _dp(np.zeros(1))
    d = dl or dict(sigma=0.0, epsInf=1.0, fD=[], gD=[], fL=[], dL=[], depsL=[])
    arrs = [_dp(np.array(d[k] if len(d[k]) else [0.0], dtype=np.float64)) for k in ("fD", "gD", "fL", "dL", "depsL")]
    if three:
        gp = _dp(np.array([three[k] for k in ("lambda_a", "lambda_b", "gamma_a", "gamma_b", "t20", "t21", "t10", "N_0")]
                          + [float(three.get("literal", 0)), 0.0]))
    else:
        gp = _dp(np.array([gain[k] for k in ("lambda_a", "lambda_b", "gamma_a", "gamma_b", "t30", "t32", "t21", "t10",
                                             "N_0")] + [gain.get("pump", 0.0)]) if gain else np.zeros(10))
    w = _dp(wave)
    rc = L.orc2d_run(p["nx"], p["ny"], p["dx"], p["dy"], p["dt"], ids2d.ctypes.data, len(m),
                     cols[0][1], cols[1][1], cols[2][1], cols[3][1],
                     1 if dl else 0, d["sigma"], d["epsInf"], len(d["fD"]), arrs[0][1], arrs[1][1],
                     len(d["fL"]), arrs[2][1], arrs[3][1], arrs[4][1], int(d.get("literal", 0)),
                     2 if three else (1 if gain else 0), gp[1], p["si"], p["sj"], w[1], p["nsteps"],
                     Ex.ctypes.data_as(C.POINTER(C.c_double)), Ey.ctypes.data_as(C.POINTER(C.c_double)),
                     Hz.ctypes.data_as(C.POINTER(C.c_double)))
    del empty
    assert rc == 0
    return Ex, Ey, Hz
