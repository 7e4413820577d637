"""cpsfdtd_b200 -- B200-native time-stepping engine for cpsFDTD workloads.

This module is a thin ctypes binding of ``libcpsfdtd.so`` (the C ABI declared
in ``include/cps_capi.h``).  All compute runs in the CUDA kernels of that
library; there is no CPU fallback: importing works without a GPU, but
creating a :class:`Grid` without the built library or without a CUDA device
raises.

``Grid.from_deck(deck)`` sets up one simulation from a
:class:`cpsfdtd_b200.decks.Deck` the same way the reference's constructors
do (Structure, CPML, Drude_Lorentz, FourLevelLaser, TF_SF, ports).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

from .decks import ID_DISPERSIVE

import numpy as np

__all__ = ["Grid", "Batch", "Server", "footprint", "CpsError", "lib", "FP64", "FP32", "PLAIN", "FUSED", "ONEPASS", "LIB_PATH"]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcpsfdtd.so")

FP64, FP32 = 0, 1
PLAIN, FUSED, ONEPASS = 0, 1, 2
MAX_POLES = 8

_lib = None


class CpsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cps error {code}: {msg}")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt", C.c_double),
                ("precision", C.c_int32), ("device", C.c_int32)]


class PmlParams(C.Structure):
    _fields_ = [("npml", C.c_int32 * 6), ("m", C.c_double), ("malp", C.c_double), ("kapmax", C.c_double),
                ("sig_ratio", C.c_double), ("alpmax", C.c_double), ("literal", C.c_int32)]


class DlParams(C.Structure):
    _fields_ = [("sigma", C.c_double), ("epsInf", C.c_double), ("nD", C.c_int32), ("nL", C.c_int32),
                ("fD", C.c_double * MAX_POLES), ("gD", C.c_double * MAX_POLES),
                ("fL", C.c_double * MAX_POLES), ("dL", C.c_double * MAX_POLES), ("depsL", C.c_double * MAX_POLES),
                ("literal", C.c_int32)]


class DrudeParams(C.Structure):
    _fields_ = [("epsInf", C.c_double), ("omegaP_hz", C.c_double), ("sigma", C.c_double), ("gamma_hz", C.c_double)]


class ThreeParams(C.Structure):
    _fields_ = [("gain_id", C.c_int32), ("lambda_a", C.c_double), ("lambda_b", C.c_double),
                ("gamma_a", C.c_double), ("gamma_b", C.c_double), ("t20", C.c_double), ("t21", C.c_double),
                ("t10", C.c_double), ("N_0", C.c_double), ("N_1", C.c_double), ("literal", C.c_int32)]


class GainParams(C.Structure):
    _fields_ = [("gain_id", C.c_int32), ("lambda_a", C.c_double), ("lambda_b", C.c_double),
                ("gamma_a", C.c_double), ("gamma_b", C.c_double), ("t30", C.c_double), ("t32", C.c_double),
                ("t21", C.c_double), ("t10", C.c_double), ("N_0", C.c_double), ("pump_rate", C.c_double)]


class TfsfParams(C.Structure):
    _fields_ = [("lambda_", C.c_double), ("dlambda", C.c_double), ("w0", C.c_double), ("z0", C.c_double),
                ("i0", C.c_int32), ("j0", C.c_int32), ("k0", C.c_int32),
                ("theta_deg", C.c_double), ("phi_deg", C.c_double), ("E0", C.c_double), ("psi_deg", C.c_double),
                ("n", C.c_int32 * 6), ("Nt", C.c_int32), ("cwmode", C.c_int32)]


class Shape(C.Structure):
    _fields_ = [("type", C.c_int32), ("material_index", C.c_int32), ("theta", C.c_double), ("phi", C.c_double),
                ("psi", C.c_double), ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double)]


SHAPE_TYPES = {"cuboid": 0, "ellipsoid": 1, "cylinder": 2, "multi": 3}


def lib():
    """Load libcpsfdtd.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cpsfdtd_b200.build`")
        L = C.CDLL(LIB_PATH)
        P, I32, I64, D, U32 = C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_uint32
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int32)
        sigs = {
            "cps_last_error": ([], C.c_char_p), "cps_version": ([], C.c_char_p),
            "cps_courant_dt": ([D, D, D], D),
            "cps_grid_create": ([C.POINTER(GridDesc), C.POINTER(P)], I32),
            "cps_grid_destroy": ([P], I32), "cps_grid_info": ([P, C.POINTER(GridDesc)], I32),
            "cps_grid_bytes": ([P, C.POINTER(I64)], I32),
            "cps_grid_set_stream": ([P, P], I32), "cps_grid_get_stream": ([P, C.POINTER(P)], I32),
            "cps_synchronize": ([P], I32),
            "cps_grid_set_media": ([P, I32, dp, dp, dp, dp], I32),
            "cps_grid_upload_ids": ([P, P], I32), "cps_grid_download_ids": ([P, P], I32),
            "cps_mesh_rasterize": ([I32, I32, I32, D, D, D, I32, C.POINTER(Shape), P, I32], I32),
            "cps_pml_init": ([P, C.POINTER(PmlParams)], I32),
            "cps_dl_init": ([P, C.POINTER(DlParams)], I32),
            "cps_drude_init": ([P, C.POINTER(DrudeParams)], I32),
            "cps_grid_rasterize": ([P, I32, C.POINTER(Shape), I32], I32),
            "cps_deck_load": ([C.c_char_p, I32, C.POINTER(P)], I32),
            "cps_field_slice": ([P, I32, I32, I32, dp], I32),
            "cps_image_png": ([C.c_char_p, I32, I32, dp, D, D], I32),
            "cps_png_rgb": ([C.c_char_p, I32, I32, C.c_void_p], I32),
            "cps_grid_energy": ([P, C.POINTER(D), C.POINTER(D)], I32),
            "cps_three_init": ([P, C.POINTER(ThreeParams)], I32),
            "cps_three_populations": ([P, dp, C.POINTER(I64)], I32),
            "cps_op_three_polarization": ([P], I32), "cps_op_three_efield": ([P], I32),
            "cps_op_three_populations": ([P], I32),
            "cps_gain_init": ([P, C.POINTER(GainParams)], I32),
            "cps_tfsf_init": ([P, C.POINTER(TfsfParams)], I32),
            "cps_tfsf_set_tables": ([P, I32, dp, dp], I32), "cps_tfsf_get_tables": ([P, I32, dp, dp], I32),
            "cps_source_add": ([P, I32, I32, I32, I32, dp, I32], I32),
            "cps_port_points_plain": ([I32, I32, I32, D, D, D, C.c_char, D, D, D, D, D, ip, ip], I32),
            "cps_port_points_spherical": ([I32, I32, I32, D, D, D, D, D, D, D, D, D, D, D, ip, ip], I32),
            "cps_port_add": ([P, I32, ip, ip], I32),
            "cps_port_set_dft": ([P, I32, I32, dp, U32], I32),
            "cps_port_read": ([P, I32, dp], I32), "cps_port_dft_read": ([P, I32, dp], I32),
            "cps_port_flux": ([P, I32, C.c_char, dp], I32),
            "cps_grid_set_step": ([P, I64], I32), "cps_grid_get_step": ([P, C.POINTER(I64)], I32),
            "cps_step": ([P, I32, I32], I32), "cps_grid_set_chunked": ([P, I32], I32),
            "cps_op_h_bulk": ([P], I32), "cps_op_e_bulk": ([P], I32), "cps_op_h_pml": ([P], I32),
            "cps_op_e_pml": ([P], I32), "cps_op_dl": ([P], I32), "cps_op_gain_polarization": ([P], I32),
            "cps_op_gain_efield": ([P], I32), "cps_op_gain_populations": ([P], I32),
            "cps_op_tfsf_h": ([P, I32, U32], I32), "cps_op_tfsf_e": ([P, I32, U32], I32),
            "cps_op_sources": ([P, I32], I32), "cps_op_port_sample": ([P, I32, I32], I32),
            "cps_grid_set_record": ([P, I32], I32),
            "cps_grid_record_stats": ([P, C.POINTER(I64), C.POINTER(I64), ip], I32),
            "cps_field_download": ([P, I32, dp], I32), "cps_field_upload": ([P, I32, dp], I32),
            "cps_field_download_f32": ([P, I32, C.POINTER(C.c_float)], I32),
            "cps_grid_reset": ([P, I64], I32), "cps_grid_check_finite": ([P, C.POINTER(I64)], I32),
            "cps_grid_set_wait_skew": ([P, I32], I32),
            "cps_gain_populations": ([P, dp, C.POINTER(I64)], I32),
            "cps_grid_launch_count": ([P, C.POINTER(I64)], I32),
            "cps_ports_flush": ([P], I32), "cps_grid_set_timing": ([P, I32], I32),
            "cps_grid_set_tile": ([P, I32, I32], I32), "cps_grid_get_tile": ([P, ip, ip], I32),
            "cps_grid_set_sweep": ([P, I32], I32),
            "cps_grid_timing": ([P, C.POINTER(D), C.POINTER(D), C.POINTER(I64)], I32),
            "cps_batch_create": ([I32, C.POINTER(P)], I32), "cps_batch_destroy": ([P], I32),
            "cps_batch_add": ([P, P], I32), "cps_batch_remove": ([P, P], I32),
            "cps_batch_info": ([P, ip, C.POINTER(I64)], I32), "cps_batch_step": ([P, I32], I32),
            "cps_batch_synchronize": ([P], I32), "cps_batch_set_tile": ([P, I32, I32, I32], I32),
            "cps_batch_get_tile": ([P, ip, ip, ip], I32), "cps_batch_set_graph": ([P, I32], I32),
            "cps_batch_get_stream": ([P, C.POINTER(P)], I32),
            "cps_batch_launch_count": ([P, C.POINTER(I64)], I32),
            "cps_batch_tune_key": ([P, C.c_char_p, I32], I32),
            "cps_batch_autotune": ([P, C.c_char_p, I32, ip], I32),
            "cps_server_create": ([P, C.POINTER(P)], I32), "cps_server_destroy": ([P], I32),
            "cps_server_submit": ([P, I64, I32, _BUILD_FN, _DONE_FN, P, C.POINTER(I64)], I32),
            "cps_server_poll": ([P, ip, ip], I32), "cps_server_drain": ([P], I32),
            "cps_server_cancel": ([P, I64], I32), "cps_server_get_stats": ([P, P], I32),
        }
        for name, (args, res) in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(code):
    if code != 0:
        raise CpsError(code, lib().cps_last_error().decode())


def _dp(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(C.POINTER(C.c_double))


def _shape_array(shapes):
    arr = (Shape * max(1, len(shapes)))()
    for n, s in enumerate(shapes):
        arr[n] = Shape(SHAPE_TYPES[s.type], s.mat, s.theta, s.phi, s.psi, s.x0, s.y0, s.z0, s.a, s.b, s.c)
    return arr


def rasterize(nx, ny, nz, dx, dy, dz, shapes) -> np.ndarray:
    """ID grid [i][j][k] of structure.txt shapes, as Structure::generate_mesh."""
    arr = _shape_array(shapes)
    ids = np.zeros((nx + 1, ny + 1, nz + 1), dtype=np.uint8)
    _check(lib().cps_mesh_rasterize(nx, ny, nz, dx, dy, dz, len(shapes), arr, ids.ctypes.data, 0))
    return ids


def image_png(path, values, cmin, cmax):
    """PNG of a 2-D array values[x][y] through the reference OutImage's colour map."""
    v = np.ascontiguousarray(values, dtype=np.float64)
    _check(lib().cps_image_png(os.fsencode(path), v.shape[0], v.shape[1], v.ctypes.data_as(C.POINTER(C.c_double)),
                               float(cmin), float(cmax)))


def port_points(deck, port) -> np.ndarray:
    """Point set [(i, j, k)] of a deck port, as the reference port constructors build it."""
    L = lib()
    q = port.params
    cnt = C.c_int32(0)
    if port.kind == "plain":
        args = (deck.nx, deck.ny, deck.nz, deck.dx, deck.dy, deck.dz, q["dir"].encode(), q["position"],
                q["w1"], q["w2"], q["h1"], q["h2"])
        _check(L.cps_port_points_plain(*args, C.byref(cnt), None))
        out = np.zeros((cnt.value, 3), dtype=np.int32)
        _check(L.cps_port_points_plain(*args, C.byref(cnt), out.ctypes.data_as(C.POINTER(C.c_int32))))
    else:
        args = (deck.nx, deck.ny, deck.nz, deck.dx, deck.dy, deck.dz, q["r"], q["xc"], q["yc"], q["zc"],
                q["theta1"], q["theta2"], q["phi1"], q["phi2"])
        _check(L.cps_port_points_spherical(*args, C.byref(cnt), None))
        out = np.zeros((cnt.value, 3), dtype=np.int32)
        _check(L.cps_port_points_spherical(*args, C.byref(cnt), out.ctypes.data_as(C.POINTER(C.c_int32))))
    return out


class Grid:
    """One simulation domain resident on one GPU."""

    def __init__(self, nx, ny, nz, dx, dy, dz, dt=0.0, precision=FP32, device=0):
        self.L = lib()
        self.h = C.c_void_p()
        self.desc = GridDesc(nx, ny, nz, dx, dy, dz, dt, precision, device)
        _check(self.L.cps_grid_create(C.byref(self.desc), C.byref(self.h)))
        info = GridDesc()
        _check(self.L.cps_grid_info(self.h, C.byref(info)))
        self.dt = info.dt
        self.shape3 = (nx + 1, ny + 1, nz + 1)
        self.precision = precision
        self.ports = []  # (npts, ncomp, nfreq)

    @classmethod
    def from_deck_dir(cls, path, precision=FP32):
        """A grid from a directory of the reference's deck files (cps_deck_load);
        its ports carry no DFT and it has no sources until they are added."""
        g = cls.__new__(cls)
        g.L = lib()
        g.h = C.c_void_p()
        _check(g.L.cps_deck_load(os.fsencode(path), precision, C.byref(g.h)))
        info = GridDesc()
        _check(g.L.cps_grid_info(g.h, C.byref(info)))
        g.desc = info
        g.dt = info.dt
        g.shape3 = (info.nx + 1, info.ny + 1, info.nz + 1)
        g.precision = precision
        g.ports = []
        return g

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.cps_grid_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------- setup
    @classmethod
    def from_deck(cls, dk, precision=FP32, ids: Optional[np.ndarray] = None, device=0, port_points_list=None,
                  device_raster=True):
        """A grid set up from a deck; the shapes of a deck without an ID array are
        rasterised on the device (device_raster=False: on the host, then uploaded)."""
        g = cls(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.dt, precision, device)
        g.set_media(dk.media)
        if ids is None and dk.ids is None and device_raster:
            g.rasterize(dk.shapes)
        else:
            if ids is None:
                ids = dk.ids if dk.ids is not None else rasterize(dk.nx, dk.ny, dk.nz, dk.dx, dk.dy, dk.dz, dk.shapes)
            g.upload_ids(ids)
        if dk.pml:
            g.pml_init(dk.pml)
        if dk.dl:
            g.dl_init(dk.dl)
        if dk.gain:
            g.gain_init(dk.gain)
        if getattr(dk, "three", None):
            g.three_init(dk.three)
        if dk.tfsf:
            g.tfsf_init(dk.tfsf_abi())
        for comp, i, j, k, wave in dk.sources:
            g.source_add(comp, i, j, k, wave)
        for n, p in enumerate(dk.ports):
            pts = port_points_list[n] if port_points_list is not None else port_points(dk, p)
            pid = g.port_add(pts)
            if p.dft_freqs is not None:
                g.port_set_dft(pid, p.dft_freqs, p.dft_mask)
        g.set_step(dk.n0)
        return g

    def set_media(self, media):
        m = np.array(media, dtype=np.float64).reshape(-1, 4)
        cols = [_dp(m[:, c]) for c in range(4)]
        _check(self.L.cps_grid_set_media(self.h, len(m), *[c[1] for c in cols]))

    def rasterize(self, shapes, keep=False):
        """Rasterise structure.txt shapes into the grid's IDs on the device."""
        _check(self.L.cps_grid_rasterize(self.h, len(shapes), _shape_array(shapes), 1 if keep else 0))

    def upload_ids(self, ids):
        ids = np.ascontiguousarray(ids, dtype=np.uint8)
        assert ids.shape == self.shape3, (ids.shape, self.shape3)
        _check(self.L.cps_grid_upload_ids(self.h, ids.ctypes.data))

    def download_ids(self):
        out = np.empty(self.shape3, dtype=np.uint8)
        _check(self.L.cps_grid_download_ids(self.h, out.ctypes.data))
        return out

    def pml_init(self, p):
        pp = PmlParams((C.c_int32 * 6)(*p["npml"]), p["m"], p["malp"], p["kapmax"], p["sig_ratio"], p["alpmax"],
                       int(p.get("literal", 0)))
        _check(self.L.cps_pml_init(self.h, C.byref(pp)))

    def dl_init(self, d):
        z = [0.0] * MAX_POLES
        def arr(v):
            return (C.c_double * MAX_POLES)(*(list(v) + z)[:MAX_POLES])
        pp = DlParams(d["sigma"], d["epsInf"], len(d["fD"]), len(d["fL"]), arr(d["fD"]), arr(d["gD"]),
                      arr(d["fL"]), arr(d["dL"]), arr(d["depsL"]), int(d.get("literal", 0)))
        _check(self.L.cps_dl_init(self.h, C.byref(pp)))

    def drude_init(self, d):
        """The single-pole Drude class (Drude.cpp): dict epsInf fP sigma gamma (Hz)."""
        pp = DrudeParams(d["epsInf"], d["fP"], d["sigma"], d["gamma"])
        _check(self.L.cps_drude_init(self.h, C.byref(pp)))

    def three_init(self, t):
        """The three-level gain class (ThreeLevel.cpp): dict lambda_a lambda_b gamma_a
        gamma_b t20 t21 t10 N_0 [N_1 gain_id literal]."""
        pp = ThreeParams(int(t.get("gain_id", 5)), t["lambda_a"], t["lambda_b"], t["gamma_a"], t["gamma_b"],
                         t["t20"], t["t21"], t["t10"], t["N_0"], t.get("N_1", 0.0), int(t.get("literal", 0)))
        _check(self.L.cps_three_init(self.h, C.byref(pp)))

    def three_populations(self):
        """[ncells][3] N0 N1 N2 of the three-level sites, cells in (i,j,k) order"""
        n = C.c_int64()
        _check(self.L.cps_three_populations(self.h, None, C.byref(n)))
        out = np.empty((n.value, 3))
        _check(self.L.cps_three_populations(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)))
        return out

    def gain_init(self, g):
        pp = GainParams(int(g.get("gain_id", 5)), g["lambda_a"], g["lambda_b"], g["gamma_a"], g["gamma_b"],
                        g["t30"], g["t32"], g["t21"], g["t10"], g["N_0"], g.get("pump", 0.0))
        _check(self.L.cps_gain_init(self.h, C.byref(pp)))

    def tfsf_init(self, t):
        pp = TfsfParams(t["lambda_"], t["dlambda"], t["w0"], t["z0"], t["i0"], t["j0"], t["k0"], t["theta"],
                        t["phi"], t["E0"], t["psi"], (C.c_int32 * 6)(*t["n6"]), t["Nt"], t["cwmode"])
        _check(self.L.cps_tfsf_init(self.h, C.byref(pp)))
        self.tfsf_Nt = t["Nt"]

    def tfsf_tables(self):
        n = self.tfsf_Nt + 1
        e, h = np.empty(n), np.empty(n)
        _check(self.L.cps_tfsf_get_tables(self.h, n, e.ctypes.data_as(C.POINTER(C.c_double)),
                                          h.ctypes.data_as(C.POINTER(C.c_double))))
        return e, h

    def source_add(self, comp, i, j, k, wave):
        w = _dp(wave)
        _check(self.L.cps_source_add(self.h, comp, i, j, k, w[1], len(w[0])))

    def port_add(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.int32).reshape(-1, 3)
        pid = C.c_int32()
        _check(self.L.cps_port_add(self.h, len(pts), pts.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(pid)))
        self.ports.append([len(pts), 0, 0])
        return pid.value

    def port_set_dft(self, pid, freqs, mask=0x3F):
        f = _dp(freqs)
        _check(self.L.cps_port_set_dft(self.h, pid, len(f[0]), f[1], mask))
        self.ports[pid][1] = bin(mask & 63).count("1")
        self.ports[pid][2] = len(f[0])

    # ---------------------------------------------------------- run
    def set_step(self, n):
        _check(self.L.cps_grid_set_step(self.h, n))

    def get_step(self):
        n = C.c_int64()
        _check(self.L.cps_grid_get_step(self.h, C.byref(n)))
        return n.value

    def step(self, n=1, path=FUSED):
        _check(self.L.cps_step(self.h, n, path))

    def sync(self):
        _check(self.L.cps_synchronize(self.h))

    def set_chunked(self, on):
        """fused steps of large grids as graph-replayed one-grid batch chunks (default on)"""
        _check(self.L.cps_grid_set_chunked(self.h, 1 if on else 0))

    def reset(self, n0=1):
        _check(self.L.cps_grid_reset(self.h, n0))

    def set_wait_skew(self, extra_bytes):
        """Test setting of the bounded device waits (cps_grid_set_wait_skew)."""
        _check(self.L.cps_grid_set_wait_skew(self.h, extra_bytes))

    def op(self, name, *args):
        _check(getattr(self.L, "cps_op_" + name)(self.h, *args))

    def set_record(self, on):
        """Queue op() calls; a whole step in the reference's order runs fused."""
        _check(self.L.cps_grid_set_record(self.h, 1 if on else 0))

    def record_stats(self):
        """(steps run fused, calls replayed one by one, calls queued now)"""
        f, r, q = C.c_int64(), C.c_int64(), C.c_int32()
        _check(self.L.cps_grid_record_stats(self.h, C.byref(f), C.byref(r), C.byref(q)))
        return f.value, r.value, q.value

    # ------------------------------------------------------- access
    def field(self, comp):
        out = np.empty(self.shape3, dtype=np.float64)
        _check(self.L.cps_field_download(self.h, comp, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def slice(self, what, axis, index):
        """One plane of component `what` (0..5) or of |E|^2 (6), cut on the device:
        [u][v] with (u, v) = (j, k), (i, k) or (i, j) for axis 0, 1, 2."""
        nu = (self.shape3[1] if axis == 0 else self.shape3[0])
        nv = (self.shape3[1] if axis == 2 else self.shape3[2])
        out = np.empty((nu, nv))
        _check(self.L.cps_field_slice(self.h, what, axis, index, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def energy(self):
        """(electric, magnetic) energy in joules, summed on the device"""
        e, h = C.c_double(), C.c_double()
        _check(self.L.cps_grid_energy(self.h, C.byref(e), C.byref(h)))
        return e.value, h.value

    def fields(self):
        return [self.field(c) for c in range(6)]

    def set_field(self, comp, a):
        a, p = _dp(a)
        assert a.shape == self.shape3
        _check(self.L.cps_field_upload(self.h, comp, p))

    def port_last(self, pid):
        out = np.empty((self.ports[pid][0], 6))
        _check(self.L.cps_port_read(self.h, pid, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def port_dft(self, pid, raw=False, out=None):
        """DFT accumulators; raw=True gives the ABI layout [ncomp][nfreq][2][npts],
        otherwise a [npts][ncomp][nfreq][2] view of it.  out: a C-contiguous
        float64 array of that many values to read into (pinned host memory
        makes the copy a direct DMA)."""
        npts, ncomp, nfreq = self.ports[pid]
        shape = (ncomp, nfreq, 2, npts)
        if out is None:
            out = np.empty(shape)
        else:
            assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == np.prod(shape)
            out = out.reshape(shape)
        _check(self.L.cps_port_dft_read(self.h, pid, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out if raw else out.transpose(3, 0, 1, 2)

    def port_flux(self, pid, normal):
        out = np.empty(self.ports[pid][2])
        _check(self.L.cps_port_flux(self.h, pid, normal.encode(), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def nonfinite(self):
        n = C.c_int64()
        _check(self.L.cps_grid_check_finite(self.h, C.byref(n)))
        return n.value

    def populations(self):
        n = C.c_int64()
        _check(self.L.cps_gain_populations(self.h, None, C.byref(n)))
        out = np.empty((n.value, 4))
        _check(self.L.cps_gain_populations(self.h, out.ctypes.data_as(C.POINTER(C.c_double)), C.byref(n)))
        return out

    def device_bytes(self):
        n = C.c_int64()
        _check(self.L.cps_grid_bytes(self.h, C.byref(n)))
        return n.value

    def launches(self):
        n = C.c_int64()
        _check(self.L.cps_grid_launch_count(self.h, C.byref(n)))
        return n.value

    def flush_ports(self):
        _check(self.L.cps_ports_flush(self.h))

    def set_timing(self, stride):
        _check(self.L.cps_grid_set_timing(self.h, stride))

    def timing(self):
        h, e, n = C.c_double(), C.c_double(), C.c_int64()
        _check(self.L.cps_grid_timing(self.h, C.byref(h), C.byref(e), C.byref(n)))
        return h.value, e.value, n.value

    def set_tile(self, rows, planes):
        _check(self.L.cps_grid_set_tile(self.h, rows, planes))

    def set_sweep(self, mode):
        """0: TMA-fed sweeps (default), 1: register sweeps."""
        _check(self.L.cps_grid_set_sweep(self.h, mode))

    def get_tile(self):
        r, p = C.c_int32(), C.c_int32()
        _check(self.L.cps_grid_get_tile(self.h, C.byref(r), C.byref(p)))
        return r.value, p.value

    def stream(self):
        p = C.c_void_p()
        _check(self.L.cps_grid_get_stream(self.h, C.byref(p)))
        return p.value


class Batch:
    """Many grids of one precision advanced together by the batched engine
    (``cps_batch_*``): sweeps either as one launch per sweep class over all
    members' tiles or as each member's own launches spread over side streams
    (the default), the rest of a step batched over members, step chunks
    replayed as CUDA graphs.  Members stay ordinary :class:`Grid` objects for
    set-up and read-out."""

    def __init__(self, precision=FP32):
        self.L = lib()
        self.h = C.c_void_p()
        _check(self.L.cps_batch_create(precision, C.byref(self.h)))
        self.members = []

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.cps_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, g: Grid):
        _check(self.L.cps_batch_add(self.h, g.h))
        self.members.append(g)

    def remove(self, g: Grid):
        _check(self.L.cps_batch_remove(self.h, g.h))
        self.members.remove(g)

    def info(self):
        n, c = C.c_int32(), C.c_int64()
        _check(self.L.cps_batch_info(self.h, C.byref(n), C.byref(c)))
        return n.value, c.value

    def step(self, n=1):
        _check(self.L.cps_batch_step(self.h, n))

    def sync(self):
        _check(self.L.cps_batch_synchronize(self.h))

    def set_tile(self, rows, planes, persistent=0):
        """Tile rows (4 or 8), planes per tile and sweep launch mode: 0 one
        launch per sweep class, one block per tile; 1 the same, persistent;
        2 each member's own launches on side streams (the default, with
        4 rows and 16 planes).  Results do not depend on the choice."""
        _check(self.L.cps_batch_set_tile(self.h, rows, planes, persistent))

    def get_tile(self):
        r, p, q = C.c_int32(), C.c_int32(), C.c_int32()
        _check(self.L.cps_batch_get_tile(self.h, C.byref(r), C.byref(p), C.byref(q)))
        return r.value, p.value, q.value

    def set_graph(self, on):
        _check(self.L.cps_batch_set_graph(self.h, 1 if on else 0))

    def stream(self):
        s = C.c_void_p()
        _check(self.L.cps_batch_get_stream(self.h, C.byref(s)))
        return s.value

    def launches(self):
        n = C.c_int64()
        _check(self.L.cps_batch_launch_count(self.h, C.byref(n)))
        return n.value

    def tune_key(self):
        buf = C.create_string_buffer(256)
        _check(self.L.cps_batch_tune_key(self.h, buf, 256))
        return buf.value.decode()

    def autotune(self, cache_path="", trial_steps=4):
        """Pick the tiling (cached per key in ``cache_path``); returns the
        number of steps every member advanced while trying candidates."""
        ran = C.c_int32()
        _check(self.L.cps_batch_autotune(self.h, cache_path.encode(), trial_steps, C.byref(ran)))
        return ran.value


class ServerConfig(C.Structure):
    _fields_ = [("precision", C.c_int32), ("max_jobs", C.c_int32), ("budget_bytes", C.c_int64),
                ("chunk_steps", C.c_int32), ("tile_rows", C.c_int32), ("tile_planes", C.c_int32),
                ("tile_persistent", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("jobs_done", "jobs_failed", "jobs_rejected", "jobs_cancelled",
                                          "jobs_live", "jobs_queued", "bytes_in_use", "chunks")] + \
               [(n, C.c_double) for n in ("latency_p50_ms", "latency_p99_ms", "wait_p50_ms", "wait_p99_ms",
                                           "run_p50_ms", "cell_updates", "span_s", "gpu_busy_s")]


_BUILD_FN = C.CFUNCTYPE(C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_void_p))
_DONE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64, C.c_void_p, C.c_int32)

# status codes of cps_capi.h
CPS_OK, CPS_E_INVALID, CPS_E_CUDA, CPS_E_NOMEM, CPS_E_STATE = 0, 1, 2, 3, 4
CPS_E_NUMERIC, CPS_E_BUDGET, CPS_E_TIMEOUT, CPS_E_CANCELLED, CPS_E_NOTFOUND = 5, 6, 7, 8, 9


def footprint(dk, precision=FP32) -> int:
    """Admission estimate of a deck's device memory in bytes: fields, IDs,
    CPML slabs, Drude-Lorentz and gain state at their cell counts, port rings
    and DFT accumulators, plus 5% for tables."""
    esz = 4 if precision == FP32 else 8
    nx, ny, nz = dk.nx, dk.ny, dk.nz
    px = (nx + 1 + 31) // 32 * 32
    cells = px * (ny + 1) * (nz + 1)
    total = 6 * cells * esz + cells
    if dk.pml:
        n = dk.pml["npml"]
        xw = sum((v + 32) // 32 * 32 for v in n[0:2] if v) * (ny + 1) * (nz + 1)
        yw = sum(v + 1 for v in n[2:4] if v) * px * (nz + 1)
        zw = sum(v + 1 for v in n[4:6] if v) * px * (ny + 1)
        total += 2 * 2 * esz * (xw + yw + zw)  # two psi per slab cell for E and for H
    ids = dk.ids
    if dk.dl:
        ndl = int((ids == ID_DISPERSIVE).sum()) if ids is not None else cells // 10
        total += ndl * (3 * (len(dk.dl.get("fD", [])) + 2 * len(dk.dl.get("fL", [])) + 1) * esz + 8)
    if dk.gain:
        gid = dk.gain.get("gain_id", 5)
        ng = int((ids == gid).sum()) if ids is not None else cells
        if precision == FP32:  # segment-dense persistent words for every cell + list-layout transients
            total += cells * 15 * 4 + ng * (9 * 4 + 8)
        else:
            total += ng * (25 * esz + 8)
    for p in dk.ports:
        npts = len(port_points(dk, p))
        nf = 0 if p.dft_freqs is None else len(p.dft_freqs)
        nc = bin(p.dft_mask & 63).count("1") if nf else 0
        total += npts * (8 + 6 * esz * (64 if nf else 1) + nc * nf * 16)
    return int(total * 1.05)


class Server:
    """Serving loop of the library (``cps_server_*``): jobs queued with a
    footprint and step count, admitted against a device-memory budget and run
    together by the batched engine; a job's ``build()`` makes its Grid when it
    is admitted and ``done(grid, status)`` reads its results when it ends (the
    server destroys the grid afterwards)."""

    def __init__(self, precision=FP32, max_jobs=64, budget_bytes=180 * 10 ** 9, chunk_steps=64, tile=None):
        self.L = lib()
        self.h = C.c_void_p()
        rows, planes, pers = tile if tile else (0, 0, 0)
        cfg = ServerConfig(precision, max_jobs, int(budget_bytes), chunk_steps, rows, planes, pers)
        _check(self.L.cps_server_create(C.byref(cfg), C.byref(self.h)))
        self._jobs = {}
        self._grids = {}
        self.errors = {}
        self._build_cb = _BUILD_FN(self._on_build)
        self._done_cb = _DONE_FN(self._on_done)

    def _on_build(self, user, jid, out):
        try:
            g = self._jobs[jid][0]()
        except CpsError as ex:
            self.errors[jid] = str(ex)
            return ex.code
        except Exception as ex:  # a malformed job fails alone
            self.errors[jid] = repr(ex)
            return CPS_E_INVALID
        self._grids[jid] = g
        out[0] = g.h.value
        return 0

    def _on_done(self, user, jid, gptr, status):
        g = self._grids.pop(jid, None)
        job = self._jobs.pop(jid, None)
        try:
            if job is not None and job[1] is not None:
                job[1](g, status)
        except Exception as ex:
            self.errors[jid] = repr(ex)
        finally:
            if g is not None:
                g.h = C.c_void_p()  # the server destroys the grid when this returns

    def submit(self, build, done, nsteps, footprint_bytes):
        jid = C.c_int64()
        _check(self.L.cps_server_submit(self.h, int(footprint_bytes), int(nsteps), self._build_cb, self._done_cb,
                                        None, C.byref(jid)))
        self._jobs[jid.value] = (build, done)
        return jid.value

    def poll(self):
        live, queued = C.c_int32(), C.c_int32()
        _check(self.L.cps_server_poll(self.h, C.byref(live), C.byref(queued)))
        return live.value, queued.value

    def drain(self):
        _check(self.L.cps_server_drain(self.h))

    def cancel(self, jid):
        _check(self.L.cps_server_cancel(self.h, jid))

    def stats(self):
        s = ServerStats()
        _check(self.L.cps_server_get_stats(self.h, C.byref(s)))
        return {n: getattr(s, n) for n, _ in ServerStats._fields_}

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.cps_server_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
