"""Regenerate tests/golden/golden.json from the reference's own code.

Needs the reference tree (built by `make -C oracle ref` into oracle/_ref).
Each case runs a deck through oracle/_ref/ref_harness (3-D) or
oracle/_ref/ref2d_harness (2-D Drude-Lorentz / gain classes) and stores the
SHA-256 of every output array plus its L2 norm, so the tests can check the
oracle restatement bit for bit without the reference being present.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

sys.path.insert(0, HERE)
import golden_cases  # noqa: E402
import oracle  # noqa: E402


def digest(a):
    a = np.ascontiguousarray(a)
    return {"sha256": hashlib.sha256(a.tobytes()).hexdigest(), "shape": list(a.shape), "dtype": str(a.dtype),
            "l2": float(np.linalg.norm(a.astype(np.float64)))}


def main():
    out = {"cases3d": {}, "cases2d": {}}
    for name, build in golden_cases.CASES_3D.items():
        dk = build()
        r = oracle.run_ref_harness(dk, record_ports=True)
        rec = {"ids": digest(r["ids"])}
        for c in ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz"):
            rec[c] = digest(r[c])
        rec["stretch"] = [digest(s) for s in r["stretch"]]
        if "tfsf" in r:
            rec["einc"] = digest(r["tfsf"][0])
            rec["hinc"] = digest(r["tfsf"][1])
        rec["ports"] = [{"points": digest(p["points"]), "last": digest(p["last"]), "series": digest(p["series"])}
                        for p in r["ports"]]
        out["cases3d"][name] = rec
        print(name, "done")
    for name, build in golden_cases.CASES_2D.items():
        args = build()
        Ex, Ey, Hz = oracle.run_ref2d(*args[:4], **args[4])
        out["cases2d"][name] = {"Ex": digest(Ex), "Ey": digest(Ey), "Hz": digest(Hz)}
        print(name, "done")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
