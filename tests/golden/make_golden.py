"""Generate tests/golden/golden.json from the reference implementation itself.

Run in a container that has the reference checkout (it needs ``oracle/_ref``, which
``make -C oracle`` builds from the reference's own lb.c / boundaries.c / unsteady.c):

    python tests/golden/make_golden.py

Every case runs the UNMODIFIED reference code (oracle/_ref/libref_lb_serial.so through the
harness oracle/ref_harness.c, and for the application-driver cases also the unmodified
unsteady.c binaries) and stores, per case, the SHA-256 of the final populations (float64,
[X][Y][9] with the ghost ring), per-direction interior sums and a fixed sample of nodes as
hex floats.  The reference has no test suite or fixtures of its own, so these digests are
what pins the oracle (tests/test_oracle_pins.py) and, through the oracle, the GPU kernels.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def summarize(lat: np.ndarray) -> dict:
    lx, ly = lat.shape[0] - 2, lat.shape[1] - 2
    inner = lat[1:lx + 1, 1:ly + 1]
    flat = inner.reshape(-1, 9)
    idx = np.unique(np.linspace(0, flat.shape[0] - 1, num=min(48, flat.shape[0])).astype(int))
    return {
        "sha256": digest(lat),
        "sha256_interior": digest(inner),
        "nan_nodes": int(np.isnan(inner).any(axis=2).sum()),
        "sums": [float(v).hex() for v in np.nansum(inner, axis=(0, 1))],
        "sample_index": [int(i) for i in idx],
        "sample": [[float(v).hex() for v in flat[i]] for i in idx],
    }


def cyl_dict(c: O.Cylinder) -> dict:
    return {"lx": c.lx, "ly": c.ly, "obst_x": c.obst_x, "obst_y": c.obst_y,
            "obst_r": c.obst_r, "umax": c.umax, "re": c.re, "wall": c.wall,
            "outlet": c.outlet}


def unsteady_dump(variant: str, lx: int, ly: int, steps: int, blk: int) -> np.ndarray:
    exe = os.path.join(ROOT, "oracle", "_ref", f"unsteady_{variant}")
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "dump.bin")
        env = dict(os.environ, STOP=str(steps), LBREF_DUMP=path)
        subprocess.run([exe, str(lx), str(ly), str(blk)], env=env, check=True,
                       capture_output=True)
        return np.fromfile(path, dtype="<f8").reshape(lx + 2, ly + 2, 9)


def main():
    cases = {}

    def cylinder_case(name, c, steps, variants, blk=1, poison=False, check_driver=False):
        outs = {v: O.run_reference(c, v, steps, poison=poison, blk=blk) for v in variants}
        base = outs[variants[0]]
        agree = {}
        for v in variants[1:]:
            same = np.array_equal(outs[v], base, equal_nan=True)
            agree[v] = bool(same)
        entry = {"kind": "cylinder", "cylinder": cyl_dict(c), "steps": steps, "blk": blk,
                 "poison_tmp": poison, "variants": variants, "variants_agree": agree}
        entry.update(summarize(base))
        if check_driver:
            dump = unsteady_dump(variants[0], c.lx, c.ly, steps, blk)
            entry["unsteady_driver_matches"] = bool(np.array_equal(dump, base, equal_nan=True))
        cases[name] = entry
        print(name, entry["sha256"][:16], agree, entry.get("unsteady_driver_matches"))

    all5 = ["origin", "combine", "tight", "tight_block", "panel"]
    cylinder_case("ref_driver_250x51_5000", O.Cylinder.reference_driver(250, 51), 5000,
                  ["origin", "combine", "tight"], check_driver=True)
    cylinder_case("baseline_250x51_5000", O.Cylinder.baseline(250, 51), 5000,
                  ["origin", "combine", "tight"])
    for s in (1, 2, 3):
        cylinder_case(f"baseline_250x51_{s}", O.Cylinder.baseline(250, 51), s, ["origin"])
        cylinder_case(f"ref_driver_250x51_{s}", O.Cylinder.reference_driver(250, 51), s,
                      ["origin"])
    cylinder_case("ref_driver_256x256_100_blk32", O.Cylinder.reference_driver(256, 256), 100,
                  all5, blk=32, check_driver=True)
    cylinder_case("baseline_256x256_100_blk32", O.Cylinder.baseline(256, 256), 100, all5, blk=32)
    cylinder_case("poison_256x256_100", O.Cylinder.reference_driver(256, 256), 100,
                  ["origin", "combine", "tight"], poison=True)
    cylinder_case("poison_256x256_10", O.Cylinder.reference_driver(256, 256), 10,
                  ["origin"], poison=True)
    for (lx, ly) in [(3, 3), (4, 2), (5, 3), (7, 4), (33, 17), (37, 29), (64, 48)]:
        cylinder_case(f"ref_driver_{lx}x{ly}_200", O.Cylinder.reference_driver(lx, ly), 200,
                      ["origin", "combine", "tight"])
        cylinder_case(f"baseline_{lx}x{ly}_200", O.Cylinder.baseline(lx, ly), 200,
                      ["origin", "combine", "tight"])

    for (lx, ly, seed) in [(12, 10, 1), (9, 7, 2), (16, 16, 3), (5, 4, 4), (40, 24, 5)]:
        st = O.random_boundary_lattice(lx, ly, seed)
        out = O.run_reference_custom(st, "origin", 40)
        entry = {"kind": "bc_kinds", "lx": lx, "ly": ly, "seed": seed, "steps": 40,
                 "omega": st.omega, "tags_present": sorted(int(t) for t in set(st.tag.ravel()))}
        entry.update(summarize(out))
        cases[f"bc_kinds_{lx}x{ly}_s{seed}"] = entry
        print(f"bc_kinds_{lx}x{ly}_s{seed}", entry["sha256"][:16])

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "source": "reference lb.c/boundaries.c/unsteady.c compiled by oracle/Makefile",
                   "cases": cases}, f, indent=1)


if __name__ == "__main__":
    main()
