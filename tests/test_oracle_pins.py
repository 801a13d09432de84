"""The CPU oracle against the reference's own outputs (CPU only).

tests/golden/golden.json holds digests of the UNMODIFIED reference (lb.c, boundaries.c and the
application driver unsteady.c, compiled by oracle/Makefile) made by tests/golden/make_golden.py.
These tests re-run the oracle restatement (oracle/lbm_oracle.c) on the same inputs and require
bit-identical populations; where the reference build (oracle/_ref) is present they also run it
live.
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import check_golden, describe_diff, same, state_of


def _cases(golden, pred):
    return [k for k, v in golden.items() if pred(v)]


def test_golden_file_is_consistent(golden):
    assert len(golden) >= 30
    # the reference's own variant-equivalence property, recorded when the golden was made
    for name, case in golden.items():
        for v, ok in case.get("variants_agree", {}).items():
            assert ok, f"{name}: reference {v} differed from {case['variants'][0]}"
        if "unsteady_driver_matches" in case:
            assert case["unsteady_driver_matches"], name


@pytest.mark.parametrize("steps_case", [
    "baseline_250x51_1", "baseline_250x51_2", "baseline_250x51_3",
    "ref_driver_250x51_1", "ref_driver_250x51_2", "ref_driver_250x51_3",
    "ref_driver_256x256_100_blk32", "baseline_256x256_100_blk32",
    "poison_256x256_10", "poison_256x256_100",
])
def test_oracle_matches_reference_digest(golden, steps_case):
    case = golden[steps_case]
    out = O.run(state_of(case), case["steps"]).lat
    assert check_golden(case, out), steps_case


def test_oracle_matches_reference_long_runs(golden):
    for name in ("ref_driver_250x51_5000", "baseline_250x51_5000"):
        case = golden[name]
        out = O.run(state_of(case), case["steps"]).lat
        assert check_golden(case, out), name


def test_oracle_matches_reference_small_and_ragged(golden):
    names = _cases(golden, lambda c: c["kind"] == "cylinder" and c["steps"] == 200)
    assert len(names) >= 14
    for name in names:
        case = golden[name]
        assert check_golden(case, O.run(state_of(case), case["steps"]).lat), name


def test_oracle_matches_reference_every_boundary_kind(golden):
    names = _cases(golden, lambda c: c["kind"] == "bc_kinds")
    seen = set()
    for name in names:
        case = golden[name]
        seen |= set(case["tags_present"])
        assert check_golden(case, O.run(state_of(case), case["steps"]).lat), name
    assert set(range(1, 19)) <= seen   # bgk, bounce-back and all 16 Zou/He + regularized rules


def test_poison_reaches_only_corners_after_10_steps(golden):
    """The stale ghost-sourced slots are read only by the 4 corner nodes (lb.c:258-267)."""
    case = golden["poison_256x256_10"]
    st = state_of(case)
    out = O.run(st, 10).lat[1:-1, 1:-1]
    bad = np.argwhere(np.isnan(out).any(axis=2))
    assert case["nan_nodes"] == len(bad) > 0
    lx, ly = 256, 256
    for X, Y in bad + 1:
        assert min(X - 1, lx - X) < 10 and min(Y - 1, ly - Y) < 10


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
def test_oracle_matches_live_reference_all_variants():
    c = O.Cylinder.reference_driver(64, 48)
    base = O.run(O.build_cylinder(c), 64).lat
    for v in ("origin", "combine", "tight", "tight_block", "panel"):
        ref = O.run_reference(c, v, 64, blk=16)
        assert same(ref, base), f"{v}: {describe_diff(ref, base)}"


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
def test_oracle_matches_live_reference_custom_lattices():
    for seed, (lx, ly) in enumerate([(6, 5), (11, 9), (20, 14)], start=11):
        st = O.random_boundary_lattice(lx, ly, seed)
        ref = O.run_reference_custom(st, "origin", 25)
        assert same(O.run(st, 25).lat, ref)


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
def test_oracle_planted_mistake_is_caught():
    """A deliberately wrong oracle input (omega off by one ulp) must not match the reference."""
    c = O.Cylinder.baseline(40, 21)
    st = O.build_cylinder(c)
    ref = O.run_reference(c, "origin", 50)
    st.omega = np.nextafter(st.omega, 2.0)
    assert not same(O.run(st, 50).lat, ref)


_PERIODIC_REF = os.path.join(os.path.dirname(O.HERE), "oracle", "_ref", "periodic_ref")


@pytest.mark.skipif(not os.path.exists(_PERIODIC_REF), reason="oracle/_ref/periodic_ref not built")
def test_reference_periodic_driver_conserves_mass(tmp_path):
    """The periodic-box driver's wrap (the reference's makePeriodic, lb.c:1783-1817) closes the
    box: the interior mass after 40 wrapped steps equals the wrapped initial state's."""
    import subprocess
    lx, ly = 77, 45
    mass = []
    for steps in (0, 40):
        d = tmp_path / str(steps)
        d.mkdir()
        subprocess.run([_PERIODIC_REF, str(lx), str(ly), str(steps), "0", str(d)], check=True,
                       timeout=120)
        f = np.fromfile(d / "lattice.bin", "<f8").reshape(lx + 2, ly + 2, 9)
        mass.append(f[1:-1, 1:-1].sum())
        assert (d / "vel.dat").read_text().count("\n") == lx * ly
    assert abs(mass[1] - mass[0]) <= 1e-13 * mass[0], mass

