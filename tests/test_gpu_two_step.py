"""Two pull steps per sweep (lbgpu_set_sweep_steps(lat, 2), the temporal-blocking kernel).

The contract: the state after any number of steps is bit-identical to single steps, in every
precision, including the ghost ring and the stale slots that only the corners consume, on
lattices smaller than one tile and spanning many, with every boundary rule of boundaries.h, a
seeded second buffer (whose ghost ring differs from the first's), read-outs between calls and
odd step counts.  FP64 results also match the reference's own digests.
"""
import numpy as np
import pytest

import lbgpu
import oracle as O
from helpers import check_golden, describe_diff, same, state_of

pytestmark = pytest.mark.gpu

SCALE = {"f16": 10, "bf16": 6}


def run(st, plan, precision, sweep, scale=None, reads=False):
    with lbgpu.Lattice(st.lx, st.ly, precision, "pull") as lat:
        if scale is not None:
            lat.set_offset_scale(scale)
        lat.set_geometry(st.omega, st.tag, st.bc, st.zgb)
        lat.set_populations(st.lat, st.tmp)
        lat.set_sweep_steps(sweep)
        seen = []
        for n in plan:
            lat.step(n)
            if reads:
                seen.append((lat.macros(), lat.moments()))
        assert lat.steps_done == sum(plan)
        return lat.populations(), seen


@pytest.mark.parametrize("precision", ["f64", "f32", "f16", "bf16"])
@pytest.mark.parametrize("size", [(23, 11), (37, 29), (70, 40), (130, 33)])
def test_two_step_sweeps_equal_single_steps(precision, size):
    st = O.random_boundary_lattice(size[0], size[1], seed=size[0] * 7 + size[1])
    plan = [1, 2, 3, 4, 7]
    one, _ = run(st, plan, precision, 1, SCALE.get(precision))
    two, _ = run(st, plan, precision, 2, SCALE.get(precision))
    assert same(two, one), (precision, size, describe_diff(two, one))


@pytest.mark.parametrize("precision", ["f64", "f16"])
def test_read_outs_between_two_step_sweeps(precision):
    st = O.build_cylinder(O.Cylinder.baseline(150, 41))
    one, r1 = run(st, [2, 5, 10], precision, 1, SCALE.get(precision), reads=True)
    two, r2 = run(st, [2, 5, 10], precision, 2, SCALE.get(precision), reads=True)
    assert same(two, one)
    for (m1, s1), (m2, s2) in zip(r1, r2):
        for a, b in zip(m1, m2):
            assert same(a, b)
        assert same(s1, s2)


@pytest.mark.parametrize("name", ["baseline_250x51_5000", "baseline_250x51_3", "ref_driver_256x256_100_blk32"])
def test_two_step_fp64_matches_reference_digests(golden, name):
    case = golden[name]
    got, _ = run(state_of(case), [case["steps"]], "f64", 2)
    assert check_golden(case, got), name


def test_two_step_fp64_matches_oracle_on_every_boundary_rule():
    st = O.random_boundary_lattice(45, 38, seed=3)
    got, _ = run(st, [9], "f64", 2)
    exp = O.run(st, 9).lat
    assert same(got, exp), describe_diff(got, exp)


def test_extrapolated_outlet_runs_single_steps():
    st = O.build_cylinder(O.Cylinder.reference_driver(120, 31))    # zero-gradient outlet
    got, _ = run(st, [6], "f64", 2)
    exp = O.run(st, 6).lat
    assert same(got, exp), describe_diff(got, exp)


def test_channel_set_up_on_the_device():
    def go(sweep):
        with lbgpu.Lattice(333, 77, "f32", "pull") as lat:
            lat.setup_cylinder(67, 39, 8, 0.03, 80.0, lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
            lat.set_sweep_steps(sweep)
            lat.step(101)
            return lat.populations()
    assert same(go(2), go(1))


def test_sweep_steps_arguments():
    with lbgpu.Lattice(40, 20, "f64", "aa") as lat:
        with pytest.raises(lbgpu.LbError) as e:
            lat.set_sweep_steps(2)
        assert e.value.code == 7
    with lbgpu.Lattice(40, 20, "f64", "pull") as lat:
        with pytest.raises(lbgpu.LbError) as e:
            lat.set_sweep_steps(3)
        assert e.value.code == 3
    lbgpu.clear_error()
