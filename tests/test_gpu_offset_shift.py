"""FP16/BF16 offsets from a per-row equilibrium (lbgpu_set_offset_shift).

The contract: with a shift profile every scheme still agrees bit for bit (pull, AA, two steps
per sweep, batch members with one or four nodes a thread): the stored values are relative to
the row that consumes them, so streaming between rows and the AA scheme's opposite slots stay
consistent.  A state close to the profile is stored almost exactly (the reason for the shift),
and the dynamics stay within the 16-bit tolerance of the unshifted form against the oracle.
"""
import numpy as np
import pytest

import lbgpu
import oracle as O
from helpers import describe_diff, same

pytestmark = pytest.mark.gpu

SCALE = {"f16": 10, "bf16": 6}


def channel(lx, ly, precision, scheme, shift, umax=0.03, re=60.0):
    lat = lbgpu.Lattice(lx, ly, precision, scheme)
    lat.set_offset_scale(SCALE[precision])
    if shift:
        lat.set_offset_shift(lbgpu.poiseuille_profile(ly, umax))
    lat.setup_cylinder(lx // 5 + 1, ly // 2 + 1, ly // 10 + 1, umax, re, lbgpu.WALL_BOUNCEBACK,
                       lbgpu.OUTLET_CONST)
    return lat


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_every_scheme_agrees_under_a_shift(precision):
    lx, ly, n = 300, 61, 57

    def alone(scheme, sweep=1):
        with channel(lx, ly, precision, scheme, True) as lat:
            if sweep == 2:
                lat.set_sweep_steps(2)
            lat.step(n)
            return lat.populations()

    ref = alone("pull")
    aa, two = alone("aa"), alone("pull", 2)
    assert same(aa, ref), describe_diff(aa, ref)
    assert same(two, ref), describe_diff(two, ref)
    for shape in [(32, 1), (128, 4)]:
        with channel(lx, ly, precision, "pull", True) as a, channel(lx, ly, precision, "aa", True) as b, \
                lbgpu.Batch(precision) as batch:
            for c in range(6):
                batch.set_shape(c, *shape)
            sa, sb = batch.add(a), batch.add(b)
            batch.step(n)
            batch.synchronize()
            got_a, got_b = a.populations(), b.populations()
            batch.remove(sa)
            batch.remove(sb)
        assert same(got_a, ref), (shape, describe_diff(got_a, ref))
        assert same(got_b, ref), shape


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_shift_on_every_boundary_rule(precision):
    st = O.random_boundary_lattice(41, 33, seed=11)
    rng = np.random.default_rng(5)
    u = rng.uniform(-0.03, 0.03, st.ly + 2)

    def run(scheme, sweep=1):
        with lbgpu.Lattice(st.lx, st.ly, precision, scheme) as lat:
            lat.set_offset_scale(SCALE[precision])
            lat.set_offset_shift(u)
            lat.set_geometry(st.omega, st.tag, st.bc, st.zgb)
            lat.set_populations(st.lat, st.tmp)
            if sweep == 2:
                lat.set_sweep_steps(2)
            lat.step(9)
            return lat.populations()

    ref = run("pull")
    assert same(run("aa"), ref)
    assert same(run("pull", 2), ref)
    exp = O.run(st, 9).lat
    f = ref[1:-1, 1:-1]
    e = exp[1:-1, 1:-1]
    assert np.abs(f - e).max() < (3e-3 if precision == "f16" else 2e-2)


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_states_near_the_profile_are_stored_almost_exactly(precision):
    st = O.build_cylinder(O.Cylinder.baseline(250, 51))
    init = st.lat[1:-1, 1:-1]
    err = {}
    for shift in (False, True):
        with lbgpu.Lattice(250, 51, precision, "pull") as lat:
            lat.set_offset_scale(SCALE[precision])
            if shift:
                lat.set_offset_shift(lbgpu.poiseuille_profile(51, 0.02))
            lat.setup_cylinder(51, 26, 6, 0.02, 100.0, lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
            err[shift] = np.abs(lat.populations()[1:-1, 1:-1] - init).max()
    assert err[True] < 1e-7 < err[False]


def test_shifted_fp16_against_the_oracle():
    """250x51 channel, 5000 steps: the shifted form within the unshifted form's tolerance."""
    st = O.build_cylinder(O.Cylinder.baseline(250, 51))
    exp = O.run(st, 5000).lat[1:-1, 1:-1]
    with channel(250, 51, "f16", "pull", True, umax=0.02, re=100.0) as lat:
        lat.step(5000)
        got = lat.populations()[1:-1, 1:-1]
    fluid = st.tag[1:-1, 1:-1] == 1

    def vel(f):
        rho = f.sum(axis=2)
        ux = (f[..., 1] + f[..., 5] + f[..., 8] - f[..., 3] - f[..., 6] - f[..., 7]) / rho
        uy = (f[..., 2] + f[..., 5] + f[..., 6] - f[..., 4] - f[..., 7] - f[..., 8]) / rho
        return ux[fluid], uy[fluid]

    gx, gy = vel(got)
    ex, ey = vel(exp)
    rel = np.sqrt(((gx - ex) ** 2 + (gy - ey) ** 2).sum() / (ex ** 2 + ey ** 2).sum())
    assert rel <= 3e-2, rel


def test_shift_arguments():
    with lbgpu.Lattice(40, 20, "f32", "pull") as lat:
        with pytest.raises(lbgpu.LbError) as e:
            lat.set_offset_shift(np.zeros(22))
        assert e.value.code == 7
    with lbgpu.Lattice(40, 20, "f16", "pull") as lat:
        with pytest.raises(ValueError):
            lat.set_offset_shift(np.zeros(21))
        bad = np.zeros(22)
        bad[3] = np.nan
        with pytest.raises(lbgpu.LbError) as e:
            lat.set_offset_shift(bad)
        assert e.value.code == 3
        lat.set_offset_shift(None)
    lbgpu.clear_error()
