"""Device FP64 reductions (mass, momentum, momentum-exchange force, kinetic energy, non-finite
count) and time-averaged velocity, against the oracle's restatement (oracle/lbm_oracle.c
orc_moments; the reference computes no forces, so its definition is stated there).

Tolerance: relative 1e-12 for FP64 states (the device sums in a fixed tree order, the oracle
left to right; the states themselves are bit-identical), exact for the non-finite count;
1e-3 relative (mass, force) for the FP32 state against the FP64 one.
"""
import numpy as np
import pytest

import lbgpu
import oracle as O

pytestmark = pytest.mark.gpu


def lattice(st, precision="f64", scheme="pull"):
    lat = lbgpu.Lattice(st.lx, st.ly, precision, scheme)
    lat.set_geometry(st.omega, st.tag, st.bc, st.zgb)
    lat.set_populations(st.lat, st.tmp)
    return lat


def close(a, b, rtol, atol=0.0):
    return abs(a - b) <= atol + rtol * max(abs(a), abs(b))


@pytest.mark.parametrize("scheme", ["pull", "aa"])
@pytest.mark.parametrize("steps", [0, 1, 37, 400])
def test_moments_match_oracle(scheme, steps):
    for cyl in (O.Cylinder.baseline(250, 51), O.Cylinder.reference_driver(200, 60)):
        st = O.build_cylinder(cyl)
        exp = O.moments(O.run(st, steps))
        with lattice(st, "f64", scheme) as lat:
            lat.step(steps)
            got = lat.moments()
            again = lat.moments()
        assert np.array_equal(got, again)           # fixed-order device sums
        assert got[6] == exp[6] == 0
        scale = abs(exp[0])
        for k in (0, 1, 2, 5, 7):
            assert close(got[k], exp[k], 1e-12, 1e-13 * scale), (k, got[k], exp[k])
        for k in (3, 4):                             # force: a sum of +- terms
            assert close(got[k], exp[k], 1e-10, 1e-12), (k, got[k], exp[k])


def test_mean_drag_is_positive_and_lift_vanishes_in_the_symmetric_channel():
    # The impulsive start sends acoustic waves through the short channel (omega = 1.97), so the
    # instantaneous drag changes sign; its time average over 2000 steps does not.  The
    # bounce-back channel with the obstacle on the centre line is mirror-symmetric: lift stays
    # at rounding level.
    cyl = O.Cylinder.baseline(250, 51)
    fx, fy = [], []
    with lattice(O.build_cylinder(cyl)) as lat:
        for _ in range(100):
            lat.step(20)
            m = lat.moments()
            fx.append(m[3])
            fy.append(m[4])
    assert np.mean(fx) > 0
    assert np.max(np.abs(fy)) < 1e-10


def test_non_finite_nodes_are_counted():
    st = O.build_cylinder(O.Cylinder.reference_driver(256, 256))
    st.tmp[:] = np.nan
    exp = O.run(st, 10)
    with lattice(st) as lat:
        lat.step(10)
        m = lat.moments()
    assert m[6] == O.moments(exp)[6] > 0


def test_fp32_moments_close_to_fp64():
    st = O.build_cylinder(O.Cylinder.baseline(250, 51))
    with lattice(st, "f64") as a, lattice(st, "f32") as b:
        a.step(300)
        b.step(300)
        ma, mb = a.moments(), b.moments()
    for k in (0, 3, 7):
        assert close(ma[k], mb[k], 1e-3), (k, ma[k], mb[k])


def test_time_averaged_velocity_matches_oracle_average():
    st = O.build_cylinder(O.Cylinder.baseline(120, 41))
    s = st
    us, vs = [], []
    for _ in range(5):
        s = O.run(s, 10)
        f = s.lat[1:-1, 1:-1]
        rho = f.sum(axis=2)
        us.append(((f[..., 1] + f[..., 5] + f[..., 8] - f[..., 3] - f[..., 6] - f[..., 7]) / rho).T)
        vs.append(((f[..., 2] + f[..., 5] + f[..., 6] - f[..., 4] - f[..., 7] - f[..., 8]) / rho).T)
    with lattice(st) as lat:
        for _ in range(5):
            lat.step(10)
            lat.velocity_accumulate()
        ux, uy, k = lat.velocity_average()
        lat.velocity_reset()
        lat.step(1)
        lat.velocity_accumulate()
        _, _, k1 = lat.velocity_average()
    assert k == 5 and k1 == 1
    assert np.allclose(ux, np.mean(us, axis=0), rtol=1e-12, atol=1e-15)
    assert np.allclose(uy, np.mean(vs, axis=0), rtol=1e-12, atol=1e-15)
