"""Stochastic rounding of FP16/BF16 stores (lbgpu_set_stochastic_rounding).

The contract: a stored value rounds up with probability equal to its discarded fraction (checked
on a uniform lattice whose every node stores the same exact value, so the share of nodes that
rounded up is the probability); the random bits depend only on (seed, collision, node,
direction), so the pull scheme, the AA scheme and two steps per sweep stay bit-identical, a seed
reproduces its run and another seed does not; and the dynamics stay within the 16-bit tolerance
against the oracle.
"""
import numpy as np
import pytest

import lbgpu
import oracle as O
from helpers import describe_diff, same

pytestmark = pytest.mark.gpu

SCALE = {"f16": 10, "bf16": 6}
W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W32 = W.astype(np.float32).astype(np.float64)   # the weights the device decodes against


def _neighbours(x, precision):
    """The two representable values lo <= x <= hi of the storage type around x > 0."""
    if precision == "f16":
        h = float(np.float16(x))
        if h > x:
            return float(np.nextafter(np.float16(h), np.float16(-1))), h
        return h, float(np.nextafter(np.float16(h), np.float16(1e4)))
    bits = int(np.array([x], np.float32).view(np.uint32)[0]) & 0xFFFF0000
    lo = float(np.array([bits], np.uint32).view(np.float32)[0])
    if lo > x:
        bits -= 0x10000
        lo = float(np.array([bits], np.uint32).view(np.float32)[0])
    hi = float(np.array([bits + 0x10000], np.uint32).view(np.float32)[0])
    return lo, hi


def _snap(x, precision):
    """Nearest value of the storage type (undoes the float rounding of a decoded read-out)."""
    if precision == "f16":
        return np.float16(x).astype(np.float64)
    b = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    b = ((b + 0x8000) & 0xFFFF0000).astype(np.uint32)
    return b.view(np.float32).astype(np.float64)


def _uniform_bgk(lx, ly, precision, delta, rs, seed=1):
    """All-BGK lattice, f_i = w_i everywhere but f_0 = w_0 + delta (no momentum), omega = 1: one
    collision stores the equilibrium E_i = w_i sum(D) 2^s at every node, the same value
    everywhere and in general between two representable ones.  Returns (decoded populations
    after one step, stored offsets of the initial state)."""
    tag = np.zeros((lx + 2, ly + 2), np.uint8)
    tag[1:-1, 1:-1] = 1
    nb = max(lx, ly) + 2
    f0 = W.copy()
    f0[0] += delta
    f = np.broadcast_to(f0, (lx + 2, ly + 2, 9)).copy()
    with lbgpu.Lattice(lx, ly, precision, "pull") as lat:
        lat.set_offset_scale(SCALE[precision])
        if rs:
            lat.set_stochastic_rounding(True, seed)
        lat.set_geometry(1.0, tag, np.zeros(16 * nb), np.zeros(ly + 2, np.uint8))
        lat.set_populations(f, f)
        d0 = _snap((lat.populations()[5, 5] - W32) * 2.0 ** SCALE[precision], precision)
        lat.step(1)
        return lat.populations(), d0


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("delta", [3.7e-4, 5.1e-4, 1.3e-4])
def test_stochastic_rounding_is_unbiased(precision, delta):
    lx = ly = 256
    s = SCALE[precision]
    got, d0 = _uniform_bgk(lx, ly, precision, delta, True)
    nearest, _ = _uniform_bgk(lx, ly, precision, delta, False)
    sum_d = float(np.sum(d0))
    tested = 0
    for group in ([0], [1, 2, 3, 4], [5, 6, 7, 8]):
        e = W32[group[0]] * sum_d                    # the stored value every node computes
        lo, hi = _neighbours(e, precision)
        p = (e - lo) / (hi - lo)
        d = (got[2:-2, 2:-2][..., group] - W32[group]) * 2.0 ** s
        up = np.abs(d - hi) < np.abs(d - lo)
        assert np.all(np.minimum(np.abs(d - hi), np.abs(d - lo)) < 0.25 * (hi - lo))
        n = up.size
        sigma = np.sqrt(max(p * (1 - p), 1e-4) / n)
        assert abs(up.mean() - p) < 5 * sigma, (precision, group, up.mean(), p)
        dn = (nearest[2:-2, 2:-2][..., group] - W32[group]) * 2.0 ** s
        rn = hi if abs(e - hi) < abs(e - lo) else lo
        assert np.all(np.abs(dn - rn) < 0.25 * (hi - lo))   # round to nearest: all the same
        tested += 0.05 < p < 0.95
    assert tested >= 2


def _channel(lx, ly, precision, scheme, shift, seed=7, rs=True, umax=0.03, re=60.0):
    lat = lbgpu.Lattice(lx, ly, precision, scheme)
    lat.set_offset_scale(lbgpu.DEFAULT_SHIFT_SCALE[precision] if shift else SCALE[precision])
    if shift:
        lat.set_offset_shift(lbgpu.poiseuille_profile(ly, umax))
    if rs:
        lat.set_stochastic_rounding(True, seed)
    lat.setup_cylinder(lx // 5 + 1, ly // 2 + 1, ly // 10 + 1, umax, re, lbgpu.WALL_BOUNCEBACK,
                       lbgpu.OUTLET_CONST)
    return lat


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("shift", [False, True])
def test_every_scheme_agrees_under_stochastic_rounding(precision, shift):
    lx, ly = 300, 61

    def alone(scheme, n, sweep=1):
        with _channel(lx, ly, precision, scheme, shift) as lat:
            if sweep == 2:
                lat.set_sweep_steps(2)
            lat.step(n)
            return lat.populations()

    for n in (1, 2, 57):
        ref = alone("pull", n)
        aa, two = alone("aa", n), alone("pull", n, 2)
        assert same(aa, ref), (n, describe_diff(aa, ref))
        assert same(two, ref), (n, describe_diff(two, ref))


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_every_boundary_rule_under_stochastic_rounding(precision):
    st = O.random_boundary_lattice(41, 33, seed=12)

    def run(scheme, seed=3, sweep=1):
        with lbgpu.Lattice(st.lx, st.ly, precision, scheme) as lat:
            lat.set_offset_scale(SCALE[precision])
            lat.set_stochastic_rounding(True, seed)
            lat.set_geometry(st.omega, st.tag, st.bc, st.zgb)
            lat.set_populations(st.lat, st.tmp)
            if sweep == 2:
                lat.set_sweep_steps(2)
            lat.step(9)
            return lat.populations()

    ref = run("pull")
    assert same(run("aa"), ref)
    assert same(run("pull", sweep=2), ref)
    exp = O.run(st, 9).lat[1:-1, 1:-1]
    assert np.abs(ref[1:-1, 1:-1] - exp).max() < (3e-3 if precision == "f16" else 2e-2)


def test_seeds_reproduce_and_differ():
    def run(seed, rs=True):
        with _channel(200, 41, "f16", "pull", False, seed=seed, rs=rs) as lat:
            lat.step(20)
            return lat.populations()

    a, b, c, rn = run(11), run(11), run(12), run(0, rs=False)
    assert same(a, b)
    assert not same(a, c)
    assert not same(a, rn)
    # the same state up to rounding: every value within a few quanta of the nearest-rounded run
    assert np.abs(a - rn).max() < 1e-4


def test_stochastic_fp16_against_the_oracle():
    """250x51 channel, 5000 steps: the stochastically rounded FP16 state against FP64."""
    st = O.build_cylinder(O.Cylinder.baseline(250, 51))
    exp = O.run(st, 5000).lat[1:-1, 1:-1]
    fluid = st.tag[1:-1, 1:-1] == 1

    def vel(f):
        rho = f.sum(axis=2)
        ux = (f[..., 1] + f[..., 5] + f[..., 8] - f[..., 3] - f[..., 6] - f[..., 7]) / rho
        uy = (f[..., 2] + f[..., 5] + f[..., 6] - f[..., 4] - f[..., 7] - f[..., 8]) / rho
        return ux[fluid], uy[fluid]

    ex, ey = vel(exp)
    rel = {}
    for rs in (False, True):
        with _channel(250, 51, "f16", "pull", False, rs=rs, umax=0.02, re=100.0) as lat:
            lat.step(5000)
            gx, gy = vel(lat.populations()[1:-1, 1:-1])
        rel[rs] = np.sqrt(((gx - ex) ** 2 + (gy - ey) ** 2).sum() / (ex ** 2 + ey ** 2).sum())
    assert rel[True] <= 3e-2, rel


def test_stochastic_rounding_arguments():
    with lbgpu.Lattice(40, 20, "f32", "pull") as lat:
        with pytest.raises(lbgpu.LbError) as e:
            lat.set_stochastic_rounding(True, 1)
        assert e.value.code == 7
    with lbgpu.Lattice(40, 20, "f16", "pull") as lat:
        with pytest.raises(lbgpu.LbError) as e:
            lbgpu._check(lbgpu.lib().lbgpu_set_stochastic_rounding(lat.h, 2, 0))
        assert e.value.code == 3
    lbgpu.clear_error()


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("shape", [(32, 1), (128, 4)])
def test_batch_members_round_like_the_lattice_alone(precision, shape):
    """Members of every scheme, some rounding stochastically and some to nearest, one of them
    switched on between calls: each ends bit-identical to its lattice stepped alone (57 steps:
    the members' own first step, a replayed 50-step chunk and an odd remainder)."""
    specs = [("pull", False, 7, True), ("aa", False, 8, True), ("pull", True, 9, True), ("pull", False, 0, False),
             ("aa", True, 10, False)]

    def make(scheme, shift, seed, rs):
        return _channel(120 + 16 * seed, 37, precision, scheme, shift, seed=seed, rs=rs)

    def alone(scheme, shift, seed, rs, late):
        with make(scheme, shift, seed, rs and not late) as lat:
            lat.step(20)
            if late:
                lat.set_stochastic_rounding(True, seed)
            lat.step(37)
            return lat.populations()

    want = [alone(sc, sh, sd, rs, late=(i == 4)) for i, (sc, sh, sd, rs) in enumerate(specs)]
    lats = [make(sc, sh, sd, rs) for sc, sh, sd, rs in specs]
    try:
        with lbgpu.Batch(precision) as batch:
            for c in range(6):
                batch.set_shape(c, *shape)
            slots = [batch.add(lat) for lat in lats]
            batch.step(20)
            batch.synchronize()
            lats[4].set_stochastic_rounding(True, 10)
            batch.step(37)
            batch.synchronize()
            got = [lat.populations() for lat in lats]
            for sl in slots:
                batch.remove(sl)
        for i, (g, w) in enumerate(zip(got, want)):
            assert same(g, w), (i, specs[i], describe_diff(g, w))
    finally:
        for lat in lats:
            lat.close()


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_stochastic_rounding_with_the_extrapolated_outlet(precision):
    """The reference driver's outlet (zero-gradient density pass before every step): pull and AA
    stay bit-identical, and the two-step setting falls back to single steps with the same bits."""
    lx, ly, n = 260, 41, 31

    def run(scheme, sweep=1):
        with lbgpu.Lattice(lx, ly, precision, scheme) as lat:
            lat.set_offset_scale(SCALE[precision])
            lat.set_stochastic_rounding(True, 9)
            lat.setup_cylinder(lx // 4, ly // 2, ly // 10 + 1, 0.03, 60.0, lbgpu.WALL_REGULARIZED,
                               lbgpu.OUTLET_ZGB)
            if sweep == 2:
                lat.set_sweep_steps(2)
            lat.step(n)
            return lat.populations()

    ref = run("pull")
    aa, two = run("aa"), run("pull", 2)
    assert same(aa, ref), describe_diff(aa, ref)
    assert same(two, ref), describe_diff(two, ref)
