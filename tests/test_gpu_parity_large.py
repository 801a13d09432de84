"""Parity at the benchmarked size, against the reference's own code.

The benchmark times the FP64 kernels on the 16384 x 4096 cylinder channel (67.1M nodes, a
4.8 GB FP64 buffer, 38x the 126 MB L2).  Here the same lattice, set up on the device, is
stepped by the pull kernel, the in-place AA pair (odd step count), the two-step sweep and the
drop-in interface (lb.h, host node arrays), and every population -- ghost ring included -- is
compared bit for bit with the reference's lb.c compiled unmodified, run from the reference's own
initial state (iniEquilibrium with the Poiseuille profile, unsteady.c:162-199).
A ragged 8190 x 2047 lattice with the application driver's own scenario (regularized walls,
zero-gradient outlet, unsteady.c:185-214) exercises partial blocks, the zero-gradient outlet
and the L2 prefetch guards off L2 in the same way.

Which reference build: the serial one (oracle/_ref/libref_lb_serial.so: collide + propagate,
lb.c:172-288).  The OpenMP build cannot pin results: bounceBack keeps its swap in a static array
(boundaries.c:49), so threads that collide bounce-back nodes at the same time overwrite each
other's populations.  On 8 host threads, after 10 steps, its result on the 4096 x 1024 channel
with bounce-back walls differed from the serial build in 67,000-75,000 slots and between two
runs; on a 1030 x 255 channel with regularized walls, where only the obstacle bounces back and
its columns are split between threads, it differed too.  The serial build is deterministic and
is the build the oracle's golden digests come from.

Tolerance: zero for FP64 (NaN payloads aside).  FP32 storage is held to the bounds written in
test_fp32_error_at_16384x4096 against the FP64 kernel after the configuration's 1,000 steps.
"""
import numpy as np
import pytest

import lbgpu
import oracle as O

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not O.ref_available(),
                       reason="reference build oracle/_ref/libref_lb_serial.so not present"),
]

BIG = O.Cylinder.baseline(16384, 4096)
RAGGED = O.Cylinder.reference_driver(8190, 2047)


def _ref_setup(c):
    return O.ref_setup(c, openmp=False)


def _ref_step(c, n):
    return O.ref_step("origin", n)


def _ref_dump(c):
    return O.ref_dump(c)


def _ref_free(c):
    O.ref_lib(openmp=False).ref_free()


def same_large(a, b, chunk=512):
    """Bit-for-bit equality (NaN payloads aside) of two [X, Y, 9] lattices, slab by slab so
    that no temporary is larger than a slab."""
    assert a.shape == b.shape, (a.shape, b.shape)
    for x0 in range(0, a.shape[0], chunk):
        sa, sb = a[x0:x0 + chunk], b[x0:x0 + chunk]
        na, nb = np.isnan(sa), np.isnan(sb)
        if not np.array_equal(na, nb):
            return False, f"NaN slots differ in columns {x0}..{x0 + chunk - 1}"
        ia = np.where(na, 0.0, sa).view(np.uint64)
        ib = np.where(nb, 0.0, sb).view(np.uint64)
        if not np.array_equal(ia, ib):
            d = np.abs(np.where(na, 0.0, sa) - np.where(nb, 0.0, sb))
            k = np.unravel_index(np.argmax(d), d.shape)
            return False, (f"{int((ia != ib).sum())} slots differ in columns {x0}..; max "
                           f"|diff| {d.max():.3e} at X={x0 + k[0]}, Y={k[1]}, i={k[2]}")
    return True, ""


def _device_lattice(c, scheme, precision="f64"):
    lat = lbgpu.Lattice(c.lx, c.ly, precision, scheme)
    lat.omega = lat.setup_cylinder(c.obst_x, c.obst_y, c.obst_r, c.umax, c.re, c.wall, c.outlet)
    return lat


def _check(lat, ref, what):
    ok, msg = same_large(lat.populations(), ref)
    assert ok, f"{what}: {msg}"


@pytest.mark.parametrize("c", [BIG, RAGGED], ids=["16384x4096", "8190x2047"])
def test_fp64_kernels_match_reference_at_size(c):
    """Set-up, 10 and 11 steps of the pull kernel, 11 of the AA pair and 10 of the two-step
    sweep, all against the reference's origin variant on the same lattice."""
    omega = _ref_setup(c)
    try:
        ref0 = _ref_dump(c)
        with _device_lattice(c, "pull") as lat:
            assert lat.omega == omega
            _check(lat, ref0, "device set-up")
            del ref0
            assert _ref_step(c, 10) == 10
            ref10 = _ref_dump(c)
            lat.step(10)
            _check(lat, ref10, "pull kernel, 10 steps")
            assert _ref_step(c, 1) == 1
            ref11 = _ref_dump(c)
            lat.step(1)
            _check(lat, ref11, "pull kernel, 11 steps")
    finally:
        _ref_free(c)
    with _device_lattice(c, "aa") as lat:
        lat.step(11)
        _check(lat, ref11, "AA pair, 11 steps")
    del ref11
    with _device_lattice(c, "pull") as lat:
        lat.set_sweep_steps(2)
        lat.step(10)
        _check(lat, ref10, "two steps per sweep, 10 steps")


@pytest.mark.parametrize("c,variant", [(BIG, "combine"), (RAGGED, "tight")],
                         ids=["16384x4096-combine", "8190x2047-tight"])
def test_dropin_interface_matches_reference_at_size(c, variant):
    """The lb.h entry points with host node arrays (the benchmark's end-to-end path for
    combine), 10 steps, against the reference's origin variant."""
    _ref_setup(c)
    try:
        _ref_step(c, 10)
        ref10 = _ref_dump(c)
    finally:
        _ref_free(c)
    got, done, _ = lbgpu.drive(c.lx, c.ly, c.obst_x, c.obst_y, c.obst_r, 10, variant,
                               umax=c.umax, re=c.re, wall=c.wall, outlet=c.outlet)
    assert done == 10
    ok, msg = same_large(got, ref10)
    assert ok, f"drop-in {variant}: {msg}"


def _velocity_error(a, b):
    """Relative L2 error of the velocity field a against b (interior nodes)."""
    num = np.sqrt(np.sum((a[1] - b[1]) ** 2 + (a[2] - b[2]) ** 2))
    den = np.sqrt(np.sum(b[1] ** 2 + b[2] ** 2))
    return float(num / den)


def test_fp32_error_at_16384x4096():
    """FP32 storage (pull and AA bit-identical to each other) against the FP64 kernel after the
    configuration's 1,000 steps: velocity relative L2 error <= 2e-4, total mass relative
    difference <= 2e-6 (measured on a B200: 1.09e-4 and 8.9e-7)."""
    with _device_lattice(BIG, "pull") as lat:
        lat.step(1000)
        m64 = lat.moments()
        f64 = lat.macros()
    with _device_lattice(BIG, "pull", "f32") as lat:
        lat.step(1000)
        m32 = lat.moments()
        f32 = lat.macros()
    with _device_lattice(BIG, "aa", "f32") as lat:
        lat.step(1000)
        for a, b in zip(lat.macros(), f32):
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), "FP32 AA vs FP32 pull"
    err = _velocity_error(f32, f64)
    mass = abs(m32[0] - m64[0]) / m64[0]
    print(f"FP32 at 16384x4096 x 1000: velocity rel L2 {err:.3e}, mass rel {mass:.3e}")
    assert m32[6] == 0
    assert err <= 2e-4, err
    assert mass <= 2e-6, mass


@pytest.mark.parametrize("precision", ["f16", "bf16"])
def test_16bit_pull_and_aa_agree_at_16384x4096(precision):
    """The 16-bit quad kernels (pull, and the AA pair at an odd count) give the same stored
    state at the benchmarked size, L2 prefetch distance of 16 rows included."""
    outs = []
    for scheme in ("pull", "aa"):
        with lbgpu.Lattice(BIG.lx, BIG.ly, precision, scheme) as lat:
            lat.set_offset_scale(lbgpu.DEFAULT_SCALE[precision])
            lat.setup_cylinder(BIG.obst_x, BIG.obst_y, BIG.obst_r, BIG.umax, BIG.re, BIG.wall,
                               BIG.outlet)
            lat.step(11)
            outs.append(lat.macros())
            assert lat.moments()[6] == 0
    for a, b in zip(*outs):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
