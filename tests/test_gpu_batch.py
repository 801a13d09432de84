"""Batches: many lattices of uneven size in one launch per step (lbgpu_batch_*).

The contract: every member's populations after a batch step are bit-identical to the same
lattice stepped alone, for both schemes and every precision, across chunk boundaries (CUDA-graph
replays of 50 steps), odd remainders, membership changes and autotuned tile shapes.
"""
import numpy as np
import pytest

import lbgpu
from helpers import describe_diff, same

pytestmark = pytest.mark.gpu

SIZES = [(96, 40), (200, 64), (64, 33), (130, 50), (257, 35), (33, 96)]


def channel(lx, ly, precision, scheme, seed):
    rng = np.random.default_rng(seed)
    r = max(2, int(round(ly / 10 * rng.uniform(0.8, 1.2))))
    ox = int(lx / 5 * rng.uniform(0.9, 1.1)) + 1
    oy = int(ly / 2 * rng.uniform(0.9, 1.1)) + 1
    lat = lbgpu.Lattice(lx, ly, precision, scheme)
    if precision in ("f16", "bf16"):
        lat.set_offset_scale(10 if precision == "f16" else 6)
    lat.setup_cylinder(ox, oy, r, rng.uniform(0.01, 0.04), rng.uniform(20, 200),
                       lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
    return lat


def alone(lx, ly, precision, scheme, seed, steps):
    with channel(lx, ly, precision, scheme, seed) as lat:
        lat.step(steps)
        return lat.populations()


@pytest.mark.parametrize("precision", ["f32", "f16", "f64"])
def test_members_match_lattices_stepped_alone(precision):
    schemes = ["pull", "aa", "pull", "aa", "pull", "aa"]
    lats = [channel(lx, ly, precision, s, k) for k, ((lx, ly), s) in enumerate(zip(SIZES, schemes))]
    with lbgpu.Batch(precision) as b:
        slots = [b.add(l) for l in lats]
        assert len(b) == len(lats)
        for n in (3, 50, 84):          # a prologue step, a full graph chunk, chunk + odd rest
            b.step(n)
        b.synchronize()
        got = [l.populations() for l in lats]
        assert all(l.steps_done == 137 for l in lats)
        for s in slots:
            b.remove(s)
    for k, ((lx, ly), s) in enumerate(zip(SIZES, schemes)):
        exp = alone(lx, ly, precision, s, k, 137)
        assert same(got[k], exp), (precision, k, s, describe_diff(got[k], exp))
    for l in lats:
        l.close()


def test_membership_changes_between_steps():
    lats = [channel(lx, ly, "f32", "pull", k) for k, (lx, ly) in enumerate(SIZES[:4])]
    with lbgpu.Batch("f32") as b:
        slots = [b.add(l) for l in lats]
        b.step(20)
        b.remove(slots[1])
        newcomer = channel(70, 45, "f32", "aa", 99)
        b.add(newcomer)
        b.step(61)
        b.synchronize()
        got = [l.populations() for l in lats] + [newcomer.populations()]
        for s in list(b.members):
            b.remove(s)
    assert same(got[0], alone(*SIZES[0], "f32", "pull", 0, 81))
    assert same(got[1], alone(*SIZES[1], "f32", "pull", 1, 20))
    assert same(got[2], alone(*SIZES[2], "f32", "pull", 2, 81))
    assert same(got[4], alone(70, 45, "f32", "aa", 99, 61))
    for l in lats + [newcomer]:
        l.close()


def test_autotuned_shapes_keep_results_exact():
    lats = [channel(lx, ly, "f32", "pull", k) for k, (lx, ly) in enumerate(SIZES[:3])]
    with lbgpu.Batch("f32") as b:
        slots = [b.add(l) for l in lats]
        best = b.autotune(2)
        classes = {lbgpu.size_class(lx * ly) for lx, ly in SIZES[:3]}
        for c in classes:
            assert b.shape(c) in ((32, 1), (64, 1), (128, 1))
            assert best[c] > 0
        assert all(best[c] == 0 for c in range(6) if c not in classes)
        assert b.threads in (128, 256, 512)
        b.step(7)
        b.synchronize()
        got = [(l.populations(), l.steps_done) for l in lats]
        for s in slots:
            b.remove(s)
    for k, (lx, ly) in enumerate(SIZES[:3]):
        pops, steps = got[k]
        assert same(pops, alone(lx, ly, "f32", "pull", k, steps)), k
    for l in lats:
        l.close()


@pytest.mark.parametrize("persistent,width,threads", [
    (True, 128, 128), (False, 128, 128), (True, 32, 128), (False, 64, 128),
    (True, 64, 256), (False, 32, 256), (True, 128, 512), (False, 32, 512)])
def test_every_launch_form_and_tile_is_exact(persistent, width, threads):
    """AA members that join at different phases run as two lists of opposite kinds."""
    lats = [channel(lx, ly, "f32", s, k) for k, ((lx, ly), s) in
            enumerate(zip(SIZES[:4], ["aa", "pull", "aa", "aa"]))]
    lats[2].step(1)                    # an AA member in the swapped phase when it joins
    with lbgpu.Batch("f32") as b:
        b.persistent = persistent
        b.threads = threads
        assert b.persistent == persistent and b.threads == threads
        for c in range(6):
            b.set_shape(c, width, 1)
        slots = [b.add(l) for l in lats]
        for n in (51, 50, 3):          # odd rest: the lists swap kinds; then a graph again
            b.step(n)
        b.synchronize()
        got = [(l.populations(), l.steps_done) for l in lats]
        for s in slots:
            b.remove(s)
    for k, ((lx, ly), s) in enumerate(zip(SIZES[:4], ["aa", "pull", "aa", "aa"])):
        pops, steps = got[k]
        assert same(pops, alone(lx, ly, "f32", s, k, steps)), (k, s, persistent, width)
    for l in lats:
        l.close()


@pytest.mark.parametrize("precision", ["f16", "bf16"])
@pytest.mark.parametrize("persistent,threads", [(True, 128), (False, 256), (False, 512)])
def test_four_nodes_a_thread_is_exact(precision, persistent, threads):
    """16-bit pull members in quad tiles (narrow ones fall back to per-node) beside AA members."""
    sizes = [(300, 40), (257, 35), (96, 40), (520, 70)]
    schemes = ["pull", "pull", "pull", "aa"]
    lats = [channel(lx, ly, precision, s, k) for k, ((lx, ly), s) in enumerate(zip(sizes, schemes))]
    with lbgpu.Batch(precision) as b:
        b.persistent = persistent
        b.threads = threads
        for c in range(6):
            b.set_shape(c, 128, 4)
            assert b.shape(c) == (128, 4)
        slots = [b.add(l) for l in lats]
        for n in (3, 50, 7):
            b.step(n)
        b.synchronize()
        got = [(l.populations(), l.steps_done) for l in lats]
        for s in slots:
            b.remove(s)
    for k, ((lx, ly), s) in enumerate(zip(sizes, schemes)):
        pops, steps = got[k]
        assert same(pops, alone(lx, ly, precision, s, k, steps)), (k, s, persistent, threads)
    for l in lats:
        l.close()


def test_batch_rejects_mismatched_members():
    with lbgpu.Batch("f32") as b, lbgpu.Lattice(40, 20, "f64") as wrong:
        with pytest.raises(lbgpu.LbError) as e:
            b.add(wrong)
        assert e.value.code == 3
    with lbgpu.Batch("f32") as b:
        with pytest.raises(lbgpu.LbError) as e:
            b.set_shape(0, 128, 4)             # four nodes a thread: 16-bit storage only
        assert e.value.code == 3
    with lbgpu.Batch("f64") as b, lbgpu.Lattice(40, 20, "f64") as zgb:
        zgb.setup_cylinder(9, 11, 3, 0.02, 100.0, lbgpu.WALL_REGULARIZED, lbgpu.OUTLET_ZGB)
        with pytest.raises(lbgpu.LbError) as e:
            b.add(zgb)
        assert e.value.code == 3


def test_scheme_tuner_reports_both_timings():
    scheme, t_pull, t_aa = lbgpu.tune_scheme("f32", 512, 128, 6)
    assert scheme in ("pull", "aa") and t_pull > 0 and t_aa > 0


@pytest.mark.parametrize("precision,passes", [("f32", 1), ("f32", 3), ("f16", 64), ("bf16", 3)])
def test_strip_lengths_are_exact(precision, passes):
    """A block stepping `passes` tiles down a member gives the same result for every strip
    length, ragged member heights included (the last strip of a member stops at its last row)."""
    schemes = ["pull", "aa", "pull", "pull", "aa", "pull"]
    steps = 57
    lats = [channel(lx, ly, precision, s, k) for k, ((lx, ly), s) in enumerate(zip(SIZES, schemes))]
    with lbgpu.Batch(precision) as b:
        for c in range(6):
            b.set_passes(c, passes)
            assert b.passes(c) == passes
            if precision != "f32":
                b.set_shape(c, 128, 4)
        for l in lats:
            b.add(l)
        b.step(steps)
        b.synchronize()
        got = [l.populations() for l in lats]
    for k, ((lx, ly), s) in enumerate(zip(SIZES, schemes)):
        assert same(got[k], alone(lx, ly, precision, s, k, steps)), (precision, passes, k, s)
    for l in lats:
        l.close()


def test_row_shifted_member_in_a_quad_batch_is_exact():
    """A 16-bit member with offsets from a banded inflow profile (the batch then runs the quad
    kernel with the shifted path) next to unshifted members: each as stepped alone."""
    steps = 53

    def make(k, lx, ly, shifted):
        lat = channel(lx, ly, "f16", "pull", k) if not shifted else None
        if shifted:
            lat = lbgpu.Lattice(lx, ly, "f16", "pull")
            lbgpu.configure_storage(lat, "f16br", 0.03, seed=7)
            lat.setup_cylinder(lx // 5 + 1, ly // 2 + 1, ly // 10 + 1, 0.03, 120.0,
                               lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
        return lat

    spec = [(0, 200, 64, True), (1, 257, 135, False), (2, 130, 70, True)]
    lats = [make(*q) for q in spec]
    with lbgpu.Batch("f16") as b:
        for c in range(6):
            b.set_shape(c, 128, 4)
        for l in lats:
            b.add(l)
        b.step(steps)
        b.synchronize()
        got = [l.populations() for l in lats]
    for (k, lx, ly, shifted), g in zip(spec, got):
        with make(k, lx, ly, shifted) as lat:
            lat.step(steps)
            assert same(g, lat.populations()), (k, shifted)
    for l in lats:
        l.close()
