"""Seeded inputs of the workload studies (CPU only): the serving stream's request mix."""
import numpy as np

import studies


def test_serving_requests_follow_the_configuration():
    reqs = studies.serving_requests(5000)
    n = np.array([q["lx"] * q["ly"] for q in reqs], dtype=np.float64)
    aspect = np.array([q["lx"] / q["ly"] for q in reqs])
    re = np.array([q["re"] for q in reqs])
    assert len(reqs) == 5000
    assert n.min() >= 0.9e4 and n.max() <= 2.1e7
    # log-uniform node counts: the median near the geometric mean of the range
    assert abs(np.log(np.median(n)) - 0.5 * (np.log(1e4) + np.log(2e7))) < 0.2
    assert aspect.min() > 1.8 and aspect.max() < 8.5
    assert re.min() >= 20 and re.max() <= 500
    assert all(q["max_steps"] == 5000 and q["tol"] == 1e-7 for q in reqs)
    # the same seed gives the same stream
    assert reqs[:5] == studies.serving_requests(5000)[:5]


def test_serving_umax_keeps_omega_at_or_below_the_edge():
    for q in studies.serving_requests(2000, seed=7):
        nu = q["umax"] * 2 * q["obst_r"] / q["re"]
        omega = 1.0 / (3.0 * nu + 0.5)
        lo, hi = studies.UMAX_RANGE
        assert lo <= q["umax"] <= hi
        if q["umax"] < hi:
            assert omega <= studies.OMEGA_MAX + 1e-12
        if q["umax"] > lo:   # raised only as far as needed
            assert omega >= studies.OMEGA_MAX - 1e-9 or q["umax"] == hi


def test_member_shape_cases_hold_the_node_count_and_their_obstacles():
    total = 16384 * 4096
    cases = studies.member_shape_cases(total)
    assert cases[0] == ("alone", 16384, 4096, 1)
    for label, lx, ly, n in cases:
        assert n * lx * ly == total, (label, lx, ly, n)
        ox, oy, r = studies.shape_obstacle(lx, ly)
        # the disk stays inside the interior, clear of the inlet column and the walls
        assert 1 < ox - r and ox + r < lx and 1 < oy - r and oy + r < ly, (lx, ly, ox, oy, r)
    shapes = [(lx, ly) for label, lx, ly, _ in cases if label == "shape"]
    assert len({lx * ly for lx, ly in shapes}) == 1
    assert shapes[0][0] > shapes[0][1] and shapes[-1][0] < shapes[-1][1]   # wide to tall
