"""Serving: continuous batching of cylinder-channel requests (lbgpu_server_*).

The contract: a request's result does not depend on what else the server was running.  Each
request's final velocity field and step count are the same, bit for bit, whether it was solved
in the batched mix, solved in the sequential mode, or set up and stepped alone through
lbgpu_step; the server never holds more device memory than its budget; and requests retire at
their step cap or as soon as their velocity change over one check interval falls below their
tolerance.
"""
import numpy as np
import pytest

import lbgpu

pytestmark = pytest.mark.gpu

CHECK = 100


def requests(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        lx = int(rng.integers(48, 260))
        ly = int(rng.integers(24, 90))
        r = max(2, ly // 10)
        out.append(dict(lx=lx, ly=ly, obst_x=lx // 5 + 1, obst_y=ly // 2 + 1, obst_r=r,
                        umax=float(rng.uniform(0.01, 0.04)), re=float(rng.uniform(10, 120)),
                        max_steps=CHECK * int(rng.integers(1, 6)),
                        tol=[0.0, 1.0, 2e-4][k % 3],
                        arrival=float(rng.uniform(0.0, 0.02)), want_fields=True))
    return out


def serve(precision, reqs, batched, budget, solo_nodes=None):
    base, _, rs = lbgpu.storage_form(precision)
    with lbgpu.Server(base, budget, CHECK, stochastic=rs) as srv:
        if solo_nodes is not None:
            srv.set_solo_nodes(solo_nodes)
        ids = [srv.submit(**q) for q in reqs]
        srv.run(batched)
        res = [srv.result(i, fields=True) for i in ids]
        return res, srv.stats()


def alone(precision, q, steps, rid):
    base, _, rs = lbgpu.storage_form(precision)
    with lbgpu.Lattice(q["lx"], q["ly"], base, "pull") as lat:
        if base in lbgpu.DEFAULT_SCALE:
            lat.set_offset_scale(lbgpu.DEFAULT_SCALE[base])
        if rs:   # the server seeds a request's rounding with its id
            lat.set_stochastic_rounding(True, rid)
        lat.setup_cylinder(q["obst_x"], q["obst_y"], q["obst_r"], q["umax"], q["re"],
                           lbgpu.WALL_BOUNCEBACK, lbgpu.OUTLET_CONST)
        lat.step(steps)
        _, ux, uy = lat.macros()
        return ux, uy


@pytest.mark.parametrize("precision,solo_nodes", [("f32", 0), ("f16", 0), ("f64", 0),
                                                 ("f32", 12000), ("f16", 12000),
                                                 ("f16r", 0), ("bf16r", 12000)])
def test_served_results_match_sequential_and_alone(precision, solo_nodes):
    """solo_nodes 0: every request a batch member; 12000: the larger ones step on their own.
    'r': stochastic rounding."""
    reqs = requests(7, 12)
    base = lbgpu.storage_form(precision)[0]
    budget = sum(lbgpu.lattice_bytes(q["lx"], q["ly"], base) + 8 * q["lx"] * q["ly"]
                 for q in reqs) // 3       # about a third of the requests fit at once
    mix, st_mix = serve(precision, reqs, True, budget, solo_nodes)
    solo = [r["solo"] for r in mix]
    if solo_nodes:
        assert any(solo) and not all(solo)
        assert solo == [int(q["lx"] * q["ly"] >= solo_nodes) for q in reqs]
    else:
        assert not any(solo)
    seq, st_seq = serve(precision, reqs, False, budget)
    assert st_mix["peak_bytes"] <= budget and st_seq["peak_bytes"] <= budget
    assert st_mix["peak_resident"] > 1 and st_seq["peak_resident"] == 1
    for k, (q, a, b) in enumerate(zip(reqs, mix, seq)):
        assert a["done"] and b["done"], k
        assert a["steps"] == b["steps"] and a["converged"] == b["converged"], k
        assert a["admit"] >= q["arrival"] and a["finish"] > a["admit"], k
        assert np.array_equal(a["ux"], b["ux"]) and np.array_equal(a["uy"], b["uy"]), k
        assert a["last_change"] == b["last_change"], k
        ux, uy = alone(precision, q, a["steps"], k)
        assert np.array_equal(a["ux"], ux) and np.array_equal(a["uy"], uy), k
        if q["tol"] == 1.0:        # any change after the first interval is below 1
            assert a["converged"] == 1 and a["steps"] == CHECK, k
        if q["tol"] == 0.0:
            assert a["converged"] == 0 and a["steps"] == q["max_steps"], k
        if a["converged"]:
            assert a["last_change"] < q["tol"], k
        else:
            assert a["steps"] == q["max_steps"], k
    assert st_mix["lattice_updates"] == st_seq["lattice_updates"]


def test_server_schemes_and_late_arrivals():
    reqs = requests(11, 6)
    for k, q in enumerate(reqs):
        q["arrival"] = 0.01 * k          # trickle in while others run
        q["tol"] = 0.0
    budget = 1 << 30
    with lbgpu.Server("f32", budget, CHECK) as srv:
        for c in range(6):
            srv.set_scheme(c, "aa")
        ids = [srv.submit(**q) for q in reqs]
        srv.run(True)
        res = [srv.result(i, fields=True) for i in ids]
    for k, (q, r) in enumerate(zip(reqs, res)):
        assert r["steps"] == q["max_steps"] and r["admit"] >= q["arrival"]
        ux, uy = alone("f32", q, r["steps"], k)
        assert np.array_equal(r["ux"], ux) and np.array_equal(r["uy"], uy)


def test_submit_rejects_bad_requests():
    with lbgpu.Server("f32", 1 << 20, CHECK) as srv:
        with pytest.raises(lbgpu.LbError) as e:
            srv.submit(64, 32, 13, 17, 3, 0.02, 50.0, max_steps=150)     # not a multiple of 100
        assert e.value.code == 3
        with pytest.raises(lbgpu.LbError) as e:
            srv.submit(4096, 1024, 800, 512, 100, 0.02, 50.0, max_steps=100)  # over the budget
        assert e.value.code == 10
    lbgpu.clear_error()
