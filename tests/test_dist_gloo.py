"""bench.py's replica plumbing at world size 2 over gloo, on the CPU.

The channel step has no exchange between GPUs (each rank runs its own lattice), so the only
multi-rank logic is the barrier around the timed region, the max of the device times over
ranks, the whole-job rate (world x nodes x steps over that max) and which rank prints.  These
run here as two spawned processes with a stand-in lattice whose timed call reports a
rank-dependent duration.
"""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

import lbgpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _FakeLattice:
    """Stands in for lbgpu.Lattice: rank r reports (r + 1) x 10 ms for any timed call."""
    rank = 0
    calls = []

    def __init__(self, nx, ny, precision, scheme):
        self.lx, self.ly = nx, ny
        self.last_launches = 7
        _FakeLattice.calls.append(("new", nx, ny, precision, scheme))

    def set_sweep_steps(self, n):
        _FakeLattice.calls.append(("sweep", n))

    def set_offset_scale(self, s):
        _FakeLattice.calls.append(("scale", s))

    def set_offset_shift(self, u):
        _FakeLattice.calls.append(("shift", len(u)))

    def setup_cylinder(self, *a):
        _FakeLattice.calls.append(("setup",) + a[:3])

    def step(self, n):
        _FakeLattice.calls.append(("step", n))

    def synchronize(self):
        pass

    def step_timed(self, n):
        _FakeLattice.calls.append(("timed", n))
        return 10.0 * (_FakeLattice.rank + 1)

    def close(self):
        _FakeLattice.calls.append(("close",))


class _FakeLbgpu:
    """The lbgpu module with the stand-in lattice (its storage helpers are the real ones)."""
    Lattice = _FakeLattice
    WALL_BOUNCEBACK, OUTLET_CONST = 0, 1
    storage_form = staticmethod(lbgpu.storage_form)
    configure_storage = staticmethod(lbgpu.configure_storage)


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "memory-aware-lbm_b200"))
    import bench

    res = {}
    d = bench.Dist()
    try:
        res["backend"] = d.backend
        res["max"] = d.max(1.5 * (rank + 1))
        d.barrier()

        _FakeLattice.rank = rank
        ms, launches, clocks = bench.time_lattice(_FakeLbgpu, 200, 50, "f16s", "pull2", 12, 3, d)
        res["time_lattice"] = [ms, launches, clocks]
        res["calls"] = [list(c) for c in _FakeLattice.calls]

        bench.reference_cpu = lambda nx, ny, steps, warmup, budget_s, variant=None: {
            "variant": "tight_openmp", "steps": 4, "seconds": 2.0, "threads": 3,
            "mlups": nx * ny * 4 / 2.0 / 1e6, "setup_s": 0.1, "probe_ms_per_step": {}}

        class Args:
            nx, ny, steps, warmup, gpus = 100, 40, 4, 3, world

        buf = io.StringIO()
        with redirect_stdout(buf):
            bench.run_reference_arm(Args, d)
        res["reference_out"] = buf.getvalue()
        d.barrier()
    finally:
        d.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


@pytest.fixture(scope="module")
def two_ranks(tmp_path_factory):
    out = tmp_path_factory.mktemp("gloo")
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True,
                       start_method="spawn")
    res = []
    for r in range(2):
        with open(out / f"rank{r}.json") as f:
            res.append(json.load(f))
    return res


def test_ranks_use_gloo_without_a_gpu(two_ranks):
    assert [r["backend"] for r in two_ranks] == ["gloo", "gloo"]


def test_max_over_ranks(two_ranks):
    assert [r["max"] for r in two_ranks] == [3.0, 3.0]


def test_timed_region_reports_the_slowest_rank_everywhere(two_ranks):
    for r in two_ranks:
        ms, launches, clocks = r["time_lattice"]
        assert ms == 20.0            # rank 1's 20 ms, not this rank's own
        assert launches == 7 and clocks is None


def test_time_lattice_sets_the_lattice_up_in_order(two_ranks):
    calls = [c[0] for c in two_ranks[0]["calls"]]
    # the offset scale and shift encode the initial state, so they precede the set-up
    assert calls == ["new", "sweep", "scale", "shift", "setup", "step", "timed", "close"]
    new = two_ranks[0]["calls"][0]
    assert new[1:] == [200, 50, "f16", "pull"]
    assert two_ranks[0]["calls"][2] == ["scale", 17]
    assert two_ranks[0]["calls"][3] == ["shift", 52]
    assert two_ranks[0]["calls"][5] == ["step", 3]
    assert two_ranks[0]["calls"][6] == ["timed", 12]


def test_reference_arm_prints_one_line_from_rank_zero(two_ranks):
    assert two_ranks[1]["reference_out"] == ""
    lines = two_ranks[0]["reference_out"].strip().splitlines()
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2
    assert line["value"] == pytest.approx(100 * 40 * 4 / 2.0 / 1e6, abs=0.01)
    assert line["cpu_baseline"]["kind"] == "reference"
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
