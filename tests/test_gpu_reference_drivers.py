"""Application drivers built on the GPU library against the same drivers built on the reference.

* The reference's own application driver unsteady.c, compiled unmodified against this
  repository's include/lb.h and linked with the GPU library (oracle/_ref/unsteady_gpu_<variant>),
  runs next to the same file linked with the reference's lb.c (oracle/_ref/unsteady_<variant>):
  the host-side zero-gradient update reading sim.lattice columns between steps
  (unsteady.c:205-214), the two-steps-per-call loop of tight/tight_block/panel
  (unsteady.c:425-429) and the timing line (unsteady.c:558).  The final lattices must be
  bit-identical and stdout identical once the timings are masked.  (The driver defines NO_SAVE,
  unsteady.c:37, so it writes no velocity files; any file it writes must match all the same.)
* periodic_driver.c (oracle/) calls makePeriodic on the initial state and after every stream,
  then saveVel and saveF: its GPU build must write exactly the reference build's files.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from helpers import check_golden, describe_diff, same

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
VARIANTS = ["origin", "combine", "tight", "tight_block", "panel"]
TIMING = re.compile(r"^time eclapsed in (\d+) steps, t_total=(\d+\.\d{3}), t_collid=(\d+\.\d{3}), "
                    r"t_stream=(\d+\.\d{3}), t_zgb=(\d+\.\d{3})$")

pytestmark = [
    pytest.mark.gpu,
    pytest.mark.skipif(not os.path.exists(os.path.join(REF, "unsteady_gpu_origin")),
                       reason="reference drivers under oracle/_ref are not built"),
]


def _run(exe, args, cwd, env=None):
    os.makedirs(cwd, exist_ok=True)
    r = subprocess.run([os.path.join(REF, exe)] + [str(a) for a in args], cwd=cwd,
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, f"{exe}: rc {r.returncode}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
    return r.stdout


def _masked(stdout):
    """stdout lines with the timing numbers masked; the timing line must parse."""
    out, timing = [], None
    for line in stdout.splitlines():
        m = TIMING.match(line)
        if m:
            timing = m
            line = f"time eclapsed in {m.group(1)} steps, t_total=*, t_collid=*, t_stream=*, t_zgb=*"
        out.append(line)
    assert timing is not None, stdout[-1000:]
    return out, timing


def _lattice(path, lx, ly):
    return np.fromfile(path, dtype="<f8").reshape(lx + 2, ly + 2, 9)


@pytest.mark.parametrize("variant", VARIANTS)
def test_unmodified_unsteady_driver_on_the_gpu_library(golden, variant, tmp_path):
    lx, ly, blk, stop = 256, 256, 32, 100
    outs = {}
    for kind, exe in (("ref", f"unsteady_{variant}"), ("gpu", f"unsteady_gpu_{variant}")):
        d = str(tmp_path / kind)
        env = dict(os.environ, STOP=str(stop), LBREF_DUMP=os.path.join(d, "lattice.bin"))
        env.pop("LBREF_POISON", None)
        stdout = _run(exe, [lx, ly, blk], d, env)
        files = sorted(f for f in os.listdir(d) if f.startswith("vel_"))
        outs[kind] = (stdout, d, files)
    (s_ref, d_ref, f_ref), (s_gpu, d_gpu, f_gpu) = outs["ref"], outs["gpu"]

    ref = _lattice(os.path.join(d_ref, "lattice.bin"), lx, ly)
    got = _lattice(os.path.join(d_gpu, "lattice.bin"), lx, ly)
    assert same(got, ref), describe_diff(got, ref)
    assert check_golden(golden["ref_driver_256x256_100_blk32"], got)

    assert f_gpu == f_ref, (f_ref, f_gpu)
    for name in f_ref:
        with open(os.path.join(d_ref, name), "rb") as a, open(os.path.join(d_gpu, name), "rb") as b:
            assert a.read() == b.read(), name

    lines_ref, t_ref = _masked(s_ref)
    lines_gpu, t_gpu = _masked(s_gpu)
    assert lines_gpu == lines_ref
    assert int(t_gpu.group(1)) == stop
    assert all(float(v) >= 0.0 for v in t_gpu.groups()[1:])


@pytest.mark.parametrize("lx,ly,variant", [(96, 64, 0), (96, 64, 1), (77, 45, 0), (130, 9, 1)])
def test_make_periodic_save_vel_save_f_match_reference(lx, ly, variant, tmp_path):
    """makePeriodic before the first step (the library wraps its host arrays) and after every
    stream (on the device), then saveVel and saveF of every population."""
    steps = 40
    dirs = {}
    for kind in ("ref", "gpu"):
        d = str(tmp_path / kind)
        _run(f"periodic_{kind}", [lx, ly, steps, variant, d], d)
        dirs[kind] = d
    ref = _lattice(os.path.join(dirs["ref"], "lattice.bin"), lx, ly)
    got = _lattice(os.path.join(dirs["gpu"], "lattice.bin"), lx, ly)
    assert same(got, ref), describe_diff(got, ref)
    for name in ["vel.dat"] + [f"f{i}.dat" for i in range(9)]:
        with open(os.path.join(dirs["ref"], name), "rb") as a, \
                open(os.path.join(dirs["gpu"], name), "rb") as b:
            assert a.read() == b.read(), name
