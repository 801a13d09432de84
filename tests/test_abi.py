"""The C ABI of liblbgpu.so on a machine without a GPU: exports, host logic, error reporting.

No kernel runs here.  The host functions the drop-in interface exports (computeMacros,
computeEquilibrium, bgk, bounceBack and the 16 boundary rules) are checked bit-for-bit against
the oracle's restatement of the reference on random nodes; the cylinder builder against the
oracle's builder; error codes for calls that need a device.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import lbgpu
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_dp = ctypes.POINTER(ctypes.c_double)

# driver-defined in the reference too (lb.h:97): the library must not define it
DRIVER_DEFINED = {"updateZeroGradientBoundary"}

RULES = ["bgk", "bounceBack",
         "upperZouHe", "lowerZouHe", "leftZouHe", "rightZouHe",
         "upperPressureZouHe", "lowerPressureZouHe", "leftPressureZouHe", "rightPressureZouHe",
         "upperRegularized", "lowerRegularized", "leftRegularized", "rightRegularized",
         "upperPressureRegularized", "lowerPressureRegularized", "leftPressureRegularized",
         "rightPressureRegularized"]


class Dynamics(ctypes.Structure):
    _fields_ = [("dynamicsFun", ctypes.c_void_p), ("selfData", ctypes.c_void_p)]


class BCData(ctypes.Structure):   # VelocityBCData and PressureBCData share this layout
    _fields_ = [("bulkDynamics", ctypes.POINTER(Dynamics)), ("a", ctypes.c_double),
                ("b", ctypes.c_double)]


def test_library_exports_every_declared_function():
    L = lbgpu.lib()
    declared = set(lbgpu.declared_functions())
    assert len(declared) > 60
    missing = [n for n in sorted(declared - DRIVER_DEFINED) if not hasattr(L, n)]
    assert not missing, missing


def test_library_exports_driver_globals():
    L = lbgpu.lib()
    for name in ("pressureBoundary", "blk_size", "myrho1", "myrho2", "iT", "count",
                 "thread_block", "NUM_THREADS", "global_CM"):
        ctypes.c_int.in_dll(L, name)   # raises ValueError when absent


def test_struct_layouts_match_the_reference_abi(tmp_path):
    # Node = 9 doubles + pointer (80 bytes), Dynamics = 2 pointers, BC data = ptr + 2 doubles
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "lb.h"
#include "boundaries.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu\n", sizeof(Node), sizeof(Dynamics), sizeof(VelocityBCData),
         sizeof(PressureBCData), offsetof(Simulation, lattice), offsetof(Simulation, tmpLattice));
  return 0; }
"""
    exe = str(tmp_path / "abi_layout")
    cfile = exe + ".c"
    with open(cfile, "w") as f:
        f.write(src)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, cfile], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert [int(v) for v in out] == [80, 16, 24, 24, 24, 32]


def _random_populations(rng):
    f = np.zeros(9)
    O.oracle_lib().orc_init_equilibrium(f.ctypes.data_as(_dp), 1 + rng.uniform(-0.05, 0.05),
                                        rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05))
    return f * (1 + rng.uniform(-0.02, 0.02, 9))


def test_host_rules_match_oracle_bit_for_bit():
    L = lbgpu.lib()
    orc = O.oracle_lib()
    rng = np.random.default_rng(7)
    omega = ctypes.c_double(1.7)
    bulk = Dynamics(ctypes.cast(L.bgk, ctypes.c_void_p).value,
                    ctypes.cast(ctypes.pointer(omega), ctypes.c_void_p).value)
    for tag, name in enumerate(RULES, start=1):
        fn = getattr(L, name)
        fn.argtypes = [_dp, ctypes.c_void_p]
        for _ in range(40):
            f = _random_populations(rng)
            p = np.array([rng.uniform(-0.03, 0.03), rng.uniform(-0.03, 0.03)])
            if "Pressure" in name:
                p[0] = rng.uniform(0.97, 1.03)
            data = BCData(ctypes.pointer(bulk), p[0], p[1])
            mine = f.copy()
            self_data = (ctypes.cast(ctypes.pointer(omega), ctypes.c_void_p) if name == "bgk"
                         else ctypes.cast(ctypes.pointer(data), ctypes.c_void_p))
            fn(mine.ctypes.data_as(_dp), self_data)
            ref = f.copy()
            orc.orc_collide_node(tag, ref.ctypes.data_as(_dp), omega.value,
                                 p.ctypes.data_as(_dp))
            assert np.array_equal(mine.view(np.uint64), ref.view(np.uint64)), name


def test_compute_macros_and_equilibrium_match_oracle():
    L = lbgpu.lib()
    orc = O.oracle_lib()
    rng = np.random.default_rng(3)
    for _ in range(200):
        f = _random_populations(rng)
        a = [np.zeros(1) for _ in range(3)]
        b = [np.zeros(1) for _ in range(3)]
        L.computeMacros(f.ctypes.data_as(_dp), *[x.ctypes.data_as(_dp) for x in a])
        orc.orc_macros(f.ctypes.data_as(_dp), *[x.ctypes.data_as(_dp) for x in b])
        assert [x[0] for x in a] == [x[0] for x in b]
        i = int(rng.integers(0, 9))
        args = (i, a[0][0], a[1][0], a[2][0], a[1][0] ** 2 + a[2][0] ** 2)
        assert L.computeEquilibrium(*args) == orc.orc_equilibrium(*args)


@pytest.mark.parametrize("c", [O.Cylinder.baseline(250, 51), O.Cylinder.reference_driver(97, 40),
                               O.Cylinder.baseline(16, 5)])
def test_cylinder_builder_matches_oracle(c):
    omega, tag, bc, zgb, f = lbgpu.build_cylinder(c.lx, c.ly, c.obst_x, c.obst_y, c.obst_r,
                                                  c.umax, c.re, c.wall, c.outlet)
    st = O.build_cylinder(c)
    assert omega == st.omega
    assert np.array_equal(tag, st.tag)
    assert np.array_equal(bc, st.bc)
    assert np.array_equal(zgb, st.zgb)
    assert np.array_equal(f, st.lat)


def test_errors_are_reported_not_raised_without_a_device():
    if lbgpu.lib().lbgpu_device_count() > 0:
        pytest.skip("a device is present")
    lbgpu.clear_error()
    with pytest.raises(lbgpu.LbError) as e:
        lbgpu.Lattice(8, 8)
    assert e.value.code == 8          # LB_ERR_NO_DEVICE
    assert lbgpu.last_error()[0] == 0  # the binding clears the error it raised
    with pytest.raises(lbgpu.LbError) as e:
        lbgpu.drive(20, 10, 5, 6, 2, 2, "origin")
    assert e.value.code == 8
    with pytest.raises(lbgpu.LbError) as e:
        lbgpu.Server("f32", 1 << 20, 100)
    assert e.value.code == 8


def test_bad_arguments_are_rejected():
    L = lbgpu.lib()
    lbgpu.clear_error()
    h = ctypes.c_void_p()
    assert L.lbgpu_create(0, 5, 0, 0, ctypes.byref(h)) == 3      # LB_ERR_ARG before any CUDA call
    assert lbgpu.last_error()[0] == 3 and "out of range" in lbgpu.last_error()[1]
    lbgpu.clear_error()
    assert L.lbgpu_create(8, 8, 9, 0, ctypes.byref(h)) == 3
    lbgpu.clear_error()
    # CUDA's 65535 grid rows bound ly (one grid row a lattice row, two ghost rows included)
    assert L.lbgpu_create(16, 65534, 0, 0, ctypes.byref(h)) == 3
    assert "65533" in lbgpu.last_error()[1]
    lbgpu.clear_error()
    assert L.lbgpu_create((1 << 20) + 1, 8, 0, 0, ctypes.byref(h)) == 3
    lbgpu.clear_error()
    with pytest.raises(lbgpu.LbError) as e:
        lbgpu.drive(-1, 10, 5, 6, 2, 2, "origin")
    assert e.value.code == 3
    lbgpu.clear_error()
    with pytest.raises(lbgpu.LbError) as e:
        lbgpu.drive(16, 65534, 5, 6, 2, 2, "origin", want_lattice=False)
    assert e.value.code == 3
    lbgpu.clear_error()
    s = ctypes.c_void_p()
    assert L.lbgpu_server_create(1, 1 << 20, 0, ctypes.byref(s)) == 3   # check interval 0
    assert L.lbgpu_server_create(7, 1 << 20, 100, ctypes.byref(s)) == 3  # no such precision
    lbgpu.clear_error()
    # the admission estimate is the sum of the lattice's allocations (two buffers vs one)
    pull = lbgpu.lattice_bytes(250, 51, "f32", "pull")
    aa = lbgpu.lattice_bytes(250, 51, "f32", "aa")
    assert pull > aa > 9 * 4 * 250 * 51


@pytest.mark.skipif(not O.ref_available(), reason="reference build oracle/_ref not present")
def test_reference_keeps_its_own_symbols_when_the_gpu_library_is_global():
    """The GPU library exports the reference's names; a process that loads it globally must
    still run the reference's own code (the reference libraries are linked -Bsymbolic)."""
    code = (
        "import ctypes, sys, json\n"
        f"sys.path[:0] = [{os.path.join(ROOT, 'oracle')!r}, {os.path.join(ROOT, 'tests')!r}]\n"
        f"ctypes.CDLL({lbgpu.LIB_PATH!r}, mode=ctypes.RTLD_GLOBAL)\n"
        "import oracle as O\n"
        "from helpers import check_golden\n"
        f"g = json.load(open({os.path.join(ROOT, 'tests', 'golden', 'golden.json')!r}))['cases']\n"
        "out = O.run_reference(O.Cylinder.reference_driver(64, 48), 'tight', 200)\n"
        "sys.exit(0 if check_golden(g['ref_driver_64x48_200'], out) else 1)\n")
    assert subprocess.run([sys.executable, "-c", code]).returncode == 0


def test_storage_names():
    """bench.py and the studies name storage forms; 's', 'b' and 'r' are 16-bit options only."""
    assert lbgpu.storage_form("f64") == ("f64", "", False)
    assert lbgpu.storage_form("f16s") == ("f16", "s", False)
    assert lbgpu.storage_form("bf16r") == ("bf16", "", True)
    assert lbgpu.storage_form("f16sr") == ("f16", "s", True)
    assert lbgpu.storage_form("f16br") == ("f16", "b", True)
    for bad in ("f32r", "f64s", "f32b", "f16rs", "f16sb", "fp16", ""):
        with pytest.raises(ValueError):
            lbgpu.storage_form(bad)


def test_banded_shift_profile():
    """Bands of SHIFT_BAND rows hold the inflow profile's value at their middle row; the ghost
    rows stay at rest, and consecutive rows inside a band share one shift velocity."""
    ly, umax = 300, 0.05
    exact = lbgpu.poiseuille_profile(ly, umax)
    band = lbgpu.banded_profile(ly, umax)
    assert band[0] == 0.0 and band[ly + 1] == 0.0
    b = lbgpu.SHIFT_BAND
    for y0 in range(1, ly + 1, b):
        y1 = min(ly, y0 + b - 1)
        assert np.all(band[y0:y1 + 1] == exact[(y0 + y1) // 2])
    assert np.max(np.abs(band - exact)) <= 4 * umax * (b / 2) / (ly - 1)


def test_stochastic_rounding_setter_rejects_a_null_lattice():
    """The setter validates its handle before touching a device (no GPU here)."""
    rc = lbgpu.lib().lbgpu_set_stochastic_rounding(None, 1, 0)
    assert rc != 0
    lbgpu.clear_error()
