"""TEST INFRASTRUCTURE ONLY: ctypes access to the CPU oracle and to the reference build.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs import
this module.  It loads

* ``oracle/liboracle.so`` -- this repository's C restatement of the reference step
  (``lbm_oracle.c``), and
* ``oracle/_ref/libref_lb_{serial,omp}.so`` -- the reference's own ``lb.c`` and
  ``boundaries.c`` compiled unmodified (``oracle/Makefile``) and driven by
  ``ref_harness.c``.

Arrays use the reference's own node order: ``f[X, Y, i]`` for X = 0..lx+1, Y = 0..ly+1
(ghost ring included) and the reference's direction order (lb.c:48-55).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

WALL_REGULARIZED, WALL_BOUNCEBACK = 0, 1
OUTLET_ZGB, OUTLET_CONST = 0, 1
VARIANTS = {"origin": 0, "combine": 1, "tight": 2, "tight_block": 3, "panel": 4}

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


@dataclass(frozen=True)
class Cylinder:
    """A cylinder-channel scenario, in the reference's 1-based node coordinates."""

    lx: int
    ly: int
    obst_x: int
    obst_y: int
    obst_r: int
    umax: float = 0.02
    re: float = 100.0
    wall: int = WALL_REGULARIZED
    outlet: int = OUTLET_ZGB

    @classmethod
    def reference_driver(cls, lx, ly):
        """The application driver's own scenario (unsteady.c:96-103, :162-214)."""
        return cls(lx, ly, lx // 4, ly // 2, ly // 10 + 1, 0.02, 100.0,
                   WALL_REGULARIZED, OUTLET_ZGB)

    @classmethod
    def baseline(cls, nx, ny, umax=0.02, re=100.0):
        """Bounce-back walls, constant-density outlet, obstacle at (nx/5+1, ny/2+1)."""
        return cls(nx, ny, nx // 5 + 1, ny // 2 + 1, ny // 10 + 1, umax, re,
                   WALL_BOUNCEBACK, OUTLET_CONST)


def _lib(path):
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
    return ctypes.CDLL(path)


_ORACLE = None


def oracle_lib():
    global _ORACLE
    if _ORACLE is None:
        lib = _lib(os.path.join(HERE, "liboracle.so"))
        lib.orc_run.restype = ctypes.c_int
        lib.orc_run.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _u8p, _dp, _u8p,
                                _dp, _dp, ctypes.c_int]
        lib.orc_build_cylinder.restype = ctypes.c_double
        lib.orc_build_cylinder.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 2 + [
            ctypes.c_int, ctypes.c_int, _u8p, _dp, _u8p, _dp, _dp]
        lib.orc_macros.argtypes = [_dp, _dp, _dp, _dp]
        lib.orc_equilibrium.restype = ctypes.c_double
        lib.orc_equilibrium.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4
        lib.orc_collide_node.argtypes = [ctypes.c_int, _dp, ctypes.c_double, _dp]
        lib.orc_init_equilibrium.argtypes = [_dp] + [ctypes.c_double] * 3
        lib.orc_moments.argtypes = [ctypes.c_int, ctypes.c_int, _u8p, _dp, _dp]
        _ORACLE = lib
    return _ORACLE


class OracleState:
    """Tags, boundary tables, outlet flags and both population buffers of one lattice."""

    def __init__(self, lx, ly, omega, tag, bc, zgb, lat, tmp):
        self.lx, self.ly, self.omega = lx, ly, omega
        self.tag, self.bc, self.zgb, self.lat, self.tmp = tag, bc, zgb, lat, tmp

    def copy(self):
        return OracleState(self.lx, self.ly, self.omega, self.tag.copy(), self.bc.copy(),
                           self.zgb.copy(), self.lat.copy(), self.tmp.copy())

    @property
    def nb(self):
        return max(self.lx, self.ly) + 2


def build_cylinder(c: Cylinder) -> OracleState:
    lib = oracle_lib()
    n = (c.lx + 2) * (c.ly + 2)
    nb = max(c.lx, c.ly) + 2
    tag = np.zeros(n, np.uint8)
    bc = np.zeros(16 * nb, np.float64)
    zgb = np.zeros(c.ly + 2, np.uint8)
    lat = np.zeros(n * 9, np.float64)
    tmp = np.zeros(n * 9, np.float64)
    omega = lib.orc_build_cylinder(c.lx, c.ly, c.obst_x, c.obst_y, c.obst_r, c.umax, c.re,
                                   c.wall, c.outlet, _ptr(tag, _u8p), _ptr(bc),
                                   _ptr(zgb, _u8p), _ptr(lat), _ptr(tmp))
    return OracleState(c.lx, c.ly, omega, tag.reshape(c.lx + 2, c.ly + 2), bc, zgb,
                       lat.reshape(c.lx + 2, c.ly + 2, 9), tmp.reshape(c.lx + 2, c.ly + 2, 9))


def run(state: OracleState, nsteps: int) -> OracleState:
    """Advance a copy of `state` by `nsteps` reference steps (origin semantics)."""
    s = state.copy()
    tag = np.ascontiguousarray(s.tag.reshape(-1))
    lat = np.ascontiguousarray(s.lat.reshape(-1))
    tmp = np.ascontiguousarray(s.tmp.reshape(-1))
    rc = oracle_lib().orc_run(s.lx, s.ly, s.omega, _ptr(tag, _u8p), _ptr(s.bc),
                              _ptr(s.zgb, _u8p), _ptr(lat), _ptr(tmp), int(nsteps))
    if rc != 0:
        raise RuntimeError("oracle: an interior node has no dynamics")
    s.lat = lat.reshape(s.lx + 2, s.ly + 2, 9)
    s.tmp = tmp.reshape(s.lx + 2, s.ly + 2, 9)
    return s


# --------------------------------------------------------------------------------------
# The reference itself (oracle/_ref), built from the reference sources by oracle/Makefile.
# --------------------------------------------------------------------------------------
_REF = {}


def ref_available(openmp=False):
    name = "libref_lb_omp.so" if openmp else "libref_lb_serial.so"
    return os.path.exists(os.path.join(REF_DIR, name))


def ref_lib(openmp=False):
    key = bool(openmp)
    if key not in _REF:
        lib = _lib(os.path.join(REF_DIR, "libref_lb_omp.so" if openmp else "libref_lb_serial.so"))
        lib.ref_setup.restype = ctypes.c_double
        lib.ref_setup.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 2 + [ctypes.c_int] * 3
        lib.ref_run.restype = ctypes.c_int
        lib.ref_run.argtypes = [ctypes.c_int] * 3
        lib.ref_dump.argtypes = [ctypes.c_int, _dp]
        lib.ref_set_blocking.argtypes = [ctypes.c_int] * 3
        lib.ref_outlet_state.argtypes = [_dp, _dp, _dp]
        lib.ref_max_threads.restype = ctypes.c_int
        lib.ref_setup_custom.restype = ctypes.c_int
        lib.ref_setup_custom.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _u8p, _dp,
                                         _u8p, _dp, _dp]
        _REF[key] = lib
    return _REF[key]


def ref_setup(c: Cylinder, poison=False, openmp=False, blk=1, tblock=1, nthreads=0):
    lib = ref_lib(openmp)
    omega = lib.ref_setup(c.lx, c.ly, c.obst_x, c.obst_y, c.obst_r, c.umax, c.re, c.wall,
                          c.outlet, 1 if poison else 0)
    lib.ref_set_blocking(blk, tblock, nthreads)
    return omega


def ref_step(variant, nsteps, openmp=False):
    return ref_lib(openmp).ref_run(VARIANTS[variant], 1 if openmp else 0, int(nsteps))


def ref_dump(c: Cylinder, which=0, openmp=False):
    out = np.zeros((c.lx + 2) * (c.ly + 2) * 9, np.float64)
    ref_lib(openmp).ref_dump(which, _ptr(out))
    return out.reshape(c.lx + 2, c.ly + 2, 9)


def ref_outlet_state(c: Cylinder, openmp=False):
    p = np.zeros(c.ly + 2)
    r1 = np.zeros(c.ly + 2)
    r2 = np.zeros(c.ly + 2)
    ref_lib(openmp).ref_outlet_state(_ptr(p), _ptr(r1), _ptr(r2))
    return p, r1, r2


def run_reference(c: Cylinder, variant: str, nsteps: int, poison=False, openmp=False,
                  blk=1, tblock=1, nthreads=0):
    """Final `lattice` of the reference after `nsteps` steps of `variant`."""
    ref_setup(c, poison=poison, openmp=openmp, blk=blk, tblock=tblock, nthreads=nthreads)
    ref_step(variant, nsteps, openmp=openmp)
    return ref_dump(c, 0, openmp=openmp)


def run_reference_custom(state: OracleState, variant: str, nsteps: int, blk=1):
    """The reference on an arbitrary tag/table lattice (ref_setup_custom): final lattice."""
    lib = ref_lib(False)
    tag = np.ascontiguousarray(state.tag.reshape(-1))
    lat = np.ascontiguousarray(state.lat.reshape(-1))
    tmp = np.ascontiguousarray(state.tmp.reshape(-1))
    bc = np.ascontiguousarray(state.bc)
    zgb = np.ascontiguousarray(state.zgb)
    lib.ref_setup_custom(state.lx, state.ly, state.omega, _ptr(tag, _u8p), _ptr(bc),
                         _ptr(zgb, _u8p), _ptr(lat), _ptr(tmp))
    lib.ref_set_blocking(blk, 1, 0)
    lib.ref_run(VARIANTS[variant], 0, int(nsteps))
    out = np.zeros(lat.size, np.float64)
    lib.ref_dump(0, _ptr(out))
    return out.reshape(state.lx + 2, state.ly + 2, 9)


def random_boundary_lattice(lx, ly, seed, omega=1.6, kinds="mixed"):
    """A small lattice whose perimeter carries every boundary kind of boundaries.h.

    Interior nodes are BGK with a few bounce-back cells; each side gets a cycle of the
    velocity/pressure Zou/He and regularized kinds of that side, so each of the 17 boundary
    functions appears.  Populations start near equilibrium with a seeded perturbation, and
    the second buffer gets seeded values too (its ghost-sourced slots feed the first step).
    """
    rng = np.random.default_rng(seed)
    n2 = (lx + 2, ly + 2)
    nb = max(lx, ly) + 2
    tag = np.zeros(n2, np.uint8)
    tag[1:lx + 1, 1:ly + 1] = 1
    inner = rng.random((lx, ly)) < 0.08
    tag[1:lx + 1, 1:ly + 1][inner] = 2
    side_kinds = {0: [3, 7, 11, 15], 1: [4, 8, 12, 16], 2: [5, 9, 13, 17], 3: [6, 10, 14, 18]}
    for X in range(1, lx + 1):
        tag[X, ly] = side_kinds[0][X % 4]
        tag[X, 1] = side_kinds[1][(X + 1) % 4]
    for Y in range(2, ly):
        tag[1, Y] = side_kinds[2][Y % 4]
        tag[lx, Y] = side_kinds[3][(Y + 2) % 4]
    bc = np.zeros((8, 2, nb))
    bc[0:4, 0, :] = rng.uniform(-0.03, 0.03, (4, nb))   # velocity ux
    bc[0:4, 1, :] = rng.uniform(-0.03, 0.03, (4, nb))   # velocity uy
    bc[4:8, 0, :] = rng.uniform(0.97, 1.03, (4, nb))    # pressure rho
    bc[4:8, 1, :] = rng.uniform(-0.02, 0.02, (4, nb))   # pressure uPar
    lib = oracle_lib()
    lat = np.zeros(n2 + (9,))
    tmp = np.zeros(n2 + (9,))
    for X in range(lx + 2):
        for Y in range(ly + 2):
            f = np.zeros(9)
            lib.orc_init_equilibrium(_ptr(f), 1.0 + rng.uniform(-0.02, 0.02),
                                     rng.uniform(-0.04, 0.04), rng.uniform(-0.04, 0.04))
            lat[X, Y] = f * (1 + rng.uniform(-0.01, 0.01, 9))
            tmp[X, Y] = f * (1 + rng.uniform(-0.01, 0.01, 9))
    zgb = np.zeros(ly + 2, np.uint8)
    return OracleState(lx, ly, omega, tag, bc.reshape(-1), zgb, lat, tmp)


def moments(state: OracleState):
    """orc_moments of a state: mass, jx, jy, Fx, Fy, kinetic energy, non-finite nodes, bulk mass."""
    tag = np.ascontiguousarray(state.tag.reshape(-1), np.uint8)
    lat = np.ascontiguousarray(state.lat.reshape(-1))
    out = np.zeros(8)
    oracle_lib().orc_moments(state.lx, state.ly, _ptr(tag, _u8p), _ptr(lat), _ptr(out))
    return out
