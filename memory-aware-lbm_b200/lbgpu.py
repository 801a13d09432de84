"""ctypes binding of liblbgpu.so (include/lb.h, include/lbgpu.h, include/lbdriver.h).

Host-side plumbing for tests and benchmarks: every call goes through the library's C ABI and
every step runs the library's sm_100a kernels.  There is no Python or CPU fallback; if the
shared library is missing, importing its functions raises.

Arrays use the reference's node order: f[X, Y, i] for X = 0..lx+1, Y = 0..ly+1 (ghost ring
included), direction order of the reference (lb.c:48-55).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liblbgpu.so")
INCLUDE_DIR = os.path.join(os.path.dirname(HERE), "include")

PRECISIONS = {"f64": 0, "f32": 1, "f16": 2, "bf16": 3}
SCHEMES = {"pull": 0, "aa": 1}
BYTES_PER_UPDATE = {"f64": 144, "f32": 72, "f16": 36, "bf16": 36}
WALL_REGULARIZED, WALL_BOUNCEBACK = 0, 1
OUTLET_ZGB, OUTLET_CONST = 0, 1
VARIANTS = {"origin": 0, "combine": 1, "tight": 2, "tight_block": 3, "panel": 4}
SYNC = {"none": 0, "outlet": 1, "full": 2}

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_vp = ctypes.c_void_p


class LbError(RuntimeError):
    """A library call returned an LB_ERR_* code."""

    def __init__(self, code, message):
        super().__init__(f"liblbgpu error {code}: {message}")
        self.code = code


class DriverConfig(ctypes.Structure):
    _fields_ = [("lx", ctypes.c_int), ("ly", ctypes.c_int), ("obst_x", ctypes.c_int),
                ("obst_y", ctypes.c_int), ("obst_r", ctypes.c_int), ("umax", ctypes.c_double),
                ("re", ctypes.c_double), ("wall", ctypes.c_int), ("outlet", ctypes.c_int),
                ("variant", ctypes.c_int), ("blk", ctypes.c_int), ("sync_mode", ctypes.c_int)]


class Request(ctypes.Structure):
    _fields_ = [("lx", ctypes.c_int), ("ly", ctypes.c_int), ("obst_x", ctypes.c_int),
                ("obst_y", ctypes.c_int), ("obst_r", ctypes.c_int), ("umax", ctypes.c_double),
                ("re", ctypes.c_double), ("max_steps", ctypes.c_int), ("tol", ctypes.c_double),
                ("arrival", ctypes.c_double), ("want_fields", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("arrival", ctypes.c_double), ("admit", ctypes.c_double),
                ("finish", ctypes.c_double), ("steps", ctypes.c_longlong),
                ("nodes", ctypes.c_longlong), ("converged", ctypes.c_int),
                ("done", ctypes.c_int), ("last_change", ctypes.c_double), ("solo", ctypes.c_int)]


_LIB = None


def lib():
    """Load liblbgpu.so (raises FileNotFoundError when it is not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is not built: run `make -C memory-aware-lbm_b200`")
    # RTLD_LOCAL: the library exports the reference's symbol names (collide, bgk, ...); they must
    # not take the place of the reference's own definitions in libraries loaded later
    L = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
    L.lbGetLastError.restype = ctypes.c_int
    L.lbGetLastErrorString.restype = ctypes.c_char_p
    L.lbgpu_set_device.argtypes = [ctypes.c_int]
    L.lbgpu_device_count.restype = ctypes.c_int
    L.lbgpu_create.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(_vp)]
    L.lbgpu_destroy.argtypes = [_vp]
    L.lbgpu_set_geometry.argtypes = [_vp, ctypes.c_double, _u8p, _dp, _u8p]
    L.lbgpu_set_populations.argtypes = [_vp, _dp, _dp]
    L.lbgpu_set_offset_scale.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_set_offset_shift.argtypes = [_vp, _dp]
    L.lbgpu_set_stochastic_rounding.argtypes = [_vp, ctypes.c_int, ctypes.c_uint]
    L.lbgpu_setup_cylinder.argtypes = [_vp] + [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [
        ctypes.c_int] * 2 + [_dp]
    L.lbgpu_build_cylinder.restype = ctypes.c_double
    L.lbgpu_build_cylinder.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 2 + [
        ctypes.c_int] * 2 + [_u8p, _dp, _u8p, _dp]
    L.lbgpu_step.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_set_sweep_steps.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_step_timed.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.lbgpu_get_populations.argtypes = [_vp, _dp]
    L.lbgpu_get_macros.argtypes = [_vp, _dp, _dp, _dp]
    L.lbgpu_get_macros_noalloc.argtypes = [_vp, _dp, _dp, _dp]
    L.lbgpu_moments.argtypes = [_vp, _dp]
    L.lbgpu_velocity_accumulate.argtypes = [_vp]
    L.lbgpu_velocity_average.argtypes = [_vp, _dp, _dp, ctypes.POINTER(ctypes.c_longlong)]
    L.lbgpu_velocity_reset.argtypes = [_vp]
    L.lbgpu_synchronize.argtypes = [_vp]
    L.lbgpu_batch_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
    L.lbgpu_batch_destroy.argtypes = [_vp]
    L.lbgpu_batch_add.argtypes = [_vp, _vp, ctypes.POINTER(ctypes.c_int)]
    L.lbgpu_batch_remove.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_batch_size.argtypes = [_vp]
    L.lbgpu_batch_step.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_batch_step_timed.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.lbgpu_batch_synchronize.argtypes = [_vp]
    L.lbgpu_batch_last_launches.argtypes = [_vp]
    L.lbgpu_batch_size_class.argtypes = [ctypes.c_longlong]
    L.lbgpu_batch_set_shape.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.lbgpu_batch_get_shape.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                        ctypes.POINTER(ctypes.c_int)]
    L.lbgpu_batch_set_passes.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.lbgpu_batch_get_passes.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_batch_set_persistent.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_batch_get_persistent.argtypes = [_vp]
    L.lbgpu_batch_set_threads.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_batch_get_threads.argtypes = [_vp]
    L.lbgpu_batch_autotune.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    L.lbgpu_tune_scheme.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_int),
                                                         ctypes.POINTER(ctypes.c_float),
                                                         ctypes.POINTER(ctypes.c_float)]
    L.lbgpu_lattice_bytes.restype = ctypes.c_size_t
    L.lbgpu_lattice_bytes.argtypes = [ctypes.c_int] * 4
    L.lbgpu_server_create.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.c_int,
                                      ctypes.POINTER(_vp)]
    L.lbgpu_server_destroy.argtypes = [_vp]
    L.lbgpu_server_set_scheme.argtypes = [_vp, ctypes.c_int, ctypes.c_int]
    L.lbgpu_server_set_shape.argtypes = [_vp] + [ctypes.c_int] * 3
    L.lbgpu_server_set_persistent.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_set_threads.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_set_solo_nodes.argtypes = [_vp, ctypes.c_longlong]
    L.lbgpu_server_set_offset_shift.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_set_stochastic_rounding.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_set_offset_scale.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_submit.argtypes = [_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int)]
    L.lbgpu_server_run.argtypes = [_vp, ctypes.c_int]
    L.lbgpu_server_result.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(Result), _dp, _dp]
    L.lbgpu_server_stats.argtypes = [_vp, _dp]
    L.lbgpu_stream.restype = _vp
    L.lbgpu_stream.argtypes = [_vp]
    L.lbgpu_steps_done.restype = ctypes.c_longlong
    L.lbgpu_steps_done.argtypes = [_vp]
    L.lbgpu_device_bytes.restype = ctypes.c_size_t
    L.lbgpu_device_bytes.argtypes = [_vp]
    L.lbgpu_last_kernel_launches.argtypes = [_vp]
    L.lbdrv_run.argtypes = [ctypes.POINTER(DriverConfig), ctypes.c_int, _dp,
                            ctypes.POINTER(ctypes.c_double)]
    L.lbdrv_last_transfer_bytes.argtypes = [ctypes.POINTER(ctypes.c_ulonglong)] * 2
    L.computeMacros.argtypes = [_dp, _dp, _dp, _dp]
    L.computeEquilibrium.restype = ctypes.c_double
    L.computeEquilibrium.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4
    _LIB = L
    return L


def last_error():
    L = lib()
    return L.lbGetLastError(), (L.lbGetLastErrorString() or b"").decode()


def clear_error():
    lib().lbClearError()


def _check(rc):
    if rc != 0:
        code, msg = last_error()
        clear_error()
        raise LbError(rc, msg)


def _p(a, t=_dp):
    return a.ctypes.data_as(t)


def build_cylinder(lx, ly, obst_x, obst_y, obst_r, umax=0.02, re=100.0, wall=WALL_REGULARIZED,
                   outlet=OUTLET_ZGB, populations=True):
    """Host arrays of the cylinder channel: (omega, tag[X,Y], bc, zgb_row, f[X,Y,9] or None)."""
    n2 = (lx + 2) * (ly + 2)
    nb = max(lx, ly) + 2
    tag = np.zeros(n2, np.uint8)
    bc = np.zeros(16 * nb)
    zgb = np.zeros(ly + 2, np.uint8)
    f = np.zeros(n2 * 9) if populations else None
    omega = lib().lbgpu_build_cylinder(lx, ly, obst_x, obst_y, obst_r, umax, re, wall, outlet,
                                       _p(tag, _u8p), _p(bc), _p(zgb, _u8p),
                                       _p(f) if f is not None else None)
    return (omega, tag.reshape(lx + 2, ly + 2), bc, zgb,
            f.reshape(lx + 2, ly + 2, 9) if f is not None else None)


class Lattice:
    """A device lattice (lbgpu_lattice): FP64/FP32/FP16/BF16 storage, pull or AA kernel."""

    def __init__(self, lx, ly, precision="f64", scheme="pull"):
        self.lx, self.ly, self.precision, self.scheme = lx, ly, precision, scheme
        h = _vp()
        _check(lib().lbgpu_create(lx, ly, PRECISIONS[precision], SCHEMES[scheme], ctypes.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().lbgpu_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_geometry(self, omega, tag, bc, zgb=None):
        tag = np.ascontiguousarray(tag, np.uint8).reshape(-1)
        bc = np.ascontiguousarray(bc, np.float64).reshape(-1)
        z = None if zgb is None else np.ascontiguousarray(zgb, np.uint8)
        _check(lib().lbgpu_set_geometry(self.h, float(omega), _p(tag, _u8p), _p(bc),
                                        None if z is None else _p(z, _u8p)))

    def set_populations(self, f, tmp=None):
        f = np.ascontiguousarray(f, np.float64).reshape(-1)
        t = None if tmp is None else np.ascontiguousarray(tmp, np.float64).reshape(-1)
        _check(lib().lbgpu_set_populations(self.h, _p(f), None if t is None else _p(t)))

    def set_offset_scale(self, scale_log2):
        _check(lib().lbgpu_set_offset_scale(self.h, int(scale_log2)))

    def set_offset_shift(self, u_row):
        """Per-row shift velocity of FP16/BF16 offsets (ly + 2 values), or None for w_i."""
        if u_row is None:
            _check(lib().lbgpu_set_offset_shift(self.h, None))
            return
        u = np.ascontiguousarray(u_row, np.float64)
        if u.shape != (self.ly + 2,):
            raise ValueError(f"shift profile needs {self.ly + 2} values")
        _check(lib().lbgpu_set_offset_shift(self.h, _p(u)))

    def set_stochastic_rounding(self, on=True, seed=0):
        """FP16/BF16 storage: round stored values stochastically (seeded, deterministic)."""
        _check(lib().lbgpu_set_stochastic_rounding(self.h, 1 if on else 0, int(seed) & 0xffffffff))

    def setup_cylinder(self, obst_x, obst_y, obst_r, umax=0.02, re=100.0, wall=WALL_REGULARIZED,
                       outlet=OUTLET_ZGB):
        om = ctypes.c_double()
        _check(lib().lbgpu_setup_cylinder(self.h, obst_x, obst_y, obst_r, umax, re, wall, outlet,
                                          ctypes.byref(om)))
        return om.value

    def set_sweep_steps(self, steps):
        """1, or 2 for two pull steps per sweep (temporal blocking)."""
        _check(lib().lbgpu_set_sweep_steps(self.h, int(steps)))

    def step(self, n):
        _check(lib().lbgpu_step(self.h, int(n)))

    def step_timed(self, n):
        ms = ctypes.c_float()
        _check(lib().lbgpu_step_timed(self.h, int(n), ctypes.byref(ms)))
        return ms.value

    def synchronize(self):
        _check(lib().lbgpu_synchronize(self.h))

    def populations(self):
        out = np.zeros((self.lx + 2) * (self.ly + 2) * 9)
        _check(lib().lbgpu_get_populations(self.h, _p(out)))
        return out.reshape(self.lx + 2, self.ly + 2, 9)

    def macros(self):
        n = self.lx * self.ly
        rho, ux, uy = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(lib().lbgpu_get_macros(self.h, _p(rho), _p(ux), _p(uy)))
        shp = (self.ly, self.lx)
        return rho.reshape(shp), ux.reshape(shp), uy.reshape(shp)

    def macros_noalloc(self):
        """lbgpu_get_macros_noalloc: the same read-out through the library's fixed scratch."""
        n = self.lx * self.ly
        rho, ux, uy = np.zeros(n), np.zeros(n), np.zeros(n)
        _check(lib().lbgpu_get_macros_noalloc(self.h, _p(rho), _p(ux), _p(uy)))
        shp = (self.ly, self.lx)
        return rho.reshape(shp), ux.reshape(shp), uy.reshape(shp)

    def moments(self):
        """FP64 sums: mass, jx, jy, Fx, Fy, kinetic energy, non-finite nodes, bulk mass."""
        out = np.zeros(8)
        _check(lib().lbgpu_moments(self.h, _p(out)))
        return out

    def velocity_accumulate(self):
        _check(lib().lbgpu_velocity_accumulate(self.h))

    def velocity_average(self):
        n = self.lx * self.ly
        ux, uy = np.zeros(n), np.zeros(n)
        k = ctypes.c_longlong()
        _check(lib().lbgpu_velocity_average(self.h, _p(ux), _p(uy), ctypes.byref(k)))
        return ux.reshape(self.ly, self.lx), uy.reshape(self.ly, self.lx), k.value

    def velocity_reset(self):
        _check(lib().lbgpu_velocity_reset(self.h))

    @property
    def stream(self):
        return lib().lbgpu_stream(self.h)

    @property
    def steps_done(self):
        return lib().lbgpu_steps_done(self.h)

    @property
    def device_bytes(self):
        return lib().lbgpu_device_bytes(self.h)

    @property
    def last_launches(self):
        return lib().lbgpu_last_kernel_launches(self.h)


DEFAULT_SCALE = {"f16": 10, "bf16": 6}
# With a row shift the stored deviations are far smaller (down to ~1e-7 of f in a smooth far
# field) while at most ~0.03: 2^17 keeps FP16 out of its subnormal range with a 15x margin below
# its largest value.  BF16 has FP32's exponent range, so its scale does not matter.
DEFAULT_SHIFT_SCALE = {"f16": 17, "bf16": 6}


def poiseuille_profile(ly, umax):
    """The cylinder channel's inflow profile per row Y = 0..ly+1 (0 in the ghost rows): the
    natural per-row shift of 16-bit offsets for that channel (lbgpu_set_offset_shift)."""
    u = np.zeros(ly + 2)
    L = ly - 1.0
    y = np.arange(ly, dtype=np.float64)
    u[1:ly + 1] = 4.0 * umax / (L * L) * (L * y - y * y)
    return u


SHIFT_BAND = 64


def banded_profile(ly, umax, band=SHIFT_BAND):
    """The inflow profile held constant over bands of `band` rows (each band takes the value of
    its middle row; 0 in the ghost rows).  Offsets streamed between two rows of one band need no
    rebase, so only the rows at a band's edge pay for it; with bands of 64 rows the stored
    offsets stay nearly as small as with the exact profile."""
    exact = poiseuille_profile(ly, umax)
    u = exact.copy()
    for y0 in range(1, ly + 1, band):
        y1 = min(ly, y0 + band - 1)
        u[y0:y1 + 1] = exact[(y0 + y1) // 2]
    return u


def storage_form(name):
    """Storage names: 'f64', 'f32', 'f16', 'bf16', and for the 16-bit types the suffixes 's'
    (offsets from the channel's inflow-profile equilibrium per row, lbgpu_set_offset_shift) or
    'b' (the same profile held constant over bands of SHIFT_BAND rows, banded_profile), and 'r'
    (stochastic rounding, lbgpu_set_stochastic_rounding), e.g. 'f16sr', 'f16br'.
    Returns (precision, shift, stochastic) with shift '' (none), 's' or 'b'."""
    import re
    m = re.fullmatch(r"(f64|f32|f16|bf16)([sb]?)(r?)", name)
    if not m or (m.group(1) in ("f64", "f32") and (m.group(2) or m.group(3))):
        raise ValueError(f"storage {name!r}")
    return m.group(1), m.group(2), bool(m.group(3))


def shift_profile(kind, ly, umax):
    """The per-row shift velocities of a storage's shift kind ('s' or 'b')."""
    return banded_profile(ly, umax) if kind == "b" else poiseuille_profile(ly, umax)


def configure_storage(lat, name, umax, seed=0):
    """Offset scale, row shift (the inflow profile of peak umax, exact or banded) and rounding of
    a storage name, applied before the initial state is written."""
    base, shift, rs = storage_form(name)
    if base in DEFAULT_SCALE:
        lat.set_offset_scale((DEFAULT_SHIFT_SCALE if shift else DEFAULT_SCALE)[base])
    if shift:
        lat.set_offset_shift(shift_profile(shift, lat.ly, umax))
    if rs:
        lat.set_stochastic_rounding(True, seed)


def cylinder_lattice(lx, ly, precision="f64", scheme="pull", umax=0.02, re=100.0,
                     wall=WALL_BOUNCEBACK, outlet=OUTLET_CONST, obst=None, scale=None):
    """A device lattice holding the channel (obstacle default (lx/5+1, ly/2+1), r = ly/10+1).
    16-bit storage uses the offset scale 2^scale (default DEFAULT_SCALE)."""
    ox, oy, r = obst if obst is not None else (lx // 5 + 1, ly // 2 + 1, ly // 10 + 1)
    lat = Lattice(lx, ly, precision, scheme)
    if precision in DEFAULT_SCALE:
        lat.set_offset_scale(DEFAULT_SCALE[precision] if scale is None else scale)
    lat.omega = lat.setup_cylinder(ox, oy, r, umax, re, wall, outlet)
    return lat


def drive(lx, ly, obst_x, obst_y, obst_r, nsteps, variant="origin", umax=0.02, re=100.0,
          wall=WALL_REGULARIZED, outlet=OUTLET_ZGB, blk=1, sync="outlet", want_lattice=True):
    """Run the C host driver (include/lbdriver.h) on the drop-in interface.

    Returns (final lattice f[X,Y,9] or None, steps run, loop wall seconds)."""
    cfg = DriverConfig(lx, ly, obst_x, obst_y, obst_r, umax, re, wall, outlet, VARIANTS[variant],
                       blk, SYNC[sync] if isinstance(sync, str) else int(sync))
    out = np.zeros((lx + 2) * (ly + 2) * 9) if want_lattice else None
    secs = ctypes.c_double()
    done = lib().lbdrv_run(ctypes.byref(cfg), int(nsteps), None if out is None else _p(out),
                           ctypes.byref(secs))
    if done < 0:
        code, msg = last_error()
        clear_error()
        raise LbError(-done, msg)
    return (out.reshape(lx + 2, ly + 2, 9) if out is not None else None), done, secs.value


def drive_transfer_bytes():
    """(host->device, device->host) bytes the calling thread's last drive() copied."""
    a, b = ctypes.c_ulonglong(), ctypes.c_ulonglong()
    lib().lbdrv_last_transfer_bytes(ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def declared_functions():
    """Names of the functions declared in include/*.h (the C ABI this library exports)."""
    import re
    names = set()
    pat = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_ ]*[\s\*]+([A-Za-z_][A-Za-z0-9_]*)\s*\(")
    for fn in sorted(os.listdir(INCLUDE_DIR)):
        if not fn.endswith(".h"):
            continue
        with open(os.path.join(INCLUDE_DIR, fn)) as fh:
            text = fh.read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for line in text.splitlines():
            if line.strip().startswith(("#", "typedef", "//", "return")):
                continue
            m = pat.match(line)
            if m and m.group(1) not in ("if", "for", "while", "switch"):
                names.add(m.group(1))
    return sorted(names)


class Batch:
    """lbgpu_batch: many lattices of one precision stepped together (one launch per step)."""

    def __init__(self, precision="f32"):
        self.precision = precision
        h = _vp()
        _check(lib().lbgpu_batch_create(PRECISIONS[precision], ctypes.byref(h)))
        self.h = h
        self.members = {}

    def close(self):
        if self.h:
            lib().lbgpu_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def add(self, lat):
        slot = ctypes.c_int()
        _check(lib().lbgpu_batch_add(self.h, lat.h, ctypes.byref(slot)))
        self.members[slot.value] = lat
        return slot.value

    def remove(self, slot):
        _check(lib().lbgpu_batch_remove(self.h, int(slot)))
        self.members.pop(slot, None)

    def __len__(self):
        return lib().lbgpu_batch_size(self.h)

    def step(self, n):
        _check(lib().lbgpu_batch_step(self.h, int(n)))

    def step_timed(self, n):
        ms = ctypes.c_float()
        _check(lib().lbgpu_batch_step_timed(self.h, int(n), ctypes.byref(ms)))
        return ms.value

    def synchronize(self):
        _check(lib().lbgpu_batch_synchronize(self.h))

    @property
    def last_launches(self):
        return lib().lbgpu_batch_last_launches(self.h)

    def set_shape(self, size_class, tile_width, nodes_per_thread=1):
        _check(lib().lbgpu_batch_set_shape(self.h, size_class, tile_width, nodes_per_thread))

    def shape(self, size_class):
        """(tile width, nodes per thread) of a size class."""
        w, n = ctypes.c_int(), ctypes.c_int()
        _check(lib().lbgpu_batch_get_shape(self.h, size_class, ctypes.byref(w), ctypes.byref(n)))
        return w.value, n.value

    def set_passes(self, size_class, passes):
        """Tiles of a size class one block steps down a member (the strip length)."""
        _check(lib().lbgpu_batch_set_passes(self.h, int(size_class), int(passes)))

    def passes(self, size_class):
        return lib().lbgpu_batch_get_passes(self.h, int(size_class))

    @property
    def persistent(self):
        return bool(lib().lbgpu_batch_get_persistent(self.h))

    @persistent.setter
    def persistent(self, on):
        _check(lib().lbgpu_batch_set_persistent(self.h, int(bool(on))))

    @property
    def threads(self):
        """Threads per tile (= nodes per tile)."""
        return lib().lbgpu_batch_get_threads(self.h)

    @threads.setter
    def threads(self, n):
        _check(lib().lbgpu_batch_set_threads(self.h, int(n)))

    def autotune(self, steps=4):
        best = (ctypes.c_float * 6)()
        _check(lib().lbgpu_batch_autotune(self.h, int(steps), best))
        return list(best)


def size_class(nodes):
    return lib().lbgpu_batch_size_class(int(nodes))


def tune_scheme(precision, lx, ly, steps=10):
    """(scheme name, ms pull, ms aa) for a channel of lx x ly."""
    s, a, b = ctypes.c_int(), ctypes.c_float(), ctypes.c_float()
    _check(lib().lbgpu_tune_scheme(PRECISIONS[precision], lx, ly, steps, ctypes.byref(s),
                                   ctypes.byref(a), ctypes.byref(b)))
    return ("aa" if s.value == 1 else "pull"), a.value, b.value


def lattice_bytes(lx, ly, precision="f32", scheme="pull"):
    return lib().lbgpu_lattice_bytes(lx, ly, PRECISIONS[precision], SCHEMES[scheme])


class Server:
    """lbgpu_server: continuous batching of cylinder-channel requests under an HBM budget."""

    def __init__(self, precision="f32", budget_bytes=8 << 30, check_every=100, scale=None,
                 shift=False, stochastic=False):
        self.precision = precision
        h = _vp()
        _check(lib().lbgpu_server_create(PRECISIONS[precision], int(budget_bytes),
                                         int(check_every), ctypes.byref(h)))
        self.h = h
        self.requests = []
        if precision in DEFAULT_SCALE:
            default = (DEFAULT_SHIFT_SCALE if shift else DEFAULT_SCALE)[precision]
            _check(lib().lbgpu_server_set_offset_scale(h, default if scale is None else int(scale)))
            if shift:
                _check(lib().lbgpu_server_set_offset_shift(h, 1))
            if stochastic:
                _check(lib().lbgpu_server_set_stochastic_rounding(h, 1))

    def close(self):
        if self.h:
            lib().lbgpu_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_scheme(self, size_class, scheme):
        _check(lib().lbgpu_server_set_scheme(self.h, int(size_class), SCHEMES[scheme]))

    def set_shape(self, size_class, tile_width, nodes_per_thread=1):
        _check(lib().lbgpu_server_set_shape(self.h, int(size_class), int(tile_width),
                                            int(nodes_per_thread)))

    def set_persistent(self, on):
        _check(lib().lbgpu_server_set_persistent(self.h, int(bool(on))))

    def set_threads(self, n):
        _check(lib().lbgpu_server_set_threads(self.h, int(n)))

    def set_solo_nodes(self, nodes):
        """Requests of at least this many nodes step on their own (0: batch every request)."""
        _check(lib().lbgpu_server_set_solo_nodes(self.h, int(nodes)))

    def submit(self, lx, ly, obst_x, obst_y, obst_r, umax, re, max_steps, tol=0.0, arrival=0.0,
               want_fields=False):
        r = Request(lx, ly, obst_x, obst_y, obst_r, umax, re, max_steps, tol, arrival,
                    int(want_fields))
        i = ctypes.c_int()
        _check(lib().lbgpu_server_submit(self.h, ctypes.byref(r), ctypes.byref(i)))
        self.requests.append(r)
        return i.value

    def run(self, batched=True):
        _check(lib().lbgpu_server_run(self.h, int(bool(batched))))

    def result(self, rid, fields=False):
        """dict of the request's record; with fields=True also (ux, uy) arrays [Y, X]."""
        res = Result()
        r = self.requests[rid]
        ux = uy = None
        if fields:
            ux = np.zeros((r.ly, r.lx))
            uy = np.zeros((r.ly, r.lx))
        _check(lib().lbgpu_server_result(self.h, int(rid), ctypes.byref(res),
                                         None if ux is None else _p(ux),
                                         None if uy is None else _p(uy)))
        out = {k: getattr(res, k) for k, _ in Result._fields_}
        if fields:
            out["ux"], out["uy"] = ux, uy
        return out

    def stats(self):
        o = (ctypes.c_double * 4)()
        _check(lib().lbgpu_server_stats(self.h, o))
        return {"makespan_s": o[0], "lattice_updates": o[1], "peak_resident": int(o[2]),
                "peak_bytes": int(o[3])}
