"""The 16-bit storage accuracy target: time-averaged velocity within 1e-3 (relative L2) of FP64.

A reduced channel in the regime of the precision workload: 4096 x 1024 (obstacle at
(nx/5+1, ny/2+1), radius ny/10+1, bounce-back walls, constant-density outlet), with the lattice
relaxation and inflow speed of the two configured cases -- omega ~ 1.0 at uMax 0.02 (Re 24.7
here, the configuration's Re 100 on its larger grid) and omega ~ 1.6 at uMax 0.05 (Re 247 here,
Re 1000 there) -- 20,000 steps, velocity averaged every 10 steps over the second half, against
the exact FP64 kernel on the same lattice.  At omega ~ 1 the channel sits deep in its slow
transient: per step a stored population changes by far less than half a quantum of its 16-bit
offset, so round-to-nearest storage stalls (asserted below, to show the case has teeth), while
stochastic rounding keeps the drift unbiased.

Measured on a B200 (relative L2 of the time-averaged velocity): omega 1.0: FP16 round-to-nearest
1.9e-2, FP16 stochastic 1.0e-4, FP16 row shift + stochastic 1.7e-4, FP32 2.1e-3; omega 1.6:
FP16 stochastic 6.6e-4, FP16 row shift + stochastic 2.1e-4, FP32 1.3e-3; the shift held
constant over bands of 64 rows ('b'), with stochastic rounding: 2.2e-4 (omega 1.0) and 3.2e-4
(omega 1.6).
"""
import numpy as np
import pytest

import lbgpu

pytestmark = pytest.mark.gpu

NX, NY, STEPS, EVERY = 4096, 1024, 20000, 10
CASES = {"omega1.0": (24.7, 0.02), "omega1.6": (247.0, 0.05)}


def averaged_velocity(storage, re, umax):
    base, shift, rs = lbgpu.storage_form(storage)
    with lbgpu.Lattice(NX, NY, base, "pull") as lat:
        lbgpu.configure_storage(lat, storage, umax, seed=20260101)
        lat.setup_cylinder(NX // 5 + 1, NY // 2 + 1, NY // 10 + 1, umax, re, lbgpu.WALL_BOUNCEBACK,
                           lbgpu.OUTLET_CONST)
        lat.step(STEPS // 2)
        for _ in range(STEPS // 2 // EVERY):
            lat.step(EVERY)
            lat.velocity_accumulate()
        ux, uy, n = lat.velocity_average()
        assert n == STEPS // 2 // EVERY
        assert lat.moments()[6] == 0
    return ux, uy


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2) /
                         np.sum(b[0] ** 2 + b[1] ** 2)))


_REF = {}


def reference(case):
    if case not in _REF:
        _REF[case] = averaged_velocity("f64", *CASES[case])
    return _REF[case]


@pytest.mark.parametrize("storage", ["f16sr", "f16br"])
@pytest.mark.parametrize("case", list(CASES))
def test_fp16_row_shift_stochastic_meets_1e3(case, storage):
    """Offsets from the inflow profile per row ('s') or per band of rows ('b')."""
    err = rel_l2(averaged_velocity(storage, *CASES[case]), reference(case))
    print(f"{case}: {storage} {err:.2e}")
    assert err <= 1e-3


def test_fp16_stochastic_meets_1e3_where_round_to_nearest_stalls():
    ref = reference("omega1.0")
    err_rs = rel_l2(averaged_velocity("f16r", *CASES["omega1.0"]), ref)
    err_rn = rel_l2(averaged_velocity("f16", *CASES["omega1.0"]), ref)
    print(f"omega 1.0: FP16 stochastic {err_rs:.2e}, round to nearest {err_rn:.2e}")
    assert err_rs <= 1e-3
    assert err_rn > 5e-3
