"""frehg_gw_init_state_static against frehg_gw_init_state, through the C ABI.

The static entry point stages the caller's IC field in one array compiled
into the library instead of a per-call device allocation; both launch the
same initial-state kernel, so the states they leave must agree bit for bit.
Two calls in a row on one handle (a water-table raster, then a 3-D head
field) are each compared with the allocating entry point on a second handle,
followed by one step from each state.  A field above the array's capacity is
rejected with FREHG_GW_EINVAL.
"""
import ctypes as C

import numpy as np
import pytest

from frehg_b200 import gw as G
from frehg_b200 import workloads

pytestmark = pytest.mark.gpu

EINVAL = 1
IC_HEAD, IC_WATER_TABLE = 1, 2
STATIC_FIELD_MAX = 262144
_dp = C.POINTER(C.c_double)


def _lib():
    lib = G.load_library()
    lib.frehg_gw_init_state_static.argtypes = [C.c_void_p, C.c_int, C.c_double, _dp]
    lib.frehg_gw_init_state_static.restype = C.c_int
    lib.frehg_gw_last_error.restype = C.c_char_p
    return lib


def _state(s):
    return {name: s.field(name) for name in ("h", "wc", "wcn")}


def _init(lib, s, fn, form, arr):
    arr = np.ascontiguousarray(arr, np.float64)
    rc = getattr(lib, fn)(s.h, form, 0.0, arr.ctypes.data_as(_dp))
    assert rc == 0, lib.frehg_gw_last_error().decode()


def test_static_init_matches_allocating_init_two_calls():
    lib = _lib()
    cfg = workloads.hillslope(24, 20, 32, n_bumps=4)
    ref = G.RichardsSolver(cfg)
    new = G.RichardsSolver(cfg)
    rng = np.random.default_rng(7)
    bot = ref.field("bot3d")                                 # (ny, nx, nz) cell bottoms
    wt = bot[:, :, 0] - rng.uniform(0.2, 2.0, size=bot.shape[:2])
    head = rng.uniform(-3.0, 0.3, size=(cfg.domain.ny, cfg.domain.nx, cfg.domain.nz))
    for form, fld in ((IC_WATER_TABLE, wt), (IC_HEAD, head)):
        _init(lib, ref, "frehg_gw_init_state", form, fld)
        _init(lib, new, "frehg_gw_init_state_static", form, fld)
        a, b = _state(ref), _state(new)
        for name in a:
            np.testing.assert_array_equal(b[name], a[name], err_msg=name)
    dt = ref.nextDt()
    ref.step(dt, dt)
    new.step(dt, dt)
    for name in ("h", "wc", "qz"):
        np.testing.assert_array_equal(new.field(name), ref.field(name), err_msg=name)
    assert new.lastSolve()[0] == ref.lastSolve()[0]
    ref.close()
    new.close()


def test_static_init_rejects_fields_above_capacity():
    lib = _lib()
    cfg = workloads.column_32x32x50(nx=72, ny=64, nz=60)
    assert 72 * 64 * 60 > STATIC_FIELD_MAX
    s = G.RichardsSolver(cfg)
    big = np.full((64, 72, 60), -1.0)
    rc = lib.frehg_gw_init_state_static(s.h, IC_HEAD, 0.0, big.ctypes.data_as(_dp))
    assert rc == EINVAL
    assert b"at most 262144" in lib.frehg_gw_last_error()
    # The water-table raster of the same domain (72 x 64 values) fits.
    wt = np.full((64, 72), -0.5)
    _init(lib, s, "frehg_gw_init_state_static", IC_WATER_TABLE, wt)
    s.close()
