"""The C ABI library loads and exports every entry point include/*.h
declares (no compute calls: this runs without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "frehg_b200", "libfrehg_gw.so")


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(frehg_gw_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_entry_points():
    names = declared_symbols()
    for required in ("frehg_gw_create", "frehg_gw_step", "frehg_gw_destroy",
                     "frehg_gw_get_field", "frehg_gw_next_dt", "frehg_gw_owned_volume"):
        assert required in names


@pytest.mark.skipif(not os.path.exists(LIB), reason="libfrehg_gw.so not built")
def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="libfrehg_gw.so not built")
def test_descriptor_layout_matches_header():
    # The ctypes mirror must agree with the C struct: compile-free check on
    # field order by name.
    from frehg_b200.abi import GwDesc, StepInfo
    text = open(os.path.join(ROOT, "include", "frehg_gw.h")).read()
    body = text[text.index("typedef struct frehg_gw_desc"):text.index("} frehg_gw_desc;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    decl = re.findall(r"(\*?\s*\w+)\s*[,;]", body.split("{", 1)[1])
    names = [d.replace("*", "").strip() for d in decl]
    assert names == [f[0] for f in GwDesc._fields_]
    body = text[text.index("typedef struct frehg_gw_step_info"):text.index("} frehg_gw_step_info;")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = [d.strip() for d in re.findall(r"(\w+)\s*;", body)]
    assert names == [f[0] for f in StepInfo._fields_]


def test_null_arguments_are_rejected_without_a_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    lib = ctypes.CDLL(LIB)
    lib.frehg_gw_create.restype = ctypes.c_int
    assert lib.frehg_gw_create(None, None) == 1  # FREHG_GW_EINVAL
    lib.frehg_gw_last_error.restype = ctypes.c_char_p
    assert b"null" in lib.frehg_gw_last_error()


def test_batch_create_rejects_bad_arguments_without_a_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    lib = ctypes.CDLL(LIB)
    lib.frehg_gw_batch_create.restype = ctypes.c_int
    out = ctypes.c_void_p()
    assert lib.frehg_gw_batch_create(None, 0, None, ctypes.byref(out)) == 1  # FREHG_GW_EINVAL
    members = (ctypes.c_void_p * 1)(None)
    assert lib.frehg_gw_batch_create(members, 1, None, ctypes.byref(out)) == 1
    assert out.value is None


def test_server_queues_and_rejects_oversized_requests_without_a_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    from frehg_b200 import workloads
    from frehg_b200.gw import FatalError
    from frehg_b200.serve import FAILED, QUEUED, PreparedRequest, RichardsServer
    req = PreparedRequest(workloads.column_32x32x50(nx=4, ny=4, nz=20), 3)
    need = req.device_bytes()
    assert need > 6 * 6 * 20 * 8 * 40  # at least 40 doubles per halo cell
    with RichardsServer(hbm_budget_bytes=need - 1) as srv:
        with pytest.raises(FatalError) as e:
            srv.submit(req)
        assert e.value.status == 3  # FREHG_GW_ENOMEM
    with RichardsServer(hbm_budget_bytes=need * 4) as srv:
        rid = srv.submit(req)
        # The server's worker thread admits queued requests on its own; without
        # a GPU that admission fails, so the request is queued until the worker
        # reaches it and failed afterwards -- never lost, never running.
        st = srv.poll(rid)
        assert st["steps"] == 3
        assert st["state"] in (QUEUED, FAILED)
        if st["state"] == QUEUED:
            assert st["queue_s"] == -1.0
        s = srv.stats()
        assert s["active"] == 0 and s["queued"] + s["completed"] == 1


def test_restore_rejects_bad_arguments_without_a_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    lib = ctypes.CDLL(LIB)
    lib.frehg_gw_restore.restype = ctypes.c_int
    lib.frehg_gw_restore.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_double]
    assert lib.frehg_gw_restore(None, None, None, None, 1.0) == 1  # FREHG_GW_EINVAL


def test_device_ordinal_of_a_null_handle_without_a_gpu():
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    lib = ctypes.CDLL(LIB)
    lib.frehg_gw_device.restype = ctypes.c_int
    lib.frehg_gw_device.argtypes = [ctypes.c_void_p]
    assert lib.frehg_gw_device(None) == -1


def test_soil_storage_shares_equal_arrays_and_keeps_uniform_fields_as_one_value():
    """A soil field uniform over the domain takes no cell array on the
    device, and equal ksx / ksy / ksz arrays are stored once: the estimate
    of the domain's device memory counts only the arrays it keeps (to the
    2 MiB page the arena rounds to)."""
    if not os.path.exists(LIB):
        pytest.skip("libfrehg_gw.so not built")
    import numpy as np

    from frehg_b200 import workloads
    from frehg_b200.serve import PreparedRequest
    nx, ny, nz = 64, 48, 96
    rng = np.random.default_rng(7)
    ks = np.exp(rng.normal(np.log(1e-5), 1.0, (ny, nx, nz)))
    alpha = rng.uniform(0.5, 3.0, (ny, nx, nz))
    vgn = rng.uniform(1.4, 2.5, (ny, nx, nz))

    def need(cell_soil):
        cfg = workloads.column_32x32x50(nx=nx, ny=ny, nz=nz)
        cfg.cell_soil = cell_soil
        return PreparedRequest(cfg, 1).device_bytes()

    array = ((nx + 2) * (ny + 2) * nz * 8 + 255) // 256 * 256
    uniform = need(None)  # every soil field uniform: no soil array
    iso = need(dict(ksx=ks, ksy=ks.copy(), ksz=ks, vg_alpha=alpha, vg_n=vgn))  # 3 arrays
    aniso = need(dict(ksx=ks, ksy=2.0 * ks, ksz=ks, vg_alpha=alpha, vg_n=vgn))  # 4 arrays
    assert abs((iso - uniform) - 3 * array) <= 2 << 20, (iso - uniform, array)
    assert abs((aniso - iso) - array) <= 2 << 20, (aniso - iso, array)
