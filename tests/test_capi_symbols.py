"""The C ABI library loads without a GPU and exports every entry point that
include/polystring_b200.h declares; no compute call is made here."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "polystring_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ps_[A-Za-z0-9_]+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    from polystring_b200 import build
    build.build()
    from polystring_b200 import capi
    return capi.load()


def test_header_declares_entry_points():
    names = _declared()
    for must in ("ps_updater_create", "ps_updater_solve", "ps_density_solve", "ps_model_ab_create",
                 "ps_model_ab_update", "ps_model_ab_H", "ps_model_ab_residual", "ps_last_error"):
        assert must in names


def test_every_declared_symbol_is_exported(lib):
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(lib):
    from polystring_b200 import capi
    bound = {n for n, _, _ in capi.SIGNATURES}
    assert set(_declared()) <= bound | {"ps_version"}


def test_version_and_error_strings(lib):
    from polystring_b200 import capi
    assert b"sm_100a" in lib.ps_version()
    assert isinstance(lib.ps_last_error(), bytes)


def test_no_gpu_fails_loudly(lib):
    """Without a CUDA device a context cannot be created; the call returns a
    CUDA error status instead of computing anything on the host."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import polystring_b200 as ps
    with pytest.raises(ps.PSError) as e:
        ps.RQM4(ps.make_cell(1, "LAMELLAR", 4.0), 64, 1, 1, 0.01)
    assert e.value.code == -3


def test_invalid_arguments_rejected_before_any_device_work(lib):
    import polystring_b200 as ps
    from polystring_b200 import capi
    h = ctypes.c_void_p()
    cell = ps.make_cell(2, "SQUARE", 4.0)
    # 2D grid with Lz != 1
    rc = lib.ps_updater_create(0, ctypes.byref(cell), 32, 32, 4, 0.01, ctypes.byref(h))
    assert rc == capi.PS_ERR_INVALID
    # unknown scheme
    rc = lib.ps_updater_create(7, ctypes.byref(cell), 32, 32, 1, 0.01, ctypes.byref(h))
    assert rc == capi.PS_ERR_INVALID
    # null output handle
    rc = lib.ps_updater_create(0, ctypes.byref(cell), 32, 32, 1, 0.01, None)
    assert rc == capi.PS_ERR_INVALID


def test_newer_entry_points_check_arguments_first(lib):
    """Batch, adjoint, checkpointed stress and the no-allocation density
    reject bad arguments with a status before any device work."""
    import polystring_b200 as ps
    from polystring_b200 import capi
    h = ctypes.c_void_p()
    out = (ctypes.c_double * 3)()
    assert lib.ps_batch_ab_create(None, 2, ctypes.byref(h)) == capi.PS_ERR_INVALID
    p = ps._params(2, (32, 32, 1), ps.make_cell(2, "SQUARE", 4.0), (21, 31), 20.0)
    assert lib.ps_batch_ab_create(ctypes.byref(p), 0, ctypes.byref(h)) == capi.PS_ERR_INVALID
    assert lib.ps_batch_ab_update(None, 1) == capi.PS_ERR_INVALID
    assert lib.ps_batch_ab_H(None, 0, out, out, out) == capi.PS_ERR_INVALID
    assert lib.ps_model_ab_stress(None, out) == capi.PS_ERR_INVALID
    assert lib.ps_model_ab_stress_checkpointed(None, 0, out) == capi.PS_ERR_INVALID
    assert lib.ps_model_ab_forward(None) == capi.PS_ERR_INVALID
    assert lib.ps_model_ab_grad_w(None, out, out, 0.0, out, out) == capi.PS_ERR_INVALID
    # the no-allocation density: size limit and rule preconditions, pointers never touched
    dummy = ctypes.c_void_p(16)
    rc = lib.ps_density_solve_device_noalloc(0, dummy, dummy, capi.PS_DENSITY_NOALLOC_MAX_LEN + 1, 4, 0.01, 1.0,
                                             dummy, None)
    assert rc == capi.PS_ERR_INVALID and b"8192" in lib.ps_last_error()
    rc = lib.ps_density_solve_device_noalloc(1, dummy, dummy, 36, 4, 0.01, 1.0, dummy, None)   # Simpson, odd n
    assert rc == capi.PS_ERR_QUADRATURE
    assert isinstance(lib.ps_tuning_log(), bytes)
