"""C ABI host logic (no GPU needed): libdglm.so loads, exports every function
include/dglm.h declares, and rejects bad arguments with status codes before
touching a device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from exadglm_b200 import capi

HEADER = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include", "dglm.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(dglm_[A-Za-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = capi.lib()
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(capi.EXPORTS)


def test_abi_version_and_orders():
    L = capi.lib()
    assert L.dglm_abi_version() == 1
    assert all(L.dglm_order_supported(n) for n in range(1, 9))
    assert not L.dglm_order_supported(0) and not L.dglm_order_supported(9)


def test_variants_are_described():
    for phys in ("euler", "advection"):
        for N in range(1, 9):
            v = capi.variants(phys, N)
            assert len(v) >= 2
            assert all(d.startswith(("simt", "dmma", "pipe-dmma", "pipe2-dmma", "tcgen05-",
                                      "mma16-", "pipe-mma16-", "tc-tmem-")) for d in v)
            assert capi.variants(phys, N, "fp64")


def test_variant_shapes_are_unique_without_smem():
    # the tuned table matches variants by description with smem=<bytes> left out
    from exadglm_b200.tune import _shape
    for phys in ("euler", "advection"):
        for N in range(1, 9):
            shapes = [_shape(d) for d in capi.variants(phys, N)]
            assert len(set(shapes)) == len(shapes), (phys, N, shapes)


def _desc(**kw):
    d = capi.Desc()
    d.N, d.physics, d.K, d.precision = 4, capi.EULER, 48, capi.PREC_FP64
    d.cfl, d.gamma, d.tau_scale, d.tmax, d.device = 0.4, 1.4, 1.2, 1.0, 0
    for k, v in kw.items():
        setattr(d, k, v)
    return d


@pytest.mark.parametrize("kw,status", [
    ({"N": 0}, capi.ERR_UNSUPPORTED), ({"N": 9}, capi.ERR_UNSUPPORTED),
    ({"physics": 7}, capi.ERR_INVALID), ({"K": 0}, capi.ERR_INVALID),
    ({"cfl": -1.0}, capi.ERR_INVALID), ({"gamma": 1.0}, capi.ERR_INVALID),
    ({"tmax": 0.0}, capi.ERR_INVALID), ({"precision": 9}, capi.ERR_INVALID),
    ({"K": 2 ** 31 // 35 + 1}, capi.ERR_UNSUPPORTED),    # K*Np past the int32 node range
    # K*4*Nfp (face points, N=1: 12 per element) past the int32 range while K*Np is not
    ({"N": 1, "K": 2 ** 31 // 12 + 1}, capi.ERR_UNSUPPORTED),
])
def test_create_rejects_bad_descriptions(kw, status):
    L = capi.lib()
    h = C.c_void_p()
    assert L.dglm_create(C.byref(_desc(**kw)), C.byref(h)) == status
    assert not h.value
    assert L.dglm_last_error()


def test_null_arguments():
    L = capi.lib()
    assert L.dglm_create(None, None) == capi.ERR_INVALID
    assert L.dglm_step(None, 1) == capi.ERR_INVALID
    assert L.dglm_set_state(None, None, 0) == capi.ERR_INVALID
    assert L.dglm_set_time(None, 0.5, 3) == capi.ERR_INVALID
    assert L.dglm_run_ensemble(None, 1, None, None, 1, None) == capi.ERR_INVALID
    assert L.dglm_destroy(None) == capi.OK


def test_per_kernel_entry_points_validate_before_launch():
    L = capi.lib()
    null = C.c_void_p(0)
    # bad order / nvar / NULL pointers are rejected without a launch
    assert L.dglm_update_ub(0, 5, 10, null, null, null, null, null) == capi.ERR_INVALID
    assert L.dglm_update_ub(4, 3, 10, null, null, null, null, null) == capi.ERR_INVALID
    assert L.dglm_lserk_stage(4, 5, 10, 0.1, 0.0, 0.1, null, null, null, null) == capi.ERR_INVALID
    assert L.dglm_update_rhs(4, 5, 10, null, null, null, null, b"x", null, null, null, null,
                             null, null) == capi.ERR_INVALID
    assert L.dglm_calc_dt(4, 0, 0.4, null, null, null) == capi.ERR_INVALID


def test_library_fails_loudly_when_missing(monkeypatch):
    monkeypatch.setattr(capi, "LIB_PATH", "/nonexistent/libdglm.so")
    monkeypatch.setattr(capi, "_lib", None)
    with pytest.raises(RuntimeError, match="missing"):
        capi.lib()


def test_handles_close_once_in_with_blocks():
    """Solver and BatchSolver release their handle on leaving a with block,
    once, also when the block raises (checked with a fake library)."""
    calls = []

    class FakeLib:
        def dglm_destroy(self, h):
            calls.append(("solver", h))

        def dglm_batch_destroy(self, h):
            calls.append(("batch", h))

    for cls, tag in ((capi.Solver, "solver"), (capi.BatchSolver, "batch")):
        obj = cls.__new__(cls)
        obj.L, obj.h = FakeLib(), 1234
        with pytest.raises(RuntimeError):
            with obj as o:
                assert o is obj
                raise RuntimeError("inside")
        obj.close()
        assert calls.count((tag, 1234)) == 1 and obj.h is None


def test_every_tuned_entry_resolves_to_its_variant(monkeypatch):
    """Each entry of tuned.json names a compiled variant (matched by shape,
    shared-memory size left out), so no pick silently falls back to variant 0
    after a variant list or description changes."""
    from exadglm_b200 import tune
    table = tune.load_cache()
    assert table, "tuned.json is empty"
    for key, ent in table.items():
        dev, physics, order, prec = key.split("|")
        monkeypatch.setattr(tune, "_device_name", lambda device=0, d=dev: d)
        v = tune.cached_variant(physics, int(order[1:]), prec)
        assert v is not None, (key, ent["desc"])
        desc = capi.variants(physics, int(order[1:]))[v]
        assert tune._shape(desc) == tune._shape(ent["desc"]), key
        assert capi.variant_precision(desc) == prec, (key, desc)
