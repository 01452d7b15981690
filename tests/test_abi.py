"""The C-ABI library on CPU: it loads, exports every entry point include/wenofv.h declares,
and rejects invalid options before touching a GPU (no compute calls here)."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    src = open(os.path.join(ROOT, "include", "wenofv.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(wenofv_[a-z_0-9]+)\s*\(", src)))


def test_header_and_binding_agree(wb):
    assert sorted(wb.EXPORTS) == declared_functions()


def test_library_exports_every_symbol(wb):
    L = wb.load()
    for name in declared_functions():
        assert hasattr(L, name), name
    assert L.wenofv_abi_version() == 2


def test_struct_layouts(wb):
    # wenofv_eq_params: int (+4 pad) + 13 doubles; wenofv_config: 2 ints, 4 doubles, 2 ints,
    # double, 7 ints (+4 pad)
    assert C.sizeof(wb.EqParams) == 112
    assert C.sizeof(wb.Config) == 88


def test_default_config_is_shipped_settings(wb):
    L = wb.load()
    c = wb.Config()
    L.wenofv_default_config(C.byref(c))
    assert (c.nx, c.ny, c.rk_method, c.cfl, c.scheme, c.pp_limiter, c.riemann_flux, c.reconstruction) == \
        (100, 100, 2, 0.5, 1, 0, 0, 1)


@pytest.mark.parametrize("field,value,code", [
    ("nx", 0, 1), ("rk_method", 3, 1), ("cfl", 0.0, 1), ("scheme", 3, 1), ("reconstruction", 5, 6), ("reconstruction", 6, 1),
    ("riemann_flux", 4, 1), ("bc", -1, 6), ("bc", 7, 6), ("precision", 9, 1), ("ref_slabs", 3, 1),
])
def test_invalid_options_rejected(wb, field, value, code):
    L = wb.load()
    c = wb.make_config(32, 32)
    setattr(c, field, value)
    h = C.c_void_p()
    rc = L.wenofv_create(C.byref(c), C.byref(wb.make_eq()), C.byref(h))
    assert rc == code and not h.value
    assert L.wenofv_last_error()


def test_invalid_equation_rejected(wb):
    L = wb.load()
    h = C.c_void_p()
    assert L.wenofv_create(C.byref(wb.make_config(8, 8)), C.byref(wb.make_eq(kind=7)), C.byref(h)) == wb.EINVAL
    assert L.wenofv_create(C.byref(wb.make_config(8, 8)), C.byref(wb.make_eq(sound1=0.0)), C.byref(h)) == wb.EINVAL
    assert L.wenofv_create(C.byref(wb.make_config(8, 8)), C.byref(wb.make_eq(kind=2, gamma=1.0)), C.byref(h)) == wb.EINVAL
    # primitive variables are defined for the two-phase model only
    assert L.wenofv_create(C.byref(wb.make_config(8, 8, recon=2)), C.byref(wb.make_eq(kind=2)), C.byref(h)) == wb.ENOTSUP
    # WENOEXP and PRIMITIVE3 have no FP32-bulk form; PRIMITIVE3 is two-phase only
    c = wb.make_config(8, 8, scheme=2, precision=wb.FP32_BULK)
    assert L.wenofv_create(C.byref(c), C.byref(wb.make_eq()), C.byref(h)) == wb.ENOTSUP
    c = wb.make_config(8, 8, recon=4, precision=wb.FP32_BULK)
    assert L.wenofv_create(C.byref(c), C.byref(wb.make_eq()), C.byref(h)) == wb.ENOTSUP
    assert L.wenofv_create(C.byref(wb.make_config(8, 8, recon=4)), C.byref(wb.make_eq(kind=2)), C.byref(h)) == wb.ENOTSUP
    # the stiffened-gas model: FP64 forms, RECONSTRUCTIONTYPE 0-1, valid phase parameters
    sg = wb.make_eq(kind=wb.EQ_TWO_PHASE_SG, rho10=1000.0, rho20=1.0, preb=1.0)
    assert L.wenofv_create(C.byref(wb.make_config(8, 8, precision=wb.FP32_BULK)), C.byref(sg), C.byref(h)) == wb.ENOTSUP
    assert L.wenofv_create(C.byref(wb.make_config(8, 8, recon=3)), C.byref(sg), C.byref(h)) == wb.ENOTSUP
    bad = wb.make_eq(kind=wb.EQ_TWO_PHASE_SG, rho10=1000.0, rho20=1.0, preb=1.0, gamma2=1.0)
    assert L.wenofv_create(C.byref(wb.make_config(8, 8)), C.byref(bad), C.byref(h)) == wb.EINVAL


def test_null_arguments(wb):
    L = wb.load()
    assert L.wenofv_create(None, None, None) == wb.EINVAL
    assert L.wenofv_upload(None, None, 0) == wb.EINVAL
    assert L.wenofv_step(None, 0.1) == wb.EINVAL
    L.wenofv_destroy(None)
    assert L.wenofv_strerror(wb.ENUMERIC)
