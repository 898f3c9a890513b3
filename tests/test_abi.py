"""The C-ABI library: loads, exports every declared symbol, matches the
header's struct layout, and validates parameters — all without a GPU."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

from conftest import ROOT
from fluid_step import _abi

HEADER = os.path.join(ROOT, "include", "fluid_step.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^FE_API [^;(]*?\b(fe_\w+)\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    import __graft_entry__  # noqa: F401  (path setup)
    from build import build
    build()
    return _abi.load_library()


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    # and the Python mirror declares a signature for each
    assert set(names) == set(_abi.SIGNATURES), set(names) ^ set(_abi.SIGNATURES)


def test_contraction_build_exports_the_same_abi(lib):
    c = _abi.load_library(build="contract")
    assert c is not lib
    for n in declared_functions():
        assert hasattr(c, n), n
    assert c.fe_abi_version() == _abi.ABI_VERSION
    with pytest.raises(ValueError):
        _abi.load_library(build="fast")


def test_struct_layout_matches_header(lib):
    fields_p = [f for f, _ in _abi.FeParams._fields_]
    fields_s = [f for f, _ in _abi.FeStats._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           'printf("%zu %zu\\n", sizeof(fe_params), sizeof(fe_stats));']
    for f in fields_p:
        src.append(f'printf("p {f} %zu\\n", offsetof(fe_params, {f}));')
    for f in fields_s:
        src.append(f'printf("s {f} %zu\\n", offsetof(fe_stats, {f}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "probe")
        subprocess.run(["gcc", "-o", exe, c], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    sp, ss = map(int, out[0].split())
    assert sp == ctypes.sizeof(_abi.FeParams) and ss == ctypes.sizeof(_abi.FeStats)
    for line in out[1:]:
        if not line:
            continue
        kind, name, off = line.split()
        cls = _abi.FeParams if kind == "p" else _abi.FeStats
        assert getattr(cls, name).offset == int(off), name


def test_default_params_match(lib):
    a = _abi.FeParams()
    lib.fe_default_params(ctypes.byref(a))
    b = _abi.default_params()
    assert bytes(a) == bytes(b)
    assert lib.fe_validate_params(ctypes.byref(a)) == _abi.FE_OK


@pytest.mark.parametrize("field,value,status", [
    ("smoothing_radius", 0.0, _abi.FE_ERR_INVALID_ARGUMENT),
    ("particle_mass", -1.0, _abi.FE_ERR_INVALID_ARGUMENT),
    ("dt", float("nan"), _abi.FE_ERR_INVALID_ARGUMENT),
    ("sort_algorithm", 7, _abi.FE_ERR_INVALID_ARGUMENT),
    ("mode", 5, _abi.FE_ERR_INVALID_ARGUMENT),
])
def test_validate_rejects(lib, field, value, status):
    p = _abi.default_params()
    setattr(p, field, value)
    assert lib.fe_validate_params(ctypes.byref(p)) == status
    assert lib.fe_last_error()


def test_validate_box_and_tolerance(lib):
    p = _abi.default_params()
    p.box_min[1] = 5.0
    assert lib.fe_validate_params(ctypes.byref(p)) == _abi.FE_ERR_INVALID_ARGUMENT
    p = _abi.default_params()
    p.solver = _abi.FE_SOLVER_TOLERANCE
    p.max_iterations = 0
    assert lib.fe_validate_params(ctypes.byref(p)) == _abi.FE_ERR_INVALID_ARGUMENT
    p = _abi.default_params()
    p.reserved[0] = 1
    assert lib.fe_validate_params(ctypes.byref(p)) == _abi.FE_ERR_INVALID_ARGUMENT


def test_null_and_status_strings(lib):
    assert lib.fe_destroy(None) == _abi.FE_OK
    assert lib.fe_prepare(None) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_neighbor_search(None) == _abi.FE_ERR_INVALID_ARGUMENT
    for code, name in _abi.STATUS_NAMES.items():
        assert lib.fe_status_string(code).decode() == name
    assert lib.fe_abi_version() == _abi.ABI_VERSION


def test_create_rejects_bad_input_before_device(lib):
    p = _abi.default_params()
    pos = (ctypes.c_float * 3)(0.0, float("nan"), 0.0)
    h = ctypes.c_void_p()
    assert lib.fe_create(ctypes.byref(p), 1, pos, None, 0, ctypes.byref(h)) == _abi.FE_ERR_NON_FINITE
    assert lib.fe_create(ctypes.byref(p), 0, pos, None, 0, ctypes.byref(h)) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_create(ctypes.byref(p), 1, None, None, 0, ctypes.byref(h)) == _abi.FE_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("cls,cname", [(_abi.FeTuning, "fe_tuning"),
                                       (_abi.FeTuneReport, "fe_tune_report")])
def test_tuning_struct_layout_matches_header(cls, cname):
    fields = [f for f, _ in cls._fields_]
    src = ["#include <stdio.h>", "#include <stddef.h>", f'#include "{HEADER}"', "int main(void){",
           f'printf("%zu\\n", sizeof({cname}));']
    for f in fields:
        src.append(f'printf("{f} %zu\\n", offsetof({cname}, {f}));')
    src.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        open(c, "w").write("\n".join(src))
        exe = os.path.join(d, "probe")
        subprocess.run(["gcc", "-o", exe, c], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    assert int(out[0]) == ctypes.sizeof(cls)
    for line in out[1:]:
        if line:
            name, off = line.split()
            assert getattr(cls, name).offset == int(off), name


def test_sort_config_rejects_non_candidates(lib):
    # shape validation happens before any device work
    assert lib.fe_sort_pairs_config(None, None, 0, 32, 9, 8, None) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_sort_pairs_config(None, None, 0, 32, 8, 5, None) == _abi.FE_ERR_INVALID_ARGUMENT


def test_state_calls_reject_null(lib):
    size = ctypes.c_size_t()
    assert lib.fe_state_size(None, ctypes.byref(size)) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_state_export(None, None, 0) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_state_import(None, None, 0) == _abi.FE_ERR_INVALID_ARGUMENT


def test_debug_hooks_validate_before_device_work(lib):
    flags = ctypes.c_uint32()
    assert lib.fe_debug_bounded_wait(0, 0, ctypes.byref(flags)) == _abi.FE_ERR_INVALID_ARGUMENT
    assert lib.fe_debug_bounded_wait(0, 10, None) == _abi.FE_ERR_INVALID_ARGUMENT
    lib.fe_debug_fail_allocation(0)
    lib.fe_debug_poison_allocations(0)


def test_header_constants_match_the_python_mirror():
    text = open(HEADER).read()
    for name, value in [("FE_STATE_VERSION", _abi.FE_STATE_VERSION),
                        ("FE_ABI_VERSION", _abi.ABI_VERSION),
                        ("FE_MAX_PARTICLES", None)]:
        m = re.search(rf"#define {name} \(?([0-9]+)u?(?: << ([0-9]+))?\)?", text)
        assert m, name
        v = int(m.group(1)) << int(m.group(2) or 0)
        if value is not None:
            assert v == value, (name, v, value)
