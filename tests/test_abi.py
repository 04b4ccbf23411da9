"""The C ABI surface: the product library loads, exports every entry point
include/hc_abi.h declares, and rejects bad options before touching a GPU.
No compute call is made here."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "hc_abi.h")


def declared_functions() -> list[str]:
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(hc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("hc_ctx_create", "hc_box_rhs", "hc_level_rk4_step", "hc_level_dt_cfl", "hc_level_valid"):
        assert must in names


def test_library_exports_every_declared_symbol(product_lib_path):
    lib = C.CDLL(product_lib_path)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header(product_lib_path):
    from heliocubed_b200 import _native
    assert set(declared_functions()) == set(_native.SIGNATURES)


def test_struct_layouts_match_header(product_lib_path):
    from heliocubed_b200 import _native
    # 16 ints + 16 doubles, 8 ints, 8 ints + 11 doubles (see hc_abi.h)
    assert C.sizeof(_native.HcParams) == 16 * 4 + 14 * 8 + 0 * 8 or C.sizeof(_native.HcParams) == 64 + 112
    assert C.sizeof(_native.HcBox) == 8 * 4
    assert C.sizeof(_native.HcInit) == 8 * 4 + 11 * 8
    assert C.sizeof(_native.HcBoxWork) == 8 * 4 + 5 * 8


@pytest.mark.parametrize("fields,code", [
    ({"spatial_order": 3}, -3), ({"limiter": 7}, -1), ({"riemann_solver": 3}, -1),
    ({"temporal_order": 2}, -3), ({"nr": 2}, -1), ({"gamma": 1.0}, -1), ({"init_condition_type": 0}, -3),
    ({"spatial_order": 4, "spatial_operator": 1}, -3), ({"spatial_order": 4, "berta_detector_type": 1}, -3),
    ({"spatial_order": 4, "berta_fallback_type": 2}, -1), ({"spatial_order": 4}, -1),  # na = 8 < 16
    # 48 (nr + 12)(na + 12)^2 >= 2^31: the level kernels index in 32 bits
    ({"nr": 4096, "na": 1024}, -1),
    # radial slabs: an offset needs a shell, and the slab must lie inside it
    ({"radial_offset": 2}, -1), ({"radial_offset": 30, "radial_cells": 36}, -1),
    ({"radial_offset": -1, "radial_cells": 36}, -1), ({"radial_cells": -4}, -1),
])
def test_bad_options_rejected(product_lib_path, fields, code):
    from heliocubed_b200 import _native
    from heliocubed_b200.level import Params
    p = Params(nr=8, na=8).to_c()
    for field, value in fields.items():
        setattr(p, field, value)
    ctx = C.c_void_p()
    rc = _native.lib().hc_ctx_create(C.byref(p), 0, C.byref(ctx))
    assert rc == code
    assert not ctx
    assert _native.lib().hc_last_error()


def test_no_device_is_an_error_not_a_fallback(product_lib_path):
    if gpu_available():
        pytest.skip("a GPU is present")
    from heliocubed_b200 import HcError, Params, Shell
    with pytest.raises(HcError):
        Shell(Params(nr=8, na=8))


def _c_name(cls_name: str) -> str:
    """HcCfFineBox -> hc_cf_fine_box."""
    return "hc" + re.sub(r"([A-Z])", lambda m: "_" + m.group(1).lower(), cls_name[2:])


def test_every_struct_layout_matches_the_compiler(tmp_path):
    """Sizes and field offsets of every ctypes mirror against what the C
    compiler lays out for the header's structs (gcc on the host)."""
    import shutil
    import subprocess
    from heliocubed_b200 import _native
    if shutil.which("gcc") is None:
        pytest.skip("no host C compiler")
    mirrors = [getattr(_native, n) for n in dir(_native)
               if n.startswith("Hc") and isinstance(getattr(_native, n), type)
               and issubclass(getattr(_native, n), C.Structure)]
    assert len(mirrors) >= 12
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    expect = []
    for cls in mirrors:
        cname = _c_name(cls.__name__)
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append(C.sizeof(cls))
        for field, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {field}));')
            expect.append(getattr(cls, field).offset)
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got == expect


def test_stage_entries_refuse_bad_arguments_on_the_host(product_lib_path):
    """The per-stage step, its stage buffer and the radial window refuse a
    null context or arguments with HC_ERR_ARG before touching a device."""
    from heliocubed_b200 import _native
    lib = _native.lib()
    data, rows, n, first = C.c_void_p(), C.c_long(), C.c_int(), C.c_int()
    assert lib.hc_level_rk4_stage(None, None, 0, 1.0, 0.0, None, None, None) == -1
    assert lib.hc_level_stage_state(None, None, 0, C.byref(data), C.byref(rows), C.byref(n), C.byref(first)) == -1
    assert lib.hc_level_set_radial_window(None, 0, 0) == -1
    assert lib.hc_last_error()
