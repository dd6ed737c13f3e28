"""CPU tests of the C ABI boundary: libtps.so loads, exports every entry point
declared in include/tps.h with the struct layouts the Python binding assumes,
and rejects invalid input with a status code and message (no GPU compute)."""
import ctypes
import os
import re
import shutil
import subprocess

import pytest

from gputensorproductsmoother_b200 import _lib as L

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(REPO, "include", "tps.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tps_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == {s[0] for s in L.SIGNATURES}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc missing")
def test_struct_layouts_match_ctypes(tmp_path):
    prog = tmp_path / "sz.c"
    prog.write_text('#include "tps.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                    'int main(void){printf("%zu %zu %zu %zu %zu\\n", sizeof(tps_problem),'
                    ' sizeof(tps_solve_opts), sizeof(tps_report), offsetof(tps_report, history),'
                    ' offsetof(tps_report, time_ms)); return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(prog), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert out == [ctypes.sizeof(L.TpsProblem), ctypes.sizeof(L.TpsSolveOpts),
                   ctypes.sizeof(L.TpsReport), L.TpsReport.history.offset, L.TpsReport.time_ms.offset]


@pytest.mark.parametrize("field,value,status", [("dim", 4, 1), ("degree", 9, 7), ("n_coarse", 1, 1),
                                                ("n_levels", 0, 1), ("relaxation", 0.0, 1)])
def test_create_rejects_invalid_problem(field, value, status):
    pb = L.TpsProblem(3, 2, 2, 3, 1.0, None, 0)
    setattr(pb, field, value)
    h = ctypes.c_void_p()
    st = L.lib().tps_create(ctypes.byref(pb), ctypes.byref(h))
    assert st == status
    assert not h.value
    assert L.lib().tps_last_error(None)


def test_null_arguments_are_rejected():
    lib = L.lib()
    assert lib.tps_create(None, None) == 1
    assert lib.tps_destroy(None) == 1
    assert lib.tps_laplace_vmult(None, 0, 0, None, None, None) == 1
    assert lib.tps_smoother_step(None, 0, 0, None, None, 0, 0, None) == 1
    assert lib.tps_level_info(None, 0, None, None) == 1
    assert lib.tps_device_status(None) == 1
    assert lib.tps_selftest_wait_timeout(None, 1000, None) == 1
    assert lib.tps_solve_host_many(None, None, 1, None, None, None) == 1


def test_alloc_failure_hook_arms_and_disarms():
    """The allocation-failure hook is host state only: arming and disarming
    it needs no device, and a negative count disarms it."""
    lib = L.lib()
    lib.tps_inject_alloc_failure(3)
    lib.tps_inject_alloc_failure(-1)
    lib.tps_inject_alloc_failure(0)
    assert L.STATUS_NAMES[8] == "TPS_ERR_TIMEOUT"


def test_create_without_device_fails_loudly():
    """On a host without a GPU a valid problem must fail with a CUDA status
    (there is no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pb = L.TpsProblem(3, 2, 2, 3, 1.0, None, 0)
    h = ctypes.c_void_p()
    st = L.lib().tps_create(ctypes.byref(pb), ctypes.byref(h))
    assert st == 2 and not h.value
    assert "cuda" in L.lib().tps_last_error(None).decode().lower()


def test_solve_opts_default():
    o = L.TpsSolveOpts()
    L.lib().tps_solve_opts_default(ctypes.byref(o))
    assert (o.driver, o.precision, o.symmetric, o.max_iter, o.use_graph) == (0, 1, 1, 100, 1)
    assert o.rel_tol == 1e-10


def test_noalloc_entry_rejects_bad_sizes_before_any_device_work():
    """tps_restrict_add_noalloc validates its arguments on the host first:
    scratch overflow in 3D, and in 2D fine levels beyond 2^31-1 DoFs per
    direction or coarse-cell tiles beyond the launch grid's y limit."""
    lib = L.lib()
    buf = ctypes.c_double()
    p = ctypes.addressof(buf)
    assert lib.tps_restrict_add_noalloc(3, 4, 64, L.TPS_F64, p, p, None) == 1
    assert b"scratch" in lib.tps_last_error(None)
    assert lib.tps_restrict_add_noalloc(2, 4, 2_000_000_000, L.TPS_F64, p, p, None) == 1
    assert b"2^31" in lib.tps_last_error(None)
    assert lib.tps_restrict_add_noalloc(2, 2, 600_000, L.TPS_F64, p, p, None) == 1
    assert b"grid" in lib.tps_last_error(None)
    assert lib.tps_restrict_add_noalloc(4, 2, 4, L.TPS_F64, p, p, None) == 1
    assert lib.tps_restrict_add_noalloc(3, 2, 4, L.TPS_F64, None, p, None) == 1
