"""The C-ABI library loads and exports every entry point include/mkb200.h declares."""
import os
import re
import subprocess

import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "mkb200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:[A-Za-z_][\w ]*[\s\*]+)(mk_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "mk_create_from_xml" in names and "mk_advance" in names and "mk_write_vtk" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = A.load()
    out = subprocess.run(["nm", "-D", "--defined-only", A.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (mk_\w+)", out))
    missing = [n for n in _declared() if n not in exported]
    assert not missing, missing
    # and the ctypes table covers them all
    assert set(_declared()) == set(A.PROTOTYPES), set(_declared()) ^ set(A.PROTOTYPES)
    for n in _declared():
        getattr(lib, n)


def test_abi_version_and_struct_sizes():
    lib = A.load()
    assert lib.mk_abi_version() == 3
    assert A.C.sizeof(A.MkParams) == 3984
    assert A.C.sizeof(A.MkDiag) == 88


def test_no_cpu_fallback_without_device(tmp_path):
    from conftest import HAVE_GPU
    if HAVE_GPU:
        pytest.skip("a device is present")
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases
    xml = cases.write(cases.poiseuille(nx=4, ny=5, nz=4), str(tmp_path / "p.xml"))
    with pytest.raises(A.MkError) as e:
        Solver(xml)
    assert e.value.status == A.MK_ERR_NODEVICE


def test_metrics_log_path_checked():
    # host-only: an unwritable metrics log path is an MK_ERR_IO status
    lib = A.load()
    assert lib.mk_set_metrics_log(b"/nonexistent_dir/x/metrics.jsonl") == A.MK_ERR_IO
    assert lib.mk_set_metrics_log(None) == A.MK_OK
