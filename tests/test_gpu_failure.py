"""Failure detection with host-side injection: every failure here is made on
the host (a non-finite field uploaded through mk_set_state, a truncated or
foreign checkpoint file, an allocation larger than the device), never by a
device fault.  Each must come back as a status code with a message, and the
context must stay usable afterwards.

The reference has no failure detection (its mkIsNan macros,
MaterKit/inc/mkGlobalDefs.h:200-242, are never called); the watchdog is the
divergence check folded into the FP64 diagnostics reduction."""
import os

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

pytestmark = pytest.mark.gpu


def _mp(casedir, prec="fp32"):
    return case_params(cases.write(cases.multiphase_bubbles(n=32, nz=32, bubbles=1, rmin=4, rmax=5, width=2.0,
                                                            precision=prec, loops=10), f"{casedir}/f_mp_{prec}.xml"))


def _dend(casedir, prec="fp32"):
    return case_params(cases.write(cases.thermal_dendrite(n=20, radius=4.0, precision=prec, loops=10),
                                   f"{casedir}/f_d_{prec}.xml"))


def _status(s, fn, *args):
    return getattr(s._lib, fn)(s.handle, *args)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
def test_nan_field_is_reported_as_diverged(casedir, prec):
    p = _mp(casedir, prec)
    s = Solver(params=p)
    phi = np.full((p.nz, p.ny, p.nx), 0.9)
    phi[5, 7, 3] = np.nan
    phi[11, 2, 9] = np.inf
    s.set_state(phi=phi)
    s.advance(3)
    d = A.MkDiag()
    assert _status(s, "mk_diagnostics", A.C.byref(d)) == A.MK_ERR_DIVERGED
    assert d.n_bad > 0
    assert b"diverged" in s._lib.mk_last_error(s.handle)
    # the context is intact: the handle keeps working and a fresh one is clean
    s.advance(2)
    assert _status(s, "mk_sync") == A.MK_OK
    s.close()
    t = Solver(params=p)
    t.advance(3)
    assert t.diagnostics()["n_bad"] == 0
    t.close()


def test_nonpositive_density_is_reported(casedir):
    p = case_params(cases.write(cases.poiseuille(nx=8, ny=6, nz=4, loops=1, precision="fp64"), f"{casedir}/f_fl.xml"))
    s = Solver(params=p)
    rho = np.ones((p.nz, p.ny, p.nx))
    rho[2, 3, 4] = -0.5
    s.set_state(rho=rho)
    d = A.MkDiag()
    assert _status(s, "mk_diagnostics", A.C.byref(d)) == A.MK_ERR_DIVERGED
    assert d.n_bad >= 1
    s.close()


def test_dendrite_nan_temperature_is_reported(casedir):
    p = _dend(casedir)
    s = Solver(params=p)
    T = np.full((p.nz, p.ny, p.nx), -p.delta)
    T[10, 10, 10] = np.nan
    s.set_state(T=T)
    s.advance(2)
    d = A.MkDiag()
    assert _status(s, "mk_diagnostics", A.C.byref(d)) == A.MK_ERR_DIVERGED
    s.close()


def test_truncated_checkpoint_is_io_error(casedir, tmp_path):
    p = _dend(casedir)
    a = Solver(params=p)
    a.advance(5)
    path = str(tmp_path / "ck.bin")
    a.checkpoint(path)
    size = os.path.getsize(path)
    for cut in (size - 1, size // 2, 40, 3):
        with open(path, "rb") as f:
            data = f.read()[:cut]
        bad = str(tmp_path / f"cut_{cut}.bin")
        with open(bad, "wb") as f:
            f.write(data)
        b = Solver(params=p)
        assert _status(b, "mk_restore", bad.encode()) == A.MK_ERR_IO, cut
        assert s_ok(b)
        b.close()
    # the intact file still restores
    b = Solver(params=p)
    b.restore(path)
    assert b.step == 5
    assert np.array_equal(a.field("phi"), b.field("phi"))
    a.close()
    b.close()


def s_ok(s):
    return s._lib.mk_sync(s.handle) == A.MK_OK


def test_foreign_and_garbage_checkpoints_rejected(casedir, tmp_path):
    a = Solver(params=_dend(casedir))
    a.advance(2)
    path = str(tmp_path / "ck_dend.bin")
    a.checkpoint(path)
    other = Solver(params=_mp(casedir))
    assert _status(other, "mk_restore", path.encode()) == A.MK_ERR_ARG
    junk = str(tmp_path / "junk.bin")
    with open(junk, "wb") as f:
        f.write(b"\x00" * 4096)
    assert _status(other, "mk_restore", junk.encode()) == A.MK_ERR_IO
    assert _status(other, "mk_restore", str(tmp_path / "missing.bin").encode()) == A.MK_ERR_IO
    assert _status(other, "mk_checkpoint", str(tmp_path / "no_dir" / "x.bin").encode()) == A.MK_ERR_IO
    other.advance(2)
    assert other.diagnostics()["n_bad"] == 0
    a.close()
    other.close()


def test_allocation_failure_is_oom(casedir):
    # a case larger than the device's memory: the first allocation fails and the
    # create call returns MK_ERR_OOM (no host-side fields are built before it)
    p = case_params(cases.write(cases.multiphase_bubbles(n=1200, bubbles=0, precision="fp64", loops=1),
                                f"{casedir}/f_huge.xml"))
    lib = A.load()
    h = A.C.c_void_p()
    assert lib.mk_create(A.C.byref(p), A.C.byref(h)) == A.MK_ERR_OOM
    assert not h.value
    assert b"allocate" in lib.mk_last_global_error()
    # the failed allocation leaves nothing behind: the next handle creates and runs
    s = Solver(params=_mp(casedir))
    s.advance(2)
    assert s.diagnostics()["n_bad"] == 0
    s.close()
