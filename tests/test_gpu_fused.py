"""The fused multiphase loop (one cooperative launch per loop: tiles publish
their phi planes with release flags, the halo planes are staged into shared
memory by the bulk-copy engine) against the two-kernel loop (phi kernel, then
collision kernel) and the oracle, and its bounded waits.

Both forms run the same per-cell arithmetic on the same populations, so they
must agree bit for bit in every storage precision; the FP64 fused form must
match the oracle to 1e-10.  The two-kernel loop is the default (the autotuner
keeps the faster form)."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle, ocase, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ["phi", "rho", "pressure", "ux", "uy", "uz"]

SHAPES = {
    # name: (nx, ny, nz, boundary, bubbles, contact angle)
    "walls_z": (32, 32, 24, "periodic periodic walls", 2, 90.0),
    "periodic_xyz": (40, 28, 20, "periodic periodic periodic", 2, 90.0),
    "ragged_x_closed": (36, 23, 17, "closed walls periodic", 1, 60.0),
    "walls_y_wetting": (64, 20, 12, "periodic walls periodic", 1, 45.0),
}


def _case(casedir, name, prec):
    nx, ny, nz, bc, nb, th = SHAPES[name]
    text = cases.multiphase_bubbles(n=nx, ny=ny, nz=nz, bubbles=nb, rmin=3.0, rmax=4.0, width=2.0, gz=-1e-5,
                                    precision=prec, loops=10, boundary=bc, contact_angle=th)
    return cases.write(text, f"{casedir}/fused_{name}_{prec}.xml")


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_fused_equals_two_kernel(casedir, name, prec):
    p = case_params(_case(casedir, name, prec))
    a, b = Solver(params=p), Solver(params=p)
    assert not a.fused, "the two-kernel loop is the default"
    a.fused = True
    assert a.fused, "the case should admit the fused loop"
    for n in (1, 1, 5):
        a.advance(n)
        b.advance(n)
        for f in FIELDS:
            x, y = a.field(f), b.field(f)
            assert np.array_equal(x, y), (name, prec, a.step, f, float(np.max(np.abs(x - y))))
    a.advance(6, graph=True)
    b.advance(6, graph=True)
    assert a.launches_per_step() == 1 and b.launches_per_step() == 2
    assert np.array_equal(a.field("phi"), b.field("phi"))


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_fused_fp64_matches_oracle(casedir, name):
    path = _case(casedir, name, "fp64")
    s = Solver(params=case_params(path))
    s.fused = True
    o = Oracle.from_xml(path)
    fl = ocase.flags(o.params) == 0
    for n in (1, 1, 1, 30):
        s.advance(n)
        o.advance(n)
        for f in ("phi", "rho"):
            e = rel_l2(s.field(f), o.field(f), fl)
            assert e <= 1e-10, (name, s.step, f, e)


def test_cases_without_fused_form(casedir):
    # x extent not a multiple of 4, or fewer than 8 planes: the two-kernel loop
    for nx, nz in ((30, 16), (32, 6)):
        path = cases.write(cases.multiphase_bubbles(n=nx, nz=nz, bubbles=0, precision="fp32", loops=1),
                           f"{casedir}/nofuse_{nx}_{nz}.xml")
        s = Solver(params=case_params(path))
        assert not s.fused
        assert s._lib.mk_set_fused(s.handle, 1) == A.MK_ERR_ARG
        s.advance(3)
        assert s.launches_per_step() == 2


def test_bounded_wait_times_out_and_recovers(casedir, tmp_path):
    # one tile never publishes its phi planes: its neighbours' waits run out
    # after their iteration limit, the launch ends, and the host reads
    # MK_ERR_TIMEOUT; the handle then runs normally again
    p = case_params(_case(casedir, "walls_z", "fp32"))
    s = Solver(params=p)
    ref = Solver(params=p)
    s.fused = True
    ref.fused = True
    s.advance(2)
    ref.advance(2)
    ck = str(tmp_path / "before.bin")
    s.checkpoint(ck)
    assert s._lib.mk_inject_fault(s.handle, 1) == A.MK_OK
    s.advance(1)
    assert s._lib.mk_sync(s.handle) == A.MK_ERR_TIMEOUT
    assert b"bounded device wait" in s._lib.mk_last_error(s.handle)
    assert s._lib.mk_sync(s.handle) == A.MK_OK  # reported once
    s.restore(ck)
    s.advance(3, graph=True)
    ref.advance(3, graph=True)
    assert s._lib.mk_sync(s.handle) == A.MK_OK
    assert np.array_equal(s.field("phi"), ref.field("phi"))
    assert s._lib.mk_inject_fault(s.handle, 7) == A.MK_ERR_ARG
