"""The multiphase collision with its phi tile staged by one TMA tensor load
per 64 x 4 block (k_mp_collide_tma, tuning phi_tile) against the
thread-per-cell collision: the same per-cell source reading the same phi
values, bit-identical with FP32, FP16 and BF16 storage and to 1e-13 with
FP64 (the compiler contracts FP64 expressions per kernel), both AA parities,
periodic, walled and closed axes, rows and planes that are not multiples of
the block; the FP64 form matches the oracle to 1e-10; cases whose x extent
is not a multiple of 4 are refused."""
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
    "walls_x_closed_z": (48, 22, 17, "walls periodic closed", 1, 60.0),
    "closed_x_walls_y": (68, 21, 12, "closed walls periodic", 1, 45.0),
    "wide_rows": (132, 18, 19, "periodic periodic walls", 1, 90.0),
}


def _case(casedir, name, prec):
    nx, ny, nz, bc, nb, th = SHAPES[name]
    text = cases.multiphase_bubbles(n=nx, ny=ny, nz=nz, bubbles=nb, rmin=3.0, rmax=4.0, width=2.0, gz=-1e-5,
                                    precision=prec, loops=10, boundary=bc, contact_angle=th)
    return cases.write(text, f"{casedir}/tile_{name}_{prec}.xml")


def _same(prec, x, y):
    if prec != "fp64":
        return np.array_equal(x, y)
    return float(np.max(np.abs(x - y))) <= 1e-13 * max(float(np.max(np.abs(y))), 1e-30)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_phi_tile_equals_thread_per_cell(casedir, name, prec):
    p = case_params(_case(casedir, name, prec))
    a, b = Solver(params=p), Solver(params=p)
    assert a.tuning["phi_tile"] == 0, "the thread-per-cell collision is the default"
    a.tuning = {"phi_tile": 1}
    assert a.tuning["phi_tile"] == 1
    for n in (1, 1, 5):
        a.advance(n)
        b.advance(n)
        for f in FIELDS:
            x, y = a.field(f), b.field(f)
            assert _same(prec, x, y), (name, prec, a.step, f, float(np.nanmax(np.abs(x - y))))
    a.advance(6, graph=True)
    b.advance(6, graph=True)
    assert _same(prec, a.field("phi"), b.field("phi"))
    assert a.diagnostics()["n_bad"] == 0


def test_phi_tile_fp64_matches_oracle(casedir):
    path = _case(casedir, "walls_x_closed_z", "fp64")
    s = Solver(params=case_params(path))
    s.tuning = {"phi_tile": 1}
    o = Oracle.from_xml(path)
    fl = ocase.flags(o.params) == 0
    for n in (1, 1, 7):
        s.advance(n)
        o.advance(n)
        for f in ("phi", "rho"):
            e = rel_l2(s.field(f), o.field(f), fl)
            assert e <= 1e-10, (s.step, f, e)


def test_phi_tile_refused_and_exclusive(casedir):
    # 30 cells along x: a row of 120 bytes is not a multiple of 16
    text = cases.multiphase_bubbles(n=30, ny=12, nz=12, bubbles=0, precision="fp32", loops=10,
                                    boundary="periodic periodic walls")
    s = Solver(params=case_params(cases.write(text, f"{casedir}/tile_refused.xml")))
    with pytest.raises(A.MkError) as e:
        s.tuning = {"phi_tile": 1}
    assert e.value.status == A.MK_ERR_ARG
    assert s.tuning["phi_tile"] == 0
    p = case_params(_case(casedir, "walls_z", "fp32"))
    t = Solver(params=p)
    for bad in ({"phi_tile": 2}, {"phi_tile": 1, "row_staged": 1}, {"phi_tile": 1, "fused": 1}):
        with pytest.raises(A.MkError):
            t.tuning = bad
    assert t.tuning["phi_tile"] == 0
