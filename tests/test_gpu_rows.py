"""The row-staged multiphase collision (k_mp_rows: whole x rows of all 38
populations staged through shared memory by the bulk-copy engine, several
rows in flight per CTA) against the thread-per-cell collision: the same
per-cell source on the same values, bit-identical with FP32 arithmetic
(FP32, FP16, BF16 storage: the packed-pair arithmetic is written out
explicitly), both AA parities, periodic, walled and closed axes (the closed
and walled x ends take the own-slot path), and on slab handles.  The FP64
arithmetic is plain expressions whose multiply-adds the compiler contracts
per kernel, so the two FP64 kernels may differ in the last bit of a few cells:
they are held to 1e-13 relative, and the FP64 row-staged form matches the
oracle to 1e-10."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as S
from _oracle import Oracle, ocase, rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ["phi", "rho", "pressure", "ux", "uy", "uz"]

SHAPES = {
    # name: (nx, ny, nz, boundary, bubbles, contact angle)
    "walls_z": (32, 32, 24, "periodic periodic walls", 2, 90.0),
    "periodic_xyz": (40, 28, 20, "periodic periodic periodic", 2, 90.0),
    "walls_x_closed_z": (48, 20, 17, "walls periodic closed", 1, 60.0),
    "closed_x_walls_y": (64, 20, 12, "closed walls periodic", 1, 45.0),
    "row_256": (256, 20, 20, "periodic periodic walls", 1, 90.0),
}


def _case(casedir, name, prec):
    nx, ny, nz, bc, nb, th = SHAPES[name]
    text = cases.multiphase_bubbles(n=nx, ny=ny, nz=nz, bubbles=nb, rmin=3.0, rmax=4.0, width=2.0, gz=-1e-5,
                                    precision=prec, loops=10, boundary=bc, contact_angle=th)
    return cases.write(text, f"{casedir}/rows_{name}_{prec}.xml")


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_row_staged_equals_thread_per_cell(casedir, name, prec):
    p = case_params(_case(casedir, name, prec))
    a, b = Solver(params=p), Solver(params=p)
    assert not a.row_staged, "the thread-per-cell collision is the default"
    a.row_staged = True
    assert a.row_staged, "the case should admit the row-staged collision"
    def same(x, y):
        if prec != "fp64":
            return np.array_equal(x, y)
        scale = max(float(np.max(np.abs(y))), 1e-30)
        return float(np.max(np.abs(x - y))) <= 1e-13 * scale

    for n in (1, 1, 5):
        a.advance(n)
        b.advance(n)
        for f in FIELDS:
            x, y = a.field(f), b.field(f)
            assert same(x, y), (name, prec, a.step, f, float(np.nanmax(np.abs(x - y))))
    a.advance(6, graph=True)
    b.advance(6, graph=True)
    assert a.launches_per_step() == 2
    assert same(a.field("phi"), b.field("phi"))


def test_row_staged_fp64_matches_oracle(casedir):
    path = _case(casedir, "walls_x_closed_z", "fp64")
    s = Solver(params=case_params(path))
    s.row_staged = True
    o = Oracle.from_xml(path)
    fl = ocase.flags(o.params) == 0
    for n in (1, 1, 7):
        s.advance(n)
        o.advance(n)
        for f in ("phi", "rho"):
            e = rel_l2(s.field(f), o.field(f), fl)
            assert e <= 1e-10, (s.step, f, e)


def test_row_staged_refused_where_not_admitted(casedir):
    # 36 cells of FP16 are 72 bytes: not a multiple of 16
    text = cases.multiphase_bubbles(n=36, ny=12, nz=12, bubbles=0, precision="fp16", loops=10,
                                    boundary="periodic periodic walls")
    s = Solver(params=case_params(cases.write(text, f"{casedir}/rows_refused.xml")))
    with pytest.raises(A.MkError) as e:
        s.row_staged = True
    assert e.value.status == A.MK_ERR_ARG
    assert not s.row_staged


@pytest.mark.parametrize("prec", ["fp64", "bf16"])
def test_row_staged_slabs_equal_whole_domain(casedir, prec):
    p = case_params(_case(casedir, "walls_x_closed_z", prec))
    whole = Solver(params=p)
    whole.row_staged = True
    slabs = [S.Slab(p, r, 3) for r in range(3)]
    for s in slabs:
        s.row_staged = True
    for k in (1, 4):
        whole.advance(k)
        S.advance_local(slabs, k)
        for f in FIELDS:
            assert np.array_equal(np.concatenate([s.owned(f) for s in slabs]), whole.field(f)), (k, f)


def test_autotune_reports_the_row_staged_form(casedir):
    p = case_params(_case(casedir, "walls_z", "fp32"))
    s = Solver(params=p)
    ref = Solver(params=p)
    t = s.autotune(2)
    if s.row_staged:
        assert t["minb"] == 0 and t["block"][0] > 0
    s.advance(4)
    ref.advance(4)
    assert np.array_equal(s.field("phi"), ref.field("phi"))


def test_tuning_roundtrip_and_checks(casedir):
    p = case_params(_case(casedir, "walls_z", "fp32"))
    s = Solver(params=p)
    t = s.tuning
    assert set(t) == {"block_x", "block_y", "minb", "fused", "row_staged", "phi_tile"}
    s.tuning = {"block_x": 32, "block_y": 4, "minb": 1, "row_staged": 1}
    assert s.tuning == dict(t, block_x=32, block_y=4, minb=1, row_staged=1)
    for bad in ({"block_x": 48}, {"block_x": 64, "block_y": 32}, {"minb": 6}, {"minb": 0}, {"row_staged": 2}):
        with pytest.raises(A.MkError) as e:
            s.tuning = bad
        assert e.value.status == A.MK_ERR_ARG, bad
    assert s.tuning["block_x"] == 32  # a refused setting changes nothing
    q = case_params(cases.write(cases.poiseuille(nx=8, ny=6, nz=6), f"{casedir}/tune_pois.xml"))
    f = Solver(params=q)
    with pytest.raises(A.MkError):
        f.tuning = {"row_staged": 1}
    # the autotuner's choice is reported and reproduces the untuned result
    ref = Solver(params=p)
    s2 = Solver(params=p)
    s2.autotune(2)
    s2.advance(4)
    ref.advance(4)
    assert np.array_equal(s2.field("phi"), ref.field("phi"))


@pytest.mark.parametrize("prec", ["fp64", "fp32", "bf16"])
@pytest.mark.parametrize("minb", [1, 3, 4, 5])
def test_occupancy_variants_agree(casedir, prec, minb):
    # the register-capped variants (minb 3, 4, 5: 112, 96, 80 registers) run
    # the same source as the 256-thread launch-bound ones
    p = case_params(_case(casedir, "walls_x_closed_z", prec))
    a, b = Solver(params=p), Solver(params=p)
    a.tuning = {"block_x": 64, "block_y": 1, "minb": minb}
    b.tuning = {"block_x": 64, "block_y": 1, "minb": 2}
    for n in (1, 1, 5):
        a.advance(n)
        b.advance(n)
    for f in FIELDS:
        x, y = a.field(f), b.field(f)
        if prec == "fp64":
            assert float(np.max(np.abs(x - y))) <= 1e-13 * max(float(np.max(np.abs(y))), 1e-30), f
        else:
            assert np.array_equal(x, y), (prec, minb, f)
