"""Packed dendrite ensemble (the seed / anisotropy / undercooling sweep of
run_solutal_dendrite and run_thermal_dendrite, MaterKit/MaterKit.cpp:633-687,
:743-788) against the same cases run one at a time.

The ensemble kernels run the single-domain cell code on a packed index, so a
domain of the ensemble must evolve bit for bit like the case alone: fields are
compared for exact equality, at both AA parities (odd loop counts exercise the
eager tail after the two-loop graphs).
"""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Ensemble, Solver, ensemble_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

pytestmark = pytest.mark.gpu


def _small(precision, model="solutal_dendrite", edges=(16, 24, 32, 24)):
    """Generator parameters shrunk to small cubes, with per-domain undercooling."""
    ps = ensemble_params(0xE45E, len(edges), precision)
    rng = np.random.default_rng(7)
    for d, (p, L) in enumerate(zip(ps, edges)):
        p.model = A.MODELS[model]
        p.nx = p.ny = p.nz = L
        p.n_objects = min(p.n_objects, 3)
        for s in range(p.n_objects):
            p.obj_radius[s] = 2.5 + 0.5 * s
            for a in range(3):
                p.obj_center[s][a] = 4.0 + (L - 8.0) * rng.random()
        p.delta = 0.45 + 0.05 * d
    return ps


def _fields(model):
    return ["phi", "dphi", "C" if model == "solutal_dendrite" else "T"]


def _check_equal(ens, singles, fields, tag):
    for d, s in enumerate(singles):
        for f in fields + ["grain"]:
            a, b = ens.field(d, f), s.field(f)
            diff = float(np.max(np.abs(a - b)))
            assert np.array_equal(a, b), f"{tag}: domain {d} field {f} max |diff| {diff:.3e}"


@pytest.mark.parametrize("precision,model", [("fp64", "solutal_dendrite"), ("bf16", "solutal_dendrite"),
                                             ("fp32", "thermal_dendrite"), ("fp16", "thermal_dendrite")])
def test_ensemble_matches_single_domains(precision, model):
    ps = _small(precision, model)
    ens = Ensemble(ps)
    singles = [Solver(params=p) for p in ps]
    assert ens.cells == sum(p.ncell() for p in ps)
    _check_equal(ens, singles, _fields(model), "initial state")
    ens.advance(21)
    for s in singles:
        s.advance(21, graph=True)
    assert ens.step == 21
    _check_equal(ens, singles, _fields(model), "after 21 loops")
    ens.advance(9)
    for s in singles:
        s.advance(9)
    _check_equal(ens, singles, _fields(model), "after 30 loops")
    # the solid fraction grew somewhere (the loops did work)
    assert any(float(np.sum(ens.field(d, "dphi") != 0.0)) > 0 for d in range(len(ps)))
    ens.close()
    for s in singles:
        s.close()


def _shaped(precision, model, shapes):
    """Box-shaped domains (nx, ny, nz), each cell count a multiple of 256."""
    ps = _small(precision, model, edges=tuple(max(sh) for sh in shapes))
    rng = np.random.default_rng(11)
    for p, sh in zip(ps, shapes):
        p.nx, p.ny, p.nz = sh
        for s in range(p.n_objects):
            for a in range(3):
                p.obj_center[s][a] = 3.0 + (sh[a] - 6.0) * rng.random() + 0.137
    return ps


# every nx even (the ensemble's phi pass takes two cells per thread, the
# domains run alone one) and one odd nx (the one-cell pass everywhere): both
# passes give the same bits
SHAPES = {"even": [(18, 16, 16), (32, 8, 24), (16, 32, 8)],
          "odd": [(18, 16, 16), (17, 16, 16), (16, 32, 8)]}


@pytest.mark.parametrize("precision,model", [("fp64", "solutal_dendrite"), ("fp32", "thermal_dendrite"),
                                             ("fp16", "thermal_dendrite"), ("bf16", "solutal_dendrite")])
@pytest.mark.parametrize("shapes", sorted(SHAPES))
def test_ensemble_box_domains_match_single_domains(precision, model, shapes):
    ps = _shaped(precision, model, SHAPES[shapes])
    ens = Ensemble(ps)
    singles = [Solver(params=p) for p in ps]
    for n in (13, 8):
        ens.advance(n)
        for s in singles:
            s.advance(n)
        _check_equal(ens, singles, _fields(model), f"{shapes} shapes after {ens.step} loops")
    ens.close()
    for s in singles:
        s.close()


@pytest.mark.parametrize("precision,model", [("fp32", "thermal_dendrite"), ("bf16", "solutal_dendrite")])
def test_ensemble_with_walls_matches_single_domains(precision, model):
    """Walls in y on one domain: the even loop's phi pass leaves the flat
    all-fluid form for the per-tile one (wall cells keep their phi)."""
    ps = _shaped(precision, model, SHAPES["even"])
    ps[1].bc[1] = A.MK_BC_WALLS
    ens = Ensemble(ps)
    singles = [Solver(params=p) for p in ps]
    for n in (13, 8):
        ens.advance(n)
        for s in singles:
            s.advance(n)
        _check_equal(ens, singles, _fields(model), f"walls after {ens.step} loops")
    ens.close()
    for s in singles:
        s.close()


def test_generated_ensemble_runs():
    ps = ensemble_params(0xE45E, 6, "bf16")
    ens = Ensemble(ps)
    ms = ens.time_advance(20)
    assert ms > 0
    for d, p in enumerate(ps):
        phi = ens.field(d, "phi", np.float32)
        c = ens.field(d, "C", np.float32)
        assert np.isfinite(phi).all() and np.isfinite(c).all()
        assert phi.shape == (p.nz, p.ny, p.nx)
        assert (phi > 0).sum() > 0  # the seeds are there
    ens.close()


def test_ensemble_errors():
    ps = _small("fp32")
    ens = Ensemble(ps)
    with pytest.raises(A.MkError):
        ens.field(len(ps), "phi")
    buf = np.empty(64 ** 3)
    lib = A.load()
    assert lib.mk_ensemble_get_field(ens._h, len(ps), A.MK_FIELD_PHI, A.MK_DTYPE_F64, buf.ctypes.data,
                                     buf.nbytes) == A.MK_ERR_ARG
    assert b"out of range" in lib.mk_ensemble_last_error(ens._h)
    assert lib.mk_ensemble_get_field(ens._h, 0, A.MK_FIELD_PHI, A.MK_DTYPE_F64, buf.ctypes.data,
                                     8) == A.MK_ERR_ARG
    with pytest.raises(A.MkError):
        ens.field(0, "T")  # solutal ensemble has no temperature
    with pytest.raises(A.MkError):
        ens.field(0, "ux")
    ens.close()
