"""Flow + solutal dendrite model (run_flow_solutal_dendrite, MaterKit.cpp:399-465)
on the GPU vs the FP64 oracle, through the C ABI: the flow lattice with porous
bounce-back and inflow / outflow faces (propagate_PBB, relaxation,
bdyVelocity), the solutal phase field (relaxation_anisotropy_solute), the
U-lattice advected by the flow with the solute's inflow face (bdy_LBflowin).

FP64 storage matches the oracle to 1e-10 relative L2 per field at loops 1, 2
and 3 and after 40 loops."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases, case_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle, rel_l2

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FIELDS = ["phi", "C", "dphi", "rho"]


def _case(prec="fp64", coll="TRT", lat="D3Q19", inlet=True, **kw):
    return cases.flow_solutal_dendrite(nx=24, ny=14, nz=12, radius=4.0, u_in=0.03, center=(8.0, 6.5, 5.5),
                                       precision=prec, collision=coll, lattice=lat, inlet=inlet, **kw)


def _pair(casedir, name, text):
    # each side resolves the file through its own case layer
    path = cases.write(text, f"{casedir}/{name}.xml")
    p = case_params(path)
    assert p.model == A.MK_MODEL_FLOW_SOLUTAL
    return p, Solver(params=p), Oracle.from_xml(path)


def _errs(s, o, fields=FIELDS):
    e = {f: rel_l2(s.field(f), o.field(f)) for f in fields}
    u = np.stack([s.field(f) for f in ("ux", "uy", "uz")])
    v = np.stack([o.field(f) for f in ("ux", "uy", "uz")])
    e["u"] = rel_l2(u, v)
    return e


@pytest.mark.parametrize("coll,lat,inlet", [("TRT", "D3Q19", True), ("MRT", "D3Q19", True), ("BGK", "D3Q27", True),
                                            ("TRT", "D3Q19", False)])
def test_flow_solutal_fp64_steps(casedir, coll, lat, inlet):
    p, s, o = _pair(casedir, f"fs_{coll}_{lat}_{int(inlet)}", _case(coll=coll, lat=lat, inlet=inlet))
    for _ in range(3):
        s.advance(1)
        o.advance(1)
        e = _errs(s, o)
        assert max(e.values()) <= FP64_TOL, (s.step, e)
    s.advance(37)
    o.advance(37)
    e = _errs(s, o)
    assert max(e.values()) <= FP64_TOL, (s.step, e)
    assert np.array_equal(s.field("flag"), o.field("flag"))
    # the solute is advected: the inflow face holds the far-field value
    if inlet:
        assert np.allclose(s.field("C")[:, :, 0], -p.delta, atol=1e-12)


def test_flow_solutal_separate_boundary_kernel_fp64(casedir):
    # nx = 33: the outflow face cell starts a warp, so the faces go through the
    # separate boundary kernel
    p, s, o = _pair(casedir, "fs_nx33", cases.flow_solutal_dendrite(nx=33, ny=10, nz=9, radius=3.0, u_in=0.03,
                                                                     center=(10.0, 4.5, 4.0), precision="fp64"))
    assert s.launches_per_step() == 4
    for n in (1, 1, 1, 20):
        s.advance(n)
        o.advance(n)
        e = _errs(s, o)
        assert max(e.values()) <= FP64_TOL, (s.step, e)


def test_flow_solutal_fp32(casedir):
    p, s, o = _pair(casedir, "fs32", _case("fp32"))
    s.advance(60)
    o.advance(60)
    e = _errs(s, o, ["phi", "C", "rho"])
    assert max(e.values()) <= 1e-5, e


@pytest.mark.parametrize("prec,tol", [("fp16", 2e-2), ("bf16", 5e-2)])
def test_flow_solutal_16bit(casedir, prec, tol):
    p, s, o = _pair(casedir, f"fs_{prec}", _case(prec))
    s.advance(60)
    o.advance(60)
    e = _errs(s, o, ["phi", "C", "rho"])
    assert max(e.values()) <= tol, e


def test_flow_solutal_graph_checkpoint_and_diagnostics(casedir, tmp_path):
    p = case_params(cases.write(_case("fp32"), f"{casedir}/fs_ck.xml"))
    a, b = Solver(params=p), Solver(params=p)
    assert a.launches_per_step() == 3
    b.advance(4)
    a.advance(4, graph=True)
    a.advance(7, graph=True)
    b.advance(7)
    for f in ["phi", "C", "ux", "rho"]:
        assert np.array_equal(a.field(f), b.field(f))
    a.checkpoint(str(tmp_path / "fs.bin"))
    a.advance(5)
    c = Solver(params=p)
    c.restore(str(tmp_path / "fs.bin"))
    c.advance(5)
    for f in ["phi", "C", "uz"]:
        assert np.array_equal(a.field(f), c.field(f))
    d = a.diagnostics()
    assert d["n_bad"] == 0 and d["max_speed"] > 0.01
    assert d["solute"] == pytest.approx(float(a.field("C").sum()), rel=1e-6)


def test_reference_call_sequence(casedir):
    # run_flow_solutal_dendrite's per-loop calls (MaterKit.cpp:430-456) drive
    # the same device loop as Solver.advance; a call out of order is refused
    from materkit_anisotropiclbm_trt_rbc_facet_b200.solver import mkFluidsMRT, mkSpace
    xml = cases.write(_case("fp32"), f"{casedir}/fs_seq.xml")
    flow = mkFluidsMRT(mkSpace(xml), precision="fp32")
    flow.initialize(xml, model=A.MK_MODEL_FLOW_SOLUTAL)
    flow.initialize_geometry()
    for loops in range(3):
        flow.propagate_PBB()
        flow.relaxation()
        flow.bdyVelocity()
        flow.phasefield_propagate()
        flow.relaxation_anisotropy_solute(loops)
        flow.solutal_propagate()
        flow.solutal_relaxation()
        flow.bdy_LBflowin()
    ref = Solver(params=case_params(xml, precision="fp32"))
    ref.advance(3)
    assert flow.solver.step == 3
    for f in ["phi", "C", "ux", "rho"]:
        assert np.array_equal(flow.solver.field(f), ref.field(f))
    with pytest.raises(A.MkError):
        flow.solutal_relaxation()
