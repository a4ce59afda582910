"""Flow + dendrite model (run_flow_thermal_dendrite) on the GPU vs the FP64
oracle, through the C ABI: porous bounce-back of the growing crystal, the
thermal lattice advected by the flow, and the inflow/outflow faces.

FP64 storage matches the oracle to 1e-10 relative L2 per field at loops 1, 2
and 3 (both AA parities and the first boundary pass) and after 40 loops.
"""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases, case_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle, rel_l2

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FIELDS = ["phi", "T", "rho"]


def _case(prec="fp64", coll="TRT", lat="D3Q19", inlet=True, **kw):
    return cases.flow_dendrite(nx=24, ny=14, nz=12, radius=4.0, u_in=0.03, center=(8.0, 6.5, 5.5), precision=prec,
                               collision=coll, lattice=lat, inlet=inlet, **kw)


def _pair(casedir, name, text):
    # each side resolves the file through its own case layer
    path = cases.write(text, f"{casedir}/{name}.xml")
    p = case_params(path)
    return p, Solver(params=p), Oracle.from_xml(path)


def _errs(s, o):
    e = {f: rel_l2(s.field(f), o.field(f)) for f in FIELDS}
    u = np.stack([s.field(f) for f in ("ux", "uy", "uz")])
    v = np.stack([o.field(f) for f in ("ux", "uy", "uz")])
    e["u"] = rel_l2(u, v)
    return e


@pytest.mark.parametrize("coll,lat,inlet", [("TRT", "D3Q19", True), ("MRT", "D3Q19", True), ("BGK", "D3Q27", True),
                                            ("TRT", "D3Q19", False)])
def test_flow_dendrite_fp64_steps(casedir, coll, lat, inlet):
    p, s, o = _pair(casedir, f"fd_{coll}_{lat}_{int(inlet)}", _case(coll=coll, lat=lat, inlet=inlet))
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
    assert (s.field("flag") == A.MK_FLAG_SOLID).sum() > 100


def test_flow_dendrite_separate_boundary_kernel_fp64(casedir):
    # nx = 33: the outflow face cell starts a warp, so the faces are applied by
    # the separate boundary kernel instead of in the collision kernels
    p, s, o = _pair(casedir, "fd_nx33", cases.flow_dendrite(nx=33, ny=10, nz=9, radius=3.0, u_in=0.03,
                                                             center=(10.0, 4.5, 4.0), precision="fp64"))
    assert s.launches_per_step() == 4
    for n in (1, 1, 1, 20):
        s.advance(n)
        o.advance(n)
        e = _errs(s, o)
        assert max(e.values()) <= FP64_TOL, (s.step, e)


def test_flow_dendrite_fp32(casedir):
    p, s, o = _pair(casedir, "fd32", _case("fp32"))
    s.advance(60)
    o.advance(60)
    e = _errs(s, o)
    assert max(e.values()) <= 1e-5, e


@pytest.mark.parametrize("prec,tol", [("fp16", 2e-2), ("bf16", 5e-2)])
def test_flow_dendrite_16bit(casedir, prec, tol):
    p, s, o = _pair(casedir, f"fd_{prec}", _case(prec))
    s.advance(60)
    o.advance(60)
    e = _errs(s, o)
    assert max(e.values()) <= tol, e


def test_flow_dendrite_launches_graph_and_checkpoint(casedir, tmp_path):
    p = case_params(cases.write(_case("fp32"), f"{casedir}/fd_ck.xml"))
    a, b = Solver(params=p), Solver(params=p)
    assert a.launches_per_step() == 3  # phi, flow (+ faces), phase field + thermal (+ faces)
    prof = a.profile(4, "collide")
    assert prof["kernel_ms"] > 0
    b.advance(4)
    a.advance(7, graph=True)
    b.advance(7)
    for f in ["phi", "T", "ux", "rho"]:
        assert np.array_equal(a.field(f), b.field(f))
    a.checkpoint(str(tmp_path / "fd.bin"))
    a.advance(5)
    c = Solver(params=p)
    c.restore(str(tmp_path / "fd.bin"))
    c.advance(5)
    for f in ["phi", "T", "ux", "uz", "rho"]:
        assert np.array_equal(a.field(f), c.field(f))
    d = a.diagnostics()
    assert d["n_bad"] == 0 and d["max_speed"] > 0.01


def test_flow_dendrite_closed_faces_conserve_mass(casedir):
    p = case_params(cases.write(_case("fp64", inlet=False), f"{casedir}/fd_mass.xml"))
    s = Solver(params=p)
    m0 = s.diagnostics()["mass"]
    s.advance(50)
    assert abs(s.diagnostics()["mass"] - m0) / m0 < 1e-12


def test_reference_call_sequence(casedir):
    # run_flow_thermal_dendrite's per-loop calls (MaterKit.cpp:499-516) drive
    # the same device loop as Solver.advance; a call out of order is refused
    from materkit_anisotropiclbm_trt_rbc_facet_b200.solver import mkFluidsMRT, mkSpace
    xml = cases.write(_case("fp32"), f"{casedir}/fd_seq.xml")
    flow = mkFluidsMRT(mkSpace(xml), precision="fp32")
    flow.initialize(xml, model=A.MK_MODEL_FLOW_DENDRITE)
    flow.initialize_geometry()
    for _ in range(3):
        flow.propagate_PBB()
        flow.relaxation()
        flow.bdyVelocity()
        flow.phasefield_propagate()
        flow.relaxation_anisotropy_thermal()
        flow.thermal_propagate()
        flow.thermal_relaxation()
        flow.bdy_flowin()
    ref = Solver(params=case_params(xml, precision="fp32"))
    ref.advance(3)
    assert flow.solver.step == 3
    for f in ["phi", "T", "ux", "rho"]:
        assert np.array_equal(flow.solver.field(f), ref.field(f))
    with pytest.raises(A.MkError):
        flow.thermal_propagate()


def test_flow_dendrite_vtk_has_flow_and_flags(casedir, tmp_path):
    p = case_params(cases.write(_case("fp32"), f"{casedir}/fd_vtk.xml"))
    s = Solver(params=p)
    s.advance(10)
    text = open(s.write_vtk(10, str(tmp_path))).read()
    assert "VECTORS velocity_vector float" in text and "SCALARS temperature float 1" in text
    vel = text.split("VECTORS velocity_vector float\n")[1].split()
    ux = np.array(vel[0::3], dtype=float).reshape(s.shape)
    assert np.allclose(ux, s.field("ux"), rtol=1e-5, atol=1e-7)
    flag = s.field("flag")
    assert set(np.unique(flag)) <= {A.MK_FLAG_FLUID, A.MK_FLAG_SOLID}
    assert np.array_equal(flag == A.MK_FLAG_SOLID, s.field("phi") > 0)
