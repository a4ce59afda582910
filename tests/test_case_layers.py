"""The library's case layer (mk_case_params / mk_case_initial_field,
csrc/mk_case.cpp) against the oracle's own (oracle/case.py), field by field.

The parity tests start the library and the oracle from their own readings of
the same XML file, so a wrong tag mapping, unit conversion, seed placement or
initial profile in either layer shows up here first.  No GPU is needed.
"""
import glob
import os

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases, case_params, ensemble_params, initial_field
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from oracle import case as K

HERE = os.path.dirname(os.path.abspath(__file__))
SHIPPED = sorted(glob.glob(os.path.join(HERE, "golden", "shipped_cases", "*.xml")))
REFERENCE_CASES = sorted(glob.glob("/root/reference/MaterKit/BoltzTechs*.xml"))

FIELDS = ["phi", "rho", "ux", "uy", "uz", "T", "C", "flag", "pressure", "dphi", "grain"]

# The five benchmark configurations at their stated sizes (parameters only)
# and at reduced sizes (parameters and initial fields).
CONFIGS = {
    "config1_poiseuille": cases.poiseuille(),
    "config2_thermal_dendrite": cases.thermal_dendrite(n=128),
    "config3_bubbles": cases.multiphase_bubbles(n=256),
    "config3_bubbles_fp16": cases.multiphase_bubbles(n=256, precision="fp16"),
    "config5_adjoint": cases.thermal_dendrite(n=96, loops=2000, eps4=0.05, delta=0.55, radius=8.0),
}
SMALL = {
    "poiseuille": cases.poiseuille(nx=9, ny=7, nz=5),
    "thermal_dendrite": cases.thermal_dendrite(n=24, radius=4.0),
    "thermal_hcp": cases.thermal_dendrite(n=20, aniso="hcp", eps2=0.02, center=(9.3, 10.1, 8.7)),
    "solutal": cases.solutal_dendrite(n=24, seeds=[((11.3, 12.1, 10.7), (10.0, 20.0, 30.0), 4.0),
                                                   ((4.0, 5.0, 17.0), (0.0, 45.0, 0.0), 2.5)]),
    "bubbles": cases.multiphase_bubbles(n=48, nz=40, bubbles=4, rmin=3, rmax=5, width=2.0),
    "bubbles_wetting": cases.multiphase_bubbles(n=32, bubbles=2, rmin=4, rmax=6, contact_angle=60.0),
    "convection": cases.convection(nx=20, ny=5, nz=12, Ra=2e4),
    "couette": cases.couette(nx=6, ny=12, nz=5, U=2e-2),
    "flow_dendrite": cases.flow_dendrite(nx=24, ny=14, nz=12, radius=4.0, u_in=0.03, center=(8.0, 6.5, 5.5)),
    "flow_solutal": cases.flow_solutal_dendrite(nx=24, ny=14, nz=12, radius=4.0, u_in=0.03, center=(8.0, 6.5, 5.5)),
    "multigrain": cases.multigrain(n=20, ny=19, nz=18, seeds=[(7.0, 9.5, 9.0, 5.0), (13.0, 9.5, 9.0, 5.0),
                                                              (10.0, 14.0, 11.0, 3.0)]),
}


def _both(path, **opt):
    return case_params(path, **opt), K.resolve(path, **opt)


def _same_params(pp, po):
    a, b = pp.to_dict(), po.values()
    diff = {k: (a[k], b[k]) for k in a if a[k] != b[k]}
    assert not diff, diff


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_params_agree(casedir, name):
    _same_params(*_both(cases.write(CONFIGS[name], f"{casedir}/cl_{name}.xml")))


def test_config3_bubbles_layout(casedir):
    # 24 bubbles of radius in [8, 16], 2W clear of the z walls and of each other
    pp, po = _both(cases.write(CONFIGS["config3_bubbles"], f"{casedir}/cl_c3.xml"))
    assert po.n_objects == 24 and po.rng_seed == 0xB200
    r = np.array(po.obj_radius[:24])
    c = np.array([list(po.obj_center[k]) for k in range(24)])
    assert r.min() >= 8.0 and r.max() <= 16.0
    assert (c[:, 2] - r >= 1 + 2 * po.width).all() and (c[:, 2] + r <= 254 - 2 * po.width).all()


@pytest.mark.parametrize("name", sorted(SMALL))
def test_initial_fields_agree(casedir, name):
    pp, po = _both(cases.write(SMALL[name], f"{casedir}/cl_s_{name}.xml"))
    _same_params(pp, po)
    for f in FIELDS:
        a, b = initial_field(pp, f), K.initial_field(po, f)
        if f in ("flag", "grain"):
            assert np.array_equal(a, b), f
        else:
            # the two layers evaluate tanh with different libraries (glibc, numpy)
            assert np.max(np.abs(a - b)) <= 4e-16 * max(1.0, np.max(np.abs(b))), (f, np.max(np.abs(a - b)))


def test_ensemble_params_agree():
    for pp, po in zip(ensemble_params(0xE45E, 48, "bf16"), K.ensemble(0xE45E, 48, "bf16")):
        _same_params(pp, po)


def test_ensemble_initial_fields_agree():
    pp, po = ensemble_params(0xE45E, 3, "fp64")[2], K.ensemble(0xE45E, 3, "fp64")[2]
    for f in ("phi", "C", "grain"):
        a, b = initial_field(pp, f), K.initial_field(po, f)
        assert np.max(np.abs(a - b)) <= 4e-16, f


def test_shipped_fixtures_present():
    assert len(SHIPPED) == 11


@pytest.mark.parametrize("path", SHIPPED, ids=os.path.basename)
def test_shipped_case_reads(path):
    # every shipped case resolves identically in both layers; they are 2-D
    # (MeshXYZ ... 1) thermal dendrites (calcMode dendrite = true, flowField = false)
    pp, po = _both(path)
    _same_params(pp, po)
    assert po.nz == 1 and po.model == K.MODEL["thermal_dendrite"]
    assert 1 <= po.n_objects <= 4
    loops, frames = K.read_parameters(path)
    assert (pp.max_loops, pp.max_frames) == (loops, frames)


def test_shipped_solutal_short_centre_list():
    # BoltzTechs - solutal.xml declares two seeds and gives one centre triple:
    # the seed with a complete centre is placed
    path = os.path.join(HERE, "golden", "shipped_cases", "boltztechs_solutal.xml")
    pp, po = _both(path)
    assert pp.n_objects == po.n_objects == 1
    assert list(po.obj_center[0]) == [64.5, 63.5, 0.0]


def test_shipped_thermal_unit_conversion():
    # thermal.xml: mk_dx 0.4, mk_dt 0.008, alphaFluid 4, W0 1, t0 1, d0 0.138486,
    # lambda < 0 (derived), iniValue -0.55
    po = K.resolve(os.path.join(HERE, "golden", "shipped_cases", "boltztechs_thermal.xml"))
    assert po.D == pytest.approx(4.0 * 0.008 / 0.16, rel=1e-15)
    assert po.W0 == pytest.approx(2.5) and po.tau0 == pytest.approx(125.0)
    assert po.lambda_ == pytest.approx(0.8839 / 0.138486, rel=1e-15)
    assert po.delta == pytest.approx(0.55) and po.eps4 == pytest.approx(0.05)
    assert list(po.bc) == [A.MK_BC_CLOSED] * 3


@pytest.mark.skipif(not REFERENCE_CASES, reason="reference tree not present")
@pytest.mark.parametrize("path", REFERENCE_CASES, ids=os.path.basename)
def test_reference_case_files_read(path):
    # the original files (GBK comments under an utf-8 declaration) read in
    # both layers and resolve as their committed fixtures do
    pp, po = _both(path)
    _same_params(pp, po)
    from golden.make_shipped_cases import fixture_name
    fixture = os.path.join(HERE, "golden", "shipped_cases", fixture_name(path))
    _same_params(case_params(fixture), po)


MALFORMED = {
    "unterminated": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry>",
    "mismatched": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geom></MaterKit>",
    "no_mesh": "<MaterKit><output><numLoops> 3 </numLoops></output></MaterKit>",
    "short_mesh": "<MaterKit><geometry><MeshXYZ> 4 4 </MeshXYZ></geometry></MaterKit>",
    "not_a_number": "<MaterKit><geometry><MeshXYZ> 4 four 4 </MeshXYZ></geometry></MaterKit>",
    "fractional_loops": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry>"
                        "<output><numLoops> 2.5 </numLoops></output></MaterKit>",
    "bad_bool": "<MaterKit><calcMode><dendrite> maybe </dendrite></calcMode>"
                "<geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry></MaterKit>",
    "bad_model": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry>"
                 "<b200><model> plasma </model></b200></MaterKit>",
    "bad_boundary": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry>"
                    "<b200><boundary> periodic walls </boundary></b200></MaterKit>",
    "empty_value": "<MaterKit><geometry><MeshXYZ> 4 4 4 </MeshXYZ></geometry>"
                   "<numerics><mk_dx></mk_dx></numerics></MaterKit>",
}


@pytest.mark.parametrize("name", sorted(MALFORMED))
def test_malformed_xml_rejected(casedir, name):
    # host-side fault injection: a corrupt case file is an MK_ERR_XML status
    # (the reference throws mkIOError, MaterKit/xml/mkTINYXMLIO.hh:40), never a crash
    path = cases.write(MALFORMED[name], f"{casedir}/bad_{name}.xml")
    lib = A.load()
    p, o = A.MkParams(), A.MkOptions.make()
    assert lib.mk_case_params(path.encode(), A.C.byref(o), A.C.byref(p)) == A.MK_ERR_XML
    assert lib.mk_last_global_error()
    with pytest.raises(K.CaseError) as ei:
        K.resolve(path)
    assert ei.value.status == A.MK_ERR_XML


def test_missing_file_rejected(casedir):
    lib = A.load()
    p, o = A.MkParams(), A.MkOptions.make()
    assert lib.mk_case_params(f"{casedir}/does_not_exist.xml".encode(), A.C.byref(o), A.C.byref(p)) == A.MK_ERR_XML


def test_invalid_combination_is_arg_error(casedir):
    # a well-formed file with an unsupported combination: MK_ERR_ARG in both layers
    text = cases.poiseuille(nx=8, ny=6, nz=4, collision="MRT", lattice="D3Q27")
    path = cases.write(text, f"{casedir}/bad_combo.xml")
    lib = A.load()
    p, o = A.MkParams(), A.MkOptions.make()
    assert lib.mk_case_params(path.encode(), A.C.byref(o), A.C.byref(p)) == A.MK_ERR_ARG
    with pytest.raises(K.CaseError) as ei:
        K.resolve(path)
    assert ei.value.status == A.MK_ERR_ARG


def test_struct_layouts_agree():
    # the oracle declares mk_params itself; both declarations must match the C header
    assert A.C.sizeof(A.MkParams) == A.C.sizeof(K.MkParams)
    for (na, ta), (nb, tb) in zip(A.MkParams._fields_, K.MkParams._fields_):
        assert na == nb and getattr(A.MkParams, na).offset == getattr(K.MkParams, nb).offset
