"""The reference-structure CPU baseline (oracle.orc.ReferenceStructure: the
method in the reference's node-object layout, mkNode, with schedule(static,
16) node sweeps) is the oracle's method bit for bit: the flow model in every
collision operator, the thermal dendrite with three anisotropy kinds and an
off-centre seed."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases
from oracle.case import resolve as case_params
from oracle.orc import ReferenceStructure
from _oracle import Oracle


def _params(casedir, name, text, **opt):
    return case_params(cases.write(text, f"{casedir}/{name}.xml"), **opt)


@pytest.mark.parametrize("coll", ["BGK", "TRT", "MRT"])
def test_flow_bitwise(casedir, coll):
    p = _params(casedir, f"aos_pois_{coll}", cases.poiseuille(nx=10, ny=12, nz=8, loops=1, collision=coll,
                                                            force=1e-5))
    o = Oracle(p)
    a = ReferenceStructure(o)
    for n in (1, 7):
        o.advance(n)
        a.advance(n)
        assert np.array_equal(a.populations(0), o.populations(0)), (coll, n)


@pytest.mark.parametrize("aniso", ["cubic", "hcp", "facet"])
def test_thermal_dendrite_bitwise(casedir, aniso):
    text = cases.thermal_dendrite(n=20, loops=1, aniso=aniso, eps2=0.02 if aniso != "cubic" else 0.0,
                                  center=(9.0, 10.5, 8.5))
    p = _params(casedir, f"aos_dend_{aniso}", text)
    o = Oracle.from_case(p)
    a = ReferenceStructure(o)
    for n in (1, 5):
        o.advance(n)
        a.advance(n)
        assert np.array_equal(a.field("phi"), o.field("phi")), n
        assert np.array_equal(a.field("T"), o.field("T")), n
        assert np.array_equal(a.populations(0), o.populations(0)), n
        assert np.array_equal(a.populations(1), o.populations(1)), n


def test_other_models_refused(casedir):
    p = _params(casedir, "aos_mp", cases.multiphase_bubbles(n=16, bubbles=0, precision="fp64", loops=1))
    with pytest.raises(ValueError):
        ReferenceStructure(Oracle.from_case(p))


def test_node_is_the_reference_node_size():
    # eleven 19-value population vectors (f, g, h, x and the helpers), the
    # scalar fields and nine (empty) vector members
    assert ReferenceStructure.node_bytes() >= 11 * 19 * 8 + 30 * 8
