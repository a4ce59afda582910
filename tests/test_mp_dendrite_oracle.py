"""The oracle's coupling of a thermal dendrite and a two-phase flow of one grid
(run_flow_multiphase_dendrite, MaterKit/MaterKit.cpp:377-397): the flow's
cells under the dendrite's solid turn solid at even loop counts and stay
solid, solid cells leave the flow's update, and the dendrite's thermal
lattice is advected by the flow's velocity."""
import numpy as np

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases
from oracle.case import flags as oflags, resolve as case_params
from _oracle import Oracle


def _pair(casedir, n=20):
    pf = case_params(cases.write(cases.multiphase_bubbles(n=n, bubbles=1, rmin=3.0, rmax=3.5, width=2.0,
                                                          gz=-1e-5, precision="fp64", loops=10),
                                 f"{casedir}/mpd_flow.xml"))
    pd = case_params(cases.write(cases.thermal_dendrite(n=n, loops=10, precision="fp64", radius=4.0,
                                                        center=(n / 2.0 - 0.5, n / 2.0 - 0.5, n / 3.0)),
                                 f"{casedir}/mpd_dend.xml"))
    return Oracle.from_case(pf), Oracle.from_case(pd)


def _solid(o):
    return o.field("flag") == 2


def test_coupling_semantics(casedir):
    f, d = _pair(casedir)
    solid_before = None
    for loop in range(8):
        d.update_velocity(f)
        d.advance(1)
        f.update_geometry(d)
        s = _solid(f)
        if f.step % 2 == 1:
            # applied only at even counts: nothing changed since the last one
            assert solid_before is not None and np.array_equal(s, solid_before)
        else:
            # every solid cell lies under the dendrite's solid or was solid before
            under = d.field("phi") > 0
            assert np.all(s <= (under | (solid_before if solid_before is not None else under)))
        if solid_before is not None:
            assert np.all(s >= solid_before)  # cumulative
        solid_before = s
        f.advance(1)
    assert solid_before.sum() > 0


def test_velocity_advects_the_thermal_lattice(casedir):
    f, d = _pair(casedir)
    _, d2 = _pair(casedir)
    f.advance(6)  # a flow with a velocity field
    d.update_velocity(f)
    d.advance(4)
    d2.advance(4)
    assert np.abs(d.field("T") - d2.field("T")).max() > 0
