"""The seeded random cases of every model (tests/_random_cases.py: random
sizes with one-cell axes, random faces per axis, random collision, lattice,
anisotropy and contact-angle variants) on the device in FP64 against the
oracle, through the C ABI: every compared field to 1e-10 relative L2 on the
fluid cells after 1, 2 and 5 loops (both AA parities and their repeats), and
with FP32 / FP16 / BF16 storage within the tolerances below after 5 loops."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases, case_params
from _oracle import Oracle, rel_l2
import _random_cases as R

pytestmark = pytest.mark.gpu

# a pressure that starts at rest is rounding noise for the first loops; a
# velocity component is judged against the flow's speed (a component that
# vanishes, across a driven channel, is rounding noise of that speed)
FLOOR = {"pressure": 1e-9}
VEL = ("ux", "uy", "uz")


@pytest.mark.parametrize("k", range(R.N_CASES))
def test_random_shape_matches_oracle(casedir, k):
    name, xml, fields = R.case(k)
    path = cases.write(xml, f"{casedir}/rnd_{name}.xml")
    s, o = Solver(params=case_params(path)), Oracle.from_xml(path)
    fl = o.field("flag") == 0
    ngr = s.params.n_objects if name.endswith("multigrain") else 0
    for n in (1, 1, 3):
        s.advance(n)
        o.advance(n)
        ref = {f: o.field(f) for f in fields}
        speed = max([float(np.max(np.abs(ref[f][fl]))) for f in VEL if f in ref] + [0.0])
        errs = {f: rel_l2(s.field(f), ref[f], fl, floor=speed if f in VEL else FLOOR.get(f, 0.0)) for f in fields}
        for j in range(ngr):
            errs[f"phi{j}"] = rel_l2(s.grain_field(j), o.grain(j), fl)
        bad = {f: e for f, e in errs.items() if not e <= 1e-10}
        assert not bad, (name, s.step, bad)


# about 4x the largest error over the 32 cases after 5 loops (FP32 1.1e-6,
# FP16 2.6e-3, BF16 1.45e-2: the vertical velocity of a convection cell)
REDUCED = {"fp32": 5e-6, "fp16": 1e-2, "bf16": 5e-2}


@pytest.mark.parametrize("prec", sorted(REDUCED))
@pytest.mark.parametrize("k", range(R.N_CASES))
def test_random_shape_reduced_storage(casedir, k, prec):
    # the same cases with FP32 / 16-bit storage against the FP64 oracle
    name, xml, fields = R.case(k)
    xml = xml.replace("<precision> fp64 </precision>", f"<precision> {prec} </precision>")
    assert f"<precision> {prec} </precision>" in xml
    path = cases.write(xml, f"{casedir}/rnd_{name}_{prec}.xml")
    s, o = Solver(params=case_params(path)), Oracle.from_xml(path)
    fl = o.field("flag") == 0
    s.advance(5)
    o.advance(5)
    ref = {f: o.field(f) for f in fields}
    speed = max([float(np.max(np.abs(ref[f][fl]))) for f in VEL if f in ref] + [0.0])
    errs = {f: rel_l2(s.field(f), ref[f], fl, floor=speed if f in VEL else FLOOR.get(f, 0.0)) for f in fields}
    bad = {f: e for f, e in errs.items() if not e <= REDUCED[prec]}
    assert not bad, (name, prec, bad)
