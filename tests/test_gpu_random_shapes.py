"""The seeded random cases of every model (tests/_random_cases.py: random
sizes with one-cell axes, random faces per axis, random collision, lattice,
anisotropy and contact-angle variants) on the device in FP64 against the
oracle, through the C ABI: every compared field to 1e-10 relative L2 on the
fluid cells after 1, 2 and 5 loops (both AA parities and their repeats)."""
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
