"""The seeded random cases of the shape sweep (tests/_random_cases.py: every
model, random sizes with one-cell axes, random faces and variants) read the
same in the library's case layer and the oracle's (parameters exactly,
initial fields to 4e-16), and the oracle advances each of them without
non-finite values.  No GPU is needed."""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases, case_params, initial_field
from oracle import case as K
from _oracle import Oracle
import _random_cases as R

FIELDS = ["phi", "rho", "ux", "uy", "uz", "T", "C", "flag", "pressure", "dphi", "grain"]


@pytest.mark.parametrize("k", range(R.N_CASES))
def test_random_case_reads_alike(casedir, k):
    name, xml, fields = R.case(k)
    path = cases.write(xml, f"{casedir}/rnd_{name}.xml")
    pp, po = case_params(path), K.resolve(path)
    a, b = pp.to_dict(), po.values()
    diff = {f: (a[f], b[f]) for f in a if a[f] != b[f]}
    assert not diff, (name, diff)
    for f in FIELDS:
        x, y = initial_field(pp, f), K.initial_field(po, f)
        if f in ("flag", "grain"):
            assert np.array_equal(x, y), (name, f)
        else:
            assert np.max(np.abs(x - y)) <= 4e-16 * max(1.0, np.max(np.abs(y))), (name, f)
    o = Oracle.from_xml(path)
    o.advance(3)
    for f in fields:
        assert np.isfinite(o.field(f)).all(), (name, f)
