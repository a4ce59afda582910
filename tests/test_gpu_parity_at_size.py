"""FP64 parity with the oracle at the benchmark configurations' own sizes.

The library and the oracle each resolve the case through their own case layer
(library: mk_case_params / its initial fields; oracle: oracle/case.py), run in
FP64 storage, and must agree to 1e-10 relative L2 per field:

* configuration 3 (the headline): 256^3 bubbles, 24 bubbles, D3Q19 MRT +
  D3Q19 Allen-Cahn, after 1, 2 and 6 loops (both AA parities);
* configuration 2: 128^3 thermal dendrite after 60 loops;
* configuration 4: the first six domains of the 48-domain solutal ensemble
  (edges 96, 64, 128, 128, 96, 48; 1-6 rotated seeds each), packed in one
  ensemble, after 30 loops.

Configuration 1 (64x32x32, 2000 loops) and configuration 5 (96^3 adjoint,
2000 loops) are checked at size in test_gpu_parity and test_gpu_adjoint.
"""
import os

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Ensemble, Solver, case_params, cases, ensemble_params
from _oracle import Oracle, ocase, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _vel_err(s, o, mask):
    a = np.stack([s.field(f)[mask] for f in ("ux", "uy", "uz")])
    b = np.stack([o.field(f)[mask] for f in ("ux", "uy", "uz")])
    return rel_l2(a, b)


def test_config3_bubbles_256_fp64(casedir):
    path = cases.write(cases.multiphase_bubbles(n=256, precision="fp64"), f"{casedir}/c3_256.xml")
    s = Solver(params=case_params(path))
    o = Oracle.from_xml(path)
    fl = ocase.flags(o.params) == 0
    for n in (1, 1, 4):
        s.advance(n)
        o.advance(n)
        errs = {f: rel_l2(s.field(f), o.field(f), fl) for f in ("phi", "rho")}
        errs["pressure"] = rel_l2(s.field("pressure"), o.field("pressure"), fl, 1e-9)
        errs["u"] = _vel_err(s, o, fl)
        print(f"256^3 bubbles FP64, loop {s.step}: {errs}")
        assert all(v <= TOL for v in errs.values()), (s.step, errs)
    s.close()
    o.close()


def test_config2_dendrite_128_fp64(casedir):
    path = cases.write(cases.thermal_dendrite(n=128, precision="fp64"), f"{casedir}/c2_128.xml")
    s = Solver(params=case_params(path))
    o = Oracle.from_xml(path)
    for n in (1, 59):
        s.advance(n, graph=n > 1)
        o.advance(n)
        errs = {f: rel_l2(s.field(f), o.field(f)) for f in ("phi", "T", "dphi")}
        print(f"128^3 thermal dendrite FP64, loop {s.step}: {errs}")
        assert all(v <= TOL for v in errs.values()), (s.step, errs)
    s.close()


def test_config4_ensemble_domains_fp64():
    nd = 6
    ens = Ensemble(ensemble_params(0xE45E, nd, "fp64"))
    oracles = [Oracle.from_case(p) for p in ocase.ensemble(0xE45E, nd, "fp64")]
    assert [o.params.nx for o in oracles] == [96, 64, 128, 128, 96, 48]
    ens.advance(30)
    for o in oracles:
        o.advance(30)
    for d, o in enumerate(oracles):
        errs = {f: rel_l2(ens.field(d, f), o.field(f)) for f in ("phi", "C", "dphi")}
        assert all(v <= TOL for v in errs.values()), (d, errs)
        assert np.array_equal(ens.field(d, "grain"), o.field("grain")), d
    ens.close()
