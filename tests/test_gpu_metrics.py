"""The JSON-lines metrics log (mk_set_metrics_log): timed advances report
MLUPS and the algorithmic GB/s, diagnostics report the conservation sums and
their drift from the handle's first diagnostics."""
import json

import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

pytestmark = pytest.mark.gpu


def test_metrics_log_lines(casedir, tmp_path):
    lib = A.load()
    log = tmp_path / "metrics.jsonl"
    assert lib.mk_set_metrics_log(str(log).encode()) == A.MK_OK
    try:
        p = case_params(cases.write(cases.multiphase_bubbles(n=32, bubbles=1, rmin=4, rmax=5, width=2.0,
                                                             precision="fp32", loops=10), f"{casedir}/met.xml"))
        s = Solver(params=p)
        d0 = s.diagnostics()
        ms = s.time_advance(10, graph=True)
        d1 = s.diagnostics()
        s.close()
    finally:
        lib.mk_set_metrics_log(None)
    lines = [json.loads(x) for x in log.read_text().splitlines()]
    assert [x["event"] for x in lines] == ["diagnostics", "time_advance", "diagnostics"]
    t = lines[1]
    assert t["loops"] == 10 and t["step"] == 10 and t["model"] == A.MK_MODEL_MULTIPHASE
    assert t["ms"] == pytest.approx(ms, rel=1e-6)
    assert t["mlups"] == pytest.approx(p.ncell() * 10 / (ms * 1e-3) / 1e6, rel=1e-6)
    assert t["gbs"] == pytest.approx(312.0 * p.ncell() * 10 / (ms * 1e-3) / 1e9, rel=1e-6)
    assert lines[0]["phi_drift"] == 0.0
    assert lines[2]["phi_sum"] == pytest.approx(d1["phi_sum"], rel=1e-15)
    assert lines[2]["phi_drift"] == pytest.approx((d1["phi_sum"] - d0["phi_sum"]) / d0["phi_sum"], abs=1e-15)
    assert abs(lines[2]["phi_drift"]) < 1e-6
