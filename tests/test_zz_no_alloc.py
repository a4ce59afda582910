"""The allocation-free statistics entry point, against the handle's own diagnostics.

mk_field_stats_noalloc serves callers that may not call cudaMalloc (their own
pool owns the device memory); its block partials sit in a fixed device array
inside the library.  Here it must reproduce the FP64 phi sum of mk_diagnostics
and the numpy statistics of the same field, on two calls in a row (the second
call reuses the scratch the first one left behind).  The device buffers of the
test itself come from torch; the entry point allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A

pytestmark = pytest.mark.gpu


def _stats(lib, field_dev, n, out_dev):
    st = lib.mk_field_stats_noalloc(C.c_void_p(field_dev.data_ptr()), n, C.c_void_p(out_dev.data_ptr()), None)
    assert st == A.MK_OK, lib.mk_noalloc_last_error().decode()


def test_noalloc_stats_match_diagnostics(tmp_path):
    import torch

    lib = A.load()
    # closed faces: every cell is fluid, so the diagnostics' phi sum covers the whole field
    p = case_params(cases.write(cases.thermal_dendrite(n=40, loops=10, precision="fp32", radius=6.0),
                                str(tmp_path / "dend.xml")))
    s = Solver(params=p)
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    for call in range(2):
        s.advance(7)
        phi = s.field("phi", dtype=np.float32).ravel()
        dev = torch.from_numpy(phi).to("cuda")
        torch.cuda.synchronize()
        _stats(lib, dev, phi.size, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        diag = s.diagnostics()
        ref = phi.astype(np.float64)
        assert abs(got[0] - diag["phi_sum"]) <= 1e-12 * max(1.0, abs(diag["phi_sum"])), (call, got[0], diag)
        assert abs(got[1] - (ref * ref).sum()) <= 1e-12 * (ref * ref).sum()
        assert got[2] == ref.min() and got[3] == ref.max()
        assert got[4] == 0.0


def test_noalloc_rejects_oversize_and_counts_nonfinite():
    import torch

    lib = A.load()
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    big = A.MK_NOALLOC_MAX_CELLS if hasattr(A, "MK_NOALLOC_MAX_CELLS") else 2048 * 256 * 64
    st = lib.mk_field_stats_noalloc(C.c_void_p(out.data_ptr()), big + 1, C.c_void_p(out.data_ptr()), None)
    assert st == A.MK_ERR_ARG
    assert b"MK_NOALLOC_MAX_CELLS" in lib.mk_noalloc_last_error()
    x = torch.tensor([1.0, float("nan"), -2.0, float("inf"), 3.5], dtype=torch.float32, device="cuda")
    _stats(lib, x, 5, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[0] == 2.5 and got[1] == 1.0 + 4.0 + 12.25 and got[2] == -2.0 and got[3] == 3.5 and got[4] == 2.0


def test_noalloc_small_call_after_large_and_empty():
    # a small call right after a large one must not read the block partials
    # the large call left in the shared scratch; n = 0 gives the empty statistics
    import torch

    lib = A.load()
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(7)
    big = rng.standard_normal(5_000_000).astype(np.float32)  # clamps to the full 2048 partial blocks
    small = rng.standard_normal(1000).astype(np.float32) + 3.0  # 4 blocks
    for host in (big, small, big[:257], small):
        dev = torch.from_numpy(host).to("cuda")
        torch.cuda.synchronize()
        _stats(lib, dev, host.size, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = host.astype(np.float64)
        assert abs(got[0] - ref.sum()) <= 1e-12 * np.abs(ref).sum(), (host.size, got[0], ref.sum())
        assert abs(got[1] - (ref * ref).sum()) <= 1e-12 * (ref * ref).sum()
        assert got[2] == ref.min() and got[3] == ref.max() and got[4] == 0.0
    _stats(lib, out, 0, out)  # the field pointer is not read when n = 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert got[0] == 0.0 and got[1] == 0.0 and got[2] == np.inf and got[3] == -np.inf and got[4] == 0.0
