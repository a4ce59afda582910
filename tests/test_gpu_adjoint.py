"""Discrete adjoint of the thermal dendrite loop on the device (mk_backward).

The device reverse sweep must equal the oracle's (the same formulas, whose
exactness is pinned against central differences in the CPU suite), match
central differences of the device forward run itself, and do so at the full
configuration-5 size (96^3, 2000 loops, checkpoints every 100 loops): loss
||phi_T - phi_target||^2 with the target produced at (eps4, Delta) =
(0.04, 0.50) and the gradient taken at (0.05, 0.55), FD step h = 1e-4,
relative agreement <= 1e-4.
"""
import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, cases, case_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from _oracle import Oracle

pytestmark = pytest.mark.gpu


def _params(casedir, n, eps4, delta, precision="fp64", aniso="cubic", eps2=0.0, radius=3.0):
    return case_params(cases.write(cases.thermal_dendrite(n=n, loops=1, radius=radius, eps4=eps4, delta=delta,
                                                          precision=precision, aniso=aniso, eps2=eps2),
                                   f"{casedir}/adj_{n}_{precision}_{aniso}.xml"))


def _phi_after(p, steps):
    s = Solver(params=p)
    s.advance(steps, graph=True)
    phi = s.field("phi")
    s.close()
    return phi


def _fd(casedir, n, steps, p0, target, radius, h=1e-4, precision="fp64"):
    def loss(p):
        p.tau0 = p0.tau0
        return float(((_phi_after(p, steps) - target) ** 2).sum())

    def mk(eps4, delta):
        return _params(casedir, n, eps4, delta, precision=precision, aniso=_aniso_name(p0), eps2=p0.eps2,
                       radius=radius)

    e4, d = p0.eps4, p0.delta
    fd = {"d_eps4": (loss(mk(e4 + h, d)) - loss(mk(e4 - h, d))) / (2 * h),
          "d_delta": (loss(mk(e4, d + h)) - loss(mk(e4, d - h))) / (2 * h)}
    pp, pm = mk(e4, d), mk(e4, d)
    pp.D += h / 4  # tau_T = 4 D + 1/2
    pm.D -= h / 4
    fd["d_tau_t"] = (loss(pp) - loss(pm)) / (2 * h)
    return fd


def _aniso_name(p):
    return {v: k for k, v in A.ANISOTROPIES.items()}[p.aniso]


@pytest.mark.parametrize("aniso,e2", [("cubic", 0.0), ("facet", 0.03), ("hcp", 0.02)])
def test_device_adjoint_equals_oracle_adjoint(casedir, aniso, e2):
    n, steps = 14, 23
    target = _phi_after(_params(casedir, n, 0.04, 0.50, aniso=aniso, eps2=e2), steps)
    p = _params(casedir, n, 0.05, 0.55, aniso=aniso, eps2=e2)
    s = Solver(params=p)
    g = s.backward(target, steps, checkpoint_every=6)  # 4 segments, the last one partial
    o = Oracle.from_case(p)  # the oracle's own initial fields of the same parameters
    r = o.backward(target, steps)
    for k in ("loss", "d_eps4", "d_delta", "d_tau_t"):
        assert g[k] == pytest.approx(r[k], rel=1e-9, abs=1e-12), (k, g[k], r[k])
    assert g["forward_loops"] == steps + steps - 1
    # the handle is left after the forward run
    assert s.step == steps
    np.testing.assert_array_equal(s.field("phi"), _phi_after(p, steps))
    s.close()


def test_device_adjoint_matches_device_central_differences(casedir):
    n, steps = 24, 80
    target = _phi_after(_params(casedir, n, 0.04, 0.50, radius=4.0), steps)
    p = _params(casedir, n, 0.05, 0.55, radius=4.0)
    g = Solver(params=p).backward(target, steps, checkpoint_every=25)
    fd = _fd(casedir, n, steps, p, target, radius=4.0)
    for k in fd:
        assert g[k] == pytest.approx(fd[k], rel=1e-4), (k, g[k], fd[k])


def test_config5_full_size_gradients(casedir):
    # 96^3, 2000 loops, checkpoints every 100 loops, seed radius 8
    n, steps = 96, 2000
    target = _phi_after(_params(casedir, n, 0.04, 0.50, radius=8.0), steps)
    p = _params(casedir, n, 0.05, 0.55, radius=8.0)
    g = Solver(params=p).backward(target, steps, checkpoint_every=100)
    assert g["loss"] > 0
    fd = _fd(casedir, n, steps, p, target, radius=8.0)
    for k in fd:
        assert g[k] == pytest.approx(fd[k], rel=1e-4), (k, g[k], fd[k])


def test_fp32_storage_adjoint_close_to_fp64(casedir):
    n, steps = 16, 40
    target = _phi_after(_params(casedir, n, 0.04, 0.50), steps)
    g64 = Solver(params=_params(casedir, n, 0.05, 0.55)).backward(target, steps, checkpoint_every=10)
    g32 = Solver(params=_params(casedir, n, 0.05, 0.55, precision="fp32")).backward(target, steps,
                                                                                     checkpoint_every=10)
    for k in ("loss", "d_eps4", "d_delta", "d_tau_t"):
        assert g32[k] == pytest.approx(g64[k], rel=2e-3), (k, g32[k], g64[k])


def test_backward_rejects_unsupported_cases(casedir):
    p = case_params(cases.write(cases.solutal_dendrite(n=16, loops=1, precision="fp64"), f"{casedir}/adj_sol.xml"))
    s = Solver(params=p)
    with pytest.raises(A.MkError, match="thermal dendrite"):
        s.backward(np.zeros(p.ncell()), 4)
    p16 = _params(casedir, 16, 0.05, 0.55, precision="fp16")
    with pytest.raises(A.MkError, match="FP64 or FP32"):
        Solver(params=p16).backward(np.zeros(p16.ncell()), 4)
