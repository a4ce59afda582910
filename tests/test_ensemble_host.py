"""Host-side logic of the dendrite ensemble: the seeded generator and the
argument checks of mk_ensemble_create (no GPU needed)."""
import ctypes as C

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import ensemble_params
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from conftest import HAVE_GPU


def test_generator_is_deterministic_and_in_range():
    a = ensemble_params(0xE45E, 48, "bf16")
    b = ensemble_params(0xE45E, 48, "bf16")
    c = ensemble_params(0xE45F, 48, "bf16")
    assert bytes(memoryview(a[7])) == bytes(memoryview(b[7]))
    assert any(bytes(memoryview(x)) != bytes(memoryview(y)) for x, y in zip(a, c))
    edges = set()
    for p in a:
        assert p.model == A.MK_MODEL_SOLUTAL_DENDRITE and p.precision == A.MK_PREC_BF16
        assert p.nx == p.ny == p.nz and p.nx in (48, 64, 80, 96, 128)
        assert p.ncell() % 256 == 0
        edges.add(p.nx)
        assert 0.02 <= p.eps4 <= 0.06
        assert 1 <= p.n_objects <= 6
        assert list(p.bc) == [A.MK_BC_CLOSED] * 3
        assert p.k_part == 0.15 and p.D == 0.1 and p.D_s == 1e-4
        for s in range(p.n_objects):
            r = p.obj_radius[s]
            assert 4.0 <= r <= 8.0
            for a_ in range(3):
                assert r + 2.0 - 1e-9 <= p.obj_center[s][a_] <= p.nx - 1 - (r + 2.0) + 1e-9
                assert -180.0 <= p.obj_angle[s][a_] <= 180.0
    assert len(edges) >= 4  # 48 draws cover the edge set


def test_generator_orientations_are_spread():
    ps = ensemble_params(1, 400, "fp32")
    ay = np.array([p.obj_angle[s][1] for p in ps for s in range(p.n_objects)])
    # a uniform rotation has sin(ay) ~ U[-1, 1]
    sy = np.sin(np.radians(ay))
    assert abs(sy.mean()) < 0.1 and 0.25 < sy.var() < 0.42


def _create(ps):
    lib = A.load()
    arr = (A.MkParams * len(ps))(*ps)
    h = C.c_void_p()
    st = lib.mk_ensemble_create(arr, len(ps), C.byref(h))
    msg = lib.mk_last_global_error().decode()
    if st == A.MK_OK:
        lib.mk_ensemble_destroy(h)
    return st, msg


def test_create_rejects_mixed_models_and_ragged_domains():
    ps = ensemble_params(5, 3, "fp32")
    ps[1].model = A.MK_MODEL_THERMAL_DENDRITE
    st, msg = _create(ps)
    assert st == A.MK_ERR_ARG and "model" in msg
    ps = ensemble_params(5, 3, "fp32")
    ps[2].precision = A.MK_PREC_FP64
    st, msg = _create(ps)
    assert st == A.MK_ERR_ARG and "precision" in msg
    ps = ensemble_params(5, 3, "fp32")
    ps[0].nx = ps[0].ny = ps[0].nz = 47  # 47^3 cells: not whole 256-cell tiles
    ps[0].n_objects = 1
    ps[0].obj_center[0][0] = ps[0].obj_center[0][1] = ps[0].obj_center[0][2] = 20.0
    st, msg = _create(ps)
    assert st == A.MK_ERR_ARG and "multiple of 256" in msg
    ps = ensemble_params(5, 2, "fp32")
    ps[0].model = A.MK_MODEL_FLOW
    ps[1].model = A.MK_MODEL_FLOW
    st, msg = _create(ps)
    assert st == A.MK_ERR_ARG


def test_generator_rejects_bad_arguments():
    lib = A.load()
    out = (A.MkParams * 1)()
    assert lib.mk_ensemble_case_params(1, 0, A.MK_PREC_FP32, out) == A.MK_ERR_ARG
    assert lib.mk_ensemble_case_params(1, 1, 9, out) == A.MK_ERR_ARG


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device path")
def test_create_without_device():
    st, msg = _create(ensemble_params(5, 2, "fp32"))
    assert st == A.MK_ERR_NODEVICE and "device" in msg
