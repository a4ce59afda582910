"""The z-slab decomposition of one multiphase domain on the device: slab
handles advanced together through the library's exchange protocol equal the
whole-domain handle bit for bit (every storage precision, periodic, walled
and closed z, one to three slabs, ragged splits), the protocol refuses
out-of-order calls, the slab diagnostics add up to the whole domain's, and
two gloo processes sharing the device reproduce the whole run through the
Python runner (host-staged exchanges; the kernels of the two processes never
wait on each other).  The NCCL transport runs its one-rank form (a periodic
axis trading with itself, the diagnostics all-reduce on the device)."""
import ctypes as C
import datetime
import os
import socket
import sys

import numpy as np
import pytest

from materkit_anisotropiclbm_trt_rbc_facet_b200 import Solver, case_params, cases
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as S

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FIELDS = ["phi", "rho", "pressure", "ux", "uy", "uz"]

SHAPES = {
    # name: (nx, ny, nz, boundary, bubbles, contact angle)
    "walls_z": (32, 32, 24, "periodic periodic walls", 2, 90.0),
    "periodic_xyz": (40, 28, 20, "periodic periodic periodic", 2, 90.0),
    "closed_z_ragged": (36, 23, 17, "walls periodic closed", 1, 60.0),
}


def _params(casedir, name, prec):
    nx, ny, nz, bc, nb, th = SHAPES[name]
    text = cases.multiphase_bubbles(n=nx, ny=ny, nz=nz, bubbles=nb, rmin=3.0, rmax=4.0, width=2.0, gz=-1e-5,
                                    precision=prec, loops=10, boundary=bc, contact_angle=th)
    return case_params(cases.write(text, f"{casedir}/slab_{name}_{prec}.xml"))


def _owned(slabs, f):
    return np.concatenate([s.owned(f) for s in slabs], axis=0)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp16", "bf16"])
@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("name", sorted(SHAPES))
def test_slabs_equal_whole_domain(casedir, name, n, prec):
    p = _params(casedir, name, prec)
    whole = Solver(params=p)
    slabs = [S.Slab(p, r, n) for r in range(n)]
    assert sum(s.nz_own for s in slabs) == p.nz
    assert all(s.params.nz == s.nz_own + 2 for s in slabs)
    for f in FIELDS:
        assert np.array_equal(_owned(slabs, f), whole.field(f)), ("initial", f)
    for k in (1, 1, 3, 4):  # odd and even counts: both AA parities end a call
        whole.advance(k)
        S.advance_local(slabs, k)
        assert all(s.step == whole.step for s in slabs)
        for f in FIELDS:
            x, y = _owned(slabs, f), whole.field(f)
            assert np.array_equal(x, y), (name, n, prec, whole.step, f, float(np.nanmax(np.abs(x - y))))


def test_slab_diagnostics_add_up(casedir):
    p = _params(casedir, "walls_z", "fp64")
    whole = Solver(params=p)
    slabs = [S.Slab(p, r, 3) for r in range(3)]
    whole.advance(9)
    S.advance_local(slabs, 9)
    parts = [s.diag_sums() for s in slabs]
    d = S.combine(sum(a for a, _ in parts), max(b for _, b in parts))
    w = whole.diagnostics()
    assert d["fluid_cells"] == whole.fluid_cells() == sum(s.fluid_cells() for s in slabs)
    for k in ("mass", "phi_sum"):
        assert d[k] == pytest.approx(w[k], rel=1e-12), k
    assert d["momentum"] == pytest.approx(w["momentum"], abs=1e-12)
    assert d["solid_frac"] == pytest.approx(w["solid_frac"], rel=1e-12)
    assert d["max_speed"] == w["max_speed"]


def test_protocol_refuses_out_of_order(casedir):
    lib = A.load()
    p = _params(casedir, "periodic_xyz", "fp32")
    s = S.Slab(p, 0, 2)
    t = S.Slab(p, 1, 2)
    assert s.next() == A.MK_SLAB_RETURN
    # the whole-domain entry points are closed on a slab handle
    for call in (lambda: lib.mk_advance(s.handle, 1), lambda: lib.mk_advance_graph(s.handle, 2),
                 lambda: lib.mk_set_fused(s.handle, 1), lambda: lib.mk_checkpoint(s.handle, b"/tmp/x.ck")):
        assert call() == A.MK_ERR_STATE
    assert lib.mk_slab_run(s.handle, A.MK_SLAB_RUN_PHI) == A.MK_ERR_STATE
    assert lib.mk_slab_done(s.handle, A.MK_SLAB_PHI) == A.MK_ERR_STATE
    assert b"MK_SLAB_RETURN" in lib.mk_last_error(s.handle)
    arr = (C.c_void_p * 2)(t.handle, s.handle)  # ranks out of place
    assert lib.mk_slab_exchange_local(arr, 2, A.MK_SLAB_RETURN) == A.MK_ERR_ARG
    arr = (C.c_void_p * 2)(s.handle, t.handle)
    assert lib.mk_slab_exchange_local(arr, 2, A.MK_SLAB_FILL) == A.MK_ERR_STATE
    assert lib.mk_slab_exchange_local(arr, 2, A.MK_SLAB_RETURN) == A.MK_OK
    assert s.next() == A.MK_SLAB_RUN_PHI
    s.run(A.MK_SLAB_RUN_PHI)
    assert s.next() == A.MK_SLAB_PHI
    assert lib.mk_slab_run(s.handle, A.MK_SLAB_RUN_COLLIDE) == A.MK_ERR_STATE
    # the slab calls are closed on a whole-domain handle
    w = Solver(params=p)
    assert lib.mk_slab_next(w.handle) == -1
    assert lib.mk_slab_run(w.handle, A.MK_SLAB_RUN_PHI) == A.MK_ERR_STATE
    n = C.c_int32()
    assert lib.mk_slab_transfers(w.handle, A.MK_SLAB_FILL, None, 0, C.byref(n)) == A.MK_ERR_STATE


def test_create_slab_checks(casedir):
    lib = A.load()
    p = _params(casedir, "walls_z", "fp32")
    h = C.c_void_p()
    assert lib.mk_create_slab(C.byref(p), 0, p.nz + 1, C.byref(h)) == A.MK_ERR_ARG
    assert lib.mk_create_slab(C.byref(p), 3, 3, C.byref(h)) == A.MK_ERR_ARG
    q = case_params(cases.write(cases.poiseuille(nx=8, ny=6, nz=6), f"{casedir}/slab_pois.xml"))
    assert lib.mk_create_slab(C.byref(q), 0, 2, C.byref(h)) == A.MK_ERR_ARG
    assert b"multiphase" in lib.mk_last_global_error()


def test_transfers_point_into_the_slab_arrays(casedir):
    p = _params(casedir, "closed_z_ragged", "bf16")
    s = S.Slab(p, 1, 3)
    host = S.plan(p, 1, 3, A.MK_SLAB_FILL)
    dev = s.transfers(A.MK_SLAB_FILL)
    assert [(x.peer, x.tag, x.send, x.offset, x.bytes) for x in host] == \
           [(x.peer, x.tag, x.send, x.offset, x.bytes) for x in dev]
    assert all(x.ptr for x in dev)
    assert len(dev) == 40 and all(x.bytes == p.nx * p.ny * 2 for x in dev)


# ------------------------------------------------------- processes on one device
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, backend, xml, loops, q):
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import case_params as cp
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as SL
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        p = cp(xml)
        s = SL.Slab(p, rank, ws)
        run = SL.SlabRun(s, SL.TorchTransport())
        run.advance(loops // 2)
        run.advance(loops - loops // 2)
        q.put((rank, run.gather("phi"), run.gather("ux"), run.diagnostics()))
        s.close()
    finally:
        dist.destroy_process_group()


def _spawn(ws, backend, xml, loops):
    import torch.multiprocessing as mp
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, backend, xml, loops, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=300) for _ in range(ws)), key=lambda t: t[0])
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return res


@pytest.mark.parametrize("name", ["periodic_xyz", "walls_z"])
def test_two_gloo_processes_equal_whole_domain(casedir, name):
    p = _params(casedir, name, "fp64")
    xml = f"{casedir}/slab_{name}_fp64.xml"
    loops = 7
    whole = Solver(params=p)
    whole.advance(loops)
    ref_phi, ref_ux = whole.field("phi"), whole.field("ux")
    wd = whole.diagnostics()
    whole.close()
    for rank, phi, ux, d in _spawn(2, "gloo", xml, loops):
        assert np.array_equal(phi, ref_phi), rank
        assert np.array_equal(ux, ref_ux), rank
        assert d["mass"] == pytest.approx(wd["mass"], rel=1e-12)
        assert d["fluid_cells"] == int(np.prod(ref_phi.shape)) - (2 * p.nx * p.ny if name == "walls_z" else 0)


def test_nccl_one_rank_periodic(casedir):
    p = _params(casedir, "periodic_xyz", "fp32")
    xml = f"{casedir}/slab_periodic_xyz_fp32.xml"
    loops = 6
    whole = Solver(params=p)
    whole.advance(loops)
    ref = whole.field("phi")
    wd = whole.diagnostics()
    whole.close()
    (_, phi, _, d), = _spawn(1, "nccl", xml, loops)
    assert np.array_equal(phi, ref)
    assert d["phi_sum"] == pytest.approx(wd["phi_sum"], rel=1e-12)
