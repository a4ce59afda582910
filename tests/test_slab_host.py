"""The z-slab decomposition on the CPU: the library's host-only transfer plan
(mk_slab_plan) and the Python runner (slab.SlabRun / TorchTransport) drive a
NumPy model of the library's AA streaming, in one process and as two or
three gloo ranks, and the split run equals the whole-domain run bit for bit
in FP64."""
import datetime
import os
import socket
import sys

import numpy as np
import pytest

from _slab_model import EZ, AAModel, global_params, plan_counts, pop_stride, whole_run
from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as S

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STAGES = (A.MK_SLAB_FILL, A.MK_SLAB_PHI, A.MK_SLAB_RETURN)
BCS = (A.MK_BC_PERIODIC, A.MK_BC_WALLS, A.MK_BC_CLOSED)


# ------------------------------------------------------------------ split
@pytest.mark.parametrize("nz,n", [(16, 1), (16, 2), (17, 3), (9, 4), (5, 5), (256, 8), (130, 7)])
def test_split_covers_the_domain_in_order(nz, n):
    parts = [S.split(nz, r, n) for r in range(n)]
    assert parts[0][0] == 0
    for (z0, k), (z1, _) in zip(parts, parts[1:]):
        assert z1 == z0 + k
    assert sum(k for _, k in parts) == nz
    assert max(k for _, k in parts) - min(k for _, k in parts) <= 1


@pytest.mark.parametrize("nz,r,n", [(4, 0, 5), (8, 2, 2), (8, -1, 2), (8, 0, 0)])
def test_split_rejects(nz, r, n):
    with pytest.raises(A.MkError) as e:
        S.split(nz, r, n)
    assert e.value.status == A.MK_ERR_ARG


# ------------------------------------------------------------------ plan
# local plane of each kind of run: (stage, upward, send) -> plane(nown)
PLANE = {
    (A.MK_SLAB_FILL, True, True): lambda n: n, (A.MK_SLAB_FILL, True, False): lambda n: 0,
    (A.MK_SLAB_FILL, False, True): lambda n: 1, (A.MK_SLAB_FILL, False, False): lambda n: n + 1,
    (A.MK_SLAB_PHI, True, True): lambda n: n, (A.MK_SLAB_PHI, True, False): lambda n: 0,
    (A.MK_SLAB_PHI, False, True): lambda n: 1, (A.MK_SLAB_PHI, False, False): lambda n: n + 1,
    (A.MK_SLAB_RETURN, True, True): lambda n: n + 1, (A.MK_SLAB_RETURN, True, False): lambda n: 1,
    (A.MK_SLAB_RETURN, False, True): lambda n: 0, (A.MK_SLAB_RETURN, False, False): lambda n: n,
}


def _lists(p, n, stage):
    return [S.plan(p, r, n, stage) for r in range(n)]


@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("prec", [A.MK_PREC_FP64, A.MK_PREC_FP32, A.MK_PREC_BF16])
def test_plan_matches_sends_with_receives(bc, n, prec):
    p = global_params(6, 5, 11, bc)
    p.precision = prec
    elem = {A.MK_PREC_FP64: 8, A.MK_PREC_FP32: 4}.get(prec, 2)
    pelem = 8 if prec == A.MK_PREC_FP64 else 4
    for stage in STAGES:
        lists = _lists(p, n, stage)
        for r, xs in enumerate(lists):
            z0, nown = S.split(p.nz, r, n)
            plane, stride = p.nx * p.ny, pop_stride(p.nx * p.ny * (nown + 2))
            keys = [(x.peer, x.tag, x.send) for x in xs]
            assert keys == sorted(keys)
            for x in xs:
                assert x.count == plane and x.ptr is None
                assert x.bytes == plane * (pelem if x.array == 2 else elem)
                upward = x.tag < 128
                if x.array == 3:
                    # a return run lands in the halo buffer: face 0 (from below) holds
                    # the e_z = +1 runs, face 1 the e_z = -1 runs, in population order
                    assert stage == A.MK_SLAB_RETURN and not x.send
                    face, lat, k = np.unravel_index(x.offset // plane, (2, 2, 5))
                    assert x.offset % plane == 0 and face == (0 if upward else 1)
                    pops = [i for i in range(19) if EZ[i] == (1 if face == 0 else -1)]
                    assert x.tag == (0 if upward else 128) + 32 * lat + pops[k]
                    continue
                lim = (nown + 2) * plane if x.array == 2 else 19 * stride
                assert 0 <= x.offset and x.offset + x.count <= lim
                pop, lz = divmod(x.offset, stride) if x.array != 2 else (0, x.offset)
                lz //= plane
                assert lz == PLANE[(stage, upward, bool(x.send))](nown), (stage, x.tag, x.send, lz)
                if x.array == 2:
                    assert stage == A.MK_SLAB_PHI
                    continue
                # FILL moves the even loop's results, RETURN the odd loop's ghost writes
                expect = -1 if (stage == A.MK_SLAB_FILL) == upward else +1
                assert EZ[pop] == expect, (stage, x.tag, pop)
            # every receive has exactly one matching send on its peer, same size
            for x in xs:
                if x.send:
                    continue
                mates = [y for y in lists[x.peer] if y.send and y.peer == r and y.tag == x.tag]
                assert len(mates) == 1 and mates[0].bytes == x.bytes
            # and the pairwise order agrees (NCCL matches in posting order)
            for q in range(n):
                mine = [x.tag for x in xs if x.send and x.peer == q]
                theirs = [y.tag for y in lists[q] if not y.send and y.peer == r]
                assert mine == theirs


def test_plan_sizes():
    p = global_params(8, 8, 12, A.MK_BC_PERIODIC)
    # interior ranks: 5 populations x 2 lattices x (send + receive) x 2 faces
    assert plan_counts(p, 1, 3) == {A.MK_SLAB_FILL: 40, A.MK_SLAB_PHI: 4, A.MK_SLAB_RETURN: 40}
    w = global_params(8, 8, 12, A.MK_BC_WALLS)
    assert plan_counts(w, 0, 3) == {A.MK_SLAB_FILL: 20, A.MK_SLAB_PHI: 2, A.MK_SLAB_RETURN: 20}
    assert plan_counts(w, 0, 1) == {A.MK_SLAB_FILL: 0, A.MK_SLAB_PHI: 0, A.MK_SLAB_RETURN: 0}
    # periodic on one rank: the slab trades with itself
    assert plan_counts(p, 0, 1) == {A.MK_SLAB_FILL: 40, A.MK_SLAB_PHI: 4, A.MK_SLAB_RETURN: 40}


def test_plan_capacity_and_stage_checked():
    import ctypes as C
    lib = A.load()
    p = global_params(8, 8, 12, A.MK_BC_PERIODIC)
    buf = (A.MkSlabXfer * 8)()
    n = C.c_int32()
    assert lib.mk_slab_plan(C.byref(p), 1, 3, A.MK_SLAB_FILL, buf, 8, C.byref(n)) == A.MK_ERR_ARG
    assert n.value == 40
    assert lib.mk_slab_plan(C.byref(p), 1, 3, A.MK_SLAB_RUN_PHI, buf, 8, C.byref(n)) == A.MK_ERR_ARG


# ------------------------------------------------------------ in-process split
class _LocalTransport:
    """In-process exchange among NumPy slabs (the copies mk_slab_exchange_local
    makes on the device)."""

    def __init__(self, slabs):
        self.slabs = slabs

    def exchange_all(self, stage):
        lists = [s.transfers(stage) for s in self.slabs]
        for r, xs in enumerate(lists):
            for x in xs:
                if x.send:
                    continue
                (y,) = [y for y in lists[x.peer] if y.send and y.peer == r and y.tag == x.tag]
                self.slabs[r].run_tensor(x).copy_(self.slabs[x.peer].run_tensor(y))
        for s in self.slabs:
            s.done(stage)


def _split_run(nx, ny, nz, bc, n, loops, bc0=0, bc1=0):
    slabs = [AAModel(nx, ny, nz, bc, r, n, bc0, bc1) for r in range(n)]
    tr = _LocalTransport(slabs)
    while True:
        act = slabs[0].next()
        if act == A.MK_SLAB_RUN_PHI and slabs[0].step == loops:
            break
        if act in S.EXCHANGES:
            tr.exchange_all(act)
        else:
            for s in slabs:
                s.run(act)
    parts = [s.owned() for s in slabs]
    return tuple(np.concatenate([p[k] for p in parts], axis=1 if k else 0) for k in range(3))


def _same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


XY = [(A.MK_BC_PERIODIC, A.MK_BC_PERIODIC), (A.MK_BC_WALLS, A.MK_BC_PERIODIC), (A.MK_BC_CLOSED, A.MK_BC_WALLS),
      (A.MK_BC_PERIODIC, A.MK_BC_CLOSED)]


@pytest.mark.parametrize("xy", XY)
@pytest.mark.parametrize("bc", BCS)
@pytest.mark.parametrize("n", [1, 2, 3])
def test_split_run_bitwise_equals_whole_domain(bc, n, xy):
    nx, ny, nz, loops = 7, 6, 10, 7
    ref = whole_run(nx, ny, nz, bc, loops, *xy).owned()
    got = _split_run(nx, ny, nz, bc, n, loops, *xy)
    for k, (a, b) in enumerate(zip(got, ref)):
        assert _same(a, b), ("phi", "g", "h")[k]
    # and the run did something: phi moved away from its start
    assert np.abs(ref[0] - AAModel(nx, ny, nz, bc, bc0=xy[0], bc1=xy[1]).owned()[0]).max() > 1e-4


def test_whole_plane_return_breaks_walled_x():
    """Returning the odd loop's ghost writes as whole plane runs, without the
    merge's open-link mask, overwrites the bounce-back slots next to an x
    wall: the split run then differs from the whole run."""
    nx, ny, nz, bc, loops = 7, 6, 10, A.MK_BC_PERIODIC, 3
    orig = AAModel._merge

    def unmasked(self):
        ok = self.nb_ok.copy()
        self.nb_ok[:] = True
        try:
            orig(self)
        finally:
            self.nb_ok = ok

    AAModel._merge = unmasked
    try:
        got = _split_run(nx, ny, nz, bc, 2, loops, A.MK_BC_WALLS, A.MK_BC_PERIODIC)
    finally:
        AAModel._merge = orig
    ref = whole_run(nx, ny, nz, bc, loops, A.MK_BC_WALLS, A.MK_BC_PERIODIC).owned()
    assert not _same(got[2], ref[2])


def test_a_dropped_transfer_is_detected():
    """A plan that loses one population run no longer matches the whole run
    (the check has teeth)."""
    nx, ny, nz, bc, loops = 6, 5, 10, A.MK_BC_PERIODIC, 5
    slabs = [AAModel(nx, ny, nz, bc, r, 2) for r in range(2)]
    orig = AAModel.transfers

    def lossy(self, stage):
        xs = orig(self, stage)
        if stage == A.MK_SLAB_FILL:
            xs = [x for x in xs if not (x.array == 1 and x.tag == 32 + 6)]
        return xs

    for s in slabs:
        s.transfers = lossy.__get__(s)
    tr = _LocalTransport(slabs)
    while not (slabs[0].next() == A.MK_SLAB_RUN_PHI and slabs[0].step == loops):
        act = slabs[0].next()
        if act in S.EXCHANGES:
            tr.exchange_all(act)
        else:
            for s in slabs:
                s.run(act)
    got = np.concatenate([s.owned()[2] for s in slabs], axis=1)
    ref = whole_run(nx, ny, nz, bc, loops).owned()[2]
    assert not _same(got, ref)


# --------------------------------------------------------------- gloo ranks
def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, case, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import torch.distributed as dist
    from _slab_model import AAModel as M
    from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as SL
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        nx, ny, nz, bc, loops, bc0, bc1 = case
        m = M(nx, ny, nz, bc, rank, ws, bc0, bc1)
        run = SL.SlabRun(m, SL.TorchTransport())
        run.advance(loops // 2)
        run.advance(loops - loops // 2)
        diag = run.diagnostics()
        q.put((rank, m.owned(), diag))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("ws,bc,xy", [(2, A.MK_BC_PERIODIC, (0, 0)), (2, A.MK_BC_WALLS, (1, 0)),
                                      (3, A.MK_BC_CLOSED, (2, 1))])
def test_gloo_ranks_bitwise_equal_whole_domain(ws, bc, xy):
    import torch.multiprocessing as mp
    case = (6, 5, 11, bc, 9) + tuple(xy)
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, ws, port, case, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in range(ws)), key=lambda t: t[0])
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ref_model = whole_run(*case)
    ref = ref_model.owned()
    for k in range(3):
        got = np.concatenate([r[1][k] for r in res], axis=1 if k else 0)
        assert _same(got, ref[k]), ("phi", "g", "h")[k]
    # one FP64 all-reduce gives every rank the global sums
    rs, _ = ref_model.diag_sums()
    for _, _, d in res:
        assert d["fluid_cells"] == int(rs[6])
        assert d["mass"] == pytest.approx(rs[0], rel=1e-13)
        assert d["phi_sum"] == pytest.approx(rs[4], rel=1e-13)
