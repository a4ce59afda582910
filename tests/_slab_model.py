"""A NumPy model of the library's in-place (AA) streaming on two D3Q19
lattices, whole-domain or as one z-slab with ghost planes, for testing the
slab decomposition on the CPU.

The layout, the AA slot rules, the neighbour validity and the ghost-plane
geometry are the library's (SoA planes of `stride` cells, index x + nx (y +
ny z); a slab's local planes 1 .. nown are its global planes z0 .. z0 + nown -
1, planes 0 and nown + 1 are ghosts that stream but never collide; a return
exchange lands in a halo buffer and merges where the source link is open).  The
collision is a made-up but strongly coupled FP64 operator: BGK on both
lattices with a force from the phi gradient and Laplacian and an interface
source on the phase lattice, so any population or phi value that crosses a
slab face wrongly changes the result.  Every cell's arithmetic is the same
elementwise sequence in both forms, so a correct decomposition reproduces the
whole-domain run bit for bit.

The slab form speaks the library's slab protocol (next / run / done /
transfers / run_tensor) and takes its transfer lists from the library's
host-only plan (mk_slab_plan), so the decomposition logic under test is the
library's and the Python runner's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from materkit_anisotropiclbm_trt_rbc_facet_b200 import _abi as A
from materkit_anisotropiclbm_trt_rbc_facet_b200 import slab as S

# D3Q19 in the library's order (rest, +-x, +-y, +-z, xy, xz, yz edges)
EX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
EY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
EZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
INV = np.array([0] + [i + 1 if i % 2 else i - 1 for i in range(1, 19)])


def pop_stride(ncell: int) -> int:
    return (ncell + 63) // 64 * 64


def global_params(nx: int, ny: int, nz: int, bc2: int, bc0: int = 0, bc1: int = 0) -> A.MkParams:
    p = A.MkParams()
    p.model = A.MK_MODEL_MULTIPHASE
    p.precision = A.MK_PREC_FP64
    p.nx, p.ny, p.nz = nx, ny, nz
    p.bc[0], p.bc[1], p.bc[2] = bc0, bc1, bc2
    return p


def _axis(c, n, bc):
    """(valid, index) of coordinates c on an x or y axis of n cells."""
    if bc == A.MK_BC_PERIODIC:
        return np.ones_like(c, dtype=bool), c % n
    valid = (c >= 0) & (c < n)
    if bc == A.MK_BC_WALLS:
        valid &= (c != 0) & (c != n - 1)
    return valid, np.clip(c, 0, n - 1)


def initial_phi(nx: int, ny: int, nz: int) -> np.ndarray:
    """A bubble off the domain centre, diffuse interface of width 4 (nz, ny, nx)."""
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    r = np.sqrt((x - 0.4 * nx) ** 2 + (y - 0.55 * ny) ** 2 + (z - 0.45 * nz) ** 2)
    return 0.5 + 0.5 * np.tanh(2.0 * (0.3 * min(nx, ny, nz) - r) / 4.0)


class AAModel:
    """Whole domain (nranks = 0) or the slab of `rank` among `nranks`; x and y
    boundaries bc0, bc1 (periodic, walls or closed) as in the library."""

    def __init__(self, nx: int, ny: int, nz: int, bc2: int, rank: int = 0, nranks: int = 0, bc0: int = 0,
                 bc1: int = 0):
        self.nx, self.ny, self.nzg, self.bc2 = nx, ny, nz, bc2
        self.bc0, self.bc1 = bc0, bc1
        self.slab = nranks > 0
        self.rank, self.nranks = rank, nranks
        self.gp = global_params(nx, ny, nz, bc2, bc0, bc1)
        if self.slab:
            self.z0, self.nown = S.split(nz, rank, nranks)
            self.nz = self.nown + 2
        else:
            self.z0, self.nown, self.nz = 0, nz, nz
        self.plane = nx * ny
        self.ncell = self.plane * self.nz
        self.stride = pop_stride(self.ncell)
        self._geometry()
        self.g = np.zeros(19 * self.stride)
        self.h = np.zeros(19 * self.stride)
        self.halo = np.zeros(20 * self.plane)  # the runs a return exchange delivers
        gphi = initial_phi(nx, ny, nz)
        lz = np.arange(self.nz)
        gz = self.z0 + lz - 1 if self.slab else lz
        gz = gz % nz if bc2 == A.MK_BC_PERIODIC else np.clip(gz, 0, nz - 1)
        self.phi = np.ascontiguousarray(gphi[gz]).ravel()
        self.step = 0
        # the initial state placed as the output of an odd loop (streamed by loop 0)
        c = self.cells
        for i in range(19):
            o = self._off_out(i, 1)
            self.g[o] = W[i]
            self.h[o] = W[i] * self.phi[c]
        self.state = A.MK_SLAB_RETURN if self.slab else None

    # -- geometry -----------------------------------------------------------
    def _open(self, q):
        ok = np.ones_like(q, dtype=bool)
        if self.bc2 != A.MK_BC_PERIODIC:
            ok &= (q >= 0) & (q < self.nzg)
        if self.bc2 == A.MK_BC_WALLS:
            ok &= (q != 0) & (q != self.nzg - 1)
        return ok

    def _zlink(self, cz):
        """(valid, local plane) of local planes cz (any integers)."""
        if self.slab:
            inside = (cz >= 0) & (cz < self.nz)
            valid = inside & self._open(self.z0 + cz - 1)
            return valid, np.where(inside, cz, 0)
        n = self.nz
        if self.bc2 == A.MK_BC_PERIODIC:
            return np.ones_like(cz, dtype=bool), cz % n
        valid = (cz >= 0) & (cz < n)
        if self.bc2 == A.MK_BC_WALLS:
            valid &= (cz != 0) & (cz != n - 1)
        return valid, np.clip(cz, 0, n - 1)

    def _geometry(self):
        z, y, x = np.meshgrid(np.arange(self.nz), np.arange(self.ny), np.arange(self.nx), indexing="ij")
        z, y, x = z.ravel(), y.ravel(), x.ravel()
        fluid = _axis(x, self.nx, self.bc0)[0] & _axis(y, self.ny, self.bc1)[0]
        if self.slab:
            fluid &= (z >= 1) & (z <= self.nz - 2) & self._open(self.z0 + z - 1)
        elif self.bc2 == A.MK_BC_WALLS:
            fluid &= (z != 0) & (z != self.nz - 1)
        self.cells = np.nonzero(fluid)[0]
        x, y, z = x[self.cells], y[self.cells], z[self.cells]
        self.cz = z
        self.nb_ok = np.zeros((19, len(self.cells)), dtype=bool)
        self.nb = np.zeros((19, len(self.cells)), dtype=np.int64)
        for i in range(19):
            okx, cx = _axis(x + EX[i], self.nx, self.bc0)
            oky, cy = _axis(y + EY[i], self.ny, self.bc1)
            okz, cz = self._zlink(z + EZ[i])
            self.nb_ok[i] = okx & oky & okz
            self.nb[i] = cx + self.nx * (cy + self.ny * cz)

    def _off_in(self, i, parity):
        c = self.cells
        if parity == 0:
            return i * self.stride + c
        j = INV[i]  # the neighbour along -e_i
        return np.where(self.nb_ok[j], INV[i] * self.stride + self.nb[j], i * self.stride + c)

    def _off_out(self, i, parity):
        c = self.cells
        if parity == 0:
            return INV[i] * self.stride + c
        return np.where(self.nb_ok[i], i * self.stride + self.nb[i], INV[i] * self.stride + c)

    # -- the two kernels of a loop ---------------------------------------------
    def phi_kernel(self):
        p = self.step & 1
        acc = np.zeros(len(self.cells))
        for i in range(19):
            acc = acc + self.h[self._off_in(i, p)]
        self.phi[self.cells] = acc

    def collide(self):
        p = self.step & 1
        c = self.cells
        gi = [self.g[self._off_in(i, p)] for i in range(19)]
        hi = [self.h[self._off_in(i, p)] for i in range(19)]
        ph = self.phi[c]
        rho = np.zeros(len(c))
        jx, jy, jz = np.zeros(len(c)), np.zeros(len(c)), np.zeros(len(c))
        for i in range(19):
            rho = rho + gi[i]
            jx = jx + EX[i] * gi[i]
            jy = jy + EY[i] * gi[i]
            jz = jz + EZ[i] * gi[i]
        gx, gy, gz, lap = np.zeros(len(c)), np.zeros(len(c)), np.zeros(len(c)), np.zeros(len(c))
        for i in range(1, 19):
            fn = np.where(self.nb_ok[i], self.phi[self.nb[i]], ph)
            gx = gx + (W[i] * EX[i]) * fn
            gy = gy + (W[i] * EY[i]) * fn
            gz = gz + (W[i] * EZ[i]) * fn
            lap = lap + W[i] * (fn - ph)
        gx, gy, gz, lap = 3.0 * gx, 3.0 * gy, 3.0 * gz, 6.0 * lap
        mu = 0.08 * ph * (ph - 1.0) * (ph - 0.5) - 0.05 * lap
        fx, fy, fz = mu * gx, mu * gy, mu * gz - 1e-5 * (ph - 0.5)
        ux, uy, uz = (jx + 0.5 * fx) / rho, (jy + 0.5 * fy) / rho, (jz + 0.5 * fz) / rho
        gn = np.sqrt(gx * gx + gy * gy + gz * gz) + 1e-12
        nx_, ny_, nz_ = gx / gn, gy / gn, gz / gn
        usq = ux * ux + uy * uy + uz * uz
        for i in range(19):
            eu = EX[i] * ux + EY[i] * uy + EZ[i] * uz
            ef = EX[i] * fx + EY[i] * fy + EZ[i] * fz
            geq = W[i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq)
            go = gi[i] - 0.9 * (gi[i] - geq) + 0.55 * W[i] * 3.0 * ef
            en = EX[i] * nx_ + EY[i] * ny_ + EZ[i] * nz_
            heq = W[i] * ph * (1.0 + 3.0 * eu) + W[i] * 0.25 * ph * (1.0 - ph) * en
            ho = hi[i] - 1.2 * (hi[i] - heq)
            o = self._off_out(i, p)
            self.g[o] = go
            self.h[o] = ho
        self.step += 1

    def advance(self, n: int):
        """Whole-domain loops (no exchanges)."""
        assert not self.slab
        for _ in range(n):
            self.phi_kernel()
            self.collide()

    # -- results ----------------------------------------------------------------
    def owned(self):
        """(phi, g, h) over the owned planes: phi (nown, ny, nx); g, h the
        post-collision populations of every cell in the layout of the last
        loop, (19, nown, ny, nx); 0 on wall cells."""
        lo = self.plane * (1 if self.slab else 0)
        hi = lo + self.plane * self.nown
        phi = self.phi[lo:hi].reshape(self.nown, self.ny, self.nx).copy()
        par = (self.step + 1) & 1
        g = np.zeros((19, self.ncell))
        h = np.zeros((19, self.ncell))
        for i in range(19):
            o = self._off_out(i, par)
            g[i, self.cells] = self.g[o]
            h[i, self.cells] = self.h[o]
        shp = (19, self.nown, self.ny, self.nx)
        return phi, g[:, lo:hi].reshape(shp), h[:, lo:hi].reshape(shp)

    # -- the slab protocol (as the library's handle) ----------------------------
    def next(self) -> int:
        return self.state

    def transfers(self, stage: int):
        return S.plan(self.gp, self.rank, self.nranks, stage)

    def run_tensor(self, x):
        import torch
        arr = (self.g, self.h, self.phi, self.halo)[x.array]
        return torch.from_numpy(arr[x.offset:x.offset + x.count])

    def _merge(self):
        """The received return runs into the owned boundary planes, except the
        slots whose source across the face is closed (the cell's own
        bounce-back wrote those)."""
        periodic = self.bc2 == A.MK_BC_PERIODIC
        faces = [f for f, has in ((0, self.rank > 0 or periodic), (1, self.rank < self.nranks - 1 or periodic))
                 if has]
        for face in faces:
            z = 1 if face == 0 else self.nown
            pops = [i for i in range(19) if EZ[i] == (1 if face == 0 else -1)]
            sel = self.cz == z
            c = self.cells[sel]
            for lat, arr in enumerate((self.g, self.h)):
                for k, i in enumerate(pops):
                    ok = self.nb_ok[INV[i]][sel]
                    src = ((face * 2 + lat) * 5 + k) * self.plane + (c - z * self.plane)
                    arr[i * self.stride + c[ok]] = self.halo[src[ok]]

    def sync(self):
        pass

    def done(self, stage: int):
        assert stage == self.state, (stage, self.state)
        if stage == A.MK_SLAB_RETURN:
            self._merge()
        self.state = A.MK_SLAB_RUN_COLLIDE if stage == A.MK_SLAB_PHI else A.MK_SLAB_RUN_PHI

    def run(self, action: int):
        assert action == self.state, (action, self.state)
        if action == A.MK_SLAB_RUN_PHI:
            self.phi_kernel()
            self.state = A.MK_SLAB_PHI
        else:
            odd = self.step & 1
            self.collide()
            self.state = A.MK_SLAB_RETURN if odd else A.MK_SLAB_FILL

    def diag_sums(self):
        c = self.cells
        lo = self.plane if self.slab else 0
        hi = lo + self.plane * self.nown
        own = c[(c >= lo) & (c < hi)]
        par = (self.step + 1) & 1
        rho = np.zeros(len(self.cells))
        for i in range(19):
            rho = rho + self.g[self._off_out(i, par)]
        keep = (c >= lo) & (c < hi)
        sums = np.array([rho[keep].sum(), 0.0, 0.0, 0.0, self.phi[own].sum(), 0.0, float(len(own)), 0.0, 0.0, 0.0])
        return sums, 0.0


def whole_run(nx, ny, nz, bc2, loops, bc0=0, bc1=0):
    m = AAModel(nx, ny, nz, bc2, bc0=bc0, bc1=bc1)
    m.advance(loops)
    return m


def plan_counts(p: A.MkParams, rank: int, nranks: int) -> dict:
    out = {}
    for st in (A.MK_SLAB_FILL, A.MK_SLAB_PHI, A.MK_SLAB_RETURN):
        n = C.c_int32()
        A.load().mk_slab_plan(C.byref(p), rank, nranks, st, None, 0, C.byref(n))
        out[st] = n.value
    return out
