"""ctypes wrapper of the FP64 CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the oracle is the checker and the timed CPU
baseline, never the thing measured or shipped.  It imports nothing from the
product package; cases come from the oracle's own case layer (``oracle.case``).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import case as K

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(ORACLE_DIR, "_build", "liboracle.so")

_lib = None


def build() -> str:
    """Build liboracle.so with the committed Makefile when a source is newer."""
    srcs = [os.path.join(ORACLE_DIR, f) for f in ("mk_oracle.cpp", "mk_oracle.hpp", "Makefile")]
    if not os.path.exists(ORACLE_LIB) or any(os.path.getmtime(s) > os.path.getmtime(ORACLE_LIB) for s in srcs):
        env = dict(os.environ)
        env.pop("CXX", None)
        subprocess.run(["make", "-C", ORACLE_DIR], check=True, capture_output=True, env=env)
    return ORACLE_LIB


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        lib = C.CDLL(build())
        D = C.POINTER(C.c_double)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(K.MkParams)] + [D] * 7
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_advance.argtypes = [C.c_void_p, C.c_int64]
        lib.orc_step.restype = C.c_int64
        lib.orc_step.argtypes = [C.c_void_p]
        lib.orc_get_field.restype = C.c_int
        lib.orc_get_field.argtypes = [C.c_void_p, C.c_int, D]
        lib.orc_get_grain_phi.restype = C.c_int
        lib.orc_get_grain_phi.argtypes = [C.c_void_p, C.c_int, D]
        lib.orc_get_populations.restype = C.c_int
        lib.orc_get_populations.argtypes = [C.c_void_p, C.c_int, D]
        lib.orc_set_threads.argtypes = [C.c_int]
        lib.orc_get_threads.restype = C.c_int
        lib.orc_anisotropy.argtypes = [C.c_int, C.c_double, C.c_double, D, D, D]
        lib.orc_backward.restype = C.c_int
        lib.orc_backward.argtypes = [C.c_void_p, D, C.c_int64, D]
        lib.orc_update_geometry.restype = C.c_int
        lib.orc_update_geometry.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_update_velocity.restype = C.c_int
        lib.orc_update_velocity.argtypes = [C.c_void_p, C.c_void_p]
        lib.orc_aos_create.restype = C.c_void_p
        lib.orc_aos_create.argtypes = [C.c_void_p]
        lib.orc_aos_destroy.argtypes = [C.c_void_p]
        lib.orc_aos_advance.argtypes = [C.c_void_p, C.c_int64]
        lib.orc_aos_get_populations.restype = C.c_int
        lib.orc_aos_get_populations.argtypes = [C.c_void_p, C.c_int, D]
        lib.orc_aos_get_field.restype = C.c_int
        lib.orc_aos_get_field.argtypes = [C.c_void_p, C.c_int, D]
        lib.orc_aos_node_bytes.restype = C.c_size_t
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _as_oracle_params(params) -> K.MkParams:
    """The parameters as the oracle's own structure (a product MkParams of the
    same C layout is copied byte for byte)."""
    if isinstance(params, K.MkParams):
        return params
    if C.sizeof(params) != C.sizeof(K.MkParams):
        raise TypeError("parameter block of another layout")
    out = K.MkParams()
    C.memmove(C.byref(out), C.byref(params), C.sizeof(out))
    return out


class Oracle:
    """One CPU case; fields come back as (nz, ny, nx) float64 arrays."""

    def __init__(self, params, phi=None, T=None, Cc=None, rho=None, u=None):
        self.lib = load()
        self.params = _as_oracle_params(params)
        keep = []

        def arr(x):
            if x is None:
                return None
            x = np.ascontiguousarray(x, dtype=np.float64).ravel()
            keep.append(x)
            return x

        phi, T, Cc, rho = arr(phi), arr(T), arr(Cc), arr(rho)
        ux = uy = uz = None
        if u is not None:
            ux, uy, uz = arr(u[0]), arr(u[1]), arr(u[2])
        self.h = self.lib.orc_create(C.byref(self.params), _ptr(phi), _ptr(T), _ptr(Cc), _ptr(rho), _ptr(ux),
                                     _ptr(uy), _ptr(uz))
        self._keep = keep

    @classmethod
    def from_case(cls, params) -> "Oracle":
        """The case started from the oracle's own initial fields."""
        p = _as_oracle_params(params)
        return cls(p, **K.oracle_fields(p))

    @classmethod
    def from_xml(cls, path: str, **overrides) -> "Oracle":
        """Resolve an XML case with the oracle's reader and start it."""
        return cls.from_case(K.resolve(path, **overrides))

    def advance(self, n: int) -> None:
        self.lib.orc_advance(self.h, int(n))

    @property
    def step(self) -> int:
        return int(self.lib.orc_step(self.h))

    def backward(self, target, steps: int) -> dict:
        """Discrete adjoint: loss and its gradient after `steps` loops."""
        t = np.ascontiguousarray(target, dtype=np.float64).ravel()
        out = np.zeros(4)
        rc = self.lib.orc_backward(self.h, _ptr(t), int(steps), _ptr(out))
        if rc != 0:
            raise RuntimeError("orc_backward failed")
        return {"loss": out[0], "d_eps4": out[1], "d_delta": out[2], "d_tau_t": out[3]}

    def field(self, name: str) -> np.ndarray:
        p = self.params
        out = np.empty(p.ncell(), dtype=np.float64)
        rc = self.lib.orc_get_field(self.h, K.FIELD[name], _ptr(out))
        if rc != 0:
            raise KeyError(name)
        return out.reshape(p.nz, p.ny, p.nx)

    def grain(self, j: int) -> np.ndarray:
        """Order parameter of grain j (multigrain model)."""
        p = self.params
        out = np.empty(p.ncell(), dtype=np.float64)
        if self.lib.orc_get_grain_phi(self.h, int(j), _ptr(out)) != 0:
            raise KeyError(j)
        return out.reshape(p.nz, p.ny, p.nx)

    def update_geometry(self, dendrite: "Oracle") -> None:
        """This multiphase flow takes the dendrite's solid (phi > 0) as geometry
        from its next even loop count."""
        if self.lib.orc_update_geometry(self.h, dendrite.h) != 0:
            raise ValueError("update_geometry: a multiphase flow and a dendrite of one grid")

    def update_velocity(self, flow: "Oracle") -> None:
        """This dendrite's scalar lattice takes the flow's velocity."""
        if self.lib.orc_update_velocity(self.h, flow.h) != 0:
            raise ValueError("update_velocity: a dendrite and a multiphase flow of one grid")

    def populations(self, which: int = 0) -> np.ndarray:
        """Post-collision populations of lattice `which`, (Q, ncell)."""
        p = self.params
        q = {0: p.lattice if p.model in (0, 4) else 7}.get(which, 7)
        out = np.empty(q * p.ncell(), dtype=np.float64)
        if self.lib.orc_get_populations(self.h, int(which), _ptr(out)) != 0:
            raise KeyError(which)
        return out.reshape(q, p.ncell())

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReferenceStructure:
    """The oracle's method in the reference's data structure: one object per
    node with every field of mkNode (MaterKit/inc/mkNode.h:128-215), node
    sweeps with schedule(static, 16) (MaterKit/src/mkFluidsUser.cpp:70).
    Started from an oracle state; the flow model (D3Q19) and the thermal
    dendrite; bit-identical to the oracle.  The CPU baseline of that layout."""

    def __init__(self, oracle: Oracle):
        self.lib = load()
        self.params = oracle.params
        self.h = self.lib.orc_aos_create(oracle.h)
        if not self.h:
            raise ValueError("the reference-structure variant covers the flow model (D3Q19) and the thermal dendrite")

    @staticmethod
    def node_bytes() -> int:
        return int(load().orc_aos_node_bytes())

    def advance(self, n: int) -> None:
        self.lib.orc_aos_advance(self.h, int(n))

    def populations(self, which: int = 0) -> np.ndarray:
        p = self.params
        q = p.lattice if p.model == 0 else 7
        out = np.empty(q * p.ncell(), dtype=np.float64)
        if self.lib.orc_aos_get_populations(self.h, int(which), _ptr(out)) != 0:
            raise KeyError(which)
        return out.reshape(q, p.ncell())

    def field(self, name: str) -> np.ndarray:
        p = self.params
        out = np.empty(p.ncell(), dtype=np.float64)
        if self.lib.orc_aos_get_field(self.h, K.FIELD[name], _ptr(out)) != 0:
            raise KeyError(name)
        return out.reshape(p.nz, p.ny, p.nx)

    def close(self):
        if self.h:
            self.lib.orc_aos_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_threads(n: int) -> None:
    load().orc_set_threads(int(n))


def threads() -> int:
    return int(load().orc_get_threads())


def rel_l2(a, b, mask=None, floor: float = 0.0) -> float:
    """||a - b|| / max(||b||, floor * sqrt(count)).

    `floor` is the smallest per-cell magnitude the field is judged against, so
    a field that is still rounding noise (a pressure one loop after rest)
    is compared in absolute terms.
    """
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if mask is not None:
        a, b = a[mask], b[mask]
    den = max(float(np.linalg.norm(b)), floor * np.sqrt(b.size))
    num = float(np.linalg.norm(a - b))
    if den == 0.0:
        return num
    return num / den


def anisotropy(kind: int, e4: float, e2: float, n):
    """a(n) and da/dn of the oracle's anisotropy kind at the unit normal n."""
    nn = np.ascontiguousarray(n, dtype=np.float64)
    a = np.zeros(1)
    g = np.zeros(3)
    load().orc_anisotropy(int(kind), float(e4), float(e2), _ptr(nn), _ptr(a), _ptr(g))
    return float(a[0]), g
