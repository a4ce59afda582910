"""Regenerate the multigrain fixtures from the reference's own solver source.

The reference's multigrain loop (run_multiPhaseField, MaterKit/MaterKit.cpp:
529-571) runs mkFluidsUser::propagate / relaxation, MaterKit/src/
mkFluidsUser.cpp:68-299, the one solver source the reference ships readable.
`make -C oracle ref` compiles that file where it lies against stand-in
declarations of its closed library (oracle/ref_stub/), for the D2Q9 velocity
set the reference ships (QF = 9) and for D3Q19.  This script runs those builds
on two periodic cases and stores the grains' order parameters after a few
loop counts:

    multigrain_ref_d2q9.npz   64 x 64 x 1, three grains (two touching), W0 1.5
    multigrain_ref_d3q19.npz  40 x 40 x 6, two touching grains, W0 0.8

Each file holds `xml` (the case, written by cases.multigrain with periodic
faces), `loops` and `phi` (loops x grains x nz x ny x nx, FP64), and `cone`:
the reference relaxes the first node of each OpenMP thread with omega_g = 1
in its phase-field source (omega_g is firstprivate and assigned after its
first use, mkFluidsUser.cpp:174-282); the build runs one thread, so only node
(0, 0, 0) is affected, and a difference born there spreads at most two cells
per loop (one streaming step, one gradient stencil).  Cells within periodic
Chebyshev distance cone * loops + 1 of that node are excluded from
comparisons.  Seed centres sit off lattice points: at a centre on a lattice
point the grain normal is regularised rounding noise, which amplifies any
last-bit difference.

    make -C oracle ref && python tests/golden/make_multigrain_ref.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases  # noqa: E402

CONE = 2  # cells per loop

FIXTURES = {
    "multigrain_ref_d2q9.npz": dict(q=9, shape=(64, 64, 1), W0=1.5, loops=(1, 4, 8),
                                     seeds=[(26.3, 32.4, 0.0, 7.0), (38.2, 31.7, 0.0, 7.0), (32.45, 44.1, 0.0, 5.0)]),
    "multigrain_ref_d3q19.npz": dict(q=19, shape=(40, 40, 6), W0=0.8, loops=(2, 5),
                                      seeds=[(16.3, 20.4, 2.6, 5.0), (24.2, 19.7, 3.1, 5.0)]),
}


def case_xml(shape, seeds, W0) -> str:
    nx, ny, nz = shape
    xml = cases.multigrain(n=nx, ny=ny, nz=nz, seeds=[tuple(s) for s in seeds], W0=W0, loops=100, precision="fp64")
    return xml.replace("<boundary> closed closed closed </boundary>",
                       "<boundary> periodic periodic periodic </boundary>")


def initial(shape, seeds, W0) -> np.ndarray:
    """-tanh((r - R)/(sqrt2 W0)) per grain, as both case layers set it up."""
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    return np.stack([-np.tanh((np.sqrt((x - a) ** 2 + (y - b) ** 2 + (z - c) ** 2) - r) / (np.sqrt(2.0) * W0))
                     for a, b, c, r in seeds]).astype(np.float64)


def cone_mask(shape, radius: int) -> np.ndarray:
    """True where a cell is farther than `radius` (periodic Chebyshev) from (0,0,0)."""
    nx, ny, nz = shape
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    d = np.maximum(np.maximum(np.minimum(x, nx - x), np.minimum(y, ny - y)), np.minimum(z, nz - z))
    return d > radius


def run(q: int, shape, W0, phi0, loops) -> np.ndarray:
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", f"libmgref_q{q}.so"))
    lib.mgref_run.argtypes = [C.c_int] * 4 + [C.c_double, C.c_void_p, C.c_int, C.c_void_p]
    assert lib.mgref_lattice() == q
    nx, ny, nz = shape
    out = np.empty_like(phi0)
    if lib.mgref_run(nx, ny, nz, phi0.shape[0], W0, phi0.ctypes.data, int(loops), out.ctypes.data) != 0:
        raise RuntimeError("mgref_run refused the case")
    return out


def main() -> None:
    for name, f in FIXTURES.items():
        phi0 = initial(f["shape"], f["seeds"], f["W0"])
        snaps = np.stack([run(f["q"], f["shape"], f["W0"], phi0, n) for n in f["loops"]])
        np.savez_compressed(os.path.join(HERE, name), xml=np.array(case_xml(f["shape"], f["seeds"], f["W0"])),
                            loops=np.array(f["loops"]), phi=snaps, cone=np.array(CONE), lattice=np.array(f["q"]))
        print(name, snaps.shape, os.path.getsize(os.path.join(HERE, name)), "bytes")


if __name__ == "__main__":
    main()
