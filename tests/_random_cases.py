"""Seeded random cases of every model for the shape sweeps: random sizes
(one-cell axes included, so 2-D and 1-D domains appear), random faces per
axis (periodic, walls, closed), random collision / lattice / anisotropy /
contact-angle variants, seeds and bubbles off lattice points.  Each case is
(name, XML text, fields to compare), FP64, deterministic in its seed."""
import re

import numpy as np

from materkit_anisotropiclbm_trt_rbc_facet_b200 import cases

MODELS = ["flow", "multiphase", "thermal", "solutal", "convection", "multigrain", "flow_dendrite", "flow_solutal"]
FIELDS = {
    "flow": ["rho", "ux", "uy", "uz"],
    "multiphase": ["phi", "rho", "pressure", "ux", "uy", "uz"],
    "thermal": ["phi", "T"],
    "solutal": ["phi", "C"],
    "convection": ["rho", "ux", "uy", "uz", "T"],
    "multigrain": ["phi", "T"],
    "flow_dendrite": ["phi", "T", "rho", "ux", "uy", "uz"],
    "flow_solutal": ["phi", "C", "rho", "ux", "uy", "uz"],
}
N_CASES = 32


def _faces(rng, sizes, allowed=("periodic", "walls", "closed")):
    out = []
    for n in sizes:
        pick = [b for b in allowed if not (b == "walls" and n < 3)]
        out.append(str(rng.choice(pick)))
    return out


def _with_faces(xml: str, faces) -> str:
    return re.sub(r"<boundary>[^<]*</boundary>", "<boundary> " + " ".join(faces) + " </boundary>", xml, count=1)


def _sizes(rng, lo=1, hi=18, min_cells=24):
    while True:
        s = [int(rng.integers(lo, hi + 1)) for _ in range(3)]
        if s[0] * s[1] * s[2] >= min_cells:
            return s


def _point(rng, sizes, margin=0.0):
    return tuple(float(rng.uniform(margin, max(margin, n - 1 - margin))) + 0.137 for n in sizes)


def _collision(rng):
    """A collision and a flow lattice (MRT is defined for D3Q19 only)."""
    coll = str(rng.choice(["BGK", "TRT", "MRT"]))
    return coll, "D3Q19" if coll == "MRT" else str(rng.choice(["D3Q19", "D3Q27"]))


def case(k: int):
    rng = np.random.default_rng(0xC0FFEE + 7919 * k)
    model = MODELS[k % len(MODELS)]
    if model == "flow":
        nx, ny, nz = _sizes(rng)
        coll, lat = _collision(rng)
        xml = cases.poiseuille(nx=nx, ny=ny, nz=nz, collision=coll, lattice=lat,
                               force=float(rng.uniform(1e-6, 1e-4)), loops=10)
        xml = _with_faces(xml, _faces(rng, (nx, ny, nz)))
    elif model == "multiphase":
        nx, ny, nz = _sizes(rng, lo=4, hi=20, min_cells=200)
        nb = int(rng.integers(0, 3)) if min(nx, ny, nz) >= 10 else 0
        xml = cases.multiphase_bubbles(n=nx, ny=ny, nz=nz, bubbles=nb, rmin=2.5, rmax=3.5, width=2.0,
                                       gz=float(rng.uniform(-1e-5, 0)), precision="fp64", loops=10,
                                       contact_angle=float(rng.choice([60.0, 90.0, 120.0])),
                                       seed=int(rng.integers(1, 1 << 30)),
                                       boundary=" ".join(_faces(rng, (nx, ny, nz))))
    elif model == "thermal":
        n = int(rng.integers(8, 20))
        aniso = str(rng.choice(["cubic", "cbc", "hcp", "facet"]))
        xml = cases.thermal_dendrite(n=n, loops=10, precision="fp64", radius=float(rng.uniform(1.5, n / 4.0)),
                                     center=_point(rng, (n, n, n), margin=n / 3.0), aniso=aniso,
                                     eps2=0.0 if aniso == "cubic" else 0.02)
        xml = _with_faces(xml, _faces(rng, (n, n, n)))
    elif model == "solutal":
        nx, ny, nz = _sizes(rng, lo=1, hi=20, min_cells=100)
        c = _point(rng, (nx, ny, nz))
        ang = tuple(float(a) for a in rng.uniform(0, 90, 3))
        xml = cases.solutal_dendrite(n=nx, ny=ny, nz=nz, loops=10, precision="fp64",
                                     seeds=[(c, ang, float(rng.uniform(1.5, 4.0)))])
        xml = _with_faces(xml, _faces(rng, (nx, ny, nz)))
    elif model == "convection":
        axis = str(rng.choice(["x", "y", "z"]))
        sizes = _sizes(rng, lo=1, hi=16, min_cells=60)
        sizes["xyz".index(axis)] = max(sizes["xyz".index(axis)], 5)
        coll, lat = _collision(rng)
        xml = cases.convection(nx=sizes[0], ny=sizes[1], nz=sizes[2], axis=axis, Ra=float(rng.uniform(1e3, 3e4)),
                               collision=coll, lattice=lat, loops=10)
    elif model == "multigrain":
        nx, ny, nz = _sizes(rng, lo=1, hi=18, min_cells=100)
        seeds = [_point(rng, (nx, ny, nz)) + (float(rng.uniform(2.0, 5.0)),) for _ in range(int(rng.integers(1, 4)))]
        xml = cases.multigrain(n=nx, ny=ny, nz=nz, seeds=seeds, W0=float(rng.uniform(0.8, 1.5)), loops=10,
                               precision="fp64")
        xml = _with_faces(xml, _faces(rng, (nx, ny, nz)))
    else:
        nx, ny, nz = _sizes(rng, lo=3, hi=18, min_cells=100)
        nx = max(nx, 3)
        gen = cases.flow_dendrite if model == "flow_dendrite" else cases.flow_solutal_dendrite
        coll, lat = _collision(rng)
        xml = gen(nx=nx, ny=ny, nz=nz, loops=10, precision="fp64", u_in=float(rng.uniform(0.0, 0.05)),
                  radius=float(rng.uniform(1.5, 4.0)), center=_point(rng, (nx, ny, nz)),
                  inlet=bool(rng.integers(0, 2)), collision=coll, lattice=lat)
    return f"{k:02d}_{model}", xml, FIELDS[model]
