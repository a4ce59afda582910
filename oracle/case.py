"""The oracle's own case layer: BoltzTechs XML -> lattice-unit parameters,
initial macroscopic fields and the seeded synthetic cases.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  It is a second,
independent restatement of the reference's case set-up path, written in numpy
with its own XML reader, so the parity tests start the oracle from values the
product's case layer (``csrc/mk_case.cpp``) did not compute:

  mkSpace(xml)                     MaterKit/inc/mkSpace.h:36 (MeshXYZ)
  readParameters(loops, frames)    MaterKit/inc/mkFunction.h:62
  initialize(xml)                  MaterKit/inc/mkFluidsMRT.h:39, mkPhaseField.h:39,
                                   mkThermalField.h:31, mkFluidsMultiphase.h:30
  initialize_geometry()            MaterKit/inc/mkFluidsMRT.h:40, readable example
                                   MaterKit/src/mkFluidsUser.cpp:44-66 (channel walls)

Physical-unit tags are converted as the XML comments describe
(MaterKit/BoltzTechs - thermal.xml:56-63): lengths in units of mk_dx, times in
units of mk_dt, so a kinematic viscosity or diffusivity becomes
value * mk_dt / mk_dx^2, an acceleration value * mk_dt^2 / mk_dx, the phase
field's W0 / mk_dx and t0 / mk_dt, and lambda = 0.8839 W0 / d0 when <lambda>
is negative (thermal.xml:61).  The optional <b200> element holds lattice-unit
values and overrides all of that.

A seed list whose <center> holds fewer than 3 * <number> values (the shipped
``BoltzTechs - solutal.xml`` declares 2 seeds and gives one centre) places the
seeds whose centre is complete: <number> is reduced to the number of full
centre triples.

The shipped XML files carry GBK-encoded comments under an utf-8 declaration;
the reader works on bytes (latin-1 decoding) and drops comments before
tokenising, so such files read.
"""
from __future__ import annotations

import ctypes as C
import math
import re

import numpy as np

# ------------------------------------------------------------------ constants
# Values of include/mkb200.h (the enums of the C ABI the oracle library shares).
MODEL = {"flow": 0, "multiphase": 1, "thermal_dendrite": 2, "solutal_dendrite": 3, "convection": 4,
         "flow_dendrite": 5, "multigrain": 6, "flow_solutal_dendrite": 7}
FLOW_COUPLED = (MODEL["flow_dendrite"], MODEL["flow_solutal_dendrite"])
DENDRITES = (MODEL["thermal_dendrite"], MODEL["solutal_dendrite"]) + FLOW_COUPLED
PRECISION = {"fp64": 0, "fp32": 1, "fp16": 2, "bf16": 3}
COLLISION = {"bgk": 0, "trt": 1, "mrt": 2}
BC_PERIODIC, BC_WALLS, BC_CLOSED = 0, 1, 2
ANISO = {"cubic": 0, "cbc": 1, "hcp": 2, "facet": 3}
FIELD = {"rho": 0, "ux": 1, "uy": 2, "uz": 3, "T": 4, "C": 5, "phi": 6, "flag": 7, "pressure": 8, "dphi": 9,
         "grain": 10}
FLAG_FLUID, FLAG_WALLS = 0, 3
MAX_OBJECTS = 64

ST_XML, ST_ARG = 1, 2


class CaseError(ValueError):
    """A case the reader rejects: status 1 (XML) or 2 (argument), as the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class MkParams(C.Structure):
    """mk_params of include/mkb200.h, field for field (the oracle library's input)."""

    _fields_ = [
        ("model", C.c_int32), ("lattice", C.c_int32), ("collision", C.c_int32), ("precision", C.c_int32),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("bc", C.c_int32 * 3),
        ("max_loops", C.c_int32), ("max_frames", C.c_int32),
        ("rho0", C.c_double), ("u0", C.c_double * 3), ("tau", C.c_double), ("magic", C.c_double),
        ("force", C.c_double * 3),
        ("rho_l", C.c_double), ("rho_g", C.c_double), ("tau_l", C.c_double), ("tau_g", C.c_double),
        ("sigma", C.c_double), ("width", C.c_double), ("mobility", C.c_double), ("contact_angle", C.c_double),
        ("eps4", C.c_double), ("W0", C.c_double), ("tau0", C.c_double), ("lambda_", C.c_double),
        ("delta", C.c_double), ("D", C.c_double), ("D_s", C.c_double), ("k_part", C.c_double),
        ("at_coef", C.c_double),
        ("n_objects", C.c_int32), ("aniso", C.c_int32),
        ("obj_center", (C.c_double * 3) * MAX_OBJECTS), ("obj_angle", (C.c_double * 3) * MAX_OBJECTS),
        ("obj_radius", C.c_double * MAX_OBJECTS), ("rng_seed", C.c_uint64),
        ("eps2", C.c_double),
        ("wall_axis", C.c_int32), ("inlet", C.c_int32), ("wall_value", C.c_double * 2),
        ("wall_u", (C.c_double * 3) * 2), ("beta", C.c_double), ("s_ref", C.c_double),
        ("grain_kappa", C.c_double), ("grain_u", C.c_double * 3),
    ]

    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def values(self) -> dict:
        """Every field as plain Python values (arrays as lists), objects cut to n_objects."""
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, C.Array):
                v = [list(x) if isinstance(x, C.Array) else x for x in v]
            out[name] = v
        for k in ("obj_center", "obj_angle", "obj_radius"):
            out[k] = out[k][: self.n_objects]
        return out


def defaults() -> MkParams:
    """The parameter set before any tag is read (the driver's defaults of
    MaterKit/MaterKit.cpp:190-191 for the loop counts)."""
    p = MkParams()
    p.model = MODEL["flow"]
    p.lattice = 19
    p.collision = COLLISION["trt"]
    p.precision = PRECISION["fp32"]
    p.nx = p.ny = p.nz = 1
    p.max_loops, p.max_frames = 300, 100
    p.rho0 = 1.0
    p.tau = 0.8
    p.magic = 3.0 / 16.0
    p.rho_l, p.rho_g = 1.0, 0.1
    p.tau_l, p.tau_g = 0.8, 0.53
    p.sigma, p.width, p.mobility, p.contact_angle = 1e-3, 4.0, 0.05, 90.0
    p.eps4, p.W0, p.lambda_, p.delta = 0.05, 1.5, 10.0, 0.55
    p.D, p.D_s, p.k_part = 0.1, 1e-4, 0.15
    p.at_coef = 1.0 / (2.0 * math.sqrt(2.0))
    p.tau0 = 0.6267 * p.lambda_ * p.W0 * p.W0 / p.D
    p.aniso = ANISO["cubic"]
    p.wall_axis = -1
    p.grain_kappa = 1.0
    p.grain_u[:] = [0.02, 0.0, 0.0]  # grain 1's equilibrium velocity (mkFluidsUser.cpp:220-226)
    return p


# ------------------------------------------------------------------ XML reader
class Node:
    __slots__ = ("name", "text", "kids")

    def __init__(self, name: str):
        self.name = name
        self.text = ""
        self.kids: list[Node] = []

    def child(self, name: str):
        for k in self.kids:
            if k.name == name:
                return k
        return None

    def find(self, path: str):
        cur = self
        for part in path.split("/"):
            if cur is None:
                return None
            cur = cur.child(part)
        return cur


_TOKEN = re.compile(r"<(/?)([A-Za-z_][\w.:\-]*)((?:[^>\"']|\"[^\"]*\"|'[^']*')*)>|([^<]+)|(<)", re.S)


def parse_xml(path: str) -> Node:
    """Element tree of an XML file; comments, processing instructions, the
    DOCTYPE and attributes are ignored, CDATA is text."""
    with open(path, "rb") as f:
        raw = f.read()
    if raw.startswith(b"\xef\xbb\xbf"):
        raw = raw[3:]
    text = raw.decode("latin-1")
    text = re.sub(r"<!--.*?-->", " ", text, flags=re.S)
    if "<!--" in text:
        raise CaseError(ST_XML, f"{path}: unterminated comment")
    text = re.sub(r"<\?.*?\?>", " ", text, flags=re.S)
    text = re.sub(r"<!DOCTYPE[^>]*>", " ", text, flags=re.I)
    text = re.sub(r"<!\[CDATA\[(.*?)\]\]>", lambda m: m.group(1), text, flags=re.S)
    stack: list[Node] = []
    root = None
    for m in _TOKEN.finditer(text):
        close, name, attrs, chars, stray = m.groups()
        if stray is not None:
            raise CaseError(ST_XML, f"{path}: malformed tag at offset {m.start()}")
        if chars is not None:
            if stack:
                stack[-1].text += chars
            elif chars.strip():
                raise CaseError(ST_XML, f"{path}: text outside the root element")
            continue
        if close:
            if not stack or stack[-1].name != name:
                raise CaseError(ST_XML, f"{path}: mismatched end tag </{name}>")
            done = stack.pop()
            if not stack:
                root = done
                break
            continue
        node = Node(name)
        if stack:
            stack[-1].kids.append(node)
        elif root is not None:
            break
        if attrs.rstrip().endswith("/"):
            if not stack:
                root = node
                break
            continue
        stack.append(node)
    if stack or root is None:
        raise CaseError(ST_XML, f"{path}: unterminated element" if stack else f"{path}: no root element")
    return root


def _number(tok: str, where: str) -> float:
    try:
        return float(tok)
    except ValueError:
        pass
    if tok[:2].lower() == "0x":
        try:
            return float(int(tok, 16))
        except ValueError:
            pass
    raise CaseError(ST_XML, f"<{where}>: cannot read '{tok}' as a number")


def numbers(node: Node) -> list[float]:
    return [_number(t, node.name) for t in node.text.split()]


def number(node: Node) -> float:
    v = numbers(node)
    if not v:
        raise CaseError(ST_XML, f"<{node.name}>: empty value")
    return v[0]


def integer(node: Node) -> int:
    v = number(node)
    if v != int(v):
        raise CaseError(ST_XML, f"<{node.name}>: not an integer")
    return int(v)


def boolean(node: Node) -> bool:
    t = node.text.strip().lower()
    if t in ("true", "1", "yes"):
        return True
    if t in ("false", "0", "no"):
        return False
    raise CaseError(ST_XML, f"<{node.name}>: cannot read '{t}' as a boolean")


def _opt(root: Node | None, path: str, default):
    n = root.find(path) if root is not None else None
    return default if n is None else number(n)


def _optv(root: Node | None, path: str):
    n = root.find(path) if root is not None else None
    return None if n is None else numbers(n)


def _word(node: Node) -> str:
    return node.text.strip().lower()


# ------------------------------------------------------------------ case resolution
def read_parameters(path: str) -> tuple[int, int]:
    """output/numLoops and output/numFrames (readParameters, mkFunction.h:62)."""
    r = parse_xml(path)
    loops = integer(r.find("output/numLoops")) if r.find("output/numLoops") is not None else 300
    frames = integer(r.find("output/numFrames")) if r.find("output/numFrames") is not None else 100
    return loops, frames


def _seeds(node: Node | None, p: MkParams) -> None:
    """<number>, <center> triples (lattice units), <angle> triples (degrees,
    ZYX), <radius> (the last radius repeats) of a seed / object list
    (MaterKit/BoltzTechs - thermal.xml:65-77)."""
    if node is None:
        return
    num = integer(node.child("number")) if node.child("number") is not None else 0
    if num < 0 or num > MAX_OBJECTS:
        raise CaseError(ST_XML, "seed/number out of range")
    cen = _optv(node, "center") or []
    ang = _optv(node, "angle") or []
    rad = _optv(node, "radius") or []
    num = min(num, len(cen) // 3)
    p.n_objects = num
    for k in range(num):
        for a in range(3):
            p.obj_center[k][a] = cen[3 * k + a]
            p.obj_angle[k][a] = ang[3 * k + a] if len(ang) >= 3 * (k + 1) else 0.0
        p.obj_radius[k] = 8.0 if not rad else (rad[k] if k < len(rad) else rad[-1])


class SplitMix64:
    """splitmix64 (Steele, Lea & Flood 2014): the generator of every seeded case."""

    M = (1 << 64) - 1

    def __init__(self, seed: int):
        self.s = seed & self.M

    def next(self) -> int:
        self.s = (self.s + 0x9E3779B97F4A7C15) & self.M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.M
        return z ^ (z >> 31)

    def uniform(self) -> float:
        """53 random bits in [0, 1)."""
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


def random_bubbles(p: MkParams, number: int, rmin: float, rmax: float, gap: float, seed: int) -> None:
    """Non-overlapping bubbles: radius U[rmin, rmax], then centres drawn until
    the bubble keeps `gap` from every earlier bubble (minimum image on periodic
    axes) and from walled (fluid span [1, n-2]) or closed ([0, n-1]) faces."""
    if number < 0 or number > MAX_OBJECTS:
        raise CaseError(ST_XML, "random/bubbles out of range")
    rng = SplitMix64(seed)
    n3 = (p.nx, p.ny, p.nz)
    for b in range(number):
        R = rmin + (rmax - rmin) * rng.uniform()
        for _ in range(100000):
            c = [0.0, 0.0, 0.0]
            fits = True
            for a in range(3):
                if p.bc[a] == BC_PERIODIC:
                    c[a] = n3[a] * rng.uniform()
                    continue
                walled = p.bc[a] == BC_WALLS
                lo = (1.0 if walled else 0.0) + R + gap
                hi = (n3[a] - 2.0 if walled else n3[a] - 1.0) - R - gap
                u = rng.uniform()
                if hi < lo:
                    fits = False
                    continue
                c[a] = lo + (hi - lo) * u
            if not fits:
                continue
            for k in range(b):
                d2 = 0.0
                for a in range(3):
                    d = abs(c[a] - p.obj_center[k][a])
                    if p.bc[a] == BC_PERIODIC and d > 0.5 * n3[a]:
                        d = n3[a] - d
                    d2 += d * d
                need = R + p.obj_radius[k] + gap
                if d2 < need * need:
                    fits = False
                    break
            if fits:
                for a in range(3):
                    p.obj_center[b][a] = c[a]
                    p.obj_angle[b][a] = 0.0
                p.obj_radius[b] = R
                break
        else:
            raise CaseError(ST_ARG, "could not place the random bubbles without overlap")
    p.n_objects = number
    p.rng_seed = seed


def validate(p: MkParams) -> None:
    """The combinations the solver accepts (CaseError with status 2 otherwise)."""
    def bad(msg):
        raise CaseError(ST_ARG, msg)

    n3 = (p.nx, p.ny, p.nz)
    if min(n3) < 1:
        bad("MeshXYZ must be positive")
    if float(p.nx) * p.ny * p.nz >= 2147483647.0 - 64.0:
        bad("domain too large")
    for a in range(3):
        if p.bc[a] not in (BC_PERIODIC, BC_WALLS, BC_CLOSED):
            bad("bad boundary kind")
        if p.bc[a] == BC_WALLS and n3[a] < 3:
            bad("a walled axis needs at least 3 cells")
    if not 0 <= p.model <= MODEL["flow_solutal_dendrite"]:
        bad("unknown model")
    if not 0 <= p.precision <= 3:
        bad("unknown precision")
    if not -1 <= p.wall_axis <= 2:
        bad("wall_axis out of range")
    if p.wall_axis >= 0:
        if p.bc[p.wall_axis] != BC_WALLS:
            bad("the plate axis must have walled faces")
        if p.model not in (MODEL["flow"], MODEL["convection"]):
            bad("plates apply to the flow and convection models")
    if p.model == MODEL["convection"] and (not p.D > 0 or p.wall_axis < 0):
        bad("convection needs a positive diffusivity and a plate axis")
    if p.inlet:
        if p.model not in (MODEL["flow"],) + FLOW_COUPLED:
            bad("inflow / outflow faces apply to the flow and flow + dendrite models")
        if p.bc[0] != BC_CLOSED or p.nx < 3 or p.wall_axis == 0:
            bad("inflow / outflow faces need closed x faces, nx >= 3 and no x plates")
    if p.model in (MODEL["flow"], MODEL["convection"]) + FLOW_COUPLED:
        if p.lattice not in (19, 27) or not 0 <= p.collision <= 2:
            bad("flow lattice / collision")
        if p.collision == COLLISION["mrt"] and p.lattice != 19:
            bad("MRT is defined for D3Q19 only")
        if not p.tau > 0.5 or (p.collision == COLLISION["trt"] and not p.magic > 0) or not p.rho0 > 0:
            bad("flow parameters out of range")
    elif p.model == MODEL["multiphase"]:
        if not (p.tau_l > 0.5 and p.tau_g > 0.5 and p.rho_l > 0 and p.rho_g > 0 and p.width > 0 and p.mobility > 0):
            bad("multiphase parameters out of range")
    if p.model == MODEL["multigrain"]:
        if not 1 <= p.n_objects <= MAX_OBJECTS or not (p.W0 > 0 and p.mobility > 0 and p.D > 0):
            bad("multigrain parameters out of range")
    if p.model in DENDRITES:
        if not (p.W0 > 0 and p.tau0 > 0 and p.D > 0):
            bad("phase-field parameters out of range")
        if not 0 <= p.n_objects <= MAX_OBJECTS or not 0 <= p.aniso <= 3:
            bad("seed count / anisotropy kind")
        if p.aniso == ANISO["facet"] and not p.eps2 > 0:
            bad("facet anisotropy needs a positive cusp width")


_MODEL_WORDS = {
    "flow": "flow", "poiseuille": "flow", "multiphase": "multiphase", "allencahn": "multiphase",
    "allen_cahn": "multiphase", "thermal_dendrite": "thermal_dendrite", "thermal": "thermal_dendrite",
    "solutal_dendrite": "solutal_dendrite", "solutal": "solutal_dendrite", "convection": "convection",
    "rbc": "convection", "rayleigh_benard": "convection", "flow_dendrite": "flow_dendrite",
    "flow_thermal_dendrite": "flow_dendrite", "flow_solutal_dendrite": "flow_solutal_dendrite",
    "flow_solutal": "flow_solutal_dendrite", "multigrain": "multigrain", "multiphasefield": "multigrain",
    "multi_phase_field": "multigrain"}
_BC_WORDS = {"periodic": BC_PERIODIC, "p": BC_PERIODIC, "walls": BC_WALLS, "wall": BC_WALLS, "w": BC_WALLS,
             "bounceback": BC_WALLS, "closed": BC_CLOSED, "noflux": BC_CLOSED, "zeroflux": BC_CLOSED,
             "c": BC_CLOSED}


def _choice(node: Node, table: dict, what: str):
    w = _word(node)
    if w not in table:
        raise CaseError(ST_XML, f"<b200><{what}>: unknown '{w}'")
    return table[w]


def resolve(path: str, model=None, precision=None, collision=None, lattice=None, magic=None) -> MkParams:
    """Parameters of an XML case in lattice units, with optional overrides
    (names or the C enum values)."""
    r = parse_xml(path)
    p = defaults()
    mesh = r.find("geometry/MeshXYZ")
    if mesh is None:
        raise CaseError(ST_XML, "missing geometry/MeshXYZ")
    m = numbers(mesh)
    if len(m) < 3:
        raise CaseError(ST_XML, "geometry/MeshXYZ needs 3 values")
    p.nx, p.ny, p.nz = int(m[0]), int(m[1]), int(m[2])
    p.max_loops, p.max_frames = read_parameters(path)
    dx, dt = _opt(r, "numerics/mk_dx", 1.0), _opt(r, "numerics/mk_dt", 1.0)
    if not (dx > 0 and dt > 0):
        raise CaseError(ST_XML, "numerics/mk_dx and mk_dt must be positive")
    grav = _optv(r, "geometry/Gravity") or []
    g_lu = [(grav[a] if a < len(grav) else 0.0) * dt * dt / dx for a in range(3)]
    visc = lambda v: v * dt / (dx * dx)  # noqa: E731  (kinematic viscosity, diffusivity)

    b = r.child("b200")
    name = None
    if b is not None and b.child("model") is not None:
        name = _choice(b.child("model"), _MODEL_WORDS, "model")
    if model is not None:
        name = model if isinstance(model, str) else [k for k, v in MODEL.items() if v == model][0]
    if name is None:
        # calcMode as the driver reads it: a dendrite in a flow, a dendrite, or a flow
        dend = boolean(r.find("calcMode/dendrite")) if r.find("calcMode/dendrite") is not None else False
        flowf = boolean(r.find("calcMode/flowField")) if r.find("calcMode/flowField") is not None else False
        name = ("flow_dendrite" if flowf else "thermal_dendrite") if dend else "flow"
    p.model = MODEL[name]
    omega_f = _opt(r, "numerics/omega_f", -1.0)

    def flow_tau():
        nu = _opt(r, "phases/fluid/kinematicViscosity", -1.0)
        if nu > 0:
            p.tau = 3.0 * visc(nu) + 0.5
        if omega_f > 0:
            p.tau = 1.0 / omega_f

    if name == "convection":
        # bdy_RBC (mkFluidsUser.cpp:362-392): plates normal to y, highValue at
        # y = 0 and lowValue at y = My - 1, gravity from geometry/Gravity
        flow_tau()
        alpha = _opt(r, "temperature/alphaFluid", -1.0)
        if alpha > 0:
            p.D = visc(alpha)
        p.beta = _opt(r, "temperature/beta", 0.0)
        hi, lo = _opt(r, "composition/highValue", 1.0), _opt(r, "composition/lowValue", 0.0)
        p.rho0 = 1.0
        p.force[:] = g_lu
        p.bc[:] = [BC_PERIODIC, BC_WALLS, BC_PERIODIC]
        p.wall_axis = 1
        p.wall_value[:] = [hi, lo]
        p.s_ref = 0.5 * (hi + lo)
        p.collision = COLLISION["trt"]
    elif name == "flow":
        flow_tau()
        p.rho0 = 1.0
        acc = _optv(r, "flow/acceleration") or []
        p.force[:] = [(acc[a] if a < len(acc) else 0.0) + g_lu[a] for a in range(3)]
        # channel walls at y = 0 and y = My - 1 (mkFluidsUser.cpp:55-58)
        p.bc[:] = [BC_PERIODIC, BC_WALLS, BC_PERIODIC]
        p.collision = COLLISION["trt"]
    elif name == "multiphase":
        nu_d = _opt(r, "multiphases/fluidDense/kinematicViscosity", -1.0)
        rho_d = _opt(r, "multiphases/fluidDense/density", -1.0)
        nu_r = _opt(r, "multiphases/fluidRare/kinematicViscosity", -1.0)
        rho_r = _opt(r, "multiphases/fluidRare/density", -1.0)
        W, M = _opt(r, "multiphases/W0", -1.0), _opt(r, "multiphases/Mobility", -1.0)
        sig, th = _opt(r, "multiphases/sigma", -1.0), _opt(r, "multiphases/contactAngle", 90.0)
        if rho_d > 0 and rho_r > 0:
            p.rho_l, p.rho_g = 1.0, rho_r / rho_d
        if nu_d > 0:
            p.tau_l = 3.0 * visc(nu_d) + 0.5
        if nu_r > 0:
            p.tau_g = 3.0 * visc(nu_r) + 0.5
        if W > 0:
            p.width = W / dx
        if M > 0:
            p.mobility = visc(M)
        if sig > 0:
            p.sigma = sig
        p.contact_angle = th
        fd = _optv(r, "multiphases/force") or []
        p.force[:] = [g_lu[a] + ((fd[a] / rho_d * dt * dt / dx) if (a < len(fd) and rho_d > 0) else 0.0)
                      for a in range(3)]
        p.bc[:] = [BC_PERIODIC, BC_WALLS, BC_PERIODIC]
        p.collision = COLLISION["mrt"]
        _seeds(r.find("phasechange/seed"), p)
    else:
        W0, t0 = _opt(r, "phasechange/W0", 1.0), _opt(r, "phasechange/t0", 1.0)
        d0, lam = _opt(r, "phasechange/d0", -1.0), _opt(r, "phasechange/lambda", -1.0)
        p.eps4 = _opt(r, "phasechange/anisotropy", p.eps4)
        p.W0, p.tau0 = W0 / dx, t0 / dt
        if lam > 0:
            p.lambda_ = lam
        elif d0 > 0:
            p.lambda_ = 0.8839 * W0 / d0
        if name == "multigrain":
            # the grains' relaxation rate 1/(dt/dx^2/cs^2 + 1/2) (mkFluidsUser.cpp:282)
            p.mobility = 1.0
        if name in ("thermal_dendrite", "flow_dendrite", "multigrain"):
            alpha = _opt(r, "temperature/alphaFluid", -1.0)
            under = _opt(r, "temperature/undercooling", p.delta)
            ini = _opt(r, "temperature/iniValue", None)
            if alpha > 0:
                p.D = visc(alpha)
            p.delta = -ini if ini is not None else under
        else:
            dl, ds = _opt(r, "composition/diffFluid", -1.0), _opt(r, "composition/diffSolid", -1.0)
            kp, iv = _opt(r, "composition/partition", -1.0), _opt(r, "composition/iniValue", None)
            if dl > 0:
                p.D = visc(dl)
            if ds >= 0:
                p.D_s = visc(ds)
            if kp > 0:
                p.k_part = kp
            if iv is not None:
                p.delta = -iv
        p.bc[:] = [BC_CLOSED] * 3
        if name in ("flow_dendrite", "flow_solutal_dendrite"):
            # inflow at x = 0 with flow/velocityInlet, outflow at x = nx - 1
            # (boundary_vel, mkFluidsUser.cpp:455-617), periodic across
            flow_tau()
            vin = _optv(r, "flow/velocityInlet") or []
            acc = _optv(r, "flow/acceleration") or []
            p.u0[:] = [(vin[a] if a < len(vin) else 0.0) * dt / dx for a in range(3)]
            p.force[:] = [(acc[a] if a < len(acc) else 0.0) + g_lu[a] for a in range(3)]
            p.rho0 = 1.0
            p.inlet = 1
            p.bc[1] = p.bc[2] = BC_PERIODIC
            p.collision = COLLISION["trt"]
        _seeds(r.find("phasechange/seed"), p)

    if b is not None:
        _b200(b, p)
    if precision is not None:
        p.precision = PRECISION[precision] if isinstance(precision, str) else int(precision)
    if collision is not None:
        p.collision = COLLISION[collision.lower()] if isinstance(collision, str) else int(collision)
    if lattice is not None:
        p.lattice = int(lattice)
    if magic is not None and magic > 0:
        p.magic = float(magic)
    validate(p)
    return p


def _b200(b: Node, p: MkParams) -> None:
    """The <b200> element: lattice-unit values and the options the reference
    selects by code path."""
    if b.child("lattice") is not None:
        p.lattice = _choice(b.child("lattice"), {"d3q19": 19, "d3q27": 27}, "lattice")
    if b.child("collision") is not None:
        p.collision = _choice(b.child("collision"), COLLISION, "collision")
    if b.child("precision") is not None:
        p.precision = _choice(b.child("precision"), {"fp64": 0, "double": 0, "fp32": 1, "float": 1, "fp16": 2,
                                                     "half": 2, "bf16": 3}, "precision")
    if b.child("boundary") is not None:
        words = b.child("boundary").text.split()
        if len(words) != 3:
            raise CaseError(ST_XML, "<b200><boundary> needs 3 values")
        for a, w in enumerate(words):
            if w.lower() not in _BC_WORDS:
                raise CaseError(ST_XML, f"<b200><boundary>: unknown '{w.lower()}'")
            p.bc[a] = _BC_WORDS[w.lower()]
    if b.child("anisotropyKind") is not None:
        p.aniso = _choice(b.child("anisotropyKind"), ANISO, "anisotropyKind")
    scalars = {"eps2": "eps2", "magic": "magic", "tau": "tau", "rho0": "rho0", "rhoL": "rho_l", "rhoG": "rho_g",
               "tauL": "tau_l", "tauG": "tau_g", "sigma": "sigma", "width": "width", "mobility": "mobility",
               "contactAngle": "contact_angle", "eps4": "eps4", "W0": "W0", "lambda": "lambda_", "delta": "delta",
               "diffusivity": "D", "diffSolid": "D_s", "partition": "k_part", "antiTrapping": "at_coef",
               "grainKappa": "grain_kappa"}
    for tag, field in scalars.items():
        if b.child(tag) is not None:
            setattr(p, field, number(b.child(tag)))
    # tau0 from the thin-interface relation tau0 = 0.6267 lambda W0^2 / D unless given
    tau0 = number(b.child("tau0")) if b.child("tau0") is not None else -1.0
    if any(b.child(t) is not None for t in ("W0", "lambda", "diffusivity")) or tau0 > 0:
        p.tau0 = tau0 if tau0 > 0 else 0.6267 * p.lambda_ * p.W0 * p.W0 / p.D
    for tag, field in (("force", "force"), ("velocity", "u0"), ("grainVelocity", "grain_u")):
        if b.child(tag) is not None:
            v = numbers(b.child(tag))
            getattr(p, field)[:] = [v[a] if a < len(v) else 0.0 for a in range(3)]
    if b.child("wallAxis") is not None:
        p.wall_axis = _choice(b.child("wallAxis"), {"x": 0, "0": 0, "y": 1, "1": 1, "z": 2, "2": 2, "none": -1,
                                                    "-1": -1}, "wallAxis")
    if b.child("wallValue") is not None:
        v = numbers(b.child("wallValue"))
        if len(v) != 2:
            raise CaseError(ST_XML, "<b200><wallValue> needs 2 values")
        p.wall_value[:] = v
    if b.child("wallVelocity") is not None:
        v = numbers(b.child("wallVelocity"))
        if len(v) != 6:
            raise CaseError(ST_XML, "<b200><wallVelocity> needs 6 values")
        p.wall_u[0][:] = v[:3]
        p.wall_u[1][:] = v[3:]
    if b.child("beta") is not None:
        p.beta = number(b.child("beta"))
    if b.child("sRef") is not None:
        p.s_ref = number(b.child("sRef"))
    if b.child("inlet") is not None:
        p.inlet = 1 if number(b.child("inlet")) != 0.0 else 0
    if b.child("objects") is not None:
        _seeds(b.child("objects"), p)
    rb = b.child("random")
    if rb is not None:
        random_bubbles(p, int(_opt(rb, "bubbles", 0.0)), _opt(rb, "radiusMin", 8.0), _opt(rb, "radiusMax", 16.0),
                       _opt(rb, "gap", 2.0 * p.width), int(_opt(rb, "seed", 0.0)))


# ------------------------------------------------------------------ initial fields
def _coords(p: MkParams):
    z, y, x = np.meshgrid(np.arange(p.nz, dtype=np.float64), np.arange(p.ny, dtype=np.float64),
                          np.arange(p.nx, dtype=np.float64), indexing="ij")
    return x, y, z


def _dist2(p: MkParams, k: int, xyz, periodic: bool):
    n3 = (p.nx, p.ny, p.nz)
    d2 = np.zeros(xyz[0].shape)
    for a in range(3):
        d = np.abs(xyz[a] - p.obj_center[k][a])
        if periodic and p.bc[a] == BC_PERIODIC:
            d = np.where(d > 0.5 * n3[a], n3[a] - d, d)
        d2 += d * d
    return d2


def bubble_phi(p: MkParams, xyz=None) -> np.ndarray:
    """Gas bubbles (phi = 0) in liquid (phi = 1): the smallest
    1/2 (1 + tanh(2 (d_k - R_k) / W)) over the bubbles, d_k with the minimum
    image on periodic axes.  A bubble is evaluated only inside its box of
    half-width R + 10 W: beyond d - R = 10 W the double-precision profile is
    exactly 1 and leaves the minimum unchanged."""
    n3 = (p.nx, p.ny, p.nz)
    ph = np.ones((p.nz, p.ny, p.nx))
    for k in range(p.n_objects):
        reach = p.obj_radius[k] + 10.0 * p.width
        idx, dist = [], []
        for a in range(3):
            c = p.obj_center[k][a]
            lo, hi = math.floor(c - reach), math.ceil(c + reach)
            if p.bc[a] == BC_PERIODIC:
                i = np.arange(n3[a]) if hi - lo + 1 >= n3[a] else np.unique(np.arange(lo, hi + 1) % n3[a])
                d = np.abs(i - c)
                d = np.where(d > 0.5 * n3[a], n3[a] - d, d)
            else:
                i = np.arange(max(lo, 0), min(hi, n3[a] - 1) + 1)
                d = np.abs(i - c)
            idx.append(i)
            dist.append(d.astype(np.float64))
        dx, dy, dz = dist[0][None, None, :], dist[1][None, :, None], dist[2][:, None, None]
        d2 = (dx * dx + dy * dy) + dz * dz
        phk = 0.5 * (1.0 + np.tanh(2.0 * (np.sqrt(d2) - p.obj_radius[k]) / p.width))
        box = np.ix_(idx[2], idx[1], idx[0])
        ph[box] = np.minimum(ph[box], phk)
    return ph


def grain_phi(p: MkParams, k: int, xyz=None) -> np.ndarray:
    """Order parameter of seed k alone (solid +1 inside): -tanh((r - R)/(sqrt 2 W0))."""
    xyz = _coords(p) if xyz is None else xyz
    return -np.tanh((np.sqrt(_dist2(p, k, xyz, False)) - p.obj_radius[k]) / (math.sqrt(2.0) * p.W0))


def seed_phi(p: MkParams, xyz=None) -> np.ndarray:
    """Solid seeds in liquid (-1): the largest single-seed profile."""
    xyz = _coords(p) if xyz is None else xyz
    ph = -np.ones(xyz[0].shape)
    for k in range(p.n_objects):
        np.maximum(ph, grain_phi(p, k, xyz), out=ph)
    return ph


def flags(p: MkParams) -> np.ndarray:
    """Node flags: 3 (walls) on the first and last cell of a walled axis, else 0."""
    xyz = _coords(p)
    n3 = (p.nx, p.ny, p.nz)
    wall = np.zeros(xyz[0].shape, dtype=bool)
    for a in range(3):
        if p.bc[a] == BC_WALLS:
            wall |= (xyz[a] == 0) | (xyz[a] == n3[a] - 1)
    return np.where(wall, float(FLAG_WALLS), float(FLAG_FLUID))


def initial_field(p: MkParams, name: str) -> np.ndarray:
    """Initial macroscopic field (nz, ny, nx) float64 of the case."""
    xyz = _coords(p)
    shape = xyz[0].shape
    dendrite = p.model in DENDRITES
    if name == "flag":
        return flags(p)
    if name == "phi":
        if p.model == MODEL["multiphase"]:
            return bubble_phi(p, xyz)
        if p.model in (MODEL["flow"], MODEL["convection"]):
            return np.zeros(shape)
        if p.model == MODEL["multigrain"]:
            # aggregate (N - 1) + sum_j phi_j (mkFluidsUser.cpp:162-168)
            agg = np.full(shape, p.n_objects - 1.0)
            for k in range(p.n_objects):
                agg += grain_phi(p, k, xyz)
            return agg
        return seed_phi(p, xyz)
    if name == "rho":
        if p.model == MODEL["multiphase"]:
            return p.rho_g + bubble_phi(p, xyz) * (p.rho_l - p.rho_g)
        return np.full(shape, p.rho0)
    if name in ("ux", "uy", "uz"):
        a = "xyz".index(name[1])
        if p.model in FLOW_COUPLED:
            ns = np.clip(0.5 * (1.0 + seed_phi(p, xyz)), 0.0, 1.0)
            return (1.0 - ns) * p.u0[a]
        if p.model in (MODEL["flow"], MODEL["convection"]):
            return np.full(shape, p.u0[a])
        return np.zeros(shape)
    if name in ("T", "C"):
        if p.model == MODEL["convection"]:
            # conduction between the half-way plates plus one roll mode of
            # amplitude 1e-2 (T_low - T_high) along the first other axis
            a = p.wall_axis
            o = 1 if a == 0 else 0
            n3 = (p.nx, p.ny, p.nz)
            lo = 1 if p.bc[a] == BC_WALLS else 0
            hi = n3[a] - 2 if p.bc[a] == BC_WALLS else n3[a] - 1
            s = np.clip((xyz[a] - lo + 0.5) / (hi - lo + 1), 0.0, 1.0)
            dT = p.wall_value[0] - p.wall_value[1]
            return p.wall_value[0] - dT * s + 1e-2 * dT * np.sin(math.pi * s) * np.cos(2.0 * math.pi * xyz[o] / n3[o])
        return np.full(shape, -p.delta)
    if name in ("pressure", "dphi"):
        return np.zeros(shape)
    if name == "grain":
        if dendrite and p.n_objects > 0:
            # nearest seed, ties to the lower index
            best = np.zeros(shape)
            bd = np.full(shape, np.inf)
            for k in range(p.n_objects):
                d2 = _dist2(p, k, xyz, False)
                closer = d2 < bd
                best[closer] = k
                bd = np.where(closer, d2, bd)
            return best
        if p.model == MODEL["multigrain"]:
            best = np.zeros(shape)
            bp = np.full(shape, -np.inf)
            for k in range(p.n_objects):
                g = grain_phi(p, k, xyz)
                larger = g > bp
                best[larger] = k
                bp = np.where(larger, g, bp)
            return best
        return np.zeros(shape)
    raise KeyError(name)


def oracle_fields(p: MkParams) -> dict:
    """The initial fields the oracle library takes (phi, T, C), keyed by its
    constructor's argument names."""
    return {"phi": initial_field(p, "phi"), "T": initial_field(p, "T"), "Cc": initial_field(p, "C")}


# ------------------------------------------------------------------ seeded ensemble
def ensemble(seed: int, n: int, precision="bf16") -> list[MkParams]:
    """The seeded solutal ensemble: n cubes with edges drawn from
    {48, 64, 80, 96, 128}, eps4 ~ U[0.02, 0.06], 1-6 seeds of radius U[4, 8]
    at uniform positions (2 cells clear of the faces) with uniformly random
    orientations (Shoemake's uniform quaternion, written as ZYX angles);
    k = 0.15, D_l = 0.1, D_s = 1e-4, W0 = 1.5, lambda = 10, Delta = 0.55."""
    if not 1 <= n <= 4096:
        raise CaseError(ST_ARG, "ensemble size out of range")
    rng = SplitMix64(seed)
    prec = PRECISION[precision] if isinstance(precision, str) else int(precision)
    out = []
    for _ in range(n):
        p = defaults()
        p.model = MODEL["solutal_dendrite"]
        p.precision = prec
        L = (48, 64, 80, 96, 128)[rng.next() % 5]
        p.nx = p.ny = p.nz = L
        p.bc[:] = [BC_CLOSED] * 3
        p.max_loops = 3000
        p.eps4 = 0.02 + 0.04 * rng.uniform()
        p.k_part, p.D, p.D_s, p.W0, p.lambda_, p.delta = 0.15, 0.1, 1e-4, 1.5, 10.0, 0.55
        p.tau0 = 0.6267 * p.lambda_ * p.W0 * p.W0 / p.D
        p.n_objects = 1 + rng.next() % 6
        for s in range(p.n_objects):
            R = 4.0 + 4.0 * rng.uniform()
            for a in range(3):
                p.obj_center[s][a] = (R + 2.0) + (L - 1 - 2.0 * (R + 2.0)) * rng.uniform()
            p.obj_radius[s] = R
            u1, u2, u3 = rng.uniform(), rng.uniform(), rng.uniform()
            qx, qy = math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2)
            qz, qw = math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3)
            r00, r10, r20 = 1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy + qz * qw), 2 * (qx * qz - qy * qw)
            r21, r22 = 2 * (qy * qz + qx * qw), 1 - 2 * (qx * qx + qy * qy)
            deg = 180.0 / math.pi
            p.obj_angle[s][0] = math.atan2(r21, r22) * deg
            p.obj_angle[s][1] = -math.asin(max(-1.0, min(1.0, r20))) * deg
            p.obj_angle[s][2] = math.atan2(r10, r00) * deg
        p.rng_seed = seed
        validate(p)
        out.append(p)
    return out
