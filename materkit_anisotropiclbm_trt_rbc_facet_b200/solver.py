"""Host-side mirror of MaterKit's solver interface on top of the C ABI.

Two layers:

* :class:`Solver` — the direct wrapper of ``include/mkb200.h`` (create from a
  BoltzTechs XML case, advance N loops, read fields, VTK output, diagnostics,
  checkpoints).
* ``mkSpace`` / ``readParameters`` / ``mkFluidsMRT`` / ``mkFluidsMultiphase`` —
  the reference's class names and call sequence (MaterKit/MaterKit.cpp:36-124,
  :244-288, :290-331, :743-788), so a MaterKit-style driver ports line by line.
  The reference calls ``propagate()`` and ``relaxation*()`` per field; here the
  device executes one fused launch sequence per loop when the loop's last
  relaxation is called.

Everything runs on the GPU through ``libmkb200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi as A


def _check(status: int, handle=None) -> None:
    if status != A.MK_OK:
        lib = A.load()
        msg = lib.mk_last_error(handle) if handle else lib.mk_last_global_error()
        raise A.MkError(status, (msg or b"").decode(errors="replace"))


def _opts(model=None, precision=None, collision=None, lattice=None, magic=None, block=None) -> A.MkOptions:
    m = A.MODELS[model] if isinstance(model, str) else (-1 if model is None else int(model))
    p = A.PRECISIONS[precision] if isinstance(precision, str) else (-1 if precision is None else int(precision))
    c = {"bgk": 0, "trt": 1, "mrt": 2}[collision.lower()] if isinstance(collision, str) else (
        -1 if collision is None else int(collision))
    lat = -1 if lattice is None else int(lattice)
    bx, by = block if block else (0, 0)
    return A.MkOptions.make(m, p, c, lat, -1.0 if magic is None else float(magic), -1, bx, by)


def readParameters(xml_path: str) -> tuple[int, int]:
    """readParameters(maxLoops, maxFrame, xml) — MaterKit/inc/mkFunction.h:62."""
    lib = A.load()
    loops, frames = C.c_int32(), C.c_int32()
    _check(lib.mk_read_parameters(os.fsencode(xml_path), C.byref(loops), C.byref(frames)))
    return loops.value, frames.value


def case_params(xml_path: str, **opts) -> A.MkParams:
    """Resolve an XML case to lattice-unit parameters (no GPU needed)."""
    lib = A.load()
    p = A.MkParams()
    o = _opts(**opts)
    _check(lib.mk_case_params(os.fsencode(xml_path), C.byref(o), C.byref(p)))
    return p


def initial_field(params: A.MkParams, field: str) -> np.ndarray:
    """Initial macroscopic field of a case as (nz, ny, nx) float64 (no GPU needed)."""
    lib = A.load()
    n = params.ncell()
    out = np.empty(n, dtype=np.float64)
    _check(lib.mk_case_initial_field(C.byref(params), A.FIELDS[field],
                                     out.ctypes.data_as(C.POINTER(C.c_double)), n))
    return out.reshape(params.nz, params.ny, params.nx)


def ensemble_params(seed: int, n_domains: int, precision: str | int = "bf16") -> list[A.MkParams]:
    """The seeded solutal ensemble: n cubes with edges from {48, 64, 80, 96, 128},
    eps4 ~ U[0.02, 0.06], 1-6 randomly oriented seeds (no GPU needed)."""
    lib = A.load()
    prec = A.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    arr = (A.MkParams * int(n_domains))()
    _check(lib.mk_ensemble_case_params(int(seed), int(n_domains), prec, arr))
    return list(arr)


class Ensemble:
    """Many dendrite domains advanced together in one packed lattice (the
    ensemble of ``run_solutal_dendrite`` / ``run_thermal_dendrite`` sweeps,
    MaterKit/MaterKit.cpp:633-687, :743-788).  Every loop is two persistent
    launches over all domains; ``advance`` replays two loops as a CUDA graph."""

    def __init__(self, params: list[A.MkParams]):
        self._lib = A.load()
        self._h = C.c_void_p()
        self.params = [p for p in params]
        arr = (A.MkParams * len(self.params))(*self.params)
        _check(self._lib.mk_ensemble_create(arr, len(self.params), C.byref(self._h)))

    def close(self) -> None:
        if self._h:
            self._lib.mk_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, status: int) -> None:
        if status != A.MK_OK:
            msg = self._lib.mk_ensemble_last_error(self._h) if self._h else self._lib.mk_last_global_error()
            raise A.MkError(status, (msg or b"").decode(errors="replace"))

    def __len__(self) -> int:
        return len(self.params)

    @property
    def cells(self) -> int:
        return int(self._lib.mk_ensemble_cells(self._h))

    @property
    def step(self) -> int:
        return int(self._lib.mk_ensemble_step(self._h))

    def advance(self, nsteps: int) -> None:
        self._chk(self._lib.mk_ensemble_advance(self._h, int(nsteps)))

    def time_advance(self, nsteps: int) -> float:
        ms = C.c_double()
        self._chk(self._lib.mk_ensemble_time_advance(self._h, int(nsteps), C.byref(ms)))
        return ms.value

    def profile(self, nsteps: int, kernel: str = "collide") -> dict:
        """Device time of one launch kind over `nsteps` eager loops (CUDA events)."""
        k, t = C.c_double(), C.c_double()
        self._chk(self._lib.mk_ensemble_profile_steps(self._h, int(nsteps), kernel.encode(), C.byref(k), C.byref(t)))
        return {"kernel_ms": k.value, "step_ms": t.value, "launches": int(nsteps)}

    @property
    def launches(self) -> int:
        return int(self._lib.mk_ensemble_launches(self._h))

    def field(self, domain: int, name: str, dtype=np.float64) -> np.ndarray:
        if not 0 <= domain < len(self.params):
            raise A.MkError(A.MK_ERR_ARG, f"domain index {domain} out of range")
        p = self.params[domain]
        dt = np.dtype(dtype)
        code = A.MK_DTYPE_F64 if dt == np.float64 else A.MK_DTYPE_F32
        out = np.empty(p.ncell(), dtype=dt)
        self._chk(self._lib.mk_ensemble_get_field(self._h, int(domain), A.FIELDS[name], code, out.ctypes.data,
                                                  out.nbytes))
        return out.reshape(p.nz, p.ny, p.nx)


class Solver:
    """One device-resident case (a handle of the C ABI)."""

    def __init__(self, xml_path: str | None = None, params: A.MkParams | None = None, **opts):
        self._lib = A.load()
        self._h = C.c_void_p()
        if params is not None:
            _check(self._lib.mk_create(C.byref(params), C.byref(self._h)))
        elif xml_path is not None:
            o = _opts(**opts)
            _check(self._lib.mk_create_from_xml(os.fsencode(xml_path), C.byref(o), C.byref(self._h)))
        else:
            raise ValueError("Solver needs xml_path or params")
        self.params = A.MkParams()
        _check(self._lib.mk_get_params(self._h, C.byref(self.params)), self._h)

    # -- lifecycle -----------------------------------------------------------
    def close(self) -> None:
        if self._h:
            self._lib.mk_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def shape(self) -> tuple[int, int, int]:
        return self.params.nz, self.params.ny, self.params.nx

    @property
    def step(self) -> int:
        return int(self._lib.mk_get_step(self._h))

    # -- stepping ------------------------------------------------------------
    def advance(self, nsteps: int, graph: bool = False) -> None:
        fn = self._lib.mk_advance_graph if graph else self._lib.mk_advance
        _check(fn(self._h, int(nsteps)), self._h)

    def sync(self) -> None:
        _check(self._lib.mk_sync(self._h), self._h)

    def stream(self) -> int:
        s = C.c_void_p()
        _check(self._lib.mk_get_stream(self._h, C.byref(s)), self._h)
        return s.value or 0

    # -- fields --------------------------------------------------------------
    def field(self, name: str, dtype=np.float64, out: np.ndarray | None = None) -> np.ndarray:
        dt = np.dtype(dtype)
        code = A.MK_DTYPE_F64 if dt == np.float64 else A.MK_DTYPE_F32
        n = self.params.ncell()
        if out is None:
            out = np.empty(n, dtype=dt)
        _check(self._lib.mk_get_field(self._h, A.FIELDS[name], code, out.ctypes.data, out.nbytes), self._h)
        return out.reshape(self.shape)

    def grain_field(self, grain: int, dtype=np.float64) -> np.ndarray:
        """Order parameter of one grain of a multigrain case, (nz, ny, nx)."""
        out = np.empty(self.shape, dtype=dtype)
        dt = A.MK_DTYPE_F64 if out.dtype == np.float64 else A.MK_DTYPE_F32
        _check(self._lib.mk_get_grain_field(self._h, int(grain), dt, out.ctypes.data_as(C.c_void_p), out.nbytes),
               self._h)
        return out

    def set_state(self, phi=None, T=None, C_=None, rho=None, u=None) -> None:
        def ptr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float64).ravel()
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_double))

        keep: list = []
        ux = uy = uz = None
        if u is not None:
            ux, uy, uz = (ptr(u[k]) for k in range(3))
        _check(self._lib.mk_set_state(self._h, ptr(phi), ptr(T), ptr(C_), ptr(rho), ux, uy, uz), self._h)

    def set_state_f32(self, phi=None, T=None, C_=None) -> None:
        keep = []

        def ptr(a):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=np.float32).ravel()
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_float))

        _check(self._lib.mk_set_state_f32(self._h, ptr(phi), ptr(T), ptr(C_)), self._h)

    # -- output --------------------------------------------------------------
    def write_vtk(self, loops: int, directory: str) -> str:
        os.makedirs(directory, exist_ok=True)
        _check(self._lib.mk_write_vtk(self._h, int(loops), os.fsencode(directory)), self._h)
        return os.path.join(directory, f"fluid_t{loops}.vtk")

    def _iso(self, iso):
        if iso is not None:
            return float(iso)
        return 0.5 if self.params.model == A.MK_MODEL_MULTIPHASE else 0.0

    def interface_points(self, iso: float | None = None) -> dict:
        """phi = iso contour points ((N, 3) VTK coordinates) and the scalar
        (T or C of the dendrite models) interpolated at them; iso defaults to 0
        (dendrites) or 1/2 (multiphase)."""
        iso = self._iso(iso)
        n = C.c_int64()
        _check(self._lib.mk_interface_points(self._h, iso, None, None, 0, C.byref(n)), self._h)
        xyz = np.zeros((max(n.value, 1), 3))
        sc = np.zeros(max(n.value, 1))
        dp = C.POINTER(C.c_double)
        _check(self._lib.mk_interface_points(self._h, iso, xyz.ctypes.data_as(dp), sc.ctypes.data_as(dp), n.value,
                                             C.byref(n)), self._h)
        return {"xyz": xyz[:n.value], "scalar": sc[:n.value], "iso": iso}

    def write_contour_csv(self, loops: int, directory: str, iso: float | None = None) -> str:
        """loops<loops>.csv of the phi = iso contour points, in the column
        layout of a ParaView contour export (order_parameter, temperature or
        solute, Points:0..2), 8 significant digits."""
        pts = self.interface_points(iso)
        os.makedirs(directory, exist_ok=True)
        path = os.path.join(directory, f"loops{loops}.csv")
        name = "X0_solutes" if self.params.model == A.MK_MODEL_SOLUTAL_DENDRITE else "temperature"
        with open(path, "w") as f:
            f.write(f'"order_parameter","{name}","Points:0","Points:1","Points:2"\n')
            for (x, y, z), v in zip(pts["xyz"], pts["scalar"]):
                f.write(f"{pts['iso']:.8g},{v:.8g},{x:.8g},{y:.8g},{z:.8g}\n")
        return path

    def tip(self, seed: int = 0, iso: float | None = None) -> dict:
        """Distances from the seed centre to the outermost interface crossing
        along +x, -x, +y, -y, +z, -z, and their change per loop since the
        previous call for the same seed."""
        t = A.MkTip()
        _check(self._lib.mk_tip_track(self._h, int(seed), self._iso(iso), C.byref(t)), self._h)
        return {"step": t.step, "length": list(t.length), "velocity": list(t.velocity)}

    def diagnostics(self, raise_on_divergence: bool = True) -> dict:
        d = A.MkDiag()
        st = self._lib.mk_diagnostics(self._h, C.byref(d))
        if st == A.MK_ERR_DIVERGED and not raise_on_divergence:
            return d.to_dict()
        _check(st, self._h)
        return d.to_dict()

    def checkpoint(self, path: str) -> None:
        _check(self._lib.mk_checkpoint(self._h, os.fsencode(path)), self._h)

    def restore(self, path: str) -> None:
        _check(self._lib.mk_restore(self._h, os.fsencode(path)), self._h)

    # -- measurement ----------------------------------------------------------
    def profile(self, nsteps: int, kernel: str = "collide") -> dict:
        k, s, n = C.c_double(), C.c_double(), C.c_int64()
        _check(self._lib.mk_profile_steps(self._h, int(nsteps), kernel.encode(), C.byref(k), C.byref(s),
                                          C.byref(n)), self._h)
        return {"kernel_ms": k.value, "step_ms": s.value, "launches": n.value}

    def time_advance(self, nsteps: int, graph: bool = True) -> float:
        """Advance with CUDA events around the launches; returns device milliseconds."""
        ms = C.c_double()
        _check(self._lib.mk_time_advance(self._h, int(nsteps), 1 if graph else 0, C.byref(ms)), self._h)
        return ms.value

    def nusselt(self) -> float:
        """Nusselt number of a convection case (FP64 reduction on the device)."""
        nu = C.c_double()
        _check(self._lib.mk_nusselt(self._h, C.byref(nu)), self._h)
        return nu.value

    def backward(self, target_phi, steps: int, checkpoint_every: int = 100) -> dict:
        """Discrete adjoint of `steps` thermal dendrite loops from the current
        state: L = sum (phi - target)^2 and dL/d eps4, dL/d Delta, dL/d tau_T.
        Leaves the state after the forward run."""
        t = np.ascontiguousarray(target_phi, dtype=np.float64).ravel()
        if t.size != self.params.ncell():
            raise ValueError("target_phi must have one value per cell")
        loss = A.MkLoss(t.ctypes.data_as(C.POINTER(C.c_double)), int(steps), int(checkpoint_every))
        g = A.MkGrad()
        _check(self._lib.mk_backward(self._h, C.byref(loss), C.byref(g)), self._h)
        return {"loss": g.loss, "d_eps4": g.d_eps4, "d_delta": g.d_delta, "d_tau_t": g.d_tau_t,
                "forward_loops": g.forward_loops}

    def autotune(self, trial_steps: int = 4) -> dict:
        """Pick the fastest launch shape / occupancy variant; the state is left unchanged."""
        bx, by, mb, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _check(self._lib.mk_autotune(self._h, int(trial_steps), C.byref(bx), C.byref(by), C.byref(mb),
                                     C.byref(ms)), self._h)
        return {"block": (bx.value, by.value), "minb": mb.value, "ms_per_step": ms.value}

    @property
    def fused(self) -> bool:
        """Whether a multiphase loop runs as a fused one-launch form."""
        return bool(self._lib.mk_get_fused(self._h))

    @fused.setter
    def fused(self, on: bool) -> None:
        _check(self._lib.mk_set_fused(self._h, 1 if on else 0), self._h)

    # -- coupling of a dendrite and a two-phase flow (run_flow_multiphase_dendrite)
    def update_geometry(self, dendrite: "Solver") -> None:
        """This multiphase flow takes the dendrite's solid (phi > 0) as geometry
        from its next even loop count (mkFluidsMultiphase::update_geometry)."""
        _check(self._lib.mk_update_geometry(self._h, dendrite.handle), self._h)

    def update_velocity(self, flow: "Solver") -> None:
        """This dendrite's scalar lattice is advected by the flow's velocity
        (mkThermalField::update_velocity)."""
        _check(self._lib.mk_update_velocity(self._h, flow.handle), self._h)

    @property
    def tuning(self) -> dict:
        """The launch configuration (block shape, occupancy variant, loop and
        collision forms) as a dict; assign a dict (or a subset) to pin it."""
        t = A.MkTuning()
        _check(self._lib.mk_get_tuning(self._h, C.byref(t)), self._h)
        return t.to_dict()

    @tuning.setter
    def tuning(self, d: dict) -> None:
        cur = self.tuning
        cur.update(d)
        t = A.MkTuning(**{k: int(v) for k, v in cur.items()})
        _check(self._lib.mk_set_tuning(self._h, C.byref(t)), self._h)

    @property
    def row_staged(self) -> bool:
        """Whether the multiphase collision stages whole x rows through shared
        memory with the bulk-copy engine."""
        return bool(self._lib.mk_get_row_staging(self._h))

    @row_staged.setter
    def row_staged(self, on: bool) -> None:
        _check(self._lib.mk_set_row_staging(self._h, 1 if on else 0), self._h)

    def bytes_per_cell(self) -> float:
        return float(self._lib.mk_bytes_per_cell(self._h))

    def fluid_cells(self) -> int:
        return int(self._lib.mk_fluid_cells(self._h))

    def launches_per_step(self) -> int:
        return int(self._lib.mk_launches_per_step(self._h))


# ---------------------------------------------------------------------------
# Reference-named interface (MaterKit/inc/mkSpace.h, mkFluidsMRT.h, mkFluidsMultiphase.h)
# ---------------------------------------------------------------------------
class mkSpace:
    """mkSpace(xml) — grid size from geometry/MeshXYZ (MaterKit/inc/mkSpace.h:36)."""

    def __init__(self, xml_path: str):
        self.xml = xml_path
        p = case_params(xml_path)
        self._m = (p.nx, p.ny, p.nz)

    def Mx(self) -> int:
        return self._m[0]

    def My(self) -> int:
        return self._m[1]

    def Mz(self) -> int:
        return self._m[2]


class _RefSolver:
    """Common part of the reference-named solver classes.

    The per-loop call sequence of the reference driver is recorded in
    ``_SEQ``; the fused device loop runs when the sequence completes.  Calls
    out of order raise MkError(MK_ERR_STATE).
    """

    _MODEL = A.MK_MODEL_FLOW
    _SEQ: dict = {}

    def __init__(self, space: mkSpace | None = None, precision: str | None = None):
        self.space = space
        self.precision = precision
        self.xml = space.xml if space else None
        self.solver: Solver | None = None
        self._pending: list[str] = []
        self._model = self._MODEL

    def reset(self, xml_path: str) -> None:
        self.xml = xml_path

    def initialize(self, xml_path: str | None = None, model: int | None = None) -> None:
        if xml_path:
            self.xml = xml_path
        if model is not None:
            self._model = model
        self.solver = Solver(self.xml, model=self._model, precision=self.precision)

    def initialize_geometry(self) -> None:
        if self.solver is None:
            raise A.MkError(A.MK_ERR_STATE, "initialize() first")

    def _call(self, name: str) -> None:
        if self.solver is None:
            raise A.MkError(A.MK_ERR_STATE, "initialize() first")
        seq = self._SEQ[self._model]
        k = len(self._pending)
        if k >= len(seq) or seq[k] != name:
            raise A.MkError(A.MK_ERR_STATE, f"{name}() out of order; this loop expects {seq}")
        self._pending.append(name)
        if len(self._pending) == len(seq):
            self._pending.clear()
            self.solver.advance(1)

    def write_vtkfile(self, loops: int, directory: str = "vtk") -> str:
        return self.solver.write_vtk(loops, directory)

    def check_variables(self, loops: int, plane: str = "x") -> dict:
        return self.solver.diagnostics()


class mkFluidsMRT(_RefSolver):
    """Flow / phase-field solver class (MaterKit/inc/mkFluidsMRT.h:26-49)."""

    _MODEL = A.MK_MODEL_FLOW
    _SEQ = {
        A.MK_MODEL_FLOW: ["propagate", "relaxation"],
        A.MK_MODEL_THERMAL_DENDRITE: ["phasefield_propagate", "relaxation_anisotropy_thermal",
                                      "thermal_propagate", "thermal_relaxation"],
        # run_flow_thermal_dendrite (MaterKit.cpp:499-516)
        A.MK_MODEL_FLOW_DENDRITE: ["propagate_PBB", "relaxation", "bdyVelocity", "phasefield_propagate",
                                   "relaxation_anisotropy_thermal", "thermal_propagate", "thermal_relaxation",
                                   "bdy_flowin"],
        # run_multiPhaseField (MaterKit.cpp:563-567)
        A.MK_MODEL_MULTIGRAIN: ["propagate", "relaxation", "thermal_propagate", "thermal_relaxation"],
        # run_solutal_dendrite (MaterKit.cpp:665-674)
        A.MK_MODEL_SOLUTAL_DENDRITE: ["phasefield_propagate", "relaxation_anisotropy_solute", "solutal_propagate",
                                      "solutal_relaxation"],
        # run_flow_solutal_dendrite (MaterKit.cpp:430-456)
        A.MK_MODEL_FLOW_SOLUTAL: ["propagate_PBB", "relaxation", "bdyVelocity", "phasefield_propagate",
                                  "relaxation_anisotropy_solute", "solutal_propagate", "solutal_relaxation",
                                  "bdy_LBflowin"],
    }

    def initialize_geometry_Poiseuille(self) -> None:
        self.initialize_geometry()

    def propagate(self) -> None:
        self._call("propagate")

    def relaxation(self) -> None:
        self._call("relaxation")

    def propagate_PBB(self) -> None:
        self._call("propagate_PBB")

    def bdyVelocity(self) -> None:
        self._call("bdyVelocity")

    def bdy_flowin(self) -> None:
        self._call("bdy_flowin")

    # mkPhaseField / mkThermalField members, called as flow.mkPhaseField::propagate() in C++
    def phasefield_propagate(self) -> None:
        self._call("phasefield_propagate")

    def relaxation_anisotropy_thermal(self) -> None:
        self._call("relaxation_anisotropy_thermal")

    def thermal_propagate(self) -> None:
        self._call("thermal_propagate")

    def thermal_relaxation(self) -> None:
        self._call("thermal_relaxation")

    # mkPhaseField / mkSolutalField members of the solutal drivers
    def relaxation_anisotropy_solute(self, loops: int | None = None) -> None:
        self._call("relaxation_anisotropy_solute")

    def solutal_propagate(self) -> None:
        self._call("solutal_propagate")

    def solutal_relaxation(self) -> None:
        self._call("solutal_relaxation")

    def bdy_LBflowin(self) -> None:
        self._call("bdy_LBflowin")


class mkFluidsMultiphase(_RefSolver):
    """Allen-Cahn two-phase flow (MaterKit/inc/mkFluidsMultiphase.h:20-99)."""

    _MODEL = A.MK_MODEL_MULTIPHASE
    _SEQ = {A.MK_MODEL_MULTIPHASE: ["propagate", "relaxation"]}

    def propagate(self) -> None:
        self._call("propagate")

    def relaxation(self) -> None:
        self._call("relaxation")
