"""ctypes declarations of ``include/mkb200.h`` and the loader of ``libmkb200.so``.

The structures below mirror the C structs field for field; ``check_layout``
compares their sizes with the values the library was compiled with.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmkb200.so")

MK_OK, MK_ERR_XML, MK_ERR_ARG, MK_ERR_CUDA, MK_ERR_DIVERGED, MK_ERR_TIMEOUT, MK_ERR_OOM, MK_ERR_IO, MK_ERR_STATE, \
    MK_ERR_NODEVICE = range(10)
STATUS_NAMES = {0: "MK_OK", 1: "MK_ERR_XML", 2: "MK_ERR_ARG", 3: "MK_ERR_CUDA", 4: "MK_ERR_DIVERGED",
                5: "MK_ERR_TIMEOUT", 6: "MK_ERR_OOM", 7: "MK_ERR_IO", 8: "MK_ERR_STATE", 9: "MK_ERR_NODEVICE"}

(MK_MODEL_FLOW, MK_MODEL_MULTIPHASE, MK_MODEL_THERMAL_DENDRITE, MK_MODEL_SOLUTAL_DENDRITE, MK_MODEL_CONVECTION,
 MK_MODEL_FLOW_DENDRITE, MK_MODEL_MULTIGRAIN, MK_MODEL_FLOW_SOLUTAL) = range(8)
MK_PREC_FP64, MK_PREC_FP32, MK_PREC_FP16, MK_PREC_BF16 = range(4)
MK_COLL_BGK, MK_COLL_TRT, MK_COLL_MRT = range(3)
MK_D3Q7, MK_D3Q19, MK_D3Q27 = 7, 19, 27
MK_BC_PERIODIC, MK_BC_WALLS, MK_BC_CLOSED = range(3)
MK_ANISO_CUBIC, MK_ANISO_CBC, MK_ANISO_HCP, MK_ANISO_FACET = range(4)
ANISOTROPIES = {"cubic": MK_ANISO_CUBIC, "cbc": MK_ANISO_CBC, "hcp": MK_ANISO_HCP, "facet": MK_ANISO_FACET}
(MK_FIELD_RHO, MK_FIELD_UX, MK_FIELD_UY, MK_FIELD_UZ, MK_FIELD_T, MK_FIELD_C, MK_FIELD_PHI, MK_FIELD_FLAG,
 MK_FIELD_PRESSURE, MK_FIELD_DPHI, MK_FIELD_GRAIN) = range(11)
MK_DTYPE_F64, MK_DTYPE_F32 = 0, 1
MK_FLAG_FLUID, MK_FLAG_INTER, MK_FLAG_SOLID, MK_FLAG_WALLS = range(4)
MK_MAX_OBJECTS = 64
MK_NOALLOC_MAX_CELLS = 2048 * 256 * 64

PRECISIONS = {"fp64": MK_PREC_FP64, "fp32": MK_PREC_FP32, "fp16": MK_PREC_FP16, "bf16": MK_PREC_BF16}
MODELS = {"flow": MK_MODEL_FLOW, "multiphase": MK_MODEL_MULTIPHASE, "thermal_dendrite": MK_MODEL_THERMAL_DENDRITE,
          "solutal_dendrite": MK_MODEL_SOLUTAL_DENDRITE, "convection": MK_MODEL_CONVECTION,
          "flow_dendrite": MK_MODEL_FLOW_DENDRITE, "multigrain": MK_MODEL_MULTIGRAIN,
          "flow_solutal_dendrite": MK_MODEL_FLOW_SOLUTAL}
FIELDS = {"rho": MK_FIELD_RHO, "ux": MK_FIELD_UX, "uy": MK_FIELD_UY, "uz": MK_FIELD_UZ, "T": MK_FIELD_T,
          "C": MK_FIELD_C, "phi": MK_FIELD_PHI, "flag": MK_FIELD_FLAG, "pressure": MK_FIELD_PRESSURE,
          "dphi": MK_FIELD_DPHI, "grain": MK_FIELD_GRAIN}


class MkParams(C.Structure):
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
        ("obj_center", (C.c_double * 3) * MK_MAX_OBJECTS), ("obj_angle", (C.c_double * 3) * MK_MAX_OBJECTS),
        ("obj_radius", C.c_double * MK_MAX_OBJECTS), ("rng_seed", C.c_uint64),
        ("eps2", C.c_double),
        ("wall_axis", C.c_int32), ("inlet", C.c_int32), ("wall_value", C.c_double * 2),
        ("wall_u", (C.c_double * 3) * 2), ("beta", C.c_double), ("s_ref", C.c_double),
        ("grain_kappa", C.c_double), ("grain_u", C.c_double * 3),
    ]

    def ncell(self) -> int:
        return self.nx * self.ny * self.nz

    def to_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if isinstance(v, C.Array):
                v = [list(x) if isinstance(x, C.Array) else x for x in v]
            out[name] = v
        out["obj_center"] = out["obj_center"][: self.n_objects]
        out["obj_angle"] = out["obj_angle"][: self.n_objects]
        out["obj_radius"] = out["obj_radius"][: self.n_objects]
        return out


class MkOptions(C.Structure):
    _fields_ = [("model", C.c_int32), ("precision", C.c_int32), ("collision", C.c_int32), ("lattice", C.c_int32),
                ("magic", C.c_double), ("device", C.c_int32), ("block_x", C.c_int32), ("block_y", C.c_int32)]

    @classmethod
    def make(cls, model=-1, precision=-1, collision=-1, lattice=-1, magic=-1.0, device=-1, block_x=0, block_y=0):
        return cls(model, precision, collision, lattice, magic, device, block_x, block_y)


class MkTip(C.Structure):
    _fields_ = [("step", C.c_int64), ("length", C.c_double * 6), ("velocity", C.c_double * 6)]


class MkDiag(C.Structure):
    _fields_ = [("step", C.c_int64), ("mass", C.c_double), ("momentum", C.c_double * 3), ("phi_sum", C.c_double),
                ("solid_frac", C.c_double), ("heat", C.c_double), ("solute", C.c_double),
                ("max_speed", C.c_double), ("n_bad", C.c_int32), ("_pad", C.c_int32)]

    def to_dict(self) -> dict:
        return {"step": self.step, "mass": self.mass, "momentum": list(self.momentum), "phi_sum": self.phi_sum,
                "solid_frac": self.solid_frac, "heat": self.heat, "solute": self.solute,
                "max_speed": self.max_speed, "n_bad": self.n_bad}


class MkLoss(C.Structure):
    _fields_ = [("target_phi", C.POINTER(C.c_double)), ("steps", C.c_int64), ("checkpoint_every", C.c_int64)]


class MkGrad(C.Structure):
    _fields_ = [("loss", C.c_double), ("d_eps4", C.c_double), ("d_delta", C.c_double), ("d_tau_t", C.c_double),
                ("forward_loops", C.c_int64)]


class MkSlabXfer(C.Structure):
    _fields_ = [("peer", C.c_int32), ("send", C.c_int32), ("tag", C.c_int32), ("array", C.c_int32),
                ("offset", C.c_int64), ("count", C.c_int64), ("bytes", C.c_int64), ("ptr", C.c_void_p)]


class MkTuning(C.Structure):
    _fields_ = [("block_x", C.c_int32), ("block_y", C.c_int32), ("minb", C.c_int32), ("fused", C.c_int32),
                ("row_staged", C.c_int32), ("phi_tile", C.c_int32)]

    def to_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


MK_SLAB_FILL, MK_SLAB_PHI, MK_SLAB_RETURN, MK_SLAB_RUN_PHI, MK_SLAB_RUN_COLLIDE = range(5)
MK_SLAB_MAX_XFER = 40

H = C.c_void_p
P = C.POINTER

# name: (restype, argtypes)
PROTOTYPES = {
    "mk_abi_version": (C.c_int32, []),
    "mk_set_device": (C.c_int, [C.c_int32]),
    "mk_version_string": (C.c_char_p, []),
    "mk_last_global_error": (C.c_char_p, []),
    "mk_read_parameters": (C.c_int, [C.c_char_p, P(C.c_int32), P(C.c_int32)]),
    "mk_case_params": (C.c_int, [C.c_char_p, P(MkOptions), P(MkParams)]),
    "mk_case_initial_field": (C.c_int, [P(MkParams), C.c_int32, P(C.c_double), C.c_size_t]),
    "mk_create_from_xml": (C.c_int, [C.c_char_p, P(MkOptions), P(H)]),
    "mk_create": (C.c_int, [P(MkParams), P(H)]),
    "mk_destroy": (C.c_int, [H]),
    "mk_last_error": (C.c_char_p, [H]),
    "mk_get_params": (C.c_int, [H, P(MkParams)]),
    "mk_get_step": (C.c_int64, [H]),
    "mk_advance": (C.c_int, [H, C.c_int64]),
    "mk_advance_graph": (C.c_int, [H, C.c_int64]),
    "mk_sync": (C.c_int, [H]),
    "mk_inject_fault": (C.c_int, [H, C.c_int32]),
    "mk_set_fused": (C.c_int, [H, C.c_int32]),
    "mk_get_fused": (C.c_int32, [H]),
    "mk_set_row_staging": (C.c_int, [H, C.c_int32]),
    "mk_update_geometry": (C.c_int, [H, H]),
    "mk_update_velocity": (C.c_int, [H, H]),
    "mk_get_tuning": (C.c_int, [H, P(MkTuning)]),
    "mk_set_tuning": (C.c_int, [H, P(MkTuning)]),
    "mk_get_row_staging": (C.c_int32, [H]),
    "mk_get_stream": (C.c_int, [H, P(C.c_void_p)]),
    "mk_get_field": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t]),
    "mk_get_grain_field": (C.c_int, [H, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t]),
    "mk_set_state": (C.c_int, [H] + [P(C.c_double)] * 7),
    "mk_set_state_f32": (C.c_int, [H] + [P(C.c_float)] * 3),
    "mk_write_vtk": (C.c_int, [H, C.c_int64, C.c_char_p]),
    "mk_diagnostics": (C.c_int, [H, P(MkDiag)]),
    "mk_interface_points": (C.c_int, [H, C.c_double, P(C.c_double), P(C.c_double), C.c_int64, P(C.c_int64)]),
    "mk_tip_track": (C.c_int, [H, C.c_int32, C.c_double, P(MkTip)]),
    "mk_checkpoint": (C.c_int, [H, C.c_char_p]),
    "mk_restore": (C.c_int, [H, C.c_char_p]),
    "mk_profile_steps": (C.c_int, [H, C.c_int64, C.c_char_p, P(C.c_double), P(C.c_double), P(C.c_int64)]),
    "mk_time_advance": (C.c_int, [H, C.c_int64, C.c_int32, P(C.c_double)]),
    "mk_autotune": (C.c_int, [H, C.c_int32, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_double)]),
    "mk_host_alloc": (C.c_int, [C.c_size_t, P(C.c_void_p)]),
    "mk_host_free": (C.c_int, [C.c_void_p]),
    "mk_backward": (C.c_int, [H, P(MkLoss), P(MkGrad)]),
    "mk_nusselt": (C.c_int, [H, P(C.c_double)]),
    "mk_ensemble_case_params": (C.c_int, [C.c_uint64, C.c_int32, C.c_int32, P(MkParams)]),
    "mk_ensemble_create": (C.c_int, [P(MkParams), C.c_int32, P(H)]),
    "mk_ensemble_destroy": (C.c_int, [H]),
    "mk_ensemble_last_error": (C.c_char_p, [H]),
    "mk_ensemble_advance": (C.c_int, [H, C.c_int64]),
    "mk_ensemble_time_advance": (C.c_int, [H, C.c_int64, P(C.c_double)]),
    "mk_ensemble_get_field": (C.c_int, [H, C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_size_t]),
    "mk_ensemble_profile_steps": (C.c_int, [H, C.c_int64, C.c_char_p, P(C.c_double), P(C.c_double)]),
    "mk_ensemble_launches": (C.c_int64, [H]),
    "mk_ensemble_cells": (C.c_int64, [H]),
    "mk_ensemble_step": (C.c_int64, [H]),
    "mk_field_stats_noalloc": (C.c_int, [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]),
    "mk_noalloc_last_error": (C.c_char_p, []),
    "mk_set_metrics_log": (C.c_int, [C.c_char_p]),
    "mk_slab_split": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, P(C.c_int32), P(C.c_int32)]),
    "mk_slab_plan": (C.c_int, [P(MkParams), C.c_int32, C.c_int32, C.c_int32, P(MkSlabXfer), C.c_int32,
                               P(C.c_int32)]),
    "mk_create_slab": (C.c_int, [P(MkParams), C.c_int32, C.c_int32, P(H)]),
    "mk_slab_info": (C.c_int, [H, P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_int32), P(C.c_int32)]),
    "mk_slab_next": (C.c_int32, [H]),
    "mk_slab_transfers": (C.c_int, [H, C.c_int32, P(MkSlabXfer), C.c_int32, P(C.c_int32)]),
    "mk_slab_done": (C.c_int, [H, C.c_int32]),
    "mk_slab_run": (C.c_int, [H, C.c_int32]),
    "mk_slab_exchange_local": (C.c_int, [P(H), C.c_int32, C.c_int32]),
    "mk_bytes_per_cell": (C.c_double, [H]),
    "mk_fluid_cells": (C.c_int64, [H]),
    "mk_launches_per_step": (C.c_int32, [H]),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree libmkb200.so.  Raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libmkb200.so is not built ({LIB_PATH}); run __graft_entry__.build() or "
                          f"python -m materkit_anisotropiclbm_trt_rbc_facet_b200._build")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(PROTOTYPES)


class MkError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
