"""ctypes binding of ``libpystarc_b200.so`` (declared in include/pystarc_b200.h).

The library is built in-tree by ``pystarc_b200.build``.  There is no fallback:
if the shared object is missing or cannot be loaded, every entry point raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpystarc_b200.so"

BD_OK, BD_ERR_ARG, BD_ERR_CUDA, BD_ERR_OOM, BD_ERR_NAN, BD_ERR_STALL, BD_ERR_STATE = 0, -1, -2, -3, -4, -5, -6
GRID_ELEC, GRID_BORN, GRID_LIG_BORN = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
TORQUE_ZERO, TORQUE_CENTROID = 0, 1
CTR_NAMES = ("started", "reacted", "escaped", "max_steps", "steps", "returns", "overlap", "bridge", "grid_evals",
             "rev_evals", "ff_evals", "nonfinite")
N_CTR = len(CTR_NAMES)
LAYOUT_STAGE_RECEPTOR, LAYOUT_WINDOWS_1, LAYOUT_WINDOWS_2, LAYOUT_CUBES_1, LAYOUT_OVERLAP_GRID = 1, 2, 4, 8, 16
LAYOUT_XY_1, LAYOUT_ZTEX_1, LAYOUT_XYTEX_1, LAYOUT_PTEX_2 = 32, 64, 128, 256
LAYOUT_DEFAULT = LAYOUT_WINDOWS_1 | LAYOUT_CUBES_1 | LAYOUT_OVERLAP_GRID | LAYOUT_XY_1 | LAYOUT_ZTEX_1
TERM_GRID, TERM_FARFIELD, TERM_REV_BORN, TERM_CONTACT, TERM_ALL = 1, 2, 4, 8, 15

_ERR_NAMES = {BD_ERR_ARG: "bad argument", BD_ERR_CUDA: "CUDA error", BD_ERR_OOM: "out of device memory",
              BD_ERR_NAN: "non-finite value", BD_ERR_STALL: "device watchdog", BD_ERR_STATE: "call out of order"}


class BdForceParams(C.Structure):
    _fields_ = [("receptor_charge", C.c_double), ("debye_length", C.c_double), ("sdie", C.c_double),
                ("alpha", C.c_double), ("use_multipole", C.c_int), ("dipole", C.c_double * 3),
                ("quadrupole", C.c_double * 9), ("four_pi_eps", C.c_double)]


class BdSimParams(C.Structure):
    _fields_ = [("n_traj", C.c_int64), ("seed", C.c_uint64), ("r_start", C.c_double), ("r_escape", C.c_double),
                ("return_prob", C.c_double), ("max_steps", C.c_int32), ("max_dt", C.c_double),
                ("min_core_dt", C.c_double), ("use_hi", C.c_int32), ("overlap", C.c_int32), ("D_t", C.c_double),
                ("D_r", C.c_double), ("q_rec_total", C.c_double), ("q_lig_total", C.c_double),
                ("adt_debye", C.c_double), ("r_hydro_rec", C.c_double), ("r_hydro_lig", C.c_double),
                ("precision", C.c_int32), ("torque_mode", C.c_int32), ("slots", C.c_int32),
                ("id_offset", C.c_int64), ("stats", C.c_int32), ("min_core_rxn_dt", C.c_double),
                ("save_interval", C.c_int32), ("trace_capacity", C.c_int64), ("hi_mode", C.c_int32),
                ("hi_kT_eta", C.c_double)]


HI_REFERENCE_GPU, HI_ZUK = 0, 1


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)
_U = C.POINTER(C.c_uint64)


class BdStatsOut(C.Structure):
    _fields_ = [("start_pos", _D), ("start_q", _D), ("min_dist", _D), ("near_miss_pos", _D), ("near_miss_q", _D),
                ("total_time", _D), ("encounter_pos", _D), ("encounter_q", _D), ("step_at_min", _I),
                ("encounter_step", _I), ("bridge", C.POINTER(C.c_int8)), ("radial", _U), ("angular", _U),
                ("milestone_out", _U), ("milestone_in", _U), ("transition", _U), ("contact", _U),
                ("radial_edges", _D), ("transition_edges", _D), ("milestone_radii", _D)]


ST_RAD_BINS, ST_THETA, ST_PHI, ST_MILESTONES, ST_TRANS = 200, 36, 72, 11, 50


class BdSurrogateParams(C.Structure):
    _fields_ = [("r_scale", C.c_double), ("rbf_centre", C.c_double * 5), ("rbf_width", C.c_double),
                ("out_scale", C.c_double * 6), ("r_min", C.c_double), ("r_max", C.c_double),
                ("threshold", C.c_double), ("force_floor", C.c_double), ("env_r0", C.c_double),
                ("env_r1", C.c_double), ("env_log", C.c_double * 32), ("terms", C.c_int32),
                ("reserved", C.c_int32)]


class BdMlpDesc(C.Structure):
    _fields_ = [("n_members", C.c_int32), ("in_dim", C.c_int32), ("hidden", C.c_int32), ("n_hidden", C.c_int32),
                ("out_dim", C.c_int32), ("reserved", C.c_int32), ("seed", C.c_uint64)]


P = C.c_void_p
dp = C.POINTER(C.c_double)
fp = C.POINTER(C.c_float)
i32p = C.POINTER(C.c_int32)
i8p = C.POINTER(C.c_int8)
u64p = C.POINTER(C.c_uint64)

# name -> (restype, argtypes); mirrors include/pystarc_b200.h
SIGNATURES = {
    "bd_version": (C.c_char_p, []),
    "bd_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "bd_destroy": (C.c_int, [P]),
    "bd_last_error": (C.c_int, [P, C.c_char_p, C.c_int]),
    "bd_set_ligand": (C.c_int, [P, C.c_int, dp, dp]),
    "bd_set_receptor": (C.c_int, [P, C.c_int, dp, dp]),
    "bd_set_contact": (C.c_int, [P, C.c_int, dp, C.c_int, dp, C.c_double, C.c_double]),
    "bd_add_grid": (C.c_int, [P, C.c_int, fp, C.c_int, C.c_int, C.c_int, dp, dp]),
    "bd_clear_grids": (C.c_int, [P]),
    "bd_set_force_params": (C.c_int, [P, C.POINTER(BdForceParams)]),
    "bd_set_reactions": (C.c_int, [P, C.c_int, dp, dp, dp, dp, C.c_int]),
    "bd_eval_forces": (C.c_int, [P, C.c_int64, P, P, C.c_int, P, P, P, C.c_int, C.c_int, P]),
    "bd_eval_forces_atoms": (C.c_int, [P, C.c_int64, P, P, P, P, P, P, C.c_int, C.c_int, P]),
    "bd_eval_overlap": (C.c_int, [P, C.c_int64, P, P, P]),
    "bd_sim_configure": (C.c_int, [P, C.POINTER(BdSimParams)]),
    "bd_sim_reset": (C.c_int, [P, P]),
    "bd_sim_run": (C.c_int, [P, C.c_int, C.c_int, P]),
    "bd_sim_counters": (C.c_int, [P, u64p, C.c_int, P]),
    "bd_sim_outcomes": (C.c_int, [P, i8p, i32p, i32p]),
    "bd_sim_stats": (C.c_int, [P, C.POINTER(BdStatsOut)]),
    "bd_sim_live": (C.c_int, [P, i32p]),
    "bd_sim_hi_diffusion": (C.c_int, [P, C.c_int, dp, dp]),
    "bd_sim_traces": (C.c_int, [P, dp, dp, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "bd_sim_capacity": (C.c_int, [P, i32p]),
    "bd_set_reaction_states": (C.c_int, [P, C.c_int, i32p, i32p, C.c_int, C.POINTER(C.c_uint8)]),
    "bd_sim_reaction_fires": (C.c_int, [P, u64p, u64p, C.c_int]),
    "bd_sim_get_states": (C.c_int, [P, i8p]),
    "bd_sim_set_states": (C.c_int, [P, i8p]),
    "bd_sim_snapshot": (C.c_int, [P, dp, dp, i32p, i32p, i32p, i8p, i32p, u64p]),
    "bd_sim_restore": (C.c_int, [P, dp, dp, i32p, i32p, i32p, i8p, C.c_int32, u64p, i8p, i32p, i32p]),
    "bd_set_launch": (C.c_int, [P, C.c_int, C.c_int]),
    "bd_get_launch": (C.c_int, [P, i32p, i32p, i32p]),
    "bd_set_layout": (C.c_int, [P, C.c_int]),
    "bd_get_layout": (C.c_int, [P, i32p]),
    "bd_sim_run_noalloc": (C.c_int, [P, C.POINTER(BdSimParams), P, P, P, P, C.c_int, C.c_int, P]),
    "bd_set_terms": (C.c_int, [P, C.c_int]),
    "bd_sim_set_surrogate": (C.c_int, [P, P, C.POINTER(BdSurrogateParams)]),
    "bd_multi_create": (C.c_int, [C.POINTER(P), C.c_int, C.POINTER(P)]),
    "bd_multi_destroy": (C.c_int, [P]),
    "bd_multi_last_error": (C.c_int, [P, C.c_char_p, C.c_int]),
    "bd_multi_reset": (C.c_int, [P, P]),
    "bd_multi_run": (C.c_int, [P, C.c_int, C.c_int, P]),
    "bd_multi_counters": (C.c_int, [P, u64p, C.c_int, P]),
    "bd_multi_live": (C.c_int, [P, i32p]),
    "bd_sim_surrogate_counters": (C.c_int, [P, u64p]),
    "bd_mlp_create": (C.c_int, [C.c_int, C.POINTER(BdMlpDesc), C.POINTER(P)]),
    "bd_mlp_destroy": (C.c_int, [P]),
    "bd_mlp_last_error": (C.c_int, [P, C.c_char_p, C.c_int]),
    "bd_mlp_n_params": (C.c_int, [P, C.POINTER(C.c_int64)]),
    "bd_mlp_get_params": (C.c_int, [P, C.c_int, fp]),
    "bd_mlp_set_params": (C.c_int, [P, C.c_int, fp]),
    "bd_mlp_forward": (C.c_int, [P, C.c_int, C.c_int64, P, P, P]),
    "bd_mlp_grad": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P]),
    "bd_mlp_train_step": (C.c_int, [P, C.c_int, C.c_int, P, P, C.c_float, P, P]),
    "bd_mlp_ensemble": (C.c_int, [P, C.c_int64, P, P, P, P]),
    "bd_mlp_train": (C.c_int, [P, C.c_int, C.c_int64, P, P, C.c_int, C.c_int, C.c_float, C.c_uint64, P, P]),
    "bd_mlp_set_inference": (C.c_int, [P, C.c_int]),
    "bd_mlp_set_gemm": (C.c_int, [P, C.c_int]),
}

_LIB = None


class BdError(RuntimeError):
    """An engine entry point returned an error status."""

    def __init__(self, code, msg):
        super().__init__(f"{_ERR_NAMES.get(code, 'error')} ({code}): {msg}")
        self.code = code


def load(path: Path | None = None):
    """Load the shared library once and bind every declared entry point."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = Path(path or os.environ.get("PYSTARC_B200_LIB", LIB_PATH))
    if not p.exists():
        raise RuntimeError(f"{p} not found: build it with `python -c 'import pystarc_b200.build as b; b.build()'`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc, handle=None):
    if rc != BD_OK:
        buf = C.create_string_buffer(1024)
        load().bd_last_error(handle, buf, 1024)
        raise BdError(rc, buf.value.decode(errors="replace"))
    return rc


def check_multi(rc, m=None):
    if rc != BD_OK:
        buf = C.create_string_buffer(1024)
        load().bd_multi_last_error(m, buf, 1024)
        raise BdError(rc, buf.value.decode(errors="replace"))
    return rc


def check_mlp(rc, m=None):
    if rc != BD_OK:
        buf = C.create_string_buffer(1024)
        load().bd_mlp_last_error(m, buf, 1024)
        raise BdError(rc, buf.value.decode(errors="replace"))
    return rc


def ptr(a, ctype=C.c_double):
    """ctypes pointer to a contiguous NumPy array."""
    return a.ctypes.data_as(C.POINTER(ctype))
