"""ctypes binding of the C ABI declared in include/bcg.h.

Only plain pointers, sizes and POD structs cross the boundary; the
structures below mirror the header byte for byte (tests check the layout
against the header).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libbcg.so")

# ---- status codes (bcg_status) -------------------------------------------
OK = 0
E_ARG = 1
E_CUDA = 2
E_BOX_OVERFLOW = 3
E_NEIGH_OVERFLOW = 4
E_OUT_OF_GRID = 5
E_NAN = 6
E_MAXCELLS = 7
E_TIMEOUT = 8
E_UNSUPPORTED = 9
E_NEED_MORE_BOXES = 10
E_NO_DEVICE = 11
E_IO = 12

# ---- field ids (bcg_field_id) --------------------------------------------
FIELDS = dict(
    HEIGHT=0, NORMAL_X=1, NORMAL_Z=2, WALL=3, DENSITY_SHIFT=4, WALL_DENSITY_SHIFT=5, INSIDE=6,
    ENV_CARBON=7, ENV_WASTE=8, ENV_OXYGEN=9, ENV_ACETATE=10, ENV_GROWTH1=11, ENV_GROWTH2=12, ENV_PH=13,
    OLDENV_CARBON=14, OLDENV_WASTE=15, OLDENV_OXYGEN=16, OLDENV_ACETATE=17,
    WALLF_CARBON=18, WALLF_WASTE=19, WALLF_OXYGEN=20, WALLF_ACETATE=21,
    OLDWALLF_CARBON=22, OLDWALLF_WASTE=23, OLDWALLF_OXYGEN=24, OLDWALLF_ACETATE=25,
    AGARF_CARBON=26, AGARF_OXYGEN=27, AGARF_ACETATE=28,
    MG_SOL_CARBON=29, MG_SOL_OXYGEN=30, MG_SOL_ACETATE=31,
    MG_RES_CARBON=32, MG_RES_OXYGEN=33, MG_RES_ACETATE=34,
    MG_ERR_CARBON=35, MG_ERR_OXYGEN=36, MG_ERR_ACETATE=37,
    DENSITY=38, ROUGH_DENSITY=39,
    ENV_HYDROX=40, ENV_ACETIC=41, ENV_BUFFER=42, ENV_GR_CAR_AER=43, ENV_GR_CAR_ANA=44, ENV_GR_ACE_AER=45,
    ENV_Q_CAR_MNT=46, ENV_Q_ACE_MNT=47, ENV_P_ACE_MNT=48, ENV_Q_OXY_MNT=49)

TIMERS = dict(MOVE_GROW=0, DIVIDE=1, NEIGHBOURS=2, MG_SOLVE=3, SWEEPS=4, DENSITY=5)

# ---- bcg_cell: byte-identical to the reference's struct Cell (208 B) ------
_V3 = ("f8", (3,))
CELL_DTYPE = np.dtype([
    ("p", _V3), ("q", _V3), ("time_p", "f8"), ("time_q", "f8"), ("age_p", "i4"), ("age_q", "i4"),
    ("length", "f8"), ("ldiv", "f8"), ("radius", "f8"), ("growth_rate", "f8"),
    ("velocity", _V3), ("angular_velocity", _V3), ("dyn_fric", _V3), ("sta_fric", _V3),
    ("type", "i4"), ("ancestor", "i4")])
assert CELL_DTYPE.itemsize == 208


class Params(ctypes.Structure):
    """Mirror of struct bcg_params."""
    _fields_ = [
        ("box_x", ctypes.c_int32),
        ("box_y", ctypes.c_int32),
        ("box_z", ctypes.c_int32),
        ("box_z_agar", ctypes.c_int32),
        ("max_levels_mg", ctypes.c_int32),
        ("filter_len", ctypes.c_int32),
        ("refinement_grid_height", ctypes.c_int32),
        ("max_cells", ctypes.c_int32),
        ("max_cells_per_box", ctypes.c_int32),
        ("max_neighbours", ctypes.c_int32),
        ("box_length", ctypes.c_double),
        ("cell_radius", ctypes.c_double),
        ("l_divide", ctypes.c_double),
        ("k_cc", ctypes.c_double),
        ("k_wc", ctypes.c_double),
        ("var_l", ctypes.c_double),
        ("var_angle", ctypes.c_double),
        ("var_pos", ctypes.c_double),
        ("viscosity", ctypes.c_double),
        ("wall_rough", ctypes.c_double),
        ("gamma_t", ctypes.c_double),
        ("cell_mu", ctypes.c_double),
        ("wall_mu", ctypes.c_double),
        ("density_threshold", ctypes.c_double),
        ("tension", ctypes.c_double),
        ("delta_h", ctypes.c_double),
        ("rc", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("t0", ctypes.c_double),
        ("t_max", ctypes.c_double),
        ("output_time", ctypes.c_double),
        ("update_time", ctypes.c_double),
        ("kc_aer", ctypes.c_double),
        ("kc_ana", ctypes.c_double),
        ("kw", ctypes.c_double),
        ("ko", ctypes.c_double),
        ("ka", ctypes.c_double),
        ("ki", ctypes.c_double),
        ("carbon_to_waste", ctypes.c_double),
        ("c_rate", ctypes.c_double),
        ("w_rate", ctypes.c_double),
        ("maintenance_rate", ctypes.c_double),
        ("q_car_aer", ctypes.c_double),
        ("q_car_ana", ctypes.c_double),
        ("q_ace_aer", ctypes.c_double),
        ("q_o2_car", ctypes.c_double),
        ("q_o2_ace", ctypes.c_double),
        ("p_ace_aer", ctypes.c_double),
        ("p_ace_ana", ctypes.c_double),
        ("diff_colony", ctypes.c_double),
        ("diff_agar", ctypes.c_double),
        ("diff_colony_carbon", ctypes.c_double),
        ("diff_agar_carbon", ctypes.c_double),
        ("diff_colony_o2", ctypes.c_double),
        ("diff_agar_o2", ctypes.c_double),
        ("diff_colony_ace", ctypes.c_double),
        ("diff_agar_ace", ctypes.c_double),
        ("max_carbon", ctypes.c_double),
        ("max_o2", ctypes.c_double),
        ("max_o2_agar", ctypes.c_double),
        ("max_growth_rate1", ctypes.c_double),
        ("max_growth_rate2", ctypes.c_double),
        ("max_gr_car_aer", ctypes.c_double),
        ("max_gr_car_ana", ctypes.c_double),
        ("max_gr_ace_aer", ctypes.c_double),
        ("cdt", ctypes.c_double),
        ("q_car_aer_nt", ctypes.c_double),
        ("q_car_ana_nt", ctypes.c_double),
        ("q_ace_aer_nt", ctypes.c_double),
        ("q_o2_car_nt", ctypes.c_double),
        ("q_o2_ace_nt", ctypes.c_double),
        ("p_ace_ana_nt", ctypes.c_double),
        ("kw_ph", ctypes.c_double),
        ("ka_ph", ctypes.c_double),
        ("kb_ph", ctypes.c_double),
        ("cb_ph", ctypes.c_double),
        ("c1_ph", ctypes.c_double),
        ("cross_feeding", ctypes.c_int32),
        ("interface_condition", ctypes.c_int32),
        ("nutrient_gsi", ctypes.c_int32),
        ("mg_levels", ctypes.c_int32),
        ("mg_vcycles", ctypes.c_int32),
        ("mg_mu1", ctypes.c_int32),
        ("mg_mu2", ctypes.c_int32),
        ("sweeps_per_solve", ctypes.c_int32),
        ("solves_per_update", ctypes.c_int32),
        ("mg_dt", ctypes.c_double),
    ]

    def copy(self):
        p = Params()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(Params))
        return p

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Rng(ctypes.Structure):
    """Mirror of struct bcg_rng (glibc rand() state)."""
    _fields_ = [("r", ctypes.c_uint32 * 34), ("pos", ctypes.c_int32)]


_VP = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_PI = ctypes.POINTER(ctypes.c_int)
_PD = ctypes.POINTER(ctypes.c_double)
_PF = ctypes.POINTER(ctypes.c_float)
_PI64 = ctypes.POINTER(ctypes.c_int64)
_SZ = ctypes.c_size_t

# name: (restype, argtypes) -- every function declared in include/bcg.h
PROTOTYPES = {
    "bcg_params_default": (_I, [ctypes.POINTER(Params)]),
    "bcg_params_finalize": (_I, [ctypes.POINTER(Params)]),
    "bcg_create": (_I, [ctypes.POINTER(Params), ctypes.POINTER(_VP)]),
    "bcg_destroy": (_I, [_VP]),
    "bcg_status_string": (ctypes.c_char_p, [_I]),
    "bcg_stream": (_VP, [_VP]),
    "bcg_synchronize": (_I, [_VP]),
    "bcg_upload_cells": (_I, [_VP, _VP, _I]),
    "bcg_download_cells": (_I, [_VP, _VP, _I, _PI]),
    "bcg_num_cells": (_I, [_VP, _PI]),
    "bcg_rebuild_neighbours": (_I, [_VP]),
    "bcg_get_neighbours": (_I, [_VP, _PI, _PI, _I]),
    "bcg_set_neighbours": (_I, [_VP, _PI, _PI, _I]),
    "bcg_move_grow": (_I, [_VP, _D, _PI, _PI64]),
    "bcg_get_dividing": (_I, [_VP, _PI, _I]),
    "bcg_divide": (_I, [_VP, _PF, _I, _D, _PI, _PI]),
    "bcg_field_size": (_I, [_VP, _I, _I, ctypes.POINTER(_SZ)]),
    "bcg_get_field": (_I, [_VP, _I, _I, _PD, _SZ]),
    "bcg_set_field": (_I, [_VP, _I, _I, _PD, _SZ]),
    "bcg_get_bbox": (_I, [_VP, _PI, _PI, _PI]),
    "bcg_update_density": (_I, [_VP]),
    "bcg_update_height": (_I, [_VP]),
    "bcg_initial_density": (_I, [_VP]),
    "bcg_nutrient_update": (_I, [_VP, _I, _I]),
    "bcg_mg_solve": (_I, [_VP, _I]),
    "bcg_colony_sweeps": (_I, [_VP, _I, _I]),
    "bcg_mg_solve_tol": (_I, [_VP, _D, _I, _I, _PI, _PD]),
    "bcg_autotune": (_I, [_VP, _I, _PI]),
    "bcg_set_pair_precision": (_I, [_VP, _I]),
    "bcg_ensemble_create": (_I, [_VP, _I, _VP]),
    "bcg_ensemble_run": (_I, [_VP, _I]),
    "bcg_ensemble_destroy": (_I, [_VP]),
    "bcg_steady_create": (_I, [_VP, _VP]),
    "bcg_steady_destroy": (_I, [_VP]),
    "bcg_steady_set_cells": (_I, [_VP, _PD, _I]),
    "bcg_steady_solve": (_I, [_VP, _PD, _PD, _D, _PD, _PI, _PI]),
    "bcg_steady_vjp": (_I, [_VP, _PD, _PD, _PD, _D]),
    "bcg_enable_timers": (_I, [_VP, _I]),
    "bcg_get_timer": (_I, [_VP, _I, _PD, _PI64]),
    "bcg_timeline_enable": (_I, [_VP, _I]),
    "bcg_timeline_read": (_I, [_VP, _PI, _PF, _I, _PI]),
    "bcg_rng_seed": (None, [ctypes.POINTER(Rng), ctypes.c_uint32]),
    "bcg_rng_next": (ctypes.c_int32, [ctypes.POINTER(Rng)]),
    "bcg_rng_skip": (None, [ctypes.POINTER(Rng), ctypes.c_int64]),
    "bcg_synth_colony": (_I, [ctypes.c_uint64, _I, _D, _D, _D, _D, _D, _D, _D, _VP, _I, _PI]),
    "bcg_sim_create": (_I, [ctypes.POINTER(Params), _VP, _I, ctypes.c_uint32, _I, ctypes.POINTER(_VP)]),
    "bcg_sim_destroy": (_I, [_VP]),
    "bcg_sim_run": (_I, [_VP, _I]),
    "bcg_sim_ctx": (_VP, [_VP]),
    "bcg_sim_time": (_I, [_VP, _PD, _PI, _PI64]),
    "bcg_sim_counters": (_I, [_VP, _PI64, _PI64]),
    "bcg_legacy_env_update": (_I, [_VP, _I, _I, _D, _PI]),
    "bcg_legacy_agar_depletion": (_I, [_VP, _PI]),
    "bcg_set_force_group": (_I, [_VP, _I]),
    "bcg_set_relax_mode": (_I, [_VP, _I]),
    "bcg_set_smoother_warps": (_I, [_VP, _I]),
    "bcg_smoother_launch_ms": (_I, [_VP, _PD]),
    "bcg_sim_lineage": (_I, [_VP, _PI, _I, _PI]),
    "bcg_sim_set_step_mode": (_I, [_VP, _I, _I]),
    "bcg_save_restart": (_I, [ctypes.c_char_p, _D, _D, _VP, _I]),
    "bcg_load_restart": (_I, [ctypes.c_char_p, _PD, _PD, _VP, _I, _PI]),
    "bcg_mean_stress": (_I, [_VP, _PD, _PD, _PI64]),
    "bcg_mean_stress_noalloc": (_I, [_VP, _PD, _PD, _PI64]),
    "bcg_write_output": (_I, [ctypes.c_char_p, _I, _I, _I, _VP, _I]),
    "bcg_writer_create": (_I, [ctypes.c_char_p, _I, _I, _I, ctypes.POINTER(_VP)]),
    "bcg_writer_wait": (_I, [_VP]),
    "bcg_writer_destroy": (_I, [_VP]),
    "bcg_output_initial": (_I, [_VP, _VP, _D]),
    "bcg_output_cells": (_I, [_VP, _VP, _I, _D, _PI64]),
    "bcg_output_fields": (_I, [_VP, _VP, _I, _D, _D]),
    "bcg_writer_lineage": (_I, [_VP, _PI, _I]),
    "bcg_sim_set_writer": (_I, [_VP, _VP, _I]),
}

OUT_CELLS = 1     # BCG_OUT_CELLS
OUT_FIELDS = 2    # BCG_OUT_FIELDS


class OutputData(ctypes.Structure):
    """Mirror of struct bcg_output_data."""
    _fields_ = [
        ("t", ctypes.c_double), ("dt", ctypes.c_double),
        ("n_cells", ctypes.c_int32), ("force_stride", ctypes.c_int32),
        ("cells", _VP), ("cell_force", _VP),
        ("n_restart", ctypes.c_int32), ("levels", ctypes.c_int32),
        ("restart_cells", _VP),
        ("box_x", ctypes.c_int32), ("box_z", ctypes.c_int32), ("box_z_agar", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("density", _VP), ("env", _VP * 17),
        ("agar", _VP), ("wall", _VP),
    ]

# library entry points outside include/bcg.h, used by tests and the benchmark
EXTRA_PROTOTYPES = {
    "bcg_kernel_launches": (ctypes.c_longlong, [_VP]),
    "bcg_set_bbox": (_I, [_VP, _I, _I, _I]),
}

TUNE = dict(FORCE_GROUP=1, SMOOTHER=2)
NOALLOC_MAX_CELLS = 32768   # BCG_NOALLOC_MAX_CELLS

_lib = None


class BcgError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = status_string(code)
        text = "{} failed: {} (status {})".format(what, msg, code) if what else "{} (status {})".format(msg, code)
        super().__init__(text)


def load(path=None):
    """Load libbcg.so (built by baccolonygrowth_b200.build).  Raises if it is
    absent: there is no fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libbcg.so is not built ({}); run baccolonygrowth_b200.build.build()".format(p))
    lib = ctypes.CDLL(p)
    for name, (res, args) in list(PROTOTYPES.items()) + list(EXTRA_PROTOTYPES.items()):
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def status_string(code):
    try:
        return load().bcg_status_string(code).decode()
    except Exception:  # library missing
        return "status {}".format(code)


def check(code, what=""):
    if code != OK:
        raise BcgError(code, what)
    return code


def ptr(a, ctype=None):
    """ctypes pointer to the data of a contiguous numpy array."""
    if ctype is None:
        return ctypes.c_void_p(a.ctypes.data)
    return a.ctypes.data_as(ctypes.POINTER(ctype))
