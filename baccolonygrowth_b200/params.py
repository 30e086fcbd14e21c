"""Parameters: defaults, the reference's key/value input format, and the
synthetic workload configurations.

`read_parameters` follows ReadParameters (AgentBasedModel-BacColonyGrowth/
InputOutput.cpp:450-677): one "key value" pair per line, values parsed with
atof/atoi semantics, unknown keys reported and ignored.
"""
import ctypes
import math
import re
import sys

from . import _abi

# input key -> (field, kind); kind "f" = atof, "i" = atoi, "b" = (bool)atoi,
# "if" = atof truncated to int (the reference assigns atof() to int globals)
INPUT_KEYS = {
    "Radius": ("cell_radius", "f"), "L_divide": ("l_divide", "f"), "k_cc": ("k_cc", "f"),
    "k_wc": ("k_wc", "f"), "var_L": ("var_l", "f"), "var_angle": ("var_angle", "f"),
    "var_pos": ("var_pos", "f"), "Viscosity": ("viscosity", "f"),
    "Growth_Rate1": ("max_growth_rate1", "f"), "Growth_Rate2": ("max_growth_rate2", "f"),
    "Wall_Rough": ("wall_rough", "f"), "Gamma": ("gamma_t", "f"), "Wall_Mu": ("wall_mu", "f"),
    "Cell_Mu": ("cell_mu", "f"), "Density_Threshold": ("density_threshold", "f"),
    "Surface_Tension": ("tension", "f"), "t_max": ("t_max", "f"), "dt": ("dt", "f"),
    "Box_x": ("box_x", "i"), "Box_y": ("box_y", "i"), "Box_z": ("box_z", "i"),
    "Box_z_agar": ("box_z_agar", "i"), "maxLevelsMG": ("max_levels_mg", "i"),
    "refinementGridHeight": ("refinement_grid_height", "i"), "Output_Time": ("output_time", "f"),
    "Update_Time": ("update_time", "f"), "KC_aer": ("kc_aer", "f"), "KC_ana": ("kc_ana", "f"),
    "KW": ("kw", "f"), "C_rate": ("c_rate", "f"), "W_rate": ("w_rate", "f"),
    "Diff_Colony": ("diff_colony", "f"), "Diff_Agar": ("diff_agar", "f"),
    "maxCarbon": ("max_carbon", "f"), "Carbon_to_Waste": ("carbon_to_waste", "f"),
    "Cdt": ("cdt", "f"), "InterfaceCondition": ("interface_condition", "if"),
    "NutrientGSI": ("nutrient_gsi", "b"), "Rc": ("rc", "f"), "CrossFeeding": ("cross_feeding", "b"),
    "Delta_H": ("delta_h", "f"), "MaintenanceRate": ("maintenance_rate", "f"),
    "FilterLen": ("filter_len", "i"), "MaxCells": ("max_cells", "i"), "KO": ("ko", "f"),
    "KA": ("ka", "f"), "KI": ("ki", "f"), "Q_Carbon_Aerobic": ("q_car_aer", "f"),
    "Q_Carbon_Anaerobic": ("q_car_ana", "f"), "Q_Acetate_Aerobic": ("q_ace_aer", "f"),
    "Q_Oxygen_Carbon": ("q_o2_car", "f"), "Q_Oxygen_Acetate": ("q_o2_ace", "f"),
    "P_Acetate_Aerobic": ("p_ace_aer", "f"), "P_Acetate_Anaerobic": ("p_ace_ana", "f"),
    "Diff_Colony_Carbon": ("diff_colony_carbon", "f"), "Diff_Agar_Carbon": ("diff_agar_carbon", "f"),
    "Diff_Colony_Oxygen": ("diff_colony_o2", "f"), "Diff_Agar_Oxygen": ("diff_agar_o2", "f"),
    "Diff_Colony_Acetate": ("diff_colony_ace", "f"), "Diff_Agar_Acetate": ("diff_agar_ace", "f"),
    "Max_Oxygen": ("max_o2", "f"),
    "Max_Growth_Rate_Carbon_Aerobic": ("max_gr_car_aer", "f"),
    "Max_Growth_Rate_Carbon_Anaerobic": ("max_gr_car_ana", "f"),
    "Max_Growth_Rate_Acetate_Aerobic": ("max_gr_ace_aer", "f"),
    "Kw": ("kw_ph", "f"), "Ka": ("ka_ph", "f"), "Kb": ("kb_ph", "f"), "Cb": ("cb_ph", "f"),
    "c1": ("c1_ph", "f"),
    "qCarAernt": ("q_car_aer_nt", "f"), "qCarAnant": ("q_car_ana_nt", "f"),
    "qAceAernt": ("q_ace_aer_nt", "f"), "qO2Carnt": ("q_o2_car_nt", "f"),
    "qO2Acent": ("q_o2_ace_nt", "f"), "pAceAnant": ("p_ace_ana_nt", "f"),
}
# keys the reference reads into state the hot path does not use
IGNORED_KEYS = {"Tortuosity", "ConvCrit", "minIter", "maxIter", "IniColonyRadius", "IniColonySize",
                "NumColonies", "ColonySeparation", "Restart", "Restart_dir", "RestartIndex",
                "qEthaAnant", "qForAnant", "Box_Dim"}

_FLOAT_PREFIX = re.compile(r"^\s*[+-]?((\d+\.?\d*)|(\.\d+))([eE][+-]?\d+)?")
_INT_PREFIX = re.compile(r"^\s*[+-]?\d+")


def atof(s):
    m = _FLOAT_PREFIX.match(s)
    return float(m.group(0)) if m else 0.0


def atoi(s):
    m = _INT_PREFIX.match(s)
    return int(m.group(0)) if m else 0


# The two C entries behind defaults() and finalize(): the library's
# bcg_params_default / bcg_params_finalize unless a caller passes another
# pair with the same signatures (the benchmark's reference arm passes the
# oracle's, so that it never loads the CUDA library).
def _param_entries(entries):
    if entries is not None:
        return entries
    lib = _abi.load()
    return lib.bcg_params_default, lib.bcg_params_finalize


def defaults(entries=None):
    """Reference defaults (Constants.cpp:1-112) from the library."""
    p = _abi.Params()
    _abi.check(_param_entries(entries)[0](ctypes.byref(p)), "bcg_params_default")
    return p


def finalize(p, entries=None):
    _abi.check(_param_entries(entries)[1](ctypes.byref(p)), "bcg_params_finalize")
    return p


def parse_parameters(text, p=None, warn=True, entries=None):
    """Apply "key value" lines to params p (defaults if None)."""
    if p is None:
        p = defaults(entries)
    for line in re.split(r"[\r\n]", text):
        parts = line.split()
        if not parts:
            continue
        key = parts[0]
        val = parts[1] if len(parts) > 1 else ""
        if key in INPUT_KEYS:
            field, kind = INPUT_KEYS[key]
            if kind == "f":
                setattr(p, field, atof(val))
            elif kind == "i":
                setattr(p, field, atoi(val))
            elif kind == "if":
                setattr(p, field, int(atof(val)))
            else:
                setattr(p, field, 1 if atoi(val) != 0 else 0)
        elif key == "Box_Dim":
            p.box_x = atoi(val)
            p.box_y = p.box_x
        elif key in IGNORED_KEYS:
            continue
        elif warn:
            print("Unknown parameter: %s " % key, file=sys.stderr)
    return p


def read_parameters(path, p=None):
    with open(path) as f:
        return parse_parameters(f.read(), p)


# --------------------------------------------------------------------------
# Workloads.  The reference is a 2-D x-z model (Box_y = 1).  Each workload
# restates one of the benchmark configurations in that geometry: cells of
# radius 0.5 um, lengths U(2, 4) um, in a half-ellipse dome of the named
# aspect ratio, sized so the cells' area fraction is `phi`.
# --------------------------------------------------------------------------
WORKLOADS = {
    # name: (cells, dome aspect height/width, box_x, box_z, box_z_agar, agar levels)
    "small_4k": (4096, 6.0 / 40.0, 256, 50, 32, 2),
    "scale_262k": (262144, 15.0 / 300.0, 2304, 128, 512, 3),
    "mixed_1m": (1048576, 25.0 / 600.0, 4608, 200, 1024, 3),
}


def shipped_input_text(which="small"):
    """The reference's shipped input file (run_sim/inputFile_20mM_{Small,Large}
    Simulation.txt) as key/value text (data/, regenerated by
    data/make_inputs.py)."""
    import os
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "%s_input.txt" % which)
    with open(path) as f:
        return f.read()


def workload_params(name, max_cells=None, entries=None):
    """Params of a named workload: the reference's small-simulation physics
    with the workload's grid."""
    cells, aspect, bx, bz, bza, lev = WORKLOADS[name]
    p = parse_parameters(shipped_input_text("small"), entries=entries)
    p.box_x, p.box_y, p.box_z, p.box_z_agar, p.max_levels_mg = bx, 1, bz, bza, lev
    p.max_cells = max_cells if max_cells else int(cells * 1.25) + 1024
    return finalize(p, entries)


def dome_size(n_cells, aspect, phi=0.45, radius=0.5, mean_len=3.0):
    """Half-ellipse width/height (um) holding n cells at area fraction phi."""
    area = n_cells * (2 * radius) * (mean_len + 2 * radius) / phi
    w = math.sqrt(area / (math.pi / 4.0 * aspect))
    return w, w * aspect


def ensemble_member(n_cells, aspect=1.0 / 20.0, phi=0.45, max_cells=None):
    """Params for one colony of an ensemble: the small-simulation physics on
    a grid sized to the colony's dome (room for the dome, the filter margins
    and growth; 2 composite agar levels of 64 rows)."""
    w, h = dome_size(n_cells, aspect, phi)
    p = finalize(parse_parameters(shipped_input_text("small")))
    bl = p.box_length
    p.box_x = max(128, int(math.ceil((w / bl + 24) / 32.0)) * 32)
    p.box_y = 1
    p.box_z = max(16, int(math.ceil(h / bl)) + 12)
    p.box_z_agar, p.max_levels_mg = 64, 2
    p.max_cells = max_cells if max_cells else int(n_cells * 1.25) + 1024
    return finalize(p)

