"""Output steps in the reference's on-disk formats (bcg_write_output and the
asynchronous bcg_writer of the C ABI).

    w = Writer("run/out", threads=16)
    w.initial(col, t)                       # Simulation.cpp:185-244, step 0
    fcw = w.cells(col, k, t)                # before MoveCell; skip fcw rand() draws
    col.move_grow(dt) ...
    w.fields(col, k, t, dt)                 # after MoveCell, before the divisions
    w.lineage(pairs)
    w.close()                               # waits for the files

`write_output` writes one step from host arrays (no GPU): `step_data`
gathers them from a Colony through the synchronous download calls.
"""
import ctypes

import numpy as np

from . import _abi

OUT_CELLS = _abi.OUT_CELLS
OUT_FIELDS = _abi.OUT_FIELDS

# Array3D<LocalEnv>::Output's members, in file order (Array.h:931-1122)
ENV_MEMBERS = ("ENV_CARBON", "ENV_ACETATE", "ENV_WASTE", "ENV_OXYGEN", "ENV_GROWTH1", "ENV_GROWTH2",
               "ENV_GR_CAR_AER", "ENV_GR_CAR_ANA", "ENV_GR_ACE_AER", "ENV_PH", "ENV_HYDROX", "ENV_BUFFER",
               "ENV_ACETIC", "ENV_Q_CAR_MNT", "ENV_Q_ACE_MNT", "ENV_P_ACE_MNT", "ENV_Q_OXY_MNT")
# LocalAga's members in the AgarField / WallField order (Array.h:419-457, 1447-1494);
# FieldAgar's WasteAgar is never written by the MG path and stays 0
AGAR_MEMBERS = ("AGARF_CARBON", "AGARF_ACETATE", None, "AGARF_OXYGEN")
WALL_MEMBERS = ("WALLF_CARBON", "WALLF_ACETATE", "WALLF_WASTE", "WALLF_OXYGEN")


class StepData:
    """Host arrays of one output step, kept alive while a bcg_output_data
    points at them."""

    def __init__(self, p, t=0.0, dt=0.0, cells=None, force=None, force_stride=5, restart=None,
                 density=None, env=None, agar=None, wall=None):
        self.p, self.t, self.dt = p, t, dt
        self.cells = None if cells is None else np.ascontiguousarray(cells, dtype=_abi.CELL_DTYPE)
        self.force = None if force is None else np.ascontiguousarray(force, dtype=np.float64)
        self.force_stride = force_stride
        self.restart = None if restart is None else np.ascontiguousarray(restart, dtype=_abi.CELL_DTYPE)
        self.density = None if density is None else np.ascontiguousarray(density, dtype=np.float64)
        self.env = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (env or [None] * 17)]
        self.agar = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (agar or [])]
        self.wall = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (wall or [])]

    def struct(self):
        d = _abi.OutputData()
        d.t, d.dt = self.t, self.dt
        if self.cells is not None:
            d.n_cells = len(self.cells)
            d.force_stride = self.force_stride
            d.cells = self.cells.ctypes.data if len(self.cells) else None
            d.cell_force = self.force.ctypes.data if self.force is not None and self.force.size else None
        d.n_restart = -1 if self.restart is None else len(self.restart)
        d.restart_cells = self.restart.ctypes.data if self.restart is not None and len(self.restart) else None
        d.levels = self.p.max_levels_mg
        d.box_x, d.box_z, d.box_z_agar = self.p.box_x, self.p.box_z, self.p.box_z_agar
        d.density = None if self.density is None else self.density.ctypes.data
        for k, a in enumerate(self.env):
            d.env[k] = None if a is None else a.ctypes.data
        self._agar_ptrs = (_abi._VP * max(1, len(self.agar)))(*[None if a is None else a.ctypes.data for a in self.agar])
        self._wall_ptrs = (_abi._VP * max(1, len(self.wall)))(*[None if a is None else a.ctypes.data for a in self.wall])
        d.agar = ctypes.cast(self._agar_ptrs, _abi._VP)
        d.wall = ctypes.cast(self._wall_ptrs, _abi._VP)
        return d


def write_output(directory, output_id, what, data, append=False, threads=0):
    """bcg_write_output: one output step's files from host data (no GPU)."""
    lib = _abi.load()
    d = data.struct()
    _abi.check(lib.bcg_write_output(str(directory).encode(), output_id, what, 1 if append else 0,
                                    ctypes.byref(d), threads), "bcg_write_output")


def step_data(col, p, t, dt, stress=None, restart=None, initial_force=None):
    """StepData of a Colony read through the synchronous calls
    (bcg_download_cells, bcg_get_field); `stress` as bcg_mean_stress returns
    it, or `initial_force` (3 per cell) for the initial block."""
    levels = p.max_levels_mg
    cells = col.cells()
    force, stride = (stress, 5) if initial_force is None else (initial_force, 3)
    env = [col.field(m) for m in ENV_MEMBERS]
    agar, wall = [], []
    for l in range(levels):
        agar += [None if m is None else col.field(m, l) for m in AGAR_MEMBERS]
        wall += [col.field(m, l) for m in WALL_MEMBERS]
    return StepData(p, t, dt, cells=cells, force=force, force_stride=stride, restart=restart,
                    density=col.field("DENSITY_SHIFT"), env=env, agar=agar, wall=wall)


class Writer:
    """bcg_writer: output steps written by a host thread from device
    snapshots, while the GPU goes on."""

    def __init__(self, directory, append=False, threads=0, max_pending=2):
        self.lib = _abi.load()
        self.h = ctypes.c_void_p()
        _abi.check(self.lib.bcg_writer_create(str(directory).encode(), 1 if append else 0, threads, max_pending,
                                              ctypes.byref(self.h)), "bcg_writer_create")

    def initial(self, col, t):
        _abi.check(self.lib.bcg_output_initial(self.h, col.h, t), "bcg_output_initial")

    def cells(self, col, output_id, t):
        """Queue the cell lines; returns mean_stress's F_cw draw count."""
        f = ctypes.c_int64(0)
        _abi.check(self.lib.bcg_output_cells(self.h, col.h, output_id, t, ctypes.byref(f)), "bcg_output_cells")
        return f.value

    def fields(self, col, output_id, t, dt):
        _abi.check(self.lib.bcg_output_fields(self.h, col.h, output_id, t, dt), "bcg_output_fields")

    def lineage(self, pairs):
        a = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
        _abi.check(self.lib.bcg_writer_lineage(self.h, _abi.ptr(a, ctypes.c_int), len(a)), "bcg_writer_lineage")

    def wait(self):
        return self.lib.bcg_writer_wait(self.h)

    def close(self):
        rc = _abi.OK
        if self.h:
            rc = self.lib.bcg_writer_destroy(self.h)
            self.h = ctypes.c_void_p()
        return rc

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
