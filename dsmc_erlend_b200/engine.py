"""Python surface of the engine, mirroring the reference's stage functions.

    sim = Engine([params])                # Setup()       (Initialization.cpp:210)
    sim.InitialConditions()               # Initialization.cpp:290
    for _ in range(n):                    # the loop of Simulation.cpp:138-199
        sim.step()                        #   Move, Boundary, Index, Collide, Sample
    cells = sim.GatherGlobalField()       # MPIManager.cpp:305, 17 moments per cell
    sim.Printing("results")               # Sampling.cpp:36

The stage functions (MoveParticles, BoundaryConditions, Indexing,
CollideParticles, Sampling, end_step) run the same kernels as step(), one
stage at a time.  Every call goes through the C ABI of include/dsmc.h.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import abi
from ._lib import check, load
from .abi import Counters, Derived, Drag, Params

_D = C.POINTER(C.c_double)


def drag_report(p: Params, d: Derived, counters: dict) -> dict:
    """dsmc_drag_report over a counters dict (as Engine.counters returns)."""
    c = Counters(**counters)
    out = Drag()
    check(load().dsmc_drag_report(C.byref(p), C.byref(d), C.byref(c), C.byref(out)),
          "dsmc_drag_report")
    return out.as_dict()


def setup(p: Params) -> Derived:
    """Setup(): derived constants of one case (raises on invalid input)."""
    d = Derived()
    check(load().dsmc_setup(C.byref(p), C.byref(d)), "dsmc_setup")
    return d


def write_field(p: Params, d: Derived, sample_step: int, cells: np.ndarray, results_dir: str):
    """Printing(): DSMC2D_Field.plt/.json under results_dir/<wall>/."""
    cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 17)
    check(load().dsmc_write_field(C.byref(p), C.byref(d), int(sample_step),
                                  cells.ctypes.data_as(C.c_void_p), str(results_dir).encode()),
          "dsmc_write_field")


class Engine:
    """One device context holding one or more independent cases."""

    def __init__(self, cases: Params | Sequence[Params], derived: Sequence[Derived] | None = None,
                 stream: int | None = None):
        lib = load()
        if isinstance(cases, Params):
            cases = [cases]
        self.params = [p.copy() for p in cases]
        n = len(self.params)
        arr = (Params * n)(*self.params)
        darr = None
        if derived is not None:
            darr = (Derived * n)(*derived)
        h = C.c_void_p()
        check(lib.dsmc_ctx_create(arr, darr, n, C.c_void_p(stream) if stream else None,
                                  C.byref(h)), "dsmc_ctx_create")
        self._h = h
        self._lib = lib
        self.derived = list(derived) if derived is not None else [setup(p) for p in self.params]
        self.n_cases = n

    # -- lifecycle ------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.dsmc_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- the time loop --------------------------------------------------------
    def InitialConditions(self):
        check(self._lib.dsmc_init_cold(self._h), "dsmc_init_cold")

    init_cold = InitialConditions

    def init_warm(self, field: np.ndarray):
        """Fills every case from the local Maxwellian of `field`: (n, ux, uy,
        T) per cell, cells x-major, cases one after another (dsmc_init_warm),
        (n, ux, uy, Txx, Tyy, Tzz, Txy) (dsmc_init_warm_tensor), or the
        two-population (n, alpha, ux_r, uy_r, Txx_r, Tyy_r, Tzz_r, Txy_r)
        (dsmc_init_warm_mixture, fields.mixture_input)."""
        f = np.ascontiguousarray(field, dtype=np.float64)
        need = sum(p.nx * p.ny for p in self.params)
        if f.shape not in ((need, 4), (need, 7), (need, 8)):
            raise ValueError(f"field must have shape ({need}, 4), ({need}, 7) or ({need}, 8), "
                             f"not {f.shape}")
        if f.shape[1] == 7:  # n, ux, uy, Txx, Tyy, Tzz, Txy: dsmc_init_warm_tensor
            check(self._lib.dsmc_init_warm_tensor(self._h, f.ctypes.data_as(_D)),
                  "dsmc_init_warm_tensor")
        elif f.shape[1] == 8:  # n, alpha, u_r, T_r tensor: dsmc_init_warm_mixture
            check(self._lib.dsmc_init_warm_mixture(self._h, f.ctypes.data_as(_D)),
                  "dsmc_init_warm_mixture")
        else:
            check(self._lib.dsmc_init_warm(self._h, f.ctypes.data_as(_D)), "dsmc_init_warm")

    def step(self, n: int = 1):
        check(self._lib.dsmc_step(self._h, int(n)), "dsmc_step")

    def step_read(self, n: int, out_address: int):
        """n steps; after step k the counters of every case are copied
        asynchronously to the Counters array at out_address (n * n_cases
        records, case-minor); complete after synchronize().  Give it
        page-locked memory for the copies to overlap the steps."""
        check(self._lib.dsmc_step_read(self._h, int(n), C.c_void_p(out_address)),
              "dsmc_step_read")

    def MoveParticles(self):
        check(self._lib.dsmc_stage_move(self._h), "dsmc_stage_move")

    def BoundaryConditions(self):
        check(self._lib.dsmc_stage_boundary(self._h), "dsmc_stage_boundary")

    def Indexing(self):
        check(self._lib.dsmc_stage_index(self._h), "dsmc_stage_index")

    def CollideParticles(self) -> int:
        check(self._lib.dsmc_stage_collide(self._h), "dsmc_stage_collide")
        return sum(self.counters(i)["collisions_last_step"] for i in range(self.n_cases))

    def Sampling(self):
        check(self._lib.dsmc_stage_sample(self._h), "dsmc_stage_sample")

    def end_step(self):
        check(self._lib.dsmc_stage_end_step(self._h), "dsmc_stage_end_step")

    def synchronize(self):
        check(self._lib.dsmc_synchronize(self._h), "device")

    # -- state ----------------------------------------------------------------
    def counters(self, case: int = 0) -> dict:
        c = Counters()
        check(self._lib.dsmc_get_counters(self._h, case, C.byref(c)), "dsmc_get_counters")
        return c.as_dict()

    def GatherGlobalField(self, case: int = 0, out: np.ndarray | None = None) -> np.ndarray:
        """Moments of every cell, shape (nx*ny, 17), CELL layout, x-major.

        `out`, when given, receives them (float64, C-contiguous, that shape) and
        is returned: a buffer kept across calls avoids touching fresh pages,
        and a pinned one (page-locked, e.g. from torch's pin_memory) is copied
        into directly by the device."""
        p = self.params[case]
        shape = (p.nx * p.ny, 17)
        if out is None:
            out = np.empty(shape, dtype=np.float64)
        elif (out.shape != shape or out.dtype != np.float64
              or not out.flags["C_CONTIGUOUS"] or not out.flags["WRITEABLE"]):
            raise ValueError(f"out must be a writeable C-contiguous float64 array of shape {shape}")
        check(self._lib.dsmc_get_fields(self._h, case, out.ctypes.data_as(C.c_void_p)),
              "dsmc_get_fields")
        return out

    fields = GatherGlobalField

    def fields_to_device(self, case: int, device_ptr: int):
        check(self._lib.dsmc_get_fields_device(self._h, case, C.c_void_p(device_ptr)),
              "dsmc_get_fields_device")

    def fields_from_device(self, case: int, device_ptr: int, sample_step: int):
        check(self._lib.dsmc_set_fields_device(self._h, case, C.c_void_p(device_ptr),
                                               int(sample_step)), "dsmc_set_fields_device")

    def particles(self, case: int = 0) -> dict:
        n = C.c_int64()
        cap = int(self.counters(case)["np"]) + 16
        arrs = [np.empty(cap, dtype=np.float64) for _ in range(5)]
        check(self._lib.dsmc_download_particles(self._h, case, *[a.ctypes.data_as(_D)
                                                                 for a in arrs],
                                                cap, C.byref(n)), "dsmc_download_particles")
        return {k: a[: n.value].copy() for k, a in zip(("x", "y", "vx", "vy", "vz"), arrs)}

    def set_particles(self, st: dict, case: int = 0):
        arrs = [np.ascontiguousarray(st[k], dtype=np.float64) for k in ("x", "y", "vx", "vy", "vz")]
        check(self._lib.dsmc_upload_particles(self._h, case, *[a.ctypes.data_as(_D) for a in arrs],
                                              len(arrs[0])), "dsmc_upload_particles")

    def cell_starts(self, case: int = 0) -> np.ndarray:
        p = self.params[case]
        out = np.empty(p.nx * p.ny + 1, dtype=np.int32)
        check(self._lib.dsmc_get_cell_starts(self._h, case,
                                             out.ctypes.data_as(C.POINTER(C.c_int32))),
              "dsmc_get_cell_starts")
        return out

    def Printing(self, results_dir: str, case: int = 0):
        write_field(self.params[case], self.derived[case], self.counters(case)["sample_step"],
                    self.GatherGlobalField(case), results_dir)

    def drag_report(self, case: int = 0) -> dict:
        """Mean drag force and Cd (Simulation.cpp:210-237): over all steps as
        the reference's expression has it, and over the sampling window."""
        return drag_report(self.params[case], self.derived[case], self.counters(case))

    def checkpoint_save(self, path: str):
        """Counters, particles and moments of every case, between steps."""
        check(self._lib.dsmc_checkpoint_save(self._h, str(path).encode()),
              "dsmc_checkpoint_save")

    def checkpoint_load(self, path: str):
        """Resumes a checkpoint of a context with the same cases."""
        check(self._lib.dsmc_checkpoint_load(self._h, str(path).encode()),
              "dsmc_checkpoint_load")

    # -- launch shapes ----------------------------------------------------------
    def launch_config(self) -> dict:
        """{kernel: (CTAs per SM, maximum)} of the tunable step kernels."""
        cur = (C.c_int32 * 32)()
        mx = (C.c_int32 * 32)()
        names = (C.c_char_p * 32)()
        n = C.c_int()
        check(self._lib.dsmc_get_launch_config(self._h, cur, mx, 32, C.byref(n), names),
              "dsmc_get_launch_config")
        return {names[i].decode(): (cur[i], mx[i]) for i in range(n.value) if mx[i] > 0}

    def set_launch_config(self, shapes: dict):
        """Sets CTAs per SM by kernel name (others kept)."""
        order = list(self._all_kernel_names())
        arr = (C.c_int32 * len(order))(*[int(shapes.get(k, 0)) for k in order])
        check(self._lib.dsmc_set_launch_config(self._h, arr, len(order)),
              "dsmc_set_launch_config")

    def autotune(self, steps_per_trial: int = 3) -> dict:
        """Times the candidate shapes of each tunable kernel on real steps of
        this run (it advances) and keeps the fastest; returns the shapes."""
        check(self._lib.dsmc_autotune(self._h, int(steps_per_trial)), "dsmc_autotune")
        return self.launch_config()

    # -- step mode ------------------------------------------------------------
    def set_step_mode(self, persistent: bool, ctas_per_sm: int = 0):
        """dsmc_step as one graph launch per step (persistent=False, the
        default) or as ONE persistent cooperative kernel for all steps of a
        call (persistent=True; grid ctas_per_sm x SMs, 0 = the most that
        fit).  Results are identical."""
        check(self._lib.dsmc_set_step_mode(self._h, 1 if persistent else 0, int(ctas_per_sm)),
              "dsmc_set_step_mode")

    def step_mode(self) -> dict:
        """{"persistent", "ctas_per_sm", "max_ctas_per_sm", "graph_launch"}."""
        v = [C.c_int() for _ in range(4)]
        check(self._lib.dsmc_get_step_mode(self._h, *[C.byref(x) for x in v]),
              "dsmc_get_step_mode")
        return {"persistent": bool(v[0].value), "ctas_per_sm": v[1].value,
                "max_ctas_per_sm": v[2].value, "graph_launch": bool(v[3].value)}

    def phase_times(self, reset: bool = False) -> dict:
        """{phase: ms} of the persistent step, summed since the last reset."""
        ms = (C.c_double * 32)()
        names = (C.c_char_p * 32)()
        n = C.c_int()
        check(self._lib.dsmc_get_phase_times(self._h, ms, 32, C.byref(n), names,
                                             1 if reset else 0), "dsmc_get_phase_times")
        return {names[i].decode(): ms[i] for i in range(n.value)}

    def grid_sync_probe(self, wait_ns: int) -> int:
        """Status of a grid-barrier wait that can never complete, bounded by
        wait_ns (DSMC_ERR_TIMEOUT expected)."""
        return int(self._lib.dsmc_grid_sync_probe(self._h, int(wait_ns)))

    def _all_kernel_names(self):
        names = (C.c_char_p * 32)()
        n = C.c_int()
        check(self._lib.dsmc_get_launch_config(self._h, None, None, 32, C.byref(n), names),
              "dsmc_get_launch_config")
        return [names[i].decode() for i in range(n.value)]

    # -- profiling ------------------------------------------------------------
    def set_profiling(self, on: bool):
        check(self._lib.dsmc_set_profiling(self._h, 1 if on else 0), "dsmc_set_profiling")

    def kernel_times(self) -> dict:
        n = C.c_int()
        ms = (C.c_double * 32)()
        launches = (C.c_int64 * 32)()
        names = (C.c_char_p * 32)()
        check(self._lib.dsmc_get_kernel_times(self._h, ms, launches, 32, C.byref(n), names),
              "dsmc_get_kernel_times")
        return {names[i].decode(): (ms[i], launches[i]) for i in range(n.value)}


def default_params() -> Params:
    return abi.default_params()
