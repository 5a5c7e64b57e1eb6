"""ctypes mirror of include/dsmc.h: parameter, derived-constant, counter and
cell structures, status codes, and the reference defaults.

The defaults are the reference's compile-time settings
(src/Initialization.cpp:11-31, src/Geometry.cpp:11-24, src/Boundary.cpp:11-13).
"""
from __future__ import annotations

import ctypes as C

OK = 0
ERR_ARGUMENT = 2
ERR_OUT_OF_DOMAIN = 20
ERR_CELL_OVERFLOW = 22
ERR_EXCHANGE = 30
ERR_CAPACITY = 31
ERR_BAD_CLL = 40
ERR_CUDA = 50
ERR_NO_DEVICE = 51
ERR_TIMEOUT = 60
ERR_STATE = 61
ERR_UNSUPPORTED = 62

# WallModel enumerator order of include/Boundary.h:3.
WALL_DIFFUSE = 0
WALL_SPECULAR = 1
WALL_CLL = 2
WALL_NAMES = {WALL_DIFFUSE: "diffuse", WALL_SPECULAR: "specular", WALL_CLL: "cll"}

FP64 = 0
FP32 = 1

# Philox stream kinds (include/dsmc_philox.h).
RNG_INIT = 1
RNG_INJECT = 2
RNG_MOVE = 3
RNG_COLLIDE = 4
RNG_USER = 5
RNG_WARM = 6

# Layout of one cell's 17 moments (include/Cell.h:4-10).
CELL_NP = 0
CELL_V = slice(1, 4)
CELL_VV = slice(4, 13)
CELL_V2V = slice(13, 16)
CELL_NC = 16


class Params(C.Structure):
    _fields_ = [
        ("x1", C.c_double), ("x2", C.c_double), ("y1", C.c_double), ("y2", C.c_double),
        ("dz", C.c_double), ("dl", C.c_double),
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("box_x", C.c_double), ("box_y", C.c_double),
        ("box_width", C.c_double), ("box_height", C.c_double),
        ("dt", C.c_double),
        ("n_step", C.c_int32), ("first_sampling_step", C.c_int32),
        ("sampling_period", C.c_int32), ("wall_model", C.c_int32),
        ("npc_free", C.c_double), ("molar_mass", C.c_double), ("ma_free", C.c_double),
        ("n_free", C.c_double), ("t_free", C.c_double), ("attack_angle", C.c_double),
        ("t_wall", C.c_double), ("d_ref", C.c_double), ("viscosity_index", C.c_double),
        ("t_ref", C.c_double), ("cll_normal", C.c_double), ("cll_tangential", C.c_double),
        ("seed", C.c_uint64),
        ("precision", C.c_int32), ("reserved1", C.c_int32),
        ("max_particles_in_cell", C.c_int32), ("reserved0", C.c_int32),
        ("capacity", C.c_int64),
    ]

    def copy(self, **overrides) -> "Params":
        p = Params()
        C.pointer(p)[0] = self
        for k, v in overrides.items():
            setattr(p, k, v)
        return p

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Drag(C.Structure):
    """dsmc_drag of include/dsmc.h: the drag block of RunSimulation."""
    _fields_ = [
        ("sampling_time", C.c_double), ("rho_free", C.c_double), ("area_ref", C.c_double),
        ("mean_force_total", C.c_double), ("cd_total", C.c_double),
        ("box_collisions", C.c_int64), ("mean_force", C.c_double), ("cd", C.c_double),
        ("box_collisions_window", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Derived(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "molecule_mass", "p_free", "u_free", "ux_free", "uy_free", "dx", "dy", "dv",
        "weight", "sigma_ref", "omega", "cr_ref", "mft_free", "mfp_free", "kn_free",
        "sc_max")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Counters(C.Structure):
    _fields_ = [
        ("np", C.c_int64), ("step", C.c_int64), ("sample_step", C.c_int64),
        ("collisions_last_step", C.c_int64), ("collisions_total", C.c_int64),
        ("drag_collision_count", C.c_int64), ("particle_steps", C.c_int64),
        ("drag_impulse_total", C.c_double), ("time", C.c_double),
        ("sample_time", C.c_double), ("drag_sampling_time", C.c_double),
        ("drag_collision_count_window", C.c_int64), ("drag_impulse_window", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def default_params() -> Params:
    """The reference's settings: 100x100 grid on [-20,20]^2, 4x4 m box,
    argon-like VHS gas at Ma 4, CLL (0.8, 0.8) walls."""
    p = Params()
    p.x1, p.x2, p.y1, p.y2 = -20.0, 20.0, -20.0, 20.0
    p.dz, p.dl = 0.1, 0.1
    p.nx, p.ny = 100, 100
    p.box_x, p.box_y, p.box_width, p.box_height = 0.0, 0.0, 4.0, 4.0
    p.dt = 1.0e-5
    p.n_step, p.first_sampling_step, p.sampling_period = 100000, 10000, 1
    p.wall_model = WALL_CLL
    p.npc_free, p.molar_mass, p.ma_free = 10.0, 0.040, 4.0
    p.n_free, p.t_free, p.attack_angle, p.t_wall = 1e17, 200.0, 0.0, 300.0
    p.d_ref, p.viscosity_index, p.t_ref = 4.17e-10, 0.81, 273.0
    p.cll_normal, p.cll_tangential = 0.8, 0.8
    p.seed = 0x5EED
    p.precision = FP64
    p.max_particles_in_cell = 0
    p.capacity = 0
    return p


def reference_case(seed: int = 1) -> Params:
    """The plain reference case: 100x100, NPCFree 10 (~1e5 particles),
    specular walls, Dt 1e-5, 4000 steps sampled after step 2000, FP64."""
    return default_params().copy(wall_model=WALL_SPECULAR, n_step=4000,
                                 first_sampling_step=2000, seed=seed)


def large_case(wall_model: int = WALL_DIFFUSE, precision: int = FP32, seed: int = 1) -> Params:
    """The HBM-roofline case: 1000x1000, NPCFree 20 (~2e7 particles), angle 10,
    Dt 1e-6, 20000 steps sampled after step 10000, FP32 state; diffuse walls at
    Tw 300 K or CLL (0.8, 0.8)."""
    return default_params().copy(nx=1000, ny=1000, npc_free=20.0, attack_angle=10.0,
                                 wall_model=wall_model, t_wall=300.0, cll_normal=0.8,
                                 cll_tangential=0.8, dt=1e-6, n_step=20000,
                                 first_sampling_step=10000, precision=precision, seed=seed)


def warm_start_case(seed: int = 1) -> Params:
    """The warm-versus-cold case: 512x512, Ma 6, n 3e17, angle 15, CLL (0.5, 0.9),
    3x5 m box, NPCFree 30 (~8e6 particles), FP32 state."""
    return default_params().copy(nx=512, ny=512, ma_free=6.0, n_free=3e17, attack_angle=15.0,
                                 wall_model=WALL_CLL, cll_normal=0.5, cll_tangential=0.9,
                                 box_width=3.0, box_height=5.0, npc_free=30.0,
                                 precision=FP32, seed=seed)
