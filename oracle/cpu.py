"""ctypes bindings of the CPU checkers.  TEST INFRASTRUCTURE ONLY.

OracleEngine wraps the C restatement (oracle/dsmc_oracle.c, built into
oracle/lib/).  RefEngine wraps the reference's own routines compiled with the
shims of oracle/ref_shim (built into oracle/_ref/ from the reference sources;
one instance per process, since the reference keeps global state).  Both
expose the same methods so a test can run either.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from dsmc_erlend_b200.abi import Counters, Derived, Params

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "lib" / "libdsmc_oracle.so"
REF_LIB = HERE / "_ref" / "libdsmc_ref.so"
REF_BASELINE = HERE / "_ref" / "dsmc_ref_baseline"

_D = C.POINTER(C.c_double)
_I32 = C.POINTER(C.c_int32)


def build_oracle() -> Path:
    """Compiles the C restatement if its library is missing or stale."""
    src = HERE / "dsmc_oracle.c"
    if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < src.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return ORACLE_LIB


def ref_available() -> bool:
    return REF_LIB.exists()


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


class _Base:
    ncell: int

    def particles(self) -> dict:
        n = self.np()
        arrs = [np.empty(n, dtype=np.float64) for _ in range(5)]
        self._call("get_particles", *[_dptr(a) for a in arrs])
        return dict(zip(("x", "y", "vx", "vy", "vz"), arrs))

    def set_particles(self, st: dict, raw: bool = False) -> int:
        arrs = [np.ascontiguousarray(st[k], dtype=np.float64) for k in ("x", "y", "vx", "vy", "vz")]
        name = "set_particles_raw" if raw else "set_particles"
        return self._status(name, *[_dptr(a) for a in arrs], C.c_int64(len(arrs[0])))

    def fields(self) -> np.ndarray:
        out = np.empty((self.ncell, 17), dtype=np.float64)
        self._call("get_fields", _dptr(out))
        return out

    def set_fields(self, f: np.ndarray, sample_step: int):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._call("set_fields", _dptr(f), C.c_int64(sample_step))

    def counters(self) -> dict:
        c = Counters()
        self._call("get_counters", C.byref(c))
        return c.as_dict()

    def step(self, n: int = 1) -> int:
        for _ in range(n):
            s = self._status("step")
            if s:
                return s
        return 0

    def stage(self, name: str) -> int:
        return self._status("stage_" + name)


class OracleEngine(_Base):
    """The C restatement of the reference time step (FP64)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(str(build_oracle()))
            L.dsmc_oracle_create.restype = C.c_void_p
            L.dsmc_oracle_create.argtypes = [C.POINTER(Params), C.POINTER(Derived), C.c_int64]
            L.dsmc_oracle_destroy.argtypes = [C.c_void_p]
            L.dsmc_oracle_np.restype = C.c_int64
            L.dsmc_oracle_np.argtypes = [C.c_void_p]
            L.dsmc_oracle_setup.argtypes = [C.POINTER(Params), C.POINTER(Derived)]
            L.dsmc_oracle_intersect.argtypes = [C.c_void_p] + [C.c_double] * 4 + [_D] * 3
            L.dsmc_oracle_inside_box.argtypes = [C.c_void_p, C.c_double, C.c_double]
            L.dsmc_oracle_scatter.argtypes = [C.c_void_p, _D, C.c_double, C.c_double,
                                              C.c_uint32, C.c_uint32, C.c_uint32]
            L.dsmc_oracle_generate.argtypes = [C.c_void_p, _D] + [C.c_double] * 4 + \
                [C.c_int, C.c_uint32, C.c_uint32, C.c_uint32]
            L.dsmc_oracle_collide_list.argtypes = [C.c_void_p, C.c_double, C.c_int, _I32,
                                                   C.c_uint32, C.c_uint32, C.c_uint32,
                                                   C.POINTER(C.c_int)]
            L.dsmc_oracle_elastic.argtypes = [C.c_void_p, _D, _D, C.c_double, C.c_uint32,
                                              C.c_uint32, C.c_uint32]
            cls._lib = L
        return cls._lib

    @classmethod
    def setup(cls, p: Params) -> tuple[int, Derived]:
        d = Derived()
        s = cls.lib().dsmc_oracle_setup(C.byref(p), C.byref(d))
        return s, d

    def __init__(self, p: Params, derived: Derived | None = None, capacity: int = 0):
        L = self.lib()
        self.p = p.copy()
        self.ncell = p.nx * p.ny
        dptr = C.byref(derived) if derived is not None else None
        self.h = L.dsmc_oracle_create(C.byref(self.p), dptr, C.c_int64(capacity))
        if not self.h:
            raise ValueError("oracle rejected the parameters")

    def __del__(self):
        if getattr(self, "h", None) and self._lib is not None:
            self._lib.dsmc_oracle_destroy(C.c_void_p(self.h))
            self.h = None

    def _fn(self, name):
        return getattr(self.lib(), "dsmc_oracle_" + name)

    def _status(self, name, *args) -> int:
        return self._fn(name)(C.c_void_p(self.h), *args)

    def _call(self, name, *args):
        s = self._status(name, *args)
        if s:
            raise RuntimeError(f"oracle {name} failed with status {s}")

    def np(self) -> int:
        return self.lib().dsmc_oracle_np(C.c_void_p(self.h))

    def init_cold(self) -> int:
        return self._status("init_cold")

    def set_step(self, step: int):
        self._call("set_step", C.c_int64(step))

    def cell_starts(self) -> np.ndarray:
        out = np.empty(self.ncell + 1, dtype=np.int32)
        self._call("get_cell_starts", out.ctypes.data_as(_I32))
        return out

    def intersect(self, x, y, dx, dy):
        t, nx, ny = C.c_double(), C.c_double(), C.c_double()
        hit = self.lib().dsmc_oracle_intersect(C.c_void_p(self.h), x, y, dx, dy, C.byref(t),
                                               C.byref(nx), C.byref(ny))
        return bool(hit), t.value, nx.value, ny.value

    def inside_box(self, x, y) -> bool:
        return bool(self.lib().dsmc_oracle_inside_box(C.c_void_p(self.h), x, y))

    def scatter(self, v, nx, ny, kind, step, entity):
        vv = np.ascontiguousarray(v, dtype=np.float64).copy()
        s = self.lib().dsmc_oracle_scatter(C.c_void_p(self.h), _dptr(vv), nx, ny, kind, step,
                                           entity)
        return s, vv

    def generate(self, rect, n_gas, ux, uy, t_gas, move_flag, kind, step, entity) -> int:
        r = np.ascontiguousarray(rect, dtype=np.float64)
        return self.lib().dsmc_oracle_generate(C.c_void_p(self.h), _dptr(r), n_gas, ux, uy,
                                               t_gas, move_flag, kind, step, entity)

    def collide_list(self, cell_volume, ipc, kind, step, entity) -> int:
        ids = np.ascontiguousarray(ipc, dtype=np.int32)
        nc = C.c_int()
        self._call("collide_list", C.c_double(cell_volume), len(ids), ids.ctypes.data_as(_I32),
                   kind, step, entity, C.byref(nc))
        return nc.value

    def elastic(self, v1, v2, cr, kind, step, entity):
        a = np.ascontiguousarray(v1, dtype=np.float64).copy()
        b = np.ascontiguousarray(v2, dtype=np.float64).copy()
        self._call("elastic", _dptr(a), _dptr(b), C.c_double(cr), kind, step, entity)
        return a, b

    def remove_inside_box(self):
        self._call("remove_inside_box")

    def remove_outside_domain(self):
        self._call("remove_outside_domain")


class RefEngine(_Base):
    """The reference's own routines under the same stream contract."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not REF_LIB.exists():
                raise FileNotFoundError(f"{REF_LIB} is not built (make -C oracle ref)")
            L = C.CDLL(str(REF_LIB))
            L.dsmc_ref_np.restype = C.c_longlong
            L.dsmc_ref_intersect.argtypes = [C.c_double] * 4 + [_D] * 3
            L.dsmc_ref_inside_box.argtypes = [C.c_double, C.c_double]
            L.dsmc_ref_scatter.argtypes = [_D, C.c_double, C.c_double, C.c_uint32, C.c_uint32,
                                           C.c_uint32]
            L.dsmc_ref_cll.argtypes = [_D] + [C.c_double] * 6
            L.dsmc_ref_select_stream.argtypes = [C.c_uint32] * 3
            L.dsmc_ref_draws.restype = C.c_ulonglong
            L.dsmc_ref_brng.restype = C.c_double
            L.dsmc_ref_gaussian.restype = C.c_double
            L.dsmc_ref_gaussian.argtypes = [C.c_double, C.c_double]
            L.dsmc_ref_poisson.argtypes = [C.c_double]
            L.dsmc_ref_set_particles.argtypes = [_D] * 5 + [C.c_longlong]
            L.dsmc_ref_set_particles_raw.argtypes = [_D] * 5 + [C.c_longlong]
            L.dsmc_ref_set_fields.argtypes = [_D, C.c_longlong]
            L.dsmc_ref_set_step.argtypes = [C.c_longlong]
            L.dsmc_ref_write_field.argtypes = [C.c_char_p]
            cls._lib = L
        return cls._lib

    def __init__(self, p: Params, derived: Derived | None = None):
        L = self.lib()
        self.p = p.copy()
        self.ncell = p.nx * p.ny
        s = L.dsmc_ref_configure(C.byref(self.p))
        if s:
            raise ValueError(f"reference Setup failed with code {s}")
        if derived is not None:
            L.dsmc_ref_set_derived(C.byref(derived))

    def derived(self) -> Derived:
        d = Derived()
        self.lib().dsmc_ref_get_derived(C.byref(d))
        return d

    def _status(self, name, *args) -> int:
        return getattr(self.lib(), "dsmc_ref_" + name)(*args)

    def _call(self, name, *args):
        s = self._status(name, *args)
        if s:
            raise RuntimeError(f"reference {name} failed with code {s}")

    def np(self) -> int:
        return self.lib().dsmc_ref_np()

    def init_cold(self) -> int:
        return self._status("init_cold")

    def set_step(self, step: int):
        self._call("set_step", C.c_longlong(step))

    def npc(self) -> np.ndarray:
        out = np.empty(self.ncell, dtype=np.int32)
        self._call("get_npc", out.ctypes.data_as(_I32))
        return out

    def cell_starts(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum(self.npc())]).astype(np.int32)

    def intersect(self, x, y, dx, dy):
        t, nx, ny = C.c_double(), C.c_double(), C.c_double()
        hit = self.lib().dsmc_ref_intersect(x, y, dx, dy, C.byref(t), C.byref(nx), C.byref(ny))
        return bool(hit), t.value, nx.value, ny.value

    def inside_box(self, x, y) -> bool:
        return bool(self.lib().dsmc_ref_inside_box(x, y))

    def scatter(self, v, nx, ny, kind, step, entity):
        vv = np.ascontiguousarray(v, dtype=np.float64).copy()
        s = self.lib().dsmc_ref_scatter(_dptr(vv), nx, ny, kind, step, entity)
        return s, vv

    def cll(self, v, m, tw, nx, ny, an, at):
        vv = np.ascontiguousarray(v, dtype=np.float64).copy()
        s = self.lib().dsmc_ref_cll(_dptr(vv), m, tw, nx, ny, an, at)
        return s, vv

    def generate(self, rect, n_gas, ux, uy, t_gas, move_flag, kind, step, entity) -> int:
        r = np.ascontiguousarray(rect, dtype=np.float64)
        L = self.lib()
        L.dsmc_ref_generate.argtypes = [_D] + [C.c_double] * 4 + [C.c_int] + [C.c_uint32] * 3
        return L.dsmc_ref_generate(_dptr(r), n_gas, ux, uy, t_gas, move_flag, kind, step, entity)

    def collide_list(self, cell_volume, ipc, kind, step, entity) -> int:
        ids = np.ascontiguousarray(ipc, dtype=np.int32)
        nc = C.c_int()
        L = self.lib()
        L.dsmc_ref_collide_list.argtypes = [C.c_double, C.c_int, _I32] + [C.c_uint32] * 3 + \
            [C.POINTER(C.c_int)]
        self._call("collide_list", cell_volume, len(ids), ids.ctypes.data_as(_I32), kind, step,
                   entity, C.byref(nc))
        return nc.value

    def elastic(self, v1, v2, cr, kind, step, entity):
        a = np.ascontiguousarray(v1, dtype=np.float64).copy()
        b = np.ascontiguousarray(v2, dtype=np.float64).copy()
        L = self.lib()
        L.dsmc_ref_elastic.argtypes = [_D, _D, C.c_double] + [C.c_uint32] * 3
        self._call("elastic", _dptr(a), _dptr(b), cr, kind, step, entity)
        return a, b

    def remove_inside_box(self):
        self._call("remove_inside_box")

    def write_field(self, directory: str | os.PathLike):
        self._call("write_field", str(directory).encode())
