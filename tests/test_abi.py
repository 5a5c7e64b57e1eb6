"""The C ABI without a GPU: the library loads, exports every entry point that
include/dsmc.h declares, and its host-only functions (defaults, Setup(),
WallModelName(), Printing()) agree with the reference."""
from __future__ import annotations

import ctypes as C
import json
import re
from pathlib import Path

import numpy as np
import pytest

from dsmc_erlend_b200 import _lib
from dsmc_erlend_b200.abi import (WALL_CLL, WALL_DIFFUSE, WALL_SPECULAR, Derived, Params,
                                  default_params)
from dsmc_erlend_b200.engine import setup, write_field
from oracle.cpu import OracleEngine, RefEngine, ref_available

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def declared_functions(headers=None) -> set[str]:
    names = set()
    for h in headers or [h for h in (ROOT / "include").glob("*.h")
                         if h.name != "dsmc_surrogate.h"]:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b(dsmc_\w+)\s*\(", text):
            name = m.group(1)
            if not name.startswith("dsmc_philox") and not name.startswith("dsmc_stream") \
                    and name not in ("dsmc_mulhilo32", "dsmc_u32_to_unit"):
                names.add(name)
    return names


def test_library_exports_every_declared_entry_point(engine_lib):
    declared = declared_functions()
    assert "dsmc_step" in declared and "dsmc_ctx_create" in declared
    missing = [n for n in sorted(declared) if not hasattr(engine_lib, n)]
    assert not missing, f"not exported: {missing}"
    assert set(_lib.SIGNATURES) <= declared


def test_surrogate_library_exports_its_header():
    from dsmc_erlend_b200 import surrogate

    declared = declared_functions([ROOT / "include" / "dsmc_surrogate.h"])
    assert "dsmc_sg_conv_fwd" in declared
    lib = surrogate.lib()
    assert not [n for n in sorted(declared) if not hasattr(lib, n)]
    assert set(surrogate._SIGS) == declared


def test_defaults_match_reference_settings(engine_lib):
    p = Params()
    engine_lib.dsmc_default_params(C.byref(p))
    assert p.as_dict() == default_params().as_dict()


@pytest.mark.parametrize("kw", [{}, {"attack_angle": 10.0, "nx": 1000, "ny": 1000,
                                     "npc_free": 20.0},
                                {"ma_free": 6.0, "n_free": 3e17, "box_width": 3.0,
                                 "box_height": 5.0, "attack_angle": 15.0}])
def test_setup_matches_oracle(engine_lib, kw):
    p = default_params().copy(**kw)
    d = setup(p)
    s, od = OracleEngine.setup(p)
    assert s == 0
    assert d.as_dict() == od.as_dict()


def test_setup_bits_equal_reference_golden(engine_lib):
    """dsmc_setup restates the reference's Gamma (src/Initialization.cpp:111-207),
    so every derived constant (CrRef, MFT, MFP, Kn included) has the bits the
    reference's own Setup gave for the golden cases."""
    import json
    from pathlib import Path

    g = json.loads((Path(__file__).resolve().parent / "golden" /
                    "reference_steps.json").read_text())
    for wall, case in g["cases"].items():
        p = Params()
        for k, v in case["params"].items():
            setattr(p, k, v)
        d = setup(p).as_dict()
        for k, v in case["derived"].items():
            assert d[k] == v, f"{wall}: {k} {d[k]!r} != {v!r}"


SETUP_CASES = [
    {},  # the reference's own settings
    {"wall_model": WALL_SPECULAR, "n_step": 4000, "first_sampling_step": 2000},  # plain case
    {"nx": 1000, "ny": 1000, "npc_free": 20.0, "attack_angle": 10.0, "dt": 1e-6,
     "wall_model": WALL_DIFFUSE},  # the large single instance
    {"nx": 512, "ny": 512, "ma_free": 6.0, "n_free": 3e17, "attack_angle": 15.0,
     "cll_normal": 0.5, "cll_tangential": 0.9, "box_width": 3.0, "box_height": 5.0,
     "npc_free": 30.0},  # warm-versus-cold case
    {"viscosity_index": 0.5, "t_ref": 300.0, "d_ref": 3.6e-10, "molar_mass": 0.028},
    {"viscosity_index": 1.0, "ma_free": 2.0, "attack_angle": -30.0},
]


@pytest.mark.skipif(not ref_available(), reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("kw", SETUP_CASES)
def test_setup_bits_equal_reference_setup(engine_lib, kw):
    """Live: the reference's own Setup(), compiled here, against dsmc_setup
    (grids above the reference's 200 x 200 capacity are cut to it)."""
    p = default_params().copy(**kw)
    p.nx, p.ny = min(p.nx, 200), min(p.ny, 200)
    want = RefEngine(p).derived().as_dict()
    got = setup(p).as_dict()
    assert got == want
    s, od = OracleEngine.setup(p)
    assert s == 0 and od.as_dict() == want


def test_setup_rejects_bad_cll(engine_lib):
    d = Derived()
    for an, at in ((-0.1, 0.5), (0.5, 1.1), (float("nan"), 0.5)):
        p = default_params().copy(wall_model=WALL_CLL, cll_normal=an, cll_tangential=at)
        assert engine_lib.dsmc_setup(C.byref(p), C.byref(d)) == 40
    # Coefficients are only checked for CLL walls (Initialization.cpp:211).
    p = default_params().copy(wall_model=WALL_DIFFUSE, cll_normal=-1.0)
    assert engine_lib.dsmc_setup(C.byref(p), C.byref(d)) == 0


def test_wall_model_names(engine_lib):
    assert engine_lib.dsmc_wall_model_name(WALL_SPECULAR) == b"specular"
    assert engine_lib.dsmc_wall_model_name(WALL_DIFFUSE) == b"diffuse"
    assert engine_lib.dsmc_wall_model_name(WALL_CLL) == b"cll"
    assert engine_lib.dsmc_wall_model_name(7) is None
    assert engine_lib.dsmc_status_string(22) == b"too many particles in cell"


def test_context_without_device_fails_cleanly(engine_lib):
    from tests.conftest import gpu_available

    if gpu_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    p = default_params()
    assert engine_lib.dsmc_ctx_create(C.byref(p), None, 1, None, C.byref(h)) == 51


@pytest.mark.parametrize("wall", ["specular", "diffuse", "cll"])
def test_printing_is_byte_identical_to_reference(engine_lib, tmp_path, wall):
    """The field of the golden case after 8 steps (reproduced bit for bit by
    the oracle) written by dsmc_write_field equals the reference's Printing()
    output of the same field."""
    g = json.loads((GOLDEN / "reference_steps.json").read_text())
    case = g["cases"][wall]
    p, d = Params(), Derived()
    for k, v in case["params"].items():
        setattr(p, k, v)
    for k, v in case["derived"].items():
        setattr(d, k, v)
    o = OracleEngine(p, d)
    o.init_cold()
    o.step(8)
    write_field(p, d, o.counters()["sample_step"], o.fields(), str(tmp_path))
    for f in ("DSMC2D_Field.plt", "DSMC2D_Field.json"):
        got = (tmp_path / wall / f).read_bytes()
        want = (GOLDEN / f"printing_{wall}_{f}").read_bytes()
        assert got == want, f


def test_drag_report_arithmetic(engine_lib):
    """dsmc_drag_report: the drag block of Simulation.cpp:210-237 (mean force
    over DragSamplingTime, Cd on BoxHeight * DZ) for both impulse totals."""
    from dsmc_erlend_b200.engine import drag_report
    from dsmc_erlend_b200.abi import reference_case

    p = reference_case()
    d = setup(p)
    c = dict(np=0, step=40, sample_step=10, collisions_last_step=0, collisions_total=0,
             drag_collision_count=120, particle_steps=0, drag_impulse_total=3.0e-18, time=0.0,
             sample_time=0.0, drag_sampling_time=2.0e-4, drag_collision_count_window=70,
             drag_impulse_window=1.5e-18)
    r = drag_report(p, d, c)
    rho = p.n_free * d.molecule_mass
    q = 0.5 * rho * d.u_free ** 2 * (p.box_height * p.dz)
    assert r["rho_free"] == rho and r["area_ref"] == p.box_height * p.dz
    assert r["mean_force_total"] == pytest.approx(3.0e-18 / 2.0e-4, rel=1e-15)
    assert r["cd_total"] == pytest.approx(3.0e-18 / 2.0e-4 / q, rel=1e-15)
    assert r["cd"] == pytest.approx(1.5e-18 / 2.0e-4 / q, rel=1e-15)
    assert r["box_collisions"] == 120 and r["box_collisions_window"] == 70
    c["drag_sampling_time"] = 0.0
    with pytest.raises(RuntimeError):
        drag_report(p, d, c)


def test_cli_lists_run_controls_and_rejects_bad_periods(engine_lib):
    import subprocess

    exe = Path(__file__).resolve().parents[1] / "dsmc_erlend_b200" / "lib" / "dsmc"
    r = subprocess.run([str(exe), "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    for flag in ("--print-period", "--checkpoint", "--checkpoint-period", "--restart", "--drag"):
        assert flag in r.stdout
    for bad in (["--print-period", "0"], ["--checkpoint-period", "2.5"], ["--restart"]):
        r = subprocess.run([str(exe), *bad], capture_output=True, text=True, timeout=60)
        assert r.returncode == 2, bad


def test_sgbench_covers_every_layer_shape():
    # The surrogate benchmark times each distinct (resolution, Cin, Cout) of
    # the network once.
    from dsmc_erlend_b200 import sgbench
    from dsmc_erlend_b200.surrogate import LAYERS, RES

    shapes = sgbench._shapes(8)
    assert shapes[0] == (8, RES, RES, LAYERS[0][3], LAYERS[0][4])
    assert len(shapes) == len({s[1:] for s in shapes})
    assert {(s[3], s[4]) for s in shapes} == {(l[3], l[4]) for l in LAYERS}
