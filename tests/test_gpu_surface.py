"""The reference-named C++ surface and the dsmc command line, on the GPU."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

from dsmc_erlend_b200.build import CLI, LIB_DIR

ROOT = Path(__file__).resolve().parent.parent
pytestmark = pytest.mark.gpu


def test_reference_style_program(cuda, engine_lib, tmp_path):
    exe = tmp_path / "surface_checks"
    from oracle.cpu import build_oracle

    olib = build_oracle().parent  # the checker: the C restatement of the reference
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", str(ROOT / "include"),
                    "-I", str(ROOT / "oracle"), "-I", "/usr/local/cuda/include",
                    str(ROOT / "tests" / "cpp" / "surface_checks.cpp"), "-o", str(exe),
                    "-L", str(LIB_DIR), "-ldsmc_b200", f"-Wl,-rpath,{LIB_DIR}",
                    "-L", str(olib), "-ldsmc_oracle", f"-Wl,-rpath,{olib}"], check=True)
    r = subprocess.run([str(exe), str(tmp_path / "results")], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "surface checks passed" in r.stdout


def test_command_line(cuda, engine_lib, tmp_path):
    assert CLI.exists(), "dsmc program not built"
    r = subprocess.run([str(CLI), "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--angle-of-attack" in r.stdout
    r = subprocess.run([str(CLI), "--aoa", "abc"], capture_output=True, text=True)
    assert r.returncode == 2 and "Invalid angle" in r.stderr
    r = subprocess.run([str(CLI), "--aoa"], capture_output=True, text=True)  # Simulation.cpp:44
    assert r.returncode == 2 and r.stderr == "--aoa requires an angle in degrees.\n"
    r = subprocess.run([str(CLI), "--aoa", "10", "--wall", "diffuse", "--nx", "50", "--ny", "50",
                        "--steps", "300", "--first-sampling-step", "100", "--results",
                        str(tmp_path)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "Time step 300" in r.stdout
    lines = (tmp_path / "diffuse" / "DSMC2D_Field.plt").read_text().splitlines()
    assert lines[1] == "ZONE I=50 J=50" and len(lines) == 2 + 2500
    meta = (tmp_path / "diffuse" / "DSMC2D_Field.json").read_text()
    assert '"angle_of_attack_degrees": 10' in meta and '"wall_model": "diffuse"' in meta
