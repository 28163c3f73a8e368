"""mriSolver flag handling (main.cpp:148-405): errors exit 1 before any GPU work."""
import subprocess

import pytest


def run(pkg, *args):
    r = subprocess.run([str(pkg.MRISOLVER), *args], capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("args,msg", [
    ((), "Usage"),
    (("-cg_num", "0", "-idir", "x"), "Zero or wrong CG"),
    (("-idir",), "Missing input directory"),
    (("-idir", "x", "-tv"), "no weight parameter"),
    (("-idir", "x", "-gridOS_Q", "1.5"), "toeplitzGridding flag is not found"),
    (("-idir", "x", "-toeplitzGridding", "-gridOS_Q", "3"), "[1.0,2.0]"),
    (("-idir", "x", "-ntime_segs", "4"), "toeplitz flag is not found"),
    (("-idir", "x", "-reuseQ", "q"), "-reuseQ flag requires"),
    (("-idir", "x", "-bogus"), "Unknown option"),
    (("-idir", "x", "-reg"), "c.rmtx not found"),
    (("-idir", "x", "-cpu"), "no CPU reconstruction path"),
])
def test_flag_errors(pkg, args, msg):
    rc, out = run(pkg, *args)
    assert rc == 1
    assert msg in out


def test_missing_input_dir_fails(pkg, tmp_path):
    rc, out = run(pkg, "-idir", str(tmp_path / "nope"), "-cg_num", "2")
    assert rc == 1
    assert "kx.dat" in out
