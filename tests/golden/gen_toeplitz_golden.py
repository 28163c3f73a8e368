"""Golden outputs of the reference's Toeplitz path, made by running the
reference's own GPU program (oracle/_ref/mriSolver_ref, built from the
reference sources by oracle/build_ref_gpu.sh) on seeded 2-D datasets.  The
reference has no CPU implementation of this path, so this is the only way to
pin the Toeplitz oracle (oracle/toeplitz.py) to the reference itself.

Needs a GPU.  Usage (repository root):

    python tests/golden/gen_toeplitz_golden.py [out_dir]

For each case the .npz holds the inputs and the reference's Q_stone.file
(-writeQ), FhD.file and out.file contents:
  toep_2d_fd.npz  32x32, 2 coils, 4 x 256 spiral, field map, -ntime_segs 4,
                  -gridOS_Q 2 -gridOS_FH 1.5, -cg_num 5 -fdp 0.01
  toep_2d_tv.npz  the same geometry, -cg_num 3 -fdp 0.01 -tv_num 2
The inputs respect the reference's assumptions (square image, |k| < N/2,
fewer than 128 samples per gridding bin, sizes divisible by 256).
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from __graft_entry__ import load_package  # noqa: E402

REF = ROOT / "oracle" / "_ref" / "mriSolver_ref"


def make_inputs(seed: int):
    load_package()
    from impatient_mri_b200 import synth
    rng = np.random.default_rng(seed)
    n, C = 32, 2
    kx, ky, t = synth.spiral(4, 256, n / 2 - 0.05, rng)
    kz = np.zeros_like(kx)
    ix, iy, iz = synth.grid_positions(n, n, 1)
    img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 6, rng))
    fm = synth.to_voxel_order(synth.field_map((n, n), rng, max_hz=20.0)).astype(np.float32)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng)])
    case = dict(kx=kx, ky=ky, kz=kz, t=t, ix=ix, iy=iy, iz=iz, fm=fm,
                sens=sens.astype(np.complex64), dims=(n, n, 1), opts=dict(use_z=0))
    y = oracle.ft(img, case, use_z=0)
    case["kdata"] = synth.add_noise(y, 40.0, rng).astype(np.complex64)
    return case


def run_case(case, flags, work: Path):
    from impatient_mri_b200 import io
    work.mkdir(parents=True, exist_ok=True)
    io.write_dataset(work, "0.2", kx=case["kx"], ky=case["ky"], kz=case["kz"], t=case["t"],
                     ix=case["ix"], iy=case["iy"], iz=case["iz"], fm=case["fm"],
                     kdata=case["kdata"], sensi=case["sens"], dims=(32, 32, 1),
                     num_coil=case["sens"].shape[0])
    cmd = [str(REF), "-idir", str(work), "-toeplitzGridding", "-writeQ", *flags]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    N = case["ix"].size
    L = int(float(flags[flags.index("-ntime_segs") + 1]))
    q = np.fromfile(work / "Q_stone.file", np.float32).reshape(L + 1, 2, 4 * N)
    fhd = np.fromfile(work / "FhD.file", np.float32).reshape(2, N)
    out = np.fromfile(work / "out.file", np.float32).reshape(2, N)
    return dict(Q=q[:, 0] + 1j * q[:, 1], fhd=fhd[0] + 1j * fhd[1], out=out[0] + 1j * out[1],
                log=r.stdout[-4000:])


def main() -> int:
    out_dir = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out_dir.mkdir(parents=True, exist_ok=True)
    if not REF.exists():
        print("oracle/_ref/mriSolver_ref missing: run oracle/build_ref_gpu.sh", file=sys.stderr)
        return 1
    case = make_inputs(31)
    runs = {
        "toep_2d_fd": ["-ntime_segs", "4", "-gridOS_Q", "2.0", "-gridOS_FH", "1.5",
                       "-cg_num", "5", "-fdp", "0.01"],
        "toep_2d_tv": ["-ntime_segs", "4", "-gridOS_Q", "2.0", "-gridOS_FH", "1.5",
                       "-cg_num", "3", "-fdp", "0.01", "-tv_num", "2"],
    }
    with tempfile.TemporaryDirectory() as td:
        for name, flags in runs.items():
            res = run_case(case, flags, Path(td) / name)
            keys = ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm", "sens", "kdata")
            np.savez_compressed(out_dir / f"{name}.npz", **{k: case[k] for k in keys},
                                dims=np.array(case["dims"]), flags=np.array(flags),
                                Q=res["Q"].astype(np.complex64),
                                fhd=res["fhd"].astype(np.complex64),
                                out=res["out"].astype(np.complex64))
            (out_dir / f"{name}.log").write_text(res["log"])
            print("wrote", name)
    return 0


if __name__ == "__main__":
    sys.exit(main())
