"""Generates the golden fixtures in tests/golden/ from the REFERENCE's own CPU
code (oracle/_ref/libref_bf64.so and libref_bf32.so, built from the reference
sources by oracle/build_ref.sh).  Run from the repository root where the
reference sources are present:

    python tests/golden/gen_golden.py

Each .npz holds the inputs (seeded, synthetic) and the reference outputs, so
tests on machines without the reference can pin the oracle and the GPU path.
Fixtures:
  ops_2d.npz      2-D 64x64, 1 coil, 1024-sample spiral, field map:
                  parallelFtCpu(x), parallelIftCpu(d) in FP64
  ops_2d_c3.npz   2-D 32x32, 3 coils: the same with SENSE
  bf_2d.npz       bruteForceCpu, 64x64, 1 coil, 4 x 1024 spiral, cg_num 3,
                  -fdp 1e-2, -tv_num 2, FP64 and FP32 builds
  bf_2d_c3.npz    bruteForceCpu, 32x32, 3 coils, cg_num 5, -fdp 1e-2 (no TV)
  bf_2d_tv_long.npz  bruteForceCpu, 64x64, 1 coil, 4 x 1024 spiral, cg_num 6,
                  -fdp 1e-3, -tv_num 3: a configuration whose CG iterates amplify
                  rounding-level perturbations (used for reported comparisons)
  bf_2d_reg.npz   bruteForceCpu with -reg, 32x32, 2 coils, cg_num 4, -fdp 1e-2,
                  -tv_num 2: the roughness matrix is the periodic difference
                  matrix of synth.fd_matrix with every entry scaled by a seeded
                  factor in [0.5, 1.5] (a generic C, not the FD stencil),
                  stored with the fixture (C_rows, C_cols, C_I, C_J, C_V)

The short runs are chosen so that a 1e-9 relative perturbation of the CG step
moves the FP64 result by less than 1e-6; longer TV runs amplify such
perturbations by 1e5 or more, so no finite-precision implementation other
than a bit-for-bit replay of the reference's operation order can match them
to 1e-4.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from __graft_entry__ import load_package  # noqa: E402

OUT = Path(__file__).resolve().parent


def small_case(n: int, n_coil: int, n_il: int, n_s: int, seed: int):
    load_package()
    from impatient_mri_b200 import synth
    rng = np.random.default_rng(seed)
    kx, ky, t = synth.spiral(n_il, n_s, n / 2, rng)
    kz = np.zeros_like(kx)
    ix, iy, iz = synth.grid_positions(n, n, 1)
    img = synth.ellipse_phantom((n, n), 6, rng)
    fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
    if n_coil == 1:
        sens = np.ones((1, n * n), np.complex64)
    else:
        sens = np.stack([synth.to_voxel_order(m) for m in
                         synth.coil_maps((n, n), n_coil, rng)]).astype(np.complex64)
    case = dict(kx=kx, ky=ky, kz=kz, t=t, ix=ix, iy=iy, iz=iz, fm=fm, sens=sens,
                x_true=synth.to_voxel_order(img).astype(np.complex64), dims=(n, n, 1),
                opts=dict(use_z=0))
    y = oracle.ref_parallel_ft(case["x_true"], case, "bf64")
    case["kdata"] = synth.add_noise(y, 40.0, rng).astype(np.complex64)
    return case, rng


def arrays(case):
    keys = ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm", "sens", "kdata", "x_true")
    return {k: case[k] for k in keys} | {"dims": np.array(case["dims"])}


def main() -> int:
    if not oracle.ref_available("bf64"):
        print("reference CPU build missing: run oracle/build_ref.sh first", file=sys.stderr)
        return 1
    for name, n, C, seed in (("ops_2d", 64, 1, 11), ("ops_2d_c3", 32, 3, 12)):
        case, rng = small_case(n, C, 4, 256, seed)
        x = (rng.standard_normal(n * n) + 1j * rng.standard_normal(n * n)).astype(np.complex64)
        M = case["kx"].size
        d = (rng.standard_normal(C * M) + 1j * rng.standard_normal(C * M)).astype(np.complex64)
        np.savez_compressed(OUT / f"{name}.npz", **arrays(case), x=x, d=d,
                            ft64=oracle.ref_parallel_ft(x, case, "bf64"),
                            ift64=oracle.ref_parallel_ift(d, case, "bf64"))
        print("wrote", name)
    for name, n, C, n_s, seed, kw in (
            ("bf_2d", 64, 1, 1024, 21, dict(cg_num=3, lam=1e-2, tv=True, tv_num=2)),
            ("bf_2d_c3", 32, 3, 256, 22, dict(cg_num=5, lam=1e-2, tv=False, tv_num=1)),
            ("bf_2d_tv_long", 64, 1, 1024, 23, dict(cg_num=6, lam=1e-3, tv=True, tv_num=3))):
        case, _ = small_case(n, C, 4, n_s, seed)
        np.savez_compressed(OUT / f"{name}.npz", **arrays(case), cg_num=kw["cg_num"],
                            lam=kw["lam"], tv=int(kw["tv"]), tv_num=kw["tv_num"],
                            x64=oracle.ref_bf_cg(case, kind="bf64", **kw),
                            x32=oracle.ref_bf_cg(case, kind="bf32", **kw))
        print("wrote", name)
    case, rng = small_case(32, 2, 4, 256, 24)
    from impatient_mri_b200 import synth
    rows, cols, I, J, V = synth.fd_matrix((32, 32))
    V = V * rng.uniform(0.5, 1.5, V.size)
    reg = (rows, cols, I, J, V)
    kw = dict(cg_num=4, lam=1e-2, tv=True, tv_num=2)
    np.savez_compressed(OUT / "bf_2d_reg.npz", **arrays(case), C_rows=rows, C_cols=cols, C_I=I,
                        C_J=J, C_V=V, cg_num=kw["cg_num"], lam=kw["lam"], tv_num=kw["tv_num"],
                        x64=oracle.ref_bf_cg_reg(case, reg, kind="bf64", **kw),
                        x32=oracle.ref_bf_cg_reg(case, reg, kind="bf32", **kw))
    print("wrote bf_2d_reg")
    return 0


if __name__ == "__main__":
    sys.exit(main())
