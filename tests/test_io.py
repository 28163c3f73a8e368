"""Input formats: the Python writers produce files the C++ reader accepts with
the reference's rules; malformed files give IMP_ERR_FORMAT instead of exiting."""
import numpy as np
import pytest

from conftest import REF_DATA


@pytest.fixture
def io(pkg):
    from impatient_mri_b200 import io as m
    return m


def _write(io, synth, d, fmt, C=2, S=1):
    rng = np.random.default_rng(0)
    kx, ky, t = synth.spiral(2, 64, 8.0, rng)
    ix, iy, iz = synth.grid_positions(16, 16, 1)
    N, M = ix.size, kx.size
    kd = (rng.standard_normal((S, C, M)) + 1j * rng.standard_normal((S, C, M))).astype(np.complex64)
    sens = (rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N))).astype(np.complex64)
    io.write_dataset(d, fmt, kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz,
                     fm=np.zeros(S * N, np.float32), kdata=kd, sensi=sens, dims=(16, 16, 1),
                     num_coil=C, num_slices=S)
    return M, N, kd, sens


@pytest.mark.parametrize("fmt", ["0.2", "1.0"])
def test_writer_reader_roundtrip(pkg, synth, io, tmp_path, fmt):
    M, N, kd, sens = _write(io, synth, tmp_path, fmt, C=2, S=2)
    info = pkg.dataset_info(str(tmp_path))
    assert (info["num_k"], info["num_i"], info["num_coil"], info["num_slices"]) == (M, N, 2, 2)
    ds = io.read_dataset(tmp_path)
    assert np.array_equal(ds["kdata_r"], kd.real.ravel())
    assert np.array_equal(ds["sensi_i"], sens.imag.ravel())


def test_one_coil_forces_unit_sensitivity(io, synth, tmp_path):
    _write(io, synth, tmp_path, "1.0", C=1)
    ds = io.read_dataset(tmp_path)
    assert np.all(ds["sensi_r"] == 1) and np.all(ds["sensi_i"] == 0)


def test_truncated_file_is_a_format_error(pkg, io, synth, tmp_path):
    _write(io, synth, tmp_path, "1.0")
    raw = (tmp_path / "kdata_r.dat").read_bytes()
    (tmp_path / "kdata_r.dat").write_bytes(raw[: len(raw) // 2])
    with pytest.raises(pkg.ImpError) as e:
        pkg.dataset_info(str(tmp_path))
    assert e.value.status == 4


def test_missing_file_is_an_io_error(pkg, io, synth, tmp_path):
    _write(io, synth, tmp_path, "0.2")
    (tmp_path / "t.dat").unlink()
    with pytest.raises(pkg.ImpError) as e:
        pkg.dataset_info(str(tmp_path))
    assert e.value.status == 3


def test_short_array_is_a_format_error(pkg, io, synth, tmp_path):
    M, N, _, _ = _write(io, synth, tmp_path, "0.2")
    io.write_v02(tmp_path / "fm.dat", np.zeros(N // 2, np.float32), N // 2)
    with pytest.raises(pkg.ImpError) as e:
        pkg.dataset_info(str(tmp_path))
    assert e.value.status == 4


@pytest.mark.parametrize("name,expect", [("64x64x1", (3770, 4096, 1, 1)),
                                         ("64x64x16-4coils", (66592, 65536, 4, 1))])
def test_reference_datasets(pkg, io, name, expect):
    if not (REF_DATA / name).exists():
        pytest.skip("reference datasets absent")
    info = pkg.dataset_info(str(REF_DATA / name))
    assert (info["num_k"], info["num_i"], info["num_coil"], info["num_slices"]) == expect
    ds = io.read_dataset(REF_DATA / name)
    assert (ds["num_k"], ds["num_i"], ds["num_coil"]) == expect[:3]
