"""mriSolver input/output file formats in Python.

Writers produce what the reference's readers accept (kernels/structures.cpp:
readDataFile :782-863 for 0.2, readDataFile_10 :866-1162 for 1.0), with the
same layout as matlab_utils/format_conversion/datawrite.m: one binary section
per coil.  Readers follow the same rules as the C++ reader in csrc/io.cpp.
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

FILES = ["kx", "ky", "kz", "kdata_r", "kdata_i", "sensi_r", "sensi_i", "fm",
         "ix", "iy", "iz", "idata_r", "idata_i", "t"]


def write_v02(fn, data, dim1: int, ncoils: int = 1, nslices: int = 1) -> None:
    a = np.ascontiguousarray(data, dtype="<f4").ravel()
    with open(fn, "wb") as f:
        f.write(struct.pack("<fiiii", 0.2, int(dim1), int(ncoils), int(nslices), a.size))
        f.write(a.tobytes())


def write_v10(fn, data, nx: int, ny: int, nz: int, coil_number: int | None = None,
              slice_number: int = 1) -> None:
    a = np.ascontiguousarray(data, dtype="<f4").ravel()
    nsec = coil_number or 1
    if a.size % nsec:
        raise ValueError("data size not divisible by coil_number")
    per = a.size // nsec
    with open(fn, "wb") as f:
        hdr = [f"version = {1.0:f}", f"xDimension = {nx}", f"yDimension = {ny}",
               f"zDimension = {nz}"]
        if coil_number is not None:
            hdr.append(f"coil_number = {coil_number}")
        hdr += [f"slice_number = {slice_number}", f"file_size = {a.size}"]
        f.write(("\n".join(hdr) + "\n").encode())
        for c in range(nsec):
            f.write(f"// Coil No. {c + 1}\nBinary_Size = {per}\nBinary:\n".encode())
            f.write(a[c * per:(c + 1) * per].tobytes())
        f.write(b"\nEOF\n")


def read_file(fn, v02: bool | None = None):
    """Returns (header dict, float32 data) of one input file."""
    raw = Path(fn).read_bytes()
    if v02 is None:
        v02 = struct.unpack("<f", raw[:4])[0] == np.float32(0.2)
    if v02:
        ver, dim1, nc, ns, size = struct.unpack("<fiiii", raw[:20])
        data = np.frombuffer(raw, "<f4", count=size, offset=20).copy()
        return dict(version=ver, per_coil=dim1, coil_number=nc, slice_number=ns), data
    hdr: dict = {}
    pos, filled, data, local_coils = 0, 0, None, -1
    while pos < len(raw):
        nl = raw.find(b"\n", pos)
        line = raw[pos:(len(raw) if nl < 0 else nl)].decode("latin1").strip()
        pos = len(raw) if nl < 0 else nl + 1
        if not line or line.startswith("//"):
            continue
        if line.startswith("EOF"):
            break
        key, _, val = (s.strip() for s in line.partition("="))
        if key == "version":
            hdr["version"] = float(val)
        elif key in ("xDimension", "yDimension", "zDimension", "slice_number"):
            hdr[key] = int(val)
        elif key == "coil_number":
            local_coils = int(val)
            hdr["coil_number"] = local_coils
        elif key == "file_size":
            size = int(val)
            hdr["file_size"] = size
            hdr["per_coil"] = size // (local_coils if local_coils > 0 else 1)
            data = np.zeros(size, np.float32)
        elif key == "Binary_Size":
            n = int(val)
            while True:
                nl = raw.find(b"\n", pos)
                b = raw[pos:nl].decode("latin1").strip()
                pos = nl + 1
                if b and not b.startswith("//"):
                    break
            if b != "Binary:":
                raise ValueError(f"{fn}: Binary_Size not followed by Binary:")
            data[filled:filled + n] = np.frombuffer(raw, "<f4", count=n, offset=pos)
            pos += 4 * n
            filled += n
    if data is None or filled != data.size:
        raise ValueError(f"{fn}: binary sections do not add up to file_size")
    return hdr, data


def write_dataset(d, fmt: str, *, kx, ky, kz, t, ix, iy, iz, fm, kdata, sensi, idata=None,
                  dims=(0, 0, 0), num_coil=1, num_slices=1) -> None:
    """Writes an mriSolver input directory.  kdata: complex [S][C][M];
    sensi: complex [C][N]; fm: [S][N]; idata: complex [S][N] (zeros if None)."""
    d = Path(d)
    d.mkdir(parents=True, exist_ok=True)
    M, N = np.size(kx), np.size(ix)
    kdata = np.asarray(kdata).reshape(num_slices, num_coil, M)
    sensi = np.asarray(sensi).reshape(num_coil, N)
    if idata is None:
        idata = np.zeros((num_slices, N), np.complex64)
    arrays = {
        "kx": (kx, 1), "ky": (ky, 1), "kz": (kz, 1), "t": (t, 1),
        "ix": (ix, 1), "iy": (iy, 1), "iz": (iz, 1), "fm": (fm, 1),
        "kdata_r": (kdata.real, num_coil), "kdata_i": (kdata.imag, num_coil),
        "sensi_r": (sensi.real, num_coil), "sensi_i": (sensi.imag, num_coil),
        "idata_r": (np.real(idata), 1), "idata_i": (np.imag(idata), 1),
    }
    nx, ny, nz = dims
    for name, (a, nc) in arrays.items():
        a = np.asarray(a, np.float32).ravel()
        if fmt == "0.2":
            # every 0.2 header states the dataset's coil count: the reference
            # keeps the count of the last file it reads (t.dat)
            per = a.size // (nc * (num_slices if name.startswith(("kdata", "idata", "fm")) else 1))
            write_v02(d / f"{name}.dat", a, per, num_coil, num_slices)
        else:
            cn = nc if name.startswith(("kdata", "sensi")) else None
            write_v10(d / f"{name}.dat", a, nx, ny, nz, cn, num_slices)


def read_dataset(d) -> dict:
    """Mirror of loadInputData (kernels/structures.cpp:569-780)."""
    d = Path(d)
    v02 = struct.unpack("<f", (d / "kx.dat").read_bytes()[:4])[0] == np.float32(0.2)
    out = dict(num_coil=1, num_slices=1, nx=0, ny=0, nz=0)
    per = {}
    for name in FILES:
        h, a = read_file(d / f"{name}.dat", v02)
        per[name] = h.get("per_coil", a.size)
        if "coil_number" in h:
            out["num_coil"] = h["coil_number"]
        if "slice_number" in h:
            out["num_slices"] = h["slice_number"]
        for k, kk in (("xDimension", "nx"), ("yDimension", "ny"), ("zDimension", "nz")):
            if k in h:
                out[kk] = h[k]
        out[name] = a
        out["version"] = h.get("version")
    out["num_k"], out["num_i"] = per["kx"], per["ix"]
    if out["num_coil"] == 1:
        n = per["sensi_r"]
        out["sensi_r"][:n] = 1.0
        out["sensi_i"][:n] = 0.0
    return out


def write_mtx(fn, rows: int, cols: int, I, J, V) -> None:
    """A sparse real matrix (0-based coordinates) as a Matrix Market coordinate
    file (c.rmtx), the format readMtxFile reads (kernels/mmio.cpp:668-830) and
    matlab_utils/create_sparse_matrix/mmwrite.m writes: 1-based "i j value"
    lines after a "rows cols nnz" line."""
    I, J, V = np.asarray(I), np.asarray(J), np.asarray(V, np.float64)
    with open(fn, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{int(rows)} {int(cols)} {I.size}\n")
        for i, j, v in zip(I.tolist(), J.tolist(), V.tolist()):
            f.write(f"{i + 1} {j + 1} {v:.17g}\n")


def read_mtx(fn):
    """(rows, cols, I, J, V) of a Matrix Market coordinate file, 0-based
    (pattern entries read as 1.0; complex matrices refused)."""
    with open(fn) as f:
        banner = f.readline().lower()
        if not banner.startswith("%%matrixmarket") or "coordinate" not in banner:
            raise ValueError(f"{fn}: not a Matrix Market coordinate file")
        if "complex" in banner:
            raise ValueError(f"{fn}: complex matrices are not supported")
        pattern = "pattern" in banner
        line = f.readline()
        while line.startswith("%") or not line.strip():
            line = f.readline()
        rows, cols, nnz = (int(x) for x in line.split()[:3])
        body = np.loadtxt(f, ndmin=2) if nnz else np.zeros((0, 2 if pattern else 3))
    I = body[:, 0].astype(np.int64) - 1
    J = body[:, 1].astype(np.int64) - 1
    V = np.ones(nnz) if pattern else body[:, 2]
    return rows, cols, I, J, V
