"""Solution output: VTK unstructured-grid files of the nodal fields and raw
restart checkpoints (off the hot path).

`write_vtu` follows the reference's `writemesh` (examples/2d_kernels/vtk.jl,
examples/3d_kernels/vtk.jl): every element is split into (Nq-1)^dim linear
sub-cells over its LGL nodes — VTK_PIXEL in 2-D, VTK_VOXEL in 3-D, corner
nodes in column-major order — and the points are all nodes in element order,
with the fields as point data.  The file is VTK XML (.vtu) with the arrays
appended as raw little-endian binary, uncompressed, as WriteVTK writes with
compress=false.

`save_checkpoint` / `load_checkpoint` store the state of a run between LSRK
steps: the 2N-storage carry is zero at a step boundary (it is scaled by
RKA[0] = 0 after the fifth stage), so the state Q, the step count and the
time are the whole restart record.
"""
from __future__ import annotations

import struct

import numpy as np

VTK_PIXEL, VTK_VOXEL = 8, 11


def subcells(dim: int, N: int, nelem: int) -> np.ndarray:
    """0-based point ids of the linear sub-cells, (nelem * N^dim, 2^dim)."""
    Nq = N + 1
    Np = Nq ** dim
    ind = np.arange(Np).reshape((Nq,) * dim, order="F")
    local = []
    if dim == 2:
        for j in range(N):
            for i in range(N):
                local.append(ind[i:i + 2, j:j + 2].ravel(order="F"))
    elif dim == 3:
        for k in range(N):
            for j in range(N):
                for i in range(N):
                    local.append(ind[i:i + 2, j:j + 2, k:k + 2].ravel(order="F"))
    else:
        raise ValueError("dim must be 2 or 3")
    local = np.array(local, dtype=np.int64)  # (N^dim, 2^dim)
    offs = (np.arange(nelem, dtype=np.int64) * Np)[:, None, None]
    return (local[None, :, :] + offs).reshape(-1, 2 ** dim)


def write_vtu(path: str, dim: int, N: int, coords, fields=()) -> str:
    """Write the nodal fields of one mesh to `path` (".vtu" is appended when
    missing).  coords: dim arrays (Np, nelem) of node coordinates; fields:
    (name, (Np, nelem) array) pairs.  Returns the file name."""
    if not path.endswith(".vtu"):
        path = path + ".vtu"
    X = [np.asarray(c, dtype=np.float64) for c in coords]
    Np, nelem = X[0].shape
    assert Np == (N + 1) ** dim and len(X) == dim
    npts = Np * nelem
    pts = np.zeros((npts, 3), dtype=np.float64)
    for c in range(dim):
        pts[:, c] = X[c].ravel(order="F")
    conn = subcells(dim, N, nelem)
    ncell = conn.shape[0]
    offsets = (np.arange(1, ncell + 1, dtype=np.int64) * conn.shape[1])
    types = np.full(ncell, VTK_PIXEL if dim == 2 else VTK_VOXEL, dtype=np.uint8)
    arrays, head, pos = [], [], 0

    def add(a: np.ndarray):
        nonlocal pos
        raw = np.ascontiguousarray(a).tobytes()
        arrays.append(struct.pack("<Q", len(raw)) + raw)
        off = pos
        pos += 8 + len(raw)
        return off

    pdata = []
    for name, v in fields:
        v = np.asarray(v, dtype=np.float64)
        assert v.shape == (Np, nelem), name
        pdata.append((name, add(v.ravel(order="F"))))
    p_off = add(pts)
    c_off, o_off, t_off = add(conn.astype(np.int64)), add(offsets), add(types)
    head.append('<?xml version="1.0"?>')
    head.append('<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" header_type="UInt64">')
    head.append('<UnstructuredGrid>')
    head.append(f'<Piece NumberOfPoints="{npts}" NumberOfCells="{ncell}">')
    head.append('<PointData>')
    for name, off in pdata:
        head.append(f'<DataArray type="Float64" Name="{name}" format="appended" offset="{off}"/>')
    head.append('</PointData>')
    head.append('<Points>')
    head.append(f'<DataArray type="Float64" NumberOfComponents="3" format="appended" offset="{p_off}"/>')
    head.append('</Points>')
    head.append('<Cells>')
    head.append(f'<DataArray type="Int64" Name="connectivity" format="appended" offset="{c_off}"/>')
    head.append(f'<DataArray type="Int64" Name="offsets" format="appended" offset="{o_off}"/>')
    head.append(f'<DataArray type="UInt8" Name="types" format="appended" offset="{t_off}"/>')
    head.append('</Cells>')
    head.append('</Piece>')
    head.append('</UnstructuredGrid>')
    head.append('<AppendedData encoding="raw">')
    with open(path, "wb") as fh:
        fh.write(("\n".join(head) + "\n_").encode())
        for a in arrays:
            fh.write(a)
        fh.write(b"\n</AppendedData>\n</VTKFile>\n")
    return path


def read_vtu(path: str) -> dict:
    """Arrays of a file written by write_vtu: {"points", "connectivity",
    "offsets", "types", <field names>} (for checking the files)."""
    import xml.etree.ElementTree as ET
    data = open(path, "rb").read()
    start = data.index(b'<AppendedData encoding="raw">')
    root = ET.fromstring(data[:start].decode() + "</VTKFile>")
    blob = data[data.index(b"_", start) + 1:]
    dtypes = {"Float64": np.float64, "Int64": np.int64, "UInt8": np.uint8}
    out = {}
    piece = root.find("UnstructuredGrid/Piece")
    out["n_points"] = int(piece.get("NumberOfPoints"))
    out["n_cells"] = int(piece.get("NumberOfCells"))
    for da in root.iter("DataArray"):
        off = int(da.get("offset"))
        n = struct.unpack("<Q", blob[off:off + 8])[0]
        a = np.frombuffer(blob[off + 8:off + 8 + n], dtype=dtypes[da.get("type")])
        name = da.get("Name") or "points"
        out[name] = a.reshape(-1, 3) if name == "points" else a
    return out


def save_checkpoint(path: str, Q: np.ndarray, step: int, t: float, dt: float, **meta) -> str:
    """Restart record of a run between LSRK steps: the full FP64 state
    (Np, nstate, nelem), the step count, the time and dt, plus any scalar
    metadata (dim, N, mesh parameters ...).  Returns the file name (.npz)."""
    if not path.endswith(".npz"):
        path = path + ".npz"
    np.savez(path, Q=np.asarray(Q, dtype=np.float64), step=np.int64(step), t=np.float64(t),
             dt=np.float64(dt), **{k: np.asarray(v) for k, v in meta.items()})
    return path


def load_checkpoint(path: str) -> dict:
    """Inverse of save_checkpoint: {"Q", "step", "t", "dt", <metadata>}."""
    with np.load(path) as z:
        out = {k: z[k] for k in z.files}
    out["Q"] = np.asfortranarray(out["Q"])
    out["step"], out["t"], out["dt"] = int(out["step"]), float(out["t"]), float(out["dt"])
    return out
