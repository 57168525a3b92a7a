"""Headless output of a run: a VTK unstructured grid of the leaf cells
(``a$D_write_vtk``, afivo/src/m_aX_io.f90:20-207, with the file layout of
afivo/src/m_vtk.f90) and the axis profile of the cylindrical diagnostics.

The reference's other output route, Silo, depends on a library that is not
available here; the VTK file is what ParaView and VisIt read directly.

File layout (m_vtk.f90): an XML header with a ``FieldData`` block (TIME as
Float64, CYCLE as Int32, ascii), one ``Piece`` whose Points (Float32 x 3),
connectivity, offsets and types (Int32) and CellData arrays (Float64) are
all ``format="appended"``; the appended section starts after ``_`` and
holds every array as a 4-byte byte count followed by its raw little-endian
values, in the order the arrays are declared. Cells are VTK pixels (type 8)
with nodes (i, j), (i+1, j), (i, j+1), (i+1, j+1). Boxes are the leaves of
levels 1..max_lvl in level-list order, cells i-fastest within a box.
"""
from __future__ import annotations

import struct
from typing import Dict, Optional, Sequence

import numpy as np

VTK_PIXEL = 8
# output names of the cell variables (src/m_streamer.f90:17-43 order) and the
# set the streamer programs write by default
CC_NAMES = ["e", "i", "e_old", "i_old", "phi", "fld", "rhs", "pho", "eps"]
DEFAULT_NAMES = ["e", "i", "phi", "fld", "rhs", "pho", "eps"]


def leaf_mesh(meta: np.ndarray, geom: np.ndarray, levels) -> Dict[str, np.ndarray]:
    """Nodes, pixel connectivity and (box id, cell slot index) of every leaf
    cell, in the order a$D_write_vtk writes them."""
    boxes = [int(i) for lvl in sorted(levels) if lvl >= 1 for i in levels[lvl][1]]
    if not boxes:
        raise ValueError("the tree has no leaves on levels >= 1")
    nc = int(meta[boxes[0], 14])
    bn = nc + 1
    ii, jj = np.meshgrid(np.arange(bn), np.arange(bn), indexing="xy")  # j slow, i fast
    ci, cj = np.meshgrid(np.arange(1, nc + 1), np.arange(1, nc + 1), indexing="xy")
    coords, conn, ids, slots = [], [], [], []
    for g, bid in enumerate(boxes):
        if int(meta[bid, 14]) != nc:
            raise ValueError("leaf boxes of different sizes")
        r0, r1, dr = geom[bid, 0], geom[bid, 1], geom[bid, 3]
        coords.append(np.stack([r0 + ii.ravel() * dr, r1 + jj.ravel() * dr], axis=1))
        node0 = g * bn * bn
        n_ix = node0 + (cj.ravel() - 1) * bn + (ci.ravel() - 1)
        conn.append(np.stack([n_ix, n_ix + 1, n_ix + bn, n_ix + bn + 1], axis=1))
        ids.append(np.full(nc * nc, bid))
        slots.append(ci.ravel() + (nc + 2) * cj.ravel())
    return {"coords": np.concatenate(coords), "connects": np.concatenate(conn).astype(np.int32),
            "box": np.concatenate(ids), "slot": np.concatenate(slots), "nc": nc, "n_boxes": len(boxes)}


def cell_values(mesh, cc: np.ndarray) -> np.ndarray:
    """Values of one downloaded cell variable (one (nc+2)^2 slot per box id)
    at the mesh's leaf cells."""
    return np.asarray(cc)[mesh["box"], mesh["slot"]]


def face_means(mesh, fx: np.ndarray, fy: np.ndarray):
    """Cell averages of a face variable: 0.5 (fx(i) + fx(i+1)) and
    0.5 (fy(j) + fy(j+1)) (a$D_write_vtk's fc_names output)."""
    nc = mesh["nc"]
    s = mesh["slot"]
    i, j = s % (nc + 2), s // (nc + 2)
    b = mesh["box"]
    xi = (i - 1) + (nc + 1) * (j - 1)
    yi = (i - 1) + nc * (j - 1)
    fxa, fya = np.asarray(fx), np.asarray(fy)
    return 0.5 * (fxa[b, xi] + fxa[b, xi + 1]), 0.5 * (fya[b, yi] + fya[b, yi + nc])


def write_vtk(filename: str, meta: np.ndarray, geom: np.ndarray, levels,
              cell_data: Dict[str, np.ndarray], time: float = 0.0, n_cycle: int = 0) -> str:
    """Write the leaf cells and ``cell_data`` (name -> values per leaf cell in
    ``leaf_mesh`` order, or a downloaded (max_id+1, (nc+2)^2) variable) to
    ``filename`` (".vtu" appended when missing). Returns the path."""
    mesh = leaf_mesh(meta, geom, levels)
    n_cells = len(mesh["box"])
    n_nodes = len(mesh["coords"])
    if not filename.endswith(".vtu"):
        filename += ".vtu"
    arrays = []  # (xml attributes, raw bytes) in declaration order
    pts = np.zeros((n_nodes, 3), dtype="<f4")
    pts[:, :2] = mesh["coords"]
    header = ['<?xml version="1.0"?>',
              '<VTKFile type="UnstructuredGrid" version="0.1" byte_order="LittleEndian">',
              '  <UnstructuredGrid>', '    <FieldData>',
              '      <DataArray type="Float64" Name="TIME" NumberOfTuples="1" format="ascii">',
              f"        {time!r}", "      </DataArray>",
              '      <DataArray type="Int32" Name="CYCLE" NumberOfTuples="1" format="ascii">',
              f"        {int(n_cycle)}", "      </DataArray>", "    </FieldData>",
              f'    <Piece NumberOfPoints="{n_nodes}" NumberOfCells="{n_cells}">']
    offset = 0

    def decl(indent, attrs, raw):
        nonlocal offset
        header.append(" " * indent + f'<DataArray {attrs} format="appended" offset="{offset}"/>')
        arrays.append(raw)
        offset += 4 + len(raw)

    header.append("      <Points>")
    decl(8, 'type="Float32" NumberOfComponents="3" Name="Points"', pts.tobytes())
    header.append("      </Points>")
    header.append("      <Cells>")
    decl(8, 'type="Int32" Name="connectivity"', mesh["connects"].astype("<i4").tobytes())
    decl(8, 'type="Int32" Name="offsets"', (4 * np.arange(1, n_cells + 1)).astype("<i4").tobytes())
    decl(8, 'type="Int32" Name="types"', np.full(n_cells, VTK_PIXEL, dtype="<i4").tobytes())
    header.append("      </Cells>")
    header.append("      <CellData>")
    for name, v in cell_data.items():
        v = np.asarray(v, dtype=np.float64)
        if v.ndim == 2:
            v = cell_values(mesh, v)
        if v.shape != (n_cells,):
            raise ValueError(f"cell data {name!r}: {v.shape} values for {n_cells} cells")
        decl(8, f'type="Float64" Name="{name}"', v.astype("<f8").tobytes())
    header.append("      </CellData>")
    header.append("    </Piece>")
    header.append("  </UnstructuredGrid>")
    header.append('  <AppendedData encoding="raw">')
    with open(filename, "wb") as fh:
        fh.write(("\n".join(header) + "\n_").encode())
        for raw in arrays:
            fh.write(struct.pack("<i", len(raw)))
            fh.write(raw)
        fh.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return filename


def read_vtk(filename: str) -> Dict[str, np.ndarray]:
    """Read back a file written by :func:`write_vtk` (the arrays by name,
    plus TIME and CYCLE)."""
    import re
    data = open(filename, "rb").read()
    start = data.index(b"<AppendedData")
    start = data.index(b"_", start) + 1
    head = data[:start].decode()
    out: Dict[str, np.ndarray] = {}
    m = re.search(r'Name="TIME"[^>]*>\s*([^<\s]+)', head)
    out["TIME"] = np.array([float(m.group(1))])
    m = re.search(r'Name="CYCLE"[^>]*>\s*([^<\s]+)', head)
    out["CYCLE"] = np.array([int(m.group(1))])
    dt = {"Float32": "<f4", "Float64": "<f8", "Int32": "<i4"}
    for m in re.finditer(r'<DataArray type="(\w+)"(?: NumberOfComponents="(\d+)")? Name="([^"]+)" '
                         r'format="appended" offset="(\d+)"/>', head):
        typ, comps, name, off = m.group(1), m.group(2), m.group(3), int(m.group(4))
        n = struct.unpack_from("<i", data, start + off)[0]
        arr = np.frombuffer(data, dtype=dt[typ], count=n // np.dtype(dt[typ]).itemsize,
                            offset=start + off + 4)
        out[name] = arr.reshape(-1, int(comps)) if comps else arr
    return out


def write_run(filename: str, sim, names: Optional[Sequence[str]] = None, n_cycle: int = 0) -> str:
    """Write a :class:`Simulation`'s leaf cells with the streamer variables
    (electron and ion density, potential, |E|, space charge, photoionization,
    eps) and the cell-averaged electron flux and field, as the streamer
    programs do with their output variable names."""
    meta, geom, levels = sim.tree.export()
    return write_state(filename, meta, geom, levels, sim.device.cc, sim.device.fc, sim.time,
                       names, n_cycle)


def write_state(filename: str, meta, geom, levels, cc, fc, time: float,
                names: Optional[Sequence[str]] = None, n_cycle: int = 0) -> str:
    """``write_run`` from any source of a run's state: cc(iv) and fc(dim, f)
    give variables in the download layout (a device run, or a checkpoint read
    on the host)."""
    names = list(names) if names is not None else list(DEFAULT_NAMES)
    mesh = leaf_mesh(meta, geom, levels)
    data = {n: cell_values(mesh, cc(CC_NAMES.index(n))) for n in names}
    fx, fy = face_means(mesh, fc(0, 0), fc(1, 0))
    data["flux_x"], data["flux_y"] = fx, fy
    return write_vtk(filename, meta, geom, levels, data, time=time, n_cycle=n_cycle)


def axis_profile(fld: np.ndarray, dens: np.ndarray, meta, geom, levels, cfg):
    """Leaf cells along the symmetry line sorted by z (metrics.line_cells):
    (z, |E|, electron density), the axis diagnostics of the cylindrical
    program (src/streamer_cyl.f90:647-956 writes such profiles)."""
    from .metrics import line_cells
    ids, cells, zs = line_cells(meta, geom, levels, cfg)
    order = np.argsort(zs, kind="stable")
    return zs[order], np.asarray(fld)[ids, cells][order], np.asarray(dens)[ids, cells][order]
