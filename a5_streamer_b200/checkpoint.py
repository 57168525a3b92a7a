"""Reading run checkpoints without a GPU.

A checkpoint (include/a5t.h a5s_checkpoint_save, `Simulation.checkpoint`)
holds a run's whole state: time, generator state, tree and every cell and
face variable. `read` parses one into host arrays in the formats the rest of
the package uses (`Tree.export`'s meta/geom/levels, `DeviceRun.cc`'s slot
layout), so that a saved run can be inspected or written out as VTK on a
machine with no device: `write_vtk(checkpoint_path, vtk_path)`.

Layout (native byte order, little-endian on every supported host):
u32 magic 'A5CK', u32 version, u64 configuration fingerprint; i32 box_size,
coord, lvls_max, min_lvl, max_lvl, max_id, n_lists, cell slot, face slot,
photoionization; f64 time; i32 rng[4]; per id 0..max_id: i32 in_use, lvl,
ix0, ix1, parent, n_cell, children[4], neighbours[4], f64 dr, r_min0,
r_min1; per list level: i32 n_ids, n_leaves, n_parents and the three lists;
f64 cc[9][max_id + 1][cell slot]; f64 fc[2][2][max_id + 1][face slot].
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

MAGIC, VERSION = 0x4B433541, 1
N_CC, N_FC = 9, 2
_REC = np.dtype([("i", "<i4", 14), ("d", "<f8", 3)])


@dataclass
class Checkpoint:
    box_size: int
    coord: int
    lvls_max: int
    min_lvl: int
    max_lvl: int
    max_id: int
    time: float
    rng: np.ndarray
    photoionization: bool
    fingerprint: int
    meta: np.ndarray                      # (max_id + 1, 16), Tree.export layout
    geom: np.ndarray                      # (max_id + 1, 4)
    levels: Dict[int, Tuple[np.ndarray, np.ndarray, np.ndarray]]
    cc: List[np.ndarray] = field(default_factory=list)   # 9 x (max_id + 1, cell slot)
    fc: List[np.ndarray] = field(default_factory=list)   # [dim * 2 + f] x (max_id + 1, face slot)

    def n_leaf_cells(self) -> int:
        """Leaf cells of the tree (leaves of levels >= 1, box_size^2 each)."""
        return sum(len(self.levels[l][1]) for l in self.levels if l >= 1) * self.box_size ** 2


def read(buf: bytes) -> Checkpoint:
    """Parse a checkpoint buffer; ValueError if it is not one of this layout."""
    if len(buf) < 80:
        raise ValueError("not a checkpoint: too short")
    magic, version, fp = struct.unpack_from("<IIQ", buf, 0)
    if magic != MAGIC:
        raise ValueError("not a checkpoint")
    if version != VERSION:
        raise ValueError(f"checkpoint version {version} not supported")
    (nc, coord, lvls_max, min_lvl, max_lvl, max_id, n_lists, cslot, fslot,
     photoi) = struct.unpack_from("<10i", buf, 16)
    if cslot != (nc + 2) ** 2 or fslot != (nc + 1) * nc or max_id < 1 or n_lists < 1:
        raise ValueError("checkpoint header out of range")
    M = max_id + 1
    need = 80 + _REC.itemsize * M + 8 * M * (N_CC * cslot + 2 * N_FC * fslot)
    if need > len(buf):
        raise ValueError("checkpoint truncated")
    (t,) = struct.unpack_from("<d", buf, 56)
    rng = np.frombuffer(buf, dtype="<i4", count=4, offset=64).astype(np.int32)
    off = 80
    rec = np.frombuffer(buf, dtype=_REC, count=M, offset=off)
    off += _REC.itemsize * M
    used = rec["i"][:, 0] != 0
    used[0] = False
    meta = np.zeros((M, 16), dtype=np.int32)
    geom = np.zeros((M, 4))
    meta[1:, 0] = rec["i"][1:, 0]
    ri = rec["i"][used]
    meta[used, 1:4] = ri[:, 1:4]
    meta[used, 5] = ri[:, 4]
    meta[used, 6:14] = ri[:, 6:14]
    meta[used, 14] = ri[:, 5]
    geom[used, 0:2] = rec["d"][used, 1:3]
    geom[used, 3] = rec["d"][used, 0]
    levels = {}
    for k in range(n_lists):
        if off + 12 > len(buf):
            raise ValueError("checkpoint truncated")
        a, b, c = struct.unpack_from("<3i", buf, off)
        off += 12
        if min(a, b, c) < 0 or off + 4 * (a + b + c) > len(buf):
            raise ValueError("checkpoint level list out of range")
        lst = np.frombuffer(buf, dtype="<i4", count=a + b + c, offset=off).astype(np.int32)
        off += 4 * (a + b + c)
        if min_lvl + k <= max_lvl:
            levels[min_lvl + k] = (lst[:a].copy(), lst[a:a + b].copy(), lst[a + b:].copy())
    if off + 8 * M * (N_CC * cslot + 2 * N_FC * fslot) != len(buf):
        raise ValueError("checkpoint length does not match its header")
    cc, fc = [], []
    for _ in range(N_CC):
        cc.append(np.frombuffer(buf, dtype="<f8", count=M * cslot, offset=off).reshape(M, cslot).copy())
        off += 8 * M * cslot
    for _ in range(2 * N_FC):
        fc.append(np.frombuffer(buf, dtype="<f8", count=M * fslot, offset=off).reshape(M, fslot).copy())
        off += 8 * M * fslot
    return Checkpoint(nc, coord, lvls_max, min_lvl, max_lvl, max_id, t, rng, bool(photoi), fp,
                      meta, geom, levels, cc, fc)


def load(path: str) -> Checkpoint:
    with open(path, "rb") as fh:
        return read(fh.read())


def write_vtk(checkpoint_path: str, filename: str, names: Optional[Sequence[str]] = None,
              n_cycle: int = 0) -> str:
    """The leaf cells of a saved run as VTK, the file output.write_run writes
    for the live run, without a device: the variables named (output.CC_NAMES;
    output.DEFAULT_NAMES by default) and the cell-averaged electron flux."""
    from . import output
    ck = load(checkpoint_path)
    return output.write_state(filename, ck.meta, ck.geom, ck.levels, lambda iv: ck.cc[iv],
                              lambda d, f: ck.fc[d * N_FC + f], ck.time, names, n_cycle)
