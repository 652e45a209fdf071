"""Test-side writer of OpenVDB .vdb files (format 222-224 layout) for the reader's tests.

It writes the layout that nm_vdb_active_voxels reads -- header, file metadata, grid
descriptors with absolute offsets, per-grid compression flags, grid metadata, transform, tree
topology (root table, 32^3 and 16^3 internal nodes, 8^3 leaves) and the leaf buffers after it --
for a given set of active voxels, with the options a file can take: raw, zip and
blosc-flagged values (blosc chunks in their uncompressed form, a negative byte count), active-
mask compression, each per-node value code, values saved as half, active tiles in place of
fully active blocks, root tiles (x, y, z, active), several grids, scale / scale-translate / affine
transforms.  No OpenVDB library or .vdb file from it exists here, so these files pin the reader
against this writer's reading of the published layout, not against OpenVDB itself.
"""
from __future__ import annotations

import struct
import zlib

import numpy as np

MAGIC = 0x56444220
ZIP, ACTIVE_MASK, BLOSC = 0x1, 0x2, 0x4


def _str(s: str | bytes) -> bytes:
    b = s.encode() if isinstance(s, str) else s
    return struct.pack("<I", len(b)) + b


def _meta(entries) -> bytes:
    """entries: (name, type name, value bytes)."""
    out = struct.pack("<I", len(entries))
    for name, tname, value in entries:
        out += _str(name) + _str(tname) + struct.pack("<I", len(value)) + value
    return out


def _mask(bits: np.ndarray) -> bytes:
    """bits (2^(3 log2dim),) bool -> little-endian 64-bit words, bit n of word n >> 6."""
    w = np.packbits(bits.astype(np.uint8), bitorder="little")
    return w.tobytes()


class _Writer:
    def __init__(self, compression: int, half: bool, codes, zip_real: bool, vt=np.float32):
        self.vt = np.dtype(vt).newbyteorder("<")
        self.compression = compression
        self.half = half
        self.codes = codes  # per-node value code, cycled
        self.k = 0
        self.zip_real = zip_real

    def values(self, vals: np.ndarray, vmask: np.ndarray) -> bytes:
        """Compressed values of one node (float32 vals, bool active mask)."""
        code = self.codes[self.k % len(self.codes)]
        self.k += 1
        out = struct.pack("<b", code)
        if code in (2, 4, 5):
            out += np.array([0.25], self.vt).tobytes()
        if code == 5:
            out += np.array([-0.25], self.vt).tobytes()
        if code in (3, 4, 5):
            sel = np.zeros(len(vmask), bool)
            sel[::3] = True
            out += _mask(sel)
        if (self.compression & ACTIVE_MASK) and code != 6:
            vals = vals[vmask]
        data = vals.astype(np.float16 if self.half else self.vt).tobytes()
        if self.compression & (ZIP | BLOSC):
            z = zlib.compress(data) if (self.compression & ZIP) and self.zip_real else None
            if z is not None and len(z) < len(data):
                out += struct.pack("<q", len(z)) + z
            else:
                out += struct.pack("<q", -len(data)) + data
        else:
            out += data
        return out


def _tree(voxels: np.ndarray, collapse: bool):
    """{root origin: {int4 origin: {leaf origin: 512-bool}}} plus active int4 tiles
    (fully active leaves when collapse)."""
    root: dict = {}
    if len(voxels):
        origins, inv = np.unique(voxels & ~7, axis=0, return_inverse=True)
        bit = ((voxels[:, 0] & 7) << 6) | ((voxels[:, 1] & 7) << 3) | (voxels[:, 2] & 7)
        masks = np.zeros((len(origins), 512), bool)
        masks[inv.reshape(-1), bit] = True
        for (x, y, z), m in zip(origins.tolist(), masks):
            r = (x & ~4095, y & ~4095, z & ~4095)
            i4 = (x & ~127, y & ~127, z & ~127)
            root.setdefault(r, {}).setdefault(i4, {})[(x, y, z)] = m
    tiles = {}
    if collapse:
        for r, n4s in root.items():
            for i4, leaves in n4s.items():
                for lf in [o for o, m in leaves.items() if m.all()]:
                    del leaves[lf]
                    tiles.setdefault(i4, []).append(lf)
    return root, tiles


def _topology(w: _Writer, root, tiles, root_tiles) -> tuple[bytes, list]:
    out = struct.pack("<i", 1)  # buffer count
    out += np.array([0.15], w.vt).tobytes()  # background
    out += struct.pack("<II", len(root_tiles), len(root))
    for x, y, z, active in root_tiles:
        out += struct.pack("<iii", x, y, z) + np.array([0.15], w.vt).tobytes() + struct.pack("<B", active)
    leaves_in_order = []
    for r in sorted(root):
        out += struct.pack("<iii", *r)
        n4s = root[r]
        cm5 = np.zeros(32 ** 3, bool)
        children5 = {}
        for i4 in n4s:
            n = (((i4[0] - r[0]) >> 7) << 10) | (((i4[1] - r[1]) >> 7) << 5) | ((i4[2] - r[2]) >> 7)
            cm5[n] = True
            children5[n] = i4
        out += _mask(cm5) + _mask(np.zeros(32 ** 3, bool))
        out += w.values(np.full(32 ** 3, 0.15, np.float32), np.zeros(32 ** 3, bool))
        for n in sorted(children5):
            i4 = children5[n]
            leaves = n4s[i4]
            cm4 = np.zeros(16 ** 3, bool)
            vm4 = np.zeros(16 ** 3, bool)
            kids = {}
            for lf in leaves:
                m = (((lf[0] - i4[0]) >> 3) << 8) | (((lf[1] - i4[1]) >> 3) << 4) | ((lf[2] - i4[2]) >> 3)
                cm4[m] = True
                kids[m] = lf
            for lf in tiles.get(i4, []):
                m = (((lf[0] - i4[0]) >> 3) << 8) | (((lf[1] - i4[1]) >> 3) << 4) | ((lf[2] - i4[2]) >> 3)
                vm4[m] = True
            vals4 = np.where(vm4, -0.05, 0.15).astype(np.float32)
            out += _mask(cm4) + _mask(vm4) + w.values(vals4, vm4)
            for m in sorted(kids):
                out += _mask(leaves[kids[m]])
                leaves_in_order.append(leaves[kids[m]])
    return out, leaves_in_order


def write_vdb(path, voxels, *, res=0.1, translation=(0.0, 0.0, 0.0), transform="UniformScaleMap",
              compression=ZIP | ACTIVE_MASK, half=False, codes=(0,), zip_real=True, collapse=False,
              root_tiles=(), grids=("grid",), version=224, value_type="float"):
    """Writes `voxels` ((n, 3) int) as the active voxels of every grid named in `grids`."""
    voxels = np.asarray(voxels, np.int64).reshape(-1, 3)
    head = struct.pack("<qI", MAGIC, version) + struct.pack("<II", 11, 0) + struct.pack("<B", 1)
    head += b"0123abcd-0123-4567-89ab-0123456789ab"[:36]
    head += _meta([("creator", "string", b"tests")])
    head += struct.pack("<i", len(grids))
    body = bytearray(head)
    for gi, name in enumerate(grids):
        w = _Writer(compression, half, codes, zip_real,
                    {"float": np.float32, "double": np.float64}.get(value_type, np.float32))
        root, tiles = _tree(voxels, collapse)
        topo, leaves = _topology(w, root, tiles, root_tiles)
        tname = f"Tree_{value_type}_5_4_3" + ("_HalfFloat" if half else "")
        desc = _str(name if gi == 0 or name != grids[0] else name + "\x1e1") + _str(tname) + _str("")
        pos_at = len(body) + len(desc)
        grid_pos = pos_at + 24
        section = struct.pack("<I", compression)
        # grid metadata as files carry it, including a binary entry of a type the reader does
        # not know (skipped by its size)
        section += _meta([("class", "string", b"level set"), ("name", "string", name.encode()),
                          ("file_bbox_min", "vec3i", struct.pack("<iii", 0, 0, 0)),
                          ("file_voxel_count", "int64", struct.pack("<q", len(voxels))),
                          ("file_delayed_load", "__delayedload", bytes(range(37)))])
        s = [res] * 3
        inv = [1.0 / res] * 3
        if transform == "UniformScaleMap":
            section += _str(transform) + struct.pack("<15d", *s, *s, *inv, *[v * v for v in inv],
                                                     *[v / 2 for v in inv])
        elif transform == "UniformScaleTranslateMap":
            section += _str(transform) + struct.pack("<18d", *translation, *s, *s, *inv,
                                                     *[v * v for v in inv], *[v / 2 for v in inv])
        elif transform == "AffineMap":
            m = np.eye(4)
            m[0, 0] = m[1, 1] = m[2, 2] = res
            m[3, :3] = translation
            section += _str(transform) + m.astype("<f8").tobytes()
        elif transform == "RotatedAffineMap":
            m = np.eye(4)
            m[0, 0] = m[1, 1] = m[2, 2] = res
            m[0, 1] = 0.01
            section += _str("AffineMap") + m.astype("<f8").tobytes()
        else:
            section += _str(transform)
        section += topo
        block_pos = grid_pos + len(section)
        buffers = bytearray()
        for mask in leaves:
            buffers += _mask(mask) + w.values(np.where(mask, -0.05, 0.15).astype(np.float32), mask)
        end_pos = block_pos + len(buffers)
        body += desc + struct.pack("<qqq", grid_pos, block_pos, end_pos) + section + buffers
    with open(path, "wb") as f:
        f.write(bytes(body))
    return path
