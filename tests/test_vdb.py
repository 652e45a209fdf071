"""OpenVDB .vdb sim grids: nm_vdb_active_voxels (host only) over files from the test-side
writer (tests/vdb_files.py) in each of the forms the reader takes, and its refusals.

Parity: no OpenVDB library or reference .vdb file exists here, so the files follow the
writer's reading of the published layout (OpenVDB io/Archive, tree nodes' readTopology);
the reader is pinned to that, not to OpenVDB itself.
"""
import numpy as np
import pytest

from nanomap_b200 import _native as N
from nanomap_b200 import api as A
from tests.vdb_files import ACTIVE_MASK, BLOSC, ZIP, write_vdb


def _voxels(seed=3, n=4000):
    """Scattered voxels, a fully active 8^3 block (a tile when collapsed), voxels across the
    origin (negative coordinates) and far apart (several root children)."""
    rng = np.random.default_rng(seed)
    v = [rng.integers(-300, 300, (n, 3))]
    b = np.stack(np.meshgrid(*[np.arange(16, 24)] * 3, indexing="ij"), -1).reshape(-1, 3)
    v.append(b)
    v.append(np.array([[5000, -7000, 12], [-4097, 4096, -1]]))
    return np.unique(np.concatenate(v), axis=0).astype(np.int32)


def _sorted(a):
    a = np.asarray(a, np.int64)
    return a[np.lexsort((a[:, 2], a[:, 1], a[:, 0]))]


@pytest.mark.parametrize("compression,codes,half,zip_real", [
    (0, (0,), False, False),
    (ACTIVE_MASK, (0, 1, 2, 3, 4, 5, 6), False, False),
    (ZIP | ACTIVE_MASK, (0,), False, True),
    (ZIP | ACTIVE_MASK, (6, 3, 5), True, True),
    (ZIP, (0, 2), False, False),
    (BLOSC | ACTIVE_MASK, (0, 4, 6), False, False),
    (BLOSC | ACTIVE_MASK, (1,), True, False),
])
@pytest.mark.parametrize("collapse", [False, True])
def test_active_voxels_every_storage_form(tmp_path, compression, codes, half, zip_real, collapse):
    v = _voxels()
    p = write_vdb(tmp_path / "g.vdb", v, res=0.05, compression=compression, codes=codes,
                  half=half, zip_real=zip_real, collapse=collapse,
                  root_tiles=[(8192, 0, 0, 0)])
    vs, tr, got = A.vdb_active_voxels(p)
    assert np.allclose(vs, 0.05) and np.allclose(tr, 0.0)
    assert np.array_equal(_sorted(got), _sorted(v))


@pytest.mark.parametrize("transform,tr", [("UniformScaleTranslateMap", (0.3, -0.2, 1.0)),
                                          ("AffineMap", (0.5, 0.0, -0.1))])
def test_transforms(tmp_path, transform, tr):
    v = _voxels(n=50)
    p = write_vdb(tmp_path / "g.vdb", v, res=0.1, transform=transform, translation=tr)
    vs, t, got = A.vdb_active_voxels(p)
    assert np.allclose(vs, 0.1) and np.allclose(t, tr)
    assert np.array_equal(_sorted(got), _sorted(v))


def test_grid_selection(tmp_path):
    """The grid named "grid" (as SimManager::loadGridFromFile), a named one, else the first."""
    v = _voxels(n=30)
    p = write_vdb(tmp_path / "two.vdb", v, grids=("density", "grid"))
    assert len(A.vdb_active_voxels(p)[2]) == len(v)
    assert len(A.vdb_active_voxels(p, "density")[2]) == len(v)
    q = write_vdb(tmp_path / "first.vdb", v, grids=("surface",))
    assert len(A.vdb_active_voxels(q)[2]) == len(v)
    with pytest.raises(N.NanomapError) as e:
        A.vdb_active_voxels(q, "grid")
    assert e.value.code == N.NM_ERR_ARG


@pytest.mark.parametrize("compression,half", [(0, False), (ZIP | ACTIVE_MASK, False),
                                              (ACTIVE_MASK, True)])
def test_double_grids(tmp_path, compression, half):
    v = _voxels(n=200)
    p = write_vdb(tmp_path / "d.vdb", v, value_type="double", compression=compression, half=half,
                  codes=(0, 5, 6), collapse=True, root_tiles=[(-8192, 0, 0, 0)])
    assert np.array_equal(_sorted(A.vdb_active_voxels(p)[2]), _sorted(v))


def test_empty_grid(tmp_path):
    e = write_vdb(tmp_path / "e.vdb", np.zeros((0, 3), np.int32))
    assert len(A.vdb_active_voxels(e)[2]) == 0


def test_refusals(tmp_path):
    v = _voxels(n=20)
    cases = {
        "version": (dict(version=220), N.NM_ERR_UNSUPPORTED),
        "bool tree": (dict(value_type="bool"), N.NM_ERR_UNSUPPORTED),
        "rotation": (dict(transform="RotatedAffineMap"), N.NM_ERR_UNSUPPORTED),
        "frustum": (dict(transform="NonlinearFrustumMap"), N.NM_ERR_UNSUPPORTED),
    }
    for name, (kw, code) in cases.items():
        p = write_vdb(tmp_path / f"{name}.vdb", v, **kw)
        with pytest.raises(N.NanomapError) as e:
            A.vdb_active_voxels(p)
        assert e.value.code == code, name
    p = write_vdb(tmp_path / "ok.vdb", v)
    raw = p.read_bytes()
    (tmp_path / "short.vdb").write_bytes(raw[: len(raw) // 2])
    (tmp_path / "magic.vdb").write_bytes(b"\0" * 8 + raw[8:])
    for name in ("short", "magic"):
        with pytest.raises(N.NanomapError) as e:
            A.vdb_active_voxels(tmp_path / f"{name}.vdb")
        assert e.value.code == N.NM_ERR_IO, name
    # an active root tile (4096^3 voxels) is beyond the reader's 2^28-voxel list
    with pytest.raises(N.NanomapError) as e:
        A.vdb_active_voxels(write_vdb(tmp_path / "tile.vdb", v, root_tiles=[(8192, 0, 0, 1)]))
    assert e.value.code == N.NM_ERR_CAPACITY
    with pytest.raises(N.NanomapError) as e:
        A.vdb_active_voxels(p, "nope")
    assert e.value.code == N.NM_ERR_ARG
    # room for fewer voxels than the grid holds
    import ctypes as C
    cnt = C.c_int64()
    buf = np.zeros((5, 3), np.int32)
    rc = N.lib().nm_vdb_active_voxels(str(p).encode(), None, None, None,
                                      buf.ctypes.data_as(N._PI32), 5, C.byref(cnt))
    assert rc == N.NM_ERR_CAPACITY and cnt.value == len(v)


@pytest.mark.parametrize("n", [0, 1, 3000])
def test_writer_round_trip(tmp_path, n):
    """nm_vdb_write_active_voxels (the caves' .vdb output) read back by nm_vdb_active_voxels."""
    v = _voxels(seed=9, n=n)[:n] if n else np.zeros((0, 3), np.int32)
    p = tmp_path / "w.vdb"
    A.vdb_write_active_voxels(p, v, 0.05)
    vs, tr, got = A.vdb_active_voxels(p)
    assert np.allclose(vs, 0.05) and np.allclose(tr, 0.0)
    assert np.array_equal(_sorted(got), _sorted(np.unique(v, axis=0)))
    A.vdb_write_active_voxels(tmp_path / "named.vdb", v, 0.05, grid="cave")
    assert len(A.vdb_active_voxels(tmp_path / "named.vdb", "cave")[2]) == len(np.unique(v, axis=0))


def test_corrupted_files_end_in_an_error_or_a_voxel_set(tmp_path):
    """Bytes overwritten or the file cut short at seeded places: every read returns a status
    (no crash, no out-of-bounds write); the voxel lists that come back fit the array."""
    rng = np.random.default_rng(21)
    v = _voxels(seed=4, n=500)
    raw = write_vdb(tmp_path / "base.vdb", v, compression=ZIP | ACTIVE_MASK, codes=(0, 3, 5, 6),
                    collapse=True, root_tiles=[(8192, 0, 0, 0)]).read_bytes()
    p = tmp_path / "m.vdb"
    for k in range(300):
        b = bytearray(raw)
        if k % 2:
            b = b[: int(rng.integers(0, len(b)))]
        else:
            for _ in range(int(rng.integers(1, 6))):
                b[int(rng.integers(0, len(b)))] = int(rng.integers(0, 256))
        p.write_bytes(bytes(b))
        try:
            vs, tr, got = A.vdb_active_voxels(p)
            assert got.ndim == 2 and got.shape[1] == 3
        except N.NanomapError as e:
            assert e.code in (N.NM_ERR_IO, N.NM_ERR_UNSUPPORTED, N.NM_ERR_ARG, N.NM_ERR_CAPACITY)


def test_writer_refusals(tmp_path):
    v = np.array([[0, 0, 0]], np.int32)
    for size in (0.0, -0.1, float("nan"), float("inf")):
        with pytest.raises(N.NanomapError) as e:
            A.vdb_write_active_voxels(tmp_path / "x.vdb", v, size)
        assert e.value.code == N.NM_ERR_ARG, size
    with pytest.raises(N.NanomapError) as e:
        A.vdb_write_active_voxels(tmp_path / "missing_dir" / "x.vdb", v, 0.1)
    assert e.value.code == N.NM_ERR_IO
