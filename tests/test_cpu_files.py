"""HDF5 files without a GPU: geometry and particle files round-trip through
the library's reader, and the bytes follow the HDF5 file-format
specification's structures (checked here by an independent parse: superblock
version 0, end-of-file address, root symbol table with its B-tree, local heap
and symbol-table node, names sorted, version-1 dataset object headers with
dataspace, datatype and contiguous layout messages)."""
import os

import numpy as np

from felbm_gpu_b200 import files, geometry


def test_geometry_round_trip(tmp_path):
    solid = geometry.spheres((10, 12, 14), 2.5, 4, 2.0, 3)
    p = str(tmp_path / "geometry.h5")
    files.write_geometry(p, solid)
    coords = files.read_dataset(p, "coords")
    nodes = geometry.site_nodes(solid)
    nz, ny, nx = solid.shape
    want = np.stack([nodes % nx, (nodes // nx) % ny, nodes // (nx * ny)], axis=1)
    assert coords.dtype == np.int32 and np.array_equal(coords, want)
    assert np.array_equal(files.read_dataset(p, "size"), want.max(axis=0) + 1)


def test_particles_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    n = 37
    pos, vel = rng.random((3, n)), rng.random((3, n))
    ids, dm, pid = np.arange(n) + 5, rng.random(n), np.arange(n, dtype=np.int32) % 2
    p = str(tmp_path / "particles_10.h5")
    files.write_particles(p, pos, vel, ids, dm, pid)
    assert np.array_equal(files.read_dataset(p, "position"), pos.T)
    assert np.array_equal(files.read_dataset(p, "velocity"), vel.T)
    assert np.array_equal(files.read_dataset(p, "id"), ids)
    assert np.array_equal(files.read_dataset(p, "Dm"), dm)
    assert np.array_equal(files.read_dataset(p, "plane_id"), pid)


def _u(b, off, n):
    return int.from_bytes(b[off:off + n], "little")


def test_structure_follows_the_specification(tmp_path):
    p = str(tmp_path / "particles_1.h5")
    files.write_particles(p, np.zeros((3, 4)), None, None, np.ones(4), None)
    b = open(p, "rb").read()
    assert b[:8] == b"\x89HDF\r\n\x1a\n" and b[8] == 0            # superblock version 0
    assert b[13] == 8 and b[14] == 8                               # offsets / lengths
    assert _u(b, 40, 8) == len(b)                                  # end-of-file address
    assert _u(b, 32, 8) == 2 ** 64 - 1 == _u(b, 48, 8)             # undefined addresses
    root, btree, heap = _u(b, 64, 8), _u(b, 80, 8), _u(b, 88, 8)
    assert _u(b, 72, 4) == 1                                       # cached symbol table
    assert b[root] == 1 and _u(b, root + 16, 2) == 0x0011          # v1 header: symbol-table message
    assert (_u(b, root + 24, 8), _u(b, root + 32, 8)) == (btree, heap)
    assert b[heap:heap + 4] == b"HEAP" and b[btree:btree + 4] == b"TREE"
    data = _u(b, heap + 24, 8)
    assert b[data] == 0                                            # offset 0: the empty name
    snod = _u(b, btree + 32, 8)
    assert b[snod:snod + 4] == b"SNOD" and b[snod + 4] == 1
    nsym = _u(b, snod + 6, 2)
    names = []
    for s in range(nsym):
        e = snod + 8 + 40 * s
        off = _u(b, e, 8)
        names.append(b[data + off:b.index(b"\0", data + off)].decode())
        oh = _u(b, e + 8, 8)
        assert b[oh] == 1 and oh % 8 == 0
        types = []
        q = oh + 16
        for _ in range(_u(b, oh + 2, 2)):
            types.append(_u(b, q, 2))
            assert _u(b, q + 2, 2) % 8 == 0
            q += 8 + _u(b, q + 2, 2)
        assert types == [0x0001, 0x0003, 0x0005, 0x0008]
    assert names == sorted(names) == ["Dm", "id", "position"]
    # the key after the child is the last name
    assert _u(b, btree + 40, 8) == _u(b, snod + 8 + 40 * (nsym - 1), 8)
    dm_oh = _u(b, snod + 8 + 8, 8)                                 # "Dm" sorts first
    # datatype of Dm: IEEE little-endian double (class 1, size 8, bias 1023)
    q = dm_oh + 16
    q += 8 + _u(b, q + 2, 2)                                       # skip the dataspace
    assert b[q + 8] & 0x0F == 1 and _u(b, q + 12, 4) == 8 and _u(b, q + 8 + 16, 4) == 1023
    os.remove(p)


def test_reader_rejects_other_files(tmp_path):
    p = str(tmp_path / "x.h5")
    open(p, "wb").write(b"not hdf5" * 40)
    try:
        files.read_dataset(p, "a")
        raise AssertionError("no error")
    except Exception as ex:
        assert "not an HDF5 file" in str(ex)


def test_series_and_stretching_text(tmp_path):
    p = str(tmp_path / "series.txt")
    st = np.array([2.0, -4.0, 6.0, 8.0, 123.5, 0.25])
    files.write_series(p, 0, st, 4, header=True)
    files.write_series(p, 10, st * 2, 4)
    lines = open(p).read().splitlines()
    assert lines[0].split()[1:] == ["iter", "max_speed", "mean_ux", "mean_uy", "mean_uz", "mean_v2",
                                    "total_order_parameter"]
    d = np.loadtxt(p)
    assert np.allclose(d[0], [0, 0.5, 0.5, -1.0, 1.5, 2.0, 123.5])
    assert np.allclose(d[1], [10, np.sqrt(0.5), 1.0, -2.0, 3.0, 4.0, 247.0])
    q = str(tmp_path / "stretching.txt")
    rows = np.array([[1, 0.1, 0.01, 0.001, 50, 0.12, np.nan, 50, 0], [2, 0.2, 0.02, 0.002, 49, 0.3, 0.1, 20, 29]])
    files.write_stretching(q, rows[:1], header=True)
    files.write_stretching(q, rows[1:])
    cols = [l for l in open(q).read().splitlines() if l.startswith("#")][-1].split()[1:]
    assert cols == ["step", "lambda", "mean_log_rho", "var_log_rho", "n_active", "lambda_w", "lambda_nw", "n_w",
                    "n_nw"]
    assert np.allclose(np.loadtxt(q), rows, equal_nan=True)


def test_particles_with_line_elements(tmp_path):
    rng = np.random.default_rng(3)
    pos, rh, lr = rng.random((3, 9)), rng.random((3, 9)), rng.random(9)
    p = str(tmp_path / "particles_5.h5")
    files.write_particles(p, pos, rho_hat=rh, log_rho=lr)
    assert np.array_equal(files.read_dataset(p, "rho_hat"), rh.T)
    assert np.array_equal(files.read_dataset(p, "log_rho"), lr)


def test_deflated_chunk_follows_the_specification(tmp_path):
    """output_deflate: one chunk per dataset through the deflate filter (the
    reference's write_fields_h5 with deflate > 0, felbm_gpu_main.cu:94-98).
    Parsed here independently: layout message version 3, class 2 (chunked)
    with the chunk dimensions and the element size, a version-1 filter
    pipeline message with filter 1 (deflate) and the level as its client
    value, and a type-1 (raw data chunk) B-tree leaf whose one key holds the
    stored size, filter mask 0 and offset 0, pointing at a zlib stream that
    inflates to the data."""
    import zlib
    rng = np.random.default_rng(1)
    arr = np.round(rng.random(5000), 3)               # compressible
    p = str(tmp_path / "output_100.h5")
    files.write_dataset(p, "concentration", arr, deflate=6)
    assert np.array_equal(files.read_dataset(p, "concentration"), arr)
    b = open(p, "rb").read()
    assert _u(b, 40, 8) == len(b) < arr.nbytes               # compressed
    btree = _u(b, 80, 8)
    snod = _u(b, btree + 32, 8)
    oh = _u(b, snod + 8 + 8, 8)
    msgs = {}
    q = oh + 16
    for _ in range(_u(b, oh + 2, 2)):
        msgs[_u(b, q, 2)] = (q + 8, _u(b, q + 2, 2))
        q += 8 + _u(b, q + 2, 2)
    assert sorted(msgs) == [0x0001, 0x0003, 0x0005, 0x0008, 0x000B]
    ly = msgs[0x0008][0]
    assert b[ly] == 3 and b[ly + 1] == 2 and b[ly + 2] == 2   # version 3, chunked, rank + 1
    cbt = _u(b, ly + 3, 8)
    assert _u(b, ly + 11, 4) == 5000 and _u(b, ly + 15, 4) == 8
    fp = msgs[0x000B][0]
    assert b[fp] == 1 and b[fp + 1] == 1                      # version 1, one filter
    assert _u(b, fp + 8, 2) == 1 and _u(b, fp + 14, 2) == 1 and _u(b, fp + 16, 4) == 6
    assert b[cbt:cbt + 4] == b"TREE" and b[cbt + 4] == 1 and b[cbt + 5] == 0 and _u(b, cbt + 6, 2) == 1
    size, mask = _u(b, cbt + 24, 4), _u(b, cbt + 28, 4)
    assert mask == 0 and _u(b, cbt + 32, 8) == 0 and _u(b, cbt + 40, 8) == 0
    chunk = _u(b, cbt + 48, 8)
    got = np.frombuffer(zlib.decompress(b[chunk:chunk + size]), np.float64)
    assert np.array_equal(got, arr)
    # the full node of 2K = 64 children is allocated, as readers expect
    assert chunk >= cbt + 24 + 65 * 24 + 64 * 8
    # level 0 stays contiguous
    q2 = str(tmp_path / "plain.h5")
    files.write_dataset(q2, "x", arr.astype(np.float32), deflate=0)
    assert np.array_equal(files.read_dataset(q2, "x"), arr.astype(np.float32))
