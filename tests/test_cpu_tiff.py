"""Segmented TIFF stacks (reference domain_geometry = 3d_image, keys of
cfg/3d_image/domain.cfg): files written here by a small baseline-TIFF
writer (TIFF 6.0: header, one image file directory per page, strips) in both
byte orders, 1/8/16 bits, uncompressed and PackBits, one or many pages per
file; read back through fe_geom_tiff_stack and checked voxel for voxel,
with the sub-volume cut and the coarsening rule (solid when at least half of
the fine voxels are) restated in numpy."""
import struct

import numpy as np
import pytest

from felbm_gpu_b200 import geometry
from felbm_gpu_b200._capi import FeError


def _packbits(data: bytes) -> bytes:
    out, i = bytearray(), 0
    while i < len(data):
        j = i
        while j + 1 < len(data) and data[j + 1] == data[i] and j - i < 127:
            j += 1
        if j > i:                                   # a run of j - i + 1 equal bytes
            out += struct.pack("b", -(j - i)) + data[i:i + 1]
            i = j + 1
        else:                                       # literals up to the next run
            k = i
            while k < len(data) and k - i < 128 and not (k + 1 < len(data) and data[k + 1] == data[k]):
                k += 1
            k = max(k, i + 1)
            out += struct.pack("b", k - i - 1) + data[i:k]
            i = k
    return bytes(out)


def write_tiff(path, pages, bits=8, big=False, packbits=False, rows_per_strip=3):
    """pages: list of 2-D uint arrays (h, w)."""
    e = ">" if big else "<"
    body = bytearray(b"MM" if big else b"II") + struct.pack(e + "HI", 42, 0)
    prev = 4                                        # where the next IFD offset goes
    for img in pages:
        h, w = img.shape
        strips = []
        for y0 in range(0, h, rows_per_strip):
            rows = img[y0:y0 + rows_per_strip]
            if bits == 1:
                raw = np.packbits(rows.astype(np.uint8) != 0, axis=1).tobytes()
            elif bits == 8:
                raw = rows.astype(np.uint8).tobytes()
            else:
                raw = rows.astype(e + "u2").tobytes()
            if packbits:
                raw = _packbits(raw)
            strips.append(raw)
        offs, counts = [], []
        for s in strips:
            offs.append(len(body))
            counts.append(len(s))
            body += s
        if len(body) % 2:
            body += b"\0"

        def arr(vals):
            nonlocal body
            at = len(body)
            body += struct.pack(e + "%dI" % len(vals), *vals)
            return at
        so = arr(offs) if len(offs) > 1 else None
        sc = arr(counts) if len(counts) > 1 else None
        entries = [(256, 4, 1, w), (257, 4, 1, h), (258, 3, 1, bits), (259, 3, 1, 32773 if packbits else 1),
                   (262, 3, 1, 1), (273, 4, len(offs), so if so is not None else offs[0]), (277, 3, 1, 1),
                   (278, 4, 1, rows_per_strip), (279, 4, len(counts), sc if sc is not None else counts[0])]
        ifd = len(body)
        body[prev:prev + 4] = struct.pack(e + "I", ifd)
        body += struct.pack(e + "H", len(entries))
        for tag, typ, cnt, val in entries:
            if typ == 3 and cnt == 1:
                body += struct.pack(e + "HHIHH", tag, typ, cnt, val, 0)
            else:
                body += struct.pack(e + "HHII", tag, typ, cnt, val)
        prev = len(body)
        body += struct.pack(e + "I", 0)
    open(path, "wb").write(bytes(body))


def _coarsen(m, levels):
    for _ in range(levels):
        f = [2 if n > 1 else 1 for n in m.shape]
        c = [n // k for n, k in zip(m.shape, f)]
        m = m[:c[0] * f[0], :c[1] * f[1], :c[2] * f[2]]
        s = m.reshape(c[0], f[0], c[1], f[1], c[2], f[2]).sum(axis=(1, 3, 5))
        m = (2 * s >= f[0] * f[1] * f[2]).astype(np.uint8)
    return m


@pytest.mark.parametrize("bits,big,packbits", [(8, False, False), (8, True, True), (16, True, False),
                                                (16, False, True), (1, False, False), (1, True, True)])
def test_stack_round_trip(tmp_path, bits, big, packbits):
    rng = np.random.default_rng(bits + 2 * big + 4 * packbits)
    vol = (rng.random((7, 13, 19)) < 0.4).astype(np.uint16) * (255 if bits == 8 else (1 if bits == 1 else 4000))
    vol[2, 3:9, :] = vol[2, 3, 0]                   # runs for PackBits
    write_tiff(tmp_path / "a.tif", list(vol[:3]), bits, big, packbits)
    write_tiff(tmp_path / "b.tif", list(vol[3:]), bits, big, packbits, rows_per_strip=13)
    got = geometry.tiff_stack(str(tmp_path))
    assert got.shape == vol.shape and np.array_equal(got, (vol != 0).astype(np.uint8))
    inv = geometry.tiff_stack(str(tmp_path), invert=True)
    assert np.array_equal(inv, (vol == 0).astype(np.uint8))
    zero = geometry.tiff_stack([tmp_path / "a.tif", tmp_path / "b.tif"], solid_nonzero=False)
    assert np.array_equal(zero, inv)


def test_subvolume_and_coarsening(tmp_path):
    rng = np.random.default_rng(5)
    vol = (rng.random((20, 18, 23)) < 0.5).astype(np.uint8)
    for z in range(vol.shape[0]):
        write_tiff(tmp_path / ("s%03d.tif" % z), [vol[z]])
    full = geometry.tiff_stack(str(tmp_path))
    assert np.array_equal(full, vol)
    sub = geometry.tiff_stack(str(tmp_path), subvolume=(3, 2, 1, 17, 15, 18))
    assert np.array_equal(sub, vol[1:19, 2:17, 3:20])
    for lv in (1, 2):
        c = geometry.tiff_stack(str(tmp_path), coarsening_levels=lv, subvolume=(3, 2, 1, 17, 15, 18))
        assert np.array_equal(c, _coarsen(vol[1:19, 2:17, 3:20], lv)), lv
    one = vol[:1]
    write_tiff(tmp_path / "plane.tif", [one[0]])
    c2 = geometry.tiff_stack([tmp_path / "plane.tif"], coarsening_levels=1)
    assert c2.shape == (1, 9, 11) and np.array_equal(c2, _coarsen(one, 1))


def test_rejected_inputs(tmp_path):
    p = tmp_path / "x.tif"
    open(p, "wb").write(b"II*\0" + b"\0" * 4)
    with pytest.raises(FeError):
        geometry.tiff_stack([p])                    # no page
    write_tiff(p, [np.ones((4, 5), np.uint8)])
    b = bytearray(open(p, "rb").read())
    i = b.find(struct.pack("<HHIHH", 259, 3, 1, 1, 0))
    b[i:i + 12] = struct.pack("<HHIHH", 259, 3, 1, 5, 0)   # LZW
    open(p, "wb").write(bytes(b))
    with pytest.raises(FeError, match="compression"):
        geometry.tiff_stack([p])
    write_tiff(tmp_path / "a.tif", [np.ones((4, 5), np.uint8)])
    write_tiff(tmp_path / "b.tif", [np.ones((4, 6), np.uint8)])
    with pytest.raises(FeError, match="page size"):
        geometry.tiff_stack([tmp_path / "a.tif", tmp_path / "b.tif"])
    with pytest.raises(FeError, match="sub-volume"):
        geometry.tiff_stack([tmp_path / "a.tif"], subvolume=(0, 0, 0, 6, 4, 1))
