"""The reference's file formats through the C ABI (CPU only, no GPU call):
Vaa3D raw stacks (.v3draw), directories of per-Z slices as a tile source,
the slice-file tile sink, and .marker files.

Format (RawFmtMngr.cpp:332-446 reads it, Bigwarp.cpp:660-751 writes it): the
key "raw_image_stack_by_hpeng", an endianness byte, an int16 data type code,
four int32 sizes (x, y, z, channels), the voxels x fastest."""
import os
import struct

import numpy as np
import pytest

from terawarp_b200 import api

KEY = b"raw_image_stack_by_hpeng"


def raw_bytes(arr, endian="<"):
    """A raw stack built by hand from the format description."""
    a = np.asarray(arr)
    if a.ndim == 3:
        a = a[None]
    c, z, y, x = a.shape
    code = a.dtype.itemsize
    hdr = KEY + (b"L" if endian == "<" else b"B") + struct.pack(endian + "h", code) + struct.pack(endian + "4i", x, y, z, c)
    return hdr + a.astype(a.dtype.newbyteorder(endian)).tobytes()


def test_written_header_is_byte_exact(tmp_path):
    vol = np.arange(2 * 3 * 5, dtype=np.uint16).reshape(2, 3, 5)
    p = tmp_path / "a.v3draw"
    api.v3draw_write(p, vol)
    data = p.read_bytes()
    assert data == raw_bytes(vol, "<")
    assert len(data) == 24 + 1 + 2 + 16 + vol.nbytes
    assert api.v3draw_header(p) == ((5, 3, 2, 1), 2)


@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
def test_round_trip_and_multichannel(tmp_path, dtype):
    rng = np.random.default_rng(1)
    vol = rng.integers(0, 200, size=(3, 7, 11, 13)).astype(dtype)  # (c, z, y, x)
    p = tmp_path / "m.v3draw"
    api.v3draw_write(p, vol)
    np.testing.assert_array_equal(api.v3draw_read(p), vol)


def test_big_endian_file_is_read_in_host_order(tmp_path):
    rng = np.random.default_rng(2)
    vol = rng.integers(0, 65535, size=(4, 6, 9)).astype(np.uint16)
    p = tmp_path / "be.v3draw"
    p.write_bytes(raw_bytes(vol, ">"))
    assert api.v3draw_header(p) == ((9, 6, 4, 1), 2)
    np.testing.assert_array_equal(api.v3draw_read(p), vol)
    np.testing.assert_array_equal(api.v3draw_read_box(p, (2, 1, 1), (5, 4, 2)), vol[1:3, 1:5, 2:7])


@pytest.mark.parametrize("box", [((0, 0, 0), (13, 11, 7)), ((3, 2, 1), (4, 5, 3)), ((12, 10, 6), (1, 1, 1)),
                                 ((0, 4, 2), (13, 3, 4))])
def test_box_reads(tmp_path, box):
    rng = np.random.default_rng(3)
    vol = rng.integers(0, 4096, size=(7, 11, 13)).astype(np.uint16)
    p = tmp_path / "b.v3draw"
    p.write_bytes(raw_bytes(vol))
    (x0, y0, z0), (nx, ny, nz) = box
    np.testing.assert_array_equal(api.v3draw_read_box(p, (x0, y0, z0), (nx, ny, nz)),
                                  vol[z0:z0 + nz, y0:y0 + ny, x0:x0 + nx])


def test_malformed_files_are_rejected(tmp_path):
    p = tmp_path / "bad.v3draw"
    p.write_bytes(b"not a raw stack at all, clearly" * 3)
    with pytest.raises(api.TeraWarpError):
        api.v3draw_header(p)
    good = raw_bytes(np.zeros((2, 2, 2), np.uint8))
    (tmp_path / "short.v3draw").write_bytes(good[:-3])  # payload shorter than the header says
    with pytest.raises(api.TeraWarpError):
        api.v3draw_read(tmp_path / "short.v3draw")
    with pytest.raises(api.TeraWarpError):
        api.v3draw_read_box(tmp_path / "short.v3draw", (0, 0, 0), (3, 1, 1))


def make_slice_dir(d, vol, names=None, extras=True):
    os.makedirs(d, exist_ok=True)
    for z in range(vol.shape[0]):
        name = names[z] if names else f"{z * 10:07d}.raw"
        (d / name).write_bytes(raw_bytes(vol[z:z + 1]))
    if extras:  # entries the listing skips (read_2Dtif_dir, dir_make.cpp:175-216)
        (d / "mdata.bin").write_bytes(b"metadata")
        (d / ".iim.format").write_bytes(b"format")


def test_slice_dir_sorted_listing_and_box_reads(tmp_path):
    rng = np.random.default_rng(4)
    vol = rng.integers(0, 4096, size=(12, 20, 33)).astype(np.uint16)
    d = tmp_path / "slices"
    # names sort in z order; created in shuffled order
    names = [f"img_{z:03d}.v3draw" for z in range(12)]
    order = rng.permutation(12)
    os.makedirs(d)
    for z in order:
        (d / names[z]).write_bytes(raw_bytes(vol[z:z + 1]))
    (d / "mdata.bin").write_bytes(b"x")
    with api.SliceDir(d, threads=3) as s:
        assert s.shape == vol.shape and s.dtype == np.uint16
        np.testing.assert_array_equal(s.read_box((0, 0, 0), (33, 20, 12)), vol)
        np.testing.assert_array_equal(s.read_box((5, 3, 2), (17, 9, 7)), vol[2:9, 3:12, 5:22])
    np.testing.assert_array_equal(api.read_slices(d), vol)


def test_slice_dir_rejects_mixed_planes(tmp_path):
    d = tmp_path / "mixed"
    make_slice_dir(d, np.zeros((3, 4, 5), np.uint8))
    (d / "0000030.raw").write_bytes(raw_bytes(np.zeros((1, 4, 6), np.uint8)))
    with pytest.raises(api.TeraWarpError):
        api.SliceDir(d)


def test_slice_writer_takes_tiles_in_any_order(tmp_path):
    """Tiles written into the slice files in shuffled order reassemble the
    volume exactly; the files are named as the reference names its stitched
    slices (z * 10, seven digits, .raw) and are valid raw stacks."""
    rng = np.random.default_rng(5)
    vol = rng.integers(0, 255, size=(9, 21, 30)).astype(np.uint8)
    d = tmp_path / "out_slice"
    tiles = [(x, y, z, min(8, 30 - x), min(6, 21 - y), min(4, 9 - z)) for z in range(0, 9, 4)
             for y in range(0, 21, 6) for x in range(0, 30, 8)]
    with api.SliceWriter(d, vol.shape, np.uint8, threads=2) as w:
        for i in rng.permutation(len(tiles)):
            x, y, z, nx, ny, nz = tiles[i]
            w.write_box((x, y, z), vol[z:z + nz, y:y + ny, x:x + nx])
    names = sorted(os.listdir(d))
    assert names == [f"{z * 10:07d}.raw" for z in range(9)]
    assert api.v3draw_header(d / names[3]) == ((30, 21, 1, 1), 1)
    np.testing.assert_array_equal(api.read_slices(d), vol)


def test_marker_files(tmp_path):
    p = tmp_path / "a.marker"
    p.write_text("##x,y,z,radius,shape,name,comment, color_r,color_g,color_b\n"
                 "10.5,20,30,0,1,,,255,0,0\n"
                 "# a comment line\n"
                 "\n"
                 " 1e1, 2.25 ,3,5,1,name,comment,0,255,0\n"
                 "garbage line\n"
                 "4,5\n")
    m = api.read_markers(p)
    np.testing.assert_array_equal(m, np.array([[10.5, 20, 30], [10, 2.25, 3]], np.float32))
    pts = np.random.default_rng(6).uniform(0, 1000, size=(50, 3)).astype(np.float32)
    api.write_markers(tmp_path / "b.marker", pts)
    np.testing.assert_array_equal(api.read_markers(tmp_path / "b.marker"), pts)
