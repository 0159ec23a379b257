"""Reference images and masks of a fit (hgx_read_image, hgx_read_mask) against the
reference's own readers (ImageData::read, EDFReader; compiled in oracle/_ref) where present,
and against the formats' definitions.  Host only: no GPU."""
import ctypes
import os
import struct

import numpy as np
import pytest

from conftest import ROOT
from hipgisaxs_b200 import HgxError
from hipgisaxs_b200.hig import read_image, read_mask

REF_SO = os.path.join(ROOT, "oracle", "_ref", "libhigref.so")


def write_edf(path, img, pad_to=512, extra_keys=0):
    """A little-endian float EDF: "key = value ;" items, '}' closing the header at the end of
    its 512-byte blocks, then the data."""
    nrow, ncol = img.shape
    items = ["HeaderID = EH:000001:000000:000000", "ByteOrder = LowByteFirst",
             "DataType = FloatValue", f"Dim_1 = {ncol}", f"Dim_2 = {nrow}",
             f"Size = {4 * img.size}", f"EDF_BinarySize = {4 * img.size}"]
    items += [f"Comment{i} = padding item number {i}" for i in range(extra_keys)]
    head = "{\n" + "".join(f"{it} ;\n" for it in items)
    nblocks = (len(head) + 2 + pad_to - 1) // pad_to
    head = head + " " * (nblocks * pad_to - len(head) - 2) + "}\n"
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(struct.pack(f"<{img.size}f", *img.astype(np.float32).ravel()))


def ref_read(path, edf):
    if not os.path.exists(REF_SO):
        return None
    L = ctypes.CDLL(REF_SO)
    L.ref_read_image.restype = ctypes.c_long
    buf = np.zeros(1 << 16)
    nc, nr = ctypes.c_int(), ctypes.c_int()
    n = L.ref_read_image(os.fsencode(path), int(edf), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                         ctypes.c_long(buf.size), ctypes.byref(nc), ctypes.byref(nr))
    assert n >= 0
    return buf[:n].copy(), nc.value, nr.value


def test_text_image(tmp_path):
    rng = np.random.default_rng(2)
    img = rng.gamma(2.0, 10.0, (6, 7))
    p = tmp_path / "ref.out"
    p.write_text("".join("\t".join(f"{v:.17g}" for v in row) + "\t\n" for row in img))
    data, nc, nr = read_image(str(p))
    assert (nc, nr) == (7, 6) and np.array_equal(data, img.ravel())
    want = ref_read(str(p), False)
    if want is not None:
        assert np.array_equal(data, want[0]) and (nc, nr) == want[1:]


def test_text_image_without_final_newline(tmp_path):
    """The reference counts the rows by its getline calls: a last line without a newline is
    read but not counted."""
    p = tmp_path / "ref.txt"
    p.write_text("1 2 3\n4 5 6\n7 8 9")
    data, nc, nr = read_image(str(p))
    assert (nc, nr) == (3, 2) and list(data) == list(range(1, 10))
    want = ref_read(str(p), False)
    if want is not None:
        assert np.array_equal(data, want[0]) and (nc, nr) == want[1:]


@pytest.mark.parametrize("extra", [0, 40])  # a one-block and a two-block header
def test_edf_image(tmp_path, extra):
    """EDF images.  The reference's reader is compared on one-block headers only: when a
    header block ends while it looks for the closing brace it reads past its 512-byte buffer
    (EDFReader::header_done, src/file/edf_reader.cpp), so its result on longer headers depends
    on heap contents."""
    rng = np.random.default_rng(3)
    img = rng.gamma(2.0, 10.0, (9, 11)).astype(np.float32)
    p = tmp_path / "ref.edf"
    write_edf(str(p), img, extra_keys=extra)
    data, nc, nr = read_image(str(p))
    assert (nc, nr) == (11, 9) and np.array_equal(data, img.astype(np.float64).ravel())
    want = ref_read(str(p), True) if extra == 0 else None
    if want is not None:
        assert np.array_equal(data, want[0]) and (nc, nr) == want[1:]


def test_masks(tmp_path):
    p = tmp_path / "mask.dat"
    p.write_text("1 0 1\n1 1 0\n")
    assert list(read_mask(str(p))) == [1, 0, 1, 1, 1, 0]
    q = tmp_path / "mask2.dat"
    q.write_text("1 0 1\n1 1 0")  # the reference drops a last value that ends the file
    assert list(read_mask(str(q))) == [1, 0, 1, 1, 1]
    e = tmp_path / "mask.edf"
    write_edf(str(e), np.array([[1, 0], [0, 2]], dtype=np.float32))
    assert list(read_mask(str(e))) == [1, 0, 0, 2]


def test_bad_files(tmp_path):
    with pytest.raises(HgxError):
        read_image(str(tmp_path / "missing.out"))
    (tmp_path / "img.png").write_text("x")
    with pytest.raises(HgxError):
        read_image(str(tmp_path / "img.png"))
    p = tmp_path / "short.edf"
    write_edf(str(p), np.ones((4, 4), dtype=np.float32))
    raw = open(p, "rb").read()
    open(p, "wb").write(raw[:-8])
    with pytest.raises(HgxError):
        read_image(str(p))
