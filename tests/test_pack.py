"""The host packing of repeated two-row FP32 uploads (lt_upload_links), without a device.

lt_pack_links_test runs the packer of lt_upload_links on the calling thread: FP64 links in the
reference layout in, the two-row FP32 device layout out (three float4 chunks per link, plane
(mu, parity), checkerboard index s = site / 2).  The layout restated here in numpy must match
it bit for bit: the FP32 values are IEEE round-to-nearest conversions of the inputs, as the
device conversion k_from_aos makes them (tests/test_gpu_parity.py checks the packed uploads
against that conversion on the device).
"""
import ctypes as C

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200 import _lib


def packed_layout(ext, links):
    """The two-row FP32 layout of the links, restated: 24 planes of V/2 float4."""
    V = int(np.prod(ext))
    vh = V // 2
    c = np.indices(ext).reshape(4, -1)                # coordinates of site i (last extent fastest)
    par = c.sum(axis=0) & 1
    s = np.arange(V) >> 1
    rows = links.reshape(V, 4, 18)[:, :, :12].astype(np.float32)   # rows 0-1, re/im interleaved
    out = np.zeros((24, vh, 4), dtype=np.float32)
    for mu in range(4):
        for p in range(2):
            m = par == p
            for ch in range(3):
                out[(mu * 2 + p) * 3 + ch, s[m]] = rows[m, mu, 4 * ch:4 * ch + 4]
    return out


def pack(ext, links):
    V = int(np.prod(ext))
    buf = np.zeros(48 * V + 4, dtype=np.float32)
    off = (-buf.ctypes.data % 16) // 4                # a 16-byte aligned view
    out = buf[off:off + 48 * V]
    e = np.array(ext, dtype=np.int32)
    _lib.check(lt.lib().lt_pack_links_test(e, np.ascontiguousarray(links).reshape(-1),
                                           out.ctypes.data_as(C.POINTER(C.c_float))))
    return out.reshape(24, V // 2, 4)


@pytest.mark.parametrize("ext", [(2, 2, 2, 2), (4, 6, 8, 10), (2, 4, 2, 6), (6, 4, 8, 2), (8, 8, 8, 8)])
def test_packing_matches_the_layout(ext):
    rng = np.random.default_rng(sum(ext))
    links = rng.standard_normal((int(np.prod(ext)), 4, 3, 3, 2))
    assert np.array_equal(pack(ext, links), packed_layout(ext, links))


def test_packing_rounds_to_nearest():
    """Values between FP32 neighbours land on the nearer one (ties to even)."""
    ext = (2, 2, 2, 2)
    links = np.full((16, 4, 3, 3, 2), 1.0 + 2.0 ** -24 + 2.0 ** -30)   # just above the tie
    got = pack(ext, links)
    assert np.all(got == np.float32(1.0 + 2.0 ** -23))
    links[...] = 1.0 + 2.0 ** -24                                      # the tie: to even
    assert np.all(pack(ext, links) == np.float32(1.0))


def test_bad_arguments_are_refused():
    links = np.zeros((16, 4, 3, 3, 2))
    buf = np.zeros(48 * 16 + 4, dtype=np.float32)
    off = (-buf.ctypes.data % 16) // 4
    ptr = buf[off:].ctypes.data_as(C.POINTER(C.c_float))
    assert lt.lib().lt_pack_links_test(np.array((2, 2, 2, 2), dtype=np.int32), links.reshape(-1), ptr) == _lib.LT_OK
    for ext in [(2, 2, 2, 3), (0, 2, 2, 2), (1 << 30, 1 << 30, 16, 2)]:
        e = np.array(ext, dtype=np.int32)
        assert lt.lib().lt_pack_links_test(e, links.reshape(-1), ptr) == _lib.LT_ERR_ARG
