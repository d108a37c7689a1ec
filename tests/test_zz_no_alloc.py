"""lt_plaquette_sum_noalloc: the allocation-free plaquette sum, for callers that may not
allocate device memory -- frameworks whose memory pool owns all device memory (a raw
cudaMalloc escapes its accounting) and timing or monitoring loops that an allocation would
stall by synchronising the device.

The caller owns every buffer: here torch allocates the input field (reference layout, on
the device) and the one-double output, outside the call under test.  The result is compared
with the C oracle's plaquette sum and with the existing entry point lt_plaquette_sum on the
same links, to the 1e-12 relative tolerance of the FP64 parity tests, on two calls in a row:
the second call runs on the static scratch left behind by the first.  Collected last (file
name) so a stop at the first failure has run every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200._lib import LT_ERR_ARG, check, lib

TOL = 1e-12


def noalloc_plaquette(links_dev, ext, out_dev, stream=None):
    e = np.ascontiguousarray(ext, dtype=np.int32)
    return lib().lt_plaquette_sum_noalloc(C.c_void_p(links_dev.data_ptr()), e, C.c_void_p(out_dev.data_ptr()),
                                          C.c_void_p(stream))


@pytest.mark.gpu
def test_noalloc_matches_plaquette_sum_twice(oracle):
    import torch

    for ext, seed in (((8, 8, 8, 8), 3), ((4, 6, 8, 10), 4)):
        links = lt.haar_links(ext, seed)
        G = lt.GaugeField(ext, "fp64")
        G.upload(links)
        lt.UpdateSweeps(G, 6.0, 3, 1, 2, seed=seed)      # not a Haar start: a partly thermalised field
        links = np.ascontiguousarray(G.download())
        expected = oracle.plaquette_sum(ext, links)
        assert lt.PlaquetteSum(G) == pytest.approx(expected, rel=TOL)

        dev = torch.from_numpy(links.reshape(-1)).to("cuda")
        out = torch.zeros(1, dtype=torch.float64, device="cuda")
        for _ in range(2):
            out.fill_(float("nan"))
            check(noalloc_plaquette(dev, ext, out))
            torch.cuda.synchronize()
            got = float(out.item())
            assert got == pytest.approx(expected, rel=TOL), (ext, got, expected)


@pytest.mark.gpu
def test_noalloc_rejects_volume_above_limit():
    import torch

    dev = torch.zeros(18, dtype=torch.float64, device="cuda")   # never read: rejected first
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert noalloc_plaquette(dev, (66, 64, 64, 64), out) == LT_ERR_ARG
    assert b"64^4" in lib().lt_last_error()
    # extents whose product wraps a 64-bit integer are refused before any multiplication wraps
    assert noalloc_plaquette(dev, (1 << 30, 1 << 30, 16, 2), out) == LT_ERR_ARG
    assert b"64^4" in lib().lt_last_error()
