"""BMW configuration files through the C ABI (lt_save_bmw / lt_load_bmw / lt_bmw_checksum).

The device packs the links and computes the Adler-64 checksum; files must be byte-identical
to the reference's SaveConfigBMW / SaveConfigBMWFull output (tests/golden/), and loading must
reproduce the reference's LoadConfigBMW(Full) bit for bit in FP64."""
import hashlib

import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import bmw_header, haar_links_numpy

pytestmark = pytest.mark.gpu


def field(ext, U, prec="fp64"):
    G = lt.GaugeField(ext, prec)
    G.upload(U)
    return G


def golden_input(golden_bmw):
    ext = tuple(int(e) for e in golden_bmw["ext"])
    return ext, haar_links_numpy(ext, int(golden_bmw["seed"]))


@pytest.mark.parametrize("full,key", [(False, "two_row"), (True, "full")])
def test_save_is_byte_identical_to_reference(golden_bmw, tmp_path, full, key):
    ext, U = golden_input(golden_bmw)
    G = field(ext, U)
    path = tmp_path / "cfg.bmw"
    ck = G.save_bmw(path, full=full)
    assert ck == str(golden_bmw[f"checksum_{key}"])
    assert hashlib.sha256(path.read_bytes()).hexdigest() == str(golden_bmw[f"sha256_{key}"])
    assert G.bmw_checksum(full=full) == int(ck, 16)


def test_load_reference_file(oracle, golden_bmw):
    ext, _ = golden_input(golden_bmw)
    G = lt.GaugeField(ext)
    ok, in_group = G.load_bmw(golden_bmw["two_row_file"])
    assert ok and in_group
    data = open(golden_bmw["two_row_file"], "rb").read()
    _, expect = oracle.bmw_decode(ext, data[4096:], False)
    assert np.array_equal(G.download(), expect)       # third row in the reference's rounding


@pytest.mark.parametrize("prec", ["fp64", "fp32", "fp32_12"])
def test_roundtrip_and_checksum_against_oracle(oracle, tmp_path, prec):
    ext = (4, 6, 8, 10)
    G = field(ext, haar_links_numpy(ext, 5), prec)
    lt.UpdateSweeps(G, 6.0, 2, 1, 2, seed=3)
    links = G.download()
    for full in (False, True):
        path = tmp_path / f"c{int(full)}.bmw"
        ck = G.save_bmw(path, full=full, overwrite=True)
        want, payload = oracle.bmw_encode(ext, links, full)
        assert int(ck, 16) == want
        assert path.read_bytes() == bmw_header(ext, want, full) + payload
        H = lt.GaugeField(ext, prec)
        ok, in_group = H.load_bmw(path, full=full)
        assert ok and in_group
        back = H.download()
        if full or prec == "fp32_12":
            assert np.array_equal(back, links)
        else:
            assert np.abs(back - links).max() < (1e-15 if prec == "fp64" else 1e-6)


def test_checksum_at_32x4_matches_oracle(oracle):
    """Full-size check: the device checksum of a 32^4 field equals the C restatement's."""
    ext = (32, 32, 32, 32)
    G = lt.GaugeField(ext, "fp32_12")
    G.SetToHaarRandom(9)
    links = G.download()
    for full in (False, True):
        want, _ = oracle.bmw_encode(ext, links, full)
        assert G.bmw_checksum(full=full) == want


def test_corrupt_and_mismatched_files(golden_bmw, tmp_path):
    ext, _ = golden_input(golden_bmw)
    data = bytearray(open(golden_bmw["two_row_file"], "rb").read())
    data[4096 + 8 * 125 + 7] ^= 0x01                 # last mantissa bit of one big-endian double
    bad = tmp_path / "bad.bmw"
    bad.write_bytes(bytes(data))
    G = lt.GaugeField(ext)
    ok, in_group = G.load_bmw(bad)
    assert not ok and in_group
    with pytest.raises(lt.LettuceError):             # shape differs from the handle's
        lt.GaugeField((2, 4, 6, 10)).load_bmw(golden_bmw["two_row_file"])
    with pytest.raises(lt.LettuceError):             # a two-row file read as #18BMW
        G.load_bmw(golden_bmw["two_row_file"], full=True)
    short = tmp_path / "short.bmw"
    short.write_bytes(bytes(data[:-8]))
    with pytest.raises(lt.LettuceError):             # truncated payload
        G.load_bmw(short)
    with pytest.raises(lt.LettuceError):             # exists, no overwrite
        G.save_bmw(bad)
