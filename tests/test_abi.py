"""CPU checks of the drop-in boundary: the C-ABI library loads, exports every symbol the
header declares, and its host-side parts (Haar start, bias potential, argument checks)
behave like the reference.  No compute call reaches a GPU here."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import lettuce_b200 as lt
from lettuce_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_built_in_tree():
    assert os.path.exists(_lib.LIB_PATH)
    assert os.path.dirname(_lib.LIB_PATH) == os.path.join(ROOT, "lettuce_b200")


def test_exports_every_declared_symbol():
    declared = lt.declared_symbols()
    assert len(declared) >= 40
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in declared if s not in exported]
    assert not missing, missing
    assert set(declared) <= set(_lib.SIGNATURES), set(declared) - set(_lib.SIGNATURES)


def test_build_targets_sm100a_only():
    """The recipe compiles every translation unit for sm_100a and nothing else (the device
    side is checked on a B200 by lt_device_arch, tests/test_gpu_exp.py)."""
    from lettuce_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "lt_selftest.cu" in build.SOURCES


def test_version():
    assert lt.lib().lt_version() >= 100


def test_haar_links_are_su3_and_seeded():
    ext = (4, 4, 4, 6)
    U = lt.haar_links(ext, 5)
    M = (U[..., 0] + 1j * U[..., 1]).reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", M, M.conj()) - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-13
    assert np.array_equal(U, lt.haar_links(ext, 5))
    assert not np.array_equal(U, lt.haar_links(ext, 6))
    # Haar moments: <|U_ij|^2> = 1/3, <Re tr U> = 0
    assert np.mean(np.abs(M) ** 2) == pytest.approx(1 / 3, abs=0.01)
    assert abs(np.mean(np.trace(M, axis1=1, axis2=2).real)) < 0.05


def test_haar_rejects_odd_extent():
    out = np.empty((4 * 4 * 4 * 5, 4, 3, 3, 2))
    code = lt.lib().lt_haar_links(np.array([4, 4, 4, 5], dtype=np.int32), C.c_uint64(1), out)
    assert code == _lib.LT_ERR_ARG
    assert b"even" in lt.lib().lt_last_error()


def test_create_rejects_bad_extents_without_device():
    with pytest.raises(lt.LettuceError) as e:
        lt.GaugeField((4, 4, 3, 4))
    assert e.value.code == _lib.LT_ERR_ARG
    h = C.c_void_p()
    assert lt.lib().lt_create(np.array([4, 4, 4, 4], dtype=np.int32), 7, C.byref(h)) == _lib.LT_ERR_ARG
    assert not h.value


def test_null_handles_are_errors():
    v = C.c_double()
    assert lt.lib().lt_plaquette_sum(None, C.byref(v)) == _lib.LT_ERR_ARG
    assert lt.lib().lt_destroy(None) == _lib.LT_OK


def test_create_rejects_oversized_lattice_without_device():
    """4 V 9 complex entries must stay below 2^31 (96^4 does not)."""
    h = C.c_void_p()
    assert lt.lib().lt_create(np.array([96, 96, 96, 96], dtype=np.int32), 0, C.byref(h)) == _lib.LT_ERR_ARG
    assert b"too large" in lt.lib().lt_last_error()
    assert lt.lib().lt_create(np.array([2, 2, 2, 0], dtype=np.int32), 0, C.byref(h)) == _lib.LT_ERR_ARG
    # extents whose product wraps 64-bit arithmetic are refused before the product is formed
    big = 1 << 30
    assert lt.lib().lt_create(np.array([big, big, 16, 2], dtype=np.int32), 0, C.byref(h)) == _lib.LT_ERR_ARG
    assert b"too large" in lt.lib().lt_last_error()
    assert not h.value


def test_exp_test_entry_checks_arguments_without_device():
    q = np.zeros(18)
    out = np.zeros(18)
    L = lt.lib()
    assert L.lt_su3_exp_test(q, out, 1, 7, 0) == _lib.LT_ERR_ARG
    assert L.lt_su3_exp_test(q, out, 1, 0, 9) == _lib.LT_ERR_ARG
    assert L.lt_su3_exp_test(q, out, -1, 0, 0) == _lib.LT_ERR_ARG
    assert L.lt_su3_exp_test(q, out, 0, 0, 0) == _lib.LT_OK


def test_entry_points_check_handles_without_device():
    """Every entry point refuses a null handle before touching a device."""
    L = lt.lib()
    v, w = C.c_double(), C.c_double()
    u = C.c_uint64(0)
    calls = {
        "lt_md_integrate": lambda: L.lt_md_integrate(None, None, 3, 6.0, 1.0, 2, 0.1, 1, None, None),
        "lt_md_trajectory": lambda: L.lt_md_trajectory(None, None, 3, 6.0, 1.0, 2, 0.1, 1, C.c_uint64(1), C.byref(u), 1,
                                                       None, None, None),
        "lt_reverse_momenta": lambda: L.lt_reverse_momenta(None),
        "lt_parity_update": lambda: L.lt_parity_update(None),
        "lt_set_gauge_action": lambda: L.lt_set_gauge_action(None, 2, 1.0, 0.0),
        "lt_overrelax_sweeps4": lambda: L.lt_overrelax_sweeps4(None, 1),
        "lt_heatbath_sweeps4": lambda: L.lt_heatbath_sweeps4(None, 6.0, 1, C.c_uint64(1), C.byref(u)),
        "lt_wilson_loop_chain": lambda: L.lt_wilson_loop_chain(None, 0, 2, 1, C.byref(v)),
        "lt_polyakov_loop": lambda: L.lt_polyakov_loop(None, C.byref(v), C.byref(w)),
        "lt_flow": lambda: L.lt_flow(None, None, 0, 0.01, 1),
        "lt_clover_timeslices": lambda: L.lt_clover_timeslices(None, None, None),
        "lt_status_word": lambda: L.lt_status_word(None, C.byref(C.c_uint32()), 0),
    }
    for name, call in calls.items():
        assert call() == _lib.LT_ERR_ARG, name
        assert b"null handle" in L.lt_last_error(), name


def test_bias_matches_reference_fixture(golden_bias):
    g = golden_bias
    for sym in (0, 1):
        b = lt.MetaBiasPotential(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0)
        for cv in g["deposits"]:
            (b.UpdatePotentialSymmetric if sym else b.UpdatePotential)(cv)
        pot = np.array([b.ReturnPotential(p) for p in g["probes"]])
        der = np.array([b.ReturnDerivative(p) for p in g["probes"]])
        np.testing.assert_allclose(pot, g[f"pot{sym}"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(der, g[f"der{sym}"], rtol=1e-10, atol=1e-10)


def test_bias_constructor_throws_like_reference():
    with pytest.raises(ValueError, match="CV_min < CV_max"):
        lt.MetaBiasPotential(1.0, -1.0, 800, 0.05, 0.08, 10, 1000)
    with pytest.raises(ValueError, match="bin_number > 0"):
        lt.MetaBiasPotential(-1.0, 1.0, 0, 0.05, 0.08, 10, 1000)


def test_bias_generate_and_grid():
    b = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
    b.GeneratePotentialFrom(lambda cv: 0.5 * cv)
    assert b.ReturnDerivative(0.123) == pytest.approx(0.5, rel=1e-12)
    assert b.grid().shape == (801,)
    assert b.ReturnPotential(9.0) == pytest.approx(4.0 + 1000.0, rel=1e-12)
