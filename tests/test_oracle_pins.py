"""Pin the C restatement (oracle/lt_oracle.c) against the reference itself.

Every oracle function is compared with the golden fixtures generated from the reference's
own code (tests/golden/gen_golden.py) and, where the reference harness is built here, with
the reference run live on fresh inputs.  Tolerance: 1e-12 relative to the field's largest
entry (FP64 on both sides; the only differences are summation order and libm rounding).
"""
import os

import numpy as np
import pytest

from ltref import DBW2, IWASAKI, LUESCHER_WEISZ, WILSON, Reference, haar_links_numpy, ref_available, rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TOL = 1e-12


def links_of(field, idx):
    return field.reshape(-1, 18)[idx]


def checksums(field):
    f = field.reshape(-1)
    w = np.arange(f.size, dtype=np.float64) % 97.0
    return np.array([f.sum(), (f * f).sum(), (w * f).sum()])


def close_ck(a, b, tol=1e-10):
    a, b = np.asarray(a), np.asarray(b)
    return np.all(np.abs(a - b) <= tol * np.maximum(1.0, np.abs(b)))


class TestGolden4:
    """4^4 fixture: Haar start, every function of the path."""

    def test_scalars(self, oracle, golden4):
        g, ext, U = golden4, golden4["ext"], golden4["U"]
        assert oracle.plaquette_sum(ext, U) == pytest.approx(float(g["plaq"]), rel=TOL)
        assert oracle.wilson_action(ext, U, 6.0) == pytest.approx(float(g["action"]), rel=TOL)
        assert oracle.topcharge(ext, U) == pytest.approx(float(g["Q"]), rel=1e-11, abs=1e-14)
        assert oracle.energy(ext, U) == pytest.approx(float(g["E"]), rel=TOL)

    def test_staples(self, oracle, golden4):
        g = golden4
        S = oracle.staples(g["ext"], g["U"])
        assert rel_err(links_of(S, g["links"]), g["staples"]) < TOL
        assert close_ck(checksums(S), g["staples_ck"])

    def test_overrelaxation_sweep(self, oracle, golden4):
        g = golden4
        O = oracle.overrelax(g["ext"], g["U"], 1)
        # a hot (Haar) start has nearly singular SU(2) projections; 1e-10 there
        assert rel_err(links_of(O, g["links"]), g["or1"]) < 1e-10
        assert oracle.plaquette_sum(g["ext"], O) == pytest.approx(float(g["or1_plaq"]), rel=1e-11)

    def test_flow_rk3(self, oracle, golden4):
        g = golden4
        F = oracle.flow_rk3(g["ext"], g["U"], 0.01, 10)
        assert rel_err(links_of(F, g["links"]), g["flow10"]) < TOL
        assert close_ck(checksums(F), g["flow10_ck"])

    def test_stout(self, oracle, golden4):
        g = golden4
        S = oracle.stout(g["ext"], g["U"], 0.12, 4)
        assert rel_err(links_of(S, g["links"]), g["stout4"]) < TOL

    def test_gauge_force(self, oracle, golden4):
        g = golden4
        F = oracle.gauge_force(g["ext"], g["U"], 6.0)
        assert rel_err(links_of(F, g["links"]), g["gforce"]) < TOL

    def test_clover_derivative(self, oracle, golden4):
        g = golden4
        D = oracle.clover_derivative(g["ext"], g["U"])
        assert rel_err(links_of(D, g["links"]), g["cderiv"]) < TOL

    def test_metad_force(self, oracle, golden4):
        g = golden4
        n = int(g["metad_nstout"])
        M, q = oracle.metad_force(g["ext"], g["U"], 0.12, n, 1.0)
        assert rel_err(links_of(M, g["links"]), g["metad"]) < 1e-11
        assert q == pytest.approx(float(g["metad_q"]), rel=1e-11)

    def test_omf2(self, oracle, golden4):
        g = golden4
        U2, P2, ho, hn = oracle.omf2(g["ext"], g["U"], g["P"], 6.0, 1.0, 10)
        assert rel_err(links_of(U2, g["links"]), g["omf2_U"]) < 1e-11
        assert rel_err(links_of(P2, g["links"]), g["omf2_P"]) < 1e-11
        assert ho == pytest.approx(g["omf2_h"][0], rel=TOL)
        assert hn == pytest.approx(g["omf2_h"][1], rel=TOL)

    def test_su3_exp(self, oracle, golden4):
        g = golden4
        out = oracle.su3_exp(g["exp_in"].reshape(-1)).reshape(g["exp_out"].shape)
        assert np.max(np.abs(out - g["exp_out"])) < 1e-13

    def test_su3_exp_branch_cases(self, oracle):
        """Every branch range of the exponential (tests/golden/ref_exp.npz): the oracle and
        the reference agree, and both agree with an independent Pade evaluation of expm."""
        import scipy.linalg as sl
        g = dict(np.load(os.path.join(GOLDEN, "ref_exp.npz")))
        out = oracle.su3_exp(g["exp_in"].reshape(-1)).reshape(g["exp_out"].shape)
        assert np.max(np.abs(out - g["exp_out"])) < 1e-13
        q = g["exp_in"].reshape(-1, 9, 2)
        Q = (q[..., 0] + 1j * q[..., 1]).reshape(-1, 3, 3)
        E = np.array([sl.expm(1j * M) for M in Q])
        R = g["exp_out"].reshape(-1, 9, 2)
        assert np.max(np.abs(E.reshape(-1, 9) - (R[..., 0] + 1j * R[..., 1]))) < 1e-13


class TestGoldenOdd:
    """4x6x8x10: uneven extents, numpy-seeded Haar start regenerated from the seed."""

    def test_input_regenerates(self, golden_odd):
        U = haar_links_numpy((4, 6, 8, 10), int(golden_odd["seed"]))
        assert close_ck(checksums(U), golden_odd["U_ck"], 1e-12)

    def test_functions(self, oracle, golden_odd):
        g = golden_odd
        ext = g["ext"]
        U = haar_links_numpy(tuple(ext), int(g["seed"]))
        assert oracle.plaquette_sum(ext, U) == pytest.approx(float(g["plaq"]), rel=TOL)
        assert oracle.topcharge(ext, U) == pytest.approx(float(g["Q"]), rel=1e-10, abs=1e-13)
        assert oracle.energy(ext, U) == pytest.approx(float(g["E"]), rel=TOL)
        assert rel_err(links_of(oracle.staples(ext, U), g["links"]), g["staples"]) < TOL
        assert rel_err(links_of(oracle.flow_rk3(ext, U, 0.01, 10), g["links"]), g["flow10"]) < TOL
        assert rel_err(links_of(oracle.stout(ext, U, 0.12, 4), g["links"]), g["stout4"]) < TOL
        assert rel_err(links_of(oracle.gauge_force(ext, U, 6.0), g["links"]), g["gforce"]) < TOL
        assert rel_err(links_of(oracle.overrelax(ext, U, 1), g["links"]), g["or1"]) < 1e-10


def test_bias_potential(oracle, golden_bias):
    """MetaBiasPotential deposits, interpolation, walls and derivative."""
    g = golden_bias
    for sym in (0, 1):
        b = oracle.lib.or_bias_create(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0)
        for cv in g["deposits"]:
            if sym:
                oracle.lib.or_bias_update_symmetric(b, cv)
            else:
                oracle.lib.or_bias_update(b, cv)
        pot = np.array([oracle.lib.or_bias_potential(b, p) for p in g["probes"]])
        der = np.array([oracle.lib.or_bias_derivative(b, p) for p in g["probes"]])
        oracle.lib.or_bias_destroy(b)
        np.testing.assert_allclose(pot, g[f"pot{sym}"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(der, g[f"der{sym}"], rtol=1e-10, atol=1e-10)


def test_bias_rejects_bad_range(oracle):
    assert not oracle.lib.or_bias_create(1.0, -1.0, 800, 0.05, 0.08, 10.0, 1000.0)
    assert not oracle.lib.or_bias_create(-1.0, 1.0, 0, 0.05, 0.08, 10.0, 1000.0)


@pytest.mark.skipif(not ref_available((8, 8, 8, 8)), reason="reference harness not built here")
class TestLiveReference:
    """Oracle vs the reference on fresh inputs (8^4, thermalised by 20 reference heatbath sweeps)."""

    def test_observables_and_flow(self, oracle):
        ext = (8, 8, 8, 8)
        ref = Reference(ext)
        U = haar_links_numpy(ext, 77)
        U, _ = ref.hb_or_chain(U, 6.0, 20, 1, 0)
        assert oracle.plaquette_sum(ext, U) == pytest.approx(ref.plaquette_sum(U), rel=TOL)
        assert oracle.topcharge(ext, U) == pytest.approx(ref.topcharge(U), rel=1e-10, abs=1e-12)
        assert rel_err(oracle.overrelax(ext, U, 1), ref.overrelax(U, 1)) < TOL
        assert rel_err(oracle.flow_rk3(ext, U, 0.01, 3), ref.flow_rk3(U, 0.01, 3)) < TOL


class TestBMW:
    """BMW configuration files (IO/config_io/bmw_format.hpp): the oracle's payload and
    Adler-64 checksum against files written by the reference's SaveConfigBMW(Full)."""

    def test_oracle_reproduces_reference_files(self, oracle, golden_bmw):
        import hashlib
        from ltref import bmw_header
        ext = tuple(int(e) for e in golden_bmw["ext"])
        U = haar_links_numpy(ext, int(golden_bmw["seed"]))
        for full, key in ((False, "two_row"), (True, "full")):
            ck, payload = oracle.bmw_encode(ext, U, full)
            assert f"{ck:x}" == str(golden_bmw[f"checksum_{key}"])
            data = bmw_header(ext, ck, full) + payload
            assert hashlib.sha256(data).hexdigest() == str(golden_bmw[f"sha256_{key}"])

    def test_oracle_decodes_reference_file(self, oracle, golden_bmw):
        ext = tuple(int(e) for e in golden_bmw["ext"])
        data = open(golden_bmw["two_row_file"], "rb").read()
        ck, U = oracle.bmw_decode(ext, data[4096:], False)
        assert f"{ck:x}" == data[:4096].split(b"\n")[0].split()[-1].decode()
        assert np.array_equal(checksums(U), golden_bmw["loaded_ck_two_row"])
        U0 = haar_links_numpy(ext, int(golden_bmw["seed"]))
        assert np.abs(U - U0).max() < 1e-15

    @pytest.mark.skipif(not ref_available((4, 6, 8, 10)), reason="reference harness not built")
    def test_live_reference_save_and_load(self, oracle, tmp_path):
        import hashlib
        from ltref import bmw_header
        ext = (4, 6, 8, 10)
        ref = Reference(ext)
        U = haar_links_numpy(ext, 23)
        for full in (False, True):
            path = tmp_path / f"c{int(full)}.bmw"
            assert ref.save_bmw(U, path, full)
            data = path.read_bytes()
            ck, payload = oracle.bmw_encode(ext, U, full)
            assert hashlib.sha256(bmw_header(ext, ck, full) + payload).digest() == hashlib.sha256(data).digest()
            ok, loaded = ref.load_bmw(path, full)
            assert ok
            _, mine = oracle.bmw_decode(ext, data[4096:], full)
            assert np.array_equal(mine, loaded)


class TestMeasurementBundle:
    """The observables of the reference driver's measurement step (SU3_main.cpp:89-235) and
    the four flow integrators (smearing/gradient_flow.hpp:31-168), against the reference."""

    def test_against_fixture(self, oracle, golden_measure):
        g = golden_measure
        ext = tuple(int(e) for e in g["ext"])
        U = g["U"]
        assert close_ck(checksums(U), g["U_ck"], 1e-12)
        m = oracle.measure(ext, U, 6.0)
        for k in ("Q_plaq", "S_improved", "W2", "W4", "W8"):
            assert m[k] == pytest.approx(float(g[k]), rel=TOL, abs=1e-14), k
        assert m["P"] == pytest.approx(complex(g["P"]), rel=TOL, abs=1e-14)
        np.testing.assert_allclose(m["q_t"], g["q_t"], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(m["e_t"], g["e_t"], rtol=TOL)
        assert m["q_t"].sum() == pytest.approx(oracle.topcharge(ext, U), rel=1e-12, abs=1e-14)
        # the reference's chained WilsonLoop along straight runs equals the loop of the end length
        for (a, b, r), want in list(zip(g["wl_chain_seq"], g["wl_chain"]))[:5]:
            assert oracle.lib.or_wilson_loop(oracle._e(ext), np.ascontiguousarray(U), int(b)) == pytest.approx(
                float(want), rel=TOL)
        for integ in range(4):
            F = oracle.flow(ext, U, 0.02, 5, integ)
            assert rel_err(links_of(F, g["links"]), g[f"flow{integ}"]) < TOL, integ
            assert close_ck(checksums(F), g[f"flow{integ}_ck"], 1e-11)

    @pytest.mark.skipif(not ref_available((4, 4, 4, 4)), reason="reference harness not built")
    def test_live_reference(self, oracle):
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 8), 5.8, 4, 3, 0)
        ref = Reference(ext).measure(U, 6.2)
        mine = oracle.measure(ext, U, 6.2)
        for k in ("Q_plaq", "S_improved", "W2", "W4", "W8", "P"):
            assert mine[k] == pytest.approx(ref[k], rel=TOL, abs=1e-14), k
        np.testing.assert_allclose(mine["q_t"], ref["q_t"], rtol=1e-10, atol=1e-14)
        np.testing.assert_allclose(mine["e_t"], ref["e_t"], rtol=TOL)


MD_CASES = [(i, False) for i in range(8)] + [(i, True) for i in (0, 1, 2, 3, 4, 5, 8, 9, 10)]


class TestMDIntegrators:
    """The eleven MD integrators of the reference (hmc_gauge.hpp:19-377,
    hmc_metadynamics.hpp:26-238) on HMCKernel and HMCMetaDKernel, and ParityUpdate
    (parity_update.hpp:22-47), against the reference."""

    @pytest.mark.parametrize("integ,metad", MD_CASES)
    def test_against_fixture(self, oracle, golden_md, integ, metad):
        g = golden_md
        ext = tuple(int(e) for e in g["ext"])
        assert close_ck(checksums(g["U"]), g["U_ck"], 1e-12) and close_ck(checksums(g["P"]), g["P_ck"], 1e-12)
        U, P, ho, hn = oracle.md_integrate(ext, g["U"], g["P"], float(g["beta"]), float(g["tau"]), int(g["n_step"]),
                                           integ, metad, float(g["rho"]), int(g["n_stout"]), float(g["slope"]))
        key = f"{'metad' if metad else 'gauge'}{integ}"
        assert rel_err(links_of(U, g["links"]), g[key + "_U"]) < 1e-12
        assert rel_err(links_of(P, g["links"]), g[key + "_P"]) < 1e-12
        assert close_ck(np.concatenate([checksums(U), checksums(P)]), g[key + "_ck"], 1e-11)
        assert ho == pytest.approx(g[key + "_h"][0], rel=1e-13)
        assert hn == pytest.approx(g[key + "_h"][1], rel=1e-13)

    def test_parity_fixture(self, oracle, golden_md):
        g = golden_md
        ext = tuple(int(e) for e in g["ext"])
        R = oracle.parity_update(ext, g["U"])
        assert np.array_equal(links_of(R, g["links"]), g["parity_U"])
        assert close_ck(checksums(R), g["parity_ck"], 0.0)
        # action unchanged, clover charge flips sign
        assert oracle.wilson_action(ext, R, 6.0) == pytest.approx(oracle.wilson_action(ext, g["U"], 6.0), rel=1e-14)
        assert oracle.topcharge(ext, R) == pytest.approx(-oracle.topcharge(ext, g["U"]), rel=1e-10, abs=1e-13)

    def test_orders(self, oracle):
        """dH falls as eps^2 (OMF2, Leapfrog-OMF4, OMF2-OMF4) and eps^4 (OMF4); the reference's
        OMF_2_OMF_4_slow runs its inner OMF4 at full steps, so the gauge part advances 2 tau and
        dH does not fall."""
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 2), 6.0, 5, 17, 0)
        P = oracle.random_momenta(ext, 9, 0)

        def ratio(integ, n, metad):
            d = []
            for k in (n, 2 * n):
                _, _, ho, hn = oracle.md_integrate(ext, U, P, 6.0, 0.5, k, integ, metad, 0.12, 1, 0.7)
                d.append(abs(hn - ho))
            return d[0] / d[1]

        assert 3.0 < ratio(3, 8, False) < 5.0
        assert 12.0 < ratio(5, 4, False) < 24.0
        assert 3.0 < ratio(8, 4, True) < 6.0
        assert 3.0 < ratio(10, 4, True) < 6.0
        assert ratio(9, 4, True) < 1.2

    @pytest.mark.skipif(not ref_available((4, 6, 8, 10)), reason="reference harness not built")
    def test_live_reference(self, oracle):
        ext = (4, 6, 8, 10)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 9), 5.9, 3, 4, 0)
        P = oracle.random_momenta(ext, 3, 1)
        ref = Reference(ext)
        for integ, metad in ((7, False), (5, True), (10, True)):
            a = oracle.md_integrate(ext, U, P, 5.9, 0.4, 2, integ, metad, 0.1, int(ref.lib.ref_n_smear_meta()), -1.3)
            b = ref.md_integrate(U, P, 5.9, 0.4, 2, integ, metad, 0.1, -1.3)
            assert rel_err(a[0], b[0]) < 1e-12 and rel_err(a[1], b[1]) < 1e-12
            assert a[3] == pytest.approx(b[3], rel=1e-13)
        assert np.array_equal(oracle.parity_update(ext, U), ref.parity_update(U))


RECT = (("lw", LUESCHER_WEISZ), ("iwasaki", IWASAKI), ("dbw2", DBW2))


class TestRectangularActions:
    """GaugeAction::Rectangular<2> (rectangular_action.hpp:23-276) staples, sweeps over
    Iterator::Checkerboard4 (iterators.hpp:141-166), gauge MD and flow, against the reference."""

    @pytest.mark.parametrize("name,act", RECT)
    def test_against_fixture(self, oracle, golden_rect, name, act):
        g = golden_rect
        ext = tuple(int(e) for e in g["ext"])
        assert close_ck(checksums(g["U"]), g["U_ck"], 1e-12) and close_ck(checksums(g["P"]), g["P_ck"], 1e-12)
        assert tuple(g[name + "_act"]) == pytest.approx(act, rel=1e-15)
        S = oracle.action_staples(ext, g["U"], act)
        assert rel_err(links_of(S, g["links"]), g[name + "_staple"]) < 1e-13
        assert close_ck(checksums(S), g[name + "_staple_ck"], 1e-11)
        R = oracle.overrelax4(ext, g["U"], 2, act)
        assert rel_err(links_of(R, g["links"]), g[name + "_or4"]) < 1e-11
        U2, P2, ho, hn = oracle.md_integrate_action(ext, g["U"], g["P"], 6.0, 0.5, 3, int(g[name + "_md_integ"]), act)
        assert rel_err(links_of(U2, g["links"]), g[name + "_md_U"]) < 1e-12
        assert rel_err(links_of(P2, g["links"]), g[name + "_md_P"]) < 1e-12
        assert ho == pytest.approx(g[name + "_md_h"][0], rel=1e-13) and hn == pytest.approx(g[name + "_md_h"][1], rel=1e-13)
        F = oracle.flow_action(ext, g["U"], 0.02, 10, 2, act)
        assert rel_err(links_of(F, g["links"]), g[name + "_flow"]) < 1e-12

    def test_wilson_checkerboard4_fixture(self, oracle, golden_rect):
        g = golden_rect
        ext = tuple(int(e) for e in g["ext"])
        R = oracle.overrelax4(ext, g["U"], 2, WILSON)
        assert rel_err(links_of(R, g["links"]), g["wilson_or4"]) < 1e-11
        # a different visiting order than Checkerboard: the fields differ
        assert rel_err(R, oracle.overrelax(ext, g["U"], 2)) > 1e-6

    def test_action_state_resets(self, oracle, golden_rect):
        g = golden_rect
        ext = tuple(int(e) for e in g["ext"])
        oracle.action_staples(ext, g["U"], DBW2)
        assert rel_err(oracle.staples(ext, g["U"]), oracle.action_staples(ext, g["U"], WILSON)) == 0.0

    def test_rect_staple_is_action_derivative(self, oracle):
        """d/dt S(exp(t X) U) at t = 0 equals -beta/3 Re tr(X U Staple^dag) summed over one link:
        the rectangle staple is the derivative of the rectangle action."""
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 6), 6.0, 2, 1, 0)
        act = IWASAKI
        S = oracle.action_staples(ext, U, act)
        rng = np.random.default_rng(3)
        site, mu = 37, 2
        H = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        X = 0.5j * (H + H.conj().T)
        X -= np.trace(X) / 3 * np.eye(3)
        Uc = U.reshape(-1, 4, 3, 3, 2)
        u = Uc[site, mu, ..., 0] + 1j * Uc[site, mu, ..., 1]
        st = S.reshape(-1, 4, 3, 3, 2)[site, mu]
        st = st[..., 0] + 1j * st[..., 1]
        want = -6.0 / 3.0 * np.real(np.trace(X @ u @ st.conj().T))

        def action_at(t):
            from scipy.linalg import expm
            V = Uc.copy()
            w = expm(t * X) @ u
            V[site, mu, ..., 0], V[site, mu, ..., 1] = w.real, w.imag
            return oracle.lib.or_rect_action(oracle._e(ext), np.ascontiguousarray(V.reshape(U.shape)), 6.0,
                                             act[1], act[2])

        h = 1e-5
        assert (action_at(h) - action_at(-h)) / (2 * h) == pytest.approx(want, rel=1e-6)

    @pytest.mark.skipif(not ref_available((4, 4, 4, 4)), reason="reference harness not built")
    def test_live_reference(self, oracle):
        ext = (4, 4, 4, 4)
        U = oracle.heatbath(ext, haar_links_numpy(ext, 9), 5.9, 3, 4, 0)
        P = oracle.random_momenta(ext, 3, 1)
        ref = Reference(ext)
        for act in (LUESCHER_WEISZ, DBW2, (2, 0.7, 0.2)):
            assert rel_err(oracle.action_staples(ext, U, act), ref.action_staples(U, act)) < 1e-13
            assert rel_err(oracle.overrelax4(ext, U, 1, act), ref.overrelax4(U, 1, act)) < 1e-11
            a = oracle.md_integrate_action(ext, U, P, 5.9, 0.3, 2, 7, act)
            b = ref.md_action(U, P, 5.9, 0.3, 2, 7, act)
            assert rel_err(a[0], b[0]) < 1e-12 and a[3] == pytest.approx(b[3], rel=1e-13)
            assert rel_err(oracle.flow_action(ext, U, 0.03, 3, 3, act), ref.flow_action(U, 0.03, 3, 3, act)) < 1e-12


class TestLargeFixtures:
    """The full-size fixtures used by the GPU parity tests at the benchmarked sizes: their
    inputs regenerate bit for bit here, and the oracle reproduces the reference's
    overrelaxation sweep at 32^4."""

    def test_32x4_input_and_overrelaxation(self, oracle):
        from ltref import checksums, large_input
        g = dict(np.load(os.path.join(GOLDEN, "ref_32x32x32x32.npz")))
        ext = tuple(int(e) for e in g["ext"])
        U = large_input(ext, int(g["seed"]), int(g["hb_seed"]), oracle)
        np.testing.assert_allclose(checksums(U), g["U_ck"], rtol=1e-13)
        O = oracle.overrelax(ext, U, 1)
        assert rel_err(O.reshape(-1, 18)[g["links"]], g["or1"]) < TOL
        assert oracle.plaquette_sum(ext, O) == pytest.approx(float(g["or1_plaq"]), rel=TOL)

    def test_16x4_metad_input(self, oracle):
        from ltref import checksums, large_input
        g = dict(np.load(os.path.join(GOLDEN, "ref_metad_16x16x16x16.npz")))
        ext = tuple(int(e) for e in g["ext"])
        U = large_input(ext, int(g["seed"]), int(g["hb_seed"]), oracle)
        np.testing.assert_allclose(checksums(U), g["U_ck"], rtol=1e-13)
        F, q = oracle.metad_force(ext, U, 0.12, int(g["metad_nstout"]), 1.0)
        assert q == pytest.approx(float(g["metad_q"]), rel=1e-11, abs=1e-12)
        assert rel_err(F.reshape(-1, 18)[g["links"]], g["metad"]) < 1e-11
