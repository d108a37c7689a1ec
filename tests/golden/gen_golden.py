"""Generate the golden fixtures in tests/golden/ from the reference's own code.

Runs the compiled reference harness (oracle/ref_harness.cpp built by oracle/build_ref.py
against the reference headers) on seeded inputs and stores inputs, sampled output links and
full-field checksums.  Needs the reference checkout (it builds the harness); the fixtures it
writes are committed so the tests never need the reference at run time.

Usage: python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from ltref import Reference, checksums, haar_links_numpy, large_input  # noqa: E402

BETA = 6.0
N_SAMPLE = 64


def sample_links(V: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(4 * V, size=N_SAMPLE, replace=False))




def take(field: np.ndarray, links: np.ndarray) -> np.ndarray:
    return field.reshape(-1, 18)[links]


def random_momenta(V: int, seed: int) -> np.ndarray:
    """Traceless anti-Hermitian momenta from numpy Gaussians (input data only)."""
    rng = np.random.default_rng(seed)
    phi = rng.standard_normal((V * 4, 8))
    s3 = np.sqrt(3.0)
    A = np.zeros((V * 4, 3, 3), dtype=np.complex128)
    A[:, 0, 0] = 1j * (phi[:, 2] + phi[:, 7] / s3)
    A[:, 0, 1] = phi[:, 1] + 1j * phi[:, 0]
    A[:, 0, 2] = phi[:, 4] + 1j * phi[:, 3]
    A[:, 1, 0] = -phi[:, 1] + 1j * phi[:, 0]
    A[:, 1, 1] = 1j * (-phi[:, 2] + phi[:, 7] / s3)
    A[:, 1, 2] = phi[:, 6] + 1j * phi[:, 5]
    A[:, 2, 0] = -phi[:, 4] + 1j * phi[:, 3]
    A[:, 2, 1] = -phi[:, 6] + 1j * phi[:, 5]
    A[:, 2, 2] = 1j * (-2.0 * phi[:, 7] / s3)
    A *= 0.5
    out = np.empty((V, 4, 3, 3, 2))
    out[..., 0] = A.real.reshape(V, 4, 3, 3)
    out[..., 1] = A.imag.reshape(V, 4, 3, 3)
    return out


def hermitian_inputs(n: int, seed: int) -> np.ndarray:
    """Traceless Hermitian matrices spanning the exponential's branches: generic, small
    (Taylor branch of xi_0), negative determinant (sign flip) and exactly degenerate (zero)."""
    rng = np.random.default_rng(seed)
    out = np.zeros((n, 3, 3, 2))
    for k in range(n):
        M = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        H = 0.5 * (M + M.conj().T)
        H -= np.trace(H) / 3.0 * np.eye(3)
        scale = [1.0, 0.01, 1e-4, 2.0][k % 4]
        H *= scale
        if k % 8 == 7:
            H = -H
        if k == n - 1:
            H[:] = 0.0
        out[k, ..., 0] = H.real
        out[k, ..., 1] = H.imag
    return out


def gen_case(ext, seed: int, full: bool) -> dict:
    ref = Reference(ext)
    V = int(np.prod(ext))
    U = haar_links_numpy(ext, seed)
    links = sample_links(V, seed + 100)
    d = {"ext": np.array(ext, dtype=np.int32), "seed": np.array(seed), "U": U, "links": links,
         "plaq": np.array(ref.plaquette_sum(U)), "action": np.array(ref.wilson_action(U, BETA)),
         "Q": np.array(ref.topcharge(U)), "E": np.array(ref.energy(U))}
    S = ref.staples(U)
    d["staples"], d["staples_ck"] = take(S, links), checksums(S)
    O = ref.overrelax(U, 1)
    d["or1"], d["or1_ck"] = take(O, links), checksums(O)
    d["or1_plaq"] = np.array(ref.plaquette_sum(O))
    F = ref.flow_rk3(U, 0.01, 10)
    d["flow10"], d["flow10_ck"] = take(F, links), checksums(F)
    p, q, e = ref.flow_rk3_measure(U, 0.01, 2, 5)
    d["flowm_plaq"], d["flowm_q"], d["flowm_e"] = p, q, e
    St = ref.stout(U, 0.12, 4)
    d["stout4"], d["stout4_ck"] = take(St, links), checksums(St)
    G = ref.gauge_force(U, BETA)
    d["gforce"], d["gforce_ck"] = take(G, links), checksums(G)
    if full:
        D = ref.clover_derivative(U)
        d["cderiv"], d["cderiv_ck"] = take(D, links), checksums(D)
        M, qm = ref.metad_force(U, 0.12, 1.0)
        d["metad"], d["metad_ck"], d["metad_q"] = take(M, links), checksums(M), np.array(qm)
        d["metad_nstout"] = np.array(ref.lib.ref_n_smear_meta())
        P = random_momenta(V, seed + 7)
        d["P"] = P
        U2, P2, ho, hn = ref.omf2(U, P, BETA, 1.0, 10)
        d["omf2_U"], d["omf2_P"], d["omf2_h"] = take(U2, links), take(P2, links), np.array([ho, hn])
        U3, P3, ho3, hn3 = ref.metad_omf2(U, P, BETA, 1.0, 4, 0.12, 0.5)
        d["momf2_U"], d["momf2_P"], d["momf2_h"] = take(U3, links), take(P3, links), np.array([ho3, hn3])
        Hm = hermitian_inputs(64, seed + 3)
        d["exp_in"], d["exp_out"] = Hm, ref.su3_exp(Hm.reshape(-1)).reshape(Hm.shape)
    return d


def gen_bias() -> dict:
    import ctypes as C  # noqa: F401
    ref = Reference((4, 4, 4, 4))
    rng = np.random.default_rng(11)
    deposits = np.concatenate([rng.normal(0.0, 1.5, 40), [7.99, -8.5, 9.0]])
    probes = np.concatenate([np.linspace(-9.0, 9.0, 181), [-8.0, 8.0, 7.99, -7.995]])
    out = {}
    for sym in (0, 1):
        pot, der = np.empty(probes.size), np.empty(probes.size)
        ref.lib.ref_bias_probe(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0, deposits, deposits.size, sym,
                               probes, probes.size, pot, der)
        out[f"pot{sym}"], out[f"der{sym}"] = pot, der
    out["deposits"], out["probes"] = deposits, probes
    return out


def gen_chain(n_chain: int = 4, n_therm: int = 300, n_meas: int = 2500) -> dict:
    """Reference heatbath + overrelaxation chains at 8^4, beta = 6 (1 + 4 sweeps per round):
    plaquette histories of n_chain chains with independent pcg64 streams and Haar starts."""
    import ctypes as C
    ext = (8, 8, 8, 8)
    ref = Reference(ext)
    ref.lib.ref_reseed.argtypes = [C.c_uint64]
    V = int(np.prod(ext))
    hist = np.empty((n_chain, n_meas))
    for c in range(n_chain):
        ref.lib.ref_reset_prng()
        ref.lib.ref_reseed(c + 1)
        U = haar_links_numpy(ext, 5 + c)
        U, _ = ref.hb_or_chain(U, BETA, n_therm, 1, 4)
        U, p = ref.hb_or_chain(U, BETA, n_meas, 1, 4)
        hist[c] = p / V / 18.0
    return {"plaq_norm": hist, "n_therm": np.array(n_therm), "beta": np.array(BETA)}


BMW_EXT = (2, 4, 6, 8)
BMW_SEED = 11


def gen_bmw() -> dict:
    """The reference's SaveConfigBMW / SaveConfigBMWFull output for a seeded Haar field on
    uneven extents: the two-row file is committed whole, the 18-real one by its digest."""
    import hashlib
    U = haar_links_numpy(BMW_EXT, BMW_SEED)
    ref = Reference(BMW_EXT)
    out = {"ext": np.array(BMW_EXT), "seed": np.array(BMW_SEED)}
    for full, name in ((False, "ref_2x4x6x8.bmw"), (True, "ref_2x4x6x8.18bmw")):
        path = os.path.join(HERE, name)
        assert ref.save_bmw(U, path, full)
        data = open(path, "rb").read()
        key = "full" if full else "two_row"
        out[f"sha256_{key}"] = np.array(hashlib.sha256(data).hexdigest())
        out[f"checksum_{key}"] = np.array(data[:4096].split(b"\n")[0].split()[-1].decode())
        ok, loaded = ref.load_bmw(path, full)
        assert ok
        out[f"loaded_ck_{key}"] = checksums(loaded)
        if full:
            os.remove(path)
    return out


def gen_measure() -> dict:
    """The reference's measurement bundle (SU3_main.cpp:89-235) and its four flow integrators on
    the 4x6x8x10 input (Haar seed 2) after 5 oracle heatbath sweeps (the tests regenerate it)."""
    from ltref import Oracle
    ext = (4, 6, 8, 10)
    U = Oracle().heatbath(ext, haar_links_numpy(ext, 2), 6.0, 5, 17, 0)
    ref = Reference(ext)
    m = ref.measure(U, 6.0)
    out = {"ext": np.array(ext), "U_ck": checksums(U)}
    for k, v in m.items():
        out[k] = np.array(v)
    # WilsonLoop<start, end, reset> with its chain kept between calls: the driver's doubling
    # sequence, a sequence with a non-power-of-two extension, and a reset away from the origin
    # followed by a non-contiguous extension
    Uc = np.ascontiguousarray(U)
    seqs = [[(0, 2, 1), (2, 4, 0), (4, 8, 0)], [(0, 3, 1), (3, 5, 0)], [(2, 3, 1), (5, 6, 0)]]
    out["wl_chain_seq"] = np.array([c for seq in seqs for c in seq])
    out["wl_chain"] = np.array([ref.lib.ref_wilson_loop_chain(Uc, a, b, r) for seq in seqs for (a, b, r) in seq])
    links = sample_links(int(np.prod(ext)), 5)
    out["links"] = links
    for integ in range(4):
        F = ref.flow(U, 0.02, 5, integ)
        out[f"flow{integ}"] = take(F, links)
        out[f"flow{integ}_ck"] = checksums(F)
    return out


def gen_md() -> dict:
    """The reference's eleven MD integrators (hmc_gauge.hpp:19-377, hmc_metadynamics.hpp:26-238;
    ids as LT_MD_*) from the measurement fixture's links and Philox momenta (seed 9, counter
    0), tau = 0.5 in 3 steps at beta = 6: gauge-only (ids 0-7) and under the linear bias
    0.7 * Q with n_smear_meta stout steps of rho = 0.12 (ids 0-5, 8-10); and ParityUpdate."""
    from ltref import Oracle
    ext = (4, 6, 8, 10)
    o = Oracle()
    U = o.heatbath(ext, haar_links_numpy(ext, 2), 6.0, 5, 17, 0)
    P = o.random_momenta(ext, 9, 0)
    ref = Reference(ext)
    links = sample_links(int(np.prod(ext)), 6)[:32]
    out = {"ext": np.array(ext), "U_ck": checksums(U), "P_ck": checksums(P), "links": links,
           "n_stout": np.array(ref.lib.ref_n_smear_meta()), "beta": np.array(6.0), "tau": np.array(0.5),
           "n_step": np.array(3), "rho": np.array(0.12), "slope": np.array(0.7)}
    cases = [(i, False) for i in range(8)] + [(i, True) for i in (0, 1, 2, 3, 4, 5, 8, 9, 10)]
    for integ, metad in cases:
        key = f"{'metad' if metad else 'gauge'}{integ}"
        U2, P2, ho, hn = ref.md_integrate(U, P, 6.0, 0.5, 3, integ, metad, 0.12, 0.7)
        out[key + "_U"], out[key + "_P"] = take(U2, links), take(P2, links)
        out[key + "_ck"] = np.concatenate([checksums(U2), checksums(P2)])
        out[key + "_h"] = np.array([ho, hn])
    R = ref.parity_update(U)
    out["parity_U"], out["parity_ck"] = take(R, links), checksums(R)
    return out


def gen_rect() -> dict:
    """Rectangular<2> gauge actions (rectangular_action.hpp:23-276: Luescher-Weisz, Iwasaki,
    DBW2) on the 8^4 input (Haar seed 4, 3 oracle heatbath sweeps at beta = 6): staples,
    2 overrelaxation sweeps over Iterator::Checkerboard4 (also with the Wilson action), gauge MD
    (OMF_4 for LW and Iwasaki, OMF_2 for DBW2; tau = 0.5, 3 steps, Philox momenta seed 9) and
    10 RK3 flow steps of 0.02."""
    from ltref import DBW2, IWASAKI, LUESCHER_WEISZ, WILSON, Oracle
    ext = (8, 8, 8, 8)
    o = Oracle()
    U = o.heatbath(ext, haar_links_numpy(ext, 4), 6.0, 3, 21, 0)
    P = o.random_momenta(ext, 9, 0)
    ref = Reference(ext)
    links = sample_links(int(np.prod(ext)), 8)[:32]
    out = {"ext": np.array(ext), "U_ck": checksums(U), "P_ck": checksums(P), "links": links}
    for name, act in (("lw", LUESCHER_WEISZ), ("iwasaki", IWASAKI), ("dbw2", DBW2), ("wilson", WILSON)):
        out[name + "_act"] = np.array(act)
        R = ref.overrelax4(U, 2, act)
        out[name + "_or4"], out[name + "_or4_ck"] = take(R, links), checksums(R)
        if name == "wilson":
            continue
        S = ref.action_staples(U, act)
        out[name + "_staple"], out[name + "_staple_ck"] = take(S, links), checksums(S)
        integ = 3 if name == "dbw2" else 5
        U2, P2, ho, hn = ref.md_action(U, P, 6.0, 0.5, 3, integ, act)
        out[name + "_md_integ"] = np.array(integ)
        out[name + "_md_U"], out[name + "_md_P"] = take(U2, links), take(P2, links)
        out[name + "_md_h"] = np.array([ho, hn])
        F = ref.flow_action(U, 0.02, 10, 2, act)
        out[name + "_flow"], out[name + "_flow_ck"] = take(F, links), checksums(F)
    return out


N_SAMPLE_LARGE = 256


def gen_large() -> dict:
    """The benchmarked 32^4 configuration: one overrelaxation sweep and 10 RK3 flow steps of
    the reference, one heatbath sweep of the C oracle (the GPU's Philox stream), and P, Q, E
    of the input, as 256 sampled links plus full-field checksums."""
    from ltref import Oracle
    o = Oracle()
    ext = (32, 32, 32, 32)
    V = int(np.prod(ext))
    ref = Reference(ext)
    U = large_input(ext, 32, 77, o)
    rng = np.random.default_rng(3232)
    links = np.sort(rng.choice(4 * V, size=N_SAMPLE_LARGE, replace=False))
    d = {"ext": np.array(ext, dtype=np.int32), "seed": np.array(32), "hb_seed": np.array(77), "links": links,
         "U_ck": checksums(U), "plaq": np.array(ref.plaquette_sum(U)), "Q": np.array(ref.topcharge(U)),
         "E": np.array(ref.energy(U))}
    O = ref.overrelax(U, 1)
    d["or1"], d["or1_ck"], d["or1_plaq"] = take(O, links), checksums(O), np.array(ref.plaquette_sum(O))
    del O
    F = ref.flow_rk3(U, 0.01, 10)
    d["flow10"], d["flow10_ck"] = take(F, links), checksums(F)
    d["flow10_plaq"], d["flow10_q"] = np.array(ref.plaquette_sum(F)), np.array(ref.topcharge(F))
    del F
    H = o.heatbath(ext, U, BETA, 1, 555, 3)
    d["hb1_oracle"], d["hb1_oracle_ck"] = take(H, links), checksums(H)
    return d


def gen_flow_large() -> dict:
    """The reference's FP64 RK3 flow (eps = 0.01) of the 32^4 parity input to t = 4, with
    the plaquette sum, clover Q and clover E at t = 0.5, 1, 1.5, ..., 4 (every 50 steps)."""
    ext = (32, 32, 32, 32)
    ref = Reference(ext)
    U = large_input(ext, 32, 77)
    p, q, e = ref.flow_rk3_measure(U, 0.01, 8, 50)
    return {"ext": np.array(ext, dtype=np.int32), "eps": np.array(0.01), "every": np.array(50),
            "t": 0.01 * 50 * np.arange(1, 9), "plaq": p, "Q": q, "E": e}


def gen_metad16() -> dict:
    """The reference's metadynamics force (4 stout steps of rho = 0.12, dV/dQ = 1) at 16^4."""
    ext = (16, 16, 16, 16)
    V = int(np.prod(ext))
    ref = Reference(ext)
    U = large_input(ext, 16, 7)
    links = sample_links(V, 1616)
    M, q = ref.metad_force(U, 0.12, 1.0)
    return {"ext": np.array(ext, dtype=np.int32), "seed": np.array(16), "hb_seed": np.array(7), "links": links,
            "U_ck": checksums(U), "metad": take(M, links), "metad_ck": checksums(M), "metad_q": np.array(q),
            "metad_nstout": np.array(ref.lib.ref_n_smear_meta()), "Q": np.array(ref.topcharge(U))}


def gen_tempering() -> dict:
    """MetadynamicsTemperingKernel::operator() of the reference (updates/tempering.hpp:51-72)
    on two thermalised 8^4 fields for five biases: flat, deposits at the candidate's charge
    (rejection), at the biased stream's charge (acceptance), CV_current beyond the grid (the
    wall), and a bias tuned so that exp(-dV) lies near the kernel's uniform."""
    from ltref import Oracle
    o = Oracle()
    ext = (8, 8, 8, 8)
    ref = Reference(ext)
    Ua = o.heatbath(ext, haar_links_numpy(ext, 81), BETA, 30, 5, 0)
    Ub = o.heatbath(ext, haar_links_numpy(ext, 82), BETA, 30, 6, 0)
    rho = 0.12
    probe = np.empty(6)
    ref.lib.ref_tempering(Ua.copy(), Ub.copy(), rho, 0.0, np.zeros(1), 0, probe)
    cv_new, q = probe[0], probe[3]
    cv_old = cv_new + 1.3
    cases = [(cv_old, np.zeros(0)), (cv_old, np.full(400, cv_new)), (cv_old, np.full(25, cv_old)),
             (9.5, np.full(5, cv_new)), (cv_new - 0.2, np.concatenate([np.full(3, cv_new), np.full(2, cv_new - 0.2)]))]
    res, dep_all, dep_n = [], [], []
    for cvo, dep in cases:
        out = np.empty(6)
        ref.lib.ref_tempering(Ua.copy(), Ub.copy(), rho, cvo, np.ascontiguousarray(dep) if dep.size else np.zeros(1),
                              int(dep.size), out)
        res.append(out)
        dep_all.append(dep)
        dep_n.append(dep.size)
    return {"ext": np.array(ext, dtype=np.int32), "rho": np.array(rho), "seeds": np.array([81, 82, 5, 6, 30]),
            "Ua_ck": checksums(Ua), "Ub_ck": checksums(Ub), "out": np.array(res),
            "deposits": np.concatenate(dep_all), "n_dep": np.array(dep_n), "cv_old": np.array([c for c, _ in cases]),
            "uniform": np.array(q)}


def gen_tensor() -> dict:
    """CalculateClover<1, 1> as a FullTensor4D and TopChargeClover(const FullTensor&) of the
    reference on a partly thermalised 4x6x8x10 field: 48 sampled sites (all 16 matrices each)
    and full-tensor checksums."""
    from ltref import Oracle
    ext = (4, 6, 8, 10)
    V = int(np.prod(ext))
    ref = Reference(ext)
    U = Oracle().heatbath(ext, haar_links_numpy(ext, 46), BETA, 3, 8, 0)
    T = np.empty((V, 4, 4, 3, 3, 2))
    q = ref.lib.ref_clover_tensor(U, T.reshape(-1))
    sites = np.sort(np.random.default_rng(4681).choice(V, size=48, replace=False))
    return {"ext": np.array(ext, dtype=np.int32), "seeds": np.array([46, 8, 3]), "U_ck": checksums(U),
            "sites": sites, "tensor": T[sites], "tensor_ck": checksums(T), "Q": np.array(q)}


def exp_inputs(seed: int) -> np.ndarray:
    """Traceless Hermitian matrices for every branch of the device exponential and of the
    reference's SU3::exp: generic (c1 > 1/2), the long (1/32 < c1 <= 1/2) and short series
    ranges, tiny arguments, negative determinants (sign flip), exactly degenerate spectra
    (theta = 0, w = 0: the Taylor branches of xi_0, xi_1), nearly degenerate ones, diagonal
    and zero matrices."""
    rng = np.random.default_rng(seed)
    out = []

    def herm(scale):
        M = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        H = 0.5 * (M + M.conj().T)
        H -= np.trace(H) / 3.0 * np.eye(3)
        return H / np.sqrt(0.5 * np.trace(H @ H).real) * scale   # scale = sqrt(c1)

    def rotate(D):
        M = rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))
        Q, _ = np.linalg.qr(M)
        return Q @ D @ Q.conj().T

    for s in (3.0, 1.5, 0.9, 0.7, 0.6, 0.5, 0.35, 0.2, 0.17, 0.12, 0.05, 1e-2, 1e-4, 1e-8):
        for _ in range(4):
            H = herm(s)
            out += [H, -H]
    for a in (0.4, 0.05, 1e-3, 1.2):
        D = np.diag([a, a, -2 * a]).astype(np.complex128)
        out += [D, -D, rotate(D), -rotate(D)]
        for eps in (1e-3, 1e-6, 1e-9):
            D2 = np.diag([a, a + eps * a, -2 * a - eps * a]).astype(np.complex128)
            out += [rotate(D2), -rotate(D2)]
    out.append(np.zeros((3, 3), dtype=np.complex128))
    A = np.array(out)
    r = np.empty(A.shape + (2,))
    r[..., 0], r[..., 1] = A.real, A.imag
    return r


def gen_exp() -> dict:
    ref = Reference((4, 4, 4, 4))
    Hm = exp_inputs(4242)
    return {"exp_in": Hm, "exp_out": ref.su3_exp(np.ascontiguousarray(Hm).reshape(-1)).reshape(Hm.shape)}


def main() -> int:
    import argparse
    import subprocess
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["chain", "bmw", "measure", "md", "rect", "large", "flow_large", "metad16",
                                       "exp", "tempering", "tensor"], default=None,
                    help="regenerate one fixture only")
    a = ap.parse_args()
    root = os.path.dirname(os.path.dirname(HERE))
    subprocess.run([sys.executable, os.path.join(root, "oracle", "build_ref.py"), "--extents", "4x4x4x4",
                    "4x6x8x10", "8x8x8x8", "2x4x6x8"], check=True)
    if a.only in ("large", "flow_large"):
        subprocess.run([sys.executable, os.path.join(root, "oracle", "build_ref.py"), "--extents", "32x32x32x32"],
                       check=True)
        out = gen_large() if a.only == "large" else gen_flow_large()
        name = "ref_32x32x32x32.npz" if a.only == "large" else "ref_flow_32x32x32x32.npz"
        np.savez_compressed(os.path.join(HERE, name), **out)
        return 0
    if a.only == "metad16":
        subprocess.run([sys.executable, os.path.join(root, "oracle", "build_ref.py"), "--extents", "16x16x16x16"],
                       check=True)
        np.savez_compressed(os.path.join(HERE, "ref_metad_16x16x16x16.npz"), **gen_metad16())
        return 0
    if a.only == "tensor":
        np.savez_compressed(os.path.join(HERE, "ref_tensor_4x6x8x10.npz"), **gen_tensor())
        return 0
    if a.only == "tempering":
        np.savez_compressed(os.path.join(HERE, "ref_tempering.npz"), **gen_tempering())
        return 0
    if a.only == "exp":
        np.savez_compressed(os.path.join(HERE, "ref_exp.npz"), **gen_exp())
        return 0
    if a.only == "chain":
        np.savez_compressed(os.path.join(HERE, "ref_chain_8x8x8x8.npz"), **gen_chain())
        return 0
    if a.only == "measure":
        np.savez_compressed(os.path.join(HERE, "ref_measure.npz"), **gen_measure())
        return 0
    if a.only == "rect":
        np.savez_compressed(os.path.join(HERE, "ref_rect.npz"), **gen_rect())
        return 0
    if a.only == "md":
        np.savez_compressed(os.path.join(HERE, "ref_md.npz"), **gen_md())
        return 0
    if a.only == "bmw":
        np.savez_compressed(os.path.join(HERE, "ref_bmw.npz"), **gen_bmw())
        return 0
    np.savez_compressed(os.path.join(HERE, "ref_4x4x4x4.npz"), **gen_case((4, 4, 4, 4), 1, True))
    b = gen_case((4, 6, 8, 10), 2, False)
    del b["U"]   # regenerated from numpy's seeded generator; checksum kept
    U = haar_links_numpy((4, 6, 8, 10), 2)
    b["U_ck"] = checksums(U)
    np.savez_compressed(os.path.join(HERE, "ref_4x6x8x10.npz"), **b)
    np.savez_compressed(os.path.join(HERE, "ref_bias.npz"), **gen_bias())
    np.savez_compressed(os.path.join(HERE, "ref_chain_8x8x8x8.npz"), **gen_chain())
    np.savez_compressed(os.path.join(HERE, "ref_bmw.npz"), **gen_bmw())
    np.savez_compressed(os.path.join(HERE, "ref_measure.npz"), **gen_measure())
    np.savez_compressed(os.path.join(HERE, "ref_md.npz"), **gen_md())
    np.savez_compressed(os.path.join(HERE, "ref_rect.npz"), **gen_rect())
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
    return 0


if __name__ == "__main__":
    sys.exit(main())
