"""ctypes bindings for the checkers used by the tests: the C restatement in oracle/ and the
compiled reference harness in oracle/_ref/ (both test infrastructure, never the product).

Fields are numpy float64 arrays in the reference AoS layout [V, 4, 3, 3, 2]
(LettuceGauge/lattice.hpp:366-382).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build_oracle() -> str:
    """Compile oracle/lt_oracle.c into oracle/liblt_oracle.so (plain gcc)."""
    src = os.path.join(ORACLE_DIR, "lt_oracle.c")
    out = os.path.join(ORACLE_DIR, "liblt_oracle.so")
    if not os.path.exists(out) or os.path.getmtime(out) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(ORACLE_DIR, "lt_oracle.h"))):
        subprocess.run(["gcc", "-std=c99", "-O2", "-fPIC", "-shared", "-ffp-contract=off",
                        "-o", out, src, "-lm"], check=True)
    return out


class Oracle:
    """The C restatement (oracle/lt_oracle.c) with runtime extents."""

    def __init__(self):
        lib = C.CDLL(build_oracle())
        d, i, u64 = C.c_double, C.c_int, C.c_uint64
        sig = {
            "or_plaquette_sum": (d, [_ip, _dp]),
            "or_wilson_action": (d, [_ip, _dp, d]),
            "or_staples": (None, [_ip, _dp, _dp]),
            "or_overrelax_sweeps": (None, [_ip, _dp, i]),
            "or_heatbath_sweeps": (None, [_ip, _dp, d, i, u64, u64]),
            "or_su3_exp": (None, [_dp, _dp, i]),
            "or_flow_rk3": (None, [_ip, _dp, _dp, d, i]),
            "or_stout": (None, [_ip, _dp, _dp, d, i]),
            "or_topcharge_clover": (d, [_ip, _dp]),
            "or_energy_clover": (d, [_ip, _dp]),
            "or_gauge_force": (None, [_ip, _dp, d, _dp]),
            "or_clover_derivative": (None, [_ip, _dp, _dp]),
            "or_metad_force": (d, [_ip, _dp, d, i, d, _dp]),
            "or_metad_charge": (d, [_ip, _dp, d, i]),
            "or_omf2": (None, [_ip, _dp, _dp, d, d, i, C.POINTER(d), C.POINTER(d)]),
            "or_random_momenta": (None, [_ip, _dp, u64, u64]),
            "or_kinetic": (d, [_ip, _dp]),
            "or_bias_create": (C.c_void_p, [d, d, i, d, d, d, d]),
            "or_bias_destroy": (None, [C.c_void_p]),
            "or_bias_update": (None, [C.c_void_p, d]),
            "or_bias_update_symmetric": (None, [C.c_void_p, d]),
            "or_bias_update_binned": (None, [C.c_void_p, d]),
            "or_bias_potential": (d, [C.c_void_p, d]),
            "or_bias_derivative": (d, [C.c_void_p, d]),
            "or_bmw_encode": (u64, [_ip, _dp, i, C.c_void_p]),
            "or_flow": (None, [_ip, _dp, _dp, d, i, i]),
            "or_flow_zeuthen": (None, [_ip, _dp, _dp, d, i, i]),
            "or_clover_timeslices": (None, [_ip, _dp, _dp, _dp]),
            "or_topcharge_plaquette": (d, [_ip, _dp]),
            "or_rect_action": (d, [_ip, _dp, d, d, d]),
            "or_wilson_loop": (d, [_ip, _dp, i]),
            "or_polyakov_loop": (None, [_ip, _dp, C.POINTER(d), C.POINTER(d)]),
            "or_bmw_decode": (u64, [_ip, C.c_void_p, i, _dp]),
            "or_md_integrate": (None, [_ip, _dp, _dp, d, d, i, i, i, d, i, d, C.POINTER(d), C.POINTER(d)]),
            "or_parity_update": (None, [_ip, _dp]),
            "or_set_gauge_action": (None, [i, d, d]),
            "or_overrelax_sweeps4": (None, [_ip, _dp, i]),
            "or_heatbath_sweeps4": (None, [_ip, _dp, d, i, u64, u64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        self.lib = lib

    @staticmethod
    def _e(ext):
        return np.ascontiguousarray(ext, dtype=np.int32)

    @contextlib.contextmanager
    def action(self, act):
        """Run the block under GaugeAction::Rectangular act = (radius, c_plaq, c_rect) (None:
        WilsonAction); the Wilson action is restored afterwards."""
        if act is not None:
            self.lib.or_set_gauge_action(int(act[0]), float(act[1]), float(act[2]))
        try:
            yield
        finally:
            self.lib.or_set_gauge_action(1, 1.0, 0.0)

    def action_staples(self, ext, U, act):
        with self.action(act):
            return self.staples(ext, np.ascontiguousarray(U))

    def overrelax4(self, ext, U, n, act=None):
        V = np.ascontiguousarray(U).copy()
        with self.action(act):
            self.lib.or_overrelax_sweeps4(self._e(ext), V, n)
        return V

    def heatbath4(self, ext, U, beta, n, seed, counter, act=None):
        V = np.ascontiguousarray(U).copy()
        with self.action(act):
            self.lib.or_heatbath_sweeps4(self._e(ext), V, beta, n, seed, counter)
        return V

    def md_integrate_action(self, ext, U, P, beta, tau, n, integrator, act):
        with self.action(act):
            return self.md_integrate(ext, U, P, beta, tau, n, integrator)

    def flow_action(self, ext, U, eps, n, integrator, act):
        with self.action(act):
            return self.flow(ext, U, eps, n, integrator)

    def plaquette_sum(self, ext, U):
        return self.lib.or_plaquette_sum(self._e(ext), U)

    def wilson_action(self, ext, U, beta):
        return self.lib.or_wilson_action(self._e(ext), U, beta)

    def staples(self, ext, U):
        out = np.empty_like(U)
        self.lib.or_staples(self._e(ext), U, out)
        return out

    def overrelax(self, ext, U, n):
        V = U.copy()
        self.lib.or_overrelax_sweeps(self._e(ext), V, n)
        return V

    def heatbath(self, ext, U, beta, n, seed, counter):
        V = U.copy()
        self.lib.or_heatbath_sweeps(self._e(ext), V, beta, n, seed, counter)
        return V

    def su3_exp(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        out = np.empty_like(Q)
        self.lib.or_su3_exp(Q, out, Q.size // 18)
        return out

    def flow_rk3(self, ext, U, eps, n):
        out = np.empty_like(U)
        self.lib.or_flow_rk3(self._e(ext), U, out, eps, n)
        return out

    def stout(self, ext, U, rho, n):
        out = np.empty_like(U)
        self.lib.or_stout(self._e(ext), U, out, rho, n)
        return out

    def topcharge(self, ext, U):
        return self.lib.or_topcharge_clover(self._e(ext), U)

    def energy(self, ext, U):
        return self.lib.or_energy_clover(self._e(ext), U)

    def gauge_force(self, ext, U, beta):
        out = np.empty_like(U)
        self.lib.or_gauge_force(self._e(ext), U, beta, out)
        return out

    def clover_derivative(self, ext, U):
        out = np.empty_like(U)
        self.lib.or_clover_derivative(self._e(ext), U, out)
        return out

    def metad_force(self, ext, U, rho, n_stout, dvdq=1.0):
        out = np.empty_like(U)
        q = self.lib.or_metad_force(self._e(ext), U, rho, n_stout, dvdq, out)
        return out, q

    def metad_charge(self, ext, U, rho, n_stout):
        return self.lib.or_metad_charge(self._e(ext), U, rho, n_stout)

    def omf2(self, ext, U, P, beta, tau, n):
        U2, P2 = U.copy(), P.copy()
        ho, hn = C.c_double(), C.c_double()
        self.lib.or_omf2(self._e(ext), U2, P2, beta, tau, n, C.byref(ho), C.byref(hn))
        return U2, P2, ho.value, hn.value

    def md_integrate(self, ext, U, P, beta, tau, n, integrator, metad=False, rho=0.12, n_stout=0, slope=0.0):
        """(U, P, H_old, H_new) after n steps of integrator (ids as LT_MD_*); MetaD with the
        linear bias slope * Q."""
        U2, P2 = np.ascontiguousarray(U).copy(), np.ascontiguousarray(P).copy()
        ho, hn = C.c_double(), C.c_double()
        self.lib.or_md_integrate(self._e(ext), U2, P2, beta, tau, n, integrator, int(metad), rho, n_stout, slope,
                                 C.byref(ho), C.byref(hn))
        return U2, P2, ho.value, hn.value

    def parity_update(self, ext, U):
        V = np.ascontiguousarray(U).copy()
        self.lib.or_parity_update(self._e(ext), V)
        return V

    def random_momenta(self, ext, seed, counter):
        V = int(np.prod(ext))
        P = np.empty((V, 4, 3, 3, 2))
        self.lib.or_random_momenta(self._e(ext), P, seed, counter)
        return P

    def flow(self, ext, U, eps, n, integrator):
        out = np.empty_like(U)
        self.lib.or_flow(self._e(ext), np.ascontiguousarray(U), out, eps, n, integrator)
        return out

    def flow_zeuthen(self, ext, U, eps, n, integrator=2):
        out = np.empty_like(U)
        self.lib.or_flow_zeuthen(self._e(ext), np.ascontiguousarray(U), out, eps, n, integrator)
        return out

    def measure(self, ext, U, beta=6.0):
        """The bundle of SU3_main.cpp:89-235 on one field: dict of the observables."""
        U = np.ascontiguousarray(U)
        e = self._e(ext)
        qt, et = np.empty(ext[0]), np.empty(ext[0])
        self.lib.or_clover_timeslices(e, U, qt, et)
        re, im = C.c_double(), C.c_double()
        self.lib.or_polyakov_loop(e, U, C.byref(re), C.byref(im))
        V = int(np.prod(ext))
        return {"q_t": qt, "e_t": et, "Q_plaq": self.lib.or_topcharge_plaquette(e, U),
                "S_improved": self.lib.or_rect_action(e, U, beta, 1 + 8 / 12, -1 / 12) / (6 * beta * V),
                "W2": self.lib.or_wilson_loop(e, U, 2), "W4": self.lib.or_wilson_loop(e, U, 4),
                "W8": self.lib.or_wilson_loop(e, U, 8), "P": complex(re.value, im.value)}

    def bmw_encode(self, ext, U, full):
        """(Adler-64 checksum, BMW payload bytes) of a field in the reference layout."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        V = int(np.prod(ext))
        payload = np.empty(V * 4 * (18 if full else 12) * 8, dtype=np.uint8)
        ck = self.lib.or_bmw_encode(self._e(ext), U, int(full), payload.ctypes.data)
        return ck, payload.tobytes()

    def bmw_decode(self, ext, payload, full):
        """(Adler-64 checksum, links) of a BMW payload."""
        V = int(np.prod(ext))
        buf = np.frombuffer(payload, dtype=np.uint8).copy()
        U = np.empty((V, 4, 3, 3, 2))
        ck = self.lib.or_bmw_decode(self._e(ext), buf.ctypes.data, int(full), U)
        return ck, U

    def kinetic(self, ext, P):
        return self.lib.or_kinetic(self._e(ext), P)


def ref_available(ext) -> bool:
    return os.path.exists(ref_lib_path(ext))


def ref_lib_path(ext) -> str:
    return os.path.join(REF_DIR, "liblt_ref_%s.so" % "x".join(str(int(e)) for e in ext))


class Reference:
    """The reference's own code, compiled per extent tuple by oracle/build_ref.py."""

    _cache: dict = {}

    def __init__(self, ext):
        key = tuple(int(e) for e in ext)
        if key not in Reference._cache:
            lib = C.CDLL(ref_lib_path(key))
            d, i = C.c_double, C.c_int
            sig = {
                "ref_extent": (i, [i]), "ref_threads": (i, []),
                "ref_plaquette_sum": (d, [_dp]), "ref_wilson_action": (d, [_dp, d]),
                "ref_staples": (None, [_dp, _dp]), "ref_or_sweeps": (None, [_dp, i]),
                "ref_reset_prng": (None, []), "ref_hb_sweeps": (None, [_dp, d, i]),
                "ref_hb_or_chain": (None, [_dp, d, i, i, i, _dp]),
                "ref_flow_rk3": (None, [_dp, _dp, d, i]),
                "ref_flow_rk3_measure": (None, [_dp, d, i, i, _dp, _dp, _dp]),
                "ref_stout": (None, [_dp, _dp, d, i]),
                "ref_topcharge_clover": (d, [_dp]), "ref_energy_clover": (d, [_dp]),
                "ref_gauge_force": (None, [_dp, d, _dp]),
                "ref_clover_derivative": (None, [_dp, _dp]),
                "ref_metad_force": (d, [_dp, d, d, _dp]),
                "ref_metad_charge": (d, [_dp, d]),
                "ref_n_smear_meta": (i, []),
                "ref_omf2": (None, [_dp, _dp, d, d, i, C.POINTER(d), C.POINTER(d)]),
                "ref_metad_omf2": (None, [_dp, _dp, d, d, i, d, d, C.POINTER(d), C.POINTER(d)]),
                "ref_bias_probe": (None, [d, d, i, d, d, d, d, _dp, i, i, _dp, i, _dp, _dp]),
                "ref_su3_exp": (None, [_dp, _dp, i]),
                "ref_save_bmw": (i, [_dp, C.c_char_p, i]),
                "ref_flow": (None, [_dp, _dp, d, i, i]),
                "ref_measure": (None, [_dp, d, _dp, _dp, _dp]),
                "ref_load_bmw": (i, [C.c_char_p, i, _dp]),
                "ref_md_integrate": (i, [_dp, _dp, d, d, i, i, i, d, d, C.POINTER(d), C.POINTER(d)]),
                "ref_parity_update": (None, [_dp]),
                "ref_action_staples": (None, [_dp, _dp, i, d, d]),
                "ref_or_sweeps4": (i, [_dp, i, i, d, d]),
                "ref_md_action": (i, [_dp, _dp, d, d, i, i, i, d, d, C.POINTER(d), C.POINTER(d)]),
                "ref_flow_action": (None, [_dp, _dp, d, i, i, i, d, d]),
                "ref_wilson_loop_chain": (d, [_dp, i, i, i]),
                "ref_tempering": (None, [_dp, _dp, d, d, _dp, i, _dp]),
                "ref_clover_tensor": (d, [_dp, _dp]),
            }
            for name, (res, args) in sig.items():
                f = getattr(lib, name)
                f.restype = res
                f.argtypes = args
            Reference._cache[key] = lib
        self.lib = Reference._cache[key]
        self.ext = key

    def plaquette_sum(self, U):
        return self.lib.ref_plaquette_sum(U)

    def wilson_action(self, U, beta):
        return self.lib.ref_wilson_action(U, beta)

    def staples(self, U):
        out = np.empty_like(U)
        self.lib.ref_staples(U, out)
        return out

    def overrelax(self, U, n):
        V = U.copy()
        self.lib.ref_or_sweeps(V, n)
        return V

    def hb_or_chain(self, U, beta, n_sweep, n_hb, n_or):
        V = U.copy()
        plaq = np.empty(n_sweep)
        self.lib.ref_hb_or_chain(V, beta, n_sweep, n_hb, n_or, plaq)
        return V, plaq

    def flow_rk3(self, U, eps, n):
        out = np.empty_like(U)
        self.lib.ref_flow_rk3(U, out, eps, n)
        return out

    def flow_rk3_measure(self, U, eps, n_meas, every):
        p, q, e = np.empty(n_meas), np.empty(n_meas), np.empty(n_meas)
        self.lib.ref_flow_rk3_measure(U, eps, n_meas, every, p, q, e)
        return p, q, e

    def stout(self, U, rho, n):
        out = np.empty_like(U)
        self.lib.ref_stout(U, out, rho, n)
        return out

    def topcharge(self, U):
        return self.lib.ref_topcharge_clover(U)

    def energy(self, U):
        return self.lib.ref_energy_clover(U)

    def gauge_force(self, U, beta):
        out = np.empty_like(U)
        self.lib.ref_gauge_force(U, beta, out)
        return out

    def clover_derivative(self, U):
        out = np.empty_like(U)
        self.lib.ref_clover_derivative(U, out)
        return out

    def metad_force(self, U, rho, slope=1.0):
        out = np.empty_like(U)
        q = self.lib.ref_metad_force(U, rho, slope, out)
        return out, q

    def metad_charge(self, U, rho):
        return self.lib.ref_metad_charge(U, rho)

    def omf2(self, U, P, beta, tau, n):
        U2, P2 = U.copy(), P.copy()
        ho, hn = C.c_double(), C.c_double()
        self.lib.ref_omf2(U2, P2, beta, tau, n, C.byref(ho), C.byref(hn))
        return U2, P2, ho.value, hn.value

    def metad_omf2(self, U, P, beta, tau, n, rho, slope):
        U2, P2 = U.copy(), P.copy()
        ho, hn = C.c_double(), C.c_double()
        self.lib.ref_metad_omf2(U2, P2, beta, tau, n, rho, slope, C.byref(ho), C.byref(hn))
        return U2, P2, ho.value, hn.value

    def md_integrate(self, U, P, beta, tau, n, integrator, metad=False, rho=0.12, slope=0.0):
        """The reference's integrator `integrator` (LT_MD_* ids) on HMCKernel or, with metad,
        HMCMetaDKernel under V(Q) = slope * Q (n_smear_meta stout steps of rho)."""
        U2, P2 = np.ascontiguousarray(U).copy(), np.ascontiguousarray(P).copy()
        ho, hn = C.c_double(), C.c_double()
        ok = self.lib.ref_md_integrate(U2, P2, beta, tau, n, integrator, int(metad), rho, slope, C.byref(ho),
                                       C.byref(hn))
        if not ok:
            raise ValueError("the reference has no such integrator/kernel combination")
        return U2, P2, ho.value, hn.value

    def parity_update(self, U):
        V = np.ascontiguousarray(U).copy()
        self.lib.ref_parity_update(V)
        return V

    def action_staples(self, U, act):
        out = np.empty_like(U)
        self.lib.ref_action_staples(np.ascontiguousarray(U), out, int(act[0]), float(act[1]), float(act[2]))
        return out

    def overrelax4(self, U, n, act):
        V = np.ascontiguousarray(U).copy()
        if not self.lib.ref_or_sweeps4(V, n, int(act[0]), float(act[1]), float(act[2])):
            raise ValueError("Checkerboard4 needs every extent a multiple of 4")
        return V

    def md_action(self, U, P, beta, tau, n, integrator, act):
        U2, P2 = np.ascontiguousarray(U).copy(), np.ascontiguousarray(P).copy()
        ho, hn = C.c_double(), C.c_double()
        if not self.lib.ref_md_action(U2, P2, beta, tau, n, integrator, int(act[0]), float(act[1]), float(act[2]),
                                      C.byref(ho), C.byref(hn)):
            raise ValueError("no such gauge integrator")
        return U2, P2, ho.value, hn.value

    def flow_action(self, U, eps, n, integrator, act):
        out = np.empty_like(U)
        self.lib.ref_flow_action(np.ascontiguousarray(U), out, eps, n, integrator, int(act[0]), float(act[1]),
                                 float(act[2]))
        return out

    def su3_exp(self, Q):
        Q = np.ascontiguousarray(Q, dtype=np.float64)
        out = np.empty_like(Q)
        self.lib.ref_su3_exp(Q, out, Q.size // 18)
        return out

    def flow(self, U, eps, n, integrator):
        out = np.empty_like(U)
        self.lib.ref_flow(np.ascontiguousarray(U), out, eps, n, integrator)
        return out

    def measure(self, U, beta=6.0):
        out, qt, et = np.empty(7), np.empty(self.ext[0]), np.empty(self.ext[0])
        self.lib.ref_measure(np.ascontiguousarray(U), beta, out, qt, et)
        return {"q_t": qt, "e_t": et, "S_improved": out[0], "Q_plaq": out[1], "W2": out[2], "W4": out[3],
                "W8": out[4], "P": complex(out[5], out[6])}

    def save_bmw(self, U, path, full):
        return bool(self.lib.ref_save_bmw(np.ascontiguousarray(U, dtype=np.float64), str(path).encode(), int(full)))

    def load_bmw(self, path, full):
        V = int(np.prod(self.ext))
        out = np.empty((V, 4, 3, 3, 2))
        ok = bool(self.lib.ref_load_bmw(str(path).encode(), int(full), out))
        return ok, out


def bmw_header(ext, checksum: int, full: bool) -> bytes:
    """The 4096-byte header SaveConfigBMW / SaveConfigBMWFull write (bmw_format.hpp:346-363)."""
    h = bytearray(b"\n" * 4096)
    line = f"{'#18BMW' if full else '#BMW'} {ext[1]} {ext[2]} {ext[3]} {ext[0]} {checksum:x}\n".encode()
    tail = b"\nGenerated with Lettuce\n\0"
    h[:len(line)] = line
    h[len(line):len(line) + len(tail)] = tail
    return bytes(h)


# GaugeAction named actions (rectangular_action.hpp:273-276) as (stencil radius, c_plaq, c_rect)
WILSON = (1, 1.0, 0.0)
LUESCHER_WEISZ = (2, 1.0 + 8.0 / 12.0, -1.0 / 12.0)
IWASAKI = (2, 1.0 + 8.0 * 0.331, -0.331)
DBW2 = (2, 1.0 + 8.0 * 1.4088, -1.4088)


def haar_links_numpy(ext, seed):
    """Haar-random SU(3) links (Mezzadri's QR method) from numpy's PCG64, used only to
    drive oracle-vs-reference pins that need no product code."""
    rng = np.random.default_rng(seed)
    V = int(np.prod(ext))
    Z = (rng.standard_normal((V * 4, 3, 3)) + 1j * rng.standard_normal((V * 4, 3, 3))) / np.sqrt(2)
    Q, R = np.linalg.qr(Z)
    d = np.diagonal(R, axis1=1, axis2=2)
    Q = Q * (d / np.abs(d))[:, None, :]
    det = np.linalg.det(Q)
    Q = Q / (det ** (1.0 / 3.0))[:, None, None]
    out = np.empty((V, 4, 3, 3, 2))
    Qr = Q.reshape(V, 4, 3, 3)
    out[..., 0] = Qr.real
    out[..., 1] = Qr.imag
    return out


def checksums(field: np.ndarray) -> np.ndarray:
    """Size-independent summary of a full field: sum, sum of squares, index-weighted sum."""
    f = np.asarray(field, dtype=np.float64).reshape(-1)
    w = np.arange(f.size, dtype=np.float64) % 97.0
    return np.array([f.sum(), (f * f).sum(), (w * f).sum()])


def large_input(ext, seed: int, hb_seed: int, oracle=None) -> np.ndarray:
    """Input of the full-size parity fixtures: numpy Haar start, then one heatbath sweep of
    the C oracle (Philox stream hb_seed, beta = 6), so that no SU(2) projection of the first
    overrelaxation sweep is near-singular.  Regenerated bit for bit on any host by the same
    two calls."""
    o = oracle or Oracle()
    return o.heatbath(ext, haar_links_numpy(ext, seed), 6.0, 1, hb_seed, 0)


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
