"""Python mirror of the reference's call surface over the C ABI.

Names, argument meaning and error behaviour follow timo-eichhorn/Lettuce (paths relative to
the reference project root); every call goes to liblettuce_b200.so.  Fields cross in the
reference layout, numpy float64 arrays of shape [V, 4, 3, 3, 2].
"""
from __future__ import annotations

import ctypes as C
import os
from types import SimpleNamespace

import numpy as np

from ._lib import PREC, LettuceError, check, lib


def _ext(ext) -> np.ndarray:
    e = np.ascontiguousarray([int(v) for v in ext], dtype=np.int32)
    if e.shape != (4,):
        raise ValueError("extents must be (Nt, Nx, Ny, Nz)")
    return e


def haar_links(ext, seed: int) -> np.ndarray:
    """Seeded Haar-random SU(3) links in the reference layout (host generator)."""
    e = _ext(ext)
    out = np.empty((int(np.prod(e)), 4, 3, 3, 2))
    check(lib().lt_haar_links(e, C.c_uint64(seed), out))
    return out


class GaugeField:
    """GaugeField4D (LettuceGauge/lattice.hpp:87-394) resident on the GPU."""

    def __init__(self, ext, prec: str = "fp64"):
        self.ext = tuple(int(v) for v in ext)
        self.prec = prec
        h = C.c_void_p()
        check(lib().lt_create(_ext(ext), PREC[prec], C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().lt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def Volume(self) -> int:
        return int(np.prod(self.ext))

    def SpatialVolume(self) -> int:
        return int(np.prod(self.ext[1:]))

    def Length(self, d: int) -> int:
        return self.ext[d]

    def upload(self, links: np.ndarray) -> None:
        a = np.ascontiguousarray(links, dtype=np.float64)
        if a.size != self.Volume() * 72:
            raise ValueError("link array has the wrong size")
        check(lib().lt_upload_links(self._h, a.reshape(-1)))

    def upload_bytes(self, links: np.ndarray) -> int:
        """Bytes the next upload(links) copies host to device (lt_upload_bytes)."""
        a = np.ascontiguousarray(links, dtype=np.float64)
        n = C.c_uint64()
        check(lib().lt_upload_bytes(self._h, a.reshape(-1), C.byref(n)))
        return int(n.value)

    def download(self) -> np.ndarray:
        out = np.empty((self.Volume(), 4, 3, 3, 2))
        check(lib().lt_download_links(self._h, out.reshape(-1)))
        return out

    def get_link(self, site: int, mu: int) -> np.ndarray:
        """operator()(link_coord) read (lattice.hpp:113-136): 3x3 complex."""
        m = np.empty(18)
        check(lib().lt_get_link(self._h, int(site), int(mu), m))
        return (m[0::2] + 1j * m[1::2]).reshape(3, 3)

    def set_link(self, site: int, mu: int, M) -> None:
        M = np.asarray(M, dtype=np.complex128).reshape(9)
        m = np.empty(18)
        m[0::2], m[1::2] = M.real, M.imag
        check(lib().lt_set_link(self._h, int(site), int(mu), m))

    def assign(self, other: "GaugeField") -> None:
        """operator= (lattice.hpp:106-112)."""
        check(lib().lt_copy(self._h, other._h))

    def SetToIdentity(self) -> None:
        check(lib().lt_set_identity(self._h))

    def SetToHaarRandom(self, seed: int) -> None:
        check(lib().lt_set_haar_random(self._h, C.c_uint64(seed)))

    def synchronize(self) -> None:
        check(lib().lt_synchronize(self._h))

    @property
    def stream(self) -> int:
        """The handle's cudaStream_t as an integer (for event timing on that stream)."""
        s = C.c_void_p()
        check(lib().lt_get_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def status_word(self, clear: bool = False) -> int:
        """The device status word (STATUS_* bits); clear=True resets it."""
        w = C.c_uint32()
        check(lib().lt_status_word(self._h, C.byref(w), int(bool(clear))))
        return w.value

    def save_bmw(self, path, full: bool = False, overwrite: bool = False) -> str:
        """SaveConfigBMW / SaveConfigBMWFull (IO/config_io/bmw_format.hpp:294-394, :564-645);
        returns the header's checksum string."""
        buf = C.create_string_buffer(17)
        check(lib().lt_save_bmw(self._h, os.fsencode(path), int(bool(full)), int(bool(overwrite)), buf))
        return buf.value.decode()

    def load_bmw(self, path, full: bool = False) -> tuple[bool, bool]:
        """LoadConfigBMW / LoadConfigBMWFull (bmw_format.hpp:153-290, :425-560); returns
        (checksum matches the header, every link passes IsGroupElement)."""
        ok, grp = C.c_int(), C.c_int()
        check(lib().lt_load_bmw(self._h, os.fsencode(path), int(bool(full)), C.byref(ok), C.byref(grp)))
        return bool(ok.value), bool(grp.value)

    def bmw_checksum(self, full: bool = False) -> int:
        """Checksum_Adler64 of the links as a BMW file would hold them."""
        v = C.c_uint64()
        check(lib().lt_bmw_checksum(self._h, int(bool(full)), C.byref(v)))
        return v.value

    def check_links(self) -> float:
        """Largest entry of |U U^dag - 1| over all links; flags NaN/Inf and unitarity loss."""
        d = C.c_double()
        check(lib().lt_check_links(self._h, C.byref(d)))
        return d.value


def Swap(U1: GaugeField, U2: GaugeField) -> None:
    """Swap (lattice.hpp:238-246): exchanges the link storage."""
    check(lib().lt_swap(U1.handle, U2.handle))


def _out1(fn, *args) -> float:
    v = C.c_double()
    check(fn(*args, C.byref(v)))
    return v.value


def PlaquetteSum(U: GaugeField) -> float:
    """observables/plaquette.hpp:26-43."""
    return _out1(lib().lt_plaquette_sum, U.handle)


class FullTensor:
    """FullTensor4D (lattice.hpp:447-590): 16 3x3 complex matrices per site in the reference
    layout [V, 4, 4, 3, 3, 2] (host memory).  CalculateClover fills it; TopChargeClover accepts
    it as the reference's TopChargeClover(const FullTensor&) does."""

    def __init__(self, ext):
        self.ext = tuple(int(e) for e in ext)
        self.data = np.zeros((int(np.prod(self.ext)), 4, 4, 3, 3, 2))
        self._field = None

    def __call__(self, site: int, mu: int, nu: int) -> np.ndarray:
        m = self.data[site, mu, nu]
        return m[..., 0] + 1j * m[..., 1]


def CalculateClover(U: GaugeField, Clov: "FullTensor | None" = None) -> FullTensor:
    """CalculateClover<1, 1> (observables/clover.hpp:94-152): the four-leaf clover C_{mu nu}
    of every site (C_{nu mu} = C_{mu nu}^dag, zero diagonal), FP64 products."""
    if Clov is None:
        Clov = FullTensor(U.ext)
    if Clov.ext != tuple(U.ext):
        raise ValueError("tensor and field extents differ")
    check(lib().lt_clover_tensor(U.handle, Clov.data.ctypes.data))
    Clov._field = U
    return Clov


def TopChargeClover(U) -> float:
    """observables/topological_charge.hpp:97-200 for a GaugeField; for a FullTensor,
    TopChargeClover(const FullTensor&) (:202-231) of the tensor as given."""
    if isinstance(U, FullTensor):
        h = U._field if U._field is not None else GaugeField(U.ext)
        q = C.c_double()
        data = np.ascontiguousarray(U.data)
        check(lib().lt_topcharge_clover_tensor(h.handle, data.ctypes.data, C.byref(q)))
        return q.value
    return _out1(lib().lt_topcharge_clover, U.handle)


def EnergyDensityClover(U: GaugeField) -> float:
    """EnergyDensity::Clover of the traceless clover field strength
    (observables/field_strength_tensor.hpp:154-175)."""
    return _out1(lib().lt_energy_clover, U.handle)


def CloverObservables(U: GaugeField) -> tuple[float, float]:
    q, e = C.c_double(), C.c_double()
    check(lib().lt_clover_observables(U.handle, C.byref(q), C.byref(e)))
    return q.value, e.value


def Staples(U: GaugeField) -> np.ndarray:
    """WilsonAction::Staple for every link (actions/gauge/rectangular_action.hpp:104-184)."""
    return WilsonAction().Staple(U)


def _set_action(U: GaugeField, action) -> None:
    """Make `action` (None: the Wilson action) the gauge action of U's device staples, sweeps,
    HMC force and Hamiltonian, and flow."""
    if action is None:
        check(lib().lt_set_gauge_action(U.handle, 1, 1.0, 0.0))
    else:
        check(lib().lt_set_gauge_action(U.handle, int(action.stencil_radius), float(action.c_plaq),
                                        float(action.c_rect)))


class ZeuthenFlow:
    """The Zeuthen flow (Ramos and Sint, arXiv:1508.05552) as the `action` of a
    GradientFlowKernel: the Luescher-Weisz force acted on by 1 + 1/12 nabla*_mu nabla_mu
    (lt_set_flow_action).  Not in the reference, which flows with its gauge actions only."""

    c_plaq, c_rect = 1.0 + 8.0 / 12.0, -1.0 / 12.0


def _set_flow(U: GaugeField, action) -> None:
    """The force of flows run into U: the Zeuthen flow, or `action`'s (None: Wilson)."""
    if isinstance(action, ZeuthenFlow) or action is ZeuthenFlow:
        check(lib().lt_set_flow_action(U.handle, 1))
        return
    check(lib().lt_set_flow_action(U.handle, 0))
    _set_action(U, action)


class WilsonAction:
    """GaugeAction::Rectangular<1> with (c_plaq, c_rect) = (1, 0)
    (actions/gauge/rectangular_action.hpp:23-294)."""

    stencil_radius, c_plaq, c_rect = 1, 1.0, 0.0

    def __init__(self, beta: float = 6.0):
        self.beta = float(beta)

    def Staple(self, U: GaugeField) -> np.ndarray:
        """Rectangular<1>::Staple for every link (rectangular_action.hpp:104-184), reference layout."""
        _set_action(U, self)
        out = np.empty((U.Volume(), 4, 3, 3, 2))
        check(lib().lt_staples(U.handle, out.reshape(-1)))
        return out

    def SetBeta(self, beta: float) -> None:
        self.beta = float(beta)

    def GetBeta(self) -> float:
        return self.beta

    def Action(self, U: GaugeField) -> float:
        return _out1(lib().lt_wilson_action, U.handle, self.beta)

    def ActionNormalized(self, U: GaugeField) -> float:
        return self.Action(U) / (6.0 * self.beta * U.Volume())

    def Force(self, U: GaugeField) -> np.ndarray:
        """beta/6 Algebra(st U^dag) per link (updates/hmc_gauge.hpp:450-464)."""
        _set_action(U, self)
        out = np.empty((U.Volume(), 4, 3, 3, 2))
        check(lib().lt_gauge_force(U.handle, self.beta, out.reshape(-1)))
        return out


class HeatbathKernel:
    """HeatbathKernel (updates/heatbath.hpp:30-130).  beta is taken at construction, like the
    reference's cached prefactor 3/beta (:40); random numbers come from Philox streams keyed
    by `seed`, one counter value per sweep."""

    def __init__(self, U: GaugeField, action=None, seed: int = 1, counter: int = 0):
        self.action = action if action is not None else WilsonAction()
        self.U, self.beta, self.seed = U, self.action.GetBeta(), int(seed)
        self.counter = C.c_uint64(counter)

    def sweeps(self, n: int) -> None:
        _set_action(self.U, self.action)
        check(lib().lt_heatbath_sweeps(self.U.handle, self.beta, int(n), C.c_uint64(self.seed), C.byref(self.counter)))

    def sweeps4(self, n: int) -> None:
        _set_action(self.U, self.action)
        check(lib().lt_heatbath_sweeps4(self.U.handle, self.beta, int(n), C.c_uint64(self.seed), C.byref(self.counter)))


class OverrelaxationSubgroupKernel:
    """OverrelaxationSubgroupKernel (updates/overrelaxation.hpp:68-117)."""

    def __init__(self, U: GaugeField, action=None):
        self.U, self.action = U, action

    def sweeps(self, n: int) -> None:
        _set_action(self.U, self.action)
        check(lib().lt_overrelax_sweeps(self.U.handle, int(n)))

    def sweeps4(self, n: int) -> None:
        _set_action(self.U, self.action)
        check(lib().lt_overrelax_sweeps4(self.U.handle, int(n)))


class Iterator:
    """Iterator::Checkerboard (iterators/iterators.hpp:65-87) and Checkerboard4 (:141-166): a
    whole sweep is one call; a per-link functor cannot cross to the device.  Checkerboard
    refuses radius-2 actions; Checkerboard4 needs every extent a multiple of 4."""

    @staticmethod
    def Checkerboard(kernel, n_sweep: int = 1) -> None:
        kernel.sweeps(n_sweep)

    @staticmethod
    def Checkerboard4(kernel, n_sweep: int = 1) -> None:
        kernel.sweeps4(n_sweep)


def UpdateSweeps(U: GaugeField, beta: float, n_sweep: int, n_hb: int, n_or: int, seed: int, counter: int = 0) -> int:
    """n_sweep rounds of (n_hb heatbath + n_or overrelaxation) with the Wilson action over
    Iterator::Checkerboard; returns the next counter."""
    _set_action(U, None)
    c = C.c_uint64(counter)
    check(lib().lt_update_sweeps(U.handle, float(beta), int(n_sweep), int(n_hb), int(n_or), C.c_uint64(seed), C.byref(c)))
    return c.value


def UpdateSweeps4(U: GaugeField, beta: float, n_sweep: int, n_hb: int, n_or: int, seed: int, counter: int = 0,
                  action=None) -> int:
    """The same rounds over Iterator::Checkerboard4 with any action (the reference driver's
    update loop, SU3_main.cpp:361-362); returns the next counter."""
    _set_action(U, action)
    c = C.c_uint64(counter)
    check(lib().lt_update_sweeps4(U.handle, float(beta), int(n_sweep), int(n_hb), int(n_or), C.c_uint64(seed),
                                  C.byref(c)))
    return c.value


class Euler:
    """Integrators::GradientFlow::Euler (smearing/gradient_flow.hpp:31-56)."""
    ID = 0

    @staticmethod
    def ReturnName() -> str:
        return "Euler/StoutSmearing"


class RK2:
    """Integrators::GradientFlow::RK2 (smearing/gradient_flow.hpp:89-118)."""
    ID = 1

    @staticmethod
    def ReturnName() -> str:
        return "RK2"


class RK3:
    """Integrators::GradientFlow::RK3 (smearing/gradient_flow.hpp:120-168)."""
    ID = 2

    @staticmethod
    def ReturnName() -> str:
        return "RK3"


class RK3W7:
    """Integrators::GradientFlow::RK3W7 (smearing/gradient_flow.hpp:170-218)."""
    ID = 3

    @staticmethod
    def ReturnName() -> str:
        return "RK3W7"


class GradientFlowKernel:
    """GradientFlowKernel (smearing/gradient_flow.hpp:252-367) with any of the integrators above."""

    def __init__(self, U_unflowed: GaugeField, U_flowed: GaugeField, integrator=RK3, action=None, epsilon: float = 0.01):
        if integrator not in (Euler, RK2, RK3, RK3W7):
            raise ValueError("integrator must be Euler, RK2, RK3 or RK3W7")
        self.integrator, self.action = integrator, action
        self.U_unflowed, self.U_flowed, self.epsilon = U_unflowed, U_flowed, float(epsilon)

    def _run(self, src: GaugeField, n_step: int) -> None:
        _set_flow(self.U_flowed, self.action)
        if self.integrator is RK3:
            check(lib().lt_flow_rk3(src.handle, self.U_flowed.handle, self.epsilon, int(n_step)))
        else:
            check(lib().lt_flow(src.handle, self.U_flowed.handle, self.integrator.ID, self.epsilon, int(n_step)))

    def __call__(self, n_step: int) -> None:
        self._run(self.U_unflowed, n_step)

    def Resume(self, n_step: int) -> None:
        self._run(self.U_flowed, n_step)

    def ReturnIntegratorName(self) -> str:
        return self.integrator.ReturnName()

    def Measure(self, n_meas: int, every: int):
        """Flow from U_unflowed with (plaquette sum, Q, E) after every `every` steps."""
        p, q, e = np.empty(n_meas), np.empty(n_meas), np.empty(n_meas)
        _set_flow(self.U_flowed, self.action)
        check(lib().lt_flow_rk3_measure(self.U_unflowed.handle, self.U_flowed.handle, self.epsilon, int(n_meas),
                                        int(every), p.ctypes.data, q.ctypes.data, e.ctypes.data))
        return p, q, e

    def FlowToT0(self, target: float = 0.3, max_steps: int = 100000) -> tuple[float, float]:
        """Flow U_unflowed into U_flowed until t^2 E = target; returns (t0, Q at the last step)."""
        t0, q = C.c_double(), C.c_double()
        _set_flow(self.U_flowed, self.action)
        check(lib().lt_flow_t0(self.U_unflowed.handle, self.U_flowed.handle, self.epsilon, float(target),
                               int(max_steps), C.byref(t0), C.byref(q)))
        return t0.value, q.value

    def SetEpsilon(self, eps: float) -> None:
        self.epsilon = float(eps)

    def GetEpsilon(self) -> float:
        return self.epsilon


def StoutSmearing4D(U_unsmeared: GaugeField, U_smeared: GaugeField, smear_param: float = 0.12) -> None:
    """smearing/stout_smearing.hpp:29-57."""
    check(lib().lt_stout(U_unsmeared.handle, U_smeared.handle, float(smear_param), 1))


def StoutSmearingN(U_in: GaugeField, U_out: GaugeField, N: int, smear_param: float = 0.12) -> None:
    """N stout steps from U_in into U_out (smearing/stout_smearing.hpp:61-76)."""
    check(lib().lt_stout(U_in.handle, U_out.handle, float(smear_param), int(N)))


class MetaBiasPotential:
    """MetaBiasPotential (actions/bias_potential/metadynamics.hpp:29-507)."""

    def __init__(self, CV_min, CV_max, bin_number, weight, width, well_tempered_parameter, threshold_weight):
        h = C.c_void_p()
        code = lib().lt_bias_create(float(CV_min), float(CV_max), int(bin_number), float(weight), float(width),
                                    float(well_tempered_parameter), float(threshold_weight), C.byref(h))
        if code != 0:
            raise ValueError(lib().lt_last_error().decode())   # the reference throws std::invalid_argument
        self._h = h
        self.bin_number = int(bin_number)
        self._cv_min = float(CV_min)
        self._bin_width = (float(CV_max) - float(CV_min)) / int(bin_number)

    @property
    def handle(self):
        return self._h

    def __del__(self):
        try:
            if self._h.value:
                lib().lt_bias_destroy(self._h)
        except Exception:
            pass

    GAUSSIAN, BINNED = 0, 1

    def SetUpdateMode(self, mode) -> None:
        """The deposit of UpdatePotential* and of MetaD trajectories: "gaussian" (the
        reference's well-tempered Gaussian, the default) or "binned" (Gaussian-free: the
        weight split linearly between the two grid points bracketing the CV, each share
        well-tempered by its point's value)."""
        m = {"gaussian": 0, "binned": 1}.get(mode, mode)
        check(lib().lt_bias_set_update_mode(self._h, int(m)))

    def GetUpdateMode(self) -> str:
        m = C.c_int()
        check(lib().lt_bias_get_update_mode(self._h, C.byref(m)))
        return ("gaussian", "binned")[m.value]

    def UpdatePotential(self, cv) -> None:
        a = np.atleast_1d(np.asarray(cv, dtype=np.float64))
        check(lib().lt_bias_update(self._h, a.ctypes.data, a.size, 0))

    def UpdatePotentialSymmetric(self, cv) -> None:
        a = np.atleast_1d(np.asarray(cv, dtype=np.float64))
        check(lib().lt_bias_update(self._h, a.ctypes.data, a.size, 1))

    def ReturnPotential(self, cv: float) -> float:
        return _out1(lib().lt_bias_potential, self._h, float(cv))

    def ReturnDerivative(self, cv: float) -> float:
        return _out1(lib().lt_bias_derivative, self._h, float(cv))

    def grid(self) -> np.ndarray:
        g = np.empty(self.bin_number + 1)
        check(lib().lt_bias_get_grid(self._h, g, g.size))
        return g

    def set_grid(self, g) -> None:
        g = np.ascontiguousarray(g, dtype=np.float64)
        check(lib().lt_bias_set_grid(self._h, g, g.size))

    def GeneratePotentialFrom(self, fn) -> None:
        """GeneratePotentialFrom (metadynamics.hpp:93-100)."""
        n = self.bin_number + 1
        self.set_grid(np.array([fn(self._cv_min + i * self._bin_width) for i in range(n)], dtype=np.float64))


class MDIntegrator:
    """One integrator of Integrators::HMC (updates/hmc_gauge.hpp:19-377,
    updates/hmc_metadynamics.hpp:26-238); ID is its LT_MD_* number in the C ABI.  gauge /
    metad say which kernels accept it (the friction variants need UpdateMomentaFriction of
    HMCKernel, the multiple-timescale ones UpdateGaugeMomenta / UpdateMetadynamicsMomenta of
    HMCMetaDKernel)."""

    def __init__(self, name: str, ID: int, gauge: bool = True, metad: bool = True):
        self.name, self.ID, self.gauge, self.metad = name, ID, gauge, metad

    def ReturnName(self) -> str:
        return self.name

    def __repr__(self) -> str:
        return f"Integrators.HMC.{self.name}"


Leapfrog_slow = MDIntegrator("Leapfrog_slow", 0)
Leapfrog = MDIntegrator("Leapfrog", 1)
OMF_2_slow = MDIntegrator("OMF_2_slow", 2)
OMF_2 = MDIntegrator("OMF_2", 3)
OMF_4_slow = MDIntegrator("OMF_4_slow", 4)
OMF_4 = MDIntegrator("OMF_4", 5)
Leapfrog_friction_slow = MDIntegrator("Leapfrog_friction_slow", 6, metad=False)
OMF_4_friction_slow = MDIntegrator("OMF_4_friction_slow", 7, metad=False)
Leapfrog_OMF_4 = MDIntegrator("Leapfrog_OMF_4", 8, gauge=False)
OMF_2_OMF_4_slow = MDIntegrator("OMF_2_OMF_4_slow", 9, gauge=False)
OMF_2_OMF_4 = MDIntegrator("OMF_2_OMF_4", 10, gauge=False)

# Integrators::HMC / Integrators::GradientFlow as in the reference's namespaces
Integrators = SimpleNamespace(
    HMC=SimpleNamespace(**{i.name: i for i in (Leapfrog_slow, Leapfrog, OMF_2_slow, OMF_2, OMF_4_slow, OMF_4,
                                               Leapfrog_friction_slow, OMF_4_friction_slow, Leapfrog_OMF_4,
                                               OMF_2_OMF_4_slow, OMF_2_OMF_4)}),
    GradientFlow=SimpleNamespace(Euler=Euler, RK2=RK2, RK3=RK3, RK3W7=RK3W7))


class HMCKernel:
    """GaugeUpdates::HMCKernel (updates/hmc_gauge.hpp:381-600) with any gauge integrator
    (OMF_2 by default; the reference driver uses OMF_4)."""

    def __init__(self, U: GaugeField, action: WilsonAction, trajectory_length: float = 1.0, seed: int = 1,
                 counter: int = 0, integrator: MDIntegrator = OMF_2):
        if not isinstance(integrator, MDIntegrator) or not integrator.gauge:
            raise ValueError(f"{integrator!r} is not an integrator of HMCKernel")
        self.U, self.beta, self.tau, self.seed = U, action.GetBeta(), float(trajectory_length), int(seed)
        self.action = action
        self.counter = C.c_uint64(counter)
        self.integrator = integrator
        self.delta_H = 0.0

    def _bias(self):
        return None

    def _rho_n(self):
        return 0.0, 0

    def __call__(self, n_step: int, metropolis_step: bool = True) -> bool:
        dH, acc, cv = C.c_double(), C.c_int(), C.c_double()
        rho, n = self._rho_n()
        _set_action(self.U, self.action)
        check(lib().lt_md_trajectory(self.U.handle, self._bias(), self.integrator.ID, self.beta, self.tau, int(n_step),
                                     rho, n, C.c_uint64(self.seed), C.byref(self.counter), int(bool(metropolis_step)),
                                     C.byref(dH), C.byref(acc), C.byref(cv)))
        self.delta_H = dH.value
        self._after(cv.value)
        return bool(acc.value)

    def _after(self, cv: float) -> None:
        pass

    def SetMomenta(self, P: np.ndarray) -> None:
        check(lib().lt_set_momenta(self.U.handle, np.ascontiguousarray(P, dtype=np.float64).reshape(-1)))

    def GetMomenta(self) -> np.ndarray:
        out = np.empty((self.U.Volume(), 4, 3, 3, 2))
        check(lib().lt_get_momenta(self.U.handle, out.reshape(-1)))
        return out

    def RandomMomentum(self, counter: int) -> None:
        check(lib().lt_random_momenta(self.U.handle, C.c_uint64(self.seed), C.c_uint64(counter)))

    def ReverseMomenta(self) -> None:
        check(lib().lt_reverse_momenta(self.U.handle))

    def Hamiltonian(self) -> float:
        _set_action(self.U, self.action)
        return _out1(lib().lt_hamiltonian, self.U.handle, self.beta)

    def Integrate(self, n_step: int) -> tuple[float, float]:
        """Molecular dynamics only, from the current links and momenta; returns (H_old, H_new)
        (with + V(CV) under MetaD)."""
        ho, hn = C.c_double(), C.c_double()
        rho, n = self._rho_n()
        _set_action(self.U, self.action)
        check(lib().lt_md_integrate(self.U.handle, self._bias(), self.integrator.ID, self.beta, self.tau, int(n_step),
                                    rho, n, C.byref(ho), C.byref(hn)))
        return ho.value, hn.value

    def ReversibilityTest(self, n_step: int, counter: int = 0) -> tuple[float, float]:
        """ReversibilityTest (hmc_gauge.hpp:585-598): random momenta, integrate, reverse the
        momenta, integrate again; returns (H_old, H_new), which agree for a reversible
        integrator.  The links end where they started."""
        self.RandomMomentum(counter)
        ho, _ = self.Integrate(n_step)
        self.ReverseMomenta()
        _, hn = self.Integrate(n_step)
        return ho, hn


class HMCMetaDKernel(HMCKernel):
    """GaugeUpdates::HMCMetaDKernel (updates/hmc_metadynamics.hpp:264-675) with any of its
    integrators (OMF_2 by default), CV = clover Q after n_smear_meta stout steps of parameter
    rho_stout_cv."""

    def __init__(self, U: GaugeField, bias: MetaBiasPotential, action: WilsonAction, trajectory_length: float = 1.0,
                 rho_stout_cv: float = 0.12, n_smear_meta: int = 4, seed: int = 1, counter: int = 0,
                 integrator: MDIntegrator = OMF_2):
        if not isinstance(integrator, MDIntegrator) or not integrator.metad:
            raise ValueError(f"{integrator!r} is not an integrator of HMCMetaDKernel")
        HMCKernel.__init__(self, U, action, trajectory_length, seed, counter, OMF_2)
        self.integrator = integrator
        self.bias, self.rho, self.n_smear = bias, float(rho_stout_cv), int(n_smear_meta)
        self.cv = 0.0

    def _bias(self):
        return self.bias.handle

    def _rho_n(self):
        return self.rho, self.n_smear

    def _after(self, cv: float) -> None:
        self.cv = cv

    def MetaCharge(self) -> float:
        return _out1(lib().lt_metad_charge, self.U.handle, self.rho, self.n_smear)

    def CalculateTopologicalForce(self, dvdq: float | None = None, download: bool = True):
        """dV/dQ * dQ_smeared/dU on the thin links; dV/dQ from the bias unless given.
        Returns (force in the reference layout or None when download is False, Q_smeared)."""
        q = C.c_double()
        if dvdq is None:
            check(lib().lt_metad_charge(self.U.handle, self.rho, self.n_smear, C.byref(q)))
            dvdq = self.bias.ReturnDerivative(q.value)
        out = np.empty((self.U.Volume(), 4, 3, 3, 2)) if download else None
        check(lib().lt_metad_force(self.U.handle, self.rho, self.n_smear, float(dvdq),
                                   out.ctypes.data if download else None, C.byref(q)))
        return out, q.value


def ParityUpdate(U: GaugeField) -> None:
    """ParityUpdate (updates/parity_update.hpp:22-47): the spatial reflection that maps Q to -Q
    and leaves the action unchanged, in place."""
    check(lib().lt_parity_update(U.handle))


class Ensemble:
    """Lattices of any even extents (one storage format) advanced together: one launch per
    (mu, parity) sub-sweep over all of them, rounds replayed as CUDA graphs, or one persistent
    launch per round (set_mode; autotune picks the faster)."""

    def __init__(self, lattices, betas, seed: int = 1):
        self.lattices = list(lattices)
        arr = (C.c_void_p * len(self.lattices))(*[g.handle.value for g in self.lattices])
        b = np.ascontiguousarray(betas, dtype=np.float64)
        h = C.c_void_p()
        check(lib().lt_ensemble_create(C.cast(arr, C.c_void_p), b, len(self.lattices), C.c_uint64(seed), C.byref(h)))
        self._h = h
        self.counter = C.c_uint64(0)

    def __del__(self):
        try:
            if self._h.value:
                lib().lt_ensemble_destroy(self._h)
        except Exception:
            pass

    def sweeps(self, n_sweep: int, n_hb: int = 1, n_or: int = 4, reverse: bool = False) -> None:
        check(lib().lt_ensemble_sweeps(self._h, int(n_sweep), int(n_hb), int(n_or), int(bool(reverse)),
                                       C.byref(self.counter)))

    def autotune(self) -> tuple[int, int]:
        a, b = C.c_int(), C.c_int()
        check(lib().lt_ensemble_autotune(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_block(self, threads_hb: int, threads_or: int) -> None:
        check(lib().lt_ensemble_set_block(self._h, int(threads_hb), int(threads_or)))

    GRAPH, PERSISTENT = 0, 1

    def set_mode(self, mode, blocks_per_sm: int = 0) -> None:
        """"graph": one batched launch per sub-sweep, replayed as a CUDA graph; "persistent":
        one cooperative launch per round with bounded grid barriers between sub-sweeps."""
        m = {"graph": 0, "persistent": 1}.get(mode, mode)
        check(lib().lt_ensemble_set_mode(self._h, int(m), int(blocks_per_sm)))

    def get_mode(self) -> tuple[str, int]:
        m, b = C.c_int(), C.c_int()
        check(lib().lt_ensemble_get_mode(self._h, C.byref(m), C.byref(b)))
        return ("graph", "persistent")[m.value], b.value

    def set_barrier_polls(self, polls: int) -> None:
        check(lib().lt_ensemble_set_barrier_polls(self._h, int(polls)))


def TemperingSwap(a: GaugeField, b: GaugeField, bias: MetaBiasPotential, scale_a: float, scale_b: float,
                  q_a: float, q_b: float, u: float) -> tuple[bool, float]:
    """Generalised MetadynamicsTemperingKernel swap (updates/tempering.hpp:51-72)."""
    acc, dE = C.c_int(), C.c_double()
    check(lib().lt_tempering_swap(a.handle, b.handle, bias.handle, float(scale_a), float(scale_b), float(q_a),
                                  float(q_b), float(u), C.byref(acc), C.byref(dE)))
    return bool(acc.value), dE.value


# ---------------------------------------------------------------- measurement bundle
def TopChargeCloverTimeslice(U: GaugeField) -> np.ndarray:
    """TopChargeCloverTimeslice for every t (observables/topological_charge.hpp:338-364)."""
    q = np.empty(U.ext[0])
    check(lib().lt_clover_timeslices(U.handle, q.ctypes.data, None))
    return q


def EnergyDensityCloverTimeslice(U: GaugeField) -> np.ndarray:
    """EnergyDensity::CloverTimeslice for every t (observables/field_strength_tensor.hpp:178-195)."""
    e = np.empty(U.ext[0])
    check(lib().lt_clover_timeslices(U.handle, None, e.ctypes.data))
    return e


def TopChargePlaquette(U: GaugeField) -> float:
    """observables/topological_charge.hpp:366-416."""
    return _out1(lib().lt_topcharge_plaquette, U.handle)


class RectangularAction:
    """GaugeAction::Rectangular<2> (actions/gauge/rectangular_action.hpp:23-246) with plaquette
    and 1x2 coefficients; SymanzikAction(beta) is the driver's tree-level Symanzik choice.
    As the action of a kernel it selects the rectangle staples (sweeps over Checkerboard4)."""

    stencil_radius = 2

    def __init__(self, beta: float, c_plaq: float, c_rect: float):
        self.beta, self.c_plaq, self.c_rect = float(beta), float(c_plaq), float(c_rect)

    def SetBeta(self, beta: float) -> None:
        self.beta = float(beta)

    def GetBeta(self) -> float:
        return self.beta

    def Staple(self, U: GaugeField) -> np.ndarray:
        """c_plaq StaplePlaq + c_rect StapleRect for every link (:187-246), reference layout."""
        _set_action(U, self)
        out = np.empty((U.Volume(), 4, 3, 3, 2))
        check(lib().lt_staples(U.handle, out.reshape(-1)))
        return out

    def Force(self, U: GaugeField) -> np.ndarray:
        """beta/6 Algebra(Staple U^dag) per link, the HMC momentum kick (hmc_gauge.hpp:450-464)."""
        _set_action(U, self)
        out = np.empty((U.Volume(), 4, 3, 3, 2))
        check(lib().lt_gauge_force(U.handle, self.beta, out.reshape(-1)))
        return out

    def Action(self, U: GaugeField) -> float:
        return _out1(lib().lt_rect_action, U.handle, self.beta, self.c_plaq, self.c_rect)

    def ActionNormalized(self, U: GaugeField) -> float:
        return self.Action(U) / (6.0 * self.beta * U.Volume())


def SymanzikAction(beta: float) -> RectangularAction:
    """Rectangular<2>(beta, 1 + 8/12, -1/12) as in SU3_main.cpp:115."""
    return RectangularAction(beta, 1.0 + 8.0 / 12.0, -1.0 / 12.0)


def LuescherWeiszAction(beta: float = 6.0) -> RectangularAction:
    """GaugeAction::LüscherWeiszAction (rectangular_action.hpp:273): tree-level Symanzik."""
    return RectangularAction(beta, 1.0 + 8.0 / 12.0, -1.0 / 12.0)


def IwasakiAction(beta: float = 6.0) -> RectangularAction:
    """GaugeAction::IwasakiAction (rectangular_action.hpp:274)."""
    return RectangularAction(beta, 1.0 + 8.0 * 0.331, -0.331)


def DBW2Action(beta: float = 6.0) -> RectangularAction:
    """GaugeAction::DBW2Action (rectangular_action.hpp:275)."""
    return RectangularAction(beta, 1.0 + 8.0 * 1.4088, -1.4088)


def WilsonLoop(U: GaugeField, L: int) -> float:
    """Square L x L Wilson loops: 1 - sum Re tr W / (18 V) (observables/wilson_loop.hpp:63-124)."""
    return _out1(lib().lt_wilson_loop, U.handle, int(L))


def WilsonLoopChain(U: GaugeField, start: int, end: int, reset: bool) -> float:
    """WilsonLoop<start, end, reset>(U, U_chain) with the chain kept in U's handle between
    calls (observables/wilson_loop.hpp:63-124)."""
    return _out1(lib().lt_wilson_loop_chain, U.handle, int(start), int(end), int(bool(reset)))


def PolyakovLoop(U: GaugeField) -> complex:
    """observables/polyakov_loop.hpp:32-49."""
    re, im = C.c_double(), C.c_double()
    check(lib().lt_polyakov_loop(U.handle, C.byref(re), C.byref(im)))
    return complex(re.value, im.value)


def Measure(U: GaugeField, beta: float) -> dict:
    """The PerformMeasurements step of the reference driver (SU3_main.cpp:117-139) on one field,
    with the normalisations of its output (:160-167)."""
    V = U.Volume()
    q_t, e_t = np.empty(U.ext[0]), np.empty(U.ext[0])
    check(lib().lt_clover_timeslices(U.handle, q_t.ctypes.data, e_t.ctypes.data))
    plaq = PlaquetteSum(U) / V
    return {"Wilson_Action": 1.0 - plaq / 18.0, "Improved_Action": SymanzikAction(beta).ActionNormalized(U),
            "Plaquette": plaq, "E_plaq": 36.0 - 2.0 * plaq, "E_clov": float(e_t.sum()), "E_clov_timeslice": e_t,
            "Wilson_loop(L=2)": WilsonLoopChain(U, 0, 2, True), "Wilson_loop(L=4)": WilsonLoopChain(U, 2, 4, False),
            "Wilson_loop(L=8)": WilsonLoopChain(U, 4, 8, False), "Polyakov_loop": PolyakovLoop(U),
            "TopChargeClov": float(q_t.sum()), "TopChargeClov_timeslice": q_t, "TopChargePlaq": TopChargePlaquette(U)}


def Observables(U: GaugeField, beta: float, n_smear: int, smear_skip: int, epsilon: float) -> list:
    """Observables (SU3_main.cpp:89-235): measurements on U and on n_smear levels of Euler
    gradient flow, smear_skip steps of size epsilon apart; one dict per level."""
    out = [Measure(U, beta)]
    if n_smear > 0:
        S = GaugeField(U.ext, U.prec)
        flow = GradientFlowKernel(U, S, Euler, None, epsilon)
        for k in range(1, n_smear + 1):
            if k == 1:
                flow(smear_skip)
            else:
                flow.Resume(smear_skip)
            out.append(Measure(S, beta))
    return out


def CloverDerivative(U: GaugeField) -> np.ndarray:
    """CloverDerivative for every link (observables/clover.hpp:279-321)."""
    out = np.empty((U.Volume(), 4, 3, 3, 2))
    check(lib().lt_clover_derivative(U.handle, out.reshape(-1)))
    return out


# Bits of GaugeField.status_word() (LT_STATUS_* of include/lettuce_b200.h)
STATUS_NONFINITE, STATUS_UNITARITY, STATUS_HB_CAP = 1, 2, 4

__all__ = ["STATUS_NONFINITE", "STATUS_UNITARITY", "STATUS_HB_CAP", "GaugeField", "Swap", "haar_links", "PlaquetteSum", "TopChargeClover", "EnergyDensityClover",
           "CloverObservables", "Staples", "WilsonAction", "HeatbathKernel", "OverrelaxationSubgroupKernel",
           "Iterator", "UpdateSweeps", "RK3", "GradientFlowKernel", "StoutSmearing4D", "StoutSmearingN",
           "MetaBiasPotential", "HMCKernel", "HMCMetaDKernel", "CloverDerivative", "LettuceError", "Ensemble",
           "TemperingSwap", "Euler", "RK2", "RK3W7", "TopChargeCloverTimeslice", "EnergyDensityCloverTimeslice",
           "TopChargePlaquette", "RectangularAction", "SymanzikAction", "WilsonLoop", "WilsonLoopChain", "PolyakovLoop",
           "Measure",
           "Observables", "MDIntegrator", "Integrators", "Leapfrog_slow", "Leapfrog", "OMF_2_slow", "OMF_2",
           "OMF_4_slow", "OMF_4", "Leapfrog_friction_slow", "OMF_4_friction_slow", "Leapfrog_OMF_4",
           "OMF_2_OMF_4_slow", "OMF_2_OMF_4", "ParityUpdate", "LuescherWeiszAction", "IwasakiAction", "DBW2Action",
           "UpdateSweeps4", "ZeuthenFlow", "FullTensor", "CalculateClover"]
