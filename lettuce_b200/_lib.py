"""Loader for the C-ABI library liblettuce_b200.so (built in-tree by lettuce_b200/build.py).

The library is the product: there is no CPU fallback.  If it is missing, importing the
package still works (so that the symbol checks and host-side helpers can report it), but
every compute call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("LETTUCE_B200_LIB", os.path.join(HERE, "liblettuce_b200.so"))
HEADER_PATH = os.path.join(os.path.dirname(HERE), "include", "lettuce_b200.h")

LT_OK, LT_ERR_ARG, LT_ERR_CUDA, LT_ERR_NOMEM, LT_ERR_STATE, LT_ERR_NUMERIC, LT_ERR_IO, LT_ERR_TIMEOUT = range(8)
PREC = {"fp64": 0, "fp32": 1, "fp32_12": 2}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_d, _i, _u64 = C.c_double, C.c_int, C.c_uint64
_pd, _pi, _pu64 = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_uint64)

# name -> argument types (all return int status except where noted)
SIGNATURES = {
    "lt_last_error": (C.c_char_p, []),
    "lt_version": (_i, []),
    "lt_create": (_i, [_ip, _i, C.POINTER(_vp)]),
    "lt_destroy": (_i, [_vp]),
    "lt_get_extents": (_i, [_vp, _ip, _pi]),
    "lt_upload_links": (_i, [_vp, _dp]),
    "lt_download_links": (_i, [_vp, _dp]),
    "lt_upload_bytes": (_i, [_vp, _dp, _pu64]),
    "lt_set_link": (_i, [_vp, C.c_int64, _i, _dp]),
    "lt_get_link": (_i, [_vp, C.c_int64, _i, _dp]),
    "lt_copy": (_i, [_vp, _vp]),
    "lt_swap": (_i, [_vp, _vp]),
    "lt_set_identity": (_i, [_vp]),
    "lt_haar_links": (_i, [_ip, _u64, _dp]),
    "lt_set_haar_random": (_i, [_vp, _u64]),
    "lt_synchronize": (_i, [_vp]),
    "lt_get_stream": (_i, [_vp, C.POINTER(_vp)]),
    "lt_status_word": (_i, [_vp, C.POINTER(C.c_uint32), _i]),
    "lt_check_links": (_i, [_vp, _pd]),
    "lt_save_bmw": (_i, [_vp, C.c_char_p, _i, _i, C.c_char_p]),
    "lt_load_bmw": (_i, [_vp, C.c_char_p, _i, _pi, _pi]),
    "lt_bmw_checksum": (_i, [_vp, _i, _pu64]),
    "lt_plaquette_sum": (_i, [_vp, _pd]),
    "lt_wilson_action": (_i, [_vp, _d, _pd]),
    "lt_topcharge_clover": (_i, [_vp, _pd]),
    "lt_energy_clover": (_i, [_vp, _pd]),
    "lt_clover_observables": (_i, [_vp, _pd, _pd]),
    "lt_staples": (_i, [_vp, _dp]),
    "lt_clover_tensor": (_i, [_vp, _vp]),
    "lt_topcharge_clover_tensor": (_i, [_vp, _vp, _pd]),
    "lt_plaquette_sum_noalloc": (_i, [_vp, _ip, _vp, _vp]),
    "lt_su3_exp_test": (_i, [_dp, _dp, _i, _i, _i]),
    "lt_device_arch": (_i, [_pi, _pi]),
    "lt_pack_links_test": (_i, [_ip, _dp, C.POINTER(C.c_float)]),
    "lt_overrelax_sweeps": (_i, [_vp, _i]),
    "lt_heatbath_sweeps": (_i, [_vp, _d, _i, _u64, _pu64]),
    "lt_update_sweeps": (_i, [_vp, _d, _i, _i, _i, _u64, _pu64]),
    "lt_overrelax_sweeps4": (_i, [_vp, _i]),
    "lt_heatbath_sweeps4": (_i, [_vp, _d, _i, _u64, _pu64]),
    "lt_update_sweeps4": (_i, [_vp, _d, _i, _i, _i, _u64, _pu64]),
    "lt_set_gauge_action": (_i, [_vp, _i, _d, _d]),
    "lt_get_gauge_action": (_i, [_vp, _pi, _pd, _pd]),
    "lt_ensemble_create": (_i, [_vp, _dp, _i, _u64, C.POINTER(_vp)]),
    "lt_ensemble_destroy": (_i, [_vp]),
    "lt_ensemble_sweeps": (_i, [_vp, _i, _i, _i, _i, _pu64]),
    "lt_ensemble_autotune": (_i, [_vp, _pi, _pi]),
    "lt_ensemble_set_block": (_i, [_vp, _i, _i]),
    "lt_ensemble_set_mode": (_i, [_vp, _i, _i]),
    "lt_ensemble_get_mode": (_i, [_vp, _pi, _pi]),
    "lt_ensemble_set_barrier_polls": (_i, [_vp, C.c_longlong]),
    "lt_tempering_swap": (_i, [_vp, _vp, _vp, _d, _d, _d, _d, _d, _pi, _pd]),
    "lt_flow_rk3": (_i, [_vp, _vp, _d, _i]),
    "lt_flow": (_i, [_vp, _vp, _i, _d, _i]),
    "lt_set_flow_action": (_i, [_vp, _i]),
    "lt_get_flow_action": (_i, [_vp, _pi]),
    "lt_clover_timeslices": (_i, [_vp, _vp, _vp]),
    "lt_topcharge_plaquette": (_i, [_vp, _pd]),
    "lt_rect_action": (_i, [_vp, _d, _d, _d, _pd]),
    "lt_wilson_loop": (_i, [_vp, _i, _pd]),
    "lt_wilson_loop_chain": (_i, [_vp, _i, _i, _i, _pd]),
    "lt_polyakov_loop": (_i, [_vp, _pd, _pd]),
    "lt_flow_rk3_measure": (_i, [_vp, _vp, _d, _i, _i, _vp, _vp, _vp]),
    "lt_flow_t0": (_i, [_vp, _vp, _d, _d, _i, _pd, _pd]),
    "lt_stout": (_i, [_vp, _vp, _d, _i]),
    "lt_gauge_force": (_i, [_vp, _d, _dp]),
    "lt_set_momenta": (_i, [_vp, _dp]),
    "lt_get_momenta": (_i, [_vp, _dp]),
    "lt_random_momenta": (_i, [_vp, _u64, _u64]),
    "lt_hamiltonian": (_i, [_vp, _d, _pd]),
    "lt_omf2": (_i, [_vp, _d, _d, _i, _pd, _pd]),
    "lt_hmc_trajectory": (_i, [_vp, _d, _d, _i, _u64, _pu64, _i, _pd, _pi]),
    "lt_clover_derivative": (_i, [_vp, _dp]),
    "lt_metad_charge": (_i, [_vp, _d, _i, _pd]),
    "lt_metad_force": (_i, [_vp, _d, _i, _d, _vp, _pd]),
    "lt_metad_omf2": (_i, [_vp, _vp, _d, _d, _i, _d, _i, _pd, _pd]),
    "lt_metad_hmc_trajectory": (_i, [_vp, _vp, _d, _d, _i, _d, _i, _u64, _pu64, _i, _pd, _pi, _pd]),
    "lt_md_integrate": (_i, [_vp, _vp, _i, _d, _d, _i, _d, _i, _pd, _pd]),
    "lt_md_trajectory": (_i, [_vp, _vp, _i, _d, _d, _i, _d, _i, _u64, _pu64, _i, _pd, _pi, _pd]),
    "lt_reverse_momenta": (_i, [_vp]),
    "lt_parity_update": (_i, [_vp]),
    "lt_bias_create": (_i, [_d, _d, _i, _d, _d, _d, _d, C.POINTER(_vp)]),
    "lt_bias_destroy": (_i, [_vp]),
    "lt_bias_update": (_i, [_vp, _vp, _i, _i]),
    "lt_bias_set_update_mode": (_i, [_vp, _i]),
    "lt_bias_get_update_mode": (_i, [_vp, _pi]),
    "lt_bias_potential": (_i, [_vp, _d, _pd]),
    "lt_bias_derivative": (_i, [_vp, _d, _pd]),
    "lt_bias_get_grid": (_i, [_vp, _dp, _i]),
    "lt_bias_set_grid": (_i, [_vp, _dp, _i]),
}


class LettuceError(RuntimeError):
    """A non-zero status from the C ABI, carrying lt_last_error()."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_LIB = None


def lib():
    """The loaded C-ABI library; raises if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m lettuce_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def check(code: int) -> None:
    if code != LT_OK:
        raise LettuceError(code, lib().lt_last_error().decode())


def declared_symbols() -> list[str]:
    """Every function name declared in include/lettuce_b200.h."""
    import re
    text = open(HEADER_PATH).read()
    return sorted(set(re.findall(r"^(?:const char\*|int)\s+(lt_\w+)\s*\(", text, flags=re.M)))
