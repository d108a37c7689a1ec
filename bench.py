#!/usr/bin/env python
"""Benchmark of the B200 pure-gauge SU(3) hot path (one JSON line on rank 0).

Workload (the large plain-vs-FP32 configuration): 32^4 SU(3) Wilson gauge theory at
beta = 6.0 from a seeded Haar-random start.  One step = one round of 1 Cabibbo-Marinari
heatbath sweep + 4 overrelaxation sweeps (5 * 4V = 20,971,520 link updates) on FP32-bulk
links.  The headline `value` is link updates/s; flow steps/s (RK3, eps = 0.01), the plain
FP64 path, the FP32/FP64 ratios and |dP| between FP32 and FP64 flows from identical
configurations are measured in the same run.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1: launched by torchrun, one rank per GPU; each rank evolves its own lattice (replicas,
weak scaling; the path has no data exchange), timed on the device, max over ranks.
--impl reference: the reference's own multi-threaded CPU code (oracle/_ref, else the C
oracle) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lettuce_b200 import bytes_model as bm  # noqa: E402

METRIC = "link updates/s & flow steps/s at 32^4: FP32-bulk vs plain FP64 GPU, dP<=1e-6"
UNIT = "link updates/s"
BETA = 6.0
SEED = 20251203
N_HB, N_OR = 1, 4
FLOW_EPS = 0.01
N_THERM = 100


def _jsonable(o):
    """numpy scalars and arrays in the JSON line"""
    if hasattr(o, "tolist"):
        return o.tolist()
    raise TypeError(f"{type(o).__name__} is not JSON serializable")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=32)
    ap.add_argument("--prec", choices=["fp32_12", "fp32", "fp64"], default="fp32_12")
    ap.add_argument("--no-extras", action="store_true", help="skip the FP64 / flow / e2e / CPU side measurements")
    ap.add_argument("--workload", choices=["sweeps", "flow", "metad"], default="sweeps",
                    help="sweeps: the headline; flow / metad: secondary rates (and ncu targets)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def flow_roofline(torch, prec: str, volume: int, ms_step: float, ms_step64: float, hbm_peak: float) -> dict:
    """RK3 flow step against both ceilings: algorithmic HBM bytes over the measured copy
    bandwidth, and algorithmic flops over the nominal CUDA-core peak (SMs x lanes x 2 x the
    measured maximum SM clock; 128 FP32 and 64 FP64 lanes per SM)."""
    props = torch.cuda.get_device_properties(0)
    mhz = 1965.0
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        mhz = float(json.load(open(p)).get("sm_max_mhz", mhz))
    f32_peak = props.multi_processor_count * 128 * 2 * mhz * 1e6 / 1e12
    f64_peak = f32_peak / 2
    links = 4 * volume
    out = {}
    for name, pr, ms, fpk in (("bulk", prec, ms_step, f32_peak if prec != "fp64" else f64_peak),
                              ("fp64", "fp64", ms_step64, f64_peak)):
        gbs = bm.flow_step_bytes_per_link(pr) * links / (ms / 1000.0) / 1e9
        tfl = bm.FLOPS["flow_step"] * links / (ms / 1000.0) / 1e12
        out[name] = {"prec": pr, "ms_per_step": ms, "hbm_gbs": gbs, "hbm_frac": gbs / hbm_peak,
                     "tflops": tfl, "alu_peak_tflops": fpk, "alu_frac": tfl / fpk}
    out["alu_peak_source"] = "nominal CUDA-core peak at the measured max SM clock"
    return out


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` recorded from an ncu capture in profiles/ (a line
    `traffic_bytes_per_launch <kernel> <bytes>`), else None."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, f)):
            parts = line.strip().strip("`").split()
            if len(parts) == 3 and parts[0] == "traffic_bytes_per_launch" and parts[1] == kernel:
                return float(parts[2])
    return None


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.rows, self.proc = index, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) > 8 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---------------------------------------------------------------------------- reference arm
def headline_config(size: int, prec: str, world: int) -> dict:
    """The workload both arms run: one step = N_HB heatbath + N_OR overrelaxation sweeps."""
    return {"workload": f"{size}^4 SU(3) Wilson beta={BETA}: {N_HB} heatbath + {N_OR} overrelaxation "
                        f"sweeps per step, {prec} links",
            "lattice": [size] * 4, "beta": BETA, "storage": prec,
            "l2": f"inputs larger than L2 ({size ** 4 * 4 * bm.LINK_BYTES[prec] / 1e6:.0f} MB of links per sweep)",
            "parallelism": f"replicas x{world}"}


def host_isa() -> str:
    """x86-64 level of this host for the timing builds of the reference: v4 (AVX-512) or v3."""
    try:
        flags = set()
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
        if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags:
            return "v4"
    except OSError:
        pass
    return "v3"


class CpuReference:
    """The reference's own OpenMP code for the path (oracle/_ref, built from the reference
    sources): the timing build (reference Makefile optimisation, contraction on, this host's
    ISA level) when present, else the parity build.  Never the product library."""

    def __init__(self, size: int):
        import ctypes as C
        self.ext = "x".join([str(size)] * 4)
        ref_dir = os.path.join(ROOT, "oracle", "_ref")
        cands = [(os.path.join(ref_dir, f"liblt_ref_fast_{self.ext}_{host_isa()}.so"),
                  f"-O3 -march=x86-64-{host_isa()} -fopenmp, contraction on"),
                 (os.path.join(ref_dir, f"liblt_ref_{self.ext}.so"), "-O3 -march=x86-64-v3 -fopenmp, no contraction")]
        self.path, self.build = next(((p, b) for p, b in cands if os.path.exists(p)), (None, None))
        if self.path is None:
            raise FileNotFoundError(f"no reference harness for {self.ext} under oracle/_ref")
        L = C.CDLL(self.path)
        dp = C.c_void_p
        L.ref_field_load.argtypes = [dp]
        L.ref_field_rounds.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int]
        L.ref_field_flow_steps.argtypes = [C.c_double, C.c_int]
        L.ref_threads.restype = C.c_int
        self.lib = L

    def load(self, links):
        import numpy as np
        a = np.ascontiguousarray(links, dtype=np.float64)
        self.lib.ref_field_load(a.ctypes.data)

    def rounds(self, n: int):
        self.lib.ref_field_rounds(BETA, n, N_HB, N_OR)

    def flow(self, n: int):
        self.lib.ref_field_flow_steps(FLOW_EPS, n)

    def threads(self) -> int:
        return int(self.lib.ref_threads())

    def metad_force_rate(self, links, n: int) -> float:
        """Force evaluations/s of the reference's HMCMetaDKernel::CalculateTopologicalForce
        (4 stout levels of rho = 0.12, a linear bias) over n timed calls after one untimed."""
        import ctypes as C
        import numpy as np
        f = self.lib.ref_metad_force_seconds
        f.restype = C.c_double
        f.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int]
        a = np.ascontiguousarray(links, dtype=np.float64)
        return n / f(a.ctypes.data, 0.12, 1.0, n)


def cpu_reference_sample(size: int, links, n_round: int, n_flow: int):
    """A bounded sample of the reference CPU path: n_round steps (1 HB + 4 OR sweeps) and
    n_flow RK3 flow steps, timed with nothing else inside the timed regions."""
    import numpy as np
    V = size ** 4
    upd = (N_HB + N_OR) * 4 * V
    try:
        ref = CpuReference(size)
    except (FileNotFoundError, OSError):
        ref = None
    if ref is not None:
        ref.load(links)
        ref.rounds(1)
        t0 = time.perf_counter()
        ref.rounds(n_round)
        dt = time.perf_counter() - t0
        t0 = time.perf_counter()
        ref.flow(n_flow)
        df = time.perf_counter() - t0
        return {"value": n_round * upd / dt, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
                "sample": f"{n_round} x (1 heatbath + 4 overrelaxation sweeps) and {n_flow} RK3 flow steps at "
                          f"{size}^4, FP64, the reference's OpenMP code ({os.path.basename(ref.path)}: {ref.build})",
                "flow_steps_per_s": n_flow / df}
    # no reference harness here: the C oracle (a single-threaded restatement), one heatbath sweep
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ltref import Oracle
    o = Oracle()
    e = np.array([size] * 4, dtype=np.int32)
    U = np.ascontiguousarray(links)
    t0 = time.perf_counter()
    o.lib.or_heatbath_sweeps(e, U, BETA, 1, 0, 0)
    dt = time.perf_counter() - t0
    return {"value": 4 * V / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 heatbath sweep at {size}^4, FP64, single-threaded C oracle"}


def run_reference(a):
    """--impl reference: the reference's CPU implementation of the headline workload on this
    host's cores, the same config, steps and warm-up as our arm; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ltref import haar_links_numpy
    size = a.size
    V = size ** 4
    upd = (N_HB + N_OR) * 4 * V
    links = haar_links_numpy((size,) * 4, SEED)
    config = headline_config(size, a.prec, world)
    try:
        ref = CpuReference(size)
    except (FileNotFoundError, OSError) as e:
        print(json.dumps({"impl": "reference", "unavailable": f"reference harness not built: {e}"}))
        return 0
    ref.load(links)
    ref.rounds(a.warmup)
    t0 = time.perf_counter()
    ref.rounds(a.steps)
    dt = time.perf_counter() - t0
    n_flow = 10
    t1 = time.perf_counter()
    ref.flow(n_flow)
    df = time.perf_counter() - t1
    value = a.steps * upd / dt
    sample = (f"{a.steps} x (1 heatbath + 4 overrelaxation sweeps) at {size}^4 after {a.warmup} warm-up steps, FP64, "
              f"the reference's OpenMP code ({os.path.basename(ref.path)}: {ref.build}), seeded Haar start")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": 1000.0 * dt / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic: seeded Haar-random SU(3) start",
            "impl": "reference", "config": config,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.threads(), "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "flow_steps_per_s": n_flow / df}
    print(json.dumps(line, default=_jsonable))
    return 0


# ---------------------------------------------------------------------------- secondary rates
def secondary_rates(lt, torch, timed, prec):
    """Rates of the other workloads, reported beside the headline:
    * metadynamics force evaluations/s at 16^4 (4 stout steps rho = 0.12, bulk FP32 storage);
    * MetaD-HMC trajectories/s at 16^4 with the Gaussian-free binned bias deposits;
    * tempering ensemble link updates/s: 8 streams of 12^4 plus 40 chains with extents drawn
      from {8,...,16}^4, beta in [5.8, 6.2], one batched round (1 HB + 4 OR) per step;
    * BMW configuration files at 32^4 (device checksum pass, save and load);
    * Iterator::Checkerboard4 rounds at 32^4 with the Wilson and the Luescher-Weisz actions;
    * the driver's measurement step at 32^4;
    * one 48^4 HMC trajectory (OMF4, tau = 1, 20 steps, bulk FP32 storage, FP64 dH), the
      Wilson flow to t0 and the Zeuthen flow's rate."""
    import numpy as np
    out = {"storage": prec}
    try:
        ext = (16,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(3)
        lt.UpdateSweeps(G, BETA, 5, 1, 4, SEED)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(BETA), 1.0, 0.12, 4)
        for _ in range(3):
            k.CalculateTopologicalForce(dvdq=1.0, download=False)
        ms = timed(G, lambda: k.CalculateTopologicalForce(dvdq=1.0, download=False), 10)
        rate = 10 / (ms / 1000.0)
        out["metad_force_evals_per_s_16^4"] = rate
        links = 4 * G.Volume()
        gbs = bm.metad_force_bytes_per_link(prec, 4) * links * rate / 1e9
        tfl = bm.FLOPS["metad_force_n4"] * links * rate / 1e12
        out["metad_force_roofline"] = {"hbm_gbs": gbs, "hbm_frac": gbs / peaks()[0], "tflops": tfl,
                                       "note": "algorithmic bytes (6.9 n + 3.5) b per link and ~70k flops per link"}
        del k, G
    except Exception as e:   # report, never hide
        out["metad_force_error"] = repr(e)
    try:
        # the metadynamics configuration: MetaD-HMC at 16^4 (OMF2, tau = 1, 10 steps; CV = clover
        # Q after 4 stout steps of rho = 0.12; bias over [-8, 8] with 800 bins, Gaussian-free
        # binned deposits after every trajectory), bulk FP32 links, FP64 bias and dH
        ext = (16,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(21)
        lt.UpdateSweeps(G, BETA, 20, 1, 4, SEED)
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 4 * 16.0 / 800, 10, 1000)
        bias.SetUpdateMode("binned")
        hmc = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(BETA), 1.0, 0.12, 4, seed=SEED)
        for _ in range(2):
            hmc(10, True)
        n_traj, acc, dH = 8, 0, []
        t0 = time.perf_counter()
        for _ in range(n_traj):
            acc += int(hmc(10, True))
            dH.append(hmc.delta_H)
        dt = time.perf_counter() - t0
        out["metad_hmc_binned_16^4"] = {"trajectories_per_s": n_traj / dt, "acceptance": acc / n_traj,
                                        "dH": dH, "deposited_grid_points": int(np.count_nonzero(bias.grid())),
                                        "integrator": "OMF2, tau = 1, 10 steps", "storage": prec}
        del hmc, G
    except Exception as e:
        out["metad_hmc_binned_error"] = repr(e)
    try:
        rng = np.random.default_rng(4)
        lats = [lt.GaugeField((12,) * 4, prec) for _ in range(8)]
        betas = [BETA] * 8
        for _ in range(40):
            e = tuple(int(v) for v in rng.choice([8, 10, 12, 14, 16], 4))
            lats.append(lt.GaugeField(e, prec))
            betas.append(float(rng.uniform(5.8, 6.2)))
        for j, g in enumerate(lats):
            g.SetToHaarRandom(100 + j)
        ens = lt.Ensemble(lats, betas, SEED)
        out["ensemble_autotuned_threads"] = ens.autotune()
        out["ensemble_autotuned_mode"] = ens.get_mode()
        ens.sweeps(3, 1, 4)
        n = 10
        ms = timed(lats[0], lambda: ens.sweeps(n, 1, 4), 1)
        upd = 5 * 4 * sum(g.Volume() for g in lats)
        out["ensemble_link_updates_per_s"] = n * upd / (ms / 1000.0)
        out["ensemble_lattices"] = len(lats)
        # both ways of running a round: a graph of 40 batched launches, or one persistent
        # cooperative launch with 39 grid barriers (at each residency)
        modes = {}
        for mode, bps in (("graph", 0), ("persistent", 0), ("persistent", 4), ("persistent", 2)):
            ens.set_mode(mode, bps)
            ens.sweeps(2, 1, 4)
            ms = timed(lats[0], lambda: ens.sweeps(n, 1, 4), 1)
            modes[f"{mode}_{ens.get_mode()[1]}"] = n * upd / (ms / 1000.0)
        out["ensemble_link_updates_per_s_by_mode"] = modes
        del ens, lats
    except Exception as e:
        out["ensemble_error"] = repr(e)
    try:
        # BMW configuration files at 32^4: the device pack + Adler-64 pass alone (links read
        # once, payload written once), and a two-row file saved and loaded through the C ABI
        # (device pass + PCIe + file system)
        import tempfile
        ext = (32,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(11)
        G.bmw_checksum()
        n = 10
        ms = timed(G, lambda: G.bmw_checksum(), n) / n
        out["bmw_checksum_call_ms_32^4"] = ms
        out["bmw_checksum_link_gbs"] = 4 * G.Volume() * bm.LINK_BYTES[prec] / (ms / 1000.0) / 1e9
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, "cfg.bmw")
            t0 = time.perf_counter()
            G.save_bmw(path, overwrite=True)
            out["bmw_save_s_32^4"] = time.perf_counter() - t0
            t0 = time.perf_counter()
            ok, grp = G.load_bmw(path)
            out["bmw_load_s_32^4"] = time.perf_counter() - t0
            out["bmw_file_mb"] = os.path.getsize(path) / 1e6
            out["bmw_roundtrip_ok"] = bool(ok and grp)
        del G
    except Exception as e:
        out["bmw_error"] = repr(e)
    try:
        # Iterator::Checkerboard4 rounds (1 HB + 4 OR) at 32^4 with the Wilson and the
        # Luescher-Weisz (rectangle) actions, the reference driver's iterator
        ext = (32,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(17)
        for name, act in (("wilson", None), ("luescher_weisz", lt.LuescherWeiszAction(BETA))):
            lt.UpdateSweeps4(G, BETA, 2, 1, 4, SEED, 0, act)
            n = 3
            ms = timed(G, lambda: lt.UpdateSweeps4(G, BETA, n, 1, 4, SEED, 0, act), 1)
            out[f"checkerboard4_{name}_link_updates_per_s_32^4"] = n * 5 * 4 * G.Volume() / (ms / 1000.0)
        del G
    except Exception as e:
        out["checkerboard4_error"] = repr(e)
    try:
        # the driver's measurement step at 32^4 (clover Q and E per timeslice, plaquette, plaquette
        # charge, Symanzik action, Wilson loops L = 2, 4, 8, Polyakov loop) from the given storage,
        # each observable a device pass plus a host read of its sums
        ext = (32,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(13)
        lt.UpdateSweeps(G, BETA, 5, 1, 4, SEED)
        lt.Measure(G, BETA)
        n = 5
        ms = timed(G, lambda: lt.Measure(G, BETA), n) / n
        out["measure_bundle_ms_32^4"] = ms
        out["wilson_loop_L8_ms_32^4"] = timed(G, lambda: lt.WilsonLoop(G, 8), n) / n
        out["polyakov_loop_ms_32^4"] = timed(G, lambda: lt.PolyakovLoop(G), n) / n
        del G
    except Exception as e:
        out["measure_error"] = repr(e)
    try:
        # 48^4 at beta = 6.3: Haar start, 200 rounds of 1 HB + 4 OR, two OMF4 trajectories (the
        # reference driver's integrator; tau = 1, 20 steps, FP32 links, FP64 dH and accept), then
        # Wilson flow to t0
        # (t^2 E = 0.3) with clover Q and E at every step
        ext = (48,) * 4
        G = lt.GaugeField(ext, prec)
        G.SetToHaarRandom(5)
        t0 = time.perf_counter()
        lt.UpdateSweeps(G, 6.3, 200, 1, 4, SEED)
        G.synchronize()
        out["hmc_48^4_therm_s_200_rounds"] = time.perf_counter() - t0
        hmc = lt.HMCKernel(G, lt.WilsonAction(6.3), 1.0, seed=7, integrator=lt.OMF_4)
        hmc(20, True)
        t0 = time.perf_counter()
        acc = hmc(20, True)
        out["hmc_48^4_s_per_trajectory"] = time.perf_counter() - t0
        out["hmc_48^4_dH"] = [hmc.delta_H]
        out["hmc_48^4_accepted"] = bool(acc)
        del hmc
        F = lt.GaugeField(ext, prec)
        flow = lt.GradientFlowKernel(G, F, lt.RK3, None, FLOW_EPS)
        t0 = time.perf_counter()
        tt0, q = flow.FlowToT0(0.3)
        out["flow_to_t0_48^4_s"] = time.perf_counter() - t0
        out["t0_48^4_beta6.3"] = tt0
        out["Q_at_t0_48^4"] = q
        # the Zeuthen flow of the same configuration: RK3 steps/s
        zflow = lt.GradientFlowKernel(G, F, lt.RK3, lt.ZeuthenFlow(), FLOW_EPS)
        zflow(2)
        n_z = 10
        ms = timed(F, lambda: zflow.Resume(n_z), 1)
        out["zeuthen_flow_steps_per_s_48^4"] = n_z / (ms / 1000.0)
        del F, G
    except Exception as e:
        out["hmc_48_error"] = repr(e)
    return out


# ---------------------------------------------------------------------------- secondary workloads
def run_secondary(a, lt, torch, ext, links, timed, barrier, max_over_ranks, world, rank, dist):
    """flow: one RK3 step (eps = 0.01) per step, flow steps/s.
    metad: one metadynamics force evaluation (4 stout steps rho = 0.12, clover Q, adjoint
    chain) per step, force evaluations/s."""
    G = lt.GaugeField(ext, a.prec)
    G.upload(links)
    lt.UpdateSweeps(G, BETA, 5, 1, 4, SEED + rank)
    if a.workload == "flow":
        H = lt.GaugeField(ext, a.prec)
        flow = lt.GradientFlowKernel(G, H, lt.RK3, None, FLOW_EPS)
        flow(1)
        step = lambda: flow.Resume(1)   # noqa: E731
        unit, launches_per_step, handle = "flow steps/s", 3, H
    else:
        bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
        k = lt.HMCMetaDKernel(G, bias, lt.WilsonAction(BETA), 1.0, 0.12, 4)
        step = lambda: k.CalculateTopologicalForce(dvdq=1.0, download=False)   # noqa: E731
        unit, launches_per_step, handle = "force evaluations/s", 4 + 2 + 2 * 4 + 3, G
    for _ in range(max(a.warmup, 3)):
        step()
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(timed(handle, lambda: [step() for _ in range(a.steps)], 1))
    line = {"metric": f"{unit} at {ext[0]}^4", "value": world * a.steps / (ms / 1000.0), "unit": unit,
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms / a.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if a.prec != "fp64" else "f64", "data": "synthetic: seeded Haar-random SU(3) start",
            "config": {"workload": f"{a.workload} at {ext[0]}^4, {a.prec} links", "lattice": list(ext),
                       "storage": a.prec}, "gpu_launches": a.steps * launches_per_step}
    if rank == 0:
        print(json.dumps(line, default=_jsonable))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------- our arm
def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)

    import numpy as np
    import torch
    import lettuce_b200 as lt

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    ext = (a.size,) * 4
    V = a.size ** 4
    links = lt.haar_links(ext, SEED + rank)

    def barrier():
        if dist:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(G, fn, n):
        """Device time (ms) of n calls of fn, CUDA events on the handle's stream."""
        s = torch.cuda.ExternalStream(G.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        G.synchronize()
        e0.record(s)
        for _ in range(n):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1)

    counter = {"c": 0}

    def sweep_round(G):
        counter["c"] = lt.UpdateSweeps(G, BETA, 1, N_HB, N_OR, SEED + rank, counter["c"])

    if a.workload != "sweeps":
        return run_secondary(a, lt, torch, ext, links, timed, barrier, max_over_ranks, world, rank, dist)

    # ---- headline: FP32-bulk sweeps
    G = lt.GaugeField(ext, a.prec)
    G.upload(links)
    for _ in range(max(a.warmup, 3)):
        sweep_round(G)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ms = timed(G, lambda: sweep_round(G), a.steps)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(ms)
    upd_per_step = (N_HB + N_OR) * 4 * V
    value = world * a.steps * upd_per_step / (ms / 1000.0)
    launches = a.steps * (N_HB + N_OR) * 8

    # ---- dominant kernel: one overrelaxation sub-sweep, per-launch duration
    n_or = 20
    or_ms = timed(G, lambda: lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(G), n_or), 1) / (8 * n_or)
    hb_ms = timed(G, lambda: lt.Iterator.Checkerboard(lt.HeatbathKernel(G, lt.WilsonAction(BETA), 5), 5), 1) / 40
    peak, peak_kind = peaks()
    alg_bytes = bm.sweep_launch_bytes(a.prec, V)   # 9 link reads/writes per update, V/2 updates
    achieved = alg_bytes / (or_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": ncu_traffic(f"k_overrelax<{a.prec}>"),
                "kernel": f"k_overrelax_staged ({a.prec})" if a.prec == "fp32_12" else f"k_overrelax ({a.prec})",
                "ms_per_launch": or_ms, "algorithmic_bytes_per_launch": alg_bytes,
                "peak_source": f"{peak_kind} hbm_gbs",
                "heatbath_ms_per_launch": hb_ms,
                "heatbath_achieved_gbs": alg_bytes / (hb_ms / 1000.0) / 1e9}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if a.prec != "fp64" else "f64",
            "data": "synthetic: seeded Haar-random SU(3) start (per rank)",
            "config": headline_config(a.size, a.prec, world),
            "roofline": roofline, "clocks": clocks.summary(), "gpu_launches": launches}

    if not a.no_extras:
        # ---- 100 further rounds (the plain-vs-FP32 protocol's thermalisation), then the identical
        # configuration flowed in FP32-bulk and in FP64 to t = 4, with P, Q and E at t = 1, 2, 3, 4
        for _ in range(N_THERM):
            sweep_round(G)
        therm = G.download()
        res = {}
        n_flow = 10
        # the bulk storage, the 18-real FP32 storage beside two-row links, and plain FP64
        precs = [a.prec] + (["fp32"] if a.prec == "fp32_12" else []) + ["fp64"]
        for prec in precs:
            A, B = lt.GaugeField(ext, prec), lt.GaugeField(ext, prec)
            A.upload(therm)
            flow = lt.GradientFlowKernel(A, B, lt.RK3, None, FLOW_EPS)
            flow(2)
            t = timed(B, lambda: flow.Resume(n_flow), 1)
            p, q, e = flow.Measure(4, 100)
            res[prec] = {"flow_steps_per_s": n_flow / (t / 1000.0), "flow_ms": t / n_flow,
                         "plaq": p / V / 18, "Q": q, "E": e}
            # sweeps in this precision
            C = lt.GaugeField(ext, prec)
            C.upload(therm)
            for _ in range(2):
                sweep_round(C)
            t = timed(C, lambda: sweep_round(C), 5)
            res[prec]["link_updates_per_s"] = 5 * upd_per_step / (t / 1000.0)
            # per-launch sub-sweep times of this precision and their HBM fractions
            o_ms = timed(C, lambda: lt.Iterator.Checkerboard(lt.OverrelaxationSubgroupKernel(C), 5), 1) / 40
            h_ms = timed(C, lambda: lt.Iterator.Checkerboard(lt.HeatbathKernel(C, lt.WilsonAction(BETA), 5), 5),
                         1) / 40
            lb = bm.sweep_launch_bytes(prec, V)
            res[prec]["sweep_roofline"] = {
                "overrelax_ms_per_launch": o_ms, "overrelax_hbm_frac": lb / (o_ms / 1000.0) / 1e9 / peak,
                "heatbath_ms_per_launch": h_ms, "heatbath_hbm_frac": lb / (h_ms / 1000.0) / 1e9 / peak,
                "algorithmic_bytes_per_launch": lb, "peak_gbs": peak}
            del A, B, C
        line["flow_steps_per_s"] = res[a.prec]["flow_steps_per_s"]
        line["fp64"] = {k: res["fp64"][k] for k in ("link_updates_per_s", "flow_steps_per_s", "sweep_roofline")}
        line["bulk_sweep_roofline"] = res[a.prec]["sweep_roofline"]
        line["fp32_over_fp64"] = {
            "link_updates": res[a.prec]["link_updates_per_s"] / res["fp64"]["link_updates_per_s"],
            "flow_steps": res[a.prec]["flow_steps_per_s"] / res["fp64"]["flow_steps_per_s"]}
        dP = [abs(x - y) for x, y in zip(res[a.prec]["plaq"], res["fp64"]["plaq"])]
        dQ = [abs(x - y) for x, y in zip(res[a.prec]["Q"], res["fp64"]["Q"])]
        line["flow_vs_fp64"] = {"t": [1.0, 2.0, 3.0, 4.0], "dP": dP, "dQ": dQ,
                                "Q_fp64": [float(x) for x in res["fp64"]["Q"]],
                                "t2E_fp64": [float(t * t * x) for t, x in zip((1, 2, 3, 4), res["fp64"]["E"])],
                                "start": f"{N_THERM} further rounds after the timed steps"}
        line["dP_flow_max"] = max(dP)
        line["dQ_flow_max"] = max(dQ)
        if "fp32" in res and a.prec != "fp32":
            r18 = res["fp32"]
            line["fp32_18"] = {
                "link_updates_per_s": r18["link_updates_per_s"], "flow_steps_per_s": r18["flow_steps_per_s"],
                "sweep_roofline": r18["sweep_roofline"],
                "over_fp64": {"link_updates": r18["link_updates_per_s"] / res["fp64"]["link_updates_per_s"],
                              "flow_steps": r18["flow_steps_per_s"] / res["fp64"]["flow_steps_per_s"]},
                "dP_vs_fp64": max(abs(x - y) for x, y in zip(r18["plaq"], res["fp64"]["plaq"])),
                "dQ_vs_fp64": max(abs(x - y) for x, y in zip(r18["Q"], res["fp64"]["Q"]))}
        # the error against the FP64 oracle: the FP64 GPU flow is pinned to the reference's own
        # FP64 flow within 1e-10 in Q and 1e-12 in P over 400 steps at 32^4
        # (tests/test_gpu_large.py::TestFlowToFour::test_fp64), so the FP32-vs-FP64 differences
        # above are the FP32 errors against the oracle to that accuracy
        line["dQ_vs_oracle_abs"] = max(dQ)
        line["dP_vs_oracle_abs"] = max(dP)
        line["error_bound_1e-6"] = {"dP": bool(max(dP) <= 1e-6), "dQ": bool(max(dQ) <= 1e-6)}
        line["dP_flow_max_rel"] = max(d / abs(p) for d, p in zip(dP, res["fp64"]["plaq"]))
        line["dQ_flow_max_rel"] = max(d / max(abs(q), 1.0) for d, q in zip(dQ, res["fp64"]["Q"]))
        line["flow_roofline"] = flow_roofline(torch, a.prec, V, res[a.prec]["flow_ms"], res["fp64"]["flow_ms"], peak)

        # ---- e2e through the public API with host buffers: H2D of the step's links from pinned
        # memory, the sweep round, D2H of the plaquette
        pinned = torch.empty(therm.size, dtype=torch.float64, pin_memory=True)
        host = pinned.numpy().reshape(therm.shape)
        host[...] = therm
        # Two handles, each driven by its own host thread (the C ABI serialises calls per handle
        # only, and ctypes releases the GIL inside them), so that one handle's upload overlaps
        # the other's sweeps; every step still uploads its whole field and reads its plaquette.
        fields = [lt.GaugeField(ext, a.prec) for _ in range(2)]
        # warm-up: two uploads per handle (a handle streamed into sets up its pinned packing
        # buffer at its second upload), a round and a plaquette
        for F in fields:
            for _ in range(2):
                F.upload(host)
            sweep_round(F)
            lt.PlaquetteSum(F)
        n_e2e = max(3, min(a.steps, 10))
        errors = []

        def e2e_worker(F, n):
            try:
                c = 0
                for _ in range(n):
                    F.upload(host)
                    c = lt.UpdateSweeps(F, BETA, 1, N_HB, N_OR, SEED + rank, c)
                    lt.PlaquetteSum(F)
            except Exception as e:   # reported below
                errors.append(e)

        workers = [threading.Thread(target=e2e_worker, args=(F, n_e2e)) for F in fields]
        barrier()
        t0 = time.perf_counter()
        for w in workers:
            w.start()
        for w in workers:
            w.join()
        dt = max_over_ranks(time.perf_counter() - t0)
        if errors:
            raise errors[0]
        # lt_upload_links reads the step's FP64 reference-layout links (host input); for two-row
        # FP32 storage it packs most of them into the stored format on the host threads and
        # copies the rest as FP64 (converted on the device): lt_upload_bytes counts what crosses
        # PCIe
        pcie = fields[0].upload_bytes(host)
        line["e2e"] = {"value": world * 2 * n_e2e * upd_per_step / dt, "unit": UNIT,
                       "h2d_bytes_per_step": pcie, "d2h_bytes_per_step": 8,
                       "host_input_bytes_per_step": int(therm.nbytes),
                       "path": "lt_upload_links (FP64 reference layout in from pinned memory: 70 % of the sites "
                               "packed to the stored format on the host threads and copied chunk by chunk, the rest "
                               "copied as FP64 and converted on the device) + lt_update_sweeps + lt_plaquette_sum, "
                               "two handles on two host threads"}
        del fields

        # ---- the other configurations' rates (each bounded to a few seconds)
        line["secondary"] = secondary_rates(lt, torch, timed, a.prec)

        # ---- CPU baseline on this host, rank 0, bounded sample
        if rank == 0:
            cb = cpu_reference_sample(a.size, therm, 2, 10)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            if "flow_steps_per_s" in cb:
                line["cpu_baseline"]["flow_steps_per_s"] = cb["flow_steps_per_s"]
                # each GPU arm over the reference's CPU code, sweeps and flow
                line["gpu_over_cpu"] = {
                    "bulk_link_updates": value / world / cb["value"],
                    "fp64_link_updates": line["fp64"]["link_updates_per_s"] / cb["value"],
                    "bulk_flow_steps": line["flow_steps_per_s"] / cb["flow_steps_per_s"],
                    "fp64_flow_steps": line["fp64"]["flow_steps_per_s"] / cb["flow_steps_per_s"]}
            # the MetaD force at 16^4 on the reference's code (3 evaluations, about 3 s on 16 cores)
            sys.path.insert(0, os.path.join(ROOT, "tests"))
            from ltref import haar_links_numpy as _haar
            try:
                ref16 = CpuReference(16)
            except (FileNotFoundError, OSError):
                ref16 = None
            if ref16 is not None and hasattr(ref16.lib, "ref_metad_force_seconds"):
                cpu_force = ref16.metad_force_rate(_haar((16,) * 4, SEED), 3)
                line["cpu_baseline"]["metad_force_evals_per_s_16^4"] = cpu_force
                gpu_force = line.get("secondary", {}).get("metad_force_evals_per_s_16^4")
                if gpu_force and "gpu_over_cpu" in line:
                    line["gpu_over_cpu"]["metad_force"] = gpu_force / cpu_force

    if rank == 0:
        print(json.dumps(line, default=_jsonable))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
