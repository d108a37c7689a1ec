"""The C++20 drop-in header (include/lettuce_gpu.hpp): a SU3_main.cpp-style program compiles
and links against the C-ABI library (CPU) and runs on the GPU with the same numbers as the
Python mirror (GPU)."""
import os
import subprocess

import pytest

import lettuce_b200 as lt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "drop_in_main.cpp")
EXE = os.path.join(ROOT, "tests", "cpp", "drop_in_main")


def build_exe():
    lib_dir = os.path.dirname(lt.LIB_PATH)
    subprocess.run(["g++", "-std=c++20", "-O2", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
                    "-L", lib_dir, "-llettuce_b200", f"-Wl,-rpath,{lib_dir}", "-o", EXE], check=True)
    return EXE


def test_dropin_compiles_and_links():
    assert os.path.exists(build_exe())


@pytest.mark.gpu
def test_dropin_runs_like_python_mirror(tmp_path):
    out = subprocess.run([build_exe(), "8", str(tmp_path / "ckpt")], capture_output=True, text=True,
                         check=True).stdout
    lines = dict((l.split()[0] + (l.split()[1] if l.startswith("flow") else ""), l) for l in out.splitlines())
    # the same sequence through the Python mirror
    G = lt.GaugeField((8, 8, 8, 8))
    G.SetToHaarRandom(2024)
    hb = lt.HeatbathKernel(G, lt.WilsonAction(6.0), seed=7)
    orx = lt.OverrelaxationSubgroupKernel(G)
    for _ in range(20):
        lt.Iterator.Checkerboard4(hb, 1)
        lt.Iterator.Checkerboard4(orx, 4)
    p = lt.PlaquetteSum(G) / 8 ** 4 / 18
    assert float(lines["plaquette"].split()[1]) == pytest.approx(p, rel=1e-14)
    assert 0.55 < p < 0.65
    assert "metad" in out and "copy" in out
    par = lines["parity"].split()
    assert abs(float(par[2])) < 1.0   # OMF_4 at 10 steps conserves H well
    assert float(par[5]) == pytest.approx(-float(par[4]), rel=1e-10, abs=1e-12)
    # measurement bundle and an Euler flow on the same thermalised field
    b = lines["bundle"].split()
    m = lt.Measure(G, 6.0)
    assert float(b[2]) == pytest.approx(m["Improved_Action"], rel=1e-13)
    assert float(b[4]) == pytest.approx(m["Wilson_loop(L=2)"], rel=1e-13)
    assert float(b[6]) == pytest.approx(m["Wilson_loop(L=4)"], rel=1e-13)
    assert complex(float(b[8]), float(b[9])) == pytest.approx(m["Polyakov_loop"], abs=1e-14)
    assert float(b[11]) == pytest.approx(m["TopChargePlaq"], abs=1e-13)
    assert float(b[13]) == pytest.approx(m["TopChargeClov"], abs=1e-13)
    assert float(b[15]) == pytest.approx(m["E_clov_timeslice"][0], rel=1e-13)
    F = lt.GaugeField((8, 8, 8, 8))
    lt.GradientFlowKernel(G, F, lt.Euler, None, 0.02)(5)
    assert float(lines["euler"].split()[2]) == pytest.approx(lt.EnergyDensityClover(F), rel=1e-13)
    tq = lines["tensor"].split()
    assert float(tq[2]) == pytest.approx(float(tq[3]), rel=1e-11, abs=1e-13)
    Fz = lt.GaugeField((8, 8, 8, 8))
    lt.GradientFlowKernel(G, Fz, lt.RK3, lt.ZeuthenFlow(), 0.01)(10)
    assert float(lines["zeuthen"].split()[2]) == pytest.approx(lt.EnergyDensityClover(Fz), rel=1e-13)
    # checkpoints: three rotations, restored field and Philox counter, a missing file rejected
    ck = lines["checkpoint"].split()
    assert int(ck[2]) == 20 + 3
    assert float(ck[5]) == float(ck[7])
    assert ck[9] == "0"
    for sub in ("", "backup1", "backup2"):
        assert (tmp_path / "ckpt" / sub / "config").exists()
