"""Ensembles: lattices of uneven extents advanced by one batched launch per sub-sweep.

Each lattice k of an ensemble draws the heatbath stream keyed seed + k, so one round on the
ensemble must reproduce, link for link, the same round run on each lattice alone through
lt_update_sweeps (same update code, same random numbers).  The tempering swap follows the
reference's MetadynamicsTemperingKernel rule (updates/tempering.hpp:51-72)."""
import numpy as np
import pytest

import lettuce_b200 as lt
from ltref import rel_err

pytestmark = pytest.mark.gpu

EXTS = [(4, 4, 4, 4), (4, 6, 8, 10), (6, 6, 6, 8), (8, 8, 8, 8)]
BETAS = [5.8, 6.0, 6.1, 6.2]


@pytest.mark.parametrize("prec", ["fp64", "fp32_12"])
def test_ensemble_matches_single_lattice(prec):
    seed = 4242
    starts = [lt.haar_links(e, 10 + k) for k, e in enumerate(EXTS)]
    lats = []
    for e, U in zip(EXTS, starts):
        G = lt.GaugeField(e, prec)
        G.upload(U)
        lats.append(G)
    ens = lt.Ensemble(lats, BETAS, seed=seed)
    ens.counter.value = 7
    ens.sweeps(2, 1, 3)
    assert ens.counter.value == 9
    for k, (e, U) in enumerate(zip(EXTS, starts)):
        H = lt.GaugeField(e, prec)
        H.upload(U)
        lt.UpdateSweeps(H, BETAS[k], 2, 1, 3, seed=seed + k, counter=7)
        # same update code and random numbers; only FMA contraction may differ between kernels
        assert rel_err(lats[k].download(), H.download()) < (1e-12 if prec == "fp64" else 1e-5), k


def test_autotune_keeps_chains_and_block_sizes_agree():
    lats = [lt.GaugeField(e, "fp32_12") for e in EXTS]
    for k, G in enumerate(lats):
        G.SetToHaarRandom(k)
    before = [G.download() for G in lats]
    ens = lt.Ensemble(lats, BETAS, seed=1)
    hb, orx = ens.autotune()
    assert hb in (64, 128, 256) and orx in (64, 128, 256)
    for G, b in zip(lats, before):
        assert np.array_equal(G.download(), b)
    # the result of a round does not depend on the block size
    results = []
    for threads in (64, 256):
        for G, b in zip(lats, before):
            G.upload(b)
        ens.set_block(threads, threads)
        ens.counter.value = 0
        ens.sweeps(1, 1, 1)
        results.append([G.download() for G in lats])
    for a, b in zip(*results):
        assert rel_err(a, b) < 1e-5


def test_reverse_round_overrelaxation_conserves_action():
    lats = [lt.GaugeField(e, "fp64") for e in EXTS]
    for k, G in enumerate(lats):
        G.SetToHaarRandom(50 + k)
        lt.UpdateSweeps(G, 6.0, 3, 1, 0, seed=k)
    p0 = [lt.PlaquetteSum(G) for G in lats]
    ens = lt.Ensemble(lats, BETAS, seed=1)
    fwd = None
    for reverse in (True, False):
        ens.sweeps(3, 0, 1, reverse=reverse)
        for G, p in zip(lats, p0):
            assert lt.PlaquetteSum(G) == pytest.approx(p, rel=1e-11)
        if fwd is None:
            fwd = [G.download() for G in lats]
    assert not np.array_equal(fwd[0], lats[0].download())


def test_pt_metad_streams_and_chains():
    from lettuce_b200.tempering import PTMetaD
    pt = PTMetaD((8, 8, 8, 8), [1.0, 2 / 3, 1 / 3, 0.0], 6.0, chains=[((6, 6, 6, 6), 5.9), ((4, 6, 8, 8), 6.1)],
                 prec="fp32", seed=3, n_smear=2)
    p0 = [lt.PlaquetteSum(G) / G.Volume() / 18 for G in pt.streams + pt.chains]
    for _ in range(12):
        pt.sweep()
    p1 = [lt.PlaquetteSum(G) / G.Volume() / 18 for G in pt.streams + pt.chains]
    assert all(b > a + 0.2 for a, b in zip(p0, p1))          # all lattices moved off the Haar start
    assert pt.stats["swap_proposals"] == 6 * 2 + 6 * 1
    assert pt.stats["bias_accept"] > 0
    g = pt.bias.grid()
    assert g.max() > 0 and np.allclose(g, g[::-1])
    assert sorted(pt.scales) == [0.0, 1 / 3, 2 / 3, 1.0]


def test_tempering_swap_rule():
    a, b = lt.GaugeField((4, 4, 4, 4)), lt.GaugeField((4, 4, 4, 4))
    a.SetToHaarRandom(1)
    b.SetToIdentity()
    Ua = a.download()
    bias = lt.MetaBiasPotential(-8, 8, 800, 0.05, 0.08, 10, 1000)
    bias.GeneratePotentialFrom(lambda q: q * q)
    # dE = (s_a - s_b) (V(q_b) - V(q_a)) = (0 - 1) (1 - 4) = 3: exp(-3) = 0.0498
    acc, dE = lt.TemperingSwap(a, b, bias, 0.0, 1.0, 2.0, 1.0, 0.9)
    assert dE == pytest.approx(3.0, rel=1e-6) and not acc
    assert np.array_equal(a.download(), Ua)
    acc, dE = lt.TemperingSwap(a, b, bias, 0.0, 1.0, 2.0, 1.0, 0.01)
    assert acc
    assert np.array_equal(b.download(), Ua)
    assert lt.PlaquetteSum(a) == pytest.approx(18 * 256, rel=1e-14)


@pytest.mark.parametrize("prec", ["fp64", "fp32_12"])
@pytest.mark.parametrize("reverse", [False, True])
def test_persistent_round_matches_graph(prec, reverse):
    """One cooperative launch per round (grid barriers between the sub-sweeps) advances every
    lattice exactly as the graph of batched launches: same sub-sweeps in the same order, same
    heatbath counters (two heatbath sweeps per round check their order)."""
    starts = [lt.haar_links(e, 30 + k) for k, e in enumerate(EXTS)]
    out = {}
    for mode in ("graph", "persistent"):
        lats = []
        for e, U in zip(EXTS, starts):
            G = lt.GaugeField(e, prec)
            G.upload(U)
            lats.append(G)
        ens = lt.Ensemble(lats, BETAS, seed=99)
        ens.set_mode(mode)
        assert ens.get_mode()[0] == mode
        ens.counter.value = 3
        ens.sweeps(2, 2, 3, reverse=reverse)
        assert ens.counter.value == 7
        out[mode] = [G.download() for G in lats]
    for a, b in zip(out["graph"], out["persistent"]):
        assert rel_err(b, a) < (1e-12 if prec == "fp64" else 1e-5)


def test_persistent_barrier_gives_up_and_recovers():
    """A wait bound of zero polls makes the grid barriers give up at once: the call returns
    LT_ERR_TIMEOUT instead of waiting, and with the default bound the same ensemble runs a
    correct round afterwards."""
    from lettuce_b200._lib import LT_ERR_TIMEOUT
    starts = [lt.haar_links(e, 50 + k) for k, e in enumerate(EXTS)]
    lats = [lt.GaugeField(e, "fp32_12") for e in EXTS]
    for G, U in zip(lats, starts):
        G.upload(U)
    ens = lt.Ensemble(lats, BETAS, seed=5)
    ens.set_mode("persistent")
    ens.set_barrier_polls(0)
    with pytest.raises(lt.LettuceError) as err:
        ens.sweeps(1, 1, 1)
    assert err.value.code == LT_ERR_TIMEOUT
    assert b"gave up" in lt.lib().lt_last_error()
    ens.set_barrier_polls(10_000_000)
    for G, U in zip(lats, starts):
        G.upload(U)
    ens.counter.value = 0
    ens.sweeps(1, 1, 1)
    got = [G.download() for G in lats]
    ref = []
    for k, (e, U) in enumerate(zip(EXTS, starts)):
        H = lt.GaugeField(e, "fp32_12")
        H.upload(U)
        lt.UpdateSweeps(H, BETAS[k], 1, 1, 1, seed=5 + k, counter=0)
        ref.append(H.download())
    for a, b in zip(got, ref):
        assert rel_err(a, b) < 1e-5


def test_autotune_chooses_a_mode():
    lats = [lt.GaugeField(e, "fp32_12") for e in EXTS]
    for k, G in enumerate(lats):
        G.SetToHaarRandom(k)
    before = [G.download() for G in lats]
    ens = lt.Ensemble(lats, BETAS, seed=1)
    ens.autotune()
    mode, bps = ens.get_mode()
    assert mode in ("graph", "persistent")
    assert (bps >= 1) if mode == "persistent" else (bps == 0)
    for G, b in zip(lats, before):
        assert np.array_equal(G.download(), b)
