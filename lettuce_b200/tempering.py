"""Parallel-tempered metadynamics over streams with scaled biases, plus independent chains.

Generalises the reference's two-stream PT-MetaD loop (SU3_main.cpp:561-633,
LettuceGauge/updates/tempering.hpp:24-73) to n streams: stream k samples
exp(-S - s_k V(Q)), s_0 = 1 carries the metadynamics bias V (well-tempered, symmetric
deposits, actions/bias_potential/metadynamics.hpp:103-147), the other scales run down to 0
(an unbiased stream).  Q is the clover charge after n_smear stout steps (MetaCharge,
updates/hmc_metadynamics.hpp:302-310).

One sweep:
  1. every lattice (streams and the independent chains) gets one round of heatbath +
     overrelaxation sweeps through one Ensemble (batched launches replayed as a CUDA graph),
     in forward or reverse sub-sweep order with probability 1/2 each (the even mixture is
     reversible with respect to exp(-S));
  2. a biased stream keeps its new configuration with probability
     min(1, exp(-s_k [V(Q_new) - V(Q_old)])) and otherwise returns to the old one -- the
     round is the proposal, this step corrects for the bias;
  3. neighbouring streams (pairs (0,1),(2,3),... then (1,2),(3,4),... alternately) propose
     exchanges with the rule of tempering.hpp:51-72 generalised to scales (lt_tempering_swap);
  4. the bias gets a symmetric deposit at the charge of stream 0.

swap_decisions() is the same exchange rule as a pure function of gathered scalars; with
streams on different GPUs it exchanges the scales instead of the configurations, so only
(Q, s) pairs cross between ranks.
"""
from __future__ import annotations

import numpy as np

from .api import Ensemble, GaugeField, MetaBiasPotential, TemperingSwap, lib
from ._lib import check

import ctypes as C


def metad_charge(U: GaugeField, rho: float, n_smear: int) -> float:
    q = C.c_double()
    check(lib().lt_metad_charge(U.handle, float(rho), int(n_smear), C.byref(q)))
    return q.value


def swap_decisions(q, scales, potential, parity: int, uniforms):
    """Exchange decisions for neighbour pairs (i, i+1), i = parity, parity + 2, ...

    q[i], scales[i]: charge and bias scale of stream i; potential: V(Q); uniforms[i]: a
    uniform number for the pair starting at i.  Returns (new_scales, accepted pairs): an
    accepted pair exchanges its two scales (equivalently its configurations).
    dE = (s_i - s_{i+1}) (V(q_{i+1}) - V(q_i)), accepted when u <= exp(-dE)."""
    s = list(scales)
    accepted = []
    for i in range(parity, len(q) - 1, 2):
        dE = (s[i] - s[i + 1]) * (potential(q[i + 1]) - potential(q[i]))
        if uniforms[i] <= np.exp(-dE):
            s[i], s[i + 1] = s[i + 1], s[i]
            accepted.append(i)
    return s, accepted


class PTMetaD:
    """Streams of one extent with bias scales `scales` (scales[0] = 1 carries the bias) plus
    independent chains [(extent, beta), ...], all advanced by one Ensemble."""

    def __init__(self, stream_ext, scales, beta: float, chains=(), prec: str = "fp32", seed: int = 1,
                 bias_args=(-8.0, 8.0, 800, 0.05, 4 * 16.0 / 800, 10.0, 1000.0), rho: float = 0.12,
                 n_smear: int = 4, n_or: int = 4):
        self.scales = [float(s) for s in scales]
        self.n_streams = len(self.scales)
        self.rho, self.n_smear, self.n_or = float(rho), int(n_smear), int(n_or)
        self.rng = np.random.default_rng(seed)
        self.streams = []
        for k in range(self.n_streams):
            G = GaugeField(stream_ext, prec)
            G.SetToHaarRandom(seed * 1000 + k)
            self.streams.append(G)
        self.chains = []
        chain_betas = []
        for j, (ext, b) in enumerate(chains):
            G = GaugeField(ext, prec)
            G.SetToHaarRandom(seed * 1000 + 500 + j)
            self.chains.append(G)
            chain_betas.append(float(b))
        self.ensemble = Ensemble(self.streams + self.chains, [beta] * self.n_streams + chain_betas, seed)
        self.backup = [GaugeField(stream_ext, prec) for _ in range(self.n_streams)]
        self.bias = MetaBiasPotential(*bias_args)
        self.q = [metad_charge(G, self.rho, self.n_smear) for G in self.streams]
        self.n_sweep = 0
        self.stats = {"bias_accept": 0, "bias_proposals": 0, "swap_accept": 0, "swap_proposals": 0}

    def link_updates_per_sweep(self) -> int:
        v = sum(G.Volume() for G in self.streams + self.chains)
        return 4 * v * (1 + self.n_or)

    def sweep(self) -> None:
        biased = [k for k in range(self.n_streams) if self.scales[k] != 0.0]
        for k in biased:
            self.backup[k].assign(self.streams[k])
        self.ensemble.sweeps(1, 1, self.n_or, reverse=bool(self.rng.integers(2)))
        q_new = [metad_charge(G, self.rho, self.n_smear) for G in self.streams]
        for k in range(self.n_streams):
            if k in biased:
                dV = self.scales[k] * (self.bias.ReturnPotential(q_new[k]) - self.bias.ReturnPotential(self.q[k]))
                self.stats["bias_proposals"] += 1
                if self.rng.random() <= np.exp(-dV):
                    self.q[k] = q_new[k]
                    self.stats["bias_accept"] += 1
                else:
                    self.streams[k].assign(self.backup[k])
            else:
                self.q[k] = q_new[k]
        parity = self.n_sweep % 2
        for i in range(parity, self.n_streams - 1, 2):
            acc, _ = TemperingSwap(self.streams[i], self.streams[i + 1], self.bias, self.scales[i],
                                   self.scales[i + 1], self.q[i], self.q[i + 1], self.rng.random())
            self.stats["swap_proposals"] += 1
            if acc:
                self.q[i], self.q[i + 1] = self.q[i + 1], self.q[i]
                self.stats["swap_accept"] += 1
        k0 = self.scales.index(1.0) if 1.0 in self.scales else 0
        self.bias.UpdatePotentialSymmetric(self.q[k0])
        self.n_sweep += 1
