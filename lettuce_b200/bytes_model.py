"""Algorithmic HBM bytes and flops per unit of work, one place for the bench's roofline figures.

b is the stored link size (144 B FP64 = 18 doubles, 72 B FP32 = 18 floats, 48 B FP32-12 = two
rows), b_alg the algebra size (8 reals: 64 B FP64, 32 B FP32).  "Algorithmic" counts each
field byte a kernel must move at least once; neighbour re-reads are not counted (they are L2's
job), so DRAM traffic measured by ncu above these figures means wasted re-reads.

* sweep (one (mu, parity) sub-sweep, heatbath or overrelaxation): V/2 active links read and
  written, the V/2 opposite-parity mu links and the 3V links of the other directions read:
  9 b per link update.
* RK3 flow step (three fused stages, U ping-pong, Z written by stages 1-2 and read by 2-3):
  3 (read U + write U) + 2 Z writes + 2 Z reads = 6 b + 4 b_alg per link.
* clover Q / E, plaquette: every link read once: 4 b per site.
* metadynamics force through n stout levels (forward 2 n b, clover + derivative about 3.5 b,
  backward about 4.9 b per level): (6.9 n + 3.5) b per link, about 70k flops per link for
  n = 4.

Flops use 198 real flops per 3x3 complex product (27 complex multiplies at 6 flops plus 18
complex additions at 2): staple about 2.5k, heatbath about 4.0k and overrelaxation about
3.9k per link update, an RK3 step about 10k per link, clover Q about 15k per site.
"""
from __future__ import annotations

LINK_BYTES = {"fp64": 144, "fp32": 72, "fp32_12": 48}
ALG_BYTES = {"fp64": 64, "fp32": 32, "fp32_12": 32}

FLOPS = {"overrelax": 3.9e3, "heatbath": 4.0e3, "flow_step": 10.0e3, "clover_site": 15.0e3,
         "metad_force_n4": 70.0e3}


def sweep_bytes_per_update(prec: str) -> int:
    return 9 * LINK_BYTES[prec]


def sweep_launch_bytes(prec: str, volume: int) -> int:
    """One (mu, parity) launch: V/2 link updates."""
    return sweep_bytes_per_update(prec) * (volume // 2)


def flow_step_bytes_per_link(prec: str) -> int:
    return 6 * LINK_BYTES[prec] + 4 * ALG_BYTES[prec]


def flow_stage_bytes(prec: str, volume: int, read_z: bool, write_z: bool) -> int:
    """One fused stage over all 4V links: U read and written, Z read and/or written."""
    per_link = 2 * LINK_BYTES[prec] + ALG_BYTES[prec] * (int(read_z) + int(write_z))
    return per_link * 4 * volume


def clover_bytes_per_site(prec: str) -> int:
    return 4 * LINK_BYTES[prec]


def metad_force_bytes_per_link(prec: str, n_stout: int) -> float:
    return (6.9 * n_stout + 3.5) * LINK_BYTES[prec]
