"""Algorithmic work counts of the pair passes, for roofline fractions.

FLOPs per pair are counted from the CUDA C++ source formulas of eval_fused.cu (an FMA counts two,
each square root, reciprocal, divide and exponential counts one), on the path most pairs take:
the long-range Taylor branch of the HCT integral (r > 4 s_j) in GB passes 1 and 3, a
non-excluded pair in pass 2, zero salt concentration (no Debye-Hueckel exponential).

  pass 1 (Born radii)        48 = coordinate difference 9 + r^2 5 + sqrt, 1/r 2
                                  + two HCT integrals 2 x 15 + psi updates 2
  pass 2 (Coulomb, LJ, GB)   79 = difference 9 + r^2 5 + q_i q_j 1 + Coulomb / LJ 21
                                  + GB pair energy and force 31 + force accumulation 12
  pass 3 (radii chain rule)  63 = difference 9 + r^2 5 + sqrt, 1/r 2
                                  + two HCT derivatives 2 x 16 + combination 3 + accumulation 12

Every unordered pair of a molecule is visited once per pass (excluded pairs still count: GB
ignores exclusions).  Padding slots of partial tiles are not counted.
"""
from __future__ import annotations

import numpy as np

FLOPS_PASS1 = 48
FLOPS_PASS2 = 79
FLOPS_PASS3 = 63
FLOPS_PER_PAIR_FORCE = FLOPS_PASS1 + FLOPS_PASS2 + FLOPS_PASS3   # force + energy evaluation
FLOPS_PER_PAIR_ENERGY = FLOPS_PASS1 + 45                         # energy only: no pass 3, no forces

# B200: 148 SMs x 128 FP32 lanes x 2 flops per FMA at the 1965 MHz maximum SM clock
SM_COUNT = 148
FP32_LANES_PER_SM = 128


def fp32_peak_tflops(sm_mhz: float = 1965.0) -> float:
    return SM_COUNT * FP32_LANES_PER_SM * 2 * sm_mhz * 1.0e6 / 1.0e12


def pair_count(natoms) -> int:
    n = np.asarray(natoms, dtype=np.int64)
    return int((n * (n - 1) // 2).sum())


def flops_per_evaluation(natoms, force: bool = True) -> float:
    return float(pair_count(natoms)) * (FLOPS_PER_PAIR_FORCE if force else FLOPS_PER_PAIR_ENERGY)
