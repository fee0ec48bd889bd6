"""Synthetic workloads of the benchmark configurations (seeded, no datasets).

Each builder returns plain Python descriptions (rule factors, leg
(sector, degeneracy) lists) so the same shapes can be instantiated with the
device facade (``tenet_b200.typed``) or with any CPU checker.

* ``u1_compose_permute``: U(1) V with charges -2..2, degeneracies
  [4, 8, 12, 8, 4]; A, B : (V x V) <- (V x V).
* ``su2_itebd``: SU(2) W with 2j = 0..4, degeneracies [40, 64, 64, 40, 16];
  P spin-1/2.
* ``hubbard_batch``: fZ2 x U(1) x SU(2) W of 60 sectors drawn from
  (parity, charge in [-7, 7], 2j in 0..6) with parity tied to half-integer
  spin; degeneracies geometric with mean 48 clipped to [1, 256]; P has
  sectors (0,0,0), (1,1,1/2), (0,2,0) of multiplicity 1.
* ``su2_heff``: SU(2) MPS x with W spins 0..4 (2j = 0..8), degeneracies
  [256, 512, 768, 1024, 1024, 768, 512, 256, 128]; MPO bond M = spins {0, 1}
  with multiplicities [2, 1]; P spin-1/2.
"""

from __future__ import annotations

import numpy as np


def u1_compose_permute():
    v = [((-2,), 4), ((-1,), 8), ((0,), 12), ((1,), 8), ((2,), 4)]
    return dict(factors=["U1"], V=v)


def su2_itebd():
    w = [((0,), 40), ((1,), 64), ((2,), 64), ((3,), 40), ((4,), 16)]
    p = [((1,), 1)]
    return dict(factors=["SU2"], W=w, P=p)


def hubbard_batch(seed: int = 0, nsectors: int = 60, mean: float = 48.0):
    rng = np.random.default_rng(seed)
    cand = [((tj % 2), q, tj) for q in range(-7, 8) for tj in range(0, 7)]
    pick = sorted(rng.choice(len(cand), size=nsectors, replace=False))
    degs = np.clip(rng.geometric(1.0 / mean, size=nsectors), 1, 256)
    w = [(cand[i], int(d)) for i, d in zip(pick, degs)]
    p = [((0, 0, 0), 1), ((1, 1, 1), 1), ((0, 2, 0), 1)]
    return dict(factors=["FZ2", "U1", "SU2"], W=w, P=p)


def su2_heff():
    w = [((tj,), d) for tj, d in zip(range(0, 9), [256, 512, 768, 1024, 1024, 768, 512, 256, 128])]
    m = [((0,), 2), ((2,), 1)]
    p = [((1,), 1)]
    return dict(factors=["SU2"], W=w, M=m, P=p)


def splitmix_normal(seed: int, n: int) -> np.ndarray:
    """N(0,1) entries from the splitmix64 stream of ``TensorMap::rand_with_seed``
    (tenet/src/typed.rs:2086-2093) through a Box-Muller map over consecutive
    uniform pairs; the reference itself has no normal sampler."""
    idx = np.arange(1, 2 * n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        v = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        v = (v ^ (v >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        v = (v ^ (v >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        v = v ^ (v >> np.uint64(31))
    u = (v >> np.uint64(11)).astype(np.float64) / float(1 << 52) - 1.0
    u1 = (1.0 - u[0::2]) * 0.5
    u2 = (u[1::2] + 1.0) * 0.5
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)
