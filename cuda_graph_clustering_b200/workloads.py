"""Seeded synthetic workloads of the benchmarks: the batched mix and the serving request stream.

Both are defined here, by this project (the reference has no batched or serving mode): every random
quantity is a draw from one sequential splitmix64 stream, using the same helpers as the solver
(DrawUnit = 24-bit float in [0, 1), DrawBelow = multiply-shift), so a master seed fixes everything.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

GAMMA = 0x9E3779B97F4A7C15
MASK = (1 << 64) - 1


def _mix(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def stream_seed(seed: int, stream: int, step: int) -> int:
    s = (seed ^ ((stream * 0xD1B54A32D192ED03) & MASK) ^ ((step * 0xA0761D6478BD642F) & MASK)) & MASK
    return (s + GAMMA) & MASK


class Draws:
    """One sequential splitmix64 stream (the solver's StreamSeed / DrawUnit / DrawBelow)."""

    def __init__(self, seed: int, stream: int):
        self.state = stream_seed(seed, stream, 0)

    def u64(self) -> int:
        self.state = (self.state + GAMMA) & MASK
        return _mix(self.state)

    def unit(self) -> float:
        return float((self.u64() >> 32) >> 8) / 16777216.0

    def below(self, bound: int) -> int:
        return ((self.u64() >> 32) * bound) >> 32


@dataclass
class Instance:
    n: int
    parts: int        # planted communities
    p_in: float
    p_out: float
    flip: float
    graph_seed: int
    k: int
    population: int
    seed: int
    iterations: int
    erdos_renyi: bool = False
    density: float = 0.0


def batched_mix(count: int = 256, master: int = 7, iterations: int = 100) -> list[Instance]:
    """The batched mix: n log-uniform in [200, 20000], k_true uniform in 2..16, planted partition into
    k_true equal-probability clusters with p_in in [0.3, 0.8], p_out in [0.01, 0.2], every pair flipped with
    probability in [0.05, 0.2]; solved with k uniform in 2..64, population in {32, 64, 128}, gww 0.1,
    `iterations` iterations without early stop."""
    d = Draws(master, 0xB47C4)
    out = []
    for _ in range(count):
        n = int(round(math.exp(math.log(200) + d.unit() * math.log(100))))
        parts = 2 + d.below(15)
        p_in = 0.3 + 0.5 * d.unit()
        p_out = 0.01 + 0.19 * d.unit()
        flip = 0.05 + 0.15 * d.unit()
        k = 2 + d.below(63)
        pop = (32, 64, 128)[d.below(3)]
        out.append(Instance(n, parts, p_in, p_out, flip, d.u64(), k, pop, d.u64(), iterations))
    return out


def serving_requests(count: int, rate: float, master: int = 11, max_n: int = 50000,
                     population: int = 64, iterations: int = 50) -> list[tuple[float, Instance]]:
    """Poisson arrivals at `rate` requests/s: (arrival time in s, instance).  Each request is an
    Erdős–Rényi or planted graph (even odds) with n log-uniform in [500, max_n], density uniform in
    [0.01, 0.5] (planted: p_in = density, p_out = density / 4, up to 8 communities), k uniform in 2..32,
    the given population and iteration count, and a per-request seed."""
    d = Draws(master, 0x5E7E)
    t = 0.0
    out = []
    for _ in range(count):
        t += -math.log(1.0 - d.unit()) / rate
        n = int(round(math.exp(math.log(500) + d.unit() * math.log(max_n / 500))))
        density = 0.01 + 0.49 * d.unit()
        er = d.below(2) == 0
        k = 2 + d.below(31)
        parts = 2 + d.below(7)
        inst = Instance(n, parts, density, density / 4, 0.0, d.u64(), k, population, d.u64(), iterations,
                        erdos_renyi=er, density=density)
        out.append((t, inst))
    return out
