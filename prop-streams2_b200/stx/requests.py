"""Requests of the serving loop (stx.serve) and the seeded served mix, kept
apart from the server so that building a request stream touches no CUDA
setting: the server module sets process-wide CUDA options when it is
imported."""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np

from . import mech as M


@dataclasses.dataclass
class Request:
    rid: int
    kind: str                      # "reactor" | "flame1d" | "tube2d"
    arrival: float                 # seconds after the start of the run
    params: dict
    steps: int = 0                 # grid solves: RK steps to take
    admitted: Optional[float] = None
    done: Optional[float] = None
    result: Optional[dict] = None

    @property
    def latency(self) -> Optional[float]:
        return None if self.done is None else self.done - self.arrival


def mixed_requests(n: int, rate: float, seed: int, mech: M.Mechanism, flame_steps: int = 20,
                   tube_steps: int = 10, frac=(0.6, 0.3, 0.1), flame_nx=(512, 4096), tube_shape=(512, 128)):
    """The served mix: Poisson arrivals at `rate` per second; 60 % 0-D reactors
    (the batched-reactor distribution), 30 % 1-D flames with nx ~ U{512..4096},
    phi ~ U(0.5, 1.5), Tu ~ U(300, 800) K, 10 % 2-D shock tubes of 512 x 128
    cells; seeded."""
    from .reactors import sample_h2air
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    kinds = rng.choice(3, size=n, p=np.asarray(frac) / np.sum(frac))
    T0, p0, Y0 = sample_h2air(n, seed + 1, mech)
    reqs = []
    for i in range(n):
        if kinds[i] == 0:
            reqs.append(Request(i, "reactor", float(t[i]), {"T0": float(T0[i]), "p0": float(p0[i]),
                                                           "Y0": Y0[:, i].copy()}))
        elif kinds[i] == 1:
            reqs.append(Request(i, "flame1d", float(t[i]),
                                {"nx": int(rng.integers(flame_nx[0], flame_nx[1] + 1)),
                                 "phi": float(rng.uniform(0.5, 1.5)), "Tu": float(rng.uniform(300.0, 800.0))},
                                steps=flame_steps))
        else:
            reqs.append(Request(i, "tube2d", float(t[i]), {"nx": tube_shape[0], "ny": tube_shape[1]},
                                steps=tube_steps))
    return reqs
