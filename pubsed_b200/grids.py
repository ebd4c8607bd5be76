"""Bin-edge grids and zone models with the reference's construction rules.

`LocGrid` reproduces locate_array's initialisers (src/utils/locate_array.cpp:
init(start, stop, del) :25-46, log_init :54-81, init(start, stop, n) :88-108);
the arithmetic is the same IEEE double sequence, so the walls are identical
to the ones the reference builds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .abi import LOC_FLEX, LOC_LIN, LOC_LOG, LOC_NONE

PI = 3.14159  # physical_constants::pi (src/utils/physical_constants.h:9)


@dataclass
class LocGrid:
    right: np.ndarray  # right walls, float64
    min: float
    delta: float
    type: int

    @property
    def n(self) -> int:
        return int(self.right.size)

    def left(self) -> np.ndarray:
        return np.concatenate([[self.min], self.right[:-1]])

    def width(self) -> np.ndarray:
        return self.right - self.left()

    def center(self) -> np.ndarray:
        return 0.5 * (self.left() + self.right)

    def delta_at(self, i: int) -> float:
        """locate_array::delta (locate_array.h:69-72)"""
        return float(self.right[0] - self.min) if i == 0 else float(self.right[i] - self.right[i - 1])

    def center_at(self, i: int) -> float:
        """locate_array::center (locate_array.h:54-57)"""
        return float(0.5 * (self.min + self.right[0])) if i == 0 else float(0.5 * (self.right[i - 1] + self.right[i]))

    def scaled(self, e: float) -> "LocGrid":
        """locate_array::scale (locate_array.cpp:540-548)"""
        d = self.delta * e if self.type == LOC_LIN else self.delta
        return LocGrid(self.right * e, self.min * e, d, self.type)


def catch_all() -> LocGrid:
    return LocGrid(np.array([math.inf]), -math.inf, 0.0, LOC_NONE)


def lin_grid(start: float, stop: float, delta: float) -> LocGrid:
    """locate_array::init(start, stop, del)"""
    if start >= stop:
        return catch_all()
    n = max(int(math.ceil((stop - start) / delta)), 1)
    x = [start + (i + 1) * delta for i in range(n - 1)] + [stop]
    return LocGrid(np.array(x, dtype=np.float64), start, delta, LOC_LIN)


def lin_grid_n(start: float, stop: float, n: int) -> LocGrid:
    """locate_array::init(start, stop, int n)"""
    if start == stop or n == 0:
        return catch_all()
    d = (stop - start) / float(n)
    x = [start + (i + 1) * d for i in range(n - 1)] + [stop]
    return LocGrid(np.array(x, dtype=np.float64), start, d, LOC_LIN)


def log_grid(start: float, stop: float, delta: float) -> LocGrid:
    """locate_array::log_init(start, stop, del)"""
    if start >= stop:
        return catch_all()
    arr = []
    v = start + start * delta
    while v < stop:
        arr.append(v)
        v = v + v * delta
    arr.append(stop)
    return LocGrid(np.array(arr, dtype=np.float64), start, delta, LOC_LOG)


def grid_from_spec(spec) -> LocGrid:
    """{start, stop, del[, log]} as transport_nu_grid / spectrum_nu_grid
    (transport_init.cpp:147-157, spectrum_array.cpp:51-62)"""
    spec = list(spec)
    if len(spec) not in (3, 4):
        raise ValueError("improperly defined nu grid; need {nu_1, nu_2, dnu, (log?)}")
    if len(spec) == 4 and spec[3] == 1:
        return log_grid(float(spec[0]), float(spec[1]), float(spec[2]))
    return lin_grid(float(spec[0]), float(spec[1]), float(spec[2]))


def log_delta_for_bins(start: float, stop: float, nbins: int) -> float:
    """Smallest-change `del` for which log_grid(start, stop, del) has exactly
    nbins bins (the while-loop can add or drop one edge)."""
    d = (stop / start) ** (1.0 / nbins) - 1.0
    for _ in range(64):
        n = log_grid(start, stop, d).n
        if n == nbins:
            return d
        d *= (1 + 1e-9) if n > nbins else (1 - 1e-9)
    raise RuntimeError("could not find a log spacing with %d bins" % nbins)


def shell_volumes(r_min: float, r_out: np.ndarray) -> np.ndarray:
    """grid_1D_sphere zone volumes (grid_1D_sphere.cpp:365-369)"""
    vol = np.empty_like(r_out)
    for i in range(r_out.size):
        r0 = r_min if i == 0 else r_out[i - 1]
        r = r_out[i]
        vol[i] = 4.0 * PI / 3.0 * (r * r * r - r0 * r0 * r0)
    return vol
