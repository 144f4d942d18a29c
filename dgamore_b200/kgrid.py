"""Host-side Brillouin-zone maps: irreducible wedge, its inverse map and multiplicities.

This is host precompute consumed by the device kernels (the (q_irr, w) work list, the IBZ->FBZ gather and the
lambda-correction weights).  It restates the upstream symmetry folding of ``KGrid``:

* ``inv_sym``  (dgamore/brillouin_zone.py:128-142): on a [0, 2pi) grid, index i > n/2 takes the value of n - i;
* ``x_y_sym`` etc. (brillouin_zone.py:145-176): element-wise minimum of the grid and its transpose, twice;
* ``set_irrk_maps`` (brillouin_zone.py:356-363): ``np.unique`` with return_index / inverse / counts.

The representative of each orbit is therefore its smallest flat index, and ``irrk_ind`` is sorted ascending,
which is also the order ``IAmNonLocal.reduce_q`` (n_point_base.py:406-424) produces for an irreducible q list.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SQUARE_2D = ("x-inv", "y-inv", "x-y-sym")
CUBIC_3D = ("x-inv", "y-inv", "z-inv", "x-y-sym", "x-z-sym", "y-z-sym")


def _inv_sym(mat: np.ndarray, axis: int) -> None:
    n = mat.shape[axis]
    half, odd = n // 2, n % 2
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    dst[axis] = slice(half + 1, None)
    src[axis] = slice(1, half + odd)
    mat[tuple(dst)] = np.flip(mat[tuple(src)], axis=axis)


def _pair_sym(mat: np.ndarray, a: int, b: int) -> None:
    if mat.shape[a] != mat.shape[b]:
        return
    merged = np.minimum(mat, mat.swapaxes(a, b))
    mat[...] = np.minimum(merged, merged.swapaxes(a, b))


def _apply(mat: np.ndarray, sym: str) -> None:
    if sym == "x-inv":
        _inv_sym(mat, 0)
    elif sym == "y-inv":
        _inv_sym(mat, 1)
    elif sym == "z-inv":
        _inv_sym(mat, 2)
    elif sym == "x-y-sym":
        _pair_sym(mat, 0, 1)
    elif sym == "x-z-sym":
        _pair_sym(mat, 0, 2)
    elif sym == "y-z-sym":
        _pair_sym(mat, 1, 2)
    else:
        raise ValueError(f"unknown symmetry {sym!r}")


@dataclass
class KGrid:
    """Momentum grid on [0, 2pi)^3 with the irreducible-wedge maps of the given index symmetries."""

    nk: tuple
    symmetries: tuple = SQUARE_2D
    irrk_ind: np.ndarray = field(init=False)
    irrk_inv: np.ndarray = field(init=False)
    irrk_count: np.ndarray = field(init=False)

    def __post_init__(self):
        self.nk = tuple(int(x) for x in self.nk)
        fbz2irrk = np.arange(int(np.prod(self.nk))).reshape(self.nk)
        for sym in self.symmetries or ():
            _apply(fbz2irrk, sym)
        _, self.irrk_ind, self.irrk_inv, self.irrk_count = np.unique(
            fbz2irrk, return_index=True, return_inverse=True, return_counts=True
        )
        self.irrk_inv = self.irrk_inv.reshape(-1)
        self.fbz2irrk = fbz2irrk

    @property
    def nk_tot(self) -> int:
        return int(np.prod(self.nk))

    @property
    def nk_irr(self) -> int:
        return int(len(self.irrk_ind))

    @property
    def kx(self):
        return np.linspace(0, 2 * np.pi, self.nk[0], endpoint=False)

    @property
    def ky(self):
        return np.linspace(0, 2 * np.pi, self.nk[1], endpoint=False)

    @property
    def kz(self):
        return np.linspace(0, 2 * np.pi, self.nk[2], endpoint=False)

    def get_q_list(self) -> np.ndarray:
        """All q-point index triples in C order (brillouin_zone.py:571-575)."""
        return np.array(np.unravel_index(np.arange(self.nk_tot), self.nk)).T

    def get_irrq_list(self) -> np.ndarray:
        """Index triples of the irreducible q points (brillouin_zone.py:577-581)."""
        return self.get_q_list()[self.irrk_ind]
