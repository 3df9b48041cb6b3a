"""Graph helpers with the behaviour of the reference's openjij/utils/graph_utils.py."""
from __future__ import annotations

import numpy as np


def qubo_to_ising(mat: np.ndarray):
    """Turns a QUBO matrix into its Ising form in place: every entry divided by
    4, then every diagonal entry increased by the sum of its (divided) row.
    The row sums do not involve other rows' diagonals, so all of them are taken
    before the diagonal changes."""
    mat /= 4
    mat[np.diag_indices_from(mat)] += mat.sum(axis=1)


def chimera_to_ind(r: int, c: int, z: int, L: int):
    """Linear index of site z (0..7) of the Chimera unit cell in row r,
    column c of an L x L grid: cells in row-major order, 8 sites each.
    Raises ValueError for a site outside the grid."""
    try:
        return int(np.ravel_multi_index((r, c, z), (L, L, 8)))
    except ValueError:
        raise ValueError(f"Chimera site (r={r}, c={c}, z={z}) is outside an L={L} grid "
                         f"(0 <= r < L, 0 <= c < L, 0 <= z < 8)") from None
