"""Graph helpers (reference: openjij/utils/graph_utils.py)."""
from __future__ import annotations

import numpy as np


def qubo_to_ising(mat: np.ndarray):
    """In place: a QUBO matrix to its Ising form (divide by 4, then add each
    row's sum to its diagonal), as openjij/utils/graph_utils.py:5-13."""
    mat /= 4
    for i in range(mat.shape[0]):
        mat[i, i] += np.sum(mat[i, :])


def chimera_to_ind(r: int, c: int, z: int, L: int):
    """1-D index r*8L + c*8 + z of Chimera site (r, c, z) on an L x L grid of
    unit cells; ValueError outside the grid (graph_utils.py:16-36)."""
    if not (0 <= r < L and 0 <= c < L and 0 <= z < 8):
        raise ValueError("0 <= r < L or 0 <= c < L or 0 <= z < 8. "
                         "your input r={}, c={}, z={}, L={}".format(r, c, z, L))
    return r * L * 8 + c * 8 + z
