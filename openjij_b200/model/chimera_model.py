"""Chimera-graph model (reference: openjij/model/chimera_model.py).

A BinaryQuadraticModel whose variables sit on an L x L grid of Chimera unit
cells, labelled either by the 1-D index i = 8 L r + 8 c + z or by the
coordinate (r, c, z).  ``validate_chimera`` checks that every coupling is a
Chimera edge; ``get_cxxjij_ising_graph`` returns the ``cxxjij.graph.Chimera``
of the Ising form, which the samplers anneal on the GPU's colour-class kernels
(a Chimera graph is bipartite: two colour classes).

Unit cell (column representation): sites 0-3 couple to 4-7 of the same cell;
sites 0-3 also to the same site of the cells above and below, sites 4-7 to the
same site of the cells left and right.
"""
from __future__ import annotations

import openjij_b200.cxxjij as cj
from openjij_b200.model.model import BinaryQuadraticModel
from openjij_b200.variable_type import SPIN

_LEFT = (0, 1, 2, 3)
_RIGHT = (4, 5, 6, 7)


def make_ChimeraModel(linear, quadratic):
    """ChimeraModel class factory (chimera_model.py:7-286)."""

    class ChimeraModel(BinaryQuadraticModel):
        """BQM on a Chimera graph of unit_num_L x unit_num_L cells."""

        def __init__(self, linear: dict = None, quadratic: dict = None, offset: float = 0.0, vartype=SPIN,
                     unit_num_L: int = 2, model=None, sparse: bool = True):
            if model is not None:
                super().__init__(dict(model.linear), dict(model.quadratic), model.offset, model.vartype,
                                 sparse=True)
            else:
                super().__init__(dict(linear or {}), dict(quadratic or {}), offset, vartype, sparse=True)
            if not unit_num_L:
                raise ValueError("Input unit_num_L which is the length of the side of the two-dimensional grid "
                                 "where chimera unit cells are arranged.")
            self.unit_num_L = unit_num_L
            self.coordinate = self._validate_indices(self.indices)
            if self.coordinate == "index":
                self._chimera_index = lambda i, L: self.chimera_coordinate(i, L)
            else:
                self._chimera_index = lambda i, L: tuple(i)
            self._to_index = lambda r, c, z, L: self.to_index(r, c, z, L)

        def _validate_indices(self, indices):
            if indices and isinstance(indices[0], int):
                return "index"
            if indices and isinstance(indices[0], (tuple, list)) and len(indices[0]) == len(indices[-1]) == 3:
                return "chimera coordinate"
            raise ValueError("In the chimera graph, index should be int or tuple or list.")

        def _site(self, v):
            """1-D Chimera index of variable v."""
            return v if isinstance(v, int) else self.to_index(*v, self.unit_num_L)

        def validate_chimera(self):
            """Every coupling must join a site to one of its Chimera neighbours
            (chimera_model.py:92-157); raises ValueError otherwise."""
            L = self.unit_num_L
            for (i, j) in self.quadratic:
                r, c, z = self._chimera_index(i, L)
                if z >= 4:
                    nbrs = [self._to_index(r, c + d, z, L) for d in (-1, 1) if 0 <= c + d < L]
                    nbrs += [self._to_index(r, c, k, L) for k in _LEFT]
                else:
                    nbrs = [self._to_index(r + d, c, z, L) for d in (-1, 1) if 0 <= r + d < L]
                    nbrs += [self._to_index(r, c, k, L) for k in _RIGHT]
                if self._site(j) not in nbrs:
                    raise ValueError("Problem graph incompatible with chimera graph.\n"
                                     f"The connectable nodes of {i} are {nbrs}, not {j}.")
            return True

        def to_index(self, r, c, i, unit_num_L):
            """1-D index 8 L r + 8 c + i of Chimera coordinate (r, c, i)."""
            return 8 * unit_num_L * r + 8 * c + i

        def chimera_coordinate(self, i, unit_num_L):
            """(r, c, z) of 1-D index i."""
            z = i % 8
            c = (i % (8 * unit_num_L) - z) // 8
            r = (i - 8 * c - z) // (8 * unit_num_L)
            return int(r), int(c), int(z)

        def _validate(self, rcz1, rcz2, L):
            r1, c1, z1 = rcz1
            r2, c2, z2 = rcz2
            if r1 == r2 and c1 == c2:
                return (z1 in _LEFT and z2 in _RIGHT) or (z2 in _LEFT and z1 in _RIGHT)
            return (c1 == c2 and abs(r1 - r2) == 1) or (r1 == r2 and abs(c1 - c2) == 1)

        def _index_validate(self, i, L):
            if isinstance(i, tuple):
                return i[0] < self.unit_num_L and i[1] < self.unit_num_L and i[2] < 8
            return 0 <= i < 8 * L * L

        def get_cxxjij_ising_graph(self):
            """``cxxjij.graph.Chimera`` of the Ising form (chimera_model.py:185-243);
            the Ising offset is ``to_ising()[2]``."""
            L = self.unit_num_L
            if not self.validate_chimera():
                raise ValueError("Problem graph incompatible with chimera graph.")
            h, J, _ = self.to_ising()
            chimera = cj.graph.Chimera(L, L)
            for i, hi in h.items():
                if not self._index_validate(i, L):
                    raise ValueError(f"Problem graph incompatible with chimera graph. Node {i}.")
                chimera[self._chimera_index(i, L)] = hi
            in_cell = (cj.graph.ChimeraDir.IN_0or4, cj.graph.ChimeraDir.IN_1or5,
                       cj.graph.ChimeraDir.IN_2or6, cj.graph.ChimeraDir.IN_3or7)
            for (i, j), Jij in J.items():
                ri, ci, zi = self._chimera_index(i, L)
                rj, cj_, zj = self._chimera_index(j, L)
                if not (self._index_validate(i, L) and self._index_validate(j, L)
                        and self._validate((ri, ci, zi), (rj, cj_, zj), L)):
                    raise ValueError("Problem graph incompatible with chimera graph.\n"
                                     f"In the {L}*{L} Chimera grid, there is no connection between node {i} "
                                     f"and node {j}.")
                if ri == rj and ci == cj_:
                    d = in_cell[zj % 4]
                elif ri - rj == -1:
                    d = cj.graph.ChimeraDir.PLUS_R
                elif ri - rj == 1:
                    d = cj.graph.ChimeraDir.MINUS_R
                elif ci - cj_ == -1:
                    d = cj.graph.ChimeraDir.PLUS_C
                else:
                    d = cj.graph.ChimeraDir.MINUS_C
                chimera[ri, ci, zi, d] = Jij
            return chimera

        def graph_sites(self):
            """Index in the Chimera graph of each variable, in variable order."""
            return [self._site(v) for v in self.variables]

    return ChimeraModel


def make_ChimeraModel_from_JSON(obj):
    label = obj["variable_labels"][0]
    if isinstance(label, list):
        label = tuple(label)
    return make_ChimeraModel({label: 1.0}, {})


def ChimeraModel(linear: dict = None, quadratic: dict = None, offset: float = 0.0, vartype=SPIN,
                 unit_num_L: int = 2, model=None):
    """ChimeraModel(linear, quadratic, offset, vartype, unit_num_L, model)
    (chimera_model.py:304-343)."""
    Model = make_ChimeraModel(linear, quadratic)
    return Model(linear, quadratic, offset, vartype, unit_num_L, model)


ChimeraModel.from_qubo = lambda Q, offset=0.0, **kwargs: make_ChimeraModel({}, Q).from_qubo(Q, offset, **kwargs)
ChimeraModel.from_ising = lambda linear, quadratic, offset=0.0, **kwargs: make_ChimeraModel(
    linear, quadratic).from_ising(linear, quadratic, offset, **kwargs)
