"""King-graph model of the CMOS annealer (reference: openjij/model/king_graph.py).

A BinaryQuadraticModel on a 2-D grid where every site couples to its eight
neighbours (king moves).  Interactions come as dicts or in the annealing
cloud's list form: [x1, y1, x2, y2, value] for a coupling and
[x, y, x, y, value] for a field.  The hardware limits (grid size and the range
of the values) depend on ``machine_type``: "ASIC" (352 x 176, |p| <= 3) or
"FPGA" (80 x 80, |p| <= 127).  The samplers anneal it through the general
sparse path, whose colour classes cover the king graph with four colours.
"""
from __future__ import annotations

from openjij_b200.model.model import BinaryQuadraticModel
from openjij_b200.variable_type import SPIN, cast_vartype

_RANGES = {"ASIC": ([0, 352], [0, 176], [-3, 3]), "FPGA": ([0, 80], [0, 80], [-127, 127])}


def make_KingGraph(linear=None, quadratic=None, king_graph=None):
    """KingGraph class factory (king_graph.py:23-170)."""

    class KingGraph(BinaryQuadraticModel):
        """BQM on the king graph of the CMOS annealer."""

        def __init__(self, linear: dict = None, quadratic: dict = None, offset: float = 0.0, king_graph=None,
                     vartype=SPIN, machine_type: str = "", sparse: bool = False):
            vartype = cast_vartype(vartype)
            self.machine_type = machine_type
            if machine_type not in _RANGES:
                raise ValueError("machine type should be ASIC or FPGA")
            self.xrange, self.yrange, self.prange = (list(r) for r in _RANGES[machine_type])
            if king_graph is not None:
                linear, quadratic = self._convert_to_BQM_format(king_graph)
            super().__init__(dict(linear or {}), dict(quadratic or {}), offset, vartype, sparse=sparse)
            if king_graph is not None and vartype == SPIN:
                self._ising_king_graph = [list(e) for e in king_graph]
            else:
                lin, quad, _ = self.to_ising()
                self._ising_king_graph = []
                for v, h in lin.items():
                    if h != 0:
                        x, y = self._convert_to_xy(v)
                        self._ising_king_graph.append([x, y, x, y, h])
                for (u, v), J in quad.items():
                    if J != 0:
                        x1, y1 = self._convert_to_xy(u)
                        x2, y2 = self._convert_to_xy(v)
                        self._ising_king_graph.append([x1, y1, x2, y2, J])
            self._validation_ising_king_graph()

        @staticmethod
        def _convert_to_BQM_format(king_graph):
            linear, quad = {}, {}
            for x1, y1, x2, y2, value in king_graph:
                if (x1, y1) == (x2, y2):
                    linear[(x1, y1)] = value
                else:
                    quad[(x1, y1), (x2, y2)] = value
            return linear, quad

        def get_ising_king_graph(self):
            return self._ising_king_graph

        def king_indices(self):
            if isinstance(self.indices[0], tuple):
                return self.indices
            return [self._convert_to_xy(i) for i in self.indices]

        def _convert_to_xy(self, index):
            if isinstance(index, tuple):
                return index[0], index[1]
            y = int(index / self.xrange[1])
            return int(index - y * self.xrange[1]), y

        def convert_to_index(self, x, y):
            return y * self.xrange[1] + x

        def _validation_ising_king_graph(self):
            """Sites inside the grid, couplings between king neighbours, values
            inside the machine's range (king_graph.py:150-170)."""
            for xi, yi, xj, yj, p in self._ising_king_graph:
                msg = f"Graph is incomplete xi: {xi}, yi: {yi}, xj: {xj}, yj: {yj}, p: {p}"
                if yi >= self.yrange[1] or yj >= self.yrange[1]:
                    raise ValueError(msg)
                if abs(xi - xj) > 1 or abs(yi - yj) > 1:
                    raise ValueError(msg)
                if not (self.prange[0] <= p <= self.prange[1]):
                    raise ValueError(msg)

        def energy(self, sample, **kwargs):
            return super().energy(sample)

        def energies(self, samples_like, **kwargs):
            return super().energies(samples_like)

    return KingGraph


def make_KingGraph_from_JSON(obj):
    label = obj["variable_labels"][0]
    if isinstance(label, list):
        label = tuple(label)
    return make_KingGraph({label: 1.0}, {})


def KingGraph(linear=None, quadratic=None, offset=0.0, king_graph=None, vartype=SPIN, machine_type=""):
    """KingGraph(linear, quadratic, offset, king_graph, vartype, machine_type)
    (king_graph.py:193-236)::

        KingGraph(machine_type="ASIC", linear={}, quadratic={(0, 1): -1.0, (1, 2): -3.0})
        KingGraph(machine_type="ASIC", king_graph=[[0, 0, 1, 0, -1.0], [1, 0, 2, 0, -3.0]])
    """
    Model = make_KingGraph(linear, quadratic, king_graph)
    return Model(linear, quadratic, offset, king_graph, vartype, machine_type)


KingGraph.from_qubo = lambda Q, offset=0.0, **kwargs: make_KingGraph({}, Q).from_qubo(Q, offset, **kwargs)
KingGraph.from_ising = lambda linear, quadratic, offset=0.0, **kwargs: make_KingGraph(
    linear, quadratic).from_ising(linear, quadratic, offset, **kwargs)
