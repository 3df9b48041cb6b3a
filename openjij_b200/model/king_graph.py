"""King-graph model of Hitachi's CMOS annealer (the behaviour of the
reference's openjij/model/king_graph.py: KingGraph, make_KingGraph,
KingGraph.from_qubo / from_ising).

Every site of a 2-D grid couples to its eight king-move neighbours.  A site is
labelled either by its (x, y) pair or by the row-major index y * width + x.
Interactions are accepted as linear / quadratic dicts or as the annealing
cloud's list, one row [x1, y1, x2, y2, value] per coupling and
[x, y, x, y, value] per field.  The machine fixes the grid and the value range:

    ============  =========  ==========  ===========
    machine_type  width (x)  height (y)  |value| <=
    ============  =========  ==========  ===========
    "ASIC"        352        176         3
    "FPGA"        80         80          127
    ============  =========  ==========  ===========

Here the model is one BinaryQuadraticModel subclass.  Its Ising rows and their
checks are numpy arrays: coordinates of every variable at once, one
vectorised test for the whole list.  The samplers anneal it on the general
sparse path, whose colour classes cover the king graph with four colours.
"""
from __future__ import annotations

import numpy as np

from openjij_b200.model.model import BinaryQuadraticModel
from openjij_b200.variable_type import SPIN, cast_vartype

# machine -> (grid width, grid height, largest |value|)
_MACHINES = {"ASIC": (352, 176, 3), "FPGA": (80, 80, 127)}


def _site_xy(labels, width):
    """(x, y) integer arrays of site labels: (x, y) pairs as given, integer
    labels split as index = y * width + x."""
    xs = np.empty(len(labels), np.int64)
    ys = np.empty(len(labels), np.int64)
    for k, v in enumerate(labels):
        if isinstance(v, tuple):
            xs[k], ys[k] = v[0], v[1]
        else:
            ys[k] = int(v / width)
            xs[k] = int(v) - ys[k] * width
    return xs, ys


class KingGraphModel(BinaryQuadraticModel):
    """BQM on the king graph of the CMOS annealer, with the machine's ranges
    (``xrange``, ``yrange``, ``prange``) and the Ising form as the annealing
    cloud's interaction list (``get_ising_king_graph``)."""

    def __init__(self, linear: dict = None, quadratic: dict = None, offset: float = 0.0, king_graph=None,
                 vartype=SPIN, machine_type: str = "", sparse: bool = False):
        vartype = cast_vartype(vartype)
        if machine_type not in _MACHINES:
            raise ValueError("machine type should be ASIC or FPGA")
        width, height, pmax = _MACHINES[machine_type]
        self.machine_type = machine_type
        self.xrange, self.yrange, self.prange = [0, width], [0, height], [-pmax, pmax]
        rows = None
        if king_graph is not None:
            rows = [list(r) for r in king_graph]
            fields = {(r[0], r[1]): r[4] for r in rows if (r[0], r[1]) == (r[2], r[3])}
            couplings = {((r[0], r[1]), (r[2], r[3])): r[4] for r in rows if (r[0], r[1]) != (r[2], r[3])}
            linear, quadratic = fields, couplings
        super().__init__(dict(linear or {}), dict(quadratic or {}), offset, vartype, sparse=sparse)
        if rows is None or vartype != SPIN:
            rows = self._ising_rows()
        self._ising_king_graph = rows
        self._check_rows()

    def _ising_rows(self):
        """The Ising form as [x1, y1, x2, y2, value] rows: the non-zero fields
        in variable order, then the non-zero couplings in the model's order."""
        lin, qv, _ = self._converted_arrays(SPIN)
        xs, ys = _site_xy(self.variables, self.xrange[1])
        f = np.flatnonzero(lin != 0.0)
        c = np.flatnonzero(qv != 0.0)
        i, j = self._qi[c], self._qj[c]
        coords = np.concatenate([np.stack([xs[f], ys[f], xs[f], ys[f]], 1),
                                 np.stack([xs[i], ys[i], xs[j], ys[j]], 1)]).tolist()
        values = np.concatenate([lin[f], qv[c]]).tolist()
        return [xy + [v] for xy, v in zip(coords, values)]

    def _check_rows(self):
        """Every row inside the grid's height, between king neighbours (or a
        site with itself) and inside the machine's value range."""
        if not self._ising_king_graph:
            return
        a = np.asarray([r[:4] for r in self._ising_king_graph], np.int64).reshape(-1, 4)
        p = np.asarray([r[4] for r in self._ising_king_graph], np.float64)
        bad = ((a[:, 1] >= self.yrange[1]) | (a[:, 3] >= self.yrange[1]) |
               (np.abs(a[:, 0] - a[:, 2]) > 1) | (np.abs(a[:, 1] - a[:, 3]) > 1) |
               (p < self.prange[0]) | (p > self.prange[1]))
        if np.any(bad):
            xi, yi, xj, yj, v = self._ising_king_graph[int(np.argmax(bad))]
            raise ValueError(f"Graph is incomplete xi: {xi}, yi: {yi}, xj: {xj}, yj: {yj}, p: {v}")

    def get_ising_king_graph(self):
        return self._ising_king_graph

    def king_indices(self):
        """The variables as (x, y) pairs."""
        if self.variables and isinstance(self.variables[0], tuple):
            return self.variables
        xs, ys = _site_xy(self.variables, self.xrange[1])
        return list(zip(xs.tolist(), ys.tolist()))

    def convert_to_index(self, x, y):
        """Row-major index y * width + x of site (x, y)."""
        return y * self.xrange[1] + x


def make_KingGraph(linear=None, quadratic=None, king_graph=None):
    """The reference's class factory: one class serves every model here."""
    return KingGraphModel


def make_KingGraph_from_JSON(obj):
    return KingGraphModel


def KingGraph(linear=None, quadratic=None, offset=0.0, king_graph=None, vartype=SPIN, machine_type=""):
    """A king-graph model from dicts or from the annealing cloud's list::

        KingGraph(machine_type="ASIC", quadratic={(0, 1): -1.0, (1, 2): -3.0})
        KingGraph(machine_type="ASIC", king_graph=[[0, 0, 1, 0, -1.0], [1, 0, 2, 0, -3.0]])
    """
    return KingGraphModel(linear, quadratic, offset, king_graph, vartype, machine_type)


def _king_from_qubo(Q, offset=0.0, **kwargs):
    return KingGraphModel.from_qubo(Q, offset, **kwargs)


def _king_from_ising(linear, quadratic, offset=0.0, **kwargs):
    return KingGraphModel.from_ising(linear, quadratic, offset, **kwargs)


KingGraph.from_qubo = _king_from_qubo
KingGraph.from_ising = _king_from_ising
