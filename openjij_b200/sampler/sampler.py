"""Base sampler (reference: openjij/sampler/sampler.py).

The reference runs ``num_reads`` reads one after another from Python
(sampler.py:116-140), each a separate C++ call.  Here all reads are replicas of
one ``cxxjij`` system and anneal together in one GPU call; per-read energies
come back from the GPU's FP64 energy kernel.  With ``reinitialize_state=False``
(reverse annealing) each read continues from the previous read's final state,
as in the reference, so those reads run one after another.
"""
from __future__ import annotations

import time

import numpy as np

import openjij_b200.cxxjij as cxxjij
from openjij_b200.model.model import BinaryQuadraticModel
from openjij_b200.sampler.response import Response
from openjij_b200.variable_type import BINARY, SPIN


def measure_time(func):
    """Decorator returning the wall time of ``func`` in seconds (sampler.py:30-46)."""

    def wrapper(*args, **kwargs):
        t0 = time.perf_counter()
        func(*args, **kwargs)
        return time.perf_counter() - t0

    return wrapper


def _as_bqm(bqm, sparse):
    if isinstance(bqm, BinaryQuadraticModel):
        if sparse != bqm.sparse:
            out = bqm.copy()
            out.sparse = sparse
            return out
        return bqm
    # any dimod-like model: linear / quadratic / offset / vartype
    return BinaryQuadraticModel(dict(bqm.linear), dict(bqm.quadratic), bqm.offset,
                                str(getattr(bqm.vartype, "name", bqm.vartype)), sparse=sparse)


def _ising_graph(model):
    """(cxxjij graph, Ising offset, sites) of a model.  A lattice model
    (ChimeraModel) returns its full lattice graph alone; ``sites`` then gives
    the lattice index of each of its variables, in variable order (None when
    graph and variables coincide)."""
    out = model.get_cxxjij_ising_graph()
    if isinstance(out, tuple):
        graph, offset = out
    else:
        graph, offset = out, model.to_ising()[2]
    sites = None
    if hasattr(model, "graph_sites") and graph.size() != len(model.variables):
        sites = np.asarray(model.graph_sites(), np.int64)
    return graph, offset, sites


def _place(s0, sites, n):
    """A state over the model's variables placed on the n lattice sites (+1 elsewhere)."""
    if sites is None:
        return s0
    full = np.ones(n, np.int8)
    full[sites] = s0
    return full


class BaseSampler:
    """Parameter handling and the batched read loop shared by SA and SQA."""

    parameters: dict = {}
    properties: dict = {}

    def _set_params(self, **kwargs):
        for key, value in kwargs.items():
            if key not in self._default_params:
                raise ValueError("Unknown parameters detected")
            self._params[key] = self._default_params[key] if value is None else value

    def _cxxjij_sampling(self, model, init_generator, algorithm, system, reinitialize_state=True,
                         seed=None, offset=0.0, sites=None):
        """Anneals ``num_reads`` replicas of ``system`` and builds the Response.

        ``init_generator(R)`` returns an [R][n] (SA) or [R][T][n] (SQA) array.
        """
        num_reads = int(self._params["num_reads"])
        schedule = self._params["schedule"]
        n = len(model.variables)

        def run(sys):
            if seed is None:
                algorithm(sys, schedule)
            else:
                algorithm(sys, int(seed), schedule)

        exec_times = []
        t0 = time.perf_counter()
        sys_info = {}
        if n == 0:
            states = np.zeros((num_reads, 0), dtype=np.int8)
            energies = np.full(num_reads, float(offset))
        elif reinitialize_state:
            system.reset_spins(init_generator(num_reads))
            dt = measure_time(run)(system)
            exec_times = [dt / num_reads] * num_reads
            states, energies, sys_info = self._get_result(system, model, sites)
            energies = energies + offset
        else:
            rows, ens, infos = [], [], []
            for _ in range(num_reads):
                exec_times.append(measure_time(run)(system))
                st, en, inf = self._get_result(system, model, sites)
                rows.append(st[0])
                ens.append(en[0])
                infos.append(inf)
            states = np.asarray(rows)
            energies = np.asarray(ens) + offset
            if infos and infos[0]:
                sys_info = {k: np.concatenate([i[k] for i in infos]) for k in infos[0]}
        sampling_time = time.perf_counter() - t0

        if model.vartype == BINARY:
            states = (states + 1) // 2
        info = {"system": sys_info} if sys_info else {}
        response = Response(np.asarray(states, dtype=np.int8), energies, model.variables, model.vartype, info)
        response.info["sampling_time"] = sampling_time * 1e6
        response.info["execution_time"] = (float(np.mean(exec_times)) * 1e6) if exec_times else 0.0
        response.info["list_exec_times"] = np.asarray(exec_times) * 1e6
        run_info = cxxjij.last_run_info()
        response.info["run"] = run_info
        # per call: accepted single-spin flips, and for the dense kernels the
        # largest deviation of the incremental FP32 fields from the exact fields
        # of the same spins (-1 where not measured)
        response.info["accepted_flips"] = run_info.get("accepted", -1.0)
        response.info["field_drift"] = run_info.get("field_drift", -1.0)
        return response

    def _get_result(self, system, model, sites=None):
        """(spins [R][n] in +-1, Ising energies [R], extra info)."""
        sol = system._spins_int8()  # get_solution of a classical system: the spins (dummy spin +1)
        energies = np.asarray(system.energies(), dtype=np.float64).reshape(-1)
        return (sol if sites is None else sol[:, sites]), energies, {}

    # ---- dimod-style entry points (sampler.py:166-248) ---------------------
    def sample(self, bqm, **parameters):  # overridden by the samplers
        raise NotImplementedError

    def sample_ising(self, h, J, **parameters):
        sparse = parameters.pop("sparse", True)
        bqm = BinaryQuadraticModel.from_ising(h, J, sparse=sparse)
        return self.sample(bqm, sparse=sparse, **parameters)

    def sample_qubo(self, Q, **parameters):
        if isinstance(Q, dict):
            sparse = parameters.pop("sparse", True)
            bqm = BinaryQuadraticModel.from_qubo(Q, sparse=sparse)
            return self.sample(bqm, sparse=sparse, **parameters)
        if isinstance(Q, np.ndarray):
            sparse = parameters.pop("sparse", False)
            bqm = BinaryQuadraticModel.from_numpy_matrix(Q, vartype="BINARY", sparse=sparse)
            return self.sample(bqm, sparse=sparse, **parameters)
        raise TypeError("Q must be either dict or np.ndarray")


def spins_from_initial_state(initial_state, model, n):
    """Validates a user initial state (sa_sampler.py:260-305) -> +-1 array [n]."""
    vals = []
    if isinstance(initial_state, dict):
        seq = [initial_state[k] for k in model.variables]
    elif isinstance(initial_state, (list, tuple, np.ndarray)):
        seq = [initial_state[k] for k in range(len(model.variables))]
    else:
        raise RuntimeError("Unsupported type of initial_state.")
    for v in seq:
        if model.vartype == BINARY:
            if v != 0 and v != 1:
                raise RuntimeError("The initial variables must be 0 or 1.")
            vals.append(2 * v - 1)
        elif model.vartype == SPIN:
            if v != -1 and v != 1:
                raise RuntimeError("The initial variables must be -1 or +1.")
            vals.append(v)
    if len(initial_state) != n:
        raise ValueError(f"the size of the initial state should be {n}")
    return np.asarray(vals, dtype=np.int8)
