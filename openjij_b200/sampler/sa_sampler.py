"""Simulated annealing sampler (reference: openjij/sampler/sa_sampler.py:42-329).

Same parameters, defaults and schedule construction as the reference's
``SASampler``; the reads anneal together on the GPU.  Differences, by design:

* reads are replicas with their own counter-based random streams, so with a
  ``seed`` the reads start from the same initial state (as in the reference,
  sa_sampler.py:253-258) but no longer repeat each other;
* ``updater`` "swendsen wang" runs the GPU Swendsen-Wang kernel (oj_sw_run);
  like the reference it always uses the sparse graph.
"""
from __future__ import annotations

import time
from typing import Optional, Union

import numpy as np

import openjij_b200.cxxjij as cxxjij
from openjij_b200.model.model import BinaryQuadraticModel
from openjij_b200.sampler.response import Response
from openjij_b200.sampler.sampler import BaseSampler, _as_bqm, _ising_graph, _place, spins_from_initial_state
from openjij_b200.variable_type import BINARY


class SASampler(BaseSampler):
    """Sampler with simulated annealing (single spin flip Metropolis)."""

    @property
    def parameters(self):
        return {"beta_min": ["parameters"], "beta_max": ["parameters"]}

    def __init__(self):
        self._default_params = {
            "beta_min": None,
            "beta_max": None,
            "num_sweeps": 1000,
            "schedule": None,
            "num_reads": 1,
        }
        self._params = self._default_params.copy()
        self._make_system = {"singlespinflip": cxxjij.system.make_classical_ising,
                             "swendsenwang": cxxjij.system.make_classical_ising}
        self._algorithm = {"singlespinflip": cxxjij.algorithm.Algorithm_SingleSpinFlip_run,
                           "swendsenwang": cxxjij.algorithm.Algorithm_SwendsenWang_run}
        self.schedule_info = {}

    def _convert_validation_schedule(self, schedule):
        """(sa_sampler.py:109-135) list of (beta, one_mc_step) -> ClassicalSchedule list."""
        if not isinstance(schedule, (list, np.ndarray)):
            raise ValueError("schedule should be list or numpy.array")
        if isinstance(schedule[0], cxxjij.utility.ClassicalSchedule):
            return list(schedule)
        if len(schedule[0]) != 2:
            raise ValueError("schedule is list of tuple or list (beta : float, step_length : int)")
        beta = np.array(schedule).T[0]
        if not np.all(0 <= beta):
            raise ValueError("schedule beta range is '0 <= beta'.")
        out = []
        for b, step in schedule:
            s = cxxjij.utility.ClassicalSchedule()
            s.one_mc_step = int(step)
            s.updater_parameter.beta = float(b)
            out.append(s)
        return out

    def sample(
        self,
        bqm: Union[BinaryQuadraticModel, object],
        beta_min: Optional[float] = None,
        beta_max: Optional[float] = None,
        num_sweeps: Optional[int] = None,
        num_reads: Optional[int] = None,
        schedule: Optional[list] = None,
        initial_state: Optional[Union[list, dict]] = None,
        updater: Optional[str] = None,
        sparse: Optional[bool] = None,
        reinitialize_state: Optional[bool] = None,
        seed: Optional[int] = None,
    ):
        if updater is None:
            updater = "single spin flip"
        if sparse is None:
            sparse = True
        if reinitialize_state is None:
            reinitialize_state = True
        name = updater.lower().replace("_", "").replace(" ", "")
        if name not in self._make_system:
            raise ValueError('updater is one of "single spin flip or swendsen wang"')
        if name == "swendsenwang":  # runs on sparse graphs only (sa_sampler.py:195-197)
            sparse = True
        model = _as_bqm(bqm, bool(sparse))
        ising_graph, offset, sites = _ising_graph(model)
        self._set_params(beta_min=beta_min, beta_max=beta_max, num_sweeps=num_sweeps,
                         num_reads=num_reads, schedule=schedule)
        if self._params["schedule"] is None:
            self._params["schedule"], beta_range = geometric_ising_beta_schedule(
                cxxgraph=ising_graph, beta_max=self._params["beta_max"],
                beta_min=self._params["beta_min"], num_sweeps=self._params["num_sweeps"], seed=seed)
            self.schedule_info = {"beta_max": beta_range[0], "beta_min": beta_range[1],
                                  "num_sweeps": self._params["num_sweeps"]}
        else:
            self._params["schedule"] = self._convert_validation_schedule(self._params["schedule"])
            self.schedule_info = {"schedule": "custom schedule"}

        n = ising_graph.size()
        if initial_state is None:
            def init_generator(R):
                if seed is not None:  # every read starts from gen_spin(seed) (sa_sampler.py:253-258)
                    return np.broadcast_to(np.asarray(ising_graph.gen_spin(int(seed)), np.int8), (R, n))
                rng = np.random.default_rng()
                return rng.choice(np.array([-1, 1], np.int8), size=(R, n))
        else:
            s0 = _place(spins_from_initial_state(initial_state, model, len(model.variables)), sites, n)

            def init_generator(R):
                return np.broadcast_to(s0, (R, len(s0)))

        algorithm = self._algorithm[name]
        system = self._make_system[name](init_generator(1), ising_graph) if n > 0 else None
        response = self._cxxjij_sampling(model, init_generator, algorithm, system, reinitialize_state,
                                         seed, offset, sites)
        response.info["schedule"] = self.schedule_info
        return response


    def sample_batch(self, models, beta_min: Optional[float] = None, beta_max: Optional[float] = None,
                     num_sweeps: Optional[int] = None, num_reads: Optional[int] = None, seed: Optional[int] = None,
                     device: int = 0):
        """Anneals many dense models of uneven size in one GPU launch (an
        extension: the reference samples one model per ``sample`` call).

        ``models``: BinaryQuadraticModels (or dimod-like models, or QUBO dicts),
        each with at most 4096 variables.  All models share one geometric
        schedule; a missing end of the beta range is estimated per model as in
        ``sample`` and the widest range over the models is used.  Returns one
        Response per model, in order.
        """
        from openjij_b200 import _native as N
        self._set_params(beta_min=beta_min, beta_max=beta_max, num_sweeps=num_sweeps, num_reads=num_reads)
        R = int(self._params["num_reads"])
        S = int(self._params["num_sweeps"])
        bqms, mats, offsets = [], [], []
        for mdl in models:
            b = BinaryQuadraticModel.from_qubo(mdl) if isinstance(mdl, dict) else _as_bqm(mdl, False)
            graph, off = b.get_cxxjij_ising_graph()
            bqms.append(b)
            mats.append(np.ascontiguousarray(graph.get_interactions(), np.float64))
            offsets.append(off)
        ctx = _batch_context(device)
        batch = N.Batch(ctx, mats)
        bmin, bmax = self._params["beta_min"], self._params["beta_max"]
        if bmin is None or bmax is None:
            # each model's random configurations as its own sample() call would
            # draw them, then the statistics of all models in one GPU call
            draws = []
            for a in mats:
                if seed is not None:
                    np.random.seed(seed)
                draws.append(_flip_spins(a.shape[0]))
            quad, lin, amin = batch.flip_stats(np.concatenate(draws) if draws else np.zeros((0, 2), np.int8),
                                               _THRESHOLD)
            lo, hi, pos = [], [], 0
            for k, a in enumerate(mats):
                nk = a.shape[0] - 1
                b1, b0 = _beta_range(quad[pos:pos + nk], lin[pos:pos + nk], amin[k], a.shape[0], S, bmin, bmax)
                pos += nk
                lo.append(b0)
                hi.append(b1)
            bmin = min(lo) if bmin is None else bmin
            bmax = max(hi) if bmax is None else bmax
        m = max(1, S // 1000)
        count = S // m
        betas = cxxjij.utility.make_classical_schedule_list(float(bmin), float(bmax), m, count)
        beta_arr = np.array([e.updater_parameter.beta for e in betas], np.float64)
        mcs = np.array([e.one_mc_step for e in betas], np.int32)
        sizes = [a.shape[0] - 1 for a in mats]
        rng = np.random.default_rng(seed)
        spins = rng.choice(np.array([-1, 1], np.int8), size=int(R * sum(sizes)))
        reads = np.full(len(mats), R, np.int32)
        energies = np.zeros(R * len(mats))
        t0 = time.perf_counter()
        st = N.sa_run_batched(batch, reads, spins, beta_arr, mcs,
                              seed=(rng.integers(0, 2 ** 63) if seed is None else int(seed)), energies=energies)
        elapsed = time.perf_counter() - t0
        out, off = [], 0
        for k, b in enumerate(bqms):
            n = sizes[k]
            st_k = spins[off: off + R * n].reshape(R, n)
            off += R * n
            if b.vartype == BINARY:
                st_k = (st_k + 1) // 2
            resp = Response(np.asarray(st_k, dtype=np.int8), energies[k * R:(k + 1) * R] + offsets[k], b.variables, b.vartype)
            resp.info["schedule"] = {"beta_min": bmin, "beta_max": bmax, "num_sweeps": S}
            resp.info["sampling_time"] = elapsed * 1e6
            resp.info["run"] = st
            resp.info["accepted_flips"] = st["accepted"]  # over the whole batch call
            resp.info["field_drift"] = st["field_drift"]
            out.append(resp)
        return out


_BATCH_CTX = {}


def _batch_context(device):
    from openjij_b200 import _native as N
    if device not in _BATCH_CTX:
        _BATCH_CTX[device] = N.Context(device)
    return _BATCH_CTX[device]


def geometric_ising_beta_schedule(cxxgraph, beta_max=None, beta_min=None, num_sweeps=1000, seed=None):
    """Geometric beta schedule (reference: sa_sampler.py:853-976).

    With both ends given the schedule is make_classical_schedule_list(beta_min,
    beta_max, m, num_sweeps // m), m = max(1, num_sweeps // 1000).  A missing
    end is estimated from the energy changes of random spin configurations,
    by the reference's procedure (median / minimum positive dE, bisection for
    beta_min, the 1/1000 final acceptance target for beta_max).  The energy
    changes and the smallest coupling magnitude come from the GPU
    (``_flip_stats``, oj_graph_flip_stats) instead of a dense matrix product and
    a pass over the whole augmented matrix; the random configurations are the
    reference's own numpy draws.
    """
    if seed is not None:
        np.random.seed(seed)
    n = cxxgraph.size() + 1  # rows of the augmented matrix
    if beta_min is None or beta_max is None:
        spins = _flip_spins(n)
        quad, lin, int_min = cxxgraph._flip_stats(spins, _THRESHOLD)
        beta_max, beta_min = _beta_range(quad, lin, int_min, n, num_sweeps, beta_min, beta_max)
    per_beta = max(1, num_sweeps // 1000)
    schedule = cxxjij.utility.make_classical_schedule_list(
        beta_min=float(beta_min), beta_max=float(beta_max), one_mc_step=per_beta,
        num_call_updater=num_sweeps // per_beta)
    return schedule, [beta_max, beta_min]


_THRESHOLD = 1e-8


def _flip_spins(n_aug):
    """The reference's random configurations: np.random.choice([-1, 1],
    (n+1, 2)) with the dummy row set to 1, drawn only when n > 0
    (sa_sampler.py:886-888); returns the n spin rows as int8."""
    if n_aug <= 1:
        return np.zeros((0, 2), np.int8)
    spins = np.random.choice([-1, 1], size=(n_aug, 2))
    spins[-1, :] = 1
    return spins[:-1].astype(np.int8)


def _beta_range(quad, lin, int_min, n_aug, num_sweeps, beta_min, beta_max):
    """beta_max, beta_min from the flip statistics (sa_sampler.py:880-965):
    quad / lin the coupling and field parts of the single-flip energy changes
    of the random configurations, int_min the smallest |entry| > 1e-8 of the
    augmented matrix, n_aug = n + 1."""
    THRESHOLD = _THRESHOLD
    dE_max, dE_min, rate_dE = 1.0, 1.0, 0.5
    if n_aug > 1:
        quad_abs = np.abs(quad)
        if np.any(quad_abs > THRESHOLD):
            rate_dE = np.max(np.abs(lin[quad_abs > THRESHOLD]) /
                             (quad_abs[quad_abs > THRESHOLD].mean() + THRESHOLD))
        positive = quad[quad > THRESHOLD]
        if len(positive) == 0:
            dE_min, dE_max = 1.0, 1.1
        else:
            dE_max = np.median(positive, axis=0).mean()
            dE_min = np.min(positive, axis=0).mean()
    n = n_aug
    prob_init = 9 / 10 - 8 / 10 * np.tanh(rate_dE / 50) + THRESHOLD
    prob_final = 1 / 1000
    if beta_min is None:
        lo, hi = -np.log(prob_init) / dE_max, -np.log(prob_init) / dE_min
        for _ in range(5):
            b = (lo + hi) / 2
            f = 2 * b * prob_init - np.exp(-b * dE_min) + np.exp(-b * dE_max)
            if abs(f) < 1e-8:
                break
            if f > 0:
                hi = b
            else:
                lo = b
        beta_min = lo
        floor = beta_min * 0.8
        beta_min = floor + (beta_min * 1.5 - floor) * np.tanh(num_sweeps / n)
    if beta_max is None:
        if not np.isfinite(int_min):  # np.min of an empty selection in the reference
            raise ValueError("zero-size array to reduction operation minimum which has no identity")
        int_min = max(int_min, dE_min / 10.0)
        b_int = -np.log(prob_final) / int_min
        b_dE = -np.log(prob_final) / dE_min
        if rate_dE < 2:
            lo, hi = min(b_dE, b_int), max(b_dE, b_int)
            beta_max = lo + (hi - lo) * np.tanh(num_sweeps / (2 * n))
        else:
            last = min(100, num_sweeps // 10 + 1)
            beta_max = -np.log(prob_final) / max(dE_min, int_min) / last
        if beta_max < beta_min:
            beta_max = beta_min * 10.0
    if rate_dE > 1:
        beta_min *= rate_dE
        beta_max *= rate_dE
    return beta_max, beta_min
