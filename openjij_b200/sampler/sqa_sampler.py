"""Simulated quantum annealing sampler (reference: openjij/sampler/sqa_sampler.py).

Discrete-time path-integral Monte Carlo with ``trotter`` slices,
H(s) = s H_p + Gamma (1 - s) sum_i sigma_i^x, same parameters and schedules as
the reference's ``SQASampler``; all reads anneal together on the GPU.  The
returned sample of each read is its lowest-energy Trotter slice
(include/openjij/result/get_solution.hpp:59-84).
"""
from __future__ import annotations

from typing import Optional, Union

import numpy as np

import openjij_b200.cxxjij as cxxjij
from openjij_b200.sampler.sampler import BaseSampler, _as_bqm, _ising_graph, _place, spins_from_initial_state


class SQASampler(BaseSampler):
    """Sampler with simulated quantum annealing."""

    @property
    def parameters(self):
        return {"beta": ["parameters"], "gamma": ["parameters"], "trotter": ["parameters"]}

    def __init__(self):
        self._default_params = {
            "beta": 5.0,
            "gamma": 1.0,
            "num_sweeps": 1000,
            "schedule": None,
            "trotter": 4,
            "num_reads": 1,
        }
        self._params = self._default_params.copy()
        self._make_system = {"singlespinflip": cxxjij.system.make_transverse_ising}
        self._algorithm = {"singlespinflip": cxxjij.algorithm.Algorithm_SingleSpinFlip_run}
        self.schedule_info = {}

    def _convert_validation_schedule(self, schedule, beta):
        """(sqa_sampler.py:86-126) [(s, mcs)] with fixed beta or [(s, beta, mcs)]."""
        if not isinstance(schedule, (list, np.ndarray)):
            raise ValueError("schedule should be list or numpy.array")
        if isinstance(schedule[0], cxxjij.utility.TransverseFieldSchedule):
            return list(schedule)
        sch = np.array(schedule).T[0]
        if not np.all((0 <= sch) & (sch <= 1)):
            raise ValueError("schedule range is '0 <= s <= 1'.")
        out = []
        if len(schedule[0]) == 2:
            for s, mcs in schedule:
                e = cxxjij.utility.TransverseFieldSchedule()
                e.one_mc_step = int(mcs)
                e.updater_parameter.beta = float(beta)
                e.updater_parameter.s = float(s)
                out.append(e)
            return out
        if len(schedule[0]) == 3:
            for s, b, mcs in schedule:
                e = cxxjij.utility.TransverseFieldSchedule()
                e.one_mc_step = int(mcs)
                e.updater_parameter.beta = float(b)
                e.updater_parameter.s = float(s)
                out.append(e)
            return out
        raise ValueError("schedule is list of tuple or list (annealing parameter s : float, "
                         "step_length : int) or (annealing parameter s : float, beta: float, "
                         "step_length : int)")

    def _get_result(self, system, model, sites=None):
        e = np.asarray(system.energies(), dtype=np.float64)  # [R][T] classical energies
        R, T = e.shape
        best = np.argmin(e, axis=1)  # first slice of minimum energy
        q_state = system._spins_int8()  # [R][T][n]
        if sites is not None:
            q_state = np.ascontiguousarray(q_state[:, :, sites])
        states = q_state[np.arange(R), best]
        info = {"trotter_state": q_state, "trotter_energies": e}
        return states, e[np.arange(R), best], info

    def sample(
        self,
        bqm,
        beta: Optional[float] = None,
        gamma: Optional[float] = None,
        num_sweeps: Optional[int] = None,
        schedule: Optional[list] = None,
        trotter: Optional[int] = None,
        num_reads: Optional[int] = None,
        initial_state: Optional[Union[list, dict]] = None,
        updater: Optional[str] = None,
        sparse: Optional[bool] = None,
        reinitialize_state: Optional[bool] = None,
        seed: Optional[int] = None,
    ):
        if sparse is None:
            sparse = True
        if reinitialize_state is None:
            reinitialize_state = True
        if updater is None:
            updater = "single spin flip"
        name = updater.lower().replace("_", "").replace(" ", "")
        if name not in self._algorithm:
            raise ValueError('updater is one of "single spin flip"')
        model = _as_bqm(bqm, bool(sparse))
        ising_graph, offset, sites = _ising_graph(model)
        self._set_params(beta=beta, gamma=gamma, num_sweeps=num_sweeps, num_reads=num_reads,
                         trotter=trotter, schedule=schedule)
        p = self._params
        if p["schedule"]:
            p["schedule"] = self._convert_validation_schedule(p["schedule"], p["beta"])
            self.schedule_info = {"schedule": "custom schedule"}
        else:
            p["schedule"], bg = quartic_ising_schedule(model, p["beta"], p["gamma"], p["num_sweeps"])
            self.schedule_info = {"beta": bg[0], "gamma": bg[1], "num_sweeps": p["num_sweeps"]}
        n = ising_graph.size()
        T = int(p["trotter"])
        if initial_state is None:
            def init_generator(R):
                if seed is not None:  # every slice of every read from gen_spin(seed) (sqa_sampler.py:228-236)
                    one = np.asarray(ising_graph.gen_spin(int(seed)), np.int8)
                    return np.broadcast_to(one, (R, T, n))
                rng = np.random.default_rng()
                return rng.choice(np.array([-1, 1], np.int8), size=(R, T, n))
        else:
            s0 = _place(spins_from_initial_state(initial_state, model, len(model.variables)), sites, n)

            def init_generator(R):
                return np.broadcast_to(s0, (R, T, len(s0)))

        system = (self._make_system[name](init_generator(1), ising_graph, float(p["gamma"]))
                  if n > 0 else None)
        response = self._cxxjij_sampling(model, init_generator, self._algorithm[name], system,
                                         reinitialize_state, seed, offset, sites)
        response.info["schedule"] = self.schedule_info
        return response


def linear_ising_schedule(model, beta, gamma, num_sweeps):
    """s linear in [0, 1] (sqa_sampler.py:307-321)."""
    schedule = cxxjij.utility.make_transverse_field_schedule_list(beta=beta, one_mc_step=1,
                                                                  num_call_updater=num_sweeps)
    return schedule, [beta, gamma]


def quartic_ising_schedule(model, beta, gamma, num_sweeps):
    """s_k = f(k/(S-1)), f(s) = s^4 (35 - 84 s + 70 s^2 - 20 s^3) (Morita and
    Nishimori, J. Math. Phys. 49, 125210 (2008); sqa_sampler.py:327-344)."""
    s = np.linspace(0, 1, num_sweeps)
    fs = s**4 * (35 - 84 * s + 70 * s**2 - 20 * s**3)
    schedule = [((beta, float(e)), 1) for e in fs]
    return schedule, [beta, gamma]
