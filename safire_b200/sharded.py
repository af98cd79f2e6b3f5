"""run_afqmc over walkers sharded across ranks, one engine per rank (one process per GPU).

Each rank's engine holds its share of the walkers (execute.cpp:135-140) and steps them with the
rank-local calls; what crosses ranks is what the reference reduces or exchanges over MPI:

  * population control: the global comb and walker exchange (safire_b200.popcontrol);
  * averagePseudoEnergy for the Eshift relaxation (average_energy.hpp:33-48): the sums
    sum w exp(dt eloc) and sum w all-reduced, then log(Re(ratio)) / dt;
  * the energy estimator's MeasurementOutput (Measurements.hpp:96-130): every observable's weighted
    sum all-reduced and divided by the all-reduced total weight.

The engine interface used: properties(), propagate / propagate_host, orthogonalize(), measure(),
dt, and the row calls of the walker exchange (exchange_device, walker_row_elems(), pack_walkers(),
unpack_walkers(), copy_walkers()) -- AfqmcEngine's, which keep the walker table on the device.
"""
import math

import numpy as np

from .popcontrol import comm_device, engine_population_control


def _allreduce(dist, values, group=None):
    """Sum of complex values over the ranks (values itself with dist None)."""
    v = np.asarray(values, dtype=np.complex128)
    if dist is None:
        return v
    import torch
    t = torch.from_numpy(v.view(np.float64).copy()).to(comm_device(dist, group))
    dist.all_reduce(t, group=group)
    return t.cpu().numpy().view(np.complex128)


def global_pseudo_energy(dist, engine, group=None):
    """averagePseudoEnergy over the ranks: log(Re(sum w e^{dt eloc} / sum w)) / dt."""
    pr = engine.properties()
    w, el = pr["WEIGHT"], pr["PSEUDO_ELOC_"]
    s = _allreduce(dist, [np.sum(w * np.exp(engine.dt * el)), np.sum(w)], group)
    return math.log((s[0] / s[1]).real) / engine.dt


def global_measure(dist, engine, group=None):
    """EnergyEstimator::measure over the ranks: each rank's normalised observables times its total
    weight, summed, over the summed total weight (the denominator MeasurementOutput all-reduces)."""
    m = engine.measure()
    keys = [k for k in m if k != "TotalWeight"]
    tw = m["TotalWeight"]
    s = _allreduce(dist, [m[k] * tw for k in keys] + [tw], group)
    out = {k: complex(s[i] / s[-1]) for i, k in enumerate(keys)}
    out["TotalWeight"] = complex(s[-1])
    return out


def run_sharded(dist, engine, steps, Eshift, comb_uniform, field_uniforms=None, ortho_interval=10,
                pop_interval=10, equilibration_steps=100, measure_interval=10, relax=None, step0=0, group=None):
    """run_afqmc's loop (run_afqmc.cpp:69-104) on this rank's walkers.  comb_uniform() is called on
    every rank at every population control (the root's draw is the one used, as the reference's
    walker_rng is drawn on the root); field_uniforms(n), when given, returns this rank's n = nwalk *
    nchol uniforms of a step (its own field stream), else the engine's Philox fields.
    Returns (Eshift, [(step, global measurement)])."""
    if relax is None:
        relax = 1 - math.exp(-10.0 / equilibration_steps) if equilibration_steps > 1 else 1.0
    meas = []
    for step in range(step0, step0 + steps):
        if field_uniforms is None:
            engine.propagate(Eshift, step)
        else:
            u = np.ascontiguousarray(np.asarray(field_uniforms(engine.W * engine.Nc), np.float64)
                                     .reshape(engine.W, engine.Nc))
            engine.propagate_host(Eshift, step, uniforms_host=u)
        if step % ortho_interval == 0:
            engine.orthogonalize()
        if step % pop_interval == 0:
            engine_population_control(dist, engine, float(comb_uniform()), group)
        if step >= equilibration_steps:
            if step % measure_interval == 0:
                meas.append((step, global_measure(dist, engine, group)))
        else:
            Eshift += relax * (global_pseudo_energy(dist, engine, group) - Eshift)
    return Eshift, meas
