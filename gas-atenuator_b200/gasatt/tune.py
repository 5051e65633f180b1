"""Autotuning of the resident simulation's run-time knobs.

The only knob that changes speed and not results is the sort period: a cell
re-sort costs a pass over the state, while the particles' drift away from
their sorted order slowly makes the gather and the deposit less local.  The
best period depends on the workload (particle speed, cell size, time step,
population), so it is measured: fresh copies of the same population are run
for a few hundred steps at each candidate period and the fastest is kept.
Results do not depend on the period (random streams are keyed on particle ids
and steps, and the deposit is an exact integer sum), so tuning never changes
the physics."""
import ctypes

import torch

from .sim import Sim

DEFAULT_SORT_PERIODS = (10, 20, 30, 40, 60)


def time_steps(sim, steps, warmup=5):
    """Device time (ms) of `steps` back-to-back steps after `warmup` steps."""
    stream = torch.cuda.current_stream(sim.device)
    sim.bind_stream(stream)
    sim.step(warmup)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def tune_sort_period(cfg, particles, candidates=DEFAULT_SORT_PERIODS, steps=200, ctx=None,
                     tables=None, device=0):
    """Sort period (from `candidates`) with the shortest time for `steps` steps
    of this configuration and population.  `particles` is the tuple accepted
    by Sim.load.  Returns (best_period, {period: ms per step})."""
    per_step = {}
    for sp in candidates:
        c = type(cfg)()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(cfg), ctypes.sizeof(cfg))
        c.sort_period = int(sp)
        sim = Sim(c, ctx=ctx, tables=tables, device=device)
        try:
            sim.load(*particles)
            per_step[int(sp)] = time_steps(sim, steps) / steps
        finally:
            sim.close()
    best = min(per_step, key=per_step.get)
    return best, per_step
