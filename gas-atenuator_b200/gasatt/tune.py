"""Autotuning of the resident simulation's launch-shape knobs.

Four knobs change speed and not results (random streams are keyed on
particle ids and steps, the deposit is an exact integer sum, and the field
update's arithmetic is the same for every patch):

  sort_period     steps between cell re-sorts: a sort costs a pass over the
                  state, while the particles' drift away from their sorted
                  order slowly makes the gather and the deposit less local;
  fdtd_tile_rows  rows R of the field update's per-warp patch (12, 16 or 20;
                  a warp computes 26 columns x R - 6 rows of output from 32 x R
                  staged points): the halo recomputed per output point against
                  the registers a warp holds and the number of patches for
                  the warps to share;
  pass_chunk      particles per chunk of the FP32 particle pass (its deposit
                  window's span against the number of chunks for the blocks
                  to balance);
  gather          where the FP32 push reads E and H: packed 2 x 2 quads the
                  field update writes beside the fields (fewer loads per
                  electron, 48 more bytes written per cell), or the fields.

The best setting depends on the workload (particle speed, cell size, time
step, population, grid), so it is measured: fresh copies of the same
population run a few hundred steps per candidate, one knob at a time with the
others at their best so far (coordinate descent), and the fastest wins.
"""
import ctypes

import torch

from . import abi
from .sim import Sim

DEFAULT_SORT_PERIODS = (10, 20, 30, 40, 60)
DEFAULT_TILE_ROWS = (12, 16, 20)
DEFAULT_CHUNKS = (1024, 1280, 1536, 1792)


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


def _copy(cfg, **changes):
    c = type(cfg)()
    ctypes.memmove(ctypes.byref(c), ctypes.byref(cfg), ctypes.sizeof(cfg))
    for k, v in changes.items():
        setattr(c, k, int(v))
    return c


def ms_per_step(cfg, particles, steps=200, ctx=None, tables=None, device=0):
    """Milliseconds per step of this configuration on a fresh copy of the
    population (`particles`: the tuple accepted by Sim.load)."""
    sim = Sim(cfg, ctx=ctx, tables=tables, device=device)
    try:
        sim.load(*particles)
        return time_steps(sim, steps) / steps
    finally:
        sim.close()


def tune_sort_period(cfg, particles, candidates=DEFAULT_SORT_PERIODS, steps=200, ctx=None,
                     tables=None, device=0):
    """Sort period (from `candidates`) with the shortest time for `steps` steps
    of this configuration and population.  Returns (best_period, {period: ms
    per step})."""
    per_step = {int(sp): ms_per_step(_copy(cfg, sort_period=sp), particles, steps, ctx, tables,
                                     device) for sp in candidates}
    best = min(per_step, key=per_step.get)
    return best, per_step


def knob_candidates(cfg):
    """The candidates of each knob for this configuration's precision form
    (the chunk size is a knob of the FP32 pass only)."""
    fp32 = cfg.precision == abi.FP32_SPLIT
    knobs = {"fdtd_tile_rows": DEFAULT_TILE_ROWS}
    if cfg.fdtd_ratio != 1:
        knobs = {}                         # only the fdtd_ratio 1 field update has tiles
    if fp32:
        knobs["pass_chunk"] = DEFAULT_CHUNKS
        knobs["gather"] = (abi.GATHER_QUADS, abi.GATHER_FIELDS)
    knobs["sort_period"] = DEFAULT_SORT_PERIODS
    return knobs


def tune(cfg, particles, knobs=None, steps=200, ctx=None, tables=None, device=0):
    """Coordinate descent over the launch-shape knobs: each knob in turn takes
    the candidate with the shortest time per step, the others held at their
    best so far.  Returns (a copy of cfg with the choices, {knob: {value: ms
    per step}})."""
    knobs = knob_candidates(cfg) if knobs is None else knobs
    best = _copy(cfg)
    table = {}
    for name, cands in knobs.items():
        per = {int(v): ms_per_step(_copy(best, **{name: v}), particles, steps, ctx, tables, device)
               for v in cands}
        setattr(best, name, min(per, key=per.get))
        table[name] = per
    return best, table
