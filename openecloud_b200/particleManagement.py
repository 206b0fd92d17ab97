"""Macro-particle management: Russian roulette and local merge/split.

Mirrors ``particleManagement`` (particleManagement.pyx): ``globalRandom``
(:35-67) and ``localRandom`` (:74-238).  Selection, cloning, sorting, splitting
and merging run on the GPU (manage.cu); the host computes only the scalar
bookkeeping the reference computes (counts, thresholds, typical velocity).

localRandom keeps the reference's thresholds, split/merge counts and
phase-space metric, but the merge pairs neighbours inside a grid cell after
ordering the merge candidates by (cell, velocity) instead of walking a
kd-tree sequentially; total weight is conserved by every merge and split.
The reference's split draws its trial positions in cell units and tests them
against the wall in metres (particleManagement.pyx:133-162), so for chambers
smaller than a metre every split is an exact duplicate at half weight; the
split here is that duplicate.
"""
import numpy as np
import torch

from . import _lib
from . import device as D
from .constants import c

_CALLS = {"n": 0}


def _next_call():
    _CALLS["n"] += 1
    return _CALLS["n"]


def _mask_clear(P):
    fails = D.zeros(1, torch.int32)
    _lib.call("oec_roulette_select", 0, 0, P._mask.data_ptr(), P._mask.shape[0], 0, 0, fails.data_ptr(),
              D.stream())


def globalRandom(gridObj, particlesObj, targetMacroParticleCount, seed=0, call=None):
    """Reference: particleManagement.pyx:35-67.  The draws are keyed by
    (seed, call); `call` defaults to a process-wide counter (a run that must
    be reproducible on its own passes its own count of management events)."""
    P = particlesObj
    P._bind(gridObj)
    n = P.getMacroParticleCount()
    target = int(targetMacroParticleCount)
    diff = n - target
    factor = float(n) / float(target)
    s = D.stream()
    call = _next_call() if call is None else int(call)
    if diff > 0:
        _lib.call("oec_scale_weights", P.c_particles(), factor, s)
        fails = D.zeros(1, torch.int32)
        _lib.call("oec_roulette_select", n, diff, P._mask.data_ptr(), P._mask.shape[0], int(seed), call,
                  fails.data_ptr(), s)
        if int(fails.item()):
            raise RuntimeError("globalRandom: selection did not converge")
        P.addAndRemoveParticles(np.zeros((0, 6)), None)
    elif target > n:
        _lib.call("oec_scale_weights", P.c_particles(), factor, s)
        rows = D.empty((-diff, 6), torch.float64)
        _lib.call("oec_clone_rows", gridObj.c_grid(), P.c_particles(), n, -diff, int(seed), call, rows.data_ptr(), s)
        _mask_clear(P)
        P.addAndRemoveParticles(rows, None)


def localRandom(gridObj, particlesObj, particleBoundaryObj, targetMacroParticleCount, phaseSpaceWeights=None,
                thresholdFactor=2., lambdavFactor=1., factorDisLimit=1., mergeScheme=0, seed=0, oversample=4,
                call=None):
    """Reference: particleManagement.pyx:74-238 (see the module docstring);
    `call` as in globalRandom."""
    P = particlesObj
    P._bind(gridObj)
    n = P.getMacroParticleCount()
    target = int(targetMacroParticleCount)
    s = D.stream()
    meanWeight = P.getMeanWeight()
    goal = meanWeight * n / target
    maxT, minT = thresholdFactor * goal, goal / thresholdFactor
    ds = min(gridObj.getDx(), gridObj.getDy())
    P.sortByColumn(5)
    # the two _searchSorted thresholds on the device: 8 bytes come back
    # instead of the weight array
    thr = D.zeros(2, torch.int32)
    _lib.call("oec_weight_thresholds", P.c_particles(), float(minT), float(maxT), thr.data_ptr(), s)
    lo_idx, hi_idx = (int(x) for x in D.to_numpy(thr))
    to_merge = lo_idx
    to_split = n - hi_idx
    if 2 * to_merge + to_split >= n:
        f = 0.95 * n / (2 * to_merge + to_split)
        to_merge, to_split = int(to_merge * f), int(to_split * f)
    new_n = n + to_split - to_merge
    if new_n > target:
        to_merge += new_n - target
    elif new_n < target:
        to_split += target - new_n
    if 2 * to_merge + to_split >= n:
        f = 0.95 * n / (2 * to_merge + to_split)
        to_merge, to_split = int(to_merge * f), int(to_split * f)
    acc = D.zeros(2, torch.float64)
    _lib.call("oec_weight_stats", P.c_particles(), acc.data_ptr(), s)
    vt = float(np.sqrt(acc[1].item())) / (n * meanWeight)
    vt = max(vt, 1.e-12 * c)
    rows = D.empty((max(to_split, 1), 6), torch.float64)
    _lib.call("oec_split_rows", gridObj.c_grid(), P.c_particles(), n, to_split, rows.data_ptr(), s)
    if phaseSpaceWeights is not None and len(phaseSpaceWeights) >= 5:
        lam = float(phaseSpaceWeights[2])
    else:
        lam = lambdavFactor * ds / vt
    _mask_clear(P)
    n_cand = min(n - to_split, max(0, int(oversample * to_merge)))
    n_cand -= n_cand % 2
    if to_merge > 0 and n_cand >= 2:
        work = D.empty(int(_lib.lib().oec_sort_work_bytes(P._cap)), torch.uint8)
        counters = D.zeros(2, torch.int32)
        _lib.call("oec_cell_merge", gridObj.c_grid(), P.c_particles(), n_cand, to_merge, lam, factorDisLimit * ds,
                  int(mergeScheme), int(seed), _next_call() if call is None else int(call), 3.0 * vt, P._mask.data_ptr(), counters.data_ptr(),
                  work.data_ptr(), s)
        localRandom.last_counters = counters.cpu().numpy()
    P.addAndRemoveParticles(rows[:to_split], None)
    localRandom.last_counts = (to_merge, to_split)
