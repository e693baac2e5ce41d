"""Autotuner for a tank or a batch: it times the launch shapes the library offers and keeps the fastest.

Knobs (``suiri_tune`` / ``suiri_batch_tune``):
  * blocks per SM of the persistent particle kernels (binning, scatter, G2P);
  * the form of the pressure solve (sor_mode): 0 one launch per colour sweep inside the sub-step graph,
    1 the whole solve as one cooperative launch with a grid barrier between sweeps, 2 two colour sweeps
    per launch over per-tile lists of active cells, 3 four sweeps per launch on shared-memory tiles with
    halos (temporal blocking).

Each candidate is timed on the device (events on the tank's or batch's stream) over a few sub-steps of the
real state, after one sub-step that captures its graph. Tuning advances the simulation by those
sub-steps.
"""

CANDIDATES = ((2, 0), (4, 0), (8, 0), (4, 2), (8, 2), (4, 3), (4, 1))


def autotune(target, dt, candidates=CANDIDATES, steps=3):
    """Return ((blocks_per_sm, sor_mode), {candidate: ms per sub-step}) and leave the best set."""
    timings = {}
    last = None
    for bps, mode in candidates:
        try:
            target.tune(bps, mode)
            target.time_substeps(dt, 1)
            timings[(bps, mode)] = target.time_substeps(dt, steps) / steps
        except Exception as e:          # a shape the device cannot launch (e.g. too large to be co-resident)
            timings[(bps, mode)] = float('inf')
            last = e
    best = min(timings, key=timings.get)
    if timings[best] == float('inf'):
        raise last
    target.tune(best[0], best[1])
    return best, timings
