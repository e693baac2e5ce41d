"""Autotuner for a tank or a batch: it times the launch shapes the library offers and keeps the fastest.

Knobs (``suiri_tune`` / ``suiri_batch_tune``, ``suiri_tune_piece`` / ``suiri_batch_tune_piece``):
  * blocks per SM of the persistent particle kernels (binning, scatter, G2P);
  * the form of the pressure solve (sor_mode): 0 one launch per colour sweep inside the sub-step graph,
    1 the whole solve as one cooperative launch with a grid barrier between sweeps, 2 two colour sweeps
    per launch over per-tile lists of active cells, 3 four sweeps per launch on shared-memory tiles with
    halos (temporal blocking), 4 the whole solve in one launch with each tank held in one thread-block
    cluster's shared memory;
  * the tile of sor_mode 4: the shared memory one CTA takes (piece_kb; 0 = the device's maximum), which
    sets the z planes per CTA and so the CTAs per tank and the cluster size.

Each candidate is timed on the device (events on the tank's or batch's stream) over a few sub-steps of the
real state, after one sub-step that captures its graph. Targets that can save and restore their state
(``save_state`` / ``restore_state``: the tanks' water copies) are put back afterwards, so tuning leaves the
simulation where it found it.
"""

CANDIDATES = ((2, 0, 0), (4, 0, 0), (8, 0, 0), (4, 2, 0), (4, 3, 0), (4, 1, 0),
              (2, 4, 0), (2, 4, 160), (2, 4, 112), (2, 4, 80), (4, 4, 0))


def autotune(target, dt, candidates=CANDIDATES, steps=3):
    """Return ((blocks_per_sm, sor_mode, piece_kb), {candidate: ms per sub-step}) and leave the best set."""
    timings = {}
    last = None
    saved = target.save_state() if hasattr(target, 'save_state') else None
    try:
        for cand in candidates:
            bps, mode = cand[0], cand[1]
            piece = cand[2] if len(cand) > 2 else 0
            try:
                target.tune_piece(piece)
                target.tune(bps, mode)
                target.time_substeps(dt, 1)
                timings[cand] = target.time_substeps(dt, steps) / steps
            except Exception as e:      # a shape the device cannot launch (too large to be co-resident, …)
                timings[cand] = float('inf')
                last = e
    finally:
        if saved is not None:
            target.restore_state(saved)
    best = min(timings, key=timings.get)
    if timings[best] == float('inf'):
        raise last
    target.tune_piece(best[2] if len(best) > 2 else 0)
    target.tune(best[0], best[1])
    return best, timings
