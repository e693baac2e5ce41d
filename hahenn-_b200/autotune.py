"""Autotuner for a tank or a batch: it times the launch shapes the library offers and keeps the fastest.

Knobs (``suiri_tune`` / ``suiri_batch_tune``, ``suiri_tune_piece`` / ``suiri_batch_tune_piece``):
  * blocks per SM of the persistent particle kernels (binning, scatter, G2P);
  * the form of the pressure solve (sor_mode): 0 one launch per colour sweep inside the sub-step graph,
    1 the whole solve as one cooperative launch with a grid barrier between sweeps, 2 two colour sweeps
    per launch over per-tile lists of active cells, 3 four sweeps per launch on shared-memory tiles with
    halos (temporal blocking), 4 the whole solve in one launch with each tank held in one thread-block
    cluster's shared memory;
  * the tile of sor_mode 4: the shared memory one CTA takes (piece_kb; 0 = the device's maximum), which
    sets the z planes per CTA and so the CTAs per tank and the cluster size;
  * the form of the grid-to-particle pass (``suiri_tune_g2p``): a grid-stride walk, its common path with the
    rare branches deferred to a second pass, or one block per brick with the brick's faces staged in shared
    memory; tried with the best of the other knobs.

A batch is tuned lane by lane (``autotune_batch``): its size lanes run concurrently, and small tanks may
prefer another form than large ones.

Each candidate is timed on the device (events on the tank's or batch's stream) over a few sub-steps of the
real state, after one sub-step that captures its graph. Targets that can save and restore their state
(``save_state`` / ``restore_state``: the tanks' water copies) are put back afterwards, so tuning leaves the
simulation where it found it.
"""

CANDIDATES = ((2, 0, 0), (4, 0, 0), (8, 0, 0), (4, 2, 0), (4, 3, 0), (4, 1, 0),
              (2, 4, 0), (2, 4, 192), (2, 4, 128), (2, 4, 96), (2, 4, 64), (4, 4, 0))


G2P_FORMS = (0, 2, 1)


def _time(target, dt, steps):
    target.time_substeps(dt, 1)                  # captures the graph of the new shape
    return target.time_substeps(dt, steps) / steps


def autotune(target, dt, candidates=CANDIDATES, steps=3, g2p_forms=G2P_FORMS):
    """Return ((blocks_per_sm, sor_mode, piece_kb, g2p_form), {candidate: ms per sub-step}) and leave the best
    set. The candidates (blocks per SM, solve form, tile) are timed with the first G2P form; the other G2P
    forms are then timed with the best of them."""
    timings = {}
    last = None
    saved = target.save_state() if hasattr(target, 'save_state') else None
    has_g2p = hasattr(target, 'tune_g2p')
    try:
        if has_g2p:
            target.tune_g2p(g2p_forms[0])
        for cand in candidates:
            key = (cand[0], cand[1], cand[2] if len(cand) > 2 else 0, g2p_forms[0])
            try:
                target.tune_piece(key[2])
                target.tune(key[0], key[1])
                timings[key] = _time(target, dt, steps)
            except Exception as e:      # a shape the device cannot launch (too large to be co-resident, …)
                timings[key] = float('inf')
                last = e
        best = min(timings, key=timings.get)
        if timings[best] == float('inf'):
            raise last
        if has_g2p:
            target.tune_piece(best[2])
            target.tune(best[0], best[1])
            for form in g2p_forms[1:]:
                key = best[:3] + (form,)
                try:
                    target.tune_g2p(form)
                    timings[key] = _time(target, dt, steps)
                except Exception as e:
                    timings[key] = float('inf')
                    last = e
            best = min((k for k in timings if k[:3] == best[:3]), key=timings.get)
    finally:
        if saved is not None:
            target.restore_state(saved)
    target.tune_piece(best[2])
    target.tune(best[0], best[1])
    if has_g2p:
        target.tune_g2p(best[3])
    return best, timings


def autotune_batch(batch, dt, candidates=CANDIDATES, steps=3, g2p_forms=G2P_FORMS):
    """Tune each size lane of a batch in turn (the others keep their settings) on the batch's sub-step time,
    with the batch's state rolled back afterwards. Returns ([best per lane], {lane: timings})."""
    saved = batch.save_state()
    best, timings = [], {}
    try:
        n = batch.lanes()
        for k in range(n):
            batch.tune_lane(k, *CANDIDATES[0][:2], 0, g2p_forms[0])
        for k in range(n):
            b, t = autotune(batch.lane(k), dt, candidates, steps, g2p_forms)
            best.append(b)
            timings[k] = t
    finally:
        batch.restore_state(saved)
    for k, b in enumerate(best):
        batch.tune_lane(k, *b)
    return best, timings
