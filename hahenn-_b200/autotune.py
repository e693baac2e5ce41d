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
simulation where it found it. The first candidate is the default; a shape that beats it on its first
reading is timed twice more beside it and kept only if its slowest reading still wins by MARGIN, since some
forms (the cluster solve beside a busy lane) swing by a fifth from one graph launch to the next.
"""

CANDIDATES = ((2, 0, 0), (4, 0, 0), (8, 0, 0), (4, 2, 0), (4, 3, 0), (4, 1, 0),
              (2, 4, 0), (2, 4, 192), (2, 4, 128), (2, 4, 96), (2, 4, 64), (4, 4, 0))


G2P_FORMS = (0, 2, 1)

MARGIN = 0.01       # a shape replaces the first (default) one only when it is faster by this fraction
CONFIRM = 2         # extra readings of the two finalists before that choice


def _time(target, dt, steps):
    target.time_substeps(dt, 1)                  # captures the graph of the new shape
    return target.time_substeps(dt, steps) / steps


def _settle(target, dt, steps, timings, keys, apply, confirm):
    """The fastest of `keys` by its first reading, checked against the first key (the default): both are
    timed `confirm` more times, interleaved, and each is scored by its slowest reading: a form whose sub-step
    time swings from one graph launch to the next counts with its bad readings. The fastest replaces the
    default only when it still wins by MARGIN."""
    default, first = keys[0], min(keys, key=timings.get)
    if first == default or timings[default] == float('inf') or confirm <= 0:
        return first
    score = {default: timings[default], first: timings[first]}
    for _ in range(confirm):
        for key in (default, first):
            apply(key)
            score[key] = max(score[key], _time(target, dt, steps))
    return first if score[first] * (1 + MARGIN) < score[default] else default


def autotune(target, dt, candidates=CANDIDATES, steps=3, g2p_forms=G2P_FORMS, confirm=CONFIRM):
    """Return ((blocks_per_sm, sor_mode, piece_kb, g2p_form), {candidate: ms per sub-step}) and leave the best
    set. The candidates (blocks per SM, solve form, tile) are timed with the first G2P form; the other G2P
    forms are then timed with the best of them. The first candidate and the first G2P form are the
    defaults: another shape is kept only when it stays faster by MARGIN over repeated readings. The timings
    returned are the first readings."""
    timings = {}
    last = None
    saved = target.save_state() if hasattr(target, 'save_state') else None
    has_g2p = hasattr(target, 'tune_g2p')

    def shape(key):
        target.tune_piece(key[2])
        target.tune(key[0], key[1])

    try:
        if has_g2p:
            target.tune_g2p(g2p_forms[0])
        keys = []
        for cand in candidates:
            key = (cand[0], cand[1], cand[2] if len(cand) > 2 else 0, g2p_forms[0])
            keys.append(key)
            try:
                shape(key)
                timings[key] = _time(target, dt, steps)
            except Exception as e:      # a shape the device cannot launch (too large to be co-resident, …)
                timings[key] = float('inf')
                last = e
        if min(timings.values()) == float('inf'):
            raise last
        best = _settle(target, dt, steps, timings, keys, shape, confirm)
        if has_g2p:
            shape(best)
            forms = [best]
            for form in g2p_forms[1:]:
                key = best[:3] + (form,)
                forms.append(key)
                try:
                    target.tune_g2p(form)
                    timings[key] = _time(target, dt, steps)
                except Exception as e:
                    timings[key] = float('inf')
                    last = e
            best = _settle(target, dt, steps, timings, forms, lambda key: target.tune_g2p(key[3]), confirm)
    finally:
        if saved is not None:
            target.restore_state(saved)
    shape(best)
    if has_g2p:
        target.tune_g2p(best[3])
    return best, timings


def autotune_batch(batch, dt, candidates=CANDIDATES, steps=3, g2p_forms=G2P_FORMS, confirm=CONFIRM):
    """Tune each size lane of a batch in turn (the others keep their settings) on the batch's sub-step time,
    with the batch's state rolled back afterwards. Returns ([best per lane], {lane: timings})."""
    saved = batch.save_state()
    best, timings = [], {}
    try:
        n = batch.lanes()
        for k in range(n):
            batch.tune_lane(k, *CANDIDATES[0][:2], 0, g2p_forms[0])
        for k in range(n):
            b, t = autotune(batch.lane(k), dt, candidates, steps, g2p_forms, confirm)
            best.append(b)
            timings[k] = t
    finally:
        batch.restore_state(saved)
    for k, b in enumerate(best):
        batch.tune_lane(k, *b)
    return best, timings
