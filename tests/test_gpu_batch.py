"""Batched ticks (evxg_batch_*) against the single-stream path.

Streams of uneven sizes, qualities and GOP positions (intra insertions at
different frames, streams that have no frame in some ticks) advance together
through batched ticks; after every tick each stream's tables (block table,
previous table, SAO table, levels) and reconstruction must equal the same
stream encoded alone through evxg_encode_frame -- bit for bit, the tolerance
of every parity test here -- in every shape of the macroblock pass, with the
host waiting after each tick and with ticks issued back to back on the two
buffer parities."""
import numpy as np
import pytest

from chicago_b200.gop import plan, unpack_frame
from chicago_b200.synth import generate

pytestmark = pytest.mark.gpu

SIZES = [(64, 48), (176, 144), (96, 64), (34, 18)]
QUALITY = [8, 4, 16, 12]


def sequences(sizes, T, qualities):
    seqs = []
    for k, (w, h) in enumerate(sizes):
        frames = generate(w, h, T, seed=100 + k, vmax=4.0 + 2 * k)
        intra = (k + 2,) if k % 2 else ()
        seqs.append((frames, plan(T, quality=qualities[k], intra_at=intra)))
    return seqs


def run_batch(sizes, qualities, ticks, shape=None, autotune=False, skip=True, pipelined=False):
    import chicago_b200 as cb
    streams = [cb.Stream(w, h) for w, h in sizes]
    alone = [cb.Stream(w, h) for w, h in sizes]
    b = cb.Batch(streams)
    if autotune:
        b.autotune()
    if shape is not None:
        b.set_shape(*shape)
    seqs = sequences(sizes, ticks + 2, qualities)
    pos = [0] * len(sizes)
    pending = {}   # parity -> (tick, frames of the tick issued on it)

    def check(par):
        for k, item in enumerate(pending.pop(par)[1]):
            if item is None:
                continue
            ti, f18 = item
            frames = seqs[k][0]
            alone[k].encode_frame(frames[ti], f18)
            want = alone[k].fetch_tables()
            got = b.output(k, par)
            for key in want:
                assert np.array_equal(got[key], want[key]), f"stream {k} {sizes[k]} frame {unpack_frame(f18)}: {key}"
            slot = unpack_frame(f18)["dpb_slot"]
            if not pipelined:   # the slot is final only until the stream's next tick
                assert np.array_equal(streams[k].fetch_planes(slot), alone[k].fetch_planes(slot)), f"stream {k}: recon"

    for t in range(ticks):
        par = t & 1
        if par in pending:
            b.wait(par)
            check(par)
        f18s = []
        for k in range(len(sizes)):
            frames, sched = seqs[k]
            if (skip and (t + k) % 3 == 2) or pos[k] >= len(sched):
                f18s.append(None)
                continue
            ti, f18 = sched[pos[k]]
            pos[k] += 1
            b.input(k, par)[:] = frames[ti]
            f18s.append((ti, f18))
        b.encode([None if x is None else x[1] for x in f18s], par)
        pending[par] = (t, f18s)
        if not pipelined:
            b.wait(par)
            check(par)
    for par in sorted(pending, key=lambda p: pending[p][0]):   # remaining ticks, in tick order
        b.wait(par)
        check(par)
    assert b.launch_count() == 18
    return b


SHAPES = [
    None,          # default: one CTA per row, grid of every SM (capped at the rows)
    (0, 3, 0),     # a small persistent grid: CTAs take several rows each
    (0, 64, 1),    # longer remaining path first
    (1, 2, 1),     # three-CTA clusters, two of them
    (1, 16, 0),
]


@pytest.mark.parametrize("shape", SHAPES)
def test_batch_matches_streams_alone(shape):
    run_batch(SIZES, QUALITY, ticks=9, shape=shape)


def test_batch_pipelined_parities():
    """Ticks issued back to back, each parity checked before it is reused."""
    run_batch(SIZES, QUALITY, ticks=8, shape=(1, 8, 1), pipelined=True)


def test_batch_after_autotune():
    """The autotuner returns the streams to their initial state."""
    import chicago_b200 as cb
    b = run_batch(SIZES[:3], QUALITY[:3], ticks=5, autotune=True, skip=False)
    form, grid, policy = b.shape
    assert form in (cb.MB_FORM_SINGLE, cb.MB_FORM_CLUSTER) and grid >= 1 and policy in (0, 1)


def test_batch_mixed_resolutions():
    """The batched configuration's sizes: 1080p, 720p and 360p in one tick."""
    run_batch([(1920, 1080), (1280, 720), (640, 360)], [8, 8, 8], ticks=3, shape=None, skip=False)
