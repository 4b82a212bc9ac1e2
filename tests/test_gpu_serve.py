"""Serving (evxg_server_*): continuous batching over live streams.

Streams of different sizes and qualities join while others are on the GPU,
submit frames interleaved with the others', insert intra frames and close at
different times; each stream's results (frame descriptor and the
serializer's tables, in bitstream order) must equal the same stream encoded
alone by the GOP-level encoder (evxg_encoder_*), bit for bit -- the tolerance
of every parity test here.  Admission by the device memory budget refuses a
stream that does not fit and admits it once another has closed."""
import time

import numpy as np
import pytest

from chicago_b200.synth import generate

pytestmark = pytest.mark.gpu

# (width, height, quality, frames, intra insertions, round it joins)
SPEC = [(64, 48, 8, 9, (), 0), (176, 144, 4, 11, (5,), 0), (96, 64, 16, 7, (), 3), (34, 18, 12, 10, (3,), 5)]


def alone(w, h, q, frames, intra_at):
    import chicago_b200 as cb
    enc = cb.Encoder(quality=q)
    for t, f in enumerate(frames):
        if t in intra_at:
            enc.insert_intra()
        enc.encode(f)
    enc.flush()
    return enc.records


@pytest.mark.timeout(300)
def test_server_results_equal_streams_alone():
    import chicago_b200 as cb
    srv = cb.Server(hbm_budget_bytes=1 << 34, max_streams=8)
    seqs = [generate(w, h, n, seed=300 + k, vmax=3.0 + k) for k, (w, h, q, n, ia, j) in enumerate(SPEC)]
    ids, pos = [None] * len(SPEC), [0] * len(SPEC)
    for rnd in range(100):
        for k, (w, h, q, n, ia, join) in enumerate(SPEC):
            if ids[k] is None and rnd >= join:
                ids[k] = srv.open(w, h, q)
            if ids[k] is None or pos[k] >= n:
                continue
            if pos[k] in ia:
                srv.insert_intra(ids[k])
            srv.submit(ids[k], seqs[k][pos[k]])
            pos[k] += 1
            if pos[k] == n:
                srv.close_stream(ids[k])
        if all(p >= s[3] for p, s in zip(pos, SPEC)):
            break
        time.sleep(0.003)   # frames keep arriving while ticks run
    srv.drain()
    for k, (w, h, q, n, ia, join) in enumerate(SPEC):
        got, want = srv.results[ids[k]], alone(w, h, q, seqs[k], ia)
        assert len(got) == len(want) == n
        for i, (g, e) in enumerate(zip(got, want)):
            assert g["frame18"] == e["frame18"], f"stream {k} record {i}: frame"
            for key in ("blocks", "prev_blocks", "sao", "levels"):
                assert np.array_equal(g[key], e[key]), f"stream {k} record {i}: {key}"
            a, r, l, d = g["times"]
            assert 0 < a <= r <= l <= d
    st = srv.stats()
    assert st["frames"] == sum(s[3] for s in SPEC) and st["rebuilds"] >= 2 and st["bytes_in_use"] == 0
    srv.close()


@pytest.mark.timeout(300)
def test_server_admission_by_memory_budget():
    import chicago_b200 as cb
    srv = cb.Server(hbm_budget_bytes=1_500_000, max_streams=8)   # room for two 176x144 streams (about 0.62 MB each)
    a, b = srv.open(176, 144), srv.open(176, 144)
    with pytest.raises(cb.EvxgError) as e:
        srv.open(176, 144)
    assert e.value.code == 7   # EVXG_ERROR_CAPACITY_LIMIT
    frames = generate(176, 144, 2, seed=7, vmax=2.0)
    srv.submit(a, frames[0])
    srv.close_stream(a)
    srv.drain()                # the closed stream's memory is back in the budget
    c = srv.open(176, 144)
    srv.submit(c, frames[1])
    srv.close_stream(b)
    srv.close_stream(c)
    srv.drain()
    assert len(srv.results[a]) == 1 and len(srv.results[c]) == 1 and len(srv.results[b]) == 0
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


@pytest.mark.timeout(300)
def test_server_admission_survives_allocation_failure():
    """Host-side fault injection: a device allocation fails while a stream is
    admitted.  The admission reports EVXG_ERROR_OUTOFMEMORY and gives its
    budget reservation back; the stream already running is unaffected and a
    later admission succeeds."""
    import chicago_b200 as cb
    srv = cb.Server(hbm_budget_bytes=1 << 34, max_streams=4)
    fa = generate(96, 64, 6, seed=51, vmax=4.0)
    fb = generate(64, 48, 5, seed=52, vmax=3.0)
    a = srv.open(96, 64, 8)
    for f in fa[:3]:
        srv.submit(a, f)
    used = srv.stats()["bytes_in_use"]
    cb.lib().evxg_inject_alloc_failures(1)   # the next stream creation's first device allocation fails
    with pytest.raises(cb.EvxgError) as e:
        srv.open(64, 48, 8)
    assert e.value.code == 3                  # EVXG_ERROR_OUTOFMEMORY
    assert srv.stats()["bytes_in_use"] == used
    for f in fa[3:]:
        srv.submit(a, f)
    b = srv.open(64, 48, 8)                   # no failure pending: admitted
    for f in fb:
        srv.submit(b, f)
    srv.close_stream(a)
    srv.close_stream(b)
    srv.drain()
    for sid, frames in ((a, fa), (b, fb)):
        want = alone(*((96, 64) if sid == a else (64, 48)), 8, frames, ())
        got = srv.results[sid]
        assert len(got) == len(want)
        for g, w_ in zip(got, want):
            assert g["frame18"] == w_["frame18"]
            for key in ("blocks", "prev_blocks", "sao", "levels"):
                assert np.array_equal(g[key], w_[key])
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


@pytest.mark.timeout(300)
def test_server_cancel_mid_gop_leaves_other_streams_alone():
    """A stream cancelled in the middle of its GOP: what it got delivered is a
    prefix of its results alone; the other streams' results equal theirs alone."""
    import chicago_b200 as cb
    srv = cb.Server(hbm_budget_bytes=1 << 34, max_streams=4)
    spec = [(96, 64, 8, 10), (64, 48, 4, 10), (80, 48, 12, 9)]
    seqs = [generate(w, h, n, seed=60 + k, vmax=4.0) for k, (w, h, q, n) in enumerate(spec)]
    ids = [srv.open(w, h, q) for (w, h, q, n) in spec]
    for t in range(10):
        for k, (w, h, q, n) in enumerate(spec):
            if k == 1 and t == 6:
                srv.cancel(ids[1])            # mid-GOP: its last frames wait for their P anchor
            if t < n and not (k == 1 and t >= 6):
                srv.submit(ids[k], seqs[k][t])
        time.sleep(0.002)
    for k in (0, 2):
        srv.close_stream(ids[k])
    srv.drain()
    for k, (w, h, q, n) in enumerate(spec):
        want = alone(w, h, q, seqs[k] if k != 1 else seqs[k][:n], ())
        got = srv.results[ids[k]]
        if k == 1:
            assert len(got) <= 6
        else:
            assert len(got) == len(want) == n
        for i, g in enumerate(got):
            assert g["frame18"] == want[i]["frame18"], f"stream {k} record {i}"
            for key in ("blocks", "prev_blocks", "sao", "levels"):
                assert np.array_equal(g[key], want[i][key]), f"stream {k} record {i}: {key}"
    with pytest.raises(cb.EvxgError):
        srv.submit(ids[1], seqs[1][0])       # a cancelled stream takes no more frames
    assert srv.stats()["bytes_in_use"] == 0
    srv.close()


@pytest.mark.timeout(300)
@pytest.mark.parametrize("cfg", ["default", "ip3"])
def test_stream_checkpoint_continues_bit_identically(cfg):
    """evxg_stream_save after frame k, evxg_stream_restore into a fresh stream:
    its following frames equal the uninterrupted stream's."""
    import chicago_b200 as cb
    from oracle_py import plan_gop, plan_ip
    b_frames, ref_count, _ = cb.CONFIGS[cfg]
    w, h, T, k = 176, 144, 10, 5
    frames = generate(w, h, T, seed=41, vmax=6.0)
    plan = plan_gop(T, quality=8) if b_frames else plan_ip(T, 8, (), ref_count)
    a = cb.Stream(w, h, cfg)
    want = []
    for ti, f18 in plan:
        a.encode_frame(frames[ti], f18)
        want.append(a.fetch_tables())
    b = cb.Stream(w, h, cfg)
    for ti, f18 in plan[:k]:
        b.encode_frame(frames[ti], f18)
    state = b.save()
    b.close()
    c = cb.Stream(w, h, cfg)
    c.restore(state)
    for i, (ti, f18) in enumerate(plan[k:], start=k):
        c.encode_frame(frames[ti], f18)
        got = c.fetch_tables()
        for key in want[i]:
            assert np.array_equal(got[key], want[i][key]), f"frame {i}: {key}"
    with pytest.raises(cb.EvxgError):   # another size
        cb.Stream(w + 16, h, cfg).restore(state)


@pytest.mark.timeout(300)
def test_server_evict_restore_continues_bit_identically():
    """A served stream evicted mid-sequence frees its device memory, refuses
    frames while evicted, and after restore its results equal the stream
    encoded alone; a neighbour keeps running meanwhile."""
    import chicago_b200 as cb
    srv = cb.Server(hbm_budget_bytes=1 << 34, max_streams=4)
    w, h, q, n = 176, 144, 8, 12
    seq = generate(w, h, n, seed=77, vmax=5.0)
    other = generate(96, 64, n, seed=78, vmax=4.0)
    sid, oid = srv.open(w, h, q), srv.open(96, 64, 8)
    for t in range(6):
        srv.submit(sid, seq[t])
        srv.submit(oid, other[t])
    srv.drain()
    before = srv.stats()["bytes_in_use"]
    srv.evict(sid)
    assert srv.stats()["bytes_in_use"] < before
    with pytest.raises(cb.EvxgError) as e:
        srv.submit(sid, seq[6])
    assert e.value.code == 15   # EVXG_ERROR_NOT_READY
    for t in range(6, 9):
        srv.submit(oid, other[t])
    srv.restore(sid)
    for t in range(6, n):
        srv.submit(sid, seq[t])
    for t in range(9, n):
        srv.submit(oid, other[t])
    srv.close_stream(sid)
    srv.close_stream(oid)
    srv.drain()
    for s_, frames, (ww, hh, qq) in ((sid, seq, (w, h, q)), (oid, other, (96, 64, 8))):
        got, want = srv.results[s_], alone(ww, hh, qq, frames, ())
        assert len(got) == len(want) == n
        for i, (g, e_) in enumerate(zip(got, want)):
            assert g["frame18"] == e_["frame18"], f"stream {s_} record {i}: frame"
            for key in ("blocks", "prev_blocks", "sao", "levels"):
                assert np.array_equal(g[key], e_[key]), f"stream {s_} record {i}: {key}"
    srv.close()
