"""Parity of the CUDA path (through the C ABI) with the oracle restatement,
stage by stage and frame by frame, and of the .evx bytes with the unmodified
reference encoder (GPU tables serialized by the reference's entropy coder).

Bit-exact is the bar: integer pixel work, mode decisions, motion vectors,
levels and the float RD costs (no FMA contraction, same operation order)."""
import functools

import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import (REF_VARIANTS, Ref, compare_blocks, join_ip_stream, pack_frame, plan_gop, plan_ip, split_stream,
                       unpack_frame)

pytestmark = pytest.mark.gpu

CASES = [  # (w, h, frames, quality, vmax, intra_at)
    (64, 48, 6, 8, 6.0, ()),
    (176, 144, 9, 8, 6.0, ()),
    (100, 60, 10, 4, 12.0, (6,)),
    (352, 288, 5, 16, 6.0, ()),
    (48, 32, 7, 31, 3.0, ()),
    (96, 64, 8, 1, 20.0, ()),
    (16, 16, 4, 8, 1.0, ()),          # one macroblock
    (34, 18, 5, 12, 4.0, ()),         # 48x32 context, heavy crop
]


FORMS = ("cluster", "single")   # three CTAs per macroblock row / one


def clip(w, h, T, vmax, seed=None, window=None, stretch=None):
    """The seeded test content; window=(first, cut) takes frames first.. of a
    longer sequence with a scene cut (the benchmark's generator); stretch
    scales the contrast about mid-grey, clipping to 0..255."""
    if window is None:
        frames = generate(w, h, T, seed=w * 7 + h if seed is None else seed, vmax=vmax)
    else:
        first, cut = window
        frames = generate(w, h, first + T, seed=seed, vmax=vmax, n_rects=4, cut_at=cut)[first:]
    if stretch is not None:
        frames = np.clip((frames.astype(np.float32) - 128.0) * stretch + 128.0, 0, 255).astype(np.uint8)
    return frames


@functools.lru_cache(maxsize=8)
def oracle_run(w, h, T, q, vmax, intra_at, cfg, seed=None, window=None, stretch=None):
    """The oracle's stage dumps of a clip (cached: the large cases serve both
    macroblock-pass forms)."""
    import chicago_b200 as cb
    from oracle_py import Oracle
    b_frames, ref_count, radius = cb.CONFIGS[cfg]
    frames = clip(w, h, T, vmax, seed, window, stretch)
    oc = Oracle().context(w, h, b_frames=b_frames, ref_count=ref_count, radius=radius)
    plan = plan_gop(T, quality=q, intra_at=intra_at) if b_frames else plan_ip(T, q, intra_at, ref_count)
    return frames, [(ti, f18, oc.encode_frame(frames[ti], f18)) for ti, f18 in plan]


def check_stream(oracle, w, h, T, q, vmax, intra_at, form="cluster", cfg="default", seed=None, window=None,
                 stretch=None):
    """Encode a seeded clip through the C ABI and compare every stage of every
    frame with the oracle restating the same reference build (cfg: "default",
    or the I/P builds "ip1" / "ip3")."""
    import chicago_b200 as cb
    frames, runs = oracle_run(w, h, T, q, vmax, tuple(intra_at), cfg, seed, window, stretch)
    st = cb.Stream(w, h, cfg)
    st.mb_form = cb.MB_FORM_CLUSTER if form == "cluster" else cb.MB_FORM_SINGLE
    for k, (ti, f18, od) in enumerate(runs):
        fr = unpack_frame(f18)
        st.encode_frame(frames[ti], f18)
        tb = st.fetch_tables()
        bad = compare_blocks(tb["blocks"], od.blocks)
        assert not bad, f"frame {k} {fr}: block fields differ {sorted(bad)}"
        assert np.array_equal(tb["levels"], od.levels), f"frame {k}: levels"
        assert np.array_equal(tb["sao"], od.sao), f"frame {k}: SAO table"
        assert np.array_equal(st.fetch_planes(4), od.src), f"frame {k}: converted source"
        assert np.array_equal(st.fetch_planes(fr["dpb_slot"]), od.final), f"frame {k}: reconstruction"
    return st


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("w,h,T,q,vmax,intra_at", CASES)
def test_gpu_matches_oracle(oracle, w, h, T, q, vmax, intra_at, form):
    check_stream(oracle, w, h, T, q, vmax, intra_at, form)


@pytest.mark.parametrize("form", FORMS)
def test_gpu_matches_oracle_1080p(oracle, form):
    """Full-size frames: I, P, reference-B and B at 1920x1080 (120x68 MBs)."""
    check_stream(oracle, 1920, 1080, 4, 8, 24.0, (), form)


IP_CASES = [  # (cfg, w, h, frames, quality, vmax, intra_at, seed)
    ("ip1", 64, 48, 6, 8, 6.0, (), None),
    ("ip1", 96, 64, 6, 1, 20.0, (), None),
    ("ip3", 176, 144, 8, 8, 3.0, (7,), 176 * 5 + 144 + 4),   # uses all three references
    ("ip3", 100, 60, 7, 4, 12.0, (4,), None),
    ("ip3", 352, 288, 5, 16, 6.0, (), None),
    ("ip3", 48, 32, 6, 31, 3.0, (), None),
]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("cfg,w,h,T,q,vmax,intra_at,seed", IP_CASES)
def test_gpu_matches_oracle_ip(oracle, cfg, w, h, T, q, vmax, intra_at, seed, form):
    """I/P builds (EVX_ENABLE_B_FRAMES 0): P frames search one or three
    references by offset from the frame index, with the distance bias."""
    check_stream(oracle, w, h, T, q, vmax, intra_at, form, cfg, seed)


@pytest.mark.parametrize("form", FORMS)
def test_gpu_matches_oracle_ip3_1080p(oracle, form):
    """Full-size I/P frames with three references: I and three P frames."""
    check_stream(oracle, 1920, 1080, 4, 8, 24.0, (), form, "ip3")


@pytest.mark.parametrize("form", FORMS)
def test_gpu_matches_oracle_4k(oracle, form):
    """3840x2160 (240x135 MBs), the served form's largest size: I, P,
    reference-B and B frames of the default build."""
    check_stream(oracle, 3840, 2160, 4, 8, 24.0, (), form, seed=4321)


@pytest.mark.parametrize("form", FORMS)
def test_gpu_matches_oracle_ip3_4k(oracle, form):
    """3840x2160 I/P frames with three references: I and two P frames."""
    check_stream(oracle, 3840, 2160, 3, 8, 24.0, (), form, "ip3", seed=4322)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("q", [4, 16])
def test_gpu_matches_oracle_1080p_scene_cut(oracle, q, form):
    """The benchmark's 1080p content around its scene cut (frames 58-62, cut at
    60) at quality 4 and 16, I/P with three references: I 58, P 59, the cut's
    I 60, P 61, P 62."""
    check_stream(oracle, 1920, 1080, 5, q, 24.0, (2,), form, "ip3", seed=1000, window=(58, 60))


@pytest.mark.parametrize("form", FORMS)
def test_gpu_matches_oracle_wide_frames(oracle, form):
    """Frames wider than the filters' shared-memory paths: at 16400 px the
    deblocking strips exceed their shared-memory window (in-place form); at
    54640 x 528 the SAO merge's hand-over words exceed shared memory too
    (memory-word form)."""
    check_stream(oracle, 16400, 32, 3, 8, 6.0, (), form, seed=77)
    check_stream(oracle, 54640, 528, 1, 8, 6.0, (), form, seed=78)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("cfg", ["default", "ip3"])
def test_gpu_matches_oracle_saturated(oracle, cfg, form):
    """Contrast stretched until large areas clip to 0 or 255.  The SAO merge
    costs an MB whose samples stay in [8, 247] from the RDO's band and
    edge-category sums, and any other MB on its pixels (where v + o may
    clamp); both kinds are frequent in every frame of this clip."""
    w, h, T = 352, 288, 6
    frames, runs = oracle_run(w, h, T, 8, 6.0, (), cfg, 91, None, 2.5)
    for _, _, od in runs:
        mbs = od.final[:w * h].reshape(h // 16, 16, w // 16, 16)
        near = ((mbs < 8) | (mbs > 247)).any(axis=(1, 3)).mean()
        assert 0.1 < near < 0.9, near
    check_stream(oracle, w, h, T, 8, 6.0, (), form, cfg, seed=91, stretch=2.5)


@pytest.mark.parametrize("variant", ["ip1", "ip3"])
def test_evx_bytes_match_stock_reference_ip(variant):
    """GOP-level encoder of an I/P configuration (C ABI) -> that reference
    build's entropy coder -> its stock .evx stream, byte for byte."""
    import chicago_b200 as cb
    if not __import__("os").path.exists(REF_VARIANTS[variant][0]):
        pytest.skip(f"reference variant {variant} not built")
    ref = Ref(variant=variant)
    w, h, T, q = 144, 96, 9, 8
    frames = generate(w, h, T, seed=6, vmax=6.0)
    stock = ref.encode_stream(frames, quality=q, intra_at=(5,))
    enc = cb.Encoder(quality=q, cfg=variant)
    for t in range(T):
        if t == 5:
            enc.insert_intra()
        enc.encode(frames[t])
    enc.flush()
    assert len(enc.records) == T
    ctx = ref.context(w, h)
    parts = [(r["frame18"], ctx.serialize(r["frame18"], r["blocks"], r["prev_blocks"], r["sao"], r["levels"]))
             for r in enc.records]
    assert join_ip_stream(stock[:14], parts) == stock


def test_evx_bytes_match_stock_reference(ref):
    """GOP-level encoder (C ABI) -> reference entropy coder -> stock .evx stream."""
    import chicago_b200 as cb
    w, h, T, q = 144, 96, 11, 8
    frames = generate(w, h, T, seed=5, vmax=8.0)
    stock = ref.encode_stream(frames, quality=q, intra_at=(7,))
    _, payloads = split_stream(stock)
    enc = cb.Encoder(quality=q)
    for t in range(T):
        if t == 7:
            enc.insert_intra()
        enc.encode(frames[t])
    enc.flush()
    assert len(enc.records) == len(payloads)
    ctx = ref.context(w, h)
    for k, r in enumerate(enc.records):
        sl = ctx.serialize(r["frame18"], r["blocks"], r["prev_blocks"], r["sao"], r["levels"])
        assert r["frame18"] + sl == payloads[k], f"frame {k} bytes differ"


def test_cluster_form_is_the_default():
    """A B200 co-schedules three-CTA clusters: streams start in the cluster form."""
    import chicago_b200 as cb
    st = cb.Stream(64, 48)
    assert st.mb_form == cb.MB_FORM_CLUSTER
    st.mb_form = cb.MB_FORM_SINGLE
    assert st.mb_form == cb.MB_FORM_SINGLE
    with pytest.raises(cb.EvxgError):
        st.mb_form = 7


def test_stream_rejects_bad_frames():
    import chicago_b200 as cb
    st = cb.Stream(64, 48)
    rgb = np.zeros((48, 64, 3), np.uint8)
    with pytest.raises(cb.EvxgError) as e:
        st.encode_frame(rgb, pack_frame(1, 0, 8, 0, 1, 5, 0, 0))
    assert e.value.code == 6
    with pytest.raises(cb.EvxgError):
        st.encode_frame(rgb, pack_frame(1, 0, 8, 0, 1, 1, 1, 0))   # reference == destination
    with pytest.raises(cb.EvxgError):
        st.encode_frame(rgb, pack_frame(0, 0, 0, 0, 1, 0, 0, 0))   # QP 0
    with pytest.raises(cb.EvxgError):
        cb.Stream(63, 48)                                           # odd width


def test_deterministic_repeat():
    """Two encodes of the same input give identical tables (no races)."""
    import chicago_b200 as cb
    w, h = 320, 192
    frames = generate(w, h, 5, seed=9, vmax=10.0)
    res = []
    for _ in range(2):
        st = cb.Stream(w, h)
        out = []
        for ti, f18 in plan_gop(5, quality=8):
            st.encode_frame(frames[ti], f18)
            out.append(st.fetch_tables())
        res.append(out)
    for a, b in zip(*res):
        for key in a:
            assert np.array_equal(a[key], b[key])


@pytest.mark.parametrize("cfg", ["default", "ip1", "ip3"])
def test_encoder_bitstream_equals_stock_stream(cfg):
    """The GOP-level encoder with its bitstream output on: GPU pixel pipeline,
    then the library's own host entropy coder -- no reference code -- give the
    stock encoder's .evx stream byte for byte (but the header's padding byte,
    which the reference leaves uninitialised)."""
    import os
    import chicago_b200 as cb
    path = REF_VARIANTS[cfg][0] if cfg != "default" else None
    if path and not os.path.exists(path):
        pytest.skip(f"reference variant {cfg} not built")
    ref = Ref(variant=None if cfg == "default" else cfg)
    w, h, T, q = 160, 96, 11, 8
    frames = generate(w, h, T, seed=12, vmax=6.0)
    stock = ref.encode_stream(frames, quality=q, intra_at=(6,))
    enc = cb.Encoder(quality=q, cfg=cfg, bitstream=True)
    for t in range(T):
        if t == 6:
            enc.insert_intra()
        enc.encode(frames[t])
    enc.flush()
    mine = bytes(enc.stream)
    assert len(mine) == len(stock)
    assert mine[:7] == stock[:7] and mine[8:] == stock[8:]


@pytest.mark.parametrize("cfg,w,h,T", [("default", 176, 144, 9), ("ip3", 352, 288, 8)])
def test_pipelined_frames_equal_synchronous_frames(cfg, w, h, T):
    """evxg_encode_frame_pipelined (uploads and downloads on the stream's copy
    stream, several frames in flight) gives every frame's tables exactly as
    evxg_encode_frame + evxg_fetch_tables do."""
    import chicago_b200 as cb
    b_frames, ref_count, _ = cb.CONFIGS[cfg]
    frames = generate(w, h, T, seed=w + T, vmax=8.0)
    plan = plan_gop(T, quality=8) if b_frames else plan_ip(T, 8, (), ref_count)
    a, b = cb.Stream(w, h, cfg), cb.Stream(w, h, cfg)
    want = []
    for ti, f18 in plan:
        a.encode_frame(frames[ti], f18)
        want.append(a.fetch_tables())
    outs, tickets = [], []
    for ti, f18 in plan:   # every frame issued before any is waited for
        o = {k: np.zeros_like(v) for k, v in want[0].items()}
        outs.append(o)
        tickets.append(b.encode_pipelined(np.ascontiguousarray(frames[ti]), f18, o))
    for k, t in enumerate(tickets):
        b.output_wait(t)
        for key in want[k]:
            assert np.array_equal(outs[k][key], want[k][key]), f"frame {k}: {key}"


@pytest.mark.parametrize("cfg", ["default", "ip3"])
def test_encoder_peek_views_match_reference(cfg):
    """evxg_encoder_peek gives the stock encoder's peek() images after every
    encode() call: source, destination slot, block types, QP, sub-pel and
    variance maps; the prediction view is not implemented in either."""
    import os
    import chicago_b200 as cb
    if cfg != "default" and not os.path.exists(REF_VARIANTS[cfg][0]):
        pytest.skip("reference variant not built")
    ref = Ref() if cfg == "default" else Ref(variant=cfg)
    w, h, T = 100, 60, 7
    frames = generate(w, h, T, seed=17, vmax=8.0)
    want = ref.peeks(frames, 8, range(7))
    enc = cb.Encoder(quality=8, cfg=cfg)
    for t in range(T):
        enc.encode(frames[t])
        for st in range(7):
            if st == 1:
                assert want[t][st] == 2
                with pytest.raises(cb.EvxgError) as e:
                    enc.peek(st, w, h)
                assert e.value.code == 2
                continue
            assert np.array_equal(enc.peek(st, w, h), want[t][st]), f"call {t}: view {st}"
    enc.close()
