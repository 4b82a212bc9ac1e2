"""The decoder's pixel half on the GPU (evxg_decode_frame through the C ABI).

Parity is against the reference's own decoder run step by step on the CPU
(engine_decode_frame, src/video/decode.cpp:560-612): the tables its
unserialize_slice produced go into the GPU decoder, whose reconstruction and
RGB24 frame must equal the reference's byte for byte -- including the default
build after an inserted intra frame, where the reference's decoder departs
from its encoder and a drop-in decoder has to depart with it.  Decoding the
tables the GPU encoder produced must give back the encoder's reconstruction."""
import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import REF_VARIANTS, Ref, plan_gop, plan_ip, split_stream, unpack_frame

pytestmark = pytest.mark.gpu

CFG_OF = {None: "default", "ip1": "ip1", "ip3": "ip3"}

REF_CASES = [  # (variant, w, h, frames, quality, vmax, intra_at); None = the default build
    (None, 176, 144, 9, 8, 6.0, ()),
    (None, 176, 144, 8, 16, 6.0, (5,)),     # the reference decoder's drift after an inserted intra frame
    (None, 100, 60, 10, 4, 12.0, (6,)),     # 16-alignment crop
    (None, 34, 18, 5, 12, 4.0, ()),         # one macroblock row pair, heavy crop
    ("ip1", 96, 64, 8, 16, 14.0, (5,)),
    ("ip3", 176, 144, 8, 8, 3.0, (7,)),
    ("ip3", 96, 64, 9, 1, 20.0, (6,)),      # finest quality, fast motion
    (None, 1920, 1080, 4, 8, 24.0, ()),
    ("ip3", 1920, 1080, 4, 8, 24.0, ()),
]


def ref_for(variant):
    import os
    if variant is None:
        return Ref()
    if not os.path.exists(REF_VARIANTS[variant][0]):
        pytest.skip(f"reference variant {variant} not built")
    return Ref(variant=variant)


def stock_payloads(ref, variant, frames, q, intra_at):
    """The stock stream's frame payloads (evx_frame + slice) in bitstream order."""
    T = frames.shape[0]
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    if variant is None:
        return split_stream(stock)[1]
    # records of an I/P build carry no size: cut them with the staged encoder's slices
    h, w = frames.shape[1:3]
    rc = ref.context(w, h)
    out = []
    for ti, f18 in plan_ip(T, quality=q, intra_at=intra_at, ref_count=REF_VARIANTS[variant][2]):
        _, sl = rc.encode_frame(frames[ti], f18)
        out.append(bytes(f18[:10]) + sl)
    assert stock[:14] + b"".join(out) == stock
    return out


@pytest.mark.parametrize("variant,w,h,T,q,vmax,intra_at", REF_CASES)
def test_decoder_matches_reference_decoder(variant, w, h, T, q, vmax, intra_at):
    import chicago_b200 as cb
    ref = ref_for(variant)
    frames = generate(w, h, T, seed=w * 3 + h + q, vmax=vmax)
    payloads = stock_payloads(ref, variant, frames, q, intra_at)
    rd = ref.decoder(w, h)
    dec = cb.Decoder(w, h, CFG_OF[variant])
    for k, p in enumerate(payloads):
        d = rd.decode_frame(p)
        fr = unpack_frame(d["frame18"])
        rgb = dec.decode_frame(d["frame18"], d["blocks"], d["sao"], d["levels"])
        slot = fr["dpb_slot"] if variant is None else fr["index"] % REF_VARIANTS[variant][2]
        assert np.array_equal(dec.fetch_planes(slot), d["final"]), f"record {k} {fr}: reconstruction"
        assert np.array_equal(rgb, d["rgb"]), f"record {k} {fr}: RGB"


ROUND_TRIP = [  # (cfg, w, h, frames, quality, vmax, intra_at)
    ("default", 176, 144, 9, 8, 6.0, (5,)),
    ("ip1", 100, 60, 8, 16, 14.0, (5,)),
    ("ip3", 352, 288, 6, 4, 8.0, ()),
    ("ip3", 1920, 1080, 3, 8, 24.0, ()),
]


@pytest.mark.parametrize("cfg,w,h,T,q,vmax,intra_at", ROUND_TRIP)
def test_decoder_reproduces_gpu_encoder(oracle, cfg, w, h, T, q, vmax, intra_at):
    """The GPU encoder's tables, decoded on the GPU, give back its reconstruction
    (every DPB slot after every frame) and the restated RGB of it."""
    import chicago_b200 as cb
    b_frames, ref_count, _ = cb.CONFIGS[cfg]
    frames = generate(w, h, T, seed=w + h + q, vmax=vmax)
    plan = plan_gop(T, quality=q, intra_at=intra_at) if b_frames else plan_ip(T, q, intra_at, ref_count)
    st, dec = cb.Stream(w, h, cfg), cb.Decoder(w, h, cfg)
    for k, (ti, f18) in enumerate(plan):
        st.encode_frame(frames[ti], f18)
        tb = st.fetch_tables()
        rgb = dec.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
        for s in range(4):
            assert np.array_equal(dec.fetch_planes(s), st.fetch_planes(s)), f"frame {k}: DPB slot {s}"
        fr = unpack_frame(f18)
        assert np.array_equal(rgb, oracle.yuv_to_rgb(st.fetch_planes(fr["dpb_slot"]), st.aw, st.ah, w, h))


def encoded_tables(w, h, T, cfg="default", q=8):
    import chicago_b200 as cb
    frames = generate(w, h, T, seed=7, vmax=6.0)
    st = cb.Stream(w, h, cfg)
    out = []
    for ti, f18 in plan_gop(T, quality=q):
        st.encode_frame(frames[ti], f18)
        out.append((f18, st.fetch_tables()))
    return out


def test_decoder_rejects_invalid_descriptors():
    """A block type the reference's decode_block rejects (decode.cpp:429) or a
    reference that is no other DPB slot makes the frame fail with
    EVXG_ERROR_INVALID_RESOURCE; the decoder then decodes correctly again."""
    import chicago_b200 as cb
    w, h = 176, 144
    seq = encoded_tables(w, h, 5)
    k = next(i for i, (_, tb) in enumerate(seq) if ((tb["blocks"].view(cb.BLOCK_DTYPE)["block_type"] & 1) == 0).any())
    for field, value in (("block_type", 5), ("block_type", 9), ("prediction_target", 7)):
        dec = cb.Decoder(w, h)
        for f18, tb in seq[:k]:
            dec.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
        f18, tb = seq[k]   # the first frame with inter blocks
        bad = tb["blocks"].copy().view(cb.BLOCK_DTYPE)
        inter = np.nonzero((bad["block_type"] & 1) == 0)[0]
        bad[field][inter[0]] = value
        with pytest.raises(cb.EvxgError) as e:
            dec.decode_frame(f18, bad.view(np.uint8), tb["sao"], tb["levels"])
        assert e.value.code == 8, e.value   # EVXG_ERROR_INVALID_RESOURCE
        dec.reset()
        ok = cb.Decoder(w, h)
        for f18, tb in seq[:k + 1]:
            a = dec.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
            b = ok.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
            assert np.array_equal(a, b)


def test_decoder_intra_wavefront_timeout_recovers():
    """The intra wavefront's waits are bounded: with a 1 ns bound an intra frame
    fails with EVXG_ERROR_OPERATION_TIMEDOUT and every CTA returns; after a
    reset and the normal bound the same frame decodes exactly."""
    import chicago_b200 as cb
    w, h = 640, 360
    f18, tb = encoded_tables(w, h, 1)[0]
    ok = cb.Decoder(w, h)
    want = ok.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
    dec = cb.Decoder(w, h)
    dec.set_timeout_ns(1)
    with pytest.raises(cb.EvxgError) as e:
        dec.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"])
    assert e.value.code == 9, e.value   # EVXG_ERROR_OPERATION_TIMEDOUT
    dec.reset()
    dec.set_timeout_ns(5_000_000_000)
    assert np.array_equal(dec.decode_frame(f18, tb["blocks"], tb["sao"], tb["levels"]), want)


STREAM_CASES = [  # (variant, w, h, frames, quality, vmax, intra_at)
    (None, 176, 144, 9, 8, 6.0, (5,)),
    (None, 100, 60, 10, 16, 12.0, ()),
    ("ip1", 96, 64, 8, 16, 14.0, (5,)),
    ("ip3", 176, 144, 8, 4, 8.0, (6,)),
    ("ip3", 1920, 1080, 4, 8, 24.0, ()),
]


@pytest.mark.parametrize("variant,w,h,T,q,vmax,intra_at", STREAM_CASES)
def test_stream_decoder_matches_reference_decoder(variant, w, h, T, q, vmax, intra_at):
    """The product decoder end to end -- header, records cut by the entropy
    decoder itself, host entropy decoding, GPU pixel half, display reorder --
    gives the stock evx3_decoder's frames.  The I/P builds' streams, which the
    stock decoder cannot take whole, are compared with it fed record by record."""
    import chicago_b200 as cb
    ref = ref_for(variant)
    frames = generate(w, h, T, seed=w + 5 * h + q, vmax=vmax)
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    mine = cb.StreamDecoder(CFG_OF[variant]).decode(stock)
    if variant is None:
        want = ref.decode_stream(stock, w, h)
    else:
        records = stock_payloads(ref, variant, frames, q, intra_at)
        records[0] = stock[:14] + records[0]
        want = ref.decode_records(records, w, h)
    assert len(mine) == len(want) == T
    for k in range(T):
        assert np.array_equal(mine[k], want[k]), f"frame {k} (display order)"


@pytest.mark.parametrize("cfg", ["default", "ip3"])
def test_tools_round_trip_matches_reference_tool(tmp_path, cfg):
    """Raw RGB file -> tools encode (GPU encoder, container) -> the reference
    tool's container byte for byte (but the stream header's uninitialised
    padding byte); tools decode -> the reference decoder's frames."""
    import chicago_b200 as cb
    from chicago_b200 import tools
    variant = None if cfg == "default" else cfg
    ref = ref_for(variant)
    w, h, T, fps, q = 176, 144, 9, 30.0, 8
    frames = generate(w, h, T, seed=21, vmax=6.0)
    src, mine, theirs, out = (str(tmp_path / n) for n in ("in.rgb", "mine.evx3", "ref.evx3", "out.rgb"))
    frames.tofile(src)
    tools.encode_file(src, mine, w, h, fps, q, cfg)
    ref.encode_container(theirs, frames, fps, q)
    a, b = open(mine, "rb").read(), open(theirs, "rb").read()
    pad = 10 + 18 + 16 + 7
    assert len(a) == len(b) and a[:pad] == b[:pad] and a[pad + 1:] == b[pad + 1:]
    tools.decode_file(mine, out, cfg)
    got = np.fromfile(out, np.uint8).reshape(-1, h, w, 3)
    stock = ref.encode_stream(frames, quality=q)
    if variant is None:
        want = ref.decode_stream(stock, w, h)
    else:
        records = stock_payloads(ref, variant, frames, q, ())
        records[0] = stock[:14] + records[0]
        want = ref.decode_records(records, w, h)
    assert got.shape[0] == T and np.array_equal(got, want)
