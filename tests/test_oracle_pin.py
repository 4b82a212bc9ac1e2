"""Pins the oracle restatement to the unmodified reference library built from
its own sources (oracle/_ref): every stage of every frame must be identical,
and the planner-driven staged reference must reproduce the stock encoder's
.evx stream byte for byte (which also pins the GOP planner)."""
import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import REF_VARIANTS, Ref, compare_blocks, join_ip_stream, plan_gop, plan_ip, split_stream, unpack_frame

CASES = [  # (w, h, frames, quality, vmax, intra_at)
    (64, 48, 6, 8, 6.0, ()),
    (176, 144, 9, 4, 6.0, ()),
    (100, 60, 10, 16, 14.0, (6,)),      # 16-alignment crop, forced intra
    (48, 32, 7, 31, 3.0, ()),           # coarsest quality
    (96, 64, 8, 1, 20.0, ()),           # finest quality, fast motion
]


@pytest.mark.parametrize("w,h,T,q,vmax,intra_at", CASES)
def test_oracle_matches_reference_stages(ref, oracle, w, h, T, q, vmax, intra_at):
    frames = generate(w, h, T, seed=w * 7 + h, vmax=vmax)
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    _, payloads = split_stream(stock)
    plan = plan_gop(T, quality=q, intra_at=intra_at)
    assert len(plan) == len(payloads)
    rc, oc = ref.context(w, h), oracle.context(w, h)
    for k, (ti, f18) in enumerate(plan):
        d, sl = rc.encode_frame(frames[ti], f18)
        assert f18 + sl == payloads[k], f"staged reference != stock encoder at frame {k}"
        od = oc.encode_frame(frames[ti], f18)
        assert not compare_blocks(d.blocks, od.blocks), f"block table differs at frame {k} {unpack_frame(f18)}"
        for nm in ("src", "levels", "recon", "deblock", "sao", "final"):
            assert np.array_equal(getattr(d, nm), getattr(od, nm)), f"{nm} differs at frame {k}"


def test_wpp_schedule_equals_raster(ref):
    """The reference's own WPP schedule reproduces its sequential raster order."""
    w, h, T = 160, 96, 5
    frames = generate(w, h, T, seed=11, vmax=8.0)
    a, b = ref.context(w, h), ref.context(w, h)
    for ti, f18 in plan_gop(T, quality=8):
        da, sa = a.encode_frame(frames[ti], f18, wpp=False)
        db, sb = b.encode_frame(frames[ti], f18, wpp=True)
        assert sa == sb and np.array_equal(da.final, db.final)


IP_CASES = [  # (variant, w, h, frames, quality, vmax, intra_at); the last two ip3 cases must use all three references
    ("ip1", 64, 48, 6, 8, 6.0, ()),
    ("ip1", 100, 60, 8, 16, 14.0, (5,)),
    ("ip3", 64, 48, 7, 8, 6.0, ()),
    ("ip3", 96, 64, 9, 1, 20.0, (6,)),
    ("ip3", 48, 32, 6, 31, 3.0, ()),
    ("ip3", 176, 144, 6, 4, 8.0, ()),
    ("ip3", 176, 144, 8, 8, 3.0, (7,)),
]
COVER = {("ip3", 176, 144)}


def variant_ref(variant):
    if not __import__("os").path.exists(REF_VARIANTS[variant][0]):
        pytest.skip(f"reference variant {variant} not built (make -C oracle variants)")
    return Ref(variant=variant)


@pytest.mark.parametrize("variant,w,h,T,q,vmax,intra_at", IP_CASES)
def test_oracle_matches_reference_ip_variants(oracle, variant, w, h, T, q, vmax, intra_at):
    """The I/P builds (EVX_ENABLE_B_FRAMES 0; one or three references): the
    planner-driven staged reference reproduces the stock stream, and the
    restatement with the same switches matches it at every stage."""
    ref = variant_ref(variant)
    _, b_frames, ref_count = REF_VARIANTS[variant]
    assert (ref.b_frames, ref.ref_count, ref.frame_bytes, ref.block_bytes) == (0, ref_count, 10, 18)
    frames = generate(w, h, T, seed=w * 5 + h + ref_count, vmax=vmax)
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    plan = plan_ip(T, quality=q, intra_at=intra_at, ref_count=ref_count)
    rc, oc = ref.context(w, h), oracle.context(w, h, b_frames=0, ref_count=ref_count)
    staged = []
    targets = set()
    for k, (ti, f18) in enumerate(plan):
        d, sl = rc.encode_frame(frames[ti], f18)
        staged.append((f18, sl))
        od = oc.encode_frame(frames[ti], f18)
        assert not compare_blocks(d.blocks, od.blocks), f"block table differs at frame {k} {unpack_frame(f18)}"
        for nm in ("src", "levels", "recon", "deblock", "sao", "final"):
            assert np.array_equal(getattr(d, nm), getattr(od, nm)), f"{nm} differs at frame {k}"
        bt = d.block_table()
        targets |= set(bt["prediction_target"][(bt["block_type"] & 1) == 0].tolist())
    assert join_ip_stream(stock[:14], staged) == stock, "staged reference != stock I/P encoder"
    if (variant, w, h) in COVER:
        assert targets == {1, 2, 3}, f"expected blocks predicted from all three references, saw {targets}"


def test_sequential_build_equals_wpp_build(ref):
    """The single-thread reference build (EVX_ENABLE_WPP 0) encodes the same
    stream as the default WPP build."""
    seq = variant_ref("seq")
    assert seq.wpp == 0 and ref.wpp == 1
    frames = generate(96, 64, 6, seed=3, vmax=8.0)
    a, b = seq.encode_stream(frames, quality=8), ref.encode_stream(frames, quality=8)
    # Byte 7 of the stream header is a struct pad byte that the reference never
    # initialises, so it differs between runs.
    assert len(a) == len(b) and a[:7] == b[:7] and a[8:] == b[8:]


DEC_CASES = [  # (variant, w, h, frames, quality, vmax, intra_at); None = the default build
    (None, 100, 60, 9, 8, 8.0, ()),
    (None, 176, 144, 8, 16, 6.0, (5,)),
    ("ip1", 64, 48, 7, 16, 6.0, ()),
    ("ip3", 176, 144, 8, 4, 8.0, (6,)),
]


def reference_records(ref, variant, frames, q, intra_at):
    """The stock stream, its frame records in bitstream order (payload =
    evx_frame + slice; record = what one decode() call reads, the first with
    the header in front) and the encoder's final reconstruction of each frame
    by display order."""
    T, h, w, _ = frames.shape
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    rc = ref.context(w, h)
    if variant is None:
        plan = plan_gop(T, quality=q, intra_at=intra_at)
    else:
        plan = plan_ip(T, quality=q, intra_at=intra_at, ref_count=REF_VARIANTS[variant][2])
    final, payloads = {}, []
    for ti, f18 in plan:
        d, sl = rc.encode_frame(frames[ti], f18)
        payloads.append(bytes(f18[:len(f18) if variant is None else 10]) + sl)
        final[unpack_frame(f18)["display_order"] if variant is None else ti] = d.final
    if variant is None:
        assert split_stream(stock)[1] == payloads
        records = [len(p).to_bytes(4, "little") + p for p in payloads]
    else:
        assert stock[:14] + b"".join(payloads) == stock
        records = list(payloads)
    records[0] = stock[:14] + records[0]
    return stock, payloads, records, final


@pytest.mark.parametrize("variant,w,h,T,q,vmax,intra_at", DEC_CASES)
def test_staged_reference_decoder_equals_stock_decoder(oracle, variant, w, h, T, q, vmax, intra_at):
    """The staged engine_decode_frame (unserialize, decode_slice, deblock, SAO,
    YUV -> RGB) gives the stock evx3_decoder's frames; its RGB is the restated
    conversion of its final reconstruction.  Without an inserted intra frame in
    the default build the decoder reproduces the encoder's reconstruction; with
    one, the reference's decoder departs from its encoder: unserialize_slice
    writes only the fields it codes, so the intra frame's descriptors keep the
    previous B frame's prediction fields, which the next P frame's motion
    vector prediction reads (the encoder cleared them)."""
    ref = Ref() if variant is None else variant_ref(variant)
    frames = generate(w, h, T, seed=w + 3 * h + q, vmax=vmax)
    stock, payloads, records, final = reference_records(ref, variant, frames, q, intra_at)
    dec = ref.decode_records(records, w, h)
    assert len(dec) == T
    if variant is None:   # the default build's records carry sizes: the whole stream decodes in one go
        assert np.array_equal(ref.decode_stream(stock, w, h), dec)
    dc = ref.decoder(w, h)
    aw, ah = (w + 15) & ~15, (h + 15) & ~15
    staged = {}
    for k, p in enumerate(payloads):
        d = dc.decode_frame(p)
        assert np.array_equal(d["rgb"], oracle.yuv_to_rgb(d["final"], aw, ah, w, h)), f"record {k}: YUV -> RGB"
        staged[unpack_frame(d["frame18"])["display_order"] if variant is None else k] = d
    for k in range(T):
        assert np.array_equal(dec[k], staged[k]["rgb"]), f"frame {k} (display order)"
    same = [np.array_equal(staged[k]["final"], final[k]) for k in range(T)]
    if variant is not None or not intra_at:
        assert all(same)
    else:
        assert not all(same)
