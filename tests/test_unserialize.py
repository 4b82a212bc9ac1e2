"""The library's host entropy decoder (evxg_unserialize_slice) against the
reference decoder's own (unserialize_slice, built from the reference's
sources and run step by step by the test harness).

For seeded stock streams of every supported build, frame by frame in
bitstream order, the decoded block table (every byte, the fields a slice does
not code included: both decoders keep earlier frames' values there), SAO
table and level planes must equal the reference decoder's, and the slice's
length must come out exact -- also when the next records follow the slice,
which is how the I/P builds' streams arrive.  Runs on the CPU: the entropy
decoder has no device part."""
import os

import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import REF_SO, REF_VARIANTS, Ref, plan_ip, split_stream, unpack_frame

CASES = [  # (cfg, w, h, frames, quality, vmax, intra_at)
    ("default", 64, 48, 7, 8, 6.0, ()),
    ("default", 176, 144, 8, 16, 6.0, (5,)),    # the reference decoder's stale fields change the next P frame
    ("default", 100, 60, 9, 4, 12.0, (6,)),
    ("default", 48, 32, 6, 31, 3.0, ()),
    ("default", 96, 64, 6, 1, 20.0, ()),
    ("ip1", 64, 48, 6, 8, 6.0, ()),
    ("ip1", 96, 64, 6, 1, 20.0, (4,)),
    ("ip3", 176, 144, 7, 8, 3.0, (6,)),
    ("ip3", 100, 60, 6, 16, 14.0, ()),
]


def reference_for(cfg):
    path = REF_SO if cfg == "default" else REF_VARIANTS[cfg][0]
    if not os.path.exists(path):
        pytest.skip(f"reference build {path} not present")
    return Ref(path)


def payloads_of(ref, cfg, frames, q, intra_at):
    """The stock stream and its frame payloads (evx_frame + slice), bitstream order."""
    import chicago_b200 as cb
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    if cb.CONFIGS[cfg][0]:
        return stock, split_stream(stock)[1]
    T, h, w = frames.shape[:3]
    rc = ref.context(w, h)
    out = []
    for ti, f18 in plan_ip(T, quality=q, intra_at=intra_at, ref_count=cb.CONFIGS[cfg][1]):
        _, sl = rc.encode_frame(frames[ti], f18)
        out.append(bytes(f18[:10]) + sl)
    assert stock[:14] + b"".join(out) == stock
    return stock, out


@pytest.mark.parametrize("cfg,w,h,T,q,vmax,intra_at", CASES)
def test_unserialize_matches_reference_decoder(cfg, w, h, T, q, vmax, intra_at):
    import chicago_b200 as cb
    ref = reference_for(cfg)
    frames = generate(w, h, T, seed=w * 3 + h + q, vmax=vmax)
    stock, payloads = payloads_of(ref, cfg, frames, q, intra_at)
    b_frames = cb.CONFIGS[cfg][0]
    fb = 18 if b_frames else 10
    aw, ah = (w + 15) & ~15, (h + 15) & ~15
    nblk = (aw // 16) * (ah // 16)
    blocks = np.zeros(nblk * 28, np.uint8)
    prev = np.zeros(nblk * 28, np.uint8)
    sao = np.zeros(nblk * 16, np.uint8)
    levels = np.zeros(aw * ah * 3 // 2, np.int16)
    rd = ref.decoder(w, h)
    rest = stock[14:]
    for k, p in enumerate(payloads):
        d = rd.decode_frame(p)
        f18 = d["frame18"]
        sl = p[fb:]
        # the slice alone, and followed by the rest of the stream
        data = sl if b_frames else rest[fb:]
        used = cb.unserialize_slice(cfg, aw, ah, f18, data, blocks, prev, sao, levels)
        assert used == len(sl), f"record {k}: slice length {used} != {len(sl)}"
        assert np.array_equal(blocks, d["blocks"]), f"record {k} {unpack_frame(f18)}: block table"
        assert np.array_equal(sao, d["sao"]), f"record {k}: SAO table"
        assert np.array_equal(levels, d["levels"]), f"record {k}: levels"
        if not (b_frames and unpack_frame(f18)["type"] == 2):
            prev[:] = blocks
        rest = rest[(4 if b_frames else 0) + len(p):]


def test_unserialize_rejects_damaged_slices():
    """A truncated slice or bytes that are no slice of the format give
    EVXG_ERROR_INVALID_RESOURCE instead of tables."""
    import chicago_b200 as cb
    ref = reference_for("default")
    w, h = 64, 48
    stock, payloads = payloads_of(ref, "default", generate(w, h, 3, seed=5, vmax=6.0), 8, ())
    nblk = 12
    tabs = [np.zeros(nblk * 28, np.uint8), np.zeros(nblk * 28, np.uint8), np.zeros(nblk * 16, np.uint8),
            np.zeros(64 * 48 * 3 // 2, np.int16)]
    f18, sl = payloads[0][:18], payloads[0][18:]
    with pytest.raises(cb.EvxgError) as e:
        cb.unserialize_slice("default", 64, 48, f18, sl[: len(sl) // 2], *tabs)
    assert e.value.code == 8
