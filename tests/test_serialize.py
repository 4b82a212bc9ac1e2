"""The library's host entropy coder (evxg_serialize_slice) against the
reference's own (serialize_slice, built from the reference's sources).

The tables come from the oracle restatement (pinned stage by stage to the
reference elsewhere) for seeded clips of every supported build -- the default
hierarchical P/B GOP and the I/P builds with one and three references --
across qualities, crops and forced intra frames; for every frame the slice
bytes must be identical, and streams assembled with evxg_stream_header and
the reference's frame framing must equal the stock encoder's stream byte for
byte (but the header's padding byte, which the reference leaves
uninitialised).  Runs on the CPU: the entropy coder has no device part."""
import os
import struct

import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import REF_SO, REF_VARIANTS, Ref, join_ip_stream, plan_gop, plan_ip, split_stream

CASES = [  # (cfg, w, h, frames, quality, vmax, intra_at)
    ("default", 64, 48, 7, 8, 6.0, ()),
    ("default", 100, 60, 9, 4, 12.0, (5,)),
    ("default", 176, 144, 6, 16, 6.0, ()),
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


@pytest.mark.parametrize("cfg,w,h,T,q,vmax,intra_at", CASES)
def test_slices_and_stream_match_reference(oracle, cfg, w, h, T, q, vmax, intra_at):
    import chicago_b200 as cb
    ref = reference_for(cfg)
    b_frames, ref_count, radius = cb.CONFIGS[cfg]
    frames = generate(w, h, T, seed=w * 3 + h + q, vmax=vmax)
    plan = plan_gop(T, quality=q, intra_at=intra_at) if b_frames else plan_ip(T, q, intra_at, ref_count)
    oc = oracle.context(w, h, b_frames=b_frames, ref_count=ref_count, radius=radius)
    rc = ref.context(w, h)
    mine = []
    for k, (ti, f18) in enumerate(plan):
        prev = oc.prev_blocks()
        od = oc.encode_frame(frames[ti], f18)
        sl = cb.serialize_slice(cfg, oc.aw, oc.ah, f18, od.blocks, prev, od.sao, oc.levels())
        _, want = rc.encode_frame(frames[ti], f18)
        assert sl == want, f"frame {k}: slice bytes differ ({len(sl)} vs {len(want)})"
        mine.append((f18, sl))
    stock = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    head = cb.stream_header(cfg, w, h)
    assert head[:7] == stock[:7] and head[8:] == stock[8:14]
    if b_frames:
        body = b"".join(struct.pack("<I", len(f18) + len(sl)) + f18 + sl for f18, sl in mine)
        assert stock[14:] == body
    else:
        assert join_ip_stream(stock[:14], mine) == stock


def test_serializer_rejects_bad_arguments():
    import ctypes as C
    import chicago_b200 as cb
    n = C.c_uint64(0)
    out = np.zeros(16, np.uint8)
    f18 = b"\0" * 18
    assert cb.lib().evxg_serialize_slice(None, 24, 16, f18, out.ctypes.data, out.ctypes.data, out.ctypes.data,
                                         out.ctypes.data, out.ctypes.data, 16, C.byref(n)) == 1
    blk = np.zeros(28, np.uint8)
    blk[0] = 1   # one intra-default block
    rc = cb.lib().evxg_serialize_slice(None, 16, 16, f18, blk.ctypes.data, np.zeros(28, np.uint8).ctypes.data,
                                       np.zeros(16, np.uint8).ctypes.data, np.zeros(384, np.int16).ctypes.data,
                                       out.ctypes.data, 1, C.byref(n))
    assert rc == 7 and n.value > 1   # EVXG_ERROR_CAPACITY_LIMIT, with the size it needs
