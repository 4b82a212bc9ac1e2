"""Pins the oracle restatement to the unmodified reference library built from
its own sources (oracle/_ref): every stage of every frame must be identical,
and the planner-driven staged reference must reproduce the stock encoder's
.evx stream byte for byte (which also pins the GOP planner)."""
import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import compare_blocks, plan_gop, split_stream, unpack_frame

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
