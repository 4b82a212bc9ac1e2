"""Regenerate the golden fixtures from the UNMODIFIED reference encoder.

Run in a container that has the reference tree (it needs oracle/_ref):
    make -C oracle ref && python tests/golden/make_golden.py

Each fixture holds the seeded RGB24 input, the frame descriptors the
reference's GOP logic chose, every stage of every frame as the reference
produced it (converted source, block table, levels, reconstruction before and
after deblocking, SAO table, final reconstruction) and the stock encoder's
.evx stream.  The GPU box has no reference tree; tests read these files.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from chicago_b200.synth import generate  # noqa: E402
from oracle_py import Ref, plan_gop  # noqa: E402

CASES = {
    "pan_q8_64x48": dict(w=64, h=48, T=6, q=8, vmax=6.0, intra_at=()),
    "crop_q4_cut_100x60": dict(w=100, h=60, T=9, q=4, vmax=12.0, intra_at=(5,)),
    "tiny_q20_32x16": dict(w=32, h=16, T=5, q=20, vmax=2.0, intra_at=()),
}


def make(name, w, h, T, q, vmax, intra_at):
    ref = Ref()
    frames = generate(w, h, T, seed=w * 7 + h, vmax=vmax)
    plan = plan_gop(T, quality=q, intra_at=intra_at)
    stream = ref.encode_stream(frames, quality=q, intra_at=intra_at)
    ctx = ref.context(w, h)
    out = dict(frames=frames, order=np.array([t for t, _ in plan]),
               frame18=np.frombuffer(b"".join(f for _, f in plan), np.uint8).reshape(-1, 18),
               stream=np.frombuffer(stream, np.uint8), quality=q)
    stages = {k: [] for k in ("src", "blocks", "levels", "recon", "deblock", "sao", "final")}
    for t, f18 in plan:
        d, _ = ctx.encode_frame(frames[t], f18)
        for k in stages:
            stages[k].append(getattr(d, k))
    for k, v in stages.items():
        out[k] = np.stack(v)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)


if __name__ == "__main__":
    for n, c in CASES.items():
        make(n, **c)
        print("wrote", n)
