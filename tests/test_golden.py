"""Committed fixtures produced by the unmodified reference encoder
(tests/golden/make_golden.py): the oracle (CPU) and the CUDA path (GPU) must
reproduce every stage of every frame they expose."""
import glob
import os

import numpy as np
import pytest

from oracle_py import BLOCK_DTYPE, BLOCK_FIELDS, split_stream, unpack_frame

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
IDS = [os.path.basename(p)[:-4] for p in FIXTURES]
STAGES = ("src", "levels", "recon", "deblock", "sao", "final")


def load(path):
    z = np.load(path)
    return {k: z[k] for k in z.files}


def same_blocks(a, b):
    ta, tb = a.view(BLOCK_DTYPE), b.view(BLOCK_DTYPE)
    return all(np.array_equal(ta[f], tb[f]) for f in BLOCK_FIELDS)


def test_fixtures_present():
    assert len(FIXTURES) >= 3


@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_oracle_reproduces_golden(oracle, path):
    g = load(path)
    T, H, W, _ = g["frames"].shape
    ctx = oracle.context(W, H)
    for k, t in enumerate(g["order"]):
        d = ctx.encode_frame(g["frames"][t], g["frame18"][k].tobytes())
        assert same_blocks(d.blocks, g["blocks"][k]), f"blocks frame {k}"
        for s in STAGES:
            assert np.array_equal(getattr(d, s), g[s][k]), f"{s} frame {k}"


def test_golden_streams_are_self_consistent():
    for path in FIXTURES:
        g = load(path)
        _, payloads = split_stream(g["stream"].tobytes())
        assert len(payloads) == len(g["order"])
        for k, p in enumerate(payloads):
            assert p[:18] == g["frame18"][k].tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("path", FIXTURES, ids=IDS)
def test_gpu_reproduces_golden(path):
    import chicago_b200 as cb
    g = load(path)
    T, H, W, _ = g["frames"].shape
    st = cb.Stream(W, H)
    for k, t in enumerate(g["order"]):
        f18 = g["frame18"][k].tobytes()
        st.encode_frame(g["frames"][t], f18)
        tb = st.fetch_tables()
        assert same_blocks(tb["blocks"], g["blocks"][k]), f"blocks frame {k}"
        assert np.array_equal(tb["levels"], g["levels"][k]), f"levels frame {k}"
        assert np.array_equal(tb["sao"], g["sao"][k]), f"sao frame {k}"
        assert np.array_equal(st.fetch_planes(4), g["src"][k]), f"src frame {k}"
        assert np.array_equal(st.fetch_planes(unpack_frame(f18)["dpb_slot"]), g["final"][k]), f"final frame {k}"
