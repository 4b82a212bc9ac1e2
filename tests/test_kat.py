"""Known-answer tests of the reference's own suite, restated against the
oracle's unit entry points (the oracle is the CPU checker of the GPU path).

Sources: tests/test_interp.cpp:79-170, tests/test_motion.cpp:209-453,
tests/test_deblock.cpp:138-160, tests/test_transform.cpp:71-85, :169-207,
tests/test_intra_pred.cpp:62-134 of the reference project."""
import ctypes as C

import numpy as np
import pytest

from oracle_py import BLOCK_DTYPE


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def planes(w, h, fill=None):
    n = w * h + 2 * (w // 2) * (h // 2)
    a = np.zeros(n, np.int16)
    if fill is not None:
        a[:] = fill
    return a


@pytest.mark.parametrize("dx,dy,quarter,val", [(1, 0, 0, 100), (0, 1, 0, 80), (1, 1, 0, 60), (1, 0, 1, 100)])
def test_interp_constant(oracle, dx, dy, quarter, val):
    ref = planes(64, 64, val)
    out = np.zeros(384, np.int16)
    oracle.lib.orc_interpolate(_p(ref), 64, 64, 16, 16, dx, dy, quarter, _p(out))
    assert (out[:256] == val).all()


def test_interp_boundary_clamping(oracle):
    ref = planes(64, 64, 50)
    out = np.zeros(384, np.int16)
    oracle.lib.orc_interpolate(_p(ref), 64, 64, 0, 0, 1, 0, 0, _p(out))
    assert out[0] >= 0
    oracle.lib.orc_interpolate(_p(ref), 64, 64, 48, 48, -1, -1, 0, _p(out))
    assert out[0] >= 0 and (out == 50).all()


def test_interp_ramp_midpoint(oracle):
    ref = planes(64, 64)
    y = ref[:64 * 64].reshape(64, 64)
    y[:] = (np.arange(64) * 4)[None, :]
    out = np.zeros(384, np.int16)
    oracle.lib.orc_interpolate(_p(ref), 64, 64, 16, 16, 1, 0, 0, _p(out))
    left = y[16:32, 16:32].astype(int)
    right = y[16:32, 17:33].astype(int)
    assert np.abs(out[:256].reshape(16, 16) - ((left + right + 1) >> 1)).max() <= 1


def test_hadamard_ones_and_checkerboard(oracle):
    inp = np.ones(16, np.int16)
    out = np.zeros(16, np.int32)
    oracle.lib.orc_hadamard_4x4(_p(inp), 4, _p(out))
    assert out[0] == 16 and (out[1:] == 0).all()
    r, c = np.indices((4, 4))
    inp = np.where((r + c) % 2 == 0, 1, -1).astype(np.int16).ravel()
    oracle.lib.orc_hadamard_4x4(_p(inp), 4, _p(out))
    assert out[0] == 0 and out[5] == 16


def test_satd_kats(oracle):
    j, i = np.indices((16, 16))
    a = ((i + j * 3) % 200).astype(np.int16).ravel()
    assert oracle.lib.orc_satd_16x16(_p(a), 16, _p(a.copy()), 16) == 0
    a = np.full(256, 100, np.int16)
    b = np.full(256, 110, np.int16)
    sad = int(np.abs(a.astype(int) - b).sum())
    assert oracle.lib.orc_satd_16x16(_p(a), 16, _p(b), 16) == sad // 2 == 1280


def _table(entries, mbw, mbh):
    t = np.zeros(mbw * mbh, BLOCK_DTYPE)
    t["block_type"] = 1
    t["intra_mode"] = 7
    for idx, (bt, mx, my) in entries.items():
        t[idx]["block_type"], t[idx]["motion_x"], t[idx]["motion_y"] = bt, mx, my
    return t.view(np.uint8)


def _pred(oracle, table, prev, mbw, idx):
    px, py = C.c_int16(), C.c_int16()
    oracle.lib.orc_mv_predictor(_p(table), None if prev is None else _p(prev), mbw, idx, C.byref(px), C.byref(py))
    return px.value, py.value


def test_mv_predictor_kats(oracle):
    mbw, mbh = 4, 4
    idx = 1 * mbw + 1
    assert _pred(oracle, _table({}, mbw, mbh), None, mbw, idx) == (0, 0)
    assert _pred(oracle, _table({idx - 1: (2, 3, -2)}, mbw, mbh), None, mbw, idx) == (3, -2)
    assert _pred(oracle, _table({idx - mbw: (2, -4, 5)}, mbw, mbh), None, mbw, idx) == (-4, 5)
    t = _table({idx - 1: (2, 1, 10), idx - mbw: (2, 5, 2), idx - mbw + 1: (2, 3, 6)}, mbw, mbh)
    assert _pred(oracle, t, None, mbw, idx) == (3, 6)                 # median of three
    t = _table({idx - 1: (2, 2, 4), idx - mbw: (2, 6, 8)}, mbw, mbh)
    assert _pred(oracle, t, None, mbw, idx) == (4, 6)                 # average of two
    t = _table({idx - 1: (2, 1, 1), idx - mbw: (2, 3, 3), idx - mbw - 1: (2, 7, 7)}, mbw, mbh)
    assert _pred(oracle, t, None, mbw, idx) == (3, 3)                 # top-right falls back to top-left
    assert _pred(oracle, _table({1: (2, 9, 9)}, mbw, mbh), None, mbw, 2) == (9, 9)      # first row: left only
    assert _pred(oracle, _table({0: (2, -6, 4)}, mbw, mbh), None, mbw, mbw) == (-6, 4)  # first column: top only
    prev = _table({idx: (2, 8, -8)}, mbw, mbh)                        # temporal candidate
    assert _pred(oracle, _table({}, mbw, mbh), prev, mbw, idx) == (8, -8)


def test_deblock_strength_kats(oracle):
    left = np.zeros(1, BLOCK_DTYPE)
    right = np.zeros(1, BLOCK_DTYPE)
    left["block_type"] = right["block_type"] = 1
    assert oracle.lib.orc_deblock_strength(0, _p(left), _p(right)) == 1
    right["block_type"] = 0
    assert oracle.lib.orc_deblock_strength(1, _p(left), _p(right)) == 2
    left["block_type"] = right["block_type"] = 4
    assert oracle.lib.orc_deblock_strength(1, _p(left), _p(right)) == 0
    right["block_type"] = 0
    assert oracle.lib.orc_deblock_strength(1, _p(left), _p(right)) == 1


def test_zero_transform(oracle):
    z = np.zeros(64, np.int16)
    out = np.ones(64, np.int16)
    oracle.lib.orc_fdct_8x8(_p(z), 8, _p(out), 8)
    assert (out == 0).all()
    out[:] = 1
    oracle.lib.orc_idct_8x8(_p(z), 8, _p(out), 8)
    assert (out == 0).all()


def test_transform_roundtrip_tolerance(oracle):
    """Ramp 10..73 round-trips within 2 (tests/test_transform.cpp:71-85)."""
    x = (10 + np.arange(64)).astype(np.int16)
    c = np.zeros(64, np.int16)
    r = np.zeros(64, np.int16)
    oracle.lib.orc_fdct_8x8(_p(x), 8, _p(c), 8)
    oracle.lib.orc_idct_8x8(_p(c), 8, _p(r), 8)
    assert np.abs(r.astype(int) - x).max() <= 2


def test_intra_dc_vertical_horizontal(oracle):
    w = h = 64
    rec = planes(w, h)
    y = rec[:w * h].reshape(h, w)
    y[15, 16:32] = 200
    y[16:32, 15] = 100
    out = np.zeros(384, np.int16)
    oracle.lib.orc_intra_predict(0, _p(rec), w, h, 16, 16, _p(out))
    assert out[0] == out[8 * 16 + 8] == out[255] == 150
    y[15, 16:32] = 10 * np.arange(16)
    oracle.lib.orc_intra_predict(1, _p(rec), w, h, 16, 16, _p(out))
    assert (out[:256].reshape(16, 16) == 10 * np.arange(16)[None, :]).all()
    y[16:32, 15] = 10 * np.arange(16)
    oracle.lib.orc_intra_predict(2, _p(rec), w, h, 16, 16, _p(out))
    assert (out[:256].reshape(16, 16) == 10 * np.arange(16)[:, None]).all()
    rec[:] = 0
    y[0:16, 15] = 200
    oracle.lib.orc_intra_predict(0, _p(rec), w, h, 16, 0, _p(out))
    assert out[0] == 200
    rec[:] = 0
    y[15, 0:16] = 200
    oracle.lib.orc_intra_predict(0, _p(rec), w, h, 0, 16, _p(out))
    assert out[0] == 200
    oracle.lib.orc_intra_predict(0, _p(planes(w, h)), w, h, 0, 0, _p(out))
    assert out[0] == 128


def test_lambda_matches_reference(oracle, ref):
    for q in range(1, 64):
        assert oracle.lib.orc_lambda(q) == ref.lam(q)
