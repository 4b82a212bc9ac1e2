"""The allocation-free macroblock pass (evxg_mb_pass_noalloc) against the
regular stream path.

That entry point exists for callers that cannot allocate device memory while
encoding -- e.g. a plugin that must take every buffer from its host
application's arena -- so the test hands it buffers it allocated itself
and checks, over two calls in a row (an I frame, then a P frame that reads
the first frame's reconstruction and block table), that the block table and
the level planes it writes are identical to what evxg_encode_frame produces
for the same frame.  Identical is the tolerance of every parity test here.

The file name sorts last so a stop-at-first-failure run has already run
every other test when it gets here.
"""
import ctypes as C

import numpy as np
import pytest

from chicago_b200.gop import plan, unpack_frame
from chicago_b200.synth import generate
from oracle_py import compare_blocks

pytestmark = pytest.mark.gpu


def test_noalloc_mb_pass_matches_stream_path_two_calls():
    import torch
    import chicago_b200 as cb

    w, h = 160, 96
    frames = generate(w, h, 3, seed=21, vmax=6.0)
    sched = plan(3, quality=8)[:2]            # I frame, then the P frame that references it
    st = cb.Stream(w, h)
    n, nblk = st.plane_elems, st.nblk
    dev = torch.device("cuda")
    src = torch.zeros(n, dtype=torch.int16, device=dev)
    dpb = [torch.zeros(n, dtype=torch.int16, device=dev) for _ in range(4)]
    levels = torch.zeros(n, dtype=torch.int16, device=dev)
    blocks = torch.zeros(nblk * 28, dtype=torch.uint8, device=dev)
    prev = torch.zeros(nblk * 28, dtype=torch.uint8, device=dev)
    dpb_ptrs = (C.c_void_p * 4)(*[t.data_ptr() for t in dpb])
    state_dpb = [np.zeros(n, np.int16) for _ in range(4)]   # stream DPB before the frame
    state_lev = np.zeros(n, np.int16)                        # stream levels before the frame
    stream = torch.cuda.current_stream()

    for ti, f18 in sched:
        st.encode_frame(frames[ti], f18)
        tb = st.fetch_tables()
        src.copy_(torch.from_numpy(st.fetch_planes(4)))
        for i in range(4):
            dpb[i].copy_(torch.from_numpy(state_dpb[i]))
        levels.copy_(torch.from_numpy(state_lev))
        prev.copy_(torch.from_numpy(tb["prev_blocks"]))
        blocks.zero_()
        torch.cuda.synchronize()
        rc = cb.lib().evxg_mb_pass_noalloc(st.aw, st.ah, f18, C.c_void_p(src.data_ptr()), dpb_ptrs,
                                           C.c_void_p(levels.data_ptr()), C.c_void_p(blocks.data_ptr()),
                                           C.c_void_p(prev.data_ptr()), C.c_void_p(stream.cuda_stream))
        assert rc == 0, cb.lib().evxg_last_error()
        got_blocks = blocks.cpu().numpy()
        assert not compare_blocks(got_blocks, tb["blocks"]), f"block table differs ({unpack_frame(f18)})"
        assert np.array_equal(levels.cpu().numpy(), tb["levels"]), f"levels differ ({unpack_frame(f18)})"
        state_dpb = [st.fetch_planes(i) for i in range(4)]
        state_lev = tb["levels"]


def test_noalloc_rejects_oversized_frames():
    import chicago_b200 as cb
    from chicago_b200.gop import pack_frame
    f18 = pack_frame(0, 0, 8, 0, 1, 0, 0, 0)
    ptrs = (C.c_void_p * 4)(1, 1, 1, 1)
    rc = cb.lib().evxg_mb_pass_noalloc(64, 16 * 5000, f18, C.c_void_p(1), ptrs, C.c_void_p(1), C.c_void_p(1),
                                       None, None)
    assert rc == 7   # EVXG_ERROR_CAPACITY_LIMIT: more macroblock rows than the fixed scratch holds
