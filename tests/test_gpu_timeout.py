"""Failure detection on the GPU, without a GPU fault.

Every device-side wait of the encoder's kernels on other CTAs (wavefront
progress, the cluster form's hand-over, the SAO merge and raster-order
application) is bounded: when it runs out it sets the stream's error word and
every CTA runs to its end, so the context stays usable.  Here the bound is set
to one nanosecond, so that the waits of a multi-row frame (row r waits for
row r-1) run out; the host must see EVXG_ERROR_OPERATION_TIMEDOUT, and after
the stream is reset and the bound restored the same sequence must again match
the oracle bit for bit -- from the stream path in both macroblock-pass forms,
a batched tick and the allocation-free pass."""
import ctypes as C

import numpy as np
import pytest

from chicago_b200.gop import plan, unpack_frame
from chicago_b200.synth import generate
from oracle_py import compare_blocks

pytestmark = pytest.mark.gpu

TIMEDOUT = 9          # EVXG_ERROR_OPERATION_TIMEDOUT (evx_status EVX_ERROR_OPERATION_TIMEDOUT)
NORMAL_NS = 5_000_000_000


def check_against_oracle(oracle, st, frames, sched, w, h):
    oc = oracle.context(w, h)
    for k, (ti, f18) in enumerate(sched):
        od = oc.encode_frame(frames[ti], f18)
        st.encode_frame(frames[ti], f18)
        tb = st.fetch_tables()
        assert not compare_blocks(tb["blocks"], od.blocks), f"frame {k}: block table"
        assert np.array_equal(tb["levels"], od.levels), f"frame {k}: levels"
        assert np.array_equal(tb["sao"], od.sao), f"frame {k}: SAO table"
        assert np.array_equal(st.fetch_planes(unpack_frame(f18)["dpb_slot"]), od.final), f"frame {k}: recon"


@pytest.mark.parametrize("form", ["cluster", "single"])
def test_stream_wait_times_out_then_recovers(oracle, form):
    import chicago_b200 as cb
    w, h = 320, 192                       # 12 macroblock rows of 20
    frames = generate(w, h, 4, seed=31, vmax=6.0)
    sched = plan(4, quality=8)             # I, P, reference B, B
    st = cb.Stream(w, h)
    st.mb_form = cb.MB_FORM_CLUSTER if form == "cluster" else cb.MB_FORM_SINGLE
    st.set_timeout_ns(1)
    for ti, f18 in sched[:2]:              # an I frame, then a P frame: both time out
        st.encode_frame(frames[ti], f18)
        with pytest.raises(cb.EvxgError) as e:
            st.sync()
        assert e.value.code == TIMEDOUT
        st.sync()                          # the error word was collected and cleared
    with pytest.raises(cb.EvxgError):
        st.set_timeout_ns(0)
    st.set_timeout_ns(NORMAL_NS)
    st.reset()
    check_against_oracle(oracle, st, frames, sched, w, h)


def test_batch_tick_times_out_then_recovers(oracle):
    import chicago_b200 as cb
    sizes = [(160, 96), (96, 64)]
    seqs = [(generate(w, h, 3, seed=40 + k, vmax=5.0), plan(3, quality=8)) for k, (w, h) in enumerate(sizes)]
    streams = [cb.Stream(w, h) for w, h in sizes]
    b = cb.Batch(streams)
    b.set_timeout_ns(1)
    for k in range(len(sizes)):
        b.input(k, 0)[:] = seqs[k][0][seqs[k][1][0][0]]
    b.encode([sq[1][0][1] for sq in seqs], 0)
    with pytest.raises(cb.EvxgError) as e:
        b.wait(0)
    assert e.value.code == TIMEDOUT
    b.close()
    for k, (w, h) in enumerate(sizes):    # every stream of the failed tick starts again
        streams[k].set_timeout_ns(NORMAL_NS)
        streams[k].reset()
        check_against_oracle(oracle, streams[k], seqs[k][0], seqs[k][1], w, h)


def test_noalloc_wait_times_out_then_recovers():
    import torch
    import chicago_b200 as cb
    w, h = 160, 96
    frames = generate(w, h, 1, seed=22, vmax=6.0)
    (ti, f18), = plan(1, quality=8)
    st = cb.Stream(w, h)
    st.encode_frame(frames[ti], f18)
    want = st.fetch_tables()
    n, nblk = st.plane_elems, st.nblk
    dev = torch.device("cuda")
    src = torch.from_numpy(st.fetch_planes(4)).to(dev)
    dpb = [torch.zeros(n, dtype=torch.int16, device=dev) for _ in range(4)]
    levels = torch.zeros(n, dtype=torch.int16, device=dev)
    blocks = torch.zeros(nblk * 28, dtype=torch.uint8, device=dev)
    ptrs = (C.c_void_p * 4)(*[t.data_ptr() for t in dpb])
    L = cb.lib()
    sp = torch.cuda.current_stream().cuda_stream

    def run():
        for t in dpb + [levels, blocks]:
            t.zero_()
        torch.cuda.synchronize()
        return L.evxg_mb_pass_noalloc(st.aw, st.ah, f18, C.c_void_p(src.data_ptr()), ptrs, C.c_void_p(levels.data_ptr()),
                                      C.c_void_p(blocks.data_ptr()), None, C.c_void_p(sp))
    try:
        assert L.evxg_mb_pass_noalloc_set_timeout_ns(1) == 0
        assert run() == TIMEDOUT
        assert b"timeout" in L.evxg_last_error()
    finally:
        assert L.evxg_mb_pass_noalloc_set_timeout_ns(NORMAL_NS) == 0
    assert run() == 0, L.evxg_last_error()
    assert not compare_blocks(blocks.cpu().numpy(), want["blocks"])
    assert np.array_equal(levels.cpu().numpy(), want["levels"])
