"""The reference-side binding (oracle/evxg_binding.cpp) on the GPU.

oracle/Makefile links the reference library without its encode.cpp and with
engine_encode_frame taken from the binding, which runs this library's GPU
pipeline and host entropy coder.  The reference's own, unmodified encoder
(create_encoder / set_quality / insert_intra / encode / flush, evx3enc.cpp)
drives it; its stream must equal the unmodified reference's byte for byte
(but the header's padding byte, which the reference leaves uninitialised),
for the default build and the I/P build with three references."""
import os

import pytest

from chicago_b200.synth import generate
from oracle_py import HERE, REF_SO, REF_VARIANTS, Ref

pytestmark = pytest.mark.gpu

GPU_SO = {"default": os.path.join(HERE, "_ref", "libevxref_gpu.so"),
          "ip3": os.path.join(HERE, "_ref", "libevxref_gpu_ip3.so")}


@pytest.mark.parametrize("cfg", ["default", "ip3"])
def test_reference_encoder_on_the_gpu_engine_gives_the_stock_stream(cfg):
    import chicago_b200 as cb
    cb.lib()   # the binding resolves the library's entry points from the same libevxg.so
    stock_so = REF_SO if cfg == "default" else REF_VARIANTS[cfg][0]
    for p in (stock_so, GPU_SO[cfg]):
        if not os.path.exists(p):
            pytest.skip(f"{p} not built (make -C oracle ref variants binding)")
    w, h, T, q = 176, 144, 10, 8
    frames = generate(w, h, T, seed=17, vmax=8.0)
    stock = Ref(stock_so).encode_stream(frames, quality=q, intra_at=(6,))
    gpu = Ref(GPU_SO[cfg]).encode_stream(frames, quality=q, intra_at=(6,))
    assert len(gpu) == len(stock)
    assert gpu[:7] == stock[:7] and gpu[8:] == stock[8:]
    again = Ref(GPU_SO[cfg]).encode_stream(frames[:4], quality=16)   # a new session on a fresh encoder
    assert again[8:] == Ref(stock_so).encode_stream(frames[:4], quality=16)[8:]
