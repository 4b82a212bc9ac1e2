"""The container (evxg_muxer / evxg_demuxer) and the tools' packet cutting
against the reference's own evx_muxer / evx_demuxer (src/muxer.cpp, built
from the reference's sources into the test harness) and its encoder tool's
packetisation (tools/evx_encode.cpp:143-275, driven here with raw RGB frames).
Runs on the CPU: nothing here has a device part."""
import os

import numpy as np
import pytest

from chicago_b200.synth import generate
from oracle_py import REF_SO, REF_VARIANTS, Ref

# Offset of the .evx stream header's padding byte inside a one-video-stream
# container (10-byte header, 18-byte descriptor, 16-byte packet header, byte 7
# of the stream header): the reference leaves it uninitialised.
PAD = 10 + 18 + 16 + 7


def reference_for(cfg):
    path = REF_SO if cfg == "default" else REF_VARIANTS[cfg][0]
    if not os.path.exists(path):
        pytest.skip(f"reference build {path} not present")
    return Ref(path)


def random_packets(seed, n=40):
    rng = np.random.default_rng(seed)
    return [(int(t), rng.integers(0, 256, int(rng.integers(1, 5000)), dtype=np.uint8).tobytes())
            for t in np.cumsum(rng.integers(0, 40000, n))]


@pytest.mark.parametrize("with_audio", [False, True])
def test_muxer_writes_the_reference_bytes(tmp_path, with_audio):
    import chicago_b200 as cb
    ref = reference_for("default")
    pk = random_packets(3 + with_audio)
    a, b = str(tmp_path / "ref.evx3"), str(tmp_path / "mine.evx3")
    ref.mux_file(a, 1280, 720, 29.97, pk, with_audio=with_audio)
    m = cb.Muxer(b)
    vid = m.add_video_stream(1280, 720, 29.97)
    if with_audio:
        m.add_audio_stream(48000, 2, 16, 5)
    m.write_header()
    for ts, p in pk:
        m.write_packet(vid, cb.STREAM_TYPE_VIDEO, ts, p)
    m.close()
    assert open(a, "rb").read() == open(b, "rb").read()


def test_demuxers_read_each_other(tmp_path):
    import chicago_b200 as cb
    ref = reference_for("default")
    pk = random_packets(11)
    a, b = str(tmp_path / "ref.evx3"), str(tmp_path / "mine.evx3")
    ref.mux_file(a, 640, 360, 25.0, pk, with_audio=True)
    d = cb.Demuxer(a)
    assert [(s.stream_type, s.stream_id, s.width, s.height) for s in d.streams] == [(0, 0, 640, 360), (1, 1, 0, 0)]
    assert abs(d.streams[0].frame_rate - 25.0) < 1e-6 and d.streams[1].sample_rate == 48000
    assert [(ts, p) for _, _, ts, p in d] == pk
    d.close()
    write = __import__("chicago_b200.tools", fromlist=["write_container"]).write_container
    write(b, 640, 360, 25.0, pk)
    n_streams, got = ref.demux_file(b)
    assert n_streams == 1 and [(ts, p) for _, ts, p in got] == pk


def test_demuxer_rejects_other_files(tmp_path):
    import chicago_b200 as cb
    bad = tmp_path / "bad.evx3"
    bad.write_bytes(b"RIFF0000WAVEfmt ")
    with pytest.raises(cb.EvxgError) as e:
        cb.Demuxer(str(bad))
    assert e.value.code == 8
    trunc = tmp_path / "trunc.evx3"
    ref = reference_for("default")
    ref.mux_file(str(trunc), 64, 48, 30.0, random_packets(5, 3))
    data = trunc.read_bytes()
    trunc.write_bytes(data[:-100])
    with pytest.raises(cb.EvxgError) as e:
        list(cb.Demuxer(str(trunc)))
    assert e.value.code == 12   # EVXG_ERROR_IO_FAILURE: the last payload is short


@pytest.mark.parametrize("cfg,q", [("default", 8), ("default", 16), ("ip3", 8), ("ip1", 4)])
def test_packets_cut_like_the_reference_tool(tmp_path, cfg, q):
    """The tools' packet cutting and timestamps over the reference encoder's
    own per-call outputs give the reference tool's container byte for byte."""
    import chicago_b200 as cb
    from chicago_b200.tools import Packetizer, write_container
    ref = reference_for(cfg)
    w, h, fps = 96, 64, 29.97
    frames = generate(w, h, 9, seed=q, vmax=6.0)
    chunks = ref.encode_stream(frames, quality=q, chunks=True)
    pk = Packetizer(bool(cb.CONFIGS[cfg][0]), fps)
    for c in chunks[:-1]:
        pk.output(c)
    if cb.CONFIGS[cfg][0]:
        pk.flushed(chunks[-1])
    a, b = str(tmp_path / "ref.evx3"), str(tmp_path / "mine.evx3")
    ref.encode_container(a, frames, fps, q)
    write_container(b, w, h, fps, pk.packets)
    ra, rb = open(a, "rb").read(), open(b, "rb").read()
    assert len(ra) == len(rb) and ra[:PAD] == rb[:PAD] and ra[PAD + 1:] == rb[PAD + 1:]
