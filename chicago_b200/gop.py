"""Frame-type / DPB-slot schedule of the EVX3 encoder, for callers that drive
the per-frame C ABI (evxg_encode_frame) themselves, e.g. the benchmark and
batched drivers.  Mirrors evx3_encoder_impl::encode / encode_gop / flush
(reference src/video/evx3enc.cpp:105-414) with the default build constants
EVX_B_FRAME_COUNT 3 and EVX_PERIODIC_INTRA_RATE 3600 (config.h:41, :121), and
its I/P path (EVX_ENABLE_B_FRAMES 0, evx3enc.cpp:137-160: every frame encoded
as it arrives, slots chosen by the frame index); the C++ encoder behind
evxg_encoder_* implements the same logic natively.
"""
from __future__ import annotations

import struct

FRAME_INTRA, FRAME_INTER, FRAME_BIDIR = 0, 1, 2
B_FRAMES, INTRA_RATE = 3, 3600


def pack_frame(ftype, index, quality, display_order, is_reference, dpb_slot, ref_fwd, ref_bwd) -> bytes:
    """The 18-byte evx_frame (reference src/video/common.h:72-87, pack(2))."""
    return struct.pack("<iIHIBBBB", ftype, index, quality, display_order, is_reference, dpb_slot, ref_fwd, ref_bwd)


def unpack_frame(b: bytes) -> dict:
    t, i, q, d, r, s, f, bw = struct.unpack("<iIHIBBBB", bytes(b[:18]))
    return dict(type=t, index=i, quality=q, display_order=d, is_reference=r, dpb_slot=s, ref_fwd=f, ref_bwd=bw)


def quality_to_qp(q: int) -> int:
    """set_quality: user quality 1..31 to the internal QP (evx3enc.cpp:64-82)."""
    q = min(max(int(q), 1), 31)
    return min(q if q <= 16 else q + ((q - 16) ** 2) // 10, 63)


class Schedule:
    """Incremental planner: feed input frame indices, get (input index, frame18)
    in encode order.  b_frames=False plans the I/P build with ref_count DPB
    slots (the frame's slots follow from its index)."""

    def __init__(self, quality: int = 8, b_frames: bool = True, ref_count: int = 4):
        self.qp = quality_to_qp(quality)
        self.b_frames, self.ref_count = b_frames, ref_count
        self.type, self.index, self.doc, self.ip, self.first = FRAME_INTRA, 0, 0, 0, True
        self.reorder = []

    def insert_intra(self):
        self.type = FRAME_INTRA

    def _slot(self, ip):
        return (ip & 0xFFFFFFFF) % 2

    def _gop(self, out):
        r, ip = self.reorder, self.ip
        p_in, p_do = r[-1]
        out.append((p_in, pack_frame(FRAME_INTER, self.index, self.qp, p_do, 1, self._slot(ip), self._slot(ip - 1), 0)))
        self.index += 1
        bc = len(r) - 1
        if bc > 0:
            ref = bc // 2
            out.append((r[ref][0], pack_frame(FRAME_BIDIR, self.index, min(self.qp + 1, 31), r[ref][1], 1, 2,
                                              self._slot(ip - 1), self._slot(ip))))
            self.index += 1
            for bi in range(bc):
                if bi == ref:
                    continue
                fw, bw = (self._slot(ip - 1), 2) if bi < ref else (2, self._slot(ip))
                out.append((r[bi][0], pack_frame(FRAME_BIDIR, self.index, min(self.qp + 2, 31), r[bi][1], 0, 3, fw, bw)))
                self.index += 1
        self.ip += 1
        self.type = FRAME_INTER
        self.reorder = []

    def push(self, t: int):
        out = []
        if not self.b_frames:   # evx3enc.cpp:137-160
            R, i = self.ref_count, self.index
            out.append((t, pack_frame(self.type, i, self.qp, self.doc, 1, i % R, (i + R - 1) % R, 0)))
            self.doc += 1
            self.type = FRAME_INTRA if (i + 1) % INTRA_RATE == 0 else FRAME_INTER
            self.index += 1
            return out
        if self.doc > 0 and self.doc % INTRA_RATE == 0:
            if self.reorder:
                self._gop(out)
            self.type, self.ip = FRAME_INTRA, 0
        as_intra = self.type == FRAME_INTRA
        if as_intra and not self.first and self.reorder:
            self._gop(out)
            self.ip = 0
        self.reorder.append((t, self.doc))
        self.doc += 1
        if self.first or as_intra:
            self.first = False
            i_in, i_do = self.reorder[0]
            out.append((i_in, pack_frame(FRAME_INTRA, self.index, self.qp, i_do, 1, self._slot(self.ip), 0, 0)))
            self.ip += 1
            self.type = FRAME_INTER
            self.index += 1
            self.reorder = []
        elif len(self.reorder) == B_FRAMES + 1:
            self._gop(out)
        return out

    def flush(self):
        out = []
        if len(self.reorder) == 1:
            p_in, p_do = self.reorder[0]
            out.append((p_in, pack_frame(FRAME_INTER, self.index, self.qp, p_do, 1, self._slot(self.ip),
                                         self._slot(self.ip - 1), 0)))
            self.index += 1
            self.ip += 1
        elif self.reorder:
            self._gop(out)
        self.reorder = []
        return out


CONFIG_GOP = {"default": (True, 4), "ip1": (False, 2), "ip3": (False, 4)}


def plan(n_frames: int, quality: int = 8, intra_at=(), cfg: str = "default"):
    """Whole-sequence schedule of the build cfg names ("default", "ip1",
    "ip3"); insert_intra() is called before each index in intra_at."""
    b_frames, ref_count = CONFIG_GOP[cfg]
    s, out = Schedule(quality, b_frames, ref_count), []
    for t in range(n_frames):
        if t in intra_at:
            s.insert_intra()
        out += s.push(t)
    return out + s.flush()
