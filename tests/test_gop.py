"""GOP / DPB-slot schedule of the reference encoder (src/video/evx3enc.cpp:105-414,
common.cpp:256-283), restated; slot KATs from tests/test_codec_roundtrip.cpp:13-32."""
from oracle_py import FRAME_BIDIR, FRAME_INTER, FRAME_INTRA, plan_gop, quality_to_qp, unpack_frame


def test_ip_slots_cycle_and_b_slots():
    plan = [unpack_frame(f) for _, f in plan_gop(17, quality=8)]
    ip = [f["dpb_slot"] for f in plan if f["type"] != FRAME_BIDIR]
    assert ip == [0, 1, 0, 1, 0]
    refb = [f for f in plan if f["type"] == FRAME_BIDIR and f["is_reference"]]
    nonref = [f for f in plan if f["type"] == FRAME_BIDIR and not f["is_reference"]]
    assert refb and all(f["dpb_slot"] == 2 for f in refb)
    assert nonref and all(f["dpb_slot"] == 3 for f in nonref)
    assert [f["index"] for f in plan] == list(range(len(plan)))


def test_encode_order_and_quality_offsets():
    plan = plan_gop(9, quality=8)
    assert [t for t, _ in plan] == [0, 4, 2, 1, 3, 8, 6, 5, 7]
    fr = [unpack_frame(f) for _, f in plan]
    assert [f["type"] for f in fr[:5]] == [FRAME_INTRA, FRAME_INTER, FRAME_BIDIR, FRAME_BIDIR, FRAME_BIDIR]
    assert [f["quality"] for f in fr[:5]] == [8, 8, 9, 10, 10]


def test_insert_intra_flushes_gop():
    fr = [(t, unpack_frame(f)) for t, f in plan_gop(8, quality=8, intra_at=(3,))]
    assert [t for t, _ in fr] == [0, 2, 1, 3, 7, 5, 4, 6]
    assert fr[3][1]["type"] == FRAME_INTRA and fr[3][1]["dpb_slot"] == 0


def test_quality_mapping():
    assert [quality_to_qp(q) for q in (0, 1, 8, 16, 17, 31, 40)] == [1, 1, 8, 16, 17, 53, 53]


def test_product_schedule_equals_restatement():
    from chicago_b200.gop import plan
    for T, q, cuts in [(1, 8, ()), (2, 8, ()), (9, 8, ()), (13, 20, (5,)), (30, 4, (3, 4, 17)), (120, 8, (60,))]:
        assert plan(T, q, cuts) == plan_gop(T, quality=q, intra_at=cuts)
