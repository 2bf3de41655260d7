"""GPU parity at the full-frame configuration: 1920x1080 (coded 1920x1088)
10-bit 4:2:0 value-noise frames encoded by the repo's GPU encoder at QP 22,
27, 32 and 37 (all tools of the frame path: 7-mode intra, CCLM, dependent
quantisation, deblocking), decoded with deblocking, SAO and ALF, every plane
compared bit-exactly with the oracle's restatement of the reference decoder.

Also: the GPU encoder's records for these pictures equal the oracle
encoder's, and a batch whose CTU-row queue is several times deeper than the
wavefront's resident warps decodes bit-exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

QPS = (22, 27, 32, 37)
SEED = 0x5EED0000


@pytest.fixture(scope="module")
def workload(ctx, pkg):
    from rustmpeg_next_b200 import synth

    return synth.encoded_workload(ctx, 4, QPS, SEED)  # 16 pictures, 4 per QP


def _picture_records(pics, cus, levels, ctus, i):
    p = pics[i]
    n = (int(p["width"]) // 32) * (int(p["height"]) // 32)
    nc = (int(p["width"]) >> int(p["ctu_log2"])) * (int(p["height"]) >> int(p["ctu_log2"]))
    c = cus[int(p["cu_offset"]):][:n]
    return p, c, ctus[int(p["ctu_offset"]):][:nc]


def test_1080p_encoded_batch_bit_exact(ctx, pkg, orc, workload):
    pics, cus, levels, ctus, aps = workload
    assert len(pics) == 16 and sorted(set(int(q) for q in pics["slice_qp"])) == list(QPS)
    out = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus, aps))
    for i in range(len(pics)):
        p, c, t = _picture_records(pics, cus, levels, ctus, i)
        rc, ref = orc.recon_frame(p, c, levels, t, aps[0])
        assert rc == 0
        for k in range(3):
            h, w = out[i][k].shape
            diff = np.argwhere(out[i][k] != ref[k][:h, :w])
            assert diff.size == 0, f"picture {i} (QP {int(p['slice_qp'])}) plane {k}: {len(diff)} samples differ"


@pytest.mark.parametrize("index", [1, 14])
def test_gpu_encoder_records_equal_oracle_encoder_at_1080p(pkg, orc, workload, index):
    from rustmpeg_next_b200 import synth

    pics, cus, levels, ctus, _ = workload
    p, c, t = _picture_records(pics, cus, levels, ctus, index)
    po, co, lo, to = synth.oracle_workload_picture(orc, index, 4, QPS, SEED)
    for f in ("luma_mode", "chroma_mode", "cbf"):
        assert np.array_equal(c[f], co[f]), f
    assert np.array_equal(t, to)
    for k in range(len(c)):
        for comp, n in ((0, 1024), (1, 256), (2, 256)):
            a, b = int(c["level_off"][k, comp]), int(co["level_off"][k, comp])
            assert (a < 0) == (b < 0)
            if a >= 0:
                assert np.array_equal(levels[a:a + n], lo[b:b + n]), (k, comp)


def test_deep_row_queue_bit_exact(ctx, pkg, orc):
    """512 pictures of 8 CTU rows: 4096 rows in the wavefront's queue, more
    than the resident warps, so rows of later pictures wait for warps that
    finished earlier pictures."""
    from rustmpeg_next_b200 import synth

    spec = [dict(width=256, height=256, bit_depth=10, chroma_format=1, ctu_log2=5, qp=22 + (i % 16))
            for i in range(512)]
    pics, cus, levels, ctus, aps = synth.random_records(
        spec, seed=77, tools=pkg.TOOL_DEP_QUANT | pkg.TOOL_DEBLOCK | pkg.TOOL_SAO | pkg.TOOL_ALF, alf_aps=True)
    out = ctx.decode_batch(pkg.Batch(pics, cus, levels, ctus, aps))
    for i in range(0, len(pics), 7):
        p, c, t = _picture_records(pics, cus, levels, ctus, i)
        rc, ref = orc.recon_frame(p, c, levels, t, aps[0])
        assert rc == 0
        for k in range(3):
            assert np.array_equal(out[i][k], ref[k]), (i, k)
