"""GPU parity: the general decoder's picture pass over batches of intra
pictures with coding trees of 4x4..128x128 blocks (vvcg_gen_prepare / run /
download): residuals (DCT-2 / implicit and explicit MTS / LFNST / transform
skip / BDPCM / dependent quantisation), intra reconstruction in dependency
levels (ISP, MRL, CCLM, chroma of split nodes), deblocking over the
transform-block maps, SAO and ALF, against the oracle's composition of its
restatements in decode order (oracle.general_picture), bit-exact on every
visible sample."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [
    dict(vis_w=200, vis_h=120, ctu=64, bd=10, qp=32, seed=1),
    dict(vis_w=128, vis_h=128, ctu=32, bd=8, qp=27, seed=2, dep_quant=True),
    dict(vis_w=256, vis_h=136, ctu=128, bd=12, qp=37, seed=3),
    dict(vis_w=96, vis_h=64, ctu=16, bd=10, qp=22, seed=4),
]


def _parts(synth, specs, tools=None):
    parts = []
    for s in specs:
        s = dict(s)
        if tools is not None:
            s["tools"] = tools
        parts.append(synth.random_general_picture(**s))
    return parts


def _check(orc, parts, got):
    for k, (part, g) in enumerate(zip(parts, got)):
        want = orc.general_picture(*part)
        for c in range(3):
            diff = np.argwhere(g[c] != want[c])
            assert diff.size == 0, f"picture {k} plane {c}: {len(diff)} samples differ, first {diff[:3].tolist()}"


@pytest.mark.parametrize("tools", [0, 2, 2 | 4, 2 | 4 | 8])
def test_general_batch_matches_oracle(ctx, pkg, orc, tools):
    from rustmpeg_next_b200 import synth

    parts = _parts(synth, SPECS, tools)
    got = ctx.decode_general(pkg.GenBatch(**synth.general_batch(parts)))
    assert ctx.gen_levels > 1
    _check(orc, parts, got)


def test_graph_replay_and_reruns_equal_the_first_run(ctx, pkg, orc):
    from rustmpeg_next_b200 import synth

    parts = _parts(synth, SPECS[:3])
    batch = pkg.GenBatch(**synth.general_batch(parts))
    first = ctx.decode_general(batch)
    ctx.gen_prepare(batch)
    for graph in (True, True, False):
        ctx.gen_run(graph)
    again = ctx.gen_download(batch.output_planes())
    for a, b in zip(first, again):
        for c in range(3):
            assert (a[c] == b[c]).all()
    _check(orc, parts, first)


def test_many_small_pictures_in_one_batch(ctx, pkg, orc):
    """Pictures of one batch share the levels: a level launch mixes groups of
    every picture."""
    from rustmpeg_next_b200 import synth

    specs = [dict(vis_w=64 + 16 * (k % 5), vis_h=48 + 8 * (k % 3), ctu=32, bd=8 + 2 * (k % 2), qp=22 + k,
                  seed=100 + k) for k in range(12)]
    parts = _parts(synth, specs)
    got = ctx.decode_general(pkg.GenBatch(**synth.general_batch(parts)))
    _check(orc, parts, got)


def test_invalid_general_batches_are_rejected(ctx, pkg):
    from rustmpeg_next_b200 import synth

    parts = _parts(synth, SPECS[:1])
    good = synth.general_batch(parts)
    cases = []
    b = dict(good, tbs=good["tbs"].copy())
    b["tbs"]["pred"]["out_off"][1] = b["tbs"]["pred"]["out_off"][0]  # two blocks on one slot range
    b["tbs"]["tu"]["out_off"][1] = b["tbs"]["tu"]["out_off"][0]
    cases.append(b)
    b = dict(good, tbs=good["tbs"].copy())
    k = int(np.argmax(b["tbs"]["pred"]["comp"] == 0))
    b["tbs"]["pred"]["x"][k] = 4000  # outside the picture
    cases.append(b)
    b = dict(good, tbs=good["tbs"].copy())
    k = int(np.argmax(b["tbs"]["coded"] != 0))
    b["tbs"]["tu"]["log2_w"][k] += 1  # residual record of another size
    cases.append(b)
    b = dict(good, group_first=good["group_first"].copy())
    b["group_first"][-1] = len(good["tbs"]) + 5  # past the blocks
    cases.append(b)
    b = dict(good, pics=good["pics"].copy())
    b["pics"]["ctu_log2"] = 3
    cases.append(b)
    for c in cases:
        with pytest.raises(pkg.InvalidInput):
            ctx.decode_general(pkg.GenBatch(**c))
    got = ctx.decode_general(pkg.GenBatch(**good))  # the context still works
    assert got[0][0].shape == (120, 200)
