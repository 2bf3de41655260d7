"""CPU: the committed strict-profile slice data (tests/golden/
strict_streams_1080p.npz, made by tests/golden/make_strict_streams.py from
the oracle's restatement of the reference's strict encoder and CABAC
writer) parses with the library's host parser, dense and sparse, on one
and on several threads into the same records, and the oracle's
decode_picture of the parsed records reproduces the encoder's
reconstruction hashed in the fixture."""
import hashlib
import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "strict_streams_1080p.npz")


def load_streams():
    z = np.load(GOLD)
    data, offs = z["data"], z["offsets"]
    w, h = int(z["width"]), int(z["height"])
    streams = [(data[offs[i]:offs[i + 1]].tobytes(), w, h, int(z["qp"][i])) for i in range(len(offs) - 1)]
    return streams, [str(s) for s in z["sha256"]]


def test_fixture_parses_and_decodes_to_the_encoder_reconstruction(pkg, orc):
    streams, hashes = load_streams()
    pics, cus, levels, used = pkg.parse_strict(streams, threads=8)
    _, cus1, levels1, _ = pkg.parse_strict(streams[:3], threads=1)
    assert (cus1 == cus[:len(cus1)]).all()
    per = (streams[0][1] // 32) * (streams[0][2] // 32)
    for i in (0, 5, 10, 15):  # one picture per QP
        c = cus[i * per:(i + 1) * per]
        dec = orc.strict_decode(c, levels, streams[i][1], streams[i][2], streams[i][3])
        h = hashlib.sha256()
        for p in dec:
            h.update(p.tobytes())
        assert h.hexdigest() == hashes[i], i


def test_sparse_parse_of_the_fixture_carries_the_same_levels(pkg):
    from rustmpeg_next_b200 import synth

    streams, _ = load_streams()
    _, cd, ld, _ = pkg.parse_strict(streams[:4], threads=4)
    ps, cs, ls, used = pkg.parse_strict(streams[:4], sparse=True, threads=4)
    assert int(used.sum()) < int(((cd["cbf"] & 1) != 0).sum()) * 1024
    _, bc, bl = synth.densify(ps, cs, ls)
    for k in range(len(cd)):
        for c, n in ((0, 1024), (1, 256), (2, 256)):
            if cd["level_off"][k, c] >= 0:
                assert (ld[cd["level_off"][k, c]:][:n] == bl[bc["level_off"][k, c]:][:n]).all()
