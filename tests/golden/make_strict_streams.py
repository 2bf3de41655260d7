"""Write tests/golden/strict_streams_1080p.npz: strict-profile slice data of
16 pictures of 1920x1088 8-bit 4:2:0 (the full-frame value-noise content,
frames 0..3, scaled to 8 bits, at QP 22 / 27 / 32 / 37), made by the
oracle's restatement of the reference's strict encoder (encode_picture's
decisions, oracle.strict_encode) and its CABAC writer (oracle.strict_write),
with the SHA-256 of each picture's reconstruction (Y, Cb, Cr bytes in that
order). The library's parser and decoder must reproduce those
reconstructions from the slice data alone.

Usage: python tests/golden/make_strict_streams.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
W, H = 1920, 1088
QPS = (22, 27, 32, 37)
FRAMES = 4


def picture(frame):
    from rustmpeg_next_b200 import synth

    y, u, v = synth.value_noise_frame(1920, 1080, 10, frame=frame)
    to8 = lambda a: (a >> 2).astype(np.uint8)  # noqa: E731
    return synth.pad_to(to8(y), W, H), synth.pad_to(to8(u), W // 2, H // 2), synth.pad_to(to8(v), W // 2, H // 2)


def digest(planes):
    h = hashlib.sha256()
    for p in planes:
        h.update(np.ascontiguousarray(p, dtype=np.uint8).tobytes())
    return h.hexdigest()


def main() -> str:
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from conftest import load_pkg

    load_pkg()
    import oracle

    oracle.build()
    data, offs, qps, hashes = [], [0], [], []
    for qp in QPS:
        for f in range(FRAMES):
            y, u, v = picture(f)
            cus, levels, rec = oracle.strict_encode(y, u, v, qp)
            b = oracle.strict_write(cus, levels, W, H, qp)
            data.append(np.frombuffer(b, np.uint8))
            offs.append(offs[-1] + len(b))
            qps.append(qp)
            hashes.append(digest(rec))
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "strict_streams_1080p.npz")
    np.savez_compressed(dst, data=np.concatenate(data), offsets=np.array(offs, np.int64), qp=np.array(qps, np.uint8),
                        width=W, height=H, sha256=np.array(hashes))
    return dst


if __name__ == "__main__":
    print(main())
