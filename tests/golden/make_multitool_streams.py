"""Write tests/golden/multitool_streams.npz: slice data of the multi-tool
stream (the reference's VvcMultiToolEncoder with default slice options: an
IDR picture, then P pictures predicting from the picture before), made by the
oracle's restatement of its encoders (encode_picture_multitool,
encode_inter_picture) and of their CABAC writes, with the SHA-256 of each
picture's reconstruction (Y, Cb, Cr bytes in that order):

- "small": the small-picture configuration, 64x64 8-bit 4:2:0, frames 0..2
  (ramp + noise + a moving square) at QP 26: I P P;
- "hd": four streams of 1920x1088 8-bit 4:2:0 (the full-frame value-noise
  content, frames 0..3 scaled to 8 bits, stream k at QP 22 / 27 / 32 / 37):
  I P P P each.

The library's parser and decoder must reproduce every reconstruction from
the slice data alone.

Usage: python tests/golden/make_multitool_streams.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
HD_W, HD_H = 1920, 1088
HD_QPS = (22, 27, 32, 37)
HD_FRAMES = 4


def hd_picture(frame):
    from rustmpeg_next_b200 import synth

    y, u, v = synth.value_noise_frame(1920, 1080, 10, frame=frame)
    to8 = lambda a: (a >> 2).astype(np.uint8)  # noqa: E731
    return (synth.pad_to(to8(y), HD_W, HD_H), synth.pad_to(to8(u), HD_W // 2, HD_H // 2),
            synth.pad_to(to8(v), HD_W // 2, HD_H // 2))


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
    from rustmpeg_next_b200 import synth

    oracle.build()
    out = {}
    sets = [("small", [[synth.config1_frame(f) for f in range(3)]], [26], 64, 64)]
    hd_frames = [hd_picture(f) for f in range(HD_FRAMES)]
    sets.append(("hd", [hd_frames] * len(HD_QPS), list(HD_QPS), HD_W, HD_H))
    for name, streams, qps, w, h in sets:
        data, offs, kinds, sid, qp_of, hashes = [], [0], [], [], [], []
        for k, (frames, qp) in enumerate(zip(streams, qps)):
            for p in oracle.multitool_stream(frames, qp, keyint=len(frames)):
                data.append(np.frombuffer(p["data"], np.uint8))
                offs.append(offs[-1] + len(p["data"]))
                kinds.append(p["kind"])
                sid.append(k)
                qp_of.append(qp)
                hashes.append(digest(p["recon"]))
        out[f"{name}_data"] = np.concatenate(data)
        out[f"{name}_offsets"] = np.array(offs, np.int64)
        out[f"{name}_kind"] = np.array(kinds)
        out[f"{name}_stream"] = np.array(sid, np.int32)
        out[f"{name}_qp"] = np.array(qp_of, np.uint8)
        out[f"{name}_size"] = np.array([w, h], np.int32)
        out[f"{name}_sha256"] = np.array(hashes)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "multitool_streams.npz")
    np.savez_compressed(dst, **out)
    return dst


if __name__ == "__main__":
    print(main())
