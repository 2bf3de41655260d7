"""Extract the reference's normative table literals into tests/golden/tables.json.

Reads the Rust sources of the reference's VVC module (the path below; run it
where the reference tree is mounted) and writes, for every table the
kernels and the oracle use, the flat list of its values in row-major order
together with the file:line of its declaration. tests/test_tables_golden.py
compares rustmpeg-next_b200/csrc/vvc_tables.h and vvc_cabac.h with that file entry by entry,
so a transcription error in the shared header cannot pass the GPU parity
tests unnoticed.

Usage: python tests/golden/make_tables.py [reference root]
"""
from __future__ import annotations

import json
import os
import re
import sys

DEFAULT_ROOT = "/root/reference"
VVC = os.path.join("crates", "rustmpeg-video", "src", "vvc")

# (file, constant) pairs, in the order the golden file lists them.
TABLES = [
    ("dct.rs", "INV_QUANT_SCALES"), ("dct.rs", "INV_QUANT_SCALES_SQRT2"),
    ("dct.rs", "QUANT_SCALES"), ("dct.rs", "QUANT_SCALES_SQRT2"),
    ("dct.rs", "DCT2_2"), ("dct.rs", "DCT2_4"), ("dct.rs", "DCT2_8"), ("dct.rs", "DCT2_16"),
    ("dct.rs", "DCT2_32"), ("dct.rs", "DCT2_64"),
    ("tr_tables.rs", "DST7_4"), ("tr_tables.rs", "DST7_8"), ("tr_tables.rs", "DST7_16"),
    ("tr_tables.rs", "DST7_32"),
    ("tr_tables.rs", "DCT8_4"), ("tr_tables.rs", "DCT8_8"), ("tr_tables.rs", "DCT8_16"),
    ("tr_tables.rs", "DCT8_32"),
    ("tr_tables.rs", "LFNST_8X8"), ("tr_tables.rs", "LFNST_4X4"), ("tr_tables.rs", "LFNST_LUT"),
    ("filter.rs", "DBF_TC_TABLE"), ("filter.rs", "DBF_BETA_TABLE"),
    ("filter.rs", "ALF_FIXED_FILTER_COEFF"), ("filter.rs", "ALF_CLASS_TO_FILTER_MAPPING"),
    ("filter.rs", "ALF_CLIP_VALS_8BIT"), ("filter.rs", "ALF_CLIP_VALS_10BIT"),
    ("filter.rs", "ALF_CLIP_VALS_12BIT"), ("filter.rs", "ALF_TRANSPOSE_PERM"),
    ("inter.rs", "LUMA_FILTER_8TAP"), ("inter.rs", "LUMA_ALT_HPEL_FILTER_8TAP"),
    ("inter.rs", "AFFINE_LUMA_FILTER_8TAP"), ("inter.rs", "BCW_WEIGHTS"),
    ("inter.rs", "GEO_DIS"), ("inter.rs", "GEO_ANGLE_TO_MASK"), ("inter.rs", "BILINEAR_FILTER_PREC4"),
    ("predict.rs", "ANG_TABLE"), ("predict.rs", "INV_ANG_TABLE"), ("predict.rs", "INTRA_FILTER_THRESHOLD"),
    ("predict.rs", "CHROMA_FILTER_4TAP"), ("predict.rs", "CCLM_DIV_SIG_TABLE"),
    ("predict.rs", "MIP_MATRIX_4X4"), ("predict.rs", "MIP_MATRIX_8X8"), ("predict.rs", "MIP_MATRIX_16X16"),
    ("cabac.rs", "CTX_INIT_I"), ("cabac.rs", "CTX_INIT_P"), ("cabac.rs", "CTX_INIT_B"), ("cabac.rs", "RENORM_LPS"),
    ("residual.rs", "PREFIX_CTX"), ("residual.rs", "MIN_IN_GROUP"), ("residual.rs", "GROUP_IDX"),
    ("residual.rs", "GO_RICE_PARS_COEFF"),
]


def _strip_comments(text: str) -> str:
    """Comments blanked out with spaces, so offsets (and line numbers) keep."""
    blank = lambda m: re.sub(r"[^\n]", " ", m.group(0))  # noqa: E731
    text = re.sub(r"/\*.*?\*/", blank, text, flags=re.S)
    return re.sub(r"//[^\n]*", blank, text)


def extract(src: str, name: str):
    """Values of `const NAME: <type> = [ ... ];` in row-major order, its
    declared dimensions and the 1-based line of the declaration."""
    clean = _strip_comments(src)
    m = re.search(r"\bconst\s+" + re.escape(name) + r"\s*:\s*(.*?)=\s*\[", clean, re.S)
    if not m:
        raise KeyError(name)
    names = {k: int(v) for k, v in re.findall(r"\bconst\s+(\w+)\s*:\s*usize\s*=\s*(\d+)\s*;", clean)}
    dims = [int(d) if d.isdigit() else names[d] for d in re.findall(r";\s*(\w+)\s*\]", m.group(1))][::-1]
    tup = re.search(r"\(([^)]*)\)", m.group(1))
    if tup:  # an array of tuples: one more dimension, the tuple's arity
        dims.append(len(tup.group(1).split(",")))
    start = m.end() - 1
    depth = 0
    for i in range(start, len(clean)):
        if clean[i] == "[":
            depth += 1
        elif clean[i] == "]":
            depth -= 1
            if depth == 0:
                body = clean[start:i + 1]
                break
    else:
        raise ValueError(f"{name}: unterminated literal")
    vals = [int(v) for v in re.findall(r"-?\d+", body)]
    n = 1
    for d in dims:
        n *= d
    if n != len(vals):
        raise ValueError(f"{name}: {len(vals)} values for dimensions {dims}")
    line = src.count("\n", 0, m.start()) + 1
    return vals, dims, line


def context_offsets(src: str):
    """The first context of every syntax element's set: the constants of
    cabac.rs's `pub mod ctx`, name -> value, and the line of the module."""
    clean = _strip_comments(src)
    start = clean.index("pub mod ctx")
    depth, i = 0, clean.index("{", start)
    for j in range(i, len(clean)):
        depth += clean[j] == "{"
        depth -= clean[j] == "}"
        if depth == 0:
            break
    body = clean[i:j]
    vals = {k: int(v) for k, v in re.findall(r"pub\s+const\s+(\w+)\s*:\s*usize\s*=\s*(\d+)\s*;", body)}
    return vals, src.count("\n", 0, start) + 1


def main(root: str = DEFAULT_ROOT) -> str:
    out = {"_source": "table literals of crates/rustmpeg-video/src/vvc/*.rs of the reference, "
                      "extracted by tests/golden/make_tables.py"}
    cache = {}
    for fname, name in TABLES:
        if fname not in cache:
            cache[fname] = open(os.path.join(root, VVC, fname)).read()
        vals, dims, line = extract(cache[fname], name)
        out[name] = {"at": f"V/{fname}:{line}", "dims": dims, "values": vals}
    offs, line = context_offsets(cache["cabac.rs"])
    out["_ctx_offsets"] = {"at": f"V/cabac.rs:{line}", "values": offs}
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tables.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    return dst


if __name__ == "__main__":
    print(main(sys.argv[1] if len(sys.argv) > 1 else DEFAULT_ROOT))
