"""C-ABI checks that need no GPU: the library builds, loads and exports every
function include/*.h declares; record layouts agree between the header, the
package's numpy dtypes and the oracle's."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            src = open(os.path.join(ROOT, "include", f)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(vvcg_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(pkg):
    pkg.build()
    lib = C.CDLL(pkg.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_context_without_gpu_reports_unavailable(pkg):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pkg.Unavailable):
        pkg.Context(0)


def test_record_layouts_match_the_header(pkg, orc):
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "vvcg.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu\n", sizeof(vvcg_cu_rec), sizeof(vvcg_pic_desc),
         sizeof(vvcg_ctu_filter), sizeof(vvcg_alf_aps), sizeof(vvcg_batch), sizeof(vvcg_mc_block),
         sizeof(vvcg_plane_out));
  printf("%zu %zu %zu %zu %zu\n", offsetof(vvcg_pic_desc, alf_aps), offsetof(vvcg_pic_desc, cu_offset),
         offsetof(vvcg_alf_aps, coeff), offsetof(vvcg_alf_aps, clip_idx), offsetof(vvcg_mc_block, out_offset));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(src, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, src], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    sizes = list(map(int, out))
    assert sizes[:7] == [pkg.CU_DTYPE.itemsize, pkg.PIC_DTYPE.itemsize, pkg.CTU_DTYPE.itemsize,
                         pkg.APS_DTYPE.itemsize, C.sizeof(pkg._Batch), pkg.MC_BLOCK_DTYPE.itemsize,
                         C.sizeof(pkg._PlaneOut)]
    assert sizes[7:] == [pkg.PIC_DTYPE.fields["alf_aps"][1], pkg.PIC_DTYPE.fields["cu_offset"][1],
                         pkg.APS_DTYPE.fields["coeff"][1], pkg.APS_DTYPE.fields["clip_idx"][1],
                         pkg.MC_BLOCK_DTYPE.fields["out_offset"][1]]
    for name in ("CU_DTYPE", "PIC_DTYPE", "CTU_DTYPE", "APS_DTYPE"):
        assert getattr(pkg, name) == getattr(orc, name), name


def test_synthetic_records_are_valid_and_deterministic(pkg, orc):
    from rustmpeg_next_b200 import synth  # noqa: E402

    spec = [dict(width=128, height=64, bit_depth=10, chroma_format=1, ctu_log2=5, qp=27),
            dict(width=64, height=64, bit_depth=8, chroma_format=3, ctu_log2=6, qp=32)]
    a = synth.random_records(spec, seed=3, tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO)
    b = synth.random_records(spec, seed=3, tools=pkg.TOOL_DEBLOCK | pkg.TOOL_SAO)
    for x, y in zip(a[:4], b[:4]):
        assert (x == y).all()
    pics, cus, levels, ctus, _ = a
    for p in pics:
        tb = min(1 << int(p["ctu_log2"]), 32)
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        rec = cus[int(p["cu_offset"]):int(p["cu_offset"]) + n]
        offs = rec["level_off"]
        assert ((offs >= 0) == ((rec["cbf"][:, None] >> np.arange(3)) & 1).astype(bool)).all()
        assert offs.max() < len(levels)
    # the oracle reconstructs them without error
    for p in pics:
        tb = min(1 << int(p["ctu_log2"]), 32)
        n = (int(p["width"]) // tb) * (int(p["height"]) // tb)
        nc = (int(p["width"]) >> int(p["ctu_log2"])) * (int(p["height"]) >> int(p["ctu_log2"]))
        rc, _ = orc.recon_frame(p, cus[int(p["cu_offset"]):][:n], levels,
                                ctus[int(p["ctu_offset"]):][:nc])
        assert rc == 0


def test_value_noise_content_shape_and_range(pkg):
    from rustmpeg_next_b200 import synth

    y, u, v = synth.value_noise_frame(256, 144, 10, frame=2)
    assert y.shape == (144, 256) and u.shape == (72, 128)
    assert y.max() <= 1023 and u.min() >= 384 and u.max() <= 640
    y2, _, _ = synth.value_noise_frame(256, 144, 10, frame=2)
    assert (y == y2).all()


# every record dtype of the package and the header struct it mirrors
RECORDS = {
    "CU_DTYPE": "vvcg_cu_rec", "SAO_DTYPE": "vvcg_sao", "CTU_DTYPE": "vvcg_ctu_filter",
    "PIC_DTYPE": "vvcg_pic_desc", "APS_DTYPE": "vvcg_alf_aps", "MC_BLOCK_DTYPE": "vvcg_mc_block",
    "LMCS_APS_DTYPE": "vvcg_lmcs_aps", "LMCS_TABLES_DTYPE": "vvcg_lmcs_tables", "CRES_DTYPE": "vvcg_cres_rec",
    "ALF_CTU_DTYPE": "vvcg_alf_ctu", "ALF_PARAMS_DTYPE": "vvcg_alf_params",
    "ISR_REQ_DTYPE": "vvcg_intra_search_req", "ISR_RES_DTYPE": "vvcg_intra_search_res",
    "CTU_SEARCH_REQ_DTYPE": "vvcg_ctu_search_req", "CTU_SEARCH_RES_DTYPE": "vvcg_ctu_search_res",
    "MV_CAND_DTYPE": "vvcg_mv_cand", "ME_REQ_DTYPE": "vvcg_me_req", "ME_RES_DTYPE": "vvcg_me_res",
    "SPLIT_REQ_DTYPE": "vvcg_split_req", "GEN_INTRA_REQ_DTYPE": "vvcg_gen_intra_req",
    "DBK_CELL_DTYPE": "vvcg_dbk_cell", "DBK_CCELL_DTYPE": "vvcg_dbk_ccell", "DBK_PARAMS_DTYPE": "vvcg_dbk_params",
    "MIP_REQ_DTYPE": "vvcg_mip_req", "MIP_RES_DTYPE": "vvcg_mip_res", "TXS_REQ_DTYPE": "vvcg_tx_search_req",
    "TXS_RES_DTYPE": "vvcg_tx_search_res", "TU_DTYPE": "vvcg_tu_rec", "CTU_MOTION_DTYPE": "vvcg_ctu_motion",
    "BDOF_REQ_DTYPE": "vvcg_bdof_req", "DMVR_REQ_DTYPE": "vvcg_dmvr_req", "AFFINE_REQ_DTYPE": "vvcg_affine_req",
    "PROF_REQ_DTYPE": "vvcg_prof_req", "CIIP_REQ_DTYPE": "vvcg_ciip_req", "GPM_REQ_DTYPE": "vvcg_gpm_req",
    "GEN_TB_DTYPE": "vvcg_gen_tb", "GEN_PIC_DTYPE": "vvcg_gen_pic",
    "INTER_CU_DTYPE": "vvcg_inter_cu", "P_PIC_DTYPE": "vvcg_p_pic",
    "STREAM_CFG_DTYPE": "vvcg_stream_cfg", "ANNEXB_INFO_DTYPE": "vvcg_annexb_info",
}


def test_every_record_dtype_matches_its_struct_field_by_field(pkg):
    missing = sorted(n for n in dir(pkg) if n.endswith("_DTYPE") and n not in RECORDS)
    assert not missing, f"record dtypes without a layout check: {missing}"
    lines, expect = [], []
    for name, struct in RECORDS.items():
        dt = getattr(pkg, name)
        lines.append(f'  printf("%zu\\n", sizeof({struct}));')
        expect.append(dt.itemsize)
        for field, (_, off) in dt.fields.items():
            lines.append(f'  printf("%zu\\n", offsetof({struct}, {field}));')
            expect.append(off)
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"vvcg.h\"\nint main(void) {\n" + "\n".join(lines) + \
        "\n  return 0;\n}\n"
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(src, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", exe, src], check=True)
        got = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    assert got == expect
