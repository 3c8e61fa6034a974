"""Register report of the sm_100a build (``nvcc -Xptxas -v``, written by
``stda_b200/build.py`` next to the sources): the kernels on the hot path keep
their state in registers (no spill stores or loads) and within the register
budget their launch shapes need."""
import os
import re

import pytest

LOG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                   "stda_b200", "csrc", "ptxas.log")

# kernel -> most registers per thread.  The HBM-bound passes need enough loads
# in flight: half of the SM's 2048 threads resident (65536 / 1024 = 64
# registers), or, for the PT column pass, which issues 2 rows x 4 primaries of
# loads per thread before using them and carries a second (error-bound)
# accumulator per primary, three 256-thread CTAs (85 registers); the
# tensor-core kernel runs one 256-thread CTA per SM.
HOT = {
    "k_tc_gemm_bf16x3": 255,
    "k_ptq_rows": 80,
    "k_ptq_cols": 85,
    "k_charges_tiled": 64,
    "k_diag_screen": 64,
}


def _report():
    if not os.path.exists(LOG):
        pytest.skip("no ptxas report: the library has not been built here")
    text = open(LOG).read()
    out = {}
    for m in re.finditer(r"Compiling entry function '(_Z\w+)' for 'sm_100a'\n(.*?)(?=ptxas info    : "
                         r"Compiling entry function|\Z)", text, re.S):
        name, body = m.group(1), m.group(2)
        spill = re.search(r"(\d+) bytes spill stores, (\d+) bytes spill loads", body)
        regs = re.search(r"Used (\d+) registers", body)
        out.setdefault(name, []).append((int(spill.group(1)) if spill else 0,
                                         int(spill.group(2)) if spill else 0,
                                         int(regs.group(1)) if regs else 0))
    return out


def test_hot_kernels_do_not_spill():
    rep = _report()
    for kernel, max_regs in HOT.items():
        hits = [v for name, vals in rep.items() if kernel in name for v in vals]
        assert hits, f"{kernel} missing from the ptxas report"
        for stores, loads, regs in hits:
            assert stores == 0 and loads == 0, (kernel, stores, loads)
            assert 0 < regs <= max_regs, (kernel, regs)
