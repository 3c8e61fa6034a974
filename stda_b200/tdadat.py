"""``tda.dat`` writer (the output contract of the sTDA path).

Formats follow ``print_tdadat`` (``stda.f:2235-2265``: header ``NM``/``UV``,
rows above E_thr dropped) and the velocity-corrected variant written by
``apbtrafo`` (``apbtrafo.f:100-243``: header ``NM``/``VELO``, every root).
Rows are ``(i4,F10.4,4f13.6)``: state, eV (x27.21139), f_L, f_V, R_L, R_V.
"""
from __future__ import annotations

import numpy as np

EH2EV_OUT = 27.21139
EH2EV_IN = 27.211385050

# atomic masses by nuclear charge (block.f:24-35); 0 where the table has none
_AMS = {1: 1.00790, 2: 4.00260, 3: 6.94000, 4: 9.01218, 5: 10.81000, 6: 12.01100, 7: 14.00670,
        8: 15.99940, 9: 18.99840, 10: 20.17900, 11: 22.98977, 12: 24.30500, 13: 26.98154,
        14: 28.08550, 15: 30.97376, 16: 32.06000, 17: 35.45300, 18: 39.94800}


def molecular_mass(Z) -> float:
    return float(sum(_AMS.get(int(round(z)), 0.0) for z in Z))


def tda_dat(sol, kw) -> str:
    velo = (not kw.rpa) and kw.velcorr
    thr = kw.e_thr_ev / EH2EV_IN
    lines = [" NM", " VELO" if velo else " UV", " MMASS", f"   {sol.xmolw:.15f}     ",
             " LFAKTOR", "  0.5", " RFAKTOR", "  1.0", " WIDTH", "  0.20", " SHIFT", "  0.00",
             " DATXY"]
    for i, om in enumerate(np.asarray(sol.omega)):
        if (not velo) and om > thr:
            continue
        lines.append("%4d%10.4f%13.6f%13.6f%13.6f%13.6f" % (
            i + 1, om * EH2EV_OUT, sol.fL[i], sol.fV[i], sol.RL[i], sol.RV[i]))
    return "\n".join(lines) + "\n"
