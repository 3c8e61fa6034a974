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

# atomic masses by nuclear charge (block.f:24-38): Z = 1-56 and 72-83 carry a mass,
# Z = 102 the hydrogen value; every other Z up to 107 contributes 0 to MMASS
_MASS_1_56 = (
    1.00790, 4.00260, 6.94000, 9.01218, 10.81000, 12.01100, 14.00670, 15.99940,
    18.99840, 20.17900, 22.98977, 24.30500, 26.98154, 28.08550, 30.97376, 32.06000,
    35.45300, 39.94800, 39.09830, 40.08000, 44.95590, 47.90000, 50.94150, 51.99600,
    54.93800, 55.84700, 58.93320, 58.71000, 63.54600, 65.38000, 69.73500, 72.59000,
    74.92160, 78.96000, 79.90400, 83.80000, 85.46780, 87.62000, 88.90590, 91.22000,
    92.90640, 95.94000, 98.90620, 101.0700, 102.9055, 106.4000, 107.8680, 112.4100,
    114.8200, 118.6900, 121.7500, 127.6000, 126.9045, 131.3000, 132.9054, 137.3300)
_MASS_72_83 = (
    178.4900, 180.9479, 183.8500, 186.2070, 190.2000, 192.2200, 195.0900, 196.9665,
    200.5900, 204.3700, 207.2000, 208.9804)
_AMS = {z: m for z, m in enumerate(_MASS_1_56, start=1)}
_AMS.update({z: m for z, m in enumerate(_MASS_72_83, start=72)})
_AMS[102] = 1.0079


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
