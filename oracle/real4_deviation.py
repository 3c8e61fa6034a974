"""How far the reference's own real*4 arithmetic sits from FP64 (TEST
INFRASTRUCTURE ONLY: runs the oracle twice, ``real4=False`` and ``real4=True``).

For each molecule it prints the CSF count, the number of roots, the largest
root difference (eV), the largest relative f_L difference over roots with
f_L > 1e-3, whether the selected CSF sets agree, and for the sTD-DFT cases the
largest relative difference of alpha(w) at w = 0 and 0.05 Eh (the reference
solves those in real*4 too, linear_response.f:23-192).

    python oracle/real4_deviation.py
"""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle.stda_fp64 import EH2EV_IN, Params, dynamic_polarizability, stda  # noqa: E402


def deviation(mol, ints, **kw):
    S, L, V, M = ints
    p = Params(**kw)
    args = (mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, p)
    a = stda(*args, real4=False)
    b = stda(*args, real4=True)
    n = min(len(a.omega), len(b.omega))
    de = float(np.abs(a.omega[:n] - b.omega[:n]).max()) * EH2EV_IN
    big = a.fL[:n] > 1e-3
    rf = float((np.abs(a.fL[:n][big] - b.fL[:n][big]) / a.fL[:n][big]).max()) if big.any() else 0.0
    ra = None
    if p.rpa:
        om = [0.0, 0.05]
        aa, ab = dynamic_polarizability(a, om), dynamic_polarizability(b, om)
        ra = float(np.abs(aa - ab).max() / np.abs(aa).max())
    return len(a.iconf), n, de, rf, bool(np.array_equal(a.iconf, b.iconf)), ra


def main():
    from stda_b200 import synth
    cases = [("benzene, sTDA", synth.benzene(with_ints=True), dict(ax=0.5, e_thr_ev=10.0)),
             ("benzene, sTD-DFT", synth.benzene(with_ints=True), dict(ax=0.5, e_thr_ev=10.0, rpa=True)),
             ("30-atom cluster", synth.random_molecule(30, seed=3, with_ints=True), dict(ax=0.5, e_thr_ev=7.0)),
             ("30-atom cluster, sTD-DFT", synth.random_molecule(30, seed=3, with_ints=True),
              dict(ax=0.5, e_thr_ev=7.0, rpa=True)),
             ("40-atom cluster", synth.random_molecule(40, seed=4, with_ints=True), dict(ax=0.5, e_thr_ev=7.0)),
             ("flake C24H12", synth.graphene_flake(2, with_ints=True), dict(ax=0.5, e_thr_ev=7.0)),
             ("flake C54H18", synth.graphene_flake(3, with_ints=True), dict(ax=0.5, e_thr_ev=7.0))]
    print("| molecule | CSFs | roots | max dE (eV) | max rel f_L | CSF set | max rel alpha(w) |")
    print("|---|---:|---:|---:|---:|---|---:|")
    for name, (mol, ints), kw in cases:
        nci, n, de, rf, same, ra = deviation(mol, ints, **kw)
        print(f"| {name} | {nci} | {n} | {de:.1e} | {rf:.1e} | {'same' if same else 'differs'} "
              f"| {'-' if ra is None else f'{ra:.1e}'} |", flush=True)


if __name__ == "__main__":
    main()
