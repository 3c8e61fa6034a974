"""Regenerate the golden fixtures from the reference's own regression data.

Reads the reference checkout's ``tests/`` folder (``run_tests.sh`` cases,
``water_sto3g.molden``, ``wavelength`` and ``expected_results/*``) and writes

* ``water_sto3g.molden``  - the input wavefunction, verbatim;
* ``wavelength``          - the response wavelengths (nm), verbatim;
* ``reference_expected.json`` - for every case: the std2 command-line keywords
  and the expected rows (``tda.dat`` DATXY rows, ``2PA-abs`` rows,
  ``beta_HRS`` rows).

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import os
import shutil
import sys

CASES = {
    # tests/run_tests.sh:22-24, 44-46, 66-68
    "EXCI_TEST1": dict(kind="tda", args=dict(ax=1.0, e_thr_ev=20.0)),
    "EXCI_TEST2": dict(kind="tda", args=dict(ax=0.5, e_thr_ev=30.0)),
    "EXCI_TEST3": dict(kind="tda", args=dict(ax=1.0, e_thr_ev=30.0, beta_j=1.0, alpha_k=3.0)),
    "BETA_TEST1": dict(kind="beta_HRS", args=dict(ax=1.0, e_thr_ev=20.0)),
    "BETA_TEST2": dict(kind="beta_HRS", args=dict(ax=0.5, e_thr_ev=30.0)),
    "BETA_TEST3": dict(kind="beta_HRS", args=dict(ax=1.0, e_thr_ev=30.0, beta_j=1.0, alpha_k=3.0)),
    "2PA_TEST1": dict(kind="2PA", args=dict(ax=1.0, e_thr_ev=20.0)),
    "2PA_TEST2": dict(kind="2PA", args=dict(ax=0.5, e_thr_ev=30.0)),
    "2PA_TEST3": dict(kind="2PA", args=dict(ax=1.0, e_thr_ev=30.0, beta_j=1.0, alpha_k=3.0)),
}


def rows_of(path, kind):
    text = open(path).read().splitlines()
    if kind == "tda":
        i = next(k for k, ln in enumerate(text) if "DATXY" in ln)
        text = text[i + 1:]
        header = [ln.strip() for ln in open(path).read().splitlines()[:i + 1]]
    else:
        header = []
    rows = [[float(t) for t in ln.split()] for ln in text if ln.strip()]
    return header, rows


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    tdir = os.path.join(ref, "tests")
    shutil.copyfile(os.path.join(tdir, "water_sto3g.molden"), os.path.join(here, "water_sto3g.molden"))
    shutil.copyfile(os.path.join(tdir, "wavelength"), os.path.join(here, "wavelength"))
    out = {}
    for name, spec in CASES.items():
        ext = ".dat" if spec["kind"] == "tda" else ".txt"
        header, rows = rows_of(os.path.join(tdir, "expected_results", name + ext), spec["kind"])
        out[name] = dict(spec, header=header, rows=rows,
                         tolerance=1e-3 if spec["kind"] != "2PA" else [1e-3, 1e-2])
    with open(os.path.join(here, "reference_expected.json"), "w") as fh:
        json.dump(out, fh, indent=1)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
