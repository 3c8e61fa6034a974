"""Served form (std2g_server_*): each result is the same alone and in the mix.

Requests of mixed size, some with alpha(w), are solved one at a time on a
single context ("alone") and then all together through the request server
("in the mix"), where they are admitted into free slots and run concurrently
on the device.  Roots must agree to 1e-9 Eh, f_L to 1e-8 relative, the CSF
lists must be identical (hash) and alpha(w) must agree to 1e-8 relative.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from stda_b200 import synth
    from stda_b200.engine import Keywords, boundary_inputs
    reqs = []
    specs = [(14, 3, 8.0, None), (30, 4, 8.5, [0.0, 0.04, 0.08]), (22, 5, 9.0, None),
             (48, 6, 8.0, None), (36, 7, 8.5, [0.0, 0.05, 0.1]), (18, 8, 9.5, None)]
    for natoms, seed, ethr, om in specs:
        mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
        reqs.append((boundary_inputs(mol, ints), Keywords(ax=0.5, e_thr_ev=ethr, nroots=8), om))
    mol, ints = synth.benzene(seed=0, with_ints=True)
    reqs.append((boundary_inputs(mol, ints), Keywords(ax=0.5, e_thr_ev=10.0, nroots=8), None))
    return reqs


def _alone(reqs, precision):
    from stda_b200.engine import Engine
    out = []
    for b, kw, om in reqs:
        eng = Engine(0, precision)
        eng.load(b)
        sol = eng.solve(kw)
        alpha = eng.polarizability(kw, om)[0] if om is not None else None
        out.append((sol, alpha))
        eng.close()
    return out


def _mix(reqs, precision, slots, budget=0):
    from stda_b200.engine import Server
    srv = Server(0, precision, slots=slots, hbm_budget=budget)
    tickets = [srv.submit(b, kw, om) for b, kw, om in reqs]
    res = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    return res, st


def _same(alone, mixed):
    for (sol, alpha), (msol, malpha, mres, timing) in zip(alone, mixed):
        assert msol.csf_hash == sol.csf_hash
        assert msol.nci == sol.nci and len(msol.omega) == len(sol.omega)
        assert np.abs(msol.omega - sol.omega).max() < 1e-9
        assert np.allclose(msol.fL, sol.fL, rtol=1e-8, atol=1e-12)
        if alpha is not None:
            assert np.abs(malpha - alpha).max() <= 1e-8 * np.abs(alpha).max()
            assert mres.max() < 1e-8
        assert timing["latency_ms"] >= timing["run_ms"] > 0


@pytest.mark.parametrize("precision", [1, 0])
def test_same_alone_and_in_the_mix(precision):
    reqs = _requests()
    alone = _alone(reqs, precision)
    mixed, st = _mix(reqs, precision, slots=3)
    _same(alone, mixed)
    assert st["submitted"] == st["completed"] == len(reqs)
    assert st["peak_in_flight"] >= 2          # requests overlapped on the device
    assert st["in_flight"] == 0


def test_admission_by_footprint():
    reqs = _requests()[:4]
    alone = _alone(reqs, 1)
    mixed, st = _mix(reqs, 1, slots=4, budget=1)   # nothing fits beside another request
    _same(alone, mixed)
    assert st["peak_in_flight"] == 1


def test_result_room_grows_on_demand():
    """A full-window request (nroots = 0) with more roots than the caller's
    room: std2g_solve reports the count with STD2G_ECAP and the binding solves
    again with enough room; the server keeps the ticket on STD2G_ECAP and the
    binding waits again.  Both return every root."""
    from stda_b200 import synth
    from stda_b200.engine import Engine, Keywords, Server, boundary_inputs
    mol, ints = synth.benzene(seed=0, with_ints=True)
    b = boundary_inputs(mol, ints)
    kw = Keywords(ax=0.5, e_thr_ev=10.0)           # every root in (0, E_thr]
    eng = Engine(0, 0)
    eng.load(b)
    ref = eng.solve(kw)
    small = eng.solve(kw, cap=4)
    eng.close()
    assert len(ref.omega) > 4 and len(small.omega) == len(ref.omega)
    assert np.abs(small.omega - ref.omega).max() < 1e-12
    srv = Server(0, 0, slots=1)
    ticket = srv.submit(b, kw, None)
    sol = srv.wait(ticket, cap=4)[0]
    srv.close()
    assert len(sol.omega) == len(ref.omega)
    assert np.abs(sol.omega - ref.omega).max() < 1e-12
    assert np.allclose(sol.fL, ref.fL, rtol=1e-10, atol=1e-14)


def test_primitive_list_requests_in_the_mix():
    """Requests that carry the primitive list instead of packed integrals
    (std2g_request.nprims > 0: the worker forms S and mu on the device with
    std2g_load_prims) give the results of the host-integral requests, also
    when both kinds share the server."""
    from stda_b200 import synth
    from stda_b200.engine import Keywords, boundary_inputs, prim_inputs
    reqs, reqs_p = [], []
    for natoms, seed, om in ((20, 31, None), (34, 32, [0.0, 0.05]), (26, 33, None)):
        mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
        kw = Keywords(ax=0.5, e_thr_ev=8.5, nroots=6)
        reqs.append((boundary_inputs(mol, ints), kw, om))
        reqs_p.append((prim_inputs(mol), kw, om))
    alone = _alone(reqs, 0)
    mixed, st = _mix(reqs_p + reqs, 0, slots=3)
    _same(alone + alone, mixed)
    assert st["completed"] == 2 * len(reqs)
