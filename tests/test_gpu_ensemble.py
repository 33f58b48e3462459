"""Ensembles: independent runs advanced with one CUDA-graph launch per step.

A parameter scan in the reference is many separate runs of
``tevol_driven_cluster.m`` / ``tevol_lattice.m`` with different grids, ``nz``,
``mu`` and seeds.  ``hqt.Ensemble`` advances such runs together.  A member's
kernels and inputs are exactly those of the run stepped alone, only the
launch is shared, so every member must come out bit-identical to its solo
run made of the same calls (uneven grids, both precisions, with and without
winding removal).  A call recomputes d_z A_t from A_t on entry, so the solo
runs are split into the same calls as the ensemble.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

VY7 = -2 * np.pi * 7 / 20

MEMBERS = [
    dict(nx=64, ny=64, nz=21, L=50.0, mu=6.0, vy=VY7, rw=True, prec="fp64", seed=0),
    dict(nx=48, ny=40, nz=17, L=30.0, mu=5.0, vy=0.0, rw=False, prec="fp64", seed=1),
    dict(nx=33, ny=33, nz=12, L=20.0, mu=7.5, vy=VY7, rw=True, prec="mixed", seed=2),
]


def member_state(hqt, m):
    prof = hqt.seed.stationary_profile(m["mu"], m["vy"])
    return hqt.seed.init_driven(m["nx"], m["ny"], m["nz"], prof, noise="complex",
                                amplitude=1e-3, seed=m["seed"])


def member_sim(hqt, m):
    return hqt.Simulation(m["nx"], m["ny"], m["nz"], Lx=m["L"], mu=m["mu"], vy=m["vy"],
                          dt=0.02, remove_winding=m["rw"], precision=m["prec"])


def test_ensemble_members_match_solo_runs(hqt, cuda):
    api = __import__(hqt.__name__ + ".api", fromlist=["to_device"])
    states = [member_state(hqt, m) for m in MEMBERS]
    solo = []
    for m, st in zip(MEMBERS, states):
        t = [api.to_device(a) for a in st]
        with member_sim(hqt, m) as sim:
            sim.step_device(*t, nsteps=20)
            sim.step_device(*t, nsteps=10)
        solo.append([api.from_device(x) for x in t])
    sims = [member_sim(hqt, m) for m in MEMBERS]
    dev_states = [[api.to_device(a) for a in st] for st in states]
    with hqt.Ensemble(sims) as ens:
        info = ens.step_device(dev_states, nsteps=20)
        info += ens.step_device(dev_states, nsteps=10)  # the graph is reused
    for s in sims:
        s.close()
    assert [i.steps_done for i in info] == [20] * 3 + [10] * 3
    assert all(i.nonfinite_step == -1 for i in info)
    for k, (m, want, got) in enumerate(zip(MEMBERS, solo, dev_states)):
        for f, (w, g) in enumerate(zip(want, got)):
            assert np.array_equal(api.from_device(g), w), (k, f)


def test_ensemble_follows_new_device_arrays(hqt, cuda):
    """Calls on other device arrays must step those arrays: the ensemble graph
    bakes in the members' state pointers and is rebuilt when they change.
    Covered: a second set alive beside the first (the first must stay as its
    own call left it), and a third set allocated after the second was freed
    (the caching allocator may hand out the same addresses)."""
    api = __import__(hqt.__name__ + ".api", fromlist=["to_device"])
    states = [member_state(hqt, m) for m in MEMBERS[:2]]
    solo = []
    for m, st in zip(MEMBERS[:2], states):
        t = [api.to_device(a) for a in st]
        with member_sim(hqt, m) as sim:
            sim.step_device(*t, nsteps=6)
        solo.append([api.from_device(x) for x in t])

    def check(sets):
        for k, (want, got) in enumerate(zip(solo, sets)):
            for f, (w, g) in enumerate(zip(want, got)):
                assert np.array_equal(api.from_device(g), w), (k, f)

    sims = [member_sim(hqt, m) for m in MEMBERS[:2]]
    first = [[api.to_device(a) for a in st] for st in states]
    second = [[api.to_device(a) for a in st] for st in states]
    with hqt.Ensemble(sims) as ens:
        ens.step_device(first, nsteps=6)
        check(first)
        ens.step_device(second, nsteps=6)
        check(second)
        check(first)  # untouched by the second call
        del second
        third = [[api.to_device(a) for a in st] for st in states]
        ens.step_device(third, nsteps=6)
        check(third)
    for s in sims:
        s.close()


def test_ensemble_reports_the_nonfinite_member(hqt, cuda):
    api = __import__(hqt.__name__ + ".api", fromlist=["to_device"])
    states = [list(member_state(hqt, m)) for m in MEMBERS[:2]]
    states[1][2] = states[1][2].copy()
    states[1][2][3, 4, 2] = np.nan
    sims = [member_sim(hqt, m) for m in MEMBERS[:2]]
    dev_states = [[api.to_device(a) for a in st] for st in states]
    with hqt.Ensemble(sims) as ens:
        with pytest.raises(hqt.NonfiniteEvolution) as e:
            ens.step_device(dev_states, nsteps=10)
    for s in sims:
        s.close()
    assert e.value.info[1].nonfinite_step == 1
    assert e.value.info[1].steps_done == 1  # stopped at its bad step
    assert e.value.info[0].nonfinite_step == -1
    assert e.value.info[0].steps_done == 10


def test_ensemble_rejects_duplicate_members(hqt, cuda):
    m = MEMBERS[0]
    with member_sim(hqt, m) as sim:
        with pytest.raises(hqt.HQTError):
            hqt.Ensemble([sim, sim])
