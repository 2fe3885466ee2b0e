"""The batched-scenario form: the scenario generator (CPU) and ensembles of
solvers advanced together through cgfd_ensemble_* (GPU), which must give
each member exactly what the member gives on its own."""
import numpy as np
import pytest

import inputs


def test_scenarios_are_seeded_and_in_range():
    a = inputs.ensemble_scenarios(6, seed=5, nt=10)
    b = inputs.ensemble_scenarios(6, seed=5, nt=10)
    for p, q in zip(a, b):
        assert (p.ni, p.nj, p.nk, p.dt) == (q.ni, q.nj, q.nk, q.dt)
        assert np.array_equal(p.T0y, q.T0y)
        assert 64 <= p.ni <= 160 and 96 <= p.nj <= 256 and 64 <= p.nk <= 128
        strength = p.mu_s[0].min() * 100e6
        # the patch is the only place above the static strength
        assert (p.T0y[0] > strength).sum() == 49
    assert len({(p.ni, p.nj, p.nk) for p in a}) == 6


def test_von_karman_statistics():
    rng = np.random.default_rng(3)
    f = inputs.von_karman(256, 128, 100.0, rng=rng)
    assert abs(f.mean()) < 1e-6 and abs(f.std() - 1.0) < 1e-6
    # correlated over ~2 km: neighbours 100 m apart are close, far ones not
    c1 = np.corrcoef(f[:, :-1].ravel(), f[:, 1:].ravel())[0, 1]
    c40 = np.corrcoef(f[:, :-40].ravel(), f[:, 40:].ravel())[0, 1]
    assert c1 > 0.9 and c40 < 0.5


def _small(n, seed):
    return inputs.ensemble_scenarios(n, seed=seed, nt=24, size_lo=(36, 60, 36), size_hi=(48, 80, 44),
                                     pml=5, margin=6)


@pytest.mark.gpu
def test_ensemble_matches_members_alone(cgfd_lib):
    from cgfd import Ensemble, Solver
    probs = _small(3, seed=11)
    alone = [Solver(p) for p in probs]
    for s in alone:
        s.run(20)
    members = [Solver(p) for p in probs]
    ens = Ensemble(members)
    ens.run(9)
    ens.run(11)
    for a, m in zip(alone, members):
        assert m.steps_done == a.steps_done == 20
        for f in ("Vs", "Slip", "Init_t0"):
            assert np.array_equal(m.fault(f), a.fault(f)), f
        for c in ("Vx", "Vy", "Txy"):
            assert np.array_equal(m.wavefield(c), a.wavefield(c)), c
        assert np.array_equal(m.stations(), a.stations())
    assert max(a.fault("Vs").max() for a in alone) > 0.05
    ens.close()


@pytest.mark.gpu
def test_ensemble_rejects_members_out_of_step(cgfd_lib):
    from cgfd import CgfdError, Ensemble, Solver
    members = [Solver(p) for p in _small(2, seed=12)]
    ens = Ensemble(members)
    ens.run(2)
    members[0].run(1)
    with pytest.raises(CgfdError, match="ERR_STATE"):
        ens.run(1)
    ens.close()
