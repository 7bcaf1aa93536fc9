"""How SurveyBatch shares device memory between surveys whose plans are not
built yet (host logic; device memory queries replaced by fixed numbers)."""
import types

import numpy as np
import torch

from pyfwi_b200.batch import SurveyBatch

GB = 1 << 30


def _survey(tnz, tnx, nt, ns, nr, built=False):
    return types.SimpleNamespace(tnz=tnz, tnx=tnx, nt=nt, nt_ext=nt, ns=ns, nr=nr,
                                 _plan=object() if built else None, memory_budget=None)


def _share(surveys, free, monkeypatch):
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda d: (free, 180 * GB))
    monkeypatch.setattr(torch.cuda, "memory_reserved", lambda d: 0)
    monkeypatch.setattr(torch.cuda, "memory_allocated", lambda d: 0)
    SurveyBatch._share_memory(types.SimpleNamespace(props=surveys, device="cuda"))


def _fixed(W):
    state = 20.0 * W.tnz * W.tnx
    return 4 * 5.0 * W.nt_ext * W.ns * W.nr * 4 + (2 * int(np.ceil(np.sqrt(W.nt))) + 8) * state + (256 << 20)


def test_every_survey_gets_its_fixed_need_and_a_share_by_storage(monkeypatch):
    small, large = _survey(168, 168, 5000, 16, 128), _survey(552, 1064, 4000, 16, 1024)
    mid = _survey(300, 600, 2000, 8, 560)
    _share([small, large, mid], 150 * GB, monkeypatch)
    budgets = [W.memory_budget for W in (small, large, mid)]
    assert sum(budgets) <= 0.8 * 150 * GB + 3
    for W in (small, large, mid):
        assert W.memory_budget >= _fixed(W)
    spare = [W.memory_budget - _fixed(W) for W in (small, large, mid)]
    storage = [W.tnz * W.tnx * W.nt * W.ns for W in (small, large, mid)]
    assert np.allclose(np.array(spare) / sum(spare), np.array(storage) / sum(storage), rtol=1e-6)


def test_built_plans_and_single_surveys_are_left_alone(monkeypatch):
    a, b = _survey(200, 200, 1000, 4, 100, built=True), _survey(200, 200, 1000, 4, 100)
    _share([a, b], 100 * GB, monkeypatch)
    assert a.memory_budget is None and b.memory_budget is None  # one survey still to build


def test_tight_memory_gives_the_fixed_need_only(monkeypatch):
    s = [_survey(400, 800, 4000, 16, 800) for _ in range(3)]
    _share(s, 1 * GB, monkeypatch)
    for W in s:
        assert W.memory_budget == int(_fixed(W))
