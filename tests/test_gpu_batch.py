"""SurveyBatch: surveys of uneven size (different grids, record lengths,
time steps, receiver layouts) evaluated together, on one stream per survey
and as one replayed CUDA graph, give each survey's own misfit and gradient."""
import numpy as np
import pytest

import cases
from conftest import load_golden
from helpers import product

pytestmark = pytest.mark.gpu

NAMES = ["tiny_s8", "tiny_dtscale", "tiny_crosswell", "tiny_dxr"]


def _inputs(dev, scale=1.0):
    import torch
    models, observed = [], []
    for n in NAMES:
        case = cases.by_name(n)
        models.append({k: torch.from_numpy(v * np.float32(scale)).to(dev) for k, v in case["model_est"].items()})
        g = load_golden(n)
        observed.append({k[6:]: torch.from_numpy(v).to(dev) for k, v in g.items() if k.startswith("d_obs_")})
    return models, observed


def _alone(models, observed):
    out = []
    for n, m, o in zip(NAMES, models, observed):
        W = product(cases.by_name(n))
        rms, g = W.misfit_gradient(m, o)
        out.append((float(rms), {k: v.cpu().numpy() for k, v in g.items()}))
    return out


def _same(a, b):
    """Gradients bit for bit; misfits to double rounding (a double atomic sum,
    whose order varies between runs)."""
    for (ra, ga), (rb, gb) in zip(a, b):
        assert abs(ra - float(rb)) <= 1e-12 * abs(ra)
        for k in ga:
            assert np.array_equal(ga[k], gb[k].cpu().numpy()), k


@pytest.mark.parametrize("graph", [False, True])
def test_uneven_surveys_match_single_runs(graph):
    import torch
    from pyfwi_b200.batch import SurveyBatch
    dev = torch.device("cuda", 0)
    models, observed = _inputs(dev)
    ref = _alone(models, observed)
    batch = SurveyBatch([product(cases.by_name(n)) for n in NAMES], graph=graph)
    for _ in range(2):  # with graph=True: capture, then a replay
        _same(ref, batch.misfit_gradient(models, observed))
    if graph:  # a replay on other models is the evaluation of those models
        models2, _ = _inputs(dev, scale=1.01)
        _same(_alone(models2, observed), batch.misfit_gradient(models2, observed))
