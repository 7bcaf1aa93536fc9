"""The orchestration of the time-lapse drivers (src/PyFWI/tl_fwi.py) without
a GPU: which vintage's data each FWI inversion of a method runs on, from
which model it starts, and how the returned differences are formed.  The
inversions are replaced by a stand-in that adds a tag to the starting model
(+1 on the baseline data, +10 on the monitor data, +100 on anything else),
so every output of a method is a known sum of tags."""
import numpy as np
import pytest
import torch

import cases
from conftest import load_golden


@pytest.fixture
def timelapse(monkeypatch):
    from pyfwi_b200 import acquisition as acq
    from pyfwi_b200.fwi import FWI
    from pyfwi_b200.processing import prepare_residual
    from pyfwi_b200.tl_fwi import TimeLapse
    case = cases.tiny_dxr()
    inpa = dict(case["inpa"], cuda_device="cpu")
    src = acq.Source(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    g = load_golden("tiny_dxr")
    b_obs = prepare_residual({k[6:]: v for k, v in g.items() if k.startswith("d_obs_")})
    m_obs = {k: 1.5 * v for k, v in b_obs.items()}
    T = TimeLapse(b_obs, m_obs, inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                  components=case["components"], chpr=case["chpr"], n_well_rec=case["n_well_rec"])
    log = []

    def fake_call(self, m0, method, iter, freqs, n_params, k_0, k_end):
        vx = self.d_obs["vx"]
        if torch.equal(vx, T._obs("b")["vx"]):
            tag, name = 1.0, "b"
        elif torch.equal(vx, T._obs("m")["vx"]):
            tag, name = 10.0, "m"
        else:
            tag, name = 100.0, "other"
        log.append((name, float(m0["vp"].flat[0])))
        return {k: v + tag for k, v in m0.items()}, np.array([0.0])
    monkeypatch.setattr(FWI, "__call__", fake_call)
    m0 = {k: np.zeros_like(v, dtype=np.float64) for k, v in case["model_est"].items()}
    return T, m0, log


def _run(T, m0, method):
    return T(m0, iter=[1], freqs=[0], tl_method=method, n_params=1, k_0=1, k_end=4)


def _v(d):
    return float(d["vp"].flat[0])


def test_parallel(timelapse):
    T, m0, log = timelapse
    out, hist = _run(T, m0, "pa")
    assert log == [("b", 0.0), ("m", 0.0)]
    assert (_v(out["b1"]), _v(out["m1"]), _v(out["dm"])) == (1.0, 10.0, 9.0)
    assert set(hist) == {"b1", "m1"}


def test_cascaded(timelapse):
    T, m0, log = timelapse
    out, _ = _run(T, m0, "cc")
    assert log == [("b", 0.0), ("m", 1.0)]
    assert (_v(out["b1"]), _v(out["m1"]), _v(out["dm"])) == (1.0, 11.0, 10.0)


def test_weighted_average(timelapse):
    T, m0, log = timelapse
    out, hist = _run(T, m0, "wa")
    assert log == [("b", 0.0), ("m", 1.0), ("b", 11.0)]
    assert (_v(out["b1"]), _v(out["m1"]), _v(out["b2"])) == (1.0, 11.0, 12.0)
    assert (_v(out["dm11"]), _v(out["dm12"])) == (10.0, -1.0)
    assert set(hist) == {"b1", "m1", "b2"}


def test_central_difference(timelapse):
    T, m0, log = timelapse
    out, _ = _run(T, m0, "cd")
    assert log == [("b", 0.0), ("m", 1.0), ("m", 0.0), ("b", 10.0)]
    b1, b1m, m1, m1b = 1.0, 11.0, 10.0, 11.0
    assert (_v(out["b1"]), _v(out["m2"]), _v(out["m1"]), _v(out["b2"])) == (b1, b1m, m1, m1b)
    assert _v(out["dm0"]) == m1 - b1 and _v(out["dm1"]) == b1m - m1b
    assert _v(out["dm34"]) == ((b1m - b1) + (m1 - m1b)) / 2


def test_cross_updating(timelapse):
    T, m0, log = timelapse
    out, _ = _run(T, m0, "cu")
    assert log == [("b", 0.0), ("m", 1.0), ("b", 11.0), ("m", 12.0)]
    assert (_v(out["dm11"]), _v(out["dm12"]), _v(out["dm21"]), _v(out["dm22"])) == (10.0, -1.0, 21.0, 10.0)
    assert all(k in out for k in ("pt_cc", "pt_wa", "pt_cu"))


def test_double_difference(timelapse, monkeypatch):
    """The second inversion runs on (monitor - baseline) + the data modelled
    from the baseline result, from the starting model."""
    T, m0, log = timelapse
    modelled = []

    def fake_forward(model, show=False):
        modelled.append(_v(model))
        return {"vx": np.full_like(T.b_dobs["vx"], 7.0, dtype=np.float32),
                "vz": np.full_like(T.b_dobs["vz"], 7.0, dtype=np.float32)}
    monkeypatch.setattr(T, "forward_modeling", fake_forward)
    out, _ = _run(T, m0, "dd")
    assert modelled == [1.0]
    assert log == [("b", 0.0), ("other", 0.0)]
    composite = T.inv_obj.d_obs["vx"].numpy()
    expect = (T.m_dobs["vx"] - T.b_dobs["vx"]) + 7.0
    assert np.allclose(composite, expect.astype(np.float32))
    assert (_v(out["b1"]), _v(out["m1"]), _v(out["dm"])) == (1.0, 100.0, 99.0)


def test_unknown_method_is_refused(timelapse):
    T, m0, _ = timelapse
    with pytest.raises(ValueError, match="time-lapse method"):
        _run(T, m0, "xx")
