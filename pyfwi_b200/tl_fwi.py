"""``TimeLapse``: PyFWI's time-lapse FWI drivers (src/PyFWI/tl_fwi.py:13-584)
on the device propagator.

Same constructor and ``__call__(b_m0, iter, freqs, tl_method, n_params,
k_0, k_end)``, the same methods and the same output dicts:

* 'pa' parallel, 'cc' cascaded, 'dd' double difference, 'wa' weighted
  average, 'cd' central difference, 'cu' cross updating: sequences of
  ``FWI`` L-BFGS inversions (method 2) over the baseline and monitor data,
  swapped through ``inv_obj.d_obs`` as the reference does;
* 'sim' simultaneous and 'cj' cascaded joint: L-BFGS over the stacked
  (baseline, monitor) model of the joint misfit (``tl_fprime``: both
  vintages' L2 misfits plus 1e-10 * 1/2 |m - b|^2), with the reference's
  settings (m=30, factr=1e-10, pgtol=1e-12, maxls=20).

The inversions run on the device L-BFGS (``FWI.optimizer``, pyfwi_b200.lbfgs)
and every misfit evaluation on the device propagator; the stacked model of
'sim' / 'cj' stays on the device between evaluations.  Returned models are
numpy dicts, as the reference returns; the wall-clock entries ('pt', ...)
time this machine."""
import copy
import timeit

import numpy as np
import torch

from . import fwi_tools as tools
from . import lbfgs as device_lbfgs
from .fwi import FWI, evaluate, observed_on_device
from .processing import prepare_residual
from .wave_propagation import WavePropagator

GAMMA = 1e-10  # weight of the baseline-monitor model difference (tl_fwi.py:175)


def dict_diff(dict1, dict2, positivity=False):
    """dict1 - dict2 per key; negative differences set to 0 with
    `positivity` (fwi_tools.py:1537-1558)."""
    out = {}
    for k in dict1:
        out[k] = dict1[k] - dict2[k]
        if positivity:
            out[k][out[k] < 0] = 0
    return out


def dict_summation(dict1, dict2, division=1.0):
    """(dict1 + dict2) / division per key (fwi_tools.py:1561-1580)."""
    return {k: (dict1[k] + dict2[k]) / division for k in dict1}


class TimeLapse(WavePropagator):
    """Time-lapse FWI of a baseline (``b_dobs``) and a monitor (``m_dobs``)
    survey; the other parameters as ``FWI``."""

    def __init__(self, b_dobs, m_dobs, inpa, src, rec_loc, model_shape, components, chpr, n_well_rec=0,
                 param_functions=None):
        super().__init__(inpa, src, rec_loc, model_shape, n_well_rec=n_well_rec, chpr=chpr, components=components)
        self.inv_obj = FWI(b_dobs, inpa, src, rec_loc, model_shape=model_shape, n_well_rec=n_well_rec, chpr=chpr,
                           components=components, param_functions=param_functions)
        self.b_dobs = copy.deepcopy(b_dobs)
        self.m_dobs = copy.deepcopy(m_dobs)
        self.n_elements = self.nz * self.nx
        self.CF = tools.CostFunction("l2")
        self.fn = self.inv_obj.fn

    def __call__(self, b_m0, iter, freqs, tl_method, n_params, k_0, k_end):
        """Run the time-lapse method `tl_method` ('pa', 'cc', 'dd', 'sim',
        'wa', 'cj', 'cd', 'cu'); returns (models dict, misfit history dict)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        if tl_method == "pa":
            return self.parallel_inversion(b_m0, freqs, iter, **kw)
        if tl_method == "cc":
            return self.cascaded_inversion(b_m0, freqs, iter, **kw)
        if tl_method == "dd":
            return self.double_difference_inversion(b_m0, freqs, iter, **kw)
        if tl_method == "sim":
            return self.sim_inversion(b_m0, freqs, iter, data_to_invert=self.b_dobs, **kw)
        if tl_method == "wa":
            return self.weighted_averaged_cascaded(b_m0, freqs, iter, **kw)
        if tl_method == "cj":
            return self.cascaded_joint(b_m0, freqs, iter, **kw)
        if tl_method == "cd":
            return self.central_difference(b_m0, freqs, iter, **kw)
        if tl_method == "cu":
            return self.cross_updating(b_m0, freqs, iter, **kw)
        raise ValueError("unknown time-lapse method %r" % (tl_method,))

    # -- one FWI on a chosen vintage ------------------------------------------

    def _invert(self, d_obs, m0, freqs, iter, n_params, k_0, k_end):
        self.inv_obj.d_obs = d_obs
        return self.inv_obj(m0, method=2, freqs=freqs, iter=iter, n_params=n_params, k_0=k_0, k_end=k_end)

    # -- joint (simultaneous) inversion ---------------------------------------

    def tl_lbfgs(self, x0, iter, freq, n_params, k0, k_end):
        """L-BFGS of the joint misfit over parameter k (baseline and monitor
        together) for k = k0-1, k0-1+n_params, ... < k_end-1 (tl_fwi.py:114-147);
        x0 is the stacked model (baseline then monitor), updated in place with
        each result rounded to float32."""
        n = self.n_elements
        dev = self.device
        x0_dev = torch.from_numpy(np.asarray(x0, np.float64)).to(dev)
        self.xrest = x0_dev.clone()
        hist = []
        for k in np.arange(k0 - 1, k_end - 1, n_params):
            k = int(k)
            m_opt = torch.cat((x0_dev[k * n:(k + n_params) * n], x0_dev[(3 + k) * n:3 * n + (k + n_params) * n]))
            res = device_lbfgs.minimize(lambda x: self.tl_fprime(x, freq, k, n_params), m_opt, m=30, factr=1e-10,
                                        pgtol=1e-12, maxfun=15000, maxiter=iter, maxls=20)
            hist.append(res.f)
            x = res.x.to(torch.float32).to(torch.float64)
            x0_dev[k * n:(k + n_params) * n] = x[:n_params * n]
            x0_dev[(3 + k) * n:(3 + k + n_params) * n] = x[n_params * n:]
        x0[:] = x0_dev.cpu().numpy()
        return x0, hist

    def tl_fprime(self, x, freq, k, n_params):
        """Joint misfit and gradient at the stacked parameter-k vector x
        (baseline block, then monitor block), the other parameters taken from
        ``self.xrest`` (tl_fwi.py:149-219)."""
        n = self.n_elements
        x1 = self.xrest
        x1[k * n:(k + n_params) * n] = x[:n_params * n]
        x1[3 * n + k * n:3 * n + (k + n_params) * n] = x[n_params * n:2 * n_params * n]
        inv = self.inv_obj
        b_pcs = self._params(x1[:3 * n])
        m_pcs = self._params(x1[3 * n:])
        b_model = self._model(inv.model_to_dv(b_pcs, inv.param_functions_args))
        m_model = self._model(inv.model_to_dv(m_pcs, inv.param_functions_args))
        b_rms, b_grad_dv = evaluate(self, b_model, self._obs("b"), inv.sd, freq)
        b = x1[k * n:(k + n_params) * n]
        m = x1[(3 + k) * n:(3 + k + n_params) * n]
        diff = m - b
        rms_diff = 0.5 * float(torch.dot(diff, diff))
        b_grad = self._grad_vec(b_grad_dv, b_pcs)
        m_rms, m_grad_dv = evaluate(self, m_model, self._obs("m"), inv.sd, freq)
        m_grad = self._grad_vec(m_grad_dv, m_pcs)
        rms = b_rms + m_rms + GAMMA * rms_diff
        grad = torch.cat((b_grad[k * n:(k + n_params) * n] + GAMMA * (b - m),
                          m_grad[k * n:(k + n_params) * n] + GAMMA * (m - b)))
        return rms, grad.to(torch.float64)

    def _obs(self, which):
        """Device copy of the baseline ('b') or monitor ('m') data, made once."""
        key = "_dev_" + which
        if getattr(self, key, None) is None:
            setattr(self, key, observed_on_device(self, self.b_dobs if which == "b" else self.m_dobs))
        return getattr(self, key)

    def _params(self, vec):
        """Parameter dict of a stacked half; numpy for user parameter functions."""
        if not self.inv_obj._default_params:
            vec = vec.cpu().numpy()
        return self.inv_obj.vec2dict(vec, self.nz, self.nx)

    def _model(self, m):
        return {k: self._to_device(m[k]) for k in ("vp", "vs", "rho")}

    def _grad_vec(self, grad_dv, pcs):
        inv = self.inv_obj
        if not inv._default_params:
            grad_dv = {k: v.cpu().numpy() for k, v in grad_dv.items()}
        g = inv.dict2vec(inv.grad_from_dv(grad_dv, inv.param_functions_args, pcs))
        return g if isinstance(g, torch.Tensor) else torch.from_numpy(np.asarray(g, np.float64)).to(self.device)

    def sim_inversion(self, b_m0, freqs, iter, n_params, k_0, k_end, data_to_invert=None):
        """Simultaneous inversion (tl_fwi.py:474-521).  With `data_to_invert`
        an FWI from b_m0 on the inversion object's current data comes first
        (the reference stores the data in ``self.dobs``, which that FWI does
        not read), and both halves start from its result."""
        rms2 = []
        tic = timeit.default_timer()
        if data_to_invert is not None:
            self.dobs = data_to_invert
            model_ref0, rms1 = self.inv_obj(b_m0, method=2, freqs=freqs, iter=iter, n_params=n_params, k_0=k_0,
                                            k_end=k_end)
            b_model0, m_model0 = copy.deepcopy(model_ref0), copy.deepcopy(model_ref0)
        else:
            b_model0, m_model0 = copy.deepcopy(b_m0), copy.deepcopy(b_m0)
        x0 = np.hstack((self.inv_obj.dict2vec(b_model0), self.inv_obj.dict2vec(m_model0)))
        for c, freq in enumerate(freqs):
            x0, hist1 = self.tl_lbfgs(x0, iter[c], freq, n_params, k_0, k_end)
            rms2.append(hist1[0])
        models = self.ins_TL_output(x0, False)
        process_time = timeit.default_timer() - tic
        inverted = {"dm": self.ins_TL_output(x0, True), "b1": models["model_b"], "m1": models["model_m"],
                    "pt": process_time}
        return inverted, {"sim": rms2}

    def ins_TL_output(self, xk, diff=True):
        """Stacked vector -> the monitor-minus-baseline dict (`diff`) or both
        models (tl_fwi.py:524-553)."""
        half = int(xk.shape[0] / 2)
        if diff:
            return self.inv_obj.vec2dict(xk[half:] - xk[:half], self.nz, self.nx)
        return {"model_b": self.inv_obj.vec2dict(xk[:half], self.nz, self.nx),
                "model_m": self.inv_obj.vec2dict(xk[half:2 * half], self.nz, self.nx)}

    # -- sequences of single-vintage inversions -------------------------------

    def parallel_inversion(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Baseline and monitor each inverted from b_m0 (tl_fwi.py:408-431)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        tic = timeit.default_timer()
        model_b1, rms1 = self._invert(self.b_dobs, b_m0, freqs, iter, **kw)
        model_m1, rms2 = self._invert(self.m_dobs, b_m0, freqs, iter, **kw)
        inverted = {"b1": model_b1, "m1": model_m1, "dm": dict_diff(model_m1, model_b1, positivity=False),
                    "pt": timeit.default_timer() - tic}
        return inverted, {"b1": rms1, "m1": rms2}

    def cascaded_inversion(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Monitor inverted from the baseline's result (tl_fwi.py:444-472)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        tic = timeit.default_timer()
        model_b1, rms1 = self._invert(self.b_dobs, b_m0, freqs, iter, **kw)
        initial = model_b1.copy()
        model_m1, rms2 = self._invert(self.m_dobs, model_b1, freqs, iter, **kw)
        inverted = {"b1": model_b1, "m1": model_m1, "dm": dict_diff(model_m1, initial, positivity=False),
                    "pt": timeit.default_timer() - tic}
        return inverted, {"b1": rms1, "m1": rms2}

    def double_difference_inversion(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Inversion of (monitor - baseline) + data of the baseline result
        from b_m0 (tl_fwi.py:433-442, Asnaashari et al. 2011)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        tic = timeit.default_timer()
        model_b1, rms1 = self._invert(self.b_dobs, b_m0, freqs, iter, **kw)
        d_ref = self.forward_modeling(model_b1, show=False)
        d_ref = prepare_residual(d_ref, s=self.inv_obj.sd)
        d_composite = dict_summation(dict_diff(self.m_dobs, self.b_dobs), d_ref)
        model_composite, rms2 = self._invert(d_composite, b_m0.copy(), freqs, iter, **kw)
        inverted = {"b1": model_b1, "m1": model_composite,
                    "dm": dict_diff(model_composite, model_b1, positivity=False),
                    "pt": timeit.default_timer() - tic}
        return inverted, {"b1": rms1, "m1": rms2}

    def weighted_averaged_cascaded(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Baseline, monitor from it, baseline again from the monitor
        (tl_fwi.py:221-255)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        m0 = copy.deepcopy(b_m0)
        model_b1, rms_b1 = self._invert(self.b_dobs, m0, freqs, iter, **kw)
        model_m1, rms_m1 = self._invert(self.m_dobs, model_b1, freqs, iter, **kw)
        model_b2, rms_b2 = self._invert(self.b_dobs, model_m1, freqs, iter, **kw)
        inverted = {"dm11": dict_diff(model_m1, model_b1), "dm12": dict_diff(model_m1, model_b2), "m1": model_m1,
                    "b1": model_b1, "b2": model_b2}
        return inverted, {"b1": rms_b1, "m1": rms_m1, "b2": rms_b2}

    def cross_updating(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Four alternating cascaded inversions (tl_fwi.py:257-303,
        Maharramov & Biondi 2014)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        m0 = copy.deepcopy(b_m0)
        tic = timeit.default_timer()
        model_b1, rms_b1 = self._invert(self.b_dobs, m0, freqs, iter, **kw)
        model_m1, rms_m1 = self._invert(self.m_dobs, model_b1, freqs, iter, **kw)
        pt_cc = timeit.default_timer() - tic
        model_b2, rms_b2 = self._invert(self.b_dobs, model_m1, freqs, iter, **kw)
        pt_wa = timeit.default_timer() - tic
        model_m2, rms_m2 = self._invert(self.m_dobs, model_b2, freqs, iter, **kw)
        pt_cu = timeit.default_timer() - tic
        inverted = {"dm11": dict_diff(model_m1, model_b1), "dm12": dict_diff(model_m1, model_b2),
                    "dm21": dict_diff(model_m2, model_b1), "dm22": dict_diff(model_m2, model_b2),
                    "b1": model_b1, "m1": model_m1, "b2": model_b2, "m2": model_m2,
                    "pt_cc": pt_cc, "pt_wa": pt_wa, "pt_cu": pt_cu}
        return inverted, {"b1": rms_b1, "m1": rms_m1, "b2": rms_b2, "m2": rms_m2}

    def central_difference(self, b_m0, freqs, iter, n_params, k_0, k_end):
        """Baseline-then-monitor and monitor-then-baseline cascades from b_m0
        (tl_fwi.py:306-354)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        m0 = copy.deepcopy(b_m0)
        tic = timeit.default_timer()
        model_b1, rms_b1 = self._invert(self.b_dobs, m0, freqs, iter, **kw)
        model_b1m, rms_b1m = self._invert(self.m_dobs, model_b1, freqs, iter, **kw)
        model_m1, rms_m1 = self._invert(self.m_dobs, m0, freqs, iter, **kw)
        model_m1b, rms_m1b = self._invert(self.b_dobs, model_m1, freqs, iter, **kw)
        inverted = {"dm0": dict_diff(model_m1, model_b1), "dm1": dict_diff(model_b1m, model_m1b),
                    "dm3": dict_diff(model_b1m, model_b1), "dm4": dict_diff(model_m1, model_m1b),
                    "dm34": dict_summation(dict_diff(model_b1m, model_b1), dict_diff(model_m1, model_m1b),
                                           division=2),
                    "b1": model_b1, "m1": model_m1, "m2": model_b1m, "b2": model_m1b,
                    "pt": timeit.default_timer() - tic}
        return inverted, {"b1": rms_b1, "m1": rms_m1, "m2": rms_b1m, "b2": rms_m1b}

    def cascaded_joint(self, m0, freqs, iter, n_params, k_0, k_end):
        """Two simultaneous inversions, the second from the average of the
        first's models (tl_fwi.py:356-406)."""
        kw = dict(n_params=n_params, k_0=k_0, k_end=k_end)
        tic = timeit.default_timer()
        model1, rms1 = self.sim_inversion(m0, freqs, iter=iter, data_to_invert=None, **kw)
        model_b1, model_m1 = model1["b1"], model1["m1"]
        ave_model = dict_summation(model_b1, model_m1, division=2)
        model_b1x, rms2 = self.sim_inversion(ave_model, freqs, iter=iter, data_to_invert=None, **kw)
        model_b1b, model_b1m = model_b1x["b1"], model_b1x["m1"]
        inverted = {"dm0": dict_diff(model_m1, model_b1), "dm7": dict_diff(model_b1m, model_b1b),
                    "dm3": dict_diff(model_b1m, model_b1), "dm6": dict_diff(model_m1, model_b1b),
                    "b1": model_b1, "m1": model_m1, "b2": model_b1b, "m2": model_b1m,
                    "pt": timeit.default_timer() - tic}
        return inverted, {"sim1": rms1, "sim2": rms2}
