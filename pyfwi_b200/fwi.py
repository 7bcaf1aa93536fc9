"""``FWI``: PyFWI's inversion driver (src/PyFWI/fwi.py:12-282) on the device
propagator.

Same constructor and ``__call__(m0, method, iter, freqs, n_params, k_0,
k_end)``.  Each misfit evaluation runs forward modelling, the L2 residual
and the adjoint gradient on the device.  ``lbfgs`` and ``cg`` run the
reference's L-BFGS-B and Polak-Ribiere+ settings with the model, gradient
and history vectors on the device (lbfgs.minimize, cg.minimize);
``inpa['optimizer'] = 'scipy'`` hands the vectors to SciPy's
``fmin_l_bfgs_b`` / ``fmin_cg`` on the host instead, as the reference does.  The multiscale frequencies
(`freqs`) low-pass the data on the device (fwi_tools.lowpass).
Regularisation terms (TV, Tikhonov, prior, parameter relations) are not
provided: asking for them raises."""
import numpy as np
import torch
from scipy.optimize import fmin_cg, fmin_l_bfgs_b

from . import acquisition as acq
from . import fwi_tools as tools
from . import cg as device_cg
from . import lbfgs as device_lbfgs
from .processing import COMPONENTS, prepare_residual
from .wave_propagation import WavePropagator


class MemoizeJac:
    """Cache (f, g) of the last point so f and its gradient cost one
    evaluation."""

    def __init__(self, fun):
        self.fun = fun
        self.x = None
        self.value = self.jac = None

    def _compute(self, x, *args):
        if self.x is None or not np.array_equal(x, self.x):
            self.x = np.asarray(x).copy()
            self.value, self.jac = self.fun(x, *args)

    def __call__(self, x, *args):
        self._compute(x, *args)
        return self.value

    def derivative(self, x, *args):
        self._compute(x, *args)
        return self.jac


def observed_on_device(W, d):
    """Observed data dict -> its nonzero components as float32 device
    tensors, missing components counted as zero (prepare_residual)."""
    obs = prepare_residual({k: W._to_device(v) for k, v in d.items()}, 1)
    return {k: v for k, v in obs.items() if bool(torch.any(v != 0))}


def evaluate(W, model, d_obs, sd, freq):
    """L2 misfit of propagator W's data at `model` against `d_obs` (device
    dict from observed_on_device) and its (vp, vs, rho) gradient on the
    device (fwi.py:228-252): forward modelling scaled by `sd`, both data
    low-passed at `freq` when it is set (cost_seismic), residual, gradient.
    Returns (float misfit, dict of device gradients)."""
    if freq:
        d_est = W.forward_modeling(model, show=False)
        d_est = {k: sd * v for k, v in d_est.items()}
        keys = [k for k in COMPONENTS if k in d_est or k in d_obs]
        like = next(iter(d_est.values()))
        est = {k: d_est[k] if k in d_est else torch.zeros_like(like) for k in keys}
        obs = {k: d_obs[k] if k in d_obs else torch.zeros_like(like) for k in keys}
        rms, adj = tools.cost_seismic(est, obs, fun=tools.CostFunction("l2"), fn=W.fn, freq=freq, order=3, axis=1)
        return float(rms.item()), W.gradient(adj, parameterization="dv")
    if sd == 1 and set(d_obs) == set(acq.section_keys(W.components)):
        # forward, misfit and gradient fused per shot group (same result)
        rms, grad_dv = W.misfit_gradient(model, d_obs, parameterization="dv")
        return float(rms.item()), grad_dv
    d_est = W.forward_modeling(model, show=False)
    d_est = {k: sd * v for k, v in d_est.items()}
    rms = torch.zeros((), dtype=torch.float64, device=W.device)
    adj = {}
    for k in COMPONENTS:
        if k in d_est or k in d_obs:
            est = d_est.get(k, torch.zeros_like(next(iter(d_est.values()))))
            obs = d_obs.get(k, torch.zeros_like(est))
            r, res = tools.CostFunction("l2")({k: est}, {k: obs})
            rms += r
            adj[k] = res[k]
    return float(rms.item()), W.gradient(adj, parameterization="dv")


class FWI(WavePropagator):
    def __init__(self, d_obs, inpa, src, rec_loc, model_shape, components, chpr, n_well_rec=0,
                 param_functions=None):
        super().__init__(inpa, src, rec_loc, model_shape, n_well_rec=n_well_rec, chpr=chpr, components=components)
        self._default_params = param_functions is None
        if param_functions is None:
            self.dict2vec = tools.vel_dict2vec
            self.vec2dict = tools.vec2vel_dict
            self.model_to_dv = lambda a, args: a
            self.grad_from_dv = lambda a, args, b: a
            self.param_functions_args = []
        else:
            self.dict2vec = param_functions["dict2vec"]
            self.vec2dict = param_functions["vec2dict"]
            self.model_to_dv = param_functions["model_to_dv"]
            self.grad_from_dv = param_functions["grad_from_dv"]
            self.param_functions_args = param_functions.get("args", [])
        for key in ("tv", "tikhonov", "prior_model", "param_relation"):
            if inpa.get(key):
                raise NotImplementedError("regularisation '%s' is not provided" % key)
        self.sd = inpa.get("sd", 1.0)
        self.optimizer = inpa.get("optimizer", "device")
        if self.optimizer not in ("device", "scipy"):
            raise ValueError("inpa['optimizer'] is 'device' or 'scipy', not %r" % (self.optimizer,))
        if inpa.get("cost_function_type", "l2") != "l2":
            raise NotImplementedError("only the 'l2' misfit is provided")
        self.grad_coeff = inpa.get("grad_coeff", [1.0, 1.0, 1.0])
        self.n_elements = self.nz * self.nx
        self.d_obs = d_obs

    @property
    def d_obs(self):
        """Observed data: the nonzero components on the device.  Assigning a
        dict (numpy or torch, any subset of components) converts it, so the
        time-lapse drivers can swap vintages as the reference does
        (tl_fwi.py: ``self.inv_obj.d_obs = self.m_dobs``)."""
        return self._d_obs

    @d_obs.setter
    def d_obs(self, d):
        self._d_obs = observed_on_device(self, d)

    def __call__(self, m0, method, iter, freqs, n_params, k_0, k_end):
        m = self.dict2vec(m0)
        method = self._method(method)
        rms = []
        k_0 = k_0 - 1
        k_end -= 1
        if k_0 + n_params > k_end:
            raise Exception("k_0 + n_params can't be larger than k_end!!")
        for c, freq in enumerate(freqs):
            m, rms0 = method(m, iter[c], freq, n_params, k_0, k_end)
            rms.append(rms0)
        return self.vec2dict(m, self.nz, self.nx), np.array(rms, dtype=object)

    def _method(self, user_method):
        if user_method in [0, "SD", "sd"]:
            raise NotImplementedError("Steepest descent is not provided yet.")
        if user_method in [1, "CG", "cg"]:
            return self.cg
        if user_method in [2, "lbfgs"]:
            return self.lbfgs
        raise ValueError("unknown optimisation method %r" % (user_method,))

    def cg(self, m0, ITER, freq, n_params=1, k0=1, k_end=2):
        """Conjugate gradient over parameters k0, k0 + n_params, ... < k_end in
        turn, ITER iterations each (fwi.py:162-195), the others held fixed."""
        if self.optimizer == "device":
            return self._device_run(device_cg.minimize, dict(gtol=1e-8, maxiter=ITER), m0, freq, n_params, k0,
                                    k_end)
        n = self.nz * self.nx
        mtotal = np.copy(m0)
        hist = []
        fun = MemoizeJac(self.fprime_single)
        for k in np.arange(k0, k_end, n_params):
            m_1, m_opt, m1 = mtotal[:k * n], mtotal[k * n:(k + n_params) * n], mtotal[(k + n_params) * n:]
            m_opt, fopt, _, _, _ = fmin_cg(fun, m_opt, fun.derivative, args=(m_1, m1, freq), gtol=1e-8, maxiter=ITER,
                                          full_output=True, disp=False)
            hist.append(fopt)
            mtotal = np.hstack((m_1, m_opt, m1))
        return mtotal, hist

    def lbfgs(self, m0, ITER, freq, n_params=1, k0=1, k_end=2):
        """L-BFGS over parameters k0, k0 + n_params, ... < k_end in turn, ITER
        iterations each (fwi.py:197-226), the others held fixed."""
        if self.optimizer == "device":
            return self._device_run(device_lbfgs.minimize, dict(m=10, factr=1e7, pgtol=1e-8, maxfun=15000,
                                                                maxiter=ITER, maxls=10), m0, freq, n_params, k0, k_end)
        n = self.nz * self.nx
        mtotal = np.copy(m0)
        hist = []
        fun = MemoizeJac(self.fprime_single)
        for k in np.arange(k0, k_end, n_params):
            m_1, m_opt, m1 = mtotal[:k * n], mtotal[k * n:(k + n_params) * n], mtotal[(k + n_params) * n:]
            m_opt, fopt, _ = fmin_l_bfgs_b(fun, m_opt, fun.derivative, args=(m_1, m1, freq), m=10, factr=1e7,
                                           pgtol=1e-8, bounds=None, maxfun=15000, maxiter=ITER,
                                           callback=None, maxls=10)
            hist.append(fopt)
            mtotal = np.hstack((m_1, m_opt, m1))
        return mtotal, hist

    def _device_run(self, minimize, settings, m0, freq, n_params, k0, k_end):
        """The parameter loop of cg / lbfgs with the optimiser on the device."""
        n = self.nz * self.nx
        mtotal = torch.from_numpy(np.asarray(m0, np.float64)).to(self.device)
        hist = []
        for k in np.arange(k0, k_end, n_params):
            m_1, m_opt, m1 = mtotal[:k * n], mtotal[k * n:(k + n_params) * n], mtotal[(k + n_params) * n:]
            res = minimize(lambda x: self.fprime_single(x, m_1, m1, freq), m_opt, **settings)
            hist.append(res.f)
            mtotal = torch.cat((m_1, res.x, m1))
        return mtotal.cpu().numpy(), hist

    def fprime(self, m0, freq):
        """Misfit and its gradient (as a vector) at model vector m0; with
        `freq` both data are low-passed first (cost_seismic, fwi.py:238-240).
        A device tensor m0 gives a device gradient."""
        if isinstance(m0, torch.Tensor) and not self._default_params:
            # user parameter functions work on numpy vectors, as in the reference
            rms, grad = self._fprime(m0.cpu().numpy(), freq)
            return rms, torch.from_numpy(grad).to(m0.device)
        return self._fprime(m0, freq)

    def _fprime(self, m0, freq):
        m_old = self.vec2dict(m0.clone() if isinstance(m0, torch.Tensor) else np.copy(m0), self.nz, self.nx)
        m_new = self.model_to_dv(m_old, self.param_functions_args)
        model = {k: self._to_device(m_new[k]) for k in ("vp", "vs", "rho")}
        rms, grad_dv = evaluate(self, model, self.d_obs, self.sd, freq)
        return self._finish(rms, grad_dv, m_old)

    def _finish(self, rms, grad_dv, m_old):
        """Gradient vector from the (vp, vs, rho) device gradient (fwi.py:243-252),
        on the device when the model vector was."""
        if not isinstance(m_old["vp"], torch.Tensor):
            grad_dv = {k: v.cpu().numpy() for k, v in grad_dv.items()}
        grad = self.grad_from_dv(grad_dv, self.param_functions_args, m_old)
        params = [*grad]
        for q in range(3):
            grad[params[q]] = grad[params[q]] * self.grad_coeff[q]
        return rms, self.dict2vec(grad)

    def fprime_single(self, m0, m_1, m1, freq):
        """Misfit and gradient of the parameters in m0, the others (m_1
        before, m1 after) fixed; the model is rounded to float32 first
        (fwi.py:255-259)."""
        if isinstance(m0, torch.Tensor):
            mtotal = torch.cat((m_1, m0, m1)).to(torch.float32)
        else:
            mtotal = np.float32(np.hstack((m_1, m0, m1)))
        s1, s0 = m_1.shape[0], m0.shape[0]
        rms, grad = self.fprime(mtotal, freq)
        return rms, grad[s1:s1 + s0]
