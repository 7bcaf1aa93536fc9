"""Batches of independent surveys of uneven size.

``SurveyBatch`` evaluates the misfit and gradient of several surveys —
different grids, record lengths, shot counts and receiver layouts — together
on one GPU.  Each survey's plan runs on its own CUDA stream, so the step
kernels of small surveys overlap instead of leaving the GPU idle between
launches.  Surveys whose plans are not built yet share the free device
memory in proportion to their every-step storage (cells x steps x shots),
so the first survey's layout does not take the memory the others need.
With ``graph=True`` the whole batch (every survey's forward,
residual and adjoint) is captured once into a single CUDA graph and each
later evaluation is one graph launch; models and observed data are copied
into the captured buffers first (the plans issue their launches straight
into that graph, whatever their number: the 32-survey uneven batch of the
benchmark, about 1.8 million launches, runs this way).

The reference evaluates one survey at a time (one ``WavePropagator`` per
model, wave_propagation.py:594-938); results here are the same as evaluating
each survey alone with ``WavePropagator.misfit_gradient``.
"""
import numpy as np
import torch

from .engine import require_cuda


class SurveyBatch:
    """propagators: WavePropagator objects (one per survey), all on one device."""

    def __init__(self, propagators, graph=False):
        if not propagators:
            raise ValueError("no survey")
        self.props = list(propagators)
        self.device = require_cuda(self.props[0].device)
        if any(torch.device(W.device) != self.device for W in self.props):
            raise ValueError("every survey of a batch must be on one device")
        self.streams = [torch.cuda.Stream(self.device) for _ in self.props]
        # the surveys run side by side: each keeps one launch per step (a
        # persistent cooperative grid per survey would compete for the SMs)
        for W in self.props:
            W.persist_allowed = False
            if W._plan is not None and W._plan.opts.persist:
                W._plan = None  # rebuilt on first use, without persistent loops
        self._share_memory()
        self.graph = graph
        self._graph = None
        self._inputs = None
        self._outputs = None

    def _share_memory(self, fraction=0.8):
        """Device memory caps for the surveys whose plans are not built:
        each gets its fixed need (the trace buffers the layout reserves, a
        recompute store of about 2 sqrt(nt) states of one shot, 256 MB) and a
        share of the rest in proportion to its every-step storage."""
        todo = [W for W in self.props if W._plan is None and W.memory_budget is None]
        if len(todo) < 2:
            return
        free, _ = torch.cuda.mem_get_info(self.device)
        free += torch.cuda.memory_reserved(self.device) - torch.cuda.memory_allocated(self.device)
        fixed, var = [], []
        for W in todo:
            state = 20.0 * int(W.tnz) * int(W.tnx)  # five float32 fields
            traces = 5.0 * int(W.nt_ext) * int(W.ns) * int(W.nr) * 4
            fixed.append(4 * traces + (2 * int(np.ceil(np.sqrt(int(W.nt)))) + 8) * state + (256 << 20))
            var.append(state * int(W.nt) * int(W.ns))
        spare = max(fraction * free - sum(fixed), 0.0)
        for W, f, v in zip(todo, fixed, var):
            W.memory_budget = int(f + spare * v / sum(var))

    def _run(self, models, observed, param):
        out = [None] * len(self.props)
        main = torch.cuda.current_stream(self.device)
        for q, (W, st) in enumerate(zip(self.props, self.streams)):
            st.wait_stream(main)
            with torch.cuda.stream(st):
                out[q] = W.misfit_gradient(models[q], observed[q], parameterization=param)
        for st in self.streams:
            main.wait_stream(st)
        return out

    def misfit_gradient(self, models, observed, parameterization="dv"):
        """models[q]: {'vp','vs','rho'} device tensors of survey q; observed[q]:
        its observed section dict (device tensors).  Returns a list of
        (rms, gradient dict) per survey, on the device."""
        if len(models) != len(self.props) or len(observed) != len(self.props):
            raise ValueError("one model and one observed section per survey")
        if not self.graph:
            return self._run(models, observed, parameterization)
        if self._graph is None:
            self._capture(models, observed, parameterization)
        with torch.no_grad():
            for (m_buf, o_buf), m, o in zip(self._inputs, models, observed):
                for k in m_buf:
                    m_buf[k].copy_(m[k])
                for k in o_buf:
                    o_buf[k].copy_(o[k])
        self._graph.replay()
        return [(rms.clone(), {k: v.clone() for k, v in g.items()}) for rms, g in self._outputs]

    def _capture(self, models, observed, param):
        # static input buffers; misfit_gradient sets the model from them with
        # device work only (the plans upload their constants on first use)
        self._inputs = [({k: v.detach().to(self.device, torch.float32).clone() for k, v in m.items()},
                         {k: v.detach().to(self.device, torch.float32).clone() for k, v in o.items()})
                        for m, o in zip(models, observed)]
        # one eager evaluation builds every plan and warms the kernels
        self._run([m for m, _ in self._inputs], [o for _, o in self._inputs], param)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._outputs = self._run([m for m, _ in self._inputs], [o for _, o in self._inputs], param)
        self._graph = g
