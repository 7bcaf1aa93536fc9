"""pyfwi_b200: PyFWI's 2-D elastic propagator and adjoint-state gradient,
rebuilt for NVIDIA B200 (sm_100a).

The modules keep PyFWI's names and call signatures (``wave_propagation``,
``torchfwi``, ``fwi``, ``tl_fwi``, ``acquisition``, ``processing``,
``grad_switcher``, ``fwi_tools``) so that code written for PyFWI's propagator
and inversion path runs unchanged; the compute runs in ``libpyfwi_b200.so``
(CUDA, C ABI in include/pyfwi_b200.h).  ``lbfgs`` and ``cg`` hold the
optimisers FWI runs with their vectors on the device, ``batch`` evaluates
surveys of different sizes together, ``autotune`` picks kernel variants."""
__version__ = "0.1.0"
