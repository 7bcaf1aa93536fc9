"""TEST INFRASTRUCTURE ONLY: inert stand-in (the reference imports matplotlib
at module level; the propagator path draws nothing unless show=True)."""
