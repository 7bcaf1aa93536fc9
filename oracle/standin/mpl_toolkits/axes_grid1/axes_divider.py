"""TEST INFRASTRUCTURE ONLY: inert stand-in."""


def make_axes_locatable(*a, **k):
    raise RuntimeError("plotting is not available in the oracle stand-in")
