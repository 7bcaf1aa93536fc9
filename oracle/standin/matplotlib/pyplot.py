"""TEST INFRASTRUCTURE ONLY: inert stand-in."""


def __getattr__(name):
    raise RuntimeError("plotting is not available in the oracle stand-in: " + name)
