"""TEST INFRASTRUCTURE ONLY: device listing for the CPU stand-in."""


def get_test_platforms_and_devices(*a, **k):
    return [("cpu-standin", ["cpu0"])]
