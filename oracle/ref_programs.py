"""TEST INFRASTRUCTURE ONLY -- compiles the reference's kernels for the
survey geometries the CPU baseline runs (see ref_build.build_for).

The geometry constants come from the oracle's restatement of the
reference set-up (oracle.OracleWavePropagator), so they are the values the
reference's own WavePreparation would bake into its macro block."""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
for p in (HERE, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)

import cases  # noqa: E402
import oracle as O  # noqa: E402
import ref_build  # noqa: E402

HOST_SAMPLE_CASES = ["c1", "c2", "c3"]


def geometry_of(case):
    inpa = case["inpa"]
    src = O.Ricker(case["src_loc"], inpa["dh"], inpa["dt"], case["src_type"])
    src.Ricker(case["fdom"])
    W = O.OracleWavePropagator(inpa, src, case["rec_loc"], case["model_est"]["vp"].shape,
                               components=case["components"], n_well_rec=case["n_well_rec"], chpr=0)
    c = W.cfg
    return W, dict(tnz=int(W.tnz), tnx=int(W.tnx), ns=int(W.ns), nr=int(W.nr), dt=W.dt, dh=W.dh,
                   npml=int(W.npml), n_main_rec=int(W.n_surface_rec), n_extera_rec=int(W.n_well_rec),
                   sdo=int(W.sdo), c=(c.c1, c.c2, c.c3, c.c4), src_depth=int(W.src_cts),
                   rec_top_left_const=int(W.rec_top_left_const), rec_top_left_var=int(W.rec_top_left_var),
                   rec_top_right_const=int(W.rec_top_right_const), rec_top_right_var=int(W.rec_top_right_var),
                   rec_surface_const=int(W.rec_surface_const), rec_surface_var=int(W.rec_surface_var))


def build_all(names=HOST_SAMPLE_CASES):
    if not os.path.isdir(ref_build.REF_SRC):
        return {}
    out = {}
    for n in names:
        _, geom = geometry_of(cases.by_name(n))
        out[n] = ref_build.build_for(n, **geom)
    return out


if __name__ == "__main__":
    print(list(build_all()))
