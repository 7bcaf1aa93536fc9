"""TEST INFRASTRUCTURE ONLY -- builds the reference's own kernels for the CPU.

PyFWI's propagator kernels are OpenCL C (src/PyFWI/elastic.cl,
elastic_surface.cl, elastic_crosswell.cl).  With a short prelude that maps
``__kernel``/``__global`` away and ``get_global_id`` onto loop indices, that
source is valid C.  This module

* ``compile_program(source)``: compiles one program text (the reference's
  macro block followed by a ``.cl`` file, as ``wave_propagation.py:409-509``
  assembles it) with gcc into ``oracle/_ref/prog_<hash>.so``.  Each kernel gets
  a ``launch_<name>(g0, g1, ...)`` wrapper that runs the NDRange ``(g0, g1)``
  with OpenMP over the first dimension and the second in order, so the run is
  deterministic;
* ``macro_text(...)``: restates the macro block of wave_propagation.py:434-490;
* ``build_for(name, geometry)``: compiles the three programs for one
  geometry from the ``.cl`` files under the reference tree and records them in
  ``oracle/_ref/manifest.json`` so that a machine without the reference tree
  can still run the compiled kernels (the CPU baseline of ``bench.py``).

Nothing from the reference tree is copied into the repository: the generated
C files and libraries live only under the git-ignored ``oracle/_ref/``.
"""
import ctypes
import hashlib
import json
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REF_OUT = os.path.join(HERE, "_ref")
REF_SRC = "/root/reference/src/PyFWI"
CC = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
CFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
          "-std=gnu11", "-w"]

PRELUDE = r"""
/* generated: OpenCL C compiled as C for a CPU run of the NDRange */
static __thread long __gid0, __gid1;
#define __kernel static inline
#define __global
#define get_global_id(k) ((k) == 0 ? __gid0 : __gid1)
"""

_KERNEL_RE = re.compile(r"__kernel\s+void\s+(\w+)\s*\(([^)]*)\)", re.S)


def parse_kernels(source):
    """[(name, [(ctype, argname), ...])] for every kernel in an OpenCL text."""
    out = []
    for m in _KERNEL_RE.finditer(source):
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.replace("__global", "").split())
            if not p:
                continue
            pname = re.findall(r"(\w+)\s*$", p)[0]
            if "*" in p:
                params.append(("float*", pname))
            elif p.startswith("int"):
                params.append(("int", pname))
            elif p.startswith("float"):
                params.append(("float", pname))
            else:
                raise ValueError("unsupported kernel parameter: " + p)
        out.append((m.group(1), params))
    return out


def _wrappers(kernels):
    lines = []
    for name, params in kernels:
        sig = ", ".join(f"{t} {n}" for t, n in params)
        args = ", ".join(n for _, n in params)
        lines.append(f"void launch_{name}(long g0, long g1{', ' if sig else ''}{sig}) {{\n"
                     f"#pragma omp parallel for schedule(static)\n"
                     f"  for (long a = 0; a < g0; ++a) {{ __gid0 = a;\n"
                     f"    for (long b = 0; b < g1; ++b) {{ __gid1 = b; {name}({args}); }} }}\n}}\n")
    return "\n".join(lines)


def compile_program(source):
    """Compile one program text; return (path of the .so, kernel table)."""
    kernels = parse_kernels(source)
    key = hashlib.sha1((source + " ".join(CFLAGS)).encode()).hexdigest()[:16]
    os.makedirs(REF_OUT, exist_ok=True)
    so = os.path.join(REF_OUT, f"prog_{key}.so")
    if not os.path.exists(so):
        c = os.path.join(REF_OUT, f"prog_{key}.c")
        with open(c, "w") as f:
            f.write(PRELUDE + source + "\n" + _wrappers(kernels))
        tmp = so + f".tmp{os.getpid()}"
        subprocess.check_call([CC] + CFLAGS + ["-o", tmp, c])
        os.replace(tmp, so)
    return so, kernels


class Program:
    """Compiled reference program; ``prog.<kernel>(gsize, *args)`` runs it."""

    def __init__(self, so, kernels):
        self.lib = ctypes.CDLL(so)
        self.kernels = {}
        for name, params in kernels:
            fn = getattr(self.lib, "launch_" + name)
            types = [ctypes.c_long, ctypes.c_long]
            for t, _ in params:
                types.append({"float*": ctypes.c_void_p, "int": ctypes.c_int, "float": ctypes.c_float}[t])
            fn.argtypes = types
            fn.restype = None
            self.kernels[name] = (fn, [t for t, _ in params])

    def launch(self, name, gsize, args):
        fn, types = self.kernels[name]
        conv = []
        for t, a in zip(types, args):
            if t == "float*":
                conv.append(a)  # already an address
            elif t == "int":
                conv.append(int(a))
            else:
                conv.append(float(a))
        fn(int(gsize[0]), int(gsize[1]), *conv)


def macro_text(tnz, tnx, ns, nr, dt, dh, npml, n_main_rec, n_extera_rec, sdo, c, src_depth,
               rec_top_left_const, rec_top_left_var, rec_top_right_const, rec_top_right_var,
               rec_surface_const, rec_surface_var):
    """The macro block of wave_propagation.py:434-490 (same names, same "%d" /
    "%f" formatting, so the same constants reach the kernels)."""
    neigh = []
    for k, sfx in ((1, ""), (2, "2"), (3, "3"), (4, "4")):
        neigh.append(f"#define below{sfx} (i+{k})*Nx + (j)")
        neigh.append(f"#define above{sfx} (i-{k})*Nx + (j)")
        neigh.append(f"#define right{sfx} (i)*Nx + (j+{k})")
        neigh.append(f"#define left{sfx} (i)*Nx + (j-{k})")
    vals = [("Nz", "%d" % tnz), ("Nx", "%d" % tnx), ("Ns", "%d" % ns), ("Nr", "%d" % nr), ("dt", "%f" % dt),
            ("dx", "%f" % dh), ("dz", "%f" % dh), ("npml", "%d" % npml), ("n_main_rec", "%d" % n_main_rec),
            ("n_extera_rec", "%d" % n_extera_rec), ("sdo", "%d" % sdo), ("c1", "%f" % c[0]), ("c2", "%f" % c[1]),
            ("c3", "%f" % c[2]), ("c4", "%f" % c[3]), ("src_depth", "%d" % src_depth),
            ("rec_top_left_const", "%d" % rec_top_left_const), ("rec_top_left_var", "%d" % rec_top_left_var),
            ("rec_top_right_const", "%d" % rec_top_right_const), ("rec_top_right_var", "%d" % rec_top_right_var),
            ("rec_surface_const", "%d" % rec_surface_const), ("rec_surface_var", "%d" % rec_surface_var)]
    body = "\n".join(f"#define {k} {v}" for k, v in vals)
    return "\n" + body + "\n#define center (i)*Nx + (j)\n" + "\n".join(neigh) + "\n"


def build_for(name, **geom):
    """Compile the three programs for one geometry (needs the reference tree)
    and record them under ``name`` in the manifest."""
    macro = macro_text(**geom)
    entry = {}
    for prog, fname in (("main", "elastic.cl"), ("surface", "elastic_surface.cl"),
                        ("crosswell", "elastic_crosswell.cl")):
        with open(os.path.join(REF_SRC, fname)) as f:
            src = f.read()
        so, kernels = compile_program(macro + src)
        entry[prog] = {"so": os.path.relpath(so, HERE), "kernels": kernels}
    entry["geom"] = {k: ([float(x) for x in v] if isinstance(v, tuple) else (v.item() if hasattr(v, "item") else v))
                     for k, v in geom.items()}
    man = load_manifest()
    man[name] = entry
    with open(os.path.join(REF_OUT, "manifest.json"), "w") as f:
        json.dump(man, f, indent=1)
    return entry


def load_manifest():
    p = os.path.join(REF_OUT, "manifest.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def load_programs(name):
    """Programs recorded under ``name``: {'main': Program, 'surface': ..., 'crosswell': ...}."""
    entry = load_manifest()[name]
    return {k: Program(os.path.join(HERE, v["so"]), [(n, [tuple(p) for p in ps]) for n, ps in v["kernels"]])
            for k, v in entry.items() if k != "geom"}
