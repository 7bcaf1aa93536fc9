"""TEST INFRASTRUCTURE ONLY: the part of pyopencl that PyFWI's propagator
touches (context, queue, mem_flags, Buffer, enqueue_copy, Program), backed by
the reference's kernels compiled for the CPU (oracle/ref_build.py).

Buffers keep a zero guard band on both sides so that the reference kernels'
out-of-range stencil reads (rows -4..-1 and Nz..Nz+3) read zero."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
import ref_build  # noqa: E402

GUARD = 1 << 16


class mem_flags:
    READ_WRITE = 1
    READ_ONLY = 2
    WRITE_ONLY = 4
    COPY_HOST_PTR = 8
    ALLOC_HOST_PTR = 16
    USE_HOST_PTR = 32


class Context:
    pass


class CommandQueue:
    def __init__(self, ctx, *a, **k):
        self.ctx = ctx

    def finish(self):
        pass


def create_some_context(*a, **k):
    return Context()


class Buffer:
    def __init__(self, ctx, flags, size=None, hostbuf=None):
        if hostbuf is None:
            n = int(size) // 4
            data = np.zeros(n, np.float32)
        else:
            data = np.ascontiguousarray(hostbuf).reshape(-1)
            if data.dtype != np.float32:
                raise TypeError("stand-in buffers are float32 only, got %s" % data.dtype)
            n = data.size
        self._store = np.zeros(n + 2 * GUARD, np.float32)
        self.view = self._store[GUARD:GUARD + n]
        if hostbuf is not None:
            self.view[:] = data

    @property
    def address(self):
        return self.view.ctypes.data


def enqueue_copy(queue, dest, src, *a, **k):
    if isinstance(dest, np.ndarray) and isinstance(src, Buffer):
        if dest.dtype != np.float32:
            raise TypeError("copy into %s" % dest.dtype)
        dest.reshape(-1)[:] = src.view[:dest.size]
    elif isinstance(dest, Buffer) and isinstance(src, np.ndarray):
        s = np.ascontiguousarray(src).reshape(-1)
        if s.dtype != np.float32:
            raise TypeError("copy from %s" % s.dtype)
        dest.view[:s.size] = s
    else:
        raise TypeError("unsupported enqueue_copy")


class _Kernel:
    def __init__(self, prog, name):
        self.prog, self.name = prog, name

    def __call__(self, queue, gsize, lsize, *args):
        conv = [a.address if isinstance(a, Buffer) else a for a in args]
        self.prog.launch(self.name, gsize, conv)


class Program:
    def __init__(self, ctx, source):
        self.source = source

    def build(self, *a, **k):
        so, kernels = ref_build.compile_program(self.source)
        self._prog = ref_build.Program(so, kernels)
        for name, _ in kernels:
            setattr(self, name, _Kernel(self._prog, name))
        return self
