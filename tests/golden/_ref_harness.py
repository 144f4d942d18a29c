"""Import harness for the upstream DGAmore package, used only to generate golden fixtures.

The upstream code imports three packages that are absent from this image (``mpi4py``, ``h5py`` and
``multimethod``).  This module installs minimal stand-ins for them before the first ``import dgamore``:

* ``mpi4py.MPI``: a single-rank communicator whose collectives are identities (the upstream test-suite
  does the same with its thread-based fake, ``tests/conftest.py:173-318``).
* ``h5py``: a ``File`` stand-in that accepts writes and ignores them (rank files written by
  ``dgamore/mpi_distributor.py:38-42``).
* ``multimethod``: a decorator that keeps every overload of a name and picks the first whose annotated
  positional parameter types accept the call's positional arguments (``dgamore/matsubara_frequencies.py:21-62``
  overloads ``wn``/``vn`` on whether the second argument is a float ``beta``).

``patch_fp64()`` replaces the ``IHaveMat.mat`` setter (``dgamore/n_point_base.py:64-74``, which casts every
array to complex64) with one that keeps complex128, which turns the upstream NumPy path into the FP64
reference the fixtures are generated from.

Nothing in the product imports this file; only ``make_golden.py`` does, in a container that has the upstream
sources.
"""

from __future__ import annotations

import inspect
import sys
import types

import numpy as np

import os

# Root of the upstream DGAmore sources (the directory holding the ``dgamore`` package); read from the
# DGAMORE_REFERENCE_ROOT environment variable, with the mount point of the fixture-generating container as default.
REFERENCE_ROOT = os.environ.get("DGAMORE_REFERENCE_ROOT", "/root/reference")


class _InPlace:
    def __repr__(self):
        return "IN_PLACE"


class _Request:
    def wait(self):
        return None

    Wait = wait


class _RequestNS:
    @staticmethod
    def Waitall(reqs):
        return None


class _Comm:
    """Single-rank communicator: every collective returns its own input."""

    rank = 0
    size = 1

    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1

    def Barrier(self):
        return None

    barrier = Barrier

    def bcast(self, obj, root=0):
        return obj

    def Bcast(self, buf, root=0):
        return buf

    def allgather(self, obj):
        return [obj]

    def gather(self, obj, root=0):
        return [obj]

    def scatter(self, objs, root=0):
        return objs[0]

    def Allreduce(self, sendbuf, recvbuf=None):
        if sendbuf is not _IN_PLACE:
            recvbuf[...] = sendbuf
        return recvbuf

    def Allgather(self, sendbuf, recvbuf):
        if sendbuf is not _IN_PLACE:
            recvbuf[0] = sendbuf
        return recvbuf

    def Alltoall(self, sendbuf, recvbuf):
        recvbuf[0] = sendbuf[0]
        return recvbuf

    def Gatherv(self, sendbuf, recvbuf, root=0):
        data = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
        target = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
        np.copyto(np.asarray(target).reshape(-1), np.asarray(data).reshape(-1))

    def Scatterv(self, sendbuf, recvbuf, root=0):
        data = sendbuf[0] if isinstance(sendbuf, (list, tuple)) else sendbuf
        target = recvbuf[0] if isinstance(recvbuf, (list, tuple)) else recvbuf
        np.copyto(np.asarray(target).reshape(-1), np.asarray(data).reshape(-1))

    def Isend(self, buf, dest=0, tag=0):
        self.__dict__.setdefault("_mailbox", {}).setdefault(tag, []).append(np.array(buf, copy=True))
        return _Request()

    def Irecv(self, buf, source=0, tag=0):
        queue = self.__dict__.setdefault("_mailbox", {}).get(tag, [])
        if not queue:
            raise RuntimeError("single-rank stand-in: receive without a matching send")
        np.copyto(buf, queue.pop(0))
        return _Request()


_IN_PLACE = _InPlace()


def _install_mpi4py():
    mpi = types.ModuleType("mpi4py.MPI")
    mpi.IN_PLACE = _IN_PLACE
    mpi.REQUEST_NULL = object()
    mpi.Comm = _Comm
    mpi.Intracomm = _Comm
    mpi.COMM_WORLD = _Comm()
    mpi.Request = _RequestNS
    mpi.Get_processor_name = lambda: "node0"
    mpi.DOUBLE_COMPLEX = mpi.COMPLEX = mpi.DOUBLE = mpi.FLOAT = mpi.INT = object()
    mpi.SUM = mpi.MAX = mpi.MIN = object()
    pkg = types.ModuleType("mpi4py")
    pkg.MPI = mpi
    sys.modules["mpi4py"] = pkg
    sys.modules["mpi4py.MPI"] = mpi


def _install_h5py():
    h5 = types.ModuleType("h5py")

    class File:
        def __init__(self, *a, **k):
            self._d = {}

        def __enter__(self):
            return self

        def __exit__(self, *a):
            return False

        def close(self):
            return None

        def create_dataset(self, name, *a, **k):
            self._d[name] = k.get("data")

        def __getitem__(self, k):
            return self._d[k]

        def __setitem__(self, k, v):
            self._d[k] = v

        def __contains__(self, k):
            return k in self._d

        def __delitem__(self, k):
            self._d.pop(k, None)

    h5.File = File
    sys.modules["h5py"] = h5


class _MultiMethod:
    """Keeps every overload of one name; dispatches on annotated positional parameter types."""

    def __init__(self, fn):
        self._overloads = []
        self.register(fn)

    def register(self, fn):
        func = fn.__func__ if isinstance(fn, staticmethod) else fn
        sig = inspect.signature(func)
        self._overloads.append((func, sig))
        return self

    def _matches(self, sig, args):
        params = [p for p in sig.parameters.values() if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD)]
        if len(args) > len(params):
            return False
        for value, p in zip(args, params):
            ann = p.annotation
            if ann is inspect.Parameter.empty:
                continue
            if ann is float:
                if not isinstance(value, (float, np.floating)) or isinstance(value, bool):
                    return False
            elif ann is int:
                if not isinstance(value, (int, np.integer)) or isinstance(value, bool):
                    return False
            elif ann is bool:
                if not isinstance(value, (bool, np.bool_)):
                    return False
        return True

    def __call__(self, *args, **kwargs):
        for func, sig in self._overloads:
            if self._matches(sig, args):
                return func(*args, **kwargs)
        raise TypeError(f"no overload matches {args!r}")

    def __get__(self, obj, objtype=None):
        return self


def _multimethod(fn):
    frame = inspect.currentframe().f_back
    name = (fn.__func__ if isinstance(fn, staticmethod) else fn).__name__
    existing = frame.f_locals.get(name)
    if isinstance(existing, _MultiMethod):
        return existing.register(fn)
    return _MultiMethod(fn)


def _install_multimethod():
    mm = types.ModuleType("multimethod")
    mm.multimethod = _multimethod
    sys.modules["multimethod"] = mm


_installed = False


def install():
    """Installs the stand-ins and puts the upstream sources on ``sys.path``."""
    global _installed
    if _installed:
        return
    _install_mpi4py()
    _install_h5py()
    _install_multimethod()
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    _installed = True


def patch_fp64():
    """Makes every upstream n-point object keep complex128 storage (the FP64 reference)."""
    install()
    from dgamore import n_point_base

    def _setter(self, value):
        if value is None:
            self._mat = None
            return
        value = np.asarray(value)
        self._mat = value.astype(np.complex128) if value.dtype != np.complex128 else value

    n_point_base.IHaveMat.mat = n_point_base.IHaveMat.mat.setter(_setter)


class FakeDistributor:
    """Single-rank stand-in for ``MpiDistributor`` (``dgamore/mpi_distributor.py:20-470``)."""

    def __init__(self, ntasks: int):
        self.my_rank = 0
        self.comm = _Comm()
        self.ntasks = ntasks
        self.my_slice = slice(0, ntasks)

    def scatter(self, x, *a, **k):
        return x

    def gather(self, x, *a, **k):
        return x

    def allreduce(self, x, *a, **k):
        return x

    def bcast(self, x, *a, **k):
        return x

    def barrier(self):
        return None

    def delete_file(self):
        return None
