"""``dropin.install()`` on the real upstream package (CPU; skipped where the upstream sources are absent).

The upstream is imported through the fixture harness (tests/golden/_ref_harness.py: stand-ins for mpi4py, h5py
and multimethod).  Every entry point in ``dropin.PATCHES`` must be replaced by the drop-in, keep the upstream's
parameter names and order, and be restored by ``uninstall()``.  Loading libdga_b200.so needs no GPU, and no
drop-in is called here.
"""

import inspect
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))


def _harness():
    import _ref_harness as harness

    if not os.path.isdir(os.path.join(harness.REFERENCE_ROOT, "dgamore")):
        pytest.skip("the upstream sources are not present")
    harness.install()
    return harness


def _params(fn):
    fn = fn.__func__ if isinstance(fn, (staticmethod, classmethod)) else fn
    return [p.name for p in inspect.signature(fn).parameters.values()]


def test_install_replaces_every_entry_with_the_upstream_signature():
    _harness()
    import importlib

    from dgamore_b200 import dropin

    originals = {}
    for mod, cls, name, _, _ in dropin.PATCHES:
        owner = getattr(importlib.import_module(f"dgamore.{mod}"), cls) if cls else importlib.import_module(
            f"dgamore.{mod}")
        originals[(mod, cls, name)] = owner.__dict__[name] if cls else getattr(owner, name)
    replaced = dropin.install()
    try:
        assert len(replaced) == len(dropin.PATCHES)
        for (mod, cls, name, fn, _), (owner, rname, original) in zip(dropin.PATCHES, replaced):
            assert rname == name and original is originals[(mod, cls, name)]
            now = owner.__dict__[name] if cls else getattr(owner, name)
            now_fn = now.__func__ if isinstance(now, staticmethod) else now
            assert now_fn is fn, name
            assert _params(fn) == _params(original), (name, _params(fn), _params(original))
        # results are built with the upstream's classes and read the upstream config module
        four_point = importlib.import_module("dgamore.four_point")
        assert dropin._state["classes"]["FourPoint"] is four_point.FourPoint
        assert dropin._state["config"] is importlib.import_module("dgamore.config")
    finally:
        dropin.uninstall()
    for mod, cls, name, _, _ in dropin.PATCHES:
        owner = getattr(importlib.import_module(f"dgamore.{mod}"), cls) if cls else importlib.import_module(
            f"dgamore.{mod}")
        now = owner.__dict__[name] if cls else getattr(owner, name)
        assert now is originals[(mod, cls, name)], name
