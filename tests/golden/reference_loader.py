"""Load the reference PY-BEMCS engine (``Python/physics_engine.py``) for fixture generation.

This helper runs only where the read-only reference checkout is mounted.  It never
ships to a GPU host and no product code imports it.  The GPU tests, ``smoke()`` and
``bench.py`` read only the committed ``.npz`` fixtures next to this file.

The reference imports ``taichi`` unconditionally (``Python/physics_engine.py:5``) and
picks its NumPy fallbacks when ``sys.frozen`` is set (``:9``).  Taichi is not
installed here, so a stub module with the few names the decorators touch stands in
for it.  The engine source itself is loaded unmodified.

``RecordingRandom`` replaces the module's ``np.random`` (through a proxy for the
``np`` global of the loaded module) so that every draw the reference consumes is
recorded in call order.  The oracle replays that record to reproduce a run exactly.
"""
import importlib.util
import os
import sys
import types

import numpy as np

# The reference checkout is named by the environment only (no default path):
#   PYBEMCS_REFERENCE=<checkout root> python tests/golden/make_golden.py
REFERENCE_ROOT = os.environ.get("PYBEMCS_REFERENCE", "")
ENGINE_PATH = os.path.join(REFERENCE_ROOT, "Python", "physics_engine.py") if REFERENCE_ROOT else ""


def reference_available():
    return bool(ENGINE_PATH) and os.path.isfile(ENGINE_PATH)


def _taichi_stub():
    ti = types.ModuleType("taichi")
    ti.kernel = lambda f: f
    ti.f32, ti.i32, ti.vulkan = "f32", "i32", "vulkan"
    ti.init = lambda *a, **k: None
    ti.types = types.SimpleNamespace(ndarray=lambda *a, **k: None)
    return ti


def load_engine(fp64=False, name=None):
    """Import a fresh copy of the reference engine module.

    ``fp64=True`` sets the module global ``_NP_FP`` to float64 before any simulator
    is built, which turns every particle and field array into float64 (the FP64 oracle
    mode).  Each call returns an independent module object.
    """
    if not reference_available():
        raise FileNotFoundError("set PYBEMCS_REFERENCE to the reference checkout root (found: "
                                f"{REFERENCE_ROOT!r})")
    sys.modules.setdefault("taichi", _taichi_stub())
    had_frozen = hasattr(sys, "frozen")
    old_frozen = getattr(sys, "frozen", None)
    sys.frozen = True
    try:
        modname = name or ("_pybemcs_ref_fp64" if fp64 else "_pybemcs_ref_fp32")
        spec = importlib.util.spec_from_file_location(modname, ENGINE_PATH)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
    finally:
        if had_frozen:
            sys.frozen = old_frozen
        else:
            del sys.frozen
    assert mod.USE_TAICHI is False
    if fp64:
        mod._NP_FP = np.float64
    return mod


class RecordingRandom:
    """Stand-in for ``numpy.random`` that draws from a seeded RandomState and records.

    Each entry of ``log`` is ``(method_name, ndarray_of_values)``; scalar results are
    stored as 0-d arrays.  Only the methods the engine calls are provided
    (``poisson``, ``uniform``, ``randn``, ``rand``, ``randint``).
    """

    def __init__(self, seed):
        self._rs = np.random.RandomState(seed)
        self.log = []

    def _rec(self, name, val):
        self.log.append((name, np.array(val)))
        return val

    def poisson(self, lam, size=None):
        return self._rec("poisson", self._rs.poisson(lam, size))

    def uniform(self, low=0.0, high=1.0, size=None):
        return self._rec("uniform", self._rs.uniform(low, high, size))

    def randn(self, *shape):
        return self._rec("randn", self._rs.randn(*shape))

    def rand(self, *shape):
        return self._rec("rand", self._rs.rand(*shape))

    def randint(self, low, high=None, size=None):
        return self._rec("randint", self._rs.randint(low, high, size))


class _NumpyProxy(types.ModuleType):
    def __init__(self, rnd):
        super().__init__("numpy_proxy")
        self.random = rnd

    def __getattr__(self, item):
        return getattr(np, item)


def install_recorder(mod, seed):
    """Route the loaded engine's ``np.random`` calls through a RecordingRandom."""
    rec = RecordingRandom(seed)
    mod.np = _NumpyProxy(rec)
    return rec
