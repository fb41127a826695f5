"""Import the reference's unmodified ``corrct`` Python with stubbed optional dependencies.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Used by
``tests/golden/make_golden.py`` to run the reference's own code (projectors,
attenuation, solvers, data terms, regularizers) on the CPU and record golden
fixtures, and by the drop-in tests, which run the reference's unchanged solvers
and projector classes on this package's GPU projectors.  It needs a directory
that holds the reference's ``corrct`` package: ``$CORRCT_SRC`` (a checkout's
``src`` directory), else ``baseline/_ref`` at the repository root (where
``pip install --no-deps --target baseline/_ref <checkout>`` puts it); where
neither exists ``load_corrct`` raises ``ImportError``.

The reference's ``corrct/__init__.py`` imports every submodule, which pulls in
scikit-image, matplotlib, xraylib and pywt at import time; none of them is
installed.  A meta-path finder serves placeholder modules for them.  The only
placeholders that are *called* on the projection path are
``skimage.transform.radon``, ``iradon`` and ``rotate``, which are bound to the
restatements in ``oracle.skimage_restated``; every other placeholder attribute
raises if it is ever called, so a golden fixture can never silently depend on a
stub.
"""

from __future__ import annotations

import importlib
import importlib.abc
import importlib.machinery
import os
import sys
import types

from . import skimage_restated

REPO_REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref")

_STUB_ROOTS = ("skimage", "matplotlib", "mpl_toolkits", "xraylib", "pywt")


class _Placeholder:
    """Stands in for classes/functions of absent libraries; fails loudly when used."""

    def __init__(self, name: str):
        self._name = name

    def __call__(self, *args, **kwargs):
        raise RuntimeError(f"stubbed dependency called: {self._name}")

    def __getattr__(self, item: str):
        if item.startswith("__"):
            raise AttributeError(item)
        return _Placeholder(f"{self._name}.{item}")

    def __mro_entries__(self, bases):
        return (object,)


class _StubModule(types.ModuleType):
    def __getattr__(self, item: str):
        if item.startswith("__"):
            raise AttributeError(item)
        return _Placeholder(f"{self.__name__}.{item}")


class _StubLoader(importlib.abc.Loader):
    def create_module(self, spec):
        mod = _StubModule(spec.name)
        mod.__path__ = []  # behave as a package so submodules resolve
        return mod

    def exec_module(self, module):
        name = module.__name__
        if name == "skimage":
            module.__version__ = "0.24.0"
        elif name == "skimage.transform":
            module.radon = skimage_restated.radon
            module.iradon = skimage_restated.iradon
            module.rotate = skimage_restated.rotate
        elif name == "pywt":
            module.version = types.SimpleNamespace(version="1.6.0")
        elif name == "xraylib":
            module.XRayInit = lambda: None  # called at import by physics/xraylib_helper.py:11


class _StubFinder(importlib.abc.MetaPathFinder):
    def find_spec(self, fullname, path, target=None):
        if fullname.split(".")[0] in _STUB_ROOTS:
            return importlib.machinery.ModuleSpec(fullname, _StubLoader(), is_package=True)
        return None


def reference_src() -> str | None:
    """The directory holding the reference's ``corrct`` package, or None."""
    for src in (os.environ.get("CORRCT_SRC"), REPO_REF):
        if src and os.path.isdir(os.path.join(src, "corrct")):
            return src
    return None


def load_corrct(src: str | None = None):
    """Return the reference ``corrct`` package imported from ``src`` (default: ``reference_src()``)
    with stubs installed."""
    src = src or reference_src()
    if src is None or not os.path.isdir(os.path.join(src, "corrct")):
        raise ImportError("the reference's corrct package was not found: set CORRCT_SRC to a checkout's src "
                          "directory or install it into baseline/_ref")
    if "corrct" in sys.modules:
        return sys.modules["corrct"]
    if not any(isinstance(f, _StubFinder) for f in sys.meta_path):
        sys.meta_path.insert(0, _StubFinder())
    if src not in sys.path:
        sys.path.insert(0, src)
    import io
    import contextlib

    with contextlib.redirect_stdout(io.StringIO()):  # import-time WARNING prints
        corrct = importlib.import_module("corrct")
    return corrct
