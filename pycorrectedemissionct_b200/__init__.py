"""B200-native attenuation-corrected emission-CT (XRF) projection path.

A drop-in projector backend for corrct's ``ProjectorAttenuationXRF`` /
``ProjectorUncorrected`` / ``AttenuationVolume`` interfaces whose forward
projection, back projection, attenuation maps and solver updates run as
hand-written sm_100a CUDA kernels behind a C-ABI shared library
(``libcorrct_b200.so``, ``include/corrct_b200.h``).  There is no CPU fallback:
every compute entry point raises if the library or a CUDA device is missing.

Public modules mirror the reference's layout: ``projectors``, ``attenuation``,
``solvers``, ``operators`` and ``backend``; ``core`` and ``engine`` hold the
batched device API (many slices per launch).
"""

__version__ = "0.1.0"

from . import phantoms  # noqa: F401  (numpy only)


def __getattr__(name):
    # heavy submodules (torch, the CUDA library) load on first use
    import importlib

    if name in ("projectors", "attenuation", "solvers", "operators", "backend", "core", "engine", "geometry", "testing"):
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
