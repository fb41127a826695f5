import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libcorrct_b200.so")


@pytest.fixture(scope="session")
def golden_cases():
    import glob

    import numpy as np

    return {os.path.basename(f)[4:-4]: dict(np.load(f)) for f in sorted(glob.glob(os.path.join(GOLDEN, "xrf_*.npz")))}


def rel_l2(a, b) -> float:
    import numpy as np

    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def report(name: str, value: float, bound: float) -> None:
    """Print an error against the FP64 oracle with its bound; with $CCT_PARITY_REPORT set, also
    append it there as one JSON line (the GPU runs collect these figures)."""
    import json

    line = {"case": name, "rel_l2": float(value), "bound": float(bound)}
    print(f"parity {name}: rel-L2 {value:.3e} (bound {bound:.0e})")
    path = os.environ.get("CCT_PARITY_REPORT")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(line) + "\n")
