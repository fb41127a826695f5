"""CPU oracle for the attenuation-corrected XRF projection path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
legs of ``bench.py`` use it, and only as the checker (or as the timed CPU
baseline).  The CUDA path never routes through it.

Contents
--------
skimage_restated
    FP64-faithful restatement of the three scikit-image primitives that the
    reference's scikit-image backend calls (``radon``, ``iradon`` with no
    filter, ``rotate`` with ``order=1``).  scikit-image itself is a third-party
    dependency of the reference that is not vendored and has no pinned version
    (``requirements.txt``: ``scikit-image[data]``), and it is not installed in
    this environment, so its algorithm is restated from its published source
    semantics.
port
    A standalone numpy port of the reference's path (``compute_attenuation``,
    ``AttenuationVolume.compute_maps``, ``ProjectorAttenuationXRF.fp/bp``,
    the MLEM / SIRT / PDHG update equations), each function citing the
    reference ``file:line`` it follows.  It runs without the reference tree,
    so it travels with the repository.
reference_import
    Imports the reference's own, unmodified ``corrct`` Python from a local
    checkout with stub modules for its unavailable plotting / xraylib / pywt
    dependencies and the restated scikit-image primitives.  Used only to
    generate the golden fixtures under ``tests/golden`` (the checkout does not
    exist where the GPU tests run).

Parity status: the reference's own Python (projectors, attenuation, solvers,
data terms, regularizers) generates the golden fixtures, so the port is pinned
to the reference's code; the three scikit-image primitives underneath are a
restatement pinned only by analytic known-answer tests (column sums at 0 deg,
lattice permutations at 90 deg, hat ridges), because scikit-image is absent.
"""
