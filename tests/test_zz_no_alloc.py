"""GPU: cct_compute_maps_noalloc, the attenuation-map entry point for callers that cannot
allocate device memory, against the regular cct_compute_maps (caller workspace).

Collected last on purpose (file name), and self-contained so it also passes alone in a fresh
process.  Two calls in a row with different inputs check that the shared static scratch
carries nothing from one call into the next.
"""

import ctypes

import numpy as np
import pytest

from conftest import rel_l2

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5  # the relative-L2 tolerance of the map parity tests


def _desc_and_tables(n, angles, det_angles, n_slices, dev, half_turns=False, maps_dtype="float32"):
    from pycorrectedemissionct_b200 import _lib, geometry

    rad32 = np.array(angles, dtype=np.float32)
    rot_in, rot_out, n_sub = geometry.attenuation_rotations(rad32, det_angles, n)
    rot_in_d = torch.from_numpy(np.ascontiguousarray(rot_in)).to(dev)
    rot_out_d = torch.from_numpy(np.ascontiguousarray(rot_out)).to(dev)
    d = _lib.MapsDesc()
    d.n, d.n_angles, d.n_det, d.n_slices = n, len(rad32), len(det_angles), n_slices
    d.n_sub, d.has_in, d.has_out = n_sub, 1, 1
    d.maps_dtype = _lib.CCT_DTYPE_BF16 if maps_dtype == "bfloat16" else _lib.CCT_DTYPE_F32
    d.rot_in, d.rot_out = rot_in_d.data_ptr(), rot_out_d.data_ptr()
    keep = [rot_in_d, rot_out_d]
    if half_turns:
        # entries (angle, partner = angle + pi): one rotation per direction serves both angles
        pairs = torch.from_numpy(geometry.half_turn_pairs(rad32)).to(dev)
        d.pairs, d.n_entries = pairs.data_ptr(), pairs.shape[0]
        keep.append(pairs)
    return d, keep, rad32


@pytest.mark.parametrize("half_turns,maps_dtype", [(False, "float32"), (True, "float32"), (True, "bfloat16")])
def test_noalloc_maps_match_workspace_maps_twice(half_turns, maps_dtype):
    """Two calls in a row with different inputs, each against cct_compute_maps with a caller
    workspace (same pairing and storage type): with every angle on its own, with half-turn pairs
    (the scratch then also holds the partners' per-column constants), and with BF16 maps."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pycorrectedemissionct_b200 import _lib, core, phantoms

    dev = torch.device("cuda", 0)
    lib = _lib.load()
    n, n_ang, det = 96, 40, [np.pi / 2, np.pi / 3]
    angles = phantoms.angles(n_ang)
    desc, keep, rad32 = _desc_and_tables(n, angles, det, 2, dev, half_turns, maps_dtype)
    tdt = torch.bfloat16 if maps_dtype == "bfloat16" else torch.float32
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        mus = np.stack([phantoms.disk_attenuation(n, phantoms.slice_rng(300 + 10 * call, k), 0.03) for k in range(2)])
        mu_in = torch.from_numpy(mus).to(dev)
        mu_out = (0.6 + 0.3 * call) * mu_in
        out = torch.full((2, n_ang, len(det), n, n), float("nan"), device=dev, dtype=tdt)
        rc = lib.cct_compute_maps_noalloc(
            ctypes.byref(desc), mu_in.data_ptr(), mu_out.data_ptr(), out.data_ptr(), stream
        )
        _lib.check(rc)
        ref = core.compute_maps(mu_in, mu_out, rad32, det, maps_dtype=maps_dtype, half_turns=half_turns)
        torch.cuda.synchronize(dev)
        assert torch.isfinite(out.float()).all()
        assert rel_l2(out.float().cpu().numpy(), ref.float().cpu().numpy()) < TOL


def test_noalloc_rejects_batches_beyond_the_scratch():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pycorrectedemissionct_b200 import _lib

    dev = torch.device("cuda", 0)
    lib = _lib.load()
    # n = 1024 pads to 1450: one angle of 4 slices with both directions needs ~67 MB > 32 MiB
    desc, keep, _ = _desc_and_tables(1024, np.linspace(0, np.pi, 2, endpoint=False), [np.pi / 2], 4, dev)
    dummy = torch.empty(1, device=dev)
    rc = lib.cct_compute_maps_noalloc(ctypes.byref(desc), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), None)
    assert rc == _lib.CCT_ERR_VALUE
    assert b"32 MiB" in lib.cct_last_error()
