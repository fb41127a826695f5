"""CPU: host logic — geometry tables equal the oracle's scikit-image matrices, the C-ABI library
loads and exports every declared symbol, argument validation paths (no GPU compute)."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from oracle import skimage_restated as skr
from pycorrectedemissionct_b200 import geometry, phantoms


def test_fp_matrices_equal_restated_radon():
    _, deg32 = geometry.backend_angles(np.linspace(0, 2 * np.pi, 37, endpoint=False))
    for n in (16, 33, 512):
        got = geometry.fp_matrices(deg32, n)
        for ii, th in enumerate(deg32):
            ref = skr.radon_matrix(th, n)
            np.testing.assert_array_equal(got[ii], ref[:2].reshape(6).astype(np.float32))


def test_bp_trig_equal_restated_iradon():
    _, deg32 = geometry.backend_angles(np.linspace(0, 2 * np.pi, 37, endpoint=False))
    got = geometry.bp_trig(deg32)
    for ii, th in enumerate(deg32):
        c, s = skr.iradon_matrix_terms(th)
        assert got[ii, 0] == c and got[ii, 1] == s


def test_rotation_matrices_equal_restated_rotate():
    rad32, _ = geometry.backend_angles(np.linspace(0, 2 * np.pi, 11, endpoint=False))
    n = 40
    _, p = geometry.padded_size(n)
    rot_in, rot_out, n_sub = geometry.attenuation_rotations(rad32, [np.pi / 2, 1.0], n)
    assert n_sub == 1 and rot_out.shape == (11, 2, 1, 2, 6)
    for ii, a in enumerate(rad32):
        deg = np.rad2deg(a)
        np.testing.assert_array_equal(rot_in[ii, 0], skr.rotate_matrix(-deg, p, p)[:2].reshape(6))
        np.testing.assert_array_equal(rot_in[ii, 1], skr.rotate_matrix(deg, p, p)[:2].reshape(6))
        ad = a + np.array([np.pi / 2, 1.0])[1] + np.pi
        np.testing.assert_array_equal(rot_out[ii, 1, 0, 0], skr.rotate_matrix(-np.rad2deg(ad), p, p)[:2].reshape(6))


def test_padded_sizes():
    assert [geometry.padded_size(n)[1] for n in (128, 256, 384, 512, 768, 1024)] == [182, 364, 544, 726, 1088, 1450]


def test_sub_angles_follow_detector_model():
    sub = geometry.detector_sub_angles(4.0, 10.0, 4)
    half = np.arctan2(1.0, 10.0)
    np.testing.assert_allclose(sub, (np.linspace(-half, half, 5)[1:] + np.linspace(-half, half, 5)[:-1]) / 2)


def test_phantoms_are_seeded_and_inside_circle():
    a = phantoms.ellipse_phantom(64, phantoms.slice_rng(5, 2))
    b = phantoms.ellipse_phantom(64, phantoms.slice_rng(5, 2))
    np.testing.assert_array_equal(a, b)
    yy, xx = np.mgrid[:64, :64] - 31.5
    assert np.all(a[(xx**2 + yy**2) > 32**2] == 0)
    mu = phantoms.disk_attenuation(64, phantoms.slice_rng(5, 3), 0.02)
    assert mu.max() <= 0.02 and mu.min() >= 0


# ------------------------------------------------------------------------------------ C ABI
HEADER = os.path.join(ROOT, "include", "corrct_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(cct_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from pycorrectedemissionct_b200 import _lib

    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 12
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, name
    assert lib.cct_abi_version() == _lib.ABI_VERSION


def test_validation_errors_map_to_value_error():
    from pycorrectedemissionct_b200 import _lib

    lib = _lib.load()
    desc = _lib.XrfDesc()
    desc.n = 1  # invalid: must be >= 2
    desc.n_angles = desc.n_det = desc.n_slices = 1
    rc = lib.cct_fp(ctypes.byref(desc), None, None, None, None)
    assert rc == _lib.CCT_ERR_VALUE
    assert b"volume side" in lib.cct_last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)
    md = _lib.MapsDesc()
    md.n, md.n_angles, md.n_det, md.n_slices, md.n_sub = 16, 4, 1, 1, 1
    out = ctypes.c_size_t(0)
    assert lib.cct_maps_workspace_size(ctypes.byref(md), 1, ctypes.byref(out)) == _lib.CCT_ERR_VALUE  # no volumes
    md.has_in = 1
    assert lib.cct_maps_workspace_size(ctypes.byref(md), 2, ctypes.byref(out)) == _lib.CCT_OK
    p = geometry.padded_size(16)[1]
    assert out.value == 2 * (p * p + p) * 4  # W planes and the per-column constants of half-turn partners
    table = (ctypes.c_int32 * 4)(0, 2, 1, 3)
    md.pairs = ctypes.cast(table, ctypes.c_void_p)
    for bad in (0, 5):  # entries must be in [1, n_angles]
        md.n_entries = bad
        assert lib.cct_maps_workspace_size(ctypes.byref(md), 1, ctypes.byref(out)) == _lib.CCT_ERR_VALUE
        assert b"n_entries" in lib.cct_last_error()
    md.n_entries = 2
    assert lib.cct_maps_workspace_size(ctypes.byref(md), 1, ctypes.byref(out)) == _lib.CCT_OK


def test_compute_paths_need_cuda():
    import torch

    if torch.cuda.is_available():
        pytest.skip("CUDA present")
    from pycorrectedemissionct_b200 import projectors

    with pytest.raises(RuntimeError, match="CUDA"):
        projectors.ProjectorUncorrected((16, 16), np.linspace(0, np.pi, 4))


def test_subset_permutation_nests_levels():
    from pycorrectedemissionct_b200.engine import subset_permutation

    for n_ang, levels in ((720, [30, 10]), (720, [24, 8, 2]), (360, [12, 4, 1]), (90, [9, 3])):
        p = subset_permutation(n_ang, levels)
        assert sorted(p.tolist()) == list(range(n_ang))
        for k in levels:
            per = n_ang // k
            for m in range(k):
                block = p[m * per : (m + 1) * per]
                assert len(set((block % k).tolist())) == 1  # one residue class: every k-th angle
                assert np.all(np.diff(np.sort(block)) == k)
    with pytest.raises(ValueError):
        subset_permutation(720, [721])
    with pytest.raises(ValueError):
        subset_permutation(720, [10, 4])


def test_subset_ranges_for_any_angle_count():
    from pycorrectedemissionct_b200.engine import subset_permutation, subset_ranges

    for n_ang, levels in ((737, [60, 30]), (91, [9, 3]), (720, [60, 30]), (97, [7])):
        p = subset_permutation(n_ang, levels)
        for k, ranges in zip(levels, subset_ranges(n_ang, levels)):
            assert len(ranges) == k
            sizes = [r.stop - r.start for r in ranges]
            assert sum(sizes) == n_ang and max(sizes) - min(sizes) <= 1
            for r in ranges:
                assert len(set((p[r] % k).tolist())) == 1


def test_half_turn_pairs():
    from pycorrectedemissionct_b200 import geometry, phantoms

    a = np.array(phantoms.angles(720), dtype=np.float32)
    p = geometry.half_turn_pairs(a)
    assert p.shape == (360, 2) and (p[:, 1] == p[:, 0] + 360).all()
    perm = np.random.default_rng(1).permutation(720)
    q = geometry.half_turn_pairs(a[perm])
    covered = np.concatenate([q[:, 0], q[q[:, 1] >= 0, 1]])
    assert sorted(covered.tolist()) == list(range(720)) and (q[:, 1] >= 0).all()
    for i, j in q:
        d = np.mod(float(a[perm][j]) - float(a[perm][i]) - np.pi + np.pi, 2 * np.pi) - np.pi
        assert abs(d) < 1e-6
    # no partners: half-turn sets, odd counts
    assert geometry.half_turn_pairs(np.array(phantoms.angles(10, 0, np.pi), dtype=np.float32)) is None
    assert geometry.half_turn_pairs(np.array(phantoms.angles(9), dtype=np.float32)) is None
    # some partners: angles 0, 90, 180 degrees -> (0, 180) paired, 90 alone
    r = geometry.half_turn_pairs(np.array([0.0, np.pi / 2, np.pi], dtype=np.float32))
    assert r.tolist() == [[0, 2], [1, -1]]
    # a repeated angle pairs once
    r = geometry.half_turn_pairs(np.array([0.0, 0.0, np.pi], dtype=np.float32))
    assert r.tolist() == [[0, 2], [1, -1]]


def test_bench_reference_arm_contract():
    """bench.py --impl reference (the oracle port on the host cores) prints one JSON line with the
    contract's keys, on a tiny workload."""
    import json
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run(
        [sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "1",
         "--n", "16", "--angles", "8", "--slices", "1", "--cpu-sample-angles", "4"],
        capture_output=True, text=True, timeout=600, check=True,
    )
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "slices/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"] == {"value": line["value"], "unit": "slices/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling", "dtype", "config"):
        assert key in line


def test_pack_waves_and_default_schedule():
    from pycorrectedemissionct_b200 import engine, stream

    rng = np.random.default_rng(4)
    jobs = []
    for k in range(40):
        n = int(rng.choice([64, 128, 256]))
        a = int(rng.integers(30, 200))
        jobs.append(stream.Job(n, np.linspace(0, 2 * np.pi, a, endpoint=False), None, None, np.zeros((a, n), np.float32),
                               method="mlem" if k % 2 else "sirt"))
    budget = 40 << 20
    waves = stream.pack_waves(jobs, budget)
    assert sorted(id(j) for w in waves for j in w) == sorted(id(j) for j in jobs)
    for w in waves:
        assert len(w) == 1 or sum(stream.job_bytes(j) for j in w) <= budget
    flat = [j for w in waves for j in w]
    keys = [(j.method, j.n, len(j.angles)) for j in flat]
    assert keys == sorted(keys)
    # a job above the budget forms its own wave
    assert stream.pack_waves(jobs[:3], 1) == [[j] for j in sorted(jobs[:3], key=lambda j: (j.method, j.n, len(j.angles)))]
    # schedules: even subset counts of ~12 angles, the second level dividing the first
    for a in (90, 360, 720, 1440, 37):
        (k1, p1), (k2, p2) = stream.default_schedule(a)
        assert k1 % 2 == 0 and k1 % k2 == 0 and (p1, p2) == (3, 2)
        engine.subset_permutation(a, [k1, k2])
    assert stream.default_schedule(720) == [(60, 3), (30, 2)]


def test_maps_geometry_cache():
    """compute_maps' host tables: built once per geometry, least recently used dropped past 16,
    safe under concurrent callers (built here on the CPU device)."""
    import concurrent.futures as cf

    import torch

    from pycorrectedemissionct_b200 import core, geometry, phantoms

    core._MAPS_TABLES.clear()
    dev = torch.device("cpu")
    a = np.array(phantoms.angles(40), dtype=np.float32)
    t1 = core._maps_tables(dev, 32, a, [np.pi / 2], None, None, 1, True)
    t2 = core._maps_tables(dev, 32, a.copy(), [np.pi / 2], None, None, 1, True)
    assert t1 is t2
    rot_in, rot_out, n_sub = geometry.attenuation_rotations(a, [np.pi / 2], 32)
    assert np.array_equal(t1[0].numpy(), rot_in) and np.array_equal(t1[1].numpy(), rot_out) and t1[2] == n_sub
    assert np.array_equal(t1[3].numpy(), geometry.half_turn_pairs(a))
    assert core._maps_tables(dev, 32, a, [np.pi / 2], None, None, 1, False)[3] is None
    with cf.ThreadPoolExecutor(8) as ex:
        outs = list(ex.map(lambda k: core._maps_tables(dev, 16 + k % 20, a, [np.pi / 2], None, None, 1, True), range(60)))
    assert all(o[0].shape == (40, 2, 6) for o in outs)
    assert len(core._MAPS_TABLES) <= core._MAPS_TABLES_MAX
    core._MAPS_TABLES.clear()


def _column_range(ax, bx, ay, by, lim0, lim1, P, widen):
    """Mirror of the maps scan's column_support (widen=True, limits (-1, n), open) and
    column_inside (widen=False, closed limits) in csrc/cct_maps.cu."""
    import math

    tlo, thi = -1e300, 1e300
    for a, b in ((ax, bx), (ay, by)):
        if abs(b) < 1e-12:
            inside = (lim0 < a < lim1) if widen else (lim0 <= a <= lim1)
            if not inside:
                return 1, 0
        else:
            t0, t1 = (lim0 - a) / b, (lim1 - a) / b
            if t0 > t1:
                t0, t1 = t1, t0
            tlo, thi = max(tlo, t0), min(thi, t1)
    if tlo > thi:
        return 1, 0
    if widen:
        return max(0, math.floor(tlo) - 1), min(P - 1, math.ceil(thi) + 1)
    return int(max(0.0, math.ceil(tlo))), int(min(P - 1.0, math.floor(thi)))


@pytest.mark.parametrize("n,n_angles", [(2, 16), (3, 16), (16, 40), (33, 36), (512, 12), (1024, 4)])
def test_maps_scan_fast_rows_stay_inside(n, n_angles):
    """The scan kernel reads mu without per-tap tests on the rows where every lane of a warp is
    inside (0.01, n - 1.01) by the FP64 column bounds; its FP32 coordinates (FMAs) there must give
    taps in [0, n - 1] for every lane, at any angle, for the incident and emitted rotations."""
    from pycorrectedemissionct_b200 import geometry

    e, P = geometry.padded_size(n)
    angles = np.concatenate([np.linspace(0, 2 * np.pi, n_angles, endpoint=False), [np.pi / 4, np.pi / 2, 1e-7, np.pi - 1e-7]])
    rot_in, rot_out, _ = geometry.attenuation_rotations(np.array(angles, dtype=np.float32), [np.pi / 2, 1.0], n)
    mats = [rot_in[a, 0] for a in range(len(angles))] + [rot_out[a, d, 0, 0] for a in range(len(angles)) for d in range(2)]

    def fma32(a, b, c):
        return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)

    checked = 0
    for Md in mats:
        m00, m01, m02 = np.float32(Md[0]), np.float32(Md[1]), np.float32(Md[2] - e)
        m10, m11, m12 = np.float32(Md[3]), np.float32(Md[4]), np.float32(Md[5] - e)
        for w0 in range(0, P, 32):
            lanes = np.minimum(np.arange(w0, w0 + 32), P - 1)
            ilo_w, ihi_w = -1, P
            for c in lanes:
                ax, ay = Md[0] * c + Md[2] - e, Md[3] * c + Md[5] - e
                lo, hi = _column_range(ax, Md[1], ay, Md[4], -1.0, float(n), P, True)
                if lo > hi:
                    lo, hi = P, -1
                ilo, ihi = _column_range(ax, Md[1], ay, Md[4], 0.01, n - 1.01, P, False) if n >= 2 else (P, -1)
                ilo, ihi = max(ilo, lo), min(ihi, hi)
                if ilo > ihi:
                    ilo, ihi = P, -1
                ilo_w, ihi_w = max(ilo_w, ilo), min(ihi_w, ihi)
            if ilo_w > ihi_w:
                continue
            rows = np.arange(ilo_w, ihi_w + 1, dtype=np.float32)[:, None]
            fc = lanes.astype(np.float32)[None, :]
            x = fma32(m01, rows, fma32(m00, fc, m02))
            y = fma32(m11, rows, fma32(m10, fc, m12))
            fx, fy = np.floor(x), np.floor(y)
            assert fx.min() >= 0 and fx.max() <= n - 2 and fy.min() >= 0 and fy.max() <= n - 2
            checked += x.size
    # below ~64 pixels every warp holds a column whose interior is empty (the whole warp takes the
    # checked path); the benchmark's sizes use the fast rows
    assert checked > 0 or n < 64


@pytest.mark.parametrize("n,n_angles", [(2, 16), (3, 16), (16, 40), (33, 36), (130, 24), (512, 12)])
def test_maps_resample_reads_only_scanned_rows(n, n_angles):
    """The scan kernel stores a column's W only on its warp's support rows [min lo, max hi] (the
    rows outside are constant and never read); mirror the resample's FP32 positions (rotate(+phi)
    of every map pixel) and check that each of its bilinear taps inside the frame lies on a row the
    scan stored for the tap's column, for the incident and emitted rotations."""
    from pycorrectedemissionct_b200 import geometry

    e, P = geometry.padded_size(n)
    angles = np.concatenate([np.linspace(0, 2 * np.pi, n_angles, endpoint=False), [np.pi / 4, np.pi / 2, 1e-7, np.pi - 1e-7]])
    rot_in, rot_out, _ = geometry.attenuation_rotations(np.array(angles, dtype=np.float32), [np.pi / 2, 1.0], n)
    pairs = [rot_in[a] for a in range(len(angles))] + [rot_out[a, d, 0] for a in range(len(angles)) for d in range(2)]

    def fma32(a, b, c):
        return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)

    ii, jj = np.meshgrid(np.arange(n, dtype=np.float32), np.arange(n, dtype=np.float32), indexing="ij")
    X, Y = jj + np.float32(e), ii + np.float32(e)
    for mats in pairs:
        Md, Mb = mats[0], mats[1]  # rotate(-phi) of the scan, rotate(+phi) of the resample
        # rows the scan stores per column: its warp's [min lo, max hi]
        wlo = np.full(P, P, dtype=np.int64)
        whi = np.full(P, -1, dtype=np.int64)
        for w0 in range(0, P, 32):
            los, his = [], []
            for c in range(w0, min(w0 + 32, P)):
                ax, ay = Md[0] * c + Md[2] - e, Md[3] * c + Md[5] - e
                lo, hi = _column_range(ax, Md[1], ay, Md[4], -1.0, float(n), P, True)
                if lo <= hi:
                    los.append(lo)
                    his.append(hi)
            if los:
                wlo[w0:w0 + 32] = min(los)
                whi[w0:w0 + 32] = max(his)
        m = [np.float32(v) for v in Mb]
        x = fma32(m[1], Y, fma32(m[0], X, m[2]))
        y = fma32(m[4], Y, fma32(m[3], X, m[5]))
        x0, y0 = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
        for dx in (0, 1):
            for dy in (0, 1):
                c, r = (x0 + dx).ravel(), (y0 + dy).ravel()
                inside = (c >= 0) & (c < P) & (r >= 0) & (r < P)
                c, r = c[inside], r[inside]
                assert np.all((r >= wlo[c]) & (r <= whi[c])), (n, np.count_nonzero((r < wlo[c]) | (r > whi[c])))


@pytest.mark.parametrize("n", [64, 130, 512])
def test_fp_chunk_boxes_hold_every_tap(n):
    """The forward projection stages a box per 64-bin x 64-row chunk (chunk_box in
    csrc/cct_project.cu, at most 96 x 100) and reads the four taps of every sample from it without
    tests: mirror the box and the FP32 sample coordinates and check every tap is inside."""
    from pycorrectedemissionct_b200 import geometry

    TC, TR, BOX_W, BOX_H = 64, 64, 100, 96
    angles = np.concatenate([np.linspace(0, 2 * np.pi, 36, endpoint=False), [np.pi / 4, 3 * np.pi / 4, 1e-6]])
    mats = geometry.fp_matrices(np.rad2deg(np.array(angles, dtype=np.float32)), n)

    def sx(ma, mb, mc, c, r):  # sample_x: fmaf(mb, r, fmaf(ma, c, mc)) in FP32
        inner = (np.float64(ma) * np.float64(c) + np.float64(mc)).astype(np.float32)
        return (np.float64(mb) * np.float64(r) + np.float64(inner)).astype(np.float32)

    for m in mats:
        m00, m01, m02, m10, m11, m12 = (np.float32(v) for v in m)
        for c0 in range(0, n, TC):
            c_last = min(c0 + TC, n) - 1
            for r0 in range(0, n, TR):
                r_last = min(r0 + TR, n) - 1
                cs = np.array([c0, c_last, c0, c_last], dtype=np.float32)
                rs = np.array([r0, r0, r_last, r_last], dtype=np.float32)
                xs, ys = sx(m00, m01, m02, cs, rs), sx(m10, m11, m12, cs, rs)
                bx0 = (int(np.floor(xs.min())) - 1) & ~3
                bx1 = int(np.floor(xs.max())) + 2
                by0 = int(np.floor(ys.min())) - 1
                by1 = int(np.floor(ys.max())) + 2
                q4 = (bx1 - bx0) // 4 + 1
                assert 4 * q4 <= BOX_W and by1 - by0 + 1 <= BOX_H
                cc, rr = np.meshgrid(np.arange(c0, c_last + 1, dtype=np.float32), np.arange(r0, r_last + 1, dtype=np.float32))
                x, y = np.floor(sx(m00, m01, m02, cc, rr)), np.floor(sx(m10, m11, m12, cc, rr))
                assert x.min() >= bx0 and x.max() + 1 <= bx0 + 4 * q4 - 1
                assert y.min() >= by0 and y.max() + 1 <= by1


def _fma32(a, b, c):
    """fmaf in FP32 (exact product in FP64, then the sum rounded to FP32)."""
    return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)


@pytest.mark.parametrize("n", [32, 130, 512, 1000])
def test_fp_pair_staged_quads_hold_every_tap(n):
    """The two-slice forward projection (fp_pair_kernel in csrc/cct_project.cu: 64 x 32 chunks in
    boxes of at most 75 x 80) stages, per box row, only the quads that fp_row_quads finds (the
    chunk's parallelogram clipped to the row's slab, widened by 0.5 and the right tap) and reads
    the taps without tests: mirror that
    FP32 arithmetic and check that every tap of every sample lies in a staged quad of its row.
    The kernel divides with __fdividef (a few ulp): that moves the range by far less than the
    0.5 margin this check leaves."""
    from pycorrectedemissionct_b200 import geometry

    TC, EPS, MARGIN, tr = 64, np.float32(0.01), np.float32(0.5), 32
    BOX_W, BOX_H = 80, 75
    angles = np.concatenate([np.linspace(0, 2 * np.pi, 40, endpoint=False),
                             [np.pi / 4, 3 * np.pi / 4, 1e-6, np.pi / 2 + 1e-7, 0.3e-3]])
    mats = geometry.fp_matrices(np.rad2deg(np.array(angles, dtype=np.float32)), n)
    f32 = np.float32

    def row_quads(px, py, y, bx0, q4):
        ylo, yhi = f32(f32(y) - f32(1)) - EPS, f32(f32(y) + f32(1)) + EPS
        xmin, xmax = f32(3e38), f32(-3e38)
        for e in range(4):
            xa, ya, xb, yb = px[e], py[e], px[(e + 1) % 4], py[(e + 1) % 4]
            t0, t1 = f32(0), f32(1)
            dy = f32(yb - ya)
            if abs(dy) < f32(1e-6):
                if ya < ylo or ya > yhi:
                    continue
            else:
                ta, tb = f32(f32(ylo - ya) / dy), f32(f32(yhi - ya) / dy)
                if ta > tb:
                    ta, tb = tb, ta
                t0, t1 = max(ta, f32(0)), min(tb, f32(1))
                if t0 > t1:
                    continue
            x0, x1 = _fma32(t0, f32(xb - xa), xa), _fma32(t1, f32(xb - xa), xa)
            xmin, xmax = min(xmin, x0, x1), max(xmax, x0, x1)
        if xmin > xmax:
            return 1, 0
        lo = int(np.floor(f32(xmin - MARGIN))) - bx0
        hi = int(np.floor(f32(xmax + MARGIN))) + 1 - bx0
        return max(lo, 0) >> 2, min(hi >> 2, q4 - 1)

    for m in mats:
        m00, m01, m02, m10, m11, m12 = (f32(v) for v in m)
        for c0 in range(0, n, TC):
            c_last = min(c0 + TC, n) - 1
            for r0 in range(0, n, tr):
                r_last = min(r0 + tr, n) - 1
                cs = np.array([c0, c_last, c_last, c0], dtype=np.float32)   # cyclic corner order
                rs = np.array([r0, r0, r_last, r_last], dtype=np.float32)
                px = _fma32(m01, rs, _fma32(m00, cs, m02))
                py = _fma32(m11, rs, _fma32(m10, cs, m12))
                bx0 = (int(np.floor(px.min())) - 1) & ~3
                bx1 = int(np.floor(px.max())) + 2
                by0 = int(np.floor(py.min())) - 1
                by1 = int(np.floor(py.max())) + 2
                q4 = (bx1 - bx0) // 4 + 1
                bh = by1 - by0 + 1
                assert 4 * q4 <= BOX_W and bh <= BOX_H
                qlo = np.empty(bh, dtype=np.int64)
                qhi = np.empty(bh, dtype=np.int64)
                for t in range(bh):
                    qlo[t], qhi[t] = row_quads(px, py, by0 + t, bx0, q4)
                cc, rr = np.meshgrid(np.arange(c0, c_last + 1, dtype=np.float32),
                                     np.arange(r0, r_last + 1, dtype=np.float32))
                pxc = _fma32(m00, cc, m02)
                pyc = _fma32(m10, cc, m12)
                x = np.floor(_fma32(m01, rr, pxc)).astype(np.int64).ravel() - bx0
                y = np.floor(_fma32(m11, rr, pyc)).astype(np.int64).ravel()
                for dy in (0, 1):
                    row = y + dy - by0
                    assert row.min() >= 0 and row.max() < bh
                    assert ((x >> 2) >= qlo[row]).all() and (((x + 1) >> 2) <= qhi[row]).all()


def test_fp_box_strides_cut_modelled_bank_conflicts():
    """The per-angle stride selectors (geometry.fp_box_strides) stay in range and lower the
    modelled shared-memory wavefronts of the taps against the fixed strides."""
    from pycorrectedemissionct_b200 import geometry

    n = 512
    mats = geometry.fp_matrices(np.linspace(0, 360, 72, endpoint=False).astype(np.float32), n)
    sel = geometry.fp_box_strides(mats)
    assert sel.shape == (72, 2) and (sel[:, 0] == 0).all()
    assert sel[:, 1].min() >= 0 and sel[:, 1].max() <= 4

    def wavefronts(m, stride, banks, lanes, rng):
        # distinct elements per bank, the largest per phase, over random 8 x 4 lattice blocks
        lc, lr = np.arange(32) % 8, np.arange(32) // 8
        total = 0
        for _ in range(16):
            c = rng.integers(0, n - 8) + lc
            r = rng.integers(0, n - 4) + lr
            fx = np.floor(m[0] * c + m[1] * r + m[2]).astype(np.int64)
            fy = np.floor(m[3] * c + m[4] * r + m[5]).astype(np.int64)
            for dy, dx in ((0, 0), (0, 1), (1, 0), (1, 1)):
                e = (fy + dy) * stride + fx + dx
                for p0 in range(0, 32, lanes):
                    u = np.unique(e[p0:p0 + lanes])
                    total += np.bincount(np.mod(u, banks), minlength=banks).max()
        return total

    for col, (strides, banks, lanes) in list(enumerate(geometry.FP_STRIDE_CHOICES))[1:]:
        chosen = sum(wavefronts(m.astype(np.float64), strides[v], banks, lanes, np.random.default_rng(k))
                     for k, (m, v) in enumerate(zip(mats, sel[:, col])))
        fixed = sum(wavefronts(m.astype(np.float64), strides[0], banks, lanes, np.random.default_rng(k))
                    for k, m in enumerate(mats))
        assert chosen < fixed, (col, chosen, fixed)


@pytest.mark.parametrize("n", [32, 130, 512])
def test_bp_staged_bins_cover_every_lookup(n):
    """The back projection stages, per 32 x 64 pixel tile and line, 80 (value, slope) pairs from
    bin kbase = floor(tmin + K) - 1 (bp_cta in csrc/cct_project.cu) and looks a pixel's pair up
    without tests: mirror the FP32 arithmetic and check every lookup of every pixel of the tile
    (rows and columns past n included, as the kernel computes them) lands in [0, 80)."""
    from pycorrectedemissionct_b200 import geometry

    TJ, TI, KW = 32, 64, 80
    angles = np.concatenate([np.linspace(0, 2 * np.pi, 90, endpoint=False), [np.pi / 4, 1e-6, np.pi / 2 + 1e-6]])
    trig = geometry.bp_trig(np.rad2deg(np.array(angles, dtype=np.float32)))
    R = K = n // 2

    def fma32(a, b, c):
        return (np.float64(a) * np.float64(b) + np.float64(c)).astype(np.float32)

    for cs, sn in trig:
        cs, sn = np.float32(cs), np.float32(sn)
        for i0 in range(0, n, TI):
            for j0 in range(0, n, TJ):
                cj0, cj1 = np.float32(j0 - R), np.float32(j0 + TJ - 1 - R)
                ci0, ci1 = np.float32(i0 - R), np.float32(i0 + TI - 1 - R)
                ts = [fma32(cj, cs, np.float32(-(ci * sn))) for cj in (cj0, cj1) for ci in (ci0, ci1)]
                tmin = min(ts)
                kbase = int(np.floor(np.float32(tmin + np.float32(K)))) - 1
                off = np.float32(K - kbase)
                jj = np.arange(j0, j0 + TJ, dtype=np.float32)[None, :]
                ii = np.arange(i0, i0 + TI, dtype=np.float32)[:, None]
                base = fma32(jj - np.float32(R), cs, off)
                idx = np.floor(fma32(-(ii - np.float32(R)), sn, base))
                assert idx.min() >= 0 and idx.max() <= KW - 1


def test_ctypes_structs_match_the_c_header(tmp_path):
    """Every ctypes descriptor in _lib has the size and field offsets of its C struct in
    include/corrct_b200.h (compiled here with gcc)."""
    import ctypes
    import shutil
    import subprocess

    from pycorrectedemissionct_b200 import _lib

    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    pairs = {"cct_xrf_desc": _lib.XrfDesc, "cct_maps_desc": _lib.MapsDesc, "cct_noise_desc": _lib.NoiseDesc,
             "cct_conv_desc": _lib.ConvDesc, "cct_solver_state": _lib.SolverState}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "corrct_b200.h"', "int main(void) {"]
    for cname, cls in pairs.items():
        lines.append(f'  printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(root, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for cname, cls in pairs.items():
        assert got[(cname, "size")] == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert got[(cname, fname)] == getattr(cls, fname).offset, (cname, fname)


def test_get_maps_binning_matches_block_means():
    """get_maps(binning=k): crop each volume axis to a multiple of k (excess split between both
    ends, the larger half at the start) and average k x k blocks, the integer branch of corrct's
    bin_imgs(auto_crop=True) (processing/pre.py:180-231)."""
    from pycorrectedemissionct_b200 import attenuation

    rng = np.random.default_rng(4)
    maps = rng.uniform(size=(5, 2, 11, 11)).astype(np.float32)   # (A, D, y, x), 11 = 3 * 3 + 2
    got = attenuation.bin_maps(maps, 3, 2)
    assert got.shape == (5, 2, 3, 3) and got.dtype == np.float32
    crop = maps[:, :, 1:10, 1:10].astype(np.float64)              # excess 2: one pixel off each end
    want = crop.reshape(5, 2, 3, 3, 3, 3).mean(axis=(3, 5))
    np.testing.assert_allclose(got, want, rtol=1e-6)
    vol = rng.uniform(size=(3, 2, 5, 8, 8)).astype(np.float32)   # (A, D, z, y, x): all three axes
    got3 = attenuation.bin_maps(vol, 2, 3)
    want3 = vol[:, :, 1:5].astype(np.float64).reshape(3, 2, 2, 2, 4, 2, 4, 2).mean(axis=(3, 5, 7))
    np.testing.assert_allclose(got3, want3, rtol=1e-6)
    with pytest.raises(NotImplementedError):
        attenuation.bin_maps(maps, 1.5, 2)


def test_quarter_turn_quads():
    """Quads of half-turn pair entries whose emitted directions (angle + detector angle + pi) are
    incident directions inside the quad: every entry in exactly one quad, and each source index
    names the angle a quarter turn on (within float32 rounding); None when the set lacks them."""
    from pycorrectedemissionct_b200 import geometry, phantoms

    for n_ang in (16, 40, 720):
        rad32 = np.array(phantoms.angles(n_ang), dtype=np.float32)
        pairs = geometry.half_turn_pairs(rad32)
        quads = geometry.quarter_turn_quads(rad32, pairs, np.pi / 2)
        assert quads is not None and quads.shape == (n_ang // 4, 6)
        entries = np.sort(quads[:, :2].ravel())
        np.testing.assert_array_equal(entries, np.arange(len(pairs)))
        for row in quads:
            ang = [pairs[row[0], 0], pairs[row[0], 1], pairs[row[1], 0], pairs[row[1], 1]]
            for k in range(4):
                want = np.mod(np.float64(rad32[ang[k]]) + np.pi / 2 + np.pi, 2 * np.pi)
                got = np.mod(np.float64(rad32[ang[row[2 + k]]]), 2 * np.pi)
                d = abs(want - got)
                assert min(d, 2 * np.pi - d) < 1e-6
    rad32 = np.array(phantoms.angles(90), dtype=np.float32)   # 270 degrees is not in the set
    assert geometry.quarter_turn_quads(rad32, geometry.half_turn_pairs(rad32), np.pi / 2) is None
    rad32 = np.array(phantoms.angles(40), dtype=np.float32)
    assert geometry.quarter_turn_quads(rad32, geometry.half_turn_pairs(rad32), np.pi / 3) is None
    assert geometry.quarter_turn_quads(rad32, None, np.pi / 2) is None
