"""Generate the golden fixtures of the XRF projection path from the reference's own Python.

Runs the unmodified reference ``corrct`` (imported through
``oracle.reference_import`` with the restated scikit-image primitives) in FP64
on seeded synthetic slices and stores inputs and outputs as ``.npz`` files next
to this script.  Needs a local checkout of the reference (``CORRCT_SRC``);
the fixtures themselves are committed so the tests do not.

Usage: ``python tests/golden/make_golden.py``
"""

from __future__ import annotations

import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.reference_import import load_corrct  # noqa: E402
from pycorrectedemissionct_b200 import phantoms  # noqa: E402

CASES = [
    # name, N, A, detector angles, detector weights, random angle weights, seed, psf + intensities
    ("n32_a16", 32, 16, [np.pi / 2], None, False, 11, False),
    ("n33_a9", 33, 9, [np.pi / 2], None, False, 12, False),
    ("n16_a7_d2", 16, 7, [np.pi / 2, np.pi / 3], [1.0, 0.5], True, 13, False),
    ("n64_a48", 64, 48, [np.pi / 2], None, False, 14, False),
    ("n32_a16_psf", 32, 16, [np.pi / 2], None, False, 15, True),
    ("n24_a10_d2_psf", 24, 10, [np.pi / 2, 2.0], [1.0, 0.7], True, 16, True),
]
ITERATIONS = 10


def make_case(corrct, name, n, n_ang, det_angles, det_weights, rand_ang_w, seed, with_psf):
    rng = phantoms.slice_rng(seed, 0)
    x = phantoms.ellipse_phantom(n, rng, num_ellipses=6, dtype=np.float64)
    mu_in = phantoms.disk_attenuation(n, rng, mu_max=0.05, num_disks=3, dtype=np.float64)
    mu_out = 0.7 * mu_in
    angles = phantoms.angles(n_ang)
    det_angles = np.array(det_angles, dtype=np.float64)
    w_ang = rng.uniform(0.5, 1.5, size=(n_ang, len(det_angles))) if rand_ang_w else None

    angles32 = np.array(angles, dtype=np.float32)
    att = corrct.physics.attenuation.AttenuationVolume(mu_in, mu_out, angles32, det_angles, dtype=np.float64)
    att.compute_maps(use_multithreading=False, verbose=False)
    maps = att.get_maps()

    psf = np.array([0.05, 0.2, 0.5, 0.15, 0.1]) if with_psf else None
    # prj_intensities cannot be passed to the reference under numpy >= 2 (projectors.py:200 builds
    # np.array(..., dtype=np.floating), which numpy 2 rejects); the port checks them instead
    intensities = None
    common = dict(
        psf=psf,
        prj_intensities=intensities,
        att_maps=maps,
        angles_detectors_rad=det_angles,
        weights_detectors=det_weights,
        weights_angles=w_ang,
        use_multithreading=False,
        backend="skimage",
        verbose=False,
    )
    p = corrct.projectors.ProjectorAttenuationXRF((n, n), angles, **common)
    ps = corrct.projectors.ProjectorAttenuationXRF((n, n), angles, is_symmetric=True, **common)
    pu = corrct.projectors.ProjectorUncorrected((n, n), angles, backend="skimage", psf=psf, prj_intensities=intensities)

    fp_att = p.fp(x)
    y = rng.uniform(0.0, 1.0, size=fp_att.shape)
    out = dict(
        n=n,
        angles=angles,
        det_angles=det_angles,
        det_weights=np.ones(len(det_angles)) if det_weights is None else np.array(det_weights, dtype=np.float64),
        weights_angles=np.ones((n_ang, len(det_angles))) if w_ang is None else w_ang,
        x=x,
        mu_in=mu_in,
        mu_out=mu_out,
        maps=maps,
        fp_att=fp_att,
        y=y,
        psf=np.zeros(0) if psf is None else psf,
        intensities=np.zeros(0) if intensities is None else intensities,
        bp_att=p.bp(y),
        bp_sym=ps.bp(y),
        fp_unc=pu.fp(x),
        bp_unc=pu.bp(np.reshape(y, (-1, n_ang, n))[0]),
    )
    # the reference's float32 default run (maps in float32 from float32 mu), for error reporting
    att32 = corrct.physics.attenuation.AttenuationVolume(
        mu_in.astype(np.float32), mu_out.astype(np.float32), angles32, det_angles
    )
    att32.compute_maps(use_multithreading=False, verbose=False)
    out["maps_ref32"] = att32.get_maps()

    if len(det_angles) == 1:
        b = phantoms.poisson_data(fp_att, 1e4, rng, dtype=np.float64)
        out["b"] = b
        mlem = corrct.solvers.MLEM(tolerance=0.0, verbose=False)
        xm, info = mlem(p, b, iterations=ITERATIONS)
        out["mlem_x"], out["mlem_res"] = xm, info.residuals[:ITERATIONS]
        sirt = corrct.solvers.SIRT(verbose=False)
        out["sirt_x"] = sirt(p, b, iterations=ITERATIONS)[0]
        pdhg = corrct.solvers.PDHG(
            data_term="kl", regularizer=corrct.regularizers.Regularizer_TV2D(1e-2), verbose=False
        )
        out["pdhg_x"] = pdhg(p, b, iterations=ITERATIONS)[0]
    np.savez_compressed(os.path.join(HERE, f"xrf_{name}.npz"), **out)
    print(f"{name}: maps {maps.shape} fp {fp_att.shape}")


def make_surface_case(corrct):
    """Finite-surface detectors with emitted sub-sampling (attenuation.py:105-120, xrf.py:243-258):
    one 10 mm^2 detector at 50 mm and 90 degrees next to a point detector at 60 degrees, 3 sub-angles."""
    n, n_ang, sub = 32, 12, 3
    rng = phantoms.slice_rng(17, 0)
    x = phantoms.ellipse_phantom(n, rng, num_ellipses=6, dtype=np.float64)
    mu_in = phantoms.disk_attenuation(n, rng, mu_max=0.05, num_disks=3, dtype=np.float64)
    mu_out = 0.7 * mu_in
    angles32 = np.array(phantoms.angles(n_ang), dtype=np.float32)
    det = corrct.physics.xrf.DetectorXRF
    detectors = [det(surface_mm2=10.0, distance_mm=50.0, angle_rad=np.pi / 2), det(surface_mm2=0.0, distance_mm=1.0, angle_rad=np.pi / 3)]
    att = corrct.physics.attenuation.AttenuationVolume(mu_in, mu_out, angles32, detectors, emitted_sub_sampling=sub, dtype=np.float64)
    att.compute_maps(use_multithreading=False, verbose=False)
    maps = att.get_maps()
    det_angles = np.array([d.angle_rad for d in detectors])
    with corrct.projectors.ProjectorAttenuationXRF(
        (n, n), angles32, att_maps=maps, angles_detectors_rad=det_angles, use_multithreading=False, verbose=False
    ) as p:
        fp_att = p.fp(x)
    np.savez_compressed(
        os.path.join(HERE, "surface_case.npz"), n=n, angles=angles32, det_angles=det_angles,
        det_surfaces=np.array([d.surface_mm2 for d in detectors]), det_distances=np.array([d.distance_mm for d in detectors]),
        sub_sampling=sub, mu_in=mu_in, mu_out=mu_out, maps=maps, x=x, fp_att=fp_att,
    )
    print(f"surface: maps {maps.shape}")


def make_mask_case(corrct):
    """MLEM, SIRT, PDHG (KL, TV2D 1e-2) and FISTA with a data mask and a cross-validation mask
    (solvers.py:333-343, 725-805, 895-984, 1115-1206, 1395-1513), and SART with the data mask
    (solvers.py:572-629), on the n32_a16 case: 10 % of the sinogram pixels are masked out, 15 %
    held out."""
    g = np.load(os.path.join(HERE, "xrf_n32_a16.npz"))
    n, angles, b = int(g["n"]), g["angles"], g["b"]
    rng = np.random.default_rng(23)
    b_mask = (rng.uniform(size=b.shape) >= 0.1).astype(np.float64)
    b_test = (rng.uniform(size=b.shape) < 0.15).astype(np.float64)
    p = corrct.projectors.ProjectorAttenuationXRF(
        (n, n), angles, att_maps=g["maps"], angles_detectors_rad=g["det_angles"], use_multithreading=False,
        backend="skimage", verbose=False,
    )
    out = dict(b_mask=b_mask, b_test_mask=b_test)
    mlem = corrct.solvers.MLEM(tolerance=0.0, verbose=False)
    xm, info = mlem(p, b, iterations=ITERATIONS, b_mask=b_mask, b_test_mask=b_test)
    out.update(mlem_x=xm, mlem_res=info.residuals[:ITERATIONS], mlem_res_cv=info.residuals_cv[:ITERATIONS],
               mlem_res0=info.residual0, mlem_res0_cv=info.residual0_cv)
    sirt = corrct.solvers.SIRT(tolerance=0.0, verbose=False)
    xs, info = sirt(p, b, iterations=ITERATIONS, b_mask=b_mask, b_test_mask=b_test)
    out.update(sirt_x=xs, sirt_res=info.residuals[:ITERATIONS], sirt_res_cv=info.residuals_cv[:ITERATIONS],
               sirt_res0=info.residual0, sirt_res0_cv=info.residual0_cv)
    pdhg = corrct.solvers.PDHG(data_term="kl", regularizer=corrct.regularizers.Regularizer_TV2D(1e-2), tolerance=0.0, verbose=False)
    xp, info = pdhg(p, b, iterations=ITERATIONS, b_mask=b_mask, b_test_mask=b_test)
    out.update(pdhg_x=xp, pdhg_res=info.residuals[:ITERATIONS], pdhg_res_cv=info.residuals_cv[:ITERATIONS],
               pdhg_res0=info.residual0, pdhg_res0_cv=info.residual0_cv)
    fista = corrct.solvers.FISTA(tolerance=0.0, verbose=False)
    xf, info = fista(p, b, iterations=ITERATIONS, b_mask=b_mask, b_test_mask=b_test)
    out.update(fista_x=xf, fista_res=info.residuals[:ITERATIONS], fista_res_cv=info.residuals_cv[:ITERATIONS],
               fista_res0=info.residual0, fista_res0_cv=info.residual0_cv)
    # without diagonal preconditioning PDHG and FISTA scale by the operator norm from a power
    # method that starts from np.random.rand (solvers.py:26-57, 120-158)
    np.random.seed(11)
    pdhg_l = corrct.solvers.PDHG(data_term="kl", regularizer=corrct.regularizers.Regularizer_TV2D(1e-2), verbose=False)
    out["pdhg_lipschitz_x"] = pdhg_l(p, b, iterations=ITERATIONS, precondition=False)[0]
    np.random.seed(12)
    out["fista_lipschitz_x"] = corrct.solvers.FISTA(verbose=False)(p, b, iterations=ITERATIONS, precondition=False)[0]
    # SART draws its angle order from np.random (solvers.py:603); its tolerance path cannot run
    # here (compute_residual, solvers.py:503-505, subtracts (A, n) data from an (n, A) stack)
    np.random.seed(5)
    out["sart_x"] = corrct.solvers.SART(verbose=False)(p, b, iterations=3, b_mask=b_mask)[0]
    np.savez_compressed(os.path.join(HERE, "mask_case.npz"), **out)
    print(f"masks: maps {g['maps'].shape}")


def make_options_case(corrct):
    """MLEM, SIRT and PDHG (KL, TV2D 1e-2) with a solution mask and clipping limits
    (solvers.py:747-752, 800-805, 966-980, 1182-1190) on the n32_a16 case."""
    g = np.load(os.path.join(HERE, "xrf_n32_a16.npz"))
    n, angles, b = int(g["n"]), g["angles"], g["b"]
    p = corrct.projectors.ProjectorAttenuationXRF(
        (n, n), angles, att_maps=g["maps"], angles_detectors_rad=g["det_angles"], use_multithreading=False,
        backend="skimage", verbose=False,
    )
    yy, xx = np.mgrid[:n, :n]
    x_mask = (np.hypot(yy - (n - 1) / 2, xx - (n - 1) / 2) <= n / 2 - 3).astype(np.float64)
    out = dict(x_mask=x_mask)
    out["mlem_x"] = corrct.solvers.MLEM(verbose=False)(p, b, iterations=ITERATIONS, x_mask=x_mask, lower_limit=0.0,
                                                        upper_limit=2.0)[0]
    out["sirt_x"] = corrct.solvers.SIRT(verbose=False)(p, b, iterations=ITERATIONS, x_mask=x_mask, lower_limit=0.0)[0]
    pdhg = corrct.solvers.PDHG(data_term="kl", regularizer=corrct.regularizers.Regularizer_TV2D(1e-2), verbose=False)
    out["pdhg_x"] = pdhg(p, b, iterations=ITERATIONS, x_mask=x_mask, lower_limit=0.0, upper_limit=3.0)[0]
    np.savez_compressed(os.path.join(HERE, "options_case.npz"), **out)
    print(f"options: maps {g['maps'].shape}")


NOISE_CASES = [
    # name, photons, efficiency, poisson, readout std, background avg, background std, seed
    ("poisson", 1e3, 0.5, True, None, None, None, 101),
    ("background_poisson_readout", 2e3, 0.25, True, 2.0, 0.01, None, 102),
    ("background_only", 5e2, 1.0, False, None, 0.02, 0.003, 103),
]


def make_noise_golden(corrct):
    """testing.add_noise (testing.py:266-320) on a small seeded sinogram after np.random.seed."""
    rng = np.random.default_rng(7)
    clean = rng.uniform(0.0, 3.0, size=(12, 20)).astype(np.float32)
    out = {"clean": clean}
    for name, photons, eff, poisson, readout, bg_avg, bg_std, seed in NOISE_CASES:
        np.random.seed(seed)
        noisy, scaled, background = corrct.testing.add_noise(
            clean, photons, add_poisson=poisson, readout_noise_std=readout, background_avg=bg_avg,
            background_std=bg_std, detection_efficiency=eff,
        )
        out[f"{name}_noisy"], out[f"{name}_scaled"], out[f"{name}_background"] = noisy, scaled, background
    np.savez_compressed(os.path.join(HERE, "noise_cases.npz"), **out)
    print(f"noise: {len(NOISE_CASES)} cases")


def main():
    corrct = load_corrct()
    with contextlib.redirect_stdout(io.StringIO()) as log:
        for case in CASES:
            make_case(corrct, *case)
        make_noise_golden(corrct)
        make_surface_case(corrct)
        make_mask_case(corrct)
        make_options_case(corrct)
    print("\n".join(line for line in log.getvalue().splitlines() if ":" in line and ("maps" in line or "noise" in line)))


if __name__ == "__main__":
    main()
