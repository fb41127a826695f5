"""The drop-in, proved with the reference's own unchanged code driving the B200 path.

Two routes a corrct user can take, each checked against the golden fixtures that corrct itself
produced on its scikit-image backend (bounds: reconstructions after 10 iterations 1e-4 relative
L2, projections 1e-5):

* corrct's solvers (MLEM, SIRT, PDHG with TV2D, FISTA, SART) unchanged, given this package's
  ``ProjectorAttenuationXRF`` as their operator (corrct: ``src/corrct/solvers.py:688-805, 867-984,
  1060-1206, 1349-1513``; SART takes the per-angle callables of ``:562-567``, because its
  projector branch tests ``isinstance(A, corrct.projectors.ProjectorUncorrected)``);
* corrct's own ``ProjectorAttenuationXRF`` built with ``backend=ProjectorBackendB200()``
  (corrct accepts backend instances, ``src/corrct/projectors.py:185-186``): its fp / bp loop over
  angles and call the backend per angle.

The reference is imported through ``oracle.reference_import`` (test infrastructure): from
``$CORRCT_SRC``, else from ``baseline/_ref``; without either the tests skip.
"""

import os

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2, report

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5
TOL_RECON = 1e-4


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


@pytest.fixture(scope="module")
def corrct():
    from oracle import reference_import

    if reference_import.reference_src() is None:
        pytest.skip("the reference's corrct package is not available (set CORRCT_SRC or install it into baseline/_ref)")
    return reference_import.load_corrct()


def test_reference_solvers_on_b200_projector(golden_cases, corrct, cuda):
    from pycorrectedemissionct_b200 import projectors

    g = golden_cases["n32_a16"]
    m = dict(np.load(os.path.join(GOLDEN, "mask_case.npz")))
    n, angles, b = int(g["n"]), g["angles"], g["b"]
    p = projectors.ProjectorAttenuationXRF((n, n), angles, att_maps=g["maps"], angles_detectors_rad=g["det_angles"])
    sv = corrct.solvers
    xm, info = sv.MLEM(tolerance=0.0, verbose=False)(p, b, iterations=10)
    e = rel_l2(xm, g["mlem_x"])
    report("corrct MLEM on the B200 projector", e, TOL_RECON)
    assert e < TOL_RECON
    np.testing.assert_allclose(info.residuals[:10], g["mlem_res"], rtol=TOL_RECON)
    e = rel_l2(sv.SIRT(verbose=False)(p, b, iterations=10)[0], g["sirt_x"])
    report("corrct SIRT on the B200 projector", e, TOL_RECON)
    assert e < TOL_RECON
    pdhg = sv.PDHG(data_term="kl", regularizer=corrct.regularizers.Regularizer_TV2D(1e-2), verbose=False)
    e = rel_l2(pdhg(p, b, iterations=10)[0], g["pdhg_x"])
    report("corrct PDHG-TV on the B200 projector", e, TOL_RECON)
    assert e < TOL_RECON
    xf, info = sv.FISTA(tolerance=0.0, verbose=False)(p, b, iterations=10, b_mask=m["b_mask"], b_test_mask=m["b_test_mask"])
    e = rel_l2(xf, m["fista_x"])
    report("corrct FISTA (masks) on the B200 projector", e, TOL_RECON)
    assert e < TOL_RECON
    np.testing.assert_allclose(info.residuals_cv[:10], m["fista_res_cv"], rtol=TOL_RECON)
    np.random.seed(5)  # SART's angle order, as drawn by the reference's own run
    xa, _ = sv.SART(verbose=False)(
        lambda x, ii: p.fp_angle(x, ii), b, 3, A_num_rows=len(angles),
        At=lambda y, ii: p.bp_angle(y, ii, single_line=True), b_mask=m["b_mask"],
    )
    e = rel_l2(xa, m["sart_x"])
    report("corrct SART on the B200 projector", e, TOL_RECON)
    assert e < TOL_RECON
    # or register the class with corrct's projector ABC: corrct's SART then takes its own
    # projector branch (fp_angle / bp_angle(single_line=True)) with the B200 projector
    corrct.projectors.ProjectorAttenuationXRF.register(projectors.ProjectorAttenuationXRF)
    assert isinstance(p, corrct.projectors.ProjectorUncorrected)
    np.random.seed(5)
    xr, _ = sv.SART(verbose=False)(p, b, 3, b_mask=m["b_mask"])
    e = rel_l2(xr, m["sart_x"])
    report("corrct SART on the registered B200 projector", e, TOL_RECON)
    assert e < TOL_RECON


def test_reference_projector_with_b200_backend(golden_cases, corrct, cuda):
    from pycorrectedemissionct_b200.backend import ProjectorBackendB200

    for case in ("n32_a16", "n16_a7_d2"):
        g = golden_cases[case]
        n = int(g["n"])
        w_ang = None if np.all(g["weights_angles"] == 1) else g["weights_angles"]
        kw = dict(att_maps=g["maps"], angles_detectors_rad=g["det_angles"], weights_detectors=g["det_weights"],
                  weights_angles=w_ang, verbose=False)
        p = corrct.projectors.ProjectorAttenuationXRF((n, n), g["angles"], backend=ProjectorBackendB200(), **kw)
        ps = corrct.projectors.ProjectorAttenuationXRF((n, n), g["angles"], backend=ProjectorBackendB200(),
                                                       is_symmetric=True, **kw)
        assert isinstance(p.projector_backend, ProjectorBackendB200)
        e = rel_l2(p.fp(g["x"]), g["fp_att"])
        report(f"corrct fp, B200 backend, {case}", e, TOL)
        assert e < TOL
        assert rel_l2(p.bp(g["y"]), g["bp_att"]) < TOL
        assert rel_l2(ps.bp(g["y"]), g["bp_sym"]) < TOL
    g = golden_cases["n32_a16"]
    n = int(g["n"])
    p = corrct.projectors.ProjectorAttenuationXRF((n, n), g["angles"], backend=ProjectorBackendB200(),
                                                  att_maps=g["maps"], angles_detectors_rad=g["det_angles"],
                                                  verbose=False)
    with p:
        xm, _ = corrct.solvers.MLEM(tolerance=0.0, verbose=False)(p, g["b"], iterations=10)
        xs, _ = corrct.solvers.SIRT(verbose=False)(p, g["b"], iterations=10)
    e = rel_l2(xm, g["mlem_x"])
    report("corrct MLEM, corrct projector, B200 backend", e, TOL_RECON)
    assert e < TOL_RECON
    assert rel_l2(xs, g["sirt_x"]) < TOL_RECON
    # corrct's SART takes its per-angle path through the projector itself here
    m = dict(np.load(os.path.join(GOLDEN, "mask_case.npz")))
    np.random.seed(5)
    xa, _ = corrct.solvers.SART(verbose=False)(p, g["b"], 3, b_mask=m["b_mask"])
    e = rel_l2(xa, m["sart_x"])
    report("corrct SART, corrct projector, B200 backend", e, TOL_RECON)
    assert e < TOL_RECON
