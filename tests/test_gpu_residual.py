"""lsmf_residual (the right-hand side of assemble_system,
mf_elasticity.h:2708-2921) against the CPU oracle's residual: internal
force in FP64 (formulations 0 and 1, per-cell shear modulus), Neumann
traction over the boundary faces of the .prm, Dirichlet entries zeroed,
and the norm; on the Cook membrane (non-affine cells) and on a box.
Tolerance 1e-12 relative (max norm) for R, 1e-12 for ||R||.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402
from prm_util import prm_text  # noqa: E402

TOL = 1e-12


def _cook(formulation, scatter="atomic"):
    prm = prm_text({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Cook", "Elements per edge": 2,
        "Global refinement": 1, "Grid scale": 1, "Cook thickness": 10, "Poisson's ratio": 0.3,
        "Shear modulus": 80.194, "Formulation": formulation, "Solver type": "MF_CG", "Preconditioner type": "jacobi",
        "MF caching": "scalar", "MF scatter": scatter, "Dirichlet IDs and expressions": "1:0,0,0",
        "Dirichlet IDs and component mask": "1:true,true,true", "Neumann IDs and expressions": "11:0,6.25*t,0"})
    om = O.Mesh(O.GEOM_COOK, (2, 2, 1), 1, (0, 0, -5), (48, 44, 5), 1.0, 2, 3)
    return lsmf.Problem(prm), om, [(1, 7)], [(11, (0, 0, 0), (0, 6.25, 0))], 0.5


def _box(formulation, scatter="atomic"):
    prm = prm_text({
        "Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Type": "Box", "Box cells": "2, 2, 2",
        "Global refinement": 1, "Poisson's ratio": 0.3, "Shear modulus": 1.0, "Formulation": formulation,
        "Solver type": "MF_CG", "Preconditioner type": "gmg", "MF caching": "tensor4" if formulation else "scalar",
        "MF scatter": scatter, "Dirichlet IDs and expressions": "4:0,0,0",
        "Dirichlet IDs and component mask": "4:true,true,true",
        "Neumann IDs and expressions": "5:0.02*t,0,-0.05*t"})
    om = O.Mesh(O.GEOM_BOX, (2, 2, 2), 1, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    return lsmf.Problem(prm), om, [(4, 7)], [(5, (0, 0, 0), (0.02, 0, -0.05))], 0.7


@pytest.mark.parametrize("geom", ["cook", "box"])
@pytest.mark.parametrize("formulation", [0, 1])
@pytest.mark.parametrize("scatter", ["atomic", "colour8"])
def test_residual_matches_oracle(geom, formulation, scatter, parity):
    pb, om, dirichlet, neumann, t = (_cook if geom == "cook" else _box)(formulation, scatter)
    assert pb.n_dofs == om.n_dofs
    rng = np.random.default_rng(5)
    amp = 0.3 if geom == "cook" else 0.01
    u = rng.uniform(-amp, amp, om.n_dofs)
    mu = (80.194 if geom == "cook" else 1.0) * rng.choice([1.0, 10.0], om.n_cells)
    pb.set_mu(mu)
    cmask = om.constraints(dirichlet)
    R_ref, nrm_ref = O.residual(om, mu, 0.3, formulation, u, neumann, t, cmask)
    du = torch.tensor(u, device="cuda")
    dR = torch.full_like(du, 3.0)
    nrm = pb.residual(du, t, dR)
    R = dR.cpu().numpy()
    parity("residual %s f%d %s" % (geom, formulation, scatter), np.max(np.abs(R - R_ref)) / np.max(np.abs(R_ref)), TOL)
    assert np.max(np.abs(R - R_ref)) <= TOL * np.max(np.abs(R_ref))
    assert abs(nrm - nrm_ref) <= TOL * nrm_ref
    assert np.all(R[cmask == 1] == 0.0)
    # u = 0: only the external load remains (and the Dirichlet zeros)
    R0_ref, _ = O.residual(om, mu, 0.3, formulation, np.zeros(om.n_dofs), neumann, t, cmask)
    pb.residual(torch.zeros_like(du), t, dR)
    assert np.max(np.abs(dR.cpu().numpy() - R0_ref)) <= TOL * np.max(np.abs(R0_ref))
