"""The matrix-based comparison path: the GPU matrix-free operator against the
assembled FP64 tangent of the whole mesh (the oracle's FEValues-style
element matrices summed, constrained rows and columns an identity block:
assemble_system's tangent part, mf_elasticity.h:2760-2843), the CPU-side
reference the reference's matrix-based solvers work on.

* vmult of every caching variant equals K x within 1e-10 (FP64) / 2e-5
  (FP32) relative;
* CG with the Jacobi preconditioner on the GPU operator and on the assembled
  matrix (deal.II SolverCG recurrences, same tolerance) take the same number
  of iterations to within 1 and reach the same solution within 1e-8.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import lsmf  # noqa: E402
import oracle as O  # noqa: E402

VARIANTS = [("tensor4", 1), ("tensor2", 1), ("scalar", 1), ("scalar", 0), ("scalar_referential", 1),
            ("tensor4_ns", 1)]


@pytest.fixture(scope="module")
def box():
    m = O.Mesh(O.GEOM_BOX, (4, 4, 4), 1, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    spec = [(4, 7), (5, 4)]
    cm = m.constraints(spec)
    gm = lsmf.Mesh("box", (4, 4, 4), 1, degree=2)
    gm.set_dirichlet(spec)
    assert np.array_equal(gm.constraint_mask(), cm)
    rng = np.random.default_rng(31)
    mu = rng.choice([1.0, 10.0], m.n_cells)
    u = 0.01 * np.sin(np.pi * m.X[:, [1, 2, 0]]).reshape(-1)
    K = {f: O.assemble_tangent(m, mu, 0.3, f, u, cm) for f in (0, 1)}
    return m, gm, cm, mu, u, K, rng


@pytest.mark.parametrize("caching,formulation", VARIANTS)
def test_vmult_equals_assembled_tangent(box, caching, formulation, parity):
    m, gm, cm, mu, u, K, rng = box
    x = rng.uniform(-1, 1, m.n_dofs)
    want = K[formulation] @ x
    for precision, tol in (("fp64", 1e-10), ("fp32", 2e-5)):
        op = lsmf.NeoHookOperator(gm, caching, formulation, precision)
        op.set_material(mu, 0.3)
        op.cache(torch.tensor(u, device="cuda", dtype=op.dtype))
        dx = torch.tensor(x, device="cuda", dtype=op.dtype)
        out = torch.empty_like(dx)
        op.vmult(out, dx)
        got = out.double().cpu().numpy()
        parity("vmult %s f%d %s vs assembled tangent" % (caching, formulation, precision),
               np.max(np.abs(got - want)) / np.max(np.abs(want)), tol)
        assert np.max(np.abs(got - want)) <= tol * np.max(np.abs(want)), (caching, precision)


@pytest.mark.parametrize("formulation,caching", [(1, "tensor4"), (0, "scalar")])
def test_jacobi_cg_iterations_match_matrix_based(box, formulation, caching):
    m, gm, cm, mu, u, K, rng = box
    b = np.where(cm == 1, 0.0, rng.uniform(-1, 1, m.n_dofs))
    tol = 1e-10 * np.linalg.norm(b)
    xk, itk, ok = O.cg_jacobi(K[formulation], b, tol, 5000, omega=1.0)
    assert ok
    op = lsmf.NeoHookOperator(gm, caching, formulation, "fp64")
    op.set_material(mu, 0.3)
    op.cache(torch.tensor(u, device="cuda"))
    op.compute_diagonal()
    # the matrix-free diagonal is the assembled matrix's diagonal
    d = op.get_matrix_diagonal().cpu().numpy()
    assert np.max(np.abs(d - K[formulation].diagonal())) <= 1e-10 * np.max(np.abs(d))
    x = torch.zeros(m.n_dofs, dtype=torch.float64, device="cuda")
    info = lsmf.cg_solve(op, x, torch.tensor(b, device="cuda"), tol, 5000, "jacobi", omega=1.0)
    assert info["converged"]
    assert abs(info["iterations"] - itk) <= 1, (info["iterations"], itk)
    assert np.max(np.abs(x.cpu().numpy() - xk)) <= 1e-8 * np.max(np.abs(xk))
