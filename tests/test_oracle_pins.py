"""Pins of the CPU oracle against the reference's own tests.

1. tests/mf_neo_hook_operator.cc and _form1.cc (reference): on one cell of
   the unit cube with a prescribed displacement, the matrix-free cell action
   (Eulerian metric, mf_nh_operator.h physics) must equal the product of an
   independently assembled element matrix with src to 1e-10 relative
   (mf_neo_hook_operator.cc:566-572).  The displacement fields restate the
   reference's Shear / Shear2 / UniaxialTension / UniaxialTension2 /
   Rotation functions (mf_neo_hook_operator.cc:37-176).
2. tests/cook_3d_quad_mf and cook_3d_lin_mf (reference .prm + .output):
   the full load-stepping Newton solve must reproduce mesh size, volume,
   Newton iteration counts and the printed displacement (6 digits).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
MU, NU = 0.4225e6, 0.3


def _fields():
    def shear(X):
        return np.stack([X[:, 1] * 0.1, 0 * X[:, 0], 0 * X[:, 0]], 1)

    def shear2(X):
        return np.stack([X[:, 1] ** 2 * 0.1, 0 * X[:, 0], 0 * X[:, 0]], 1)

    def uni(X):
        return np.stack([X[:, 0] * 0.1, 0 * X[:, 0], 0 * X[:, 0]], 1)

    def uni2(X):
        return np.stack([X[:, 0] ** 2 * 0.1, 0 * X[:, 0], 0 * X[:, 0]], 1)

    def rotation(X):
        # rotation about z by the angle 0.6 z
        a = 0.6 * X[:, 2]
        c, s = np.cos(a), np.sin(a)
        return np.stack([c * X[:, 0] - s * X[:, 1], s * X[:, 0] + c * X[:, 1], X[:, 2]], 1)

    # (field, degree) pairs of the 3D block of the reference main()
    return [("shear", shear, 1), ("shear2", shear2, 2), ("uniaxial", uni, 1),
            ("uniaxial2", uni2, 2), ("rotation", rotation, 1)]


@pytest.mark.parametrize("name,field,p", _fields(), ids=[f[0] for f in _fields()])
@pytest.mark.parametrize("formulation,caching", [(0, "scalar"), (1, "scalar"), (1, "tensor2"), (1, "tensor4"),
                                                 (1, "scalar_referential"), (1, "tensor4_ns")])
def test_single_cell_mf_vs_matrix(name, field, p, formulation, caching):
    m = O.Mesh(O.GEOM_BOX, (1, 1, 1), 0, (0, 0, 0), (1, 1, 1), 1.0, p, p + 1)
    # the reference interpolates the field itself as the displacement (for
    # Rotation that is the rotated position, mf_neo_hook_operator.cc:166-174)
    u = field(m.X).reshape(-1)
    K = O.element_matrix(m, 0, MU, NU, formulation, u)
    rng = np.random.default_rng(1)
    src = rng.random(m.n_dofs)
    ncn = (p + 1) ** 3
    loc = np.array([src[3 * m.cell_nodes[0, a] + c] for c in range(3) for a in range(ncn)])
    ref = K @ loc
    op = O.Operator(m, caching, formulation)
    op.set_material(MU, NU)
    op.set_constraints(np.zeros(m.n_dofs, np.uint8))
    assert op.cache(u) == 0
    dst = op.vmult(src)
    got = np.array([dst[3 * m.cell_nodes[0, a] + c] for c in range(3) for a in range(ncn)])
    assert np.all(np.abs(got - ref) < 1e-10 * np.abs(ref))
    assert np.max(np.abs(K - K.T)) <= 1e-12 * np.max(np.abs(K))


def _golden():
    with open(os.path.join(HERE, "golden", "cook_3d_goldens.json")) as f:
        return json.load(f)


def _cook_args(prm):
    p = int(prm["Polynomial degree"])
    q = int(prm["Quadrature order"])
    n = int(prm["Elements per edge"])
    return dict(geometry=O.GEOM_COOK, coarse=(n, n, 1), n_refinements=0, lo=(0, 0, -0.5), hi=(48, 44, 0.5),
                scale=float(prm["Grid scale"]), p=p, q=q, caching="scalar",
                formulation=int(prm["Formulation"]), mu=float(prm["Shear modulus"]), nu=float(prm["Poisson's ratio"]),
                # 1:0,0,0 all components; 2:false,false,true (never on a face, reference quirk)
                dirichlet=[(1, 7, (0, 0, 0)), (2, 4, (0, 0, 0))],
                # 11:0,t/(16.0e-6),0
                neumann=[(11, (0, 0, 0), (0, 1.0 / 16.0e-6, 0))],
                end_time=float(prm["End time"]), dt=float(prm["Time step size"]),
                max_nr=int(prm["Max iterations Newton-Raphson"]), tol_f=float(prm["Tolerance force"]),
                tol_u=float(prm["Tolerance displacement"]), tol_lin=float(prm["Residual"]),
                max_it_mult=int(prm["Max iteration multiplier"]), precond=prm["Preconditioner type"],
                relaxation=float(prm["Preconditioner relaxation"]),
                output_point=[float(v) for v in prm["Output points"].split(",")])


@pytest.mark.parametrize("case", ["cook_3d_quad_mf", "cook_3d_lin_mf"])
def test_cook_3d_golden(case):
    g = _golden()[case]
    res = O.newton(**_cook_args(g["prm"]))
    out = g["output"]
    assert res["rc"] == 0
    assert res["n_cells"] == out["n_cells"] and res["n_dofs"] == out["n_dofs"]
    assert float("%g" % res["volume"]) == out["volume"]
    assert len(res["steps"]) == len(out["steps"])
    for s, gs in zip(res["steps"], out["steps"]):
        assert s["newton_iterations"] == gs["newton_iterations"]
        for c in range(3):
            assert float("%g" % s["point_u"][c]) == gs["displacement"][c], (case, s, gs)


def test_gmg_matches_jacobi_solution():
    """Preconditioner choice must not change the converged Newton solution."""
    kw = dict(geometry=O.GEOM_COOK, coarse=(2, 2, 1), n_refinements=1, lo=(0, 0, -5), hi=(48, 44, 5), scale=1.0,
              p=2, q=3, formulation=1, caching="tensor4", mu=80.194, nu=0.3, dirichlet=[(1, 7, (0, 0, 0))],
              neumann=[(11, (0, 0, 0), (0, 6.25, 0))], end_time=0.4, dt=0.2, tol_lin=1e-8,
              output_point=(48, 60, 5), return_u=True)
    a = O.newton(precond="jacobi", **kw)
    b = O.newton(precond="gmg", level_fp32=True, **kw)
    assert a["rc"] == 0 and b["rc"] == 0
    assert [s["newton_iterations"] for s in a["steps"]] == [s["newton_iterations"] for s in b["steps"]]
    assert np.max(np.abs(a["u"] - b["u"])) <= 1e-8 * np.max(np.abs(a["u"]))
    assert sum(s["cg_iterations"] for s in b["steps"]) < sum(s["cg_iterations"] for s in a["steps"]) / 5


def _adjoint_kw(formulation):
    # 4^3 Q2 box, bottom clamped, traction on the top face, solved tightly
    return dict(geometry=O.GEOM_BOX, coarse=(2, 2, 2), n_refinements=1, p=2, q=3,
                caching="tensor4" if formulation == 1 else "scalar", formulation=formulation, mu=1.0, nu=0.3,
                dirichlet=[(4, 7, (0, 0, 0))], neumann=[(5, (0, 0, 0), (0.02, 0, -0.05))], end_time=1.0, dt=1.0,
                tol_lin=1e-13, tol_f=1e-11, tol_u=1e-10, max_nr=25, precond="gmg", level_fp32=False)


@pytest.mark.parametrize("formulation", [0, 1])
def test_oracle_adjoint_gradient_matches_its_finite_differences(formulation):
    """The oracle's FP64 adjoint gradient (tau differentiated in mu, adjoint
    CG) against central differences of its own Newton solves: it is the
    reference gradient the device adjoint is checked against."""
    kw = _adjoint_kw(formulation)
    m = O.Mesh(O.GEOM_BOX, (2, 2, 2), 1, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    rng = np.random.default_rng(17)
    theta = rng.normal(0.0, 0.3, m.n_cells)
    target = rng.uniform(-1e-3, 1e-3, m.n_dofs)
    J, grad, u = O.adjoint(theta, target, 5, **kw)
    assert J > 0 and np.all(np.isfinite(grad)) and np.max(np.abs(grad)) > 0
    top = np.repeat(np.isclose(m.X[:, 2], 1.0), 3)
    assert abs(J - 0.5 * np.sum((u[top] - target[top]) ** 2)) <= 1e-14 * J
    h = 1e-6
    fd, ad = [], []
    for _ in range(4):
        v = rng.normal(size=m.n_cells)
        v /= np.linalg.norm(v)
        jp = O.adjoint(theta + h * v, target, 5, **kw)[0]
        jm = O.adjoint(theta - h * v, target, 5, **kw)[0]
        fd.append((jp - jm) / (2 * h))
        ad.append(grad @ v)
    fd, ad = np.array(fd), np.array(ad)
    assert np.max(np.abs(fd - ad)) <= 1e-6 * np.max(np.abs(fd)), (fd, ad)


@pytest.mark.parametrize("formulation,caching", [(1, "tensor4"), (0, "scalar"), (1, "tensor4_ns")])
def test_matrix_based_tangent_equals_matrix_free_operator(formulation, caching):
    """The reference's test method (matrix-free cell action = FEValues element
    matrix, tests/mf_neo_hook_operator.cc) on a whole 4^3 Q2 mesh with
    constraints: the assembled tangent times a vector equals the oracle's
    matrix-free vmult, and Jacobi-CG on the matrix converges like CG on the
    matrix-free operator (same iterations)."""
    m = O.Mesh(O.GEOM_BOX, (2, 2, 2), 1, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    cm = m.constraints([(4, 7), (5, 4)])
    rng = np.random.default_rng(9)
    mu = rng.choice([1.0, 10.0], m.n_cells)
    u = 0.01 * np.sin(np.pi * m.X[:, [1, 2, 0]]).reshape(-1)
    K = O.assemble_tangent(m, mu, 0.3, formulation, u, cm)
    op = O.Operator(m, caching, formulation)
    op.set_material(mu, 0.3)
    op.set_constraints(cm)
    op.cache(u)
    x = rng.uniform(-1, 1, m.n_dofs)
    assert np.max(np.abs(K @ x - op.vmult(x))) <= 1e-10 * np.max(np.abs(op.vmult(x)))
    assert abs((K - K.T).max()) <= 1e-10 * abs(K).max()     # the tangent is symmetric
    b = np.where(cm == 1, 0.0, rng.uniform(-1, 1, m.n_dofs))
    xk, itk, ok = O.cg_jacobi(K, b, 1e-10 * np.linalg.norm(b), 5000)
    assert ok and np.linalg.norm(op.vmult(xk) - b) <= 1.01e-10 * np.linalg.norm(b)


def test_oracle_cached_volume_ratio_matches_det_f():
    """The reference's consistency check of the formulation-0 cache
    (mf_nh_operator.h:1131-1156) on the oracle: JxW_ref / JxW_cur * det F = 1
    at every point, det F = c^-3 from the cached c = J^(-1/3), JxW_ref = h^3
    times the Gauss weight on the box mesh."""
    m = O.Mesh(O.GEOM_BOX, (2, 2, 2), 1, (0, 0, 0), (1, 1, 1), 1.0, 2, 3)
    rng = np.random.default_rng(4)
    op = O.Operator(m, "scalar", 0)
    op.set_material(rng.choice([1.0, 10.0], m.n_cells), 0.3)
    op.set_constraints(m.constraints([(4, 7)]))
    assert op.cache(rng.uniform(-0.01, 0.01, m.n_dofs)) == 0
    c = op.table(0).reshape(-1, 27)
    jxw = op.table(5).reshape(-1, 27)
    g = np.array([5.0, 8.0, 5.0]) / 18.0
    wq = (g[None, None, :] * g[None, :, None] * g[:, None, None]).reshape(-1)
    ratio = (0.25 ** 3 * wq[None, :]) / jxw * c ** -3.0
    assert np.max(np.abs(ratio - 1.0)) < 1e-12
