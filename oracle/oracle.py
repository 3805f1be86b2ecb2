"""ctypes binding of the CPU oracle (oracle/_build/liborc.so).

TEST INFRASTRUCTURE ONLY: the oracle is the checker for the CUDA path.  Only
tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
The library restates davydden/large-strain-matrix-free's NeoHookOperator
(include/mf_nh_operator.h), material (include/material.h) and driver
(include/mf_elasticity.h) in plain C++; see oracle/src/oracle.h.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc.so")

GEOM_BOX, GEOM_COOK = 0, 1
CACHE = {"scalar": 0, "tensor2": 1, "tensor4": 2, "scalar_referential": 3, "tensor4_ns": 4}


def build():
    """Compile the oracle with its Makefile (g++, OpenMP)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)
        L.orc_mesh_new.restype = vp
        L.orc_mesh_new.argtypes = [ctypes.c_int, ip, ctypes.c_int, dp, dp, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, vp]
        L.orc_mesh_free.argtypes = [vp]
        L.orc_mesh_sizes.argtypes = [vp, ip]
        L.orc_mesh_arrays.argtypes = [vp, vp, vp, vp, vp]
        L.orc_mesh_volume.restype = ctypes.c_double
        L.orc_mesh_volume.argtypes = [vp]
        L.orc_mesh_constraints.argtypes = [vp, ctypes.c_int, ip, ip, vp]
        L.orc_basis.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
        L.orc_op_new.restype = vp
        L.orc_op_new.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.orc_op_free.argtypes = [vp]
        L.orc_op_set_material.argtypes = [vp, dp, ctypes.c_double]
        L.orc_op_set_constraints.argtypes = [vp, vp]
        L.orc_op_cache.restype = ctypes.c_int
        L.orc_op_cache.argtypes = [vp, vp]
        L.orc_op_vmult.argtypes = [vp, vp, vp]
        L.orc_op_apply_inhom.argtypes = [vp, vp, vp]
        L.orc_op_diagonal.argtypes = [vp, vp, vp]
        L.orc_op_cell_apply.argtypes = [vp, ctypes.c_int, vp, vp]
        L.orc_op_get_table.restype = ctypes.c_long
        L.orc_op_get_table.argtypes = [vp, ctypes.c_int, vp]
        L.orc_residual.restype = ctypes.c_double
        L.orc_residual.argtypes = [vp, dp, ctypes.c_double, ctypes.c_int, dp, ctypes.c_int, ip, dp,
                                   ctypes.c_double, vp, dp]
        L.orc_element_matrix.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_int, dp, dp]
        L.orc_transfer_new.restype = vp
        L.orc_transfer_new.argtypes = [vp, vp]
        L.orc_transfer_free.argtypes = [vp]
        L.orc_transfer_prolongate.argtypes = [vp, vp, dp, dp]
        L.orc_transfer_restrict.argtypes = [vp, vp, dp, dp]
        L.orc_transfer_interpolate.argtypes = [vp, dp, dp]
        L.orc_newton.restype = ctypes.c_int
        L.orc_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def basis(p, q):
    nodes, qp, qw = np.zeros(p + 1), np.zeros(q), np.zeros(q)
    N, D = np.zeros((q, p + 1)), np.zeros((q, p + 1))
    lib().orc_basis(p, q, _dp(nodes), _dp(qp), _dp(qw), _dp(N), _dp(D))
    return nodes, qp, qw, N, D


class Mesh:
    """Structured hex mesh (box / Cook membrane) with an optional coarse mask."""

    def __init__(self, geometry=GEOM_BOX, coarse=(1, 1, 1), level=0, lo=(0, 0, 0), hi=(1, 1, 1),
                 scale=1.0, p=2, q=3, coarse_active=None):
        self.p, self.q = p, q
        c = np.array(coarse, dtype=np.int32)
        lo_ = np.array(lo, dtype=np.float64)
        hi_ = np.array(hi, dtype=np.float64)
        mask = None
        if coarse_active is not None:
            mask = np.ascontiguousarray(coarse_active, dtype=np.uint8)
        self._mask = mask
        self.h = lib().orc_mesh_new(geometry, _ip(c), level, _dp(lo_), _dp(hi_), scale, p, q,
                                    _p(mask) if mask is not None else None)
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())
        s = np.zeros(9, dtype=np.int32)
        lib().orc_mesh_sizes(self.h, _ip(s))
        self.n_cells, self.n_nodes = int(s[0]), int(s[1])
        self.nc, self.nn, self.n_bfaces = tuple(s[2:5]), tuple(s[5:8]), int(s[8])
        self.n_dofs = 3 * self.n_nodes
        ncn = (p + 1) ** 3
        self.X = np.zeros((self.n_nodes, 3))
        self.cell_nodes = np.zeros((self.n_cells, ncn), dtype=np.int32)
        self.cell_ijk = np.zeros((self.n_cells, 3), dtype=np.int32)
        self.bfaces = np.zeros((self.n_bfaces, 3), dtype=np.int32)
        lib().orc_mesh_arrays(self.h, _p(self.X), _p(self.cell_nodes), _p(self.cell_ijk), _p(self.bfaces))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mesh_free(self.h)
            self.h = None

    def volume(self):
        return lib().orc_mesh_volume(self.h)

    def constraints(self, specs):
        """specs: list of (boundary_id, component_mask_bits) -> uint8 per dof."""
        ids = np.array([s[0] for s in specs] or [0], dtype=np.int32)
        masks = np.array([s[1] for s in specs] or [0], dtype=np.int32)
        out = np.zeros(self.n_dofs, dtype=np.uint8)
        lib().orc_mesh_constraints(self.h, len(specs), _ip(ids), _ip(masks), _p(out))
        return out


class Operator:
    """NeoHookOperator restatement: initialize / cache / vmult / compute_diagonal."""

    def __init__(self, mesh, caching="tensor4", formulation=1, fp32=False):
        self.mesh, self.fp32 = mesh, fp32
        self.dtype = np.float32 if fp32 else np.float64
        self.h = lib().orc_op_new(mesh.h, CACHE[caching], formulation, int(fp32))
        if not self.h:
            raise RuntimeError(lib().orc_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_op_free(self.h)
            self.h = None

    def set_material(self, mu_cell, nu):
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_cell, dtype=np.float64), (self.mesh.n_cells,)))
        self._mu = mu
        lib().orc_op_set_material(self.h, _dp(mu), nu)

    def set_constraints(self, mask):
        self._mask = np.ascontiguousarray(mask, dtype=np.uint8)
        lib().orc_op_set_constraints(self.h, _p(self._mask))

    def cache(self, u):
        u = np.ascontiguousarray(u, dtype=self.dtype)
        return lib().orc_op_cache(self.h, _p(u))

    def vmult(self, src):
        src = np.ascontiguousarray(src, dtype=self.dtype)
        dst = np.zeros_like(src)
        lib().orc_op_vmult(self.h, _p(dst), _p(src))
        return dst

    def apply_inhomogeneous(self, g):
        g = np.ascontiguousarray(g, dtype=self.dtype)
        dst = np.zeros_like(g)
        lib().orc_op_apply_inhom(self.h, _p(dst), _p(g))
        return dst

    def diagonal(self):
        d = np.zeros(self.mesh.n_dofs, dtype=self.dtype)
        inv = np.zeros_like(d)
        lib().orc_op_diagonal(self.h, _p(d), _p(inv))
        return d, inv

    def cell_apply(self, cell, local_in):
        li = np.ascontiguousarray(local_in, dtype=self.dtype)
        out = np.zeros_like(li)
        lib().orc_op_cell_apply(self.h, cell, _p(li), _p(out))
        return out

    def table(self, which):
        n = lib().orc_op_get_table(self.h, which, None)
        out = np.zeros(n, dtype=self.dtype)
        lib().orc_op_get_table(self.h, which, _p(out))
        return out


def residual(mesh, mu_cell, nu, formulation, u, neumann, time, cmask):
    """neumann: list of (id, a[3], b[3]) with traction a + b*t."""
    mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_cell, dtype=np.float64), (mesh.n_cells,)))
    ids = np.array([n[0] for n in neumann] or [0], dtype=np.int32)
    ab = np.array([list(n[1]) + list(n[2]) for n in neumann] or [[0] * 6], dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.float64)
    R = np.zeros(mesh.n_dofs)
    cm = np.ascontiguousarray(cmask, dtype=np.uint8)
    nrm = lib().orc_residual(mesh.h, _dp(mu), nu, formulation, _dp(u), len(neumann), _ip(ids), _dp(ab),
                             time, _p(cm), _dp(R))
    return R, nrm


def assemble_tangent(mesh, mu_cell, nu, formulation, u, cmask):
    """The matrix-based tangent of the whole mesh (FEValues-style element
    matrices summed, constrained rows and columns an identity block) as a
    scipy CSR matrix."""
    import scipy.sparse as sp
    L = lib()
    L.orc_assemble_coo.restype = ctypes.c_long
    mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_cell, dtype=np.float64), (mesh.n_cells,)))
    u = np.ascontiguousarray(u, dtype=np.float64)
    cm = np.ascontiguousarray(cmask, dtype=np.uint8)
    args = [mesh.h, _p(mu), ctypes.c_double(nu), ctypes.c_int(formulation), _p(u), _p(cm)]
    n = L.orc_assemble_coo(*args, None, None, None)
    rows, cols, vals = np.zeros(n, dtype=np.int32), np.zeros(n, dtype=np.int32), np.zeros(n)
    L.orc_assemble_coo(*args, _p(rows), _p(cols), _p(vals))
    keep = rows >= 0
    return sp.csr_matrix((vals[keep], (rows[keep], cols[keep])), shape=(mesh.n_dofs, mesh.n_dofs))


def cg_jacobi(K, b, tol_abs, max_it, omega=1.0):
    """deal.II SolverCG with PreconditionJacobi (omega D^-1) on an assembled
    matrix: g = K x - b, convergence on ||g|| <= tol_abs from x = 0.  Returns
    (x, iterations, converged)."""
    invd = omega / K.diagonal()
    x = np.zeros_like(b)
    g = -b.copy()
    res = np.linalg.norm(g)
    if res <= tol_abs:
        return x, 0, True
    h = invd * g
    d = -h
    gh = g @ h
    it = 0
    while it < max_it:
        it += 1
        h = K @ d
        alpha = gh / (d @ h)
        x += alpha * d
        g += alpha * h
        res = np.linalg.norm(g)
        if res <= tol_abs:
            return x, it, True
        h = invd * g
        gh_new = g @ h
        d = -h + (gh_new / gh) * d
        gh = gh_new
    return x, it, False


def element_matrix(mesh, cell, mu, nu, formulation, u):
    nd = 3 * (mesh.p + 1) ** 3
    K = np.zeros((nd, nd))
    u = np.ascontiguousarray(u, dtype=np.float64)
    lib().orc_element_matrix(mesh.h, cell, mu, nu, formulation, _dp(u), _dp(K))
    return K


class Transfer:
    def __init__(self, coarse, fine):
        self.c, self.f = coarse, fine
        self.h = lib().orc_transfer_new(coarse.h, fine.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_transfer_free(self.h)
            self.h = None

    def prolongate(self, ccmask, src):
        cm = np.ascontiguousarray(ccmask, dtype=np.uint8)
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros(self.f.n_dofs)
        lib().orc_transfer_prolongate(self.h, _p(cm), _dp(src), _dp(dst))
        return dst

    def restrict(self, ccmask, src):
        cm = np.ascontiguousarray(ccmask, dtype=np.uint8)
        src = np.ascontiguousarray(src, dtype=np.float64)
        dst = np.zeros(self.c.n_dofs)
        lib().orc_transfer_restrict(self.h, _p(cm), _dp(src), _dp(dst))
        return dst

    def interpolate(self, fine_u):
        fu = np.ascontiguousarray(fine_u, dtype=np.float64)
        cu = np.zeros(self.c.n_dofs)
        lib().orc_transfer_interpolate(self.h, _dp(fu), _dp(cu))
        return cu


class GMG:
    """The oracle's V-cycle preconditioner (levels 0..n_refinements)."""

    def __init__(self, geometry, coarse, n_refinements, lo, hi, scale, p, q, caching, formulation, fp32, mu_fine, nu,
                 dirichlet, u, degree=5, smoothing_range=20.0, eig_its=30, coarse_chebyshev=True,
                 coarse_accurate_eig=True, coarse_active=None):
        L = lib()
        L.orc_gmg_new.restype = ctypes.c_void_p
        L.orc_gmg_vmult.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        L.orc_gmg_level_info.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.orc_gmg_free.argtypes = [ctypes.c_void_p]
        c = np.array(coarse, dtype=np.int32)
        lo_, hi_ = np.array(lo, dtype=np.float64), np.array(hi, dtype=np.float64)
        mu = np.ascontiguousarray(mu_fine, dtype=np.float64)
        ids = np.array([d[0] for d in dirichlet] or [0], dtype=np.int32)
        masks = np.array([d[1] for d in dirichlet] or [0], dtype=np.int32)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        self._act = None if coarse_active is None else np.ascontiguousarray(coarse_active, dtype=np.uint8)
        self.h = L.orc_gmg_new(ctypes.c_int(geometry), _ip(c), ctypes.c_int(n_refinements), _dp(lo_), _dp(hi_),
                               ctypes.c_double(scale), ctypes.c_int(p), ctypes.c_int(q), ctypes.c_int(CACHE[caching]),
                               ctypes.c_int(formulation), ctypes.c_int(int(fp32)), _dp(mu), ctypes.c_double(nu),
                               ctypes.c_int(len(dirichlet)), _ip(ids), _ip(masks), _dp(uu), ctypes.c_int(degree),
                               ctypes.c_double(smoothing_range), ctypes.c_int(eig_its),
                               ctypes.c_int(int(coarse_chebyshev)), ctypes.c_int(int(coarse_accurate_eig)),
                               _p(self._act) if self._act is not None else None)
        if not self.h:
            raise RuntimeError(L.orc_last_error().decode())
        self.n = uu.size
        self.n_levels = n_refinements + 1

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_gmg_free(self.h)
            self.h = None

    def vmult(self, src):
        s = np.ascontiguousarray(src, dtype=np.float64)
        d = np.zeros_like(s)
        lib().orc_gmg_vmult(self.h, _dp(d), _dp(s))
        return d

    def level_info(self, l):
        out = np.zeros(6)
        lib().orc_gmg_level_info(self.h, l, _dp(out))
        return out


class NewtonParams(ctypes.Structure):
    _fields_ = ([(n, ctypes.c_double * 3) for n in ("lo", "hi")] +
                [(n, ctypes.c_double) for n in ("scale", "mu", "nu", "end_time", "dt", "tol_f", "tol_u",
                                                 "tol_f_abs", "tol_u_abs", "tol_lin", "relaxation",
                                                 "smoothing_range")] +
                [("output_point", ctypes.c_double * 3), ("geometry", ctypes.c_int),
                 ("coarse", ctypes.c_int * 3)] +
                [(n, ctypes.c_int) for n in ("n_refinements", "p", "q", "caching", "formulation", "max_nr",
                                              "max_it_mult", "precond", "cheb_degree", "cheb_eig_its",
                                              "coarse_chebyshev", "coarse_accurate_eig", "level_fp32",
                                              "has_output_point", "n_dirichlet", "n_neumann")] +
                [("dir_ids", ctypes.c_int * 8), ("dir_masks", ctypes.c_int * 8),
                 ("dir_values", ctypes.c_double * 24), ("neu_ids", ctypes.c_int * 8),
                 ("neu_ab", ctypes.c_double * 48)])


def _splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


def void_mask(cells, count, radius, seed, lo=(0, 0, 0), hi=(1, 1, 1)):
    """Coarse-cell mask of the heterogeneous-voids geometry (the benchmark's
    "unit cube with seeded non-overlapping spherical voids"): sphere centres
    drawn uniformly (splitmix64 stream of the seed) inside the box shrunk by
    the radius, a candidate kept when it is at least 2.5 radii from every
    kept centre, until `count` are kept; a coarse cell is removed (0) when
    its centre lies inside a sphere.  Returns uint8[cz][cy][cx] flattened,
    x fastest."""
    state = (seed * 0x2545F4914F6CDD1D + 1) & 0xFFFFFFFFFFFFFFFF
    centres, tries = [], 0
    while len(centres) < count and tries < 100000:
        tries += 1
        pt = []
        for d in range(3):
            state, z = _splitmix64(state)
            u01 = (z >> 11) * (1.0 / 9007199254740992.0)
            pt.append(lo[d] + radius + u01 * ((hi[d] - lo[d]) - 2 * radius))
        if all(np.sqrt(sum((pt[d] - c[d]) ** 2 for d in range(3))) >= 2.0 * radius * 1.25 for c in centres):
            centres.append(pt)
    nx, ny, nz = cells
    act = np.ones(nx * ny * nz, dtype=np.uint8)
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                x = (lo[0] + (i + 0.5) * (hi[0] - lo[0]) / nx, lo[1] + (j + 0.5) * (hi[1] - lo[1]) / ny,
                     lo[2] + (k + 0.5) * (hi[2] - lo[2]) / nz)
                for c in centres:
                    if sum((x[d] - c[d]) ** 2 for d in range(3)) < radius * radius:
                        act[(k * ny + j) * nx + i] = 0
    return act


def _params(geometry=GEOM_BOX, coarse=(1, 1, 1), n_refinements=0, lo=(0, 0, 0), hi=(1, 1, 1), scale=1.0,
           p=2, q=3, caching="tensor4", formulation=1, mu=1.0, nu=0.3, mu_fine=None,
           dirichlet=(), neumann=(), end_time=1.0, dt=0.1, max_nr=10, tol_f=1e-9, tol_u=1e-6,
           tol_f_abs=0.0, tol_u_abs=0.0, tol_lin=1e-6, max_it_mult=1, precond="gmg", relaxation=0.65,
           cheb_degree=5, cheb_eig_its=30, smoothing_range=20.0, coarse_chebyshev=True,
           coarse_accurate_eig=True, level_fp32=True, output_point=None):
    """The flat parameter block of orc_newton / orc_adjoint."""
    P = NewtonParams()
    for k in range(3):
        P.lo[k], P.hi[k], P.coarse[k] = lo[k], hi[k], coarse[k]
    P.scale, P.mu, P.nu, P.end_time, P.dt = scale, mu, nu, end_time, dt
    P.tol_f, P.tol_u, P.tol_f_abs, P.tol_u_abs, P.tol_lin = tol_f, tol_u, tol_f_abs, tol_u_abs, tol_lin
    P.relaxation, P.smoothing_range = relaxation, smoothing_range
    P.geometry, P.n_refinements, P.p, P.q = geometry, n_refinements, p, q
    P.caching, P.formulation, P.max_nr, P.max_it_mult = CACHE[caching], formulation, max_nr, max_it_mult
    P.precond = {"none": 0, "jacobi": 1, "gmg": 2}[precond]
    P.cheb_degree, P.cheb_eig_its = cheb_degree, cheb_eig_its
    P.coarse_chebyshev, P.coarse_accurate_eig, P.level_fp32 = int(coarse_chebyshev), int(coarse_accurate_eig), int(level_fp32)
    if output_point is not None:
        P.has_output_point = 1
        for k in range(3):
            P.output_point[k] = output_point[k]
    P.n_dirichlet = len(dirichlet)
    for i, (bid, mask, vals) in enumerate(dirichlet):
        P.dir_ids[i], P.dir_masks[i] = bid, mask
        for c in range(3):
            P.dir_values[3 * i + c] = vals[c]
    P.n_neumann = len(neumann)
    for i, (bid, a, b) in enumerate(neumann):
        P.neu_ids[i] = bid
        for c in range(3):
            P.neu_ab[6 * i + c], P.neu_ab[6 * i + 3 + c] = a[c], b[c]
    return P


def newton(geometry=GEOM_BOX, coarse=(1, 1, 1), n_refinements=0, lo=(0, 0, 0), hi=(1, 1, 1), scale=1.0,
           p=2, q=3, caching="tensor4", formulation=1, mu=1.0, nu=0.3, mu_fine=None,
           dirichlet=(), neumann=(), end_time=1.0, dt=0.1, max_nr=10, tol_f=1e-9, tol_u=1e-6,
           tol_f_abs=0.0, tol_u_abs=0.0, tol_lin=1e-6, max_it_mult=1, precond="gmg", relaxation=0.65,
           cheb_degree=5, cheb_eig_its=30, smoothing_range=20.0, coarse_chebyshev=True,
           coarse_accurate_eig=True, level_fp32=True, output_point=None, return_u=False, coarse_active=None):
    """Run the oracle's load-stepping Newton solve.

    dirichlet: list of (id, comp_mask_bits, (v0, v1, v2)) — values are the
    increment imposed at the first Newton iteration of each step.
    neumann: list of (id, a[3], b[3]) with traction a + b * t.
    coarse_active: optional coarse-cell mask (uint8, x fastest), e.g. void_mask().
    """
    P = _params(geometry, coarse, n_refinements, lo, hi, scale, p, q, caching, formulation, mu, nu, mu_fine,
                dirichlet, neumann, end_time, dt, max_nr, tol_f, tol_u, tol_f_abs, tol_u_abs, tol_lin, max_it_mult,
                precond, relaxation, cheb_degree, cheb_eig_its, smoothing_range, coarse_chebyshev,
                coarse_accurate_eig, level_fp32, output_point)
    n_cells, n_dofs, nsteps = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    vol = ctypes.c_double()
    max_steps = 1000
    steps = np.zeros((max_steps, 7))
    cg = np.zeros(100000, dtype=np.int32)
    hist = np.full((20000, 3), -1.0)
    mu_arr = None if mu_fine is None else np.ascontiguousarray(mu_fine, dtype=np.float64)
    # size the displacement output from a mesh of the same description
    act = None if coarse_active is None else np.ascontiguousarray(coarse_active, dtype=np.uint8)
    m = Mesh(geometry, coarse, n_refinements, lo, hi, scale, p, q, coarse_active=act)
    u = np.zeros(m.n_dofs)
    rc = lib().orc_newton(ctypes.byref(P), _p(mu_arr) if mu_arr is not None else None,
                          ctypes.byref(n_cells), ctypes.byref(n_dofs), ctypes.byref(vol), max_steps,
                          _p(steps), ctypes.byref(nsteps), _p(u), _p(cg), len(cg),
                          _p(act) if act is not None else None, _p(hist), len(hist))
    out = {"rc": rc, "n_cells": n_cells.value, "n_dofs": n_dofs.value, "volume": vol.value,
           "steps": [{"time": s[0], "newton_iterations": int(s[1]), "converged": bool(s[2]),
                      "point_u": s[3:6].copy(), "cg_iterations": int(s[6])}
                     for s in steps[:nsteps.value]]}
    hist = hist[hist[:, 0] >= 0]
    for i, s in enumerate(out["steps"]):
        h = hist[hist[:, 0] == i]
        s["rel_res"], s["rel_upd"] = h[:, 1].copy(), h[:, 2].copy()
    if return_u:
        out["u"] = u
    return out


def adjoint(log_mu, u_target, obj_id, coarse_active=None, **kw):
    """The oracle's FP64 adjoint gradient: forward Newton solve with mu =
    exp(log_mu) per fine cell (keyword arguments as for newton()), then
    K(u) lambda = dJ/du by CG with the FP64 V-cycle to 1e-13, then
    dJ/dlog mu_c = lambda . dR/dlog mu_c with tau differentiated in mu.
    Returns (J, grad per cell, u)."""
    keys = _params.__code__.co_varnames[:_params.__code__.co_argcount]
    P = _params(**{k: v for k, v in kw.items() if k in keys})
    act = None if coarse_active is None else np.ascontiguousarray(coarse_active, dtype=np.uint8)
    m = Mesh(P.geometry, tuple(P.coarse), P.n_refinements, tuple(P.lo), tuple(P.hi), P.scale, P.p, P.q,
             coarse_active=act)
    lm = np.ascontiguousarray(log_mu, dtype=np.float64)
    tg = np.ascontiguousarray(u_target, dtype=np.float64)
    assert lm.size == m.n_cells and tg.size == m.n_dofs
    J = ctypes.c_double()
    g = np.zeros(m.n_cells)
    u = np.zeros(m.n_dofs)
    rc = lib().orc_adjoint(ctypes.byref(P), _p(act) if act is not None else None, _p(lm), _p(tg),
                           ctypes.c_int(obj_id), ctypes.byref(J), _p(g), _p(u))
    if rc != 0:
        raise RuntimeError("oracle adjoint failed (%d): %s" % (rc, lib().orc_last_error().decode()))
    return J.value, g, u
