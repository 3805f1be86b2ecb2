"""Python host mirror of the reference's NeoHookOperator surface over liblsmf.

The product is liblsmf.so (hand-written sm_100a kernels + host C++ behind
the C ABI of include/lsmf.h).  This module only binds that ABI with ctypes,
using torch CUDA tensors as device buffers (plumbing): method names and
argument meanings follow NeoHookOperator (mf_nh_operator.h:147-296) —
initialize / set_material / cache / vmult / vmult_add / Tvmult /
compute_diagonal / get_matrix_diagonal_inverse / precondition_Jacobi / el /
m / n / memory_consumption / clear.  Errors raise LsmfError carrying the
lsmf_status.  There is no CPU fallback: without the library or a GPU every
call fails loudly.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblsmf.so")

CACHING = {"scalar": 0, "tensor2": 1, "tensor4": 2, "scalar_referential": 3, "tensor4_ns": 4}
GEOM = {"box": 0, "cook": 1}
SCATTER = {"atomic": 0, "colour8": 1, "nodesum": 2}
MASK_ZERO, MASK_MPI, MASK_RW, MASK_SF, MASK_QD, MASK_DEFAULT = 1, 2, 4, 8, 16, 31


class LsmfError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("lsmf status %d: %s" % (status, msg))
        self.status = status


class MeshDesc(ctypes.Structure):
    _fields_ = [("geometry", ctypes.c_int), ("coarse", ctypes.c_int * 3), ("n_refinements", ctypes.c_int),
                ("lo", ctypes.c_double * 3), ("hi", ctypes.c_double * 3), ("scale", ctypes.c_double),
                ("degree", ctypes.c_int), ("n_q_points_1d", ctypes.c_int),
                ("coarse_active", ctypes.c_void_p)]


class GmgDesc(ctypes.Structure):
    _fields_ = [("caching", ctypes.c_int), ("formulation", ctypes.c_int), ("precision", ctypes.c_int),
                ("smoother_degree", ctypes.c_int), ("smoothing_range", ctypes.c_double),
                ("eig_cg_iterations", ctypes.c_int), ("coarse_chebyshev", ctypes.c_int),
                ("coarse_accurate_eig", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("residual", ctypes.c_double), ("converged", ctypes.c_int)]


class NewtonInfo(ctypes.Structure):
    _fields_ = [("n_steps", ctypes.c_int), ("newton_iterations", ctypes.c_int * 256),
                ("cg_iterations", ctypes.c_int * 256), ("point_u", (ctypes.c_double * 3) * 256),
                ("time_residual", ctypes.c_double), ("time_setup", ctypes.c_double),
                ("time_solve", ctypes.c_double)]


_lib = None
vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)

# every function of include/lsmf.h: name -> (restype, argtypes)
SIGNATURES = {
    "lsmf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "lsmf_last_error": (ctypes.c_char_p, []),
    "lsmf_version": (ctypes.c_char_p, []),
    "lsmf_mesh_create": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.POINTER(vp)]),
    "lsmf_mesh_destroy": (None, [vp]),
    "lsmf_mesh_info": (ctypes.c_int, [vp, ctypes.c_int, ip, ip, ip]),
    "lsmf_mesh_n_levels": (ctypes.c_int, [vp]),
    "lsmf_mesh_arrays": (ctypes.c_int, [vp, ctypes.c_int, vp, vp, vp]),
    "lsmf_mesh_set_dirichlet": (ctypes.c_int, [vp, ctypes.c_int, ip, ip]),
    "lsmf_mesh_constraint_mask": (ctypes.c_int, [vp, ctypes.c_int, vp]),
    "lsmf_operator_create": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                            ctypes.POINTER(vp)]),
    "lsmf_operator_destroy": (None, [vp]),
    "lsmf_operator_set_material": (ctypes.c_int, [vp, dp, ctypes.c_double]),
    "lsmf_operator_cache": (ctypes.c_int, [vp, vp]),
    "lsmf_operator_vmult": (ctypes.c_int, [vp, vp, vp, ctypes.c_uint]),
    "lsmf_operator_vmult_add": (ctypes.c_int, [vp, vp, vp]),
    "lsmf_operator_compute_diagonal": (ctypes.c_int, [vp]),
    "lsmf_operator_get_diagonal": (ctypes.c_int, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp)]),
    "lsmf_operator_precondition_jacobi": (ctypes.c_int, [vp, vp, vp, ctypes.c_double]),
    "lsmf_operator_m": (ctypes.c_int, [vp]),
    "lsmf_operator_n": (ctypes.c_int, [vp]),
    "lsmf_operator_el": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, dp]),
    "lsmf_operator_memory_consumption": (ctypes.c_size_t, [vp]),
    "lsmf_operator_set_stream": (ctypes.c_int, [vp, vp]),
    "lsmf_operator_set_option": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    "lsmf_operator_sync": (ctypes.c_int, [vp]),
    "lsmf_operator_get_table": (ctypes.c_int, [vp, ctypes.c_int, dp, ctypes.POINTER(ctypes.c_size_t)]),
    "lsmf_gmg_create": (ctypes.c_int, [vp, ctypes.POINTER(GmgDesc), ctypes.POINTER(vp)]),
    "lsmf_gmg_destroy": (None, [vp]),
    "lsmf_gmg_set_material": (ctypes.c_int, [vp, dp, ctypes.c_double]),
    "lsmf_gmg_setup": (ctypes.c_int, [vp, vp]),
    "lsmf_gmg_vmult": (ctypes.c_int, [vp, vp, vp]),
    "lsmf_gmg_level_info": (ctypes.c_int, [vp, ctypes.c_int, dp]),
    "lsmf_gmg_set_stream": (ctypes.c_int, [vp, vp]),
    "lsmf_gmg_set_option": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int]),
    "lsmf_gmg_level_operator": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(vp)]),
    "lsmf_cg_solve": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, vp, vp, vp, ctypes.c_double,
                                     ctypes.c_int, ctypes.POINTER(SolveInfo)]),
    "lsmf_problem_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(vp)]),
    "lsmf_prm_validate": (ctypes.c_int, [ctypes.c_char_p]),
    "lsmf_problem_destroy": (None, [vp]),
    "lsmf_problem_set_mu": (ctypes.c_int, [vp, dp]),
    "lsmf_problem_info": (ctypes.c_int, [vp, ip, ip, dp]),
    "lsmf_problem_run": (ctypes.c_int, [vp, ctypes.POINTER(NewtonInfo)]),
    "lsmf_problem_set_stream": (ctypes.c_int, [vp, vp]),
    "lsmf_problem_get_solution": (ctypes.c_int, [vp, dp]),
    "lsmf_residual": (ctypes.c_int, [vp, vp, ctypes.c_double, vp, dp]),
    "lsmf_adjoint_forward": (ctypes.c_int, [vp, dp, dp, ctypes.c_int, dp]),
    "lsmf_adjoint_backward": (ctypes.c_int, [vp, dp]),
    "lsmf_residual_norm_noalloc": (ctypes.c_int, [vp, vp, vp, vp]),
    "lsmf_mesh_create_part": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.c_int, ctypes.POINTER(vp)]),
    "lsmf_partition_layout": (ctypes.c_int, [ctypes.POINTER(MeshDesc), ctypes.c_int, ctypes.c_int, ip, ip, vp, ip, vp,
                                             ip, vp]),
    "lsmf_dist_create_group": (ctypes.c_int, [ctypes.c_int, vp, ctypes.POINTER(vp)]),
    "lsmf_dist_nccl_unique_id": (ctypes.c_int, [vp]),
    "lsmf_dist_create_nccl": (ctypes.c_int, [vp, vp, ctypes.POINTER(vp)]),
    "lsmf_dist_destroy": (None, [vp]),
    "lsmf_dist_vmult": (ctypes.c_int, [vp, vp, vp]),
    "lsmf_operator_get_option": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "lsmf_dist_set_exchange": (ctypes.c_int, [vp, ctypes.c_int]),
    "lsmf_dist_get_exchange": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int)]),
    "lsmf_dist_dot": (ctypes.c_int, [vp, vp, vp, dp]),
    "lsmf_dist_cg_solve": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_double, vp, vp, ctypes.c_double, ctypes.c_int,
                                          ctypes.POINTER(SolveInfo)]),
}


def _release(obj, destroy_name):
    """Destroy the handle of obj once.  The destroy function is taken from the
    library object the handle came from (obj._L), so this also works while
    the interpreter shuts down and module globals are already gone."""
    h = getattr(obj, "h", None)
    L = getattr(obj, "_L", None)
    if h and L is not None:
        obj.h = None
        getattr(L, destroy_name)(h)


def lib():
    """Load liblsmf.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LsmfError(-1, "liblsmf.so not built: run large-strain-matrix-free_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is not None:
                f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise LsmfError(status, "%s: %s" % (lib().lsmf_status_string(status).decode(),
                                            lib().lsmf_last_error().decode()))


def _dptr(t):
    import torch
    if not isinstance(t, torch.Tensor) or not t.is_cuda or not t.is_contiguous():
        raise LsmfError(1, "device buffers must be contiguous torch CUDA tensors")
    return ctypes.c_void_p(t.data_ptr())


def _mesh_desc(geometry="box", coarse=(1, 1, 1), n_refinements=0, lo=(0, 0, 0), hi=(1, 1, 1), scale=1.0, degree=2,
               n_q_points_1d=None, coarse_active=None):
    """lsmf_mesh_desc and the mask array it points to (kept alive by the caller)."""
    d = MeshDesc()
    d.geometry = GEOM[geometry] if isinstance(geometry, str) else int(geometry)
    for k in range(3):
        d.coarse[k], d.lo[k], d.hi[k] = coarse[k], lo[k], hi[k]
    d.n_refinements, d.scale, d.degree = n_refinements, scale, degree
    d.n_q_points_1d = degree + 1 if n_q_points_1d is None else n_q_points_1d
    mask = None
    if coarse_active is not None:
        mask = np.ascontiguousarray(coarse_active, dtype=np.uint8)
        d.coarse_active = mask.ctypes.data
    return d, mask


def partition_layout(n_parts, part, **mesh_kw):
    """Host-only layout of z-slab part `part` of `n_parts` (no GPU needed):
    whole-mesh node number of each local node, the local nodes shared with
    part - 1 (owned here) and with part + 1 (ghosts here)."""
    d, mask = _mesh_desc(**mesh_kw)
    nn, ng, nlo, nup = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    check(lib().lsmf_partition_layout(ctypes.byref(d), n_parts, part, ctypes.byref(nn), ctypes.byref(ng), None,
                                      ctypes.byref(nlo), None, ctypes.byref(nup), None))
    gn = np.zeros(nn.value, dtype=np.int32)
    lo_ = np.zeros(max(1, nlo.value), dtype=np.int32)
    up_ = np.zeros(max(1, nup.value), dtype=np.int32)
    check(lib().lsmf_partition_layout(ctypes.byref(d), n_parts, part, ctypes.byref(nn), ctypes.byref(ng),
                                      gn.ctypes.data, ctypes.byref(nlo), lo_.ctypes.data, ctypes.byref(nup),
                                      up_.ctypes.data))
    del mask
    return {"n_nodes": nn.value, "n_global_nodes": ng.value, "global_node": gn,
            "lower_shared": lo_[:nlo.value].copy(), "upper_shared": up_[:nup.value].copy()}


class Mesh:
    """Structured hex mesh hierarchy (levels 0..n_refinements); with
    n_parts > 1 the z-slab part `part` of that partition."""

    def __init__(self, geometry="box", coarse=(1, 1, 1), n_refinements=0, lo=(0, 0, 0), hi=(1, 1, 1),
                 scale=1.0, degree=2, n_q_points_1d=None, coarse_active=None, n_parts=1, part=0):
        d, self._mask = _mesh_desc(geometry, coarse, n_refinements, lo, hi, scale, degree, n_q_points_1d,
                                   coarse_active)
        h = vp()
        if n_parts > 1:
            check(lib().lsmf_mesh_create_part(ctypes.byref(d), n_parts, part, ctypes.byref(h)))
        else:
            check(lib().lsmf_mesh_create(ctypes.byref(d), ctypes.byref(h)))
        self._L = lib()
        self.h = h
        self.degree = degree
        self.n_levels = lib().lsmf_mesh_n_levels(h)

    def __del__(self, _release=_release):  # bound now: module globals are gone at exit
        _release(self, "lsmf_mesh_destroy")

    def info(self, level=-1):
        nc, nn, nd = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(lib().lsmf_mesh_info(self.h, level, ctypes.byref(nc), ctypes.byref(nn), ctypes.byref(nd)))
        return nc.value, nn.value, nd.value

    def arrays(self, level=-1):
        nc, nn, _ = self.info(level)
        X = np.zeros((nn, 3))
        cn = np.zeros((nc, (self.degree + 1) ** 3), dtype=np.int32)
        ijk = np.zeros((nc, 3), dtype=np.int32)
        check(lib().lsmf_mesh_arrays(self.h, level, X.ctypes.data, cn.ctypes.data, ijk.ctypes.data))
        return X, cn, ijk

    def set_dirichlet(self, specs):
        """specs: [(boundary_id, component_bits), ...]"""
        ids = np.array([s[0] for s in specs] or [0], dtype=np.int32)
        masks = np.array([s[1] for s in specs] or [0], dtype=np.int32)
        check(lib().lsmf_mesh_set_dirichlet(self.h, len(specs), ids.ctypes.data_as(ip), masks.ctypes.data_as(ip)))

    def constraint_mask(self, level=-1):
        _, _, nd = self.info(level)
        m = np.zeros(nd, dtype=np.uint8)
        check(lib().lsmf_mesh_constraint_mask(self.h, level, m.ctypes.data))
        return m


class NeoHookOperator:
    """initialize(): choose caching (scalar / tensor2 / tensor4) and precision."""

    def __init__(self, mesh, caching="tensor4", formulation=1, precision="fp64", level=-1):
        self.mesh = mesh
        self.fp32 = precision in ("fp32", "float", 1)
        h = vp()
        cach = CACHING[caching] if isinstance(caching, str) else int(caching)
        check(lib().lsmf_operator_create(mesh.h, level, cach, formulation, 1 if self.fp32 else 0, ctypes.byref(h)))
        self._L = lib()
        self.h = h
        self.level = level
        self._u = None

    def clear(self, _release=_release):  # bound now: module globals are gone at exit
        _release(self, "lsmf_operator_destroy")

    __del__ = clear

    @property
    def dtype(self):
        import torch
        return torch.float32 if self.fp32 else torch.float64

    def m(self):
        return lib().lsmf_operator_m(self.h)

    def n(self):
        return lib().lsmf_operator_n(self.h)

    def set_material(self, mu_per_cell, nu):
        nc, _, _ = self.mesh.info(self.level)
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_per_cell, dtype=np.float64), (nc,)))
        check(lib().lsmf_operator_set_material(self.h, mu.ctypes.data_as(dp), nu))

    def cache(self, u):
        """u: device tensor of the operator's precision (borrowed)."""
        self._u = u
        check(lib().lsmf_operator_cache(self.h, _dptr(u)))

    def vmult(self, dst, src, mask=MASK_DEFAULT):
        check(lib().lsmf_operator_vmult(self.h, _dptr(dst), _dptr(src), mask))

    def vmult_add(self, dst, src):
        check(lib().lsmf_operator_vmult_add(self.h, _dptr(dst), _dptr(src)))

    Tvmult = vmult
    Tvmult_add = vmult_add

    def compute_diagonal(self):
        check(lib().lsmf_operator_compute_diagonal(self.h))

    def _diag_tensors(self):
        d, inv = vp(), vp()
        check(lib().lsmf_operator_get_diagonal(self.h, ctypes.byref(d), ctypes.byref(inv)))
        n = self.m()
        return [device_view(p.value, n, self.fp32).clone() for p in (d, inv)]

    def get_matrix_diagonal_inverse(self):
        return self._diag_tensors()[1]

    def get_matrix_diagonal(self):
        return self._diag_tensors()[0]

    def el(self, row, col):
        v = ctypes.c_double()
        check(lib().lsmf_operator_el(self.h, int(row), int(col), ctypes.byref(v)))
        return v.value

    def precondition_Jacobi(self, dst, src, omega):
        check(lib().lsmf_operator_precondition_jacobi(self.h, _dptr(dst), _dptr(src), omega))

    def set_pipeline(self, stages):
        """Ring depth (0..3) of the bulk-copy record pipeline in vmult; 0 =
        plain loads, -1 = the measured default (one stage for the large-record
        variants of degree 1 or 2 while a record fits in 24 KB, else plain
        loads).  True/False
        select 2/0."""
        if stages is True:
            stages = 2
        check(lib().lsmf_operator_set_option(self.h, 1, int(stages)))

    def set_basic_kernel(self, enable):
        """Use the basic vmult kernel (shared-memory sweeps, plain loads)."""
        check(lib().lsmf_operator_set_option(self.h, 2, int(bool(enable))))

    def set_max_warps(self, w):
        check(lib().lsmf_operator_set_option(self.h, 3, int(w)))

    def set_wait_tries(self, tries):
        """Bound of the pipelined kernel's wait for a cell record (-1 =
        default; 0 makes every wait run out at once, for tests)."""
        check(lib().lsmf_operator_set_option(self.h, 4, int(tries)))

    def set_scatter(self, mode):
        """'atomic' (default), 'colour8' (8 colour launches, plain adds:
        bit-reproducible) or 'nodesum' (one cell loop into a per-cell buffer,
        then per-node sums in cell order: bit-reproducible)."""
        check(lib().lsmf_operator_set_option(self.h, 5, SCATTER[mode] if isinstance(mode, str) else int(mode)))

    def set_record_prefetch(self, mode):
        """L1 prefetch of the cell record with plain loads: 0 none, 1 this
        cell's, 2 the next cell's, -1 the measured default."""
        check(lib().lsmf_operator_set_option(self.h, 6, int(mode)))

    def set_cell_pairs(self, mode):
        """FP32 operators: 1 = two cells per warp in packed f32x2 arithmetic,
        0 = one cell per warp, -1 = the measured default (pairs for Q1
        tensor2 / scalar, Q2 tensor2 / scalar / scalar_referential, Q4
        scalar_referential; formulation 1)."""
        check(lib().lsmf_operator_set_option(self.h, 7, int(mode)))

    def set_chunks(self, k):
        """Atomic-scatter vmult cell loop in k (2..8) concurrent cell chunks,
        each zeroing its own range of dst first; 1 = one launch, -1 = the
        measured default."""
        check(lib().lsmf_operator_set_option(self.h, 8, int(k)))

    def get_option(self, option):
        """lsmf_operator_get_option: the option as set; for 8 (chunks) the
        chunk count the next vmult cell loop runs in."""
        v = ctypes.c_int()
        check(lib().lsmf_operator_get_option(self.h, int(option), ctypes.byref(v)))
        return v.value

    def sync(self):
        """Wait for the operator's stream; raises LsmfError (status 8) if a
        bounded device wait ran out since the last call."""
        check(lib().lsmf_operator_sync(self.h))

    def set_stream(self, stream):
        """Order every call on a CUDA stream (torch.cuda.Stream or raw handle)."""
        h = getattr(stream, "cuda_stream", stream)
        check(lib().lsmf_operator_set_stream(self.h, vp(h)))

    def residual_norm_noalloc(self, x, b, out):
        """out[0] = ||b - A x|| without any device allocation (FP64 operators
        up to 2,097,152 dofs; the scratch is a static device array)."""
        check(lib().lsmf_residual_norm_noalloc(self.h, _dptr(x), _dptr(b), _dptr(out)))

    def memory_consumption(self):
        return lib().lsmf_operator_memory_consumption(self.h)

    def table(self, which):
        cnt = ctypes.c_size_t()
        check(lib().lsmf_operator_get_table(self.h, which, None, ctypes.byref(cnt)))
        out = np.zeros(cnt.value)
        check(lib().lsmf_operator_get_table(self.h, which, out.ctypes.data_as(dp), ctypes.byref(cnt)))
        return out


class GMG:
    """Geometric multigrid V-cycle (PreconditionMG of mf_elasticity.h:2079-2238):
    level operators of the given caching / precision, Chebyshev smoothing,
    Chebyshev coarse solver, matrix-free transfer."""

    def __init__(self, mesh, caching="tensor4", formulation=1, precision="fp32", degree=5, smoothing_range=20.0,
                 eig_cg_iterations=30, coarse_chebyshev=True, coarse_accurate_eig=True):
        d = GmgDesc()
        d.caching = CACHING[caching] if isinstance(caching, str) else int(caching)
        d.formulation = formulation
        d.precision = 1 if precision in ("fp32", "float", 1) else 0
        d.smoother_degree, d.smoothing_range, d.eig_cg_iterations = degree, smoothing_range, eig_cg_iterations
        d.coarse_chebyshev, d.coarse_accurate_eig = int(coarse_chebyshev), int(coarse_accurate_eig)
        h = vp()
        check(lib().lsmf_gmg_create(mesh.h, ctypes.byref(d), ctypes.byref(h)))
        self._L = lib()
        self.h, self.mesh = h, mesh

    def __del__(self, _release=_release):  # bound now: module globals are gone at exit
        _release(self, "lsmf_gmg_destroy")

    def set_material(self, mu_fine, nu):
        nc, _, _ = self.mesh.info(-1)
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_fine, dtype=np.float64), (nc,)))
        check(lib().lsmf_gmg_set_material(self.h, mu.ctypes.data_as(dp), nu))

    def setup(self, u_fine):
        self._u = u_fine
        check(lib().lsmf_gmg_setup(self.h, _dptr(u_fine)))

    def vmult(self, dst, src):
        check(lib().lsmf_gmg_vmult(self.h, _dptr(dst), _dptr(src)))

    def set_graph(self, enable):
        """Replay the V-cycle as one CUDA graph (default) or launch kernel by kernel."""
        check(lib().lsmf_gmg_set_option(self.h, 1, int(bool(enable))))

    def set_scatter(self, mode):
        """'atomic' (default) or 'colour8' for every level cell loop and transfer."""
        check(lib().lsmf_gmg_set_option(self.h, 2, SCATTER[mode] if isinstance(mode, str) else int(mode)))


    def level_option(self, level, option, value):
        """lsmf_operator_set_option on the operator of a level (effective
        from the next set-up)."""
        h = vp()
        check(lib().lsmf_gmg_level_operator(self.h, level, ctypes.byref(h)))
        check(lib().lsmf_operator_set_option(h, option, value))

    def level_info(self, level):
        out = np.zeros(6)
        check(lib().lsmf_gmg_level_info(self.h, level, out.ctypes.data_as(dp)))
        return out


def cg_solve(op, x, b, tol, max_it, precond="gmg", gmg=None, omega=1.0):
    """SolverCG: solve op x = b to ||b - op x|| <= tol (x holds the initial guess)."""
    info = SolveInfo()
    pc = {"none": 0, "jacobi": 1, "gmg": 2}[precond]
    st = lib().lsmf_cg_solve(op.h, pc, omega, gmg.h if gmg is not None else None, _dptr(x), _dptr(b), tol, max_it,
                             ctypes.byref(info))
    if st not in (0, 5):
        check(st)
    return {"iterations": info.iterations, "residual": info.residual, "converged": bool(info.converged),
            "status": st}


def _ptr_array(tensors):
    arr = (ctypes.c_void_p * len(tensors))(*[_dptr(t).value for t in tensors])
    return arr


class Dist:
    """The distributed operator over z-slab parts (update_ghost_values, cell
    loop, compress(add) around every vmult; all-reduced CG scalars).  Build
    it with group(ops) (all parts in this process) or nccl(op, id) (one part
    per process).  Vectors are lists of the local vectors of the parts this
    object holds (one tensor for nccl)."""

    def __init__(self, h, n_local):
        self._L = lib()
        self.h, self.n_local = h, n_local

    @classmethod
    def group(cls, ops):
        h = vp()
        arr = (ctypes.c_void_p * len(ops))(*[o.h.value for o in ops])
        check(lib().lsmf_dist_create_group(len(ops), arr, ctypes.byref(h)))
        obj = cls(h, len(ops))
        obj._ops = list(ops)
        return obj

    @staticmethod
    def nccl_unique_id():
        buf = (ctypes.c_ubyte * 128)()
        check(lib().lsmf_dist_nccl_unique_id(buf))
        return bytes(buf)

    @classmethod
    def nccl(cls, op, uid):
        h = vp()
        buf = (ctypes.c_ubyte * 128).from_buffer_copy(uid)
        check(lib().lsmf_dist_create_nccl(op.h, buf, ctypes.byref(h)))
        obj = cls(h, 1)
        obj._ops = [op]
        return obj

    def __del__(self, _release=_release):  # bound now: module globals are gone at exit
        _release(self, "lsmf_dist_destroy")

    EXCHANGE = {"packed": 0, "fused": 1}

    def set_exchange(self, mode):
        """"packed" (update_ghost_values / compress(add) through buffers) or
        "fused" (group objects: the cell loops read and add to the
        neighbours' vectors directly)."""
        check(lib().lsmf_dist_set_exchange(self.h, self.EXCHANGE[mode] if isinstance(mode, str) else int(mode)))

    def exchange(self):
        m = ctypes.c_int()
        check(lib().lsmf_dist_get_exchange(self.h, ctypes.byref(m)))
        return {v: k for k, v in self.EXCHANGE.items()}[m.value]

    def vmult(self, dsts, srcs):
        check(lib().lsmf_dist_vmult(self.h, _ptr_array(dsts), _ptr_array(srcs)))

    def dot(self, a, b):
        out = ctypes.c_double()
        check(lib().lsmf_dist_dot(self.h, _ptr_array(a), _ptr_array(b), ctypes.byref(out)))
        return out.value

    def cg_solve(self, xs, bs, tol, max_it, precond="jacobi", omega=1.0):
        info = SolveInfo()
        st = lib().lsmf_dist_cg_solve(self.h, {"none": 0, "jacobi": 1}[precond], omega, _ptr_array(xs),
                                      _ptr_array(bs), tol, max_it, ctypes.byref(info))
        if st not in (0, 5):
            check(st)
        return {"iterations": info.iterations, "residual": info.residual, "converged": bool(info.converged),
                "status": st}


def prm_validate(prm_text):
    """Parse and check a .prm text on the host; returns (status, message)."""
    st = lib().lsmf_prm_validate(prm_text.encode())
    return st, (lib().lsmf_last_error().decode() if st else "")


class Problem:
    """A reference-format .prm problem (Solid of mf_elasticity.h): mesh,
    boundary conditions, loads, FP64 fine operator, optional GMG, and the
    device load-stepping Newton driver."""

    def __init__(self, prm_text):
        h = vp()
        check(lib().lsmf_problem_create(prm_text.encode(), ctypes.byref(h)))
        self._L = lib()
        self.h = h
        nc, nd, vol = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        check(lib().lsmf_problem_info(h, ctypes.byref(nc), ctypes.byref(nd), ctypes.byref(vol)))
        self.n_cells, self.n_dofs, self.volume = nc.value, nd.value, vol.value

    def __del__(self, _release=_release):  # bound now: module globals are gone at exit
        _release(self, "lsmf_problem_destroy")

    def set_mu(self, mu_per_cell):
        mu = np.ascontiguousarray(np.broadcast_to(np.asarray(mu_per_cell, dtype=np.float64), (self.n_cells,)))
        check(lib().lsmf_problem_set_mu(self.h, mu.ctypes.data_as(dp)))

    def set_stream(self, stream):
        check(lib().lsmf_problem_set_stream(self.h, vp(getattr(stream, "cuda_stream", stream))))

    def run(self, raise_on_error=True):
        info = NewtonInfo()
        st = lib().lsmf_problem_run(self.h, ctypes.byref(info))
        if raise_on_error:
            check(st)
        steps = [{"newton_iterations": info.newton_iterations[i], "cg_iterations": info.cg_iterations[i],
                  "point_u": [info.point_u[i][c] for c in range(3)]} for i in range(info.n_steps)]
        return {"status": st, "steps": steps, "time_residual": info.time_residual,
                "time_setup": info.time_setup, "time_solve": info.time_solve}

    def residual(self, u, t, R):
        """assemble_system's right-hand side R = f_ext(t) - f_int(u), Dirichlet
        entries zeroed, into the device vector R; returns ||R||."""
        nrm = ctypes.c_double()
        check(lib().lsmf_residual(self.h, _dptr(u), float(t), _dptr(R), ctypes.byref(nrm)))
        return nrm.value

    def solution(self):
        u = np.zeros(self.n_dofs)
        check(lib().lsmf_problem_get_solution(self.h, u.ctypes.data_as(dp)))
        return u

    def adjoint_forward(self, log_mu, u_target, obj_id):
        lm = np.ascontiguousarray(log_mu, dtype=np.float64)
        ut = np.ascontiguousarray(u_target, dtype=np.float64)
        J = ctypes.c_double()
        check(lib().lsmf_adjoint_forward(self.h, lm.ctypes.data_as(dp), ut.ctypes.data_as(dp), obj_id,
                                         ctypes.byref(J)))
        return J.value

    def adjoint_backward(self):
        g = np.zeros(self.n_cells)
        check(lib().lsmf_adjoint_backward(self.h, g.ctypes.data_as(dp)))
        return g


class _DevArray:
    """__cuda_array_interface__ view of a device buffer owned by liblsmf."""

    def __init__(self, ptr, n, fp32):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4" if fp32 else "<f8",
                                         "data": (ptr, False), "version": 3, "strides": None}


def device_view(ptr, n, fp32=False):
    import torch
    return torch.as_tensor(_DevArray(ptr, n, fp32), device="cuda")
