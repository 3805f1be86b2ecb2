"""C ABI checks that need no GPU: liblsmf.so loads, exports every function
declared in include/lsmf.h, and rejects bad .prm input on the host."""
import ctypes
import os
import re

import pytest

import lsmf
from prm_util import prm_text

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "lsmf.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lsmf_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(lsmf.LIB_PATH)
    names = _declared()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert not [n for n in names if n not in lsmf.SIGNATURES]


def test_status_strings():
    assert lsmf.lib().lsmf_status_string(0) == b"ok"
    assert b"det_F" in lsmf.lib().lsmf_status_string(3)
    assert lsmf.lib().lsmf_version().startswith(b"lsmf")


BASE = {"Polynomial degree": 2, "Quadrature order": 3, "Dimension": 3, "Elements per edge": 4,
        "Grid scale": "1e-3", "Solver type": "MF_CG", "Preconditioner type": "gmg", "MF caching": "tensor4",
        "Formulation": 1, "Dirichlet IDs and expressions": "1:0,0,0",
        "Dirichlet IDs and component mask": "1:true,true,true",
        "Neumann IDs and expressions": "11:0,t/(16.0e-6),0", "Output points": "48.0e-3, 60.0e-3, 0.5e-3"}


def test_prm_valid():
    st, msg = lsmf.prm_validate(prm_text(BASE))
    assert st == 0, msg


@pytest.mark.parametrize("precond", ["gmg", "gmg-gc", "jacobi", "none"])
def test_prm_every_preconditioner(precond):
    st, msg = lsmf.prm_validate(prm_text(dict(BASE, **{"Preconditioner type": precond})))
    assert st == 0, msg


@pytest.mark.parametrize("caching", ["scalar", "tensor2", "tensor4", "scalar_referential", "tensor4_ns"])
def test_prm_every_caching(caching):
    st, msg = lsmf.prm_validate(prm_text(dict(BASE, **{"MF caching": caching})))
    assert st == 0, msg


@pytest.mark.parametrize("scatter", ["atomic", "colour8", "nodesum"])
def test_prm_every_scatter(scatter):
    st, msg = lsmf.prm_validate(prm_text(dict(BASE, **{"MF scatter": scatter})))
    assert st == 0, msg


@pytest.mark.parametrize("change,status", [
    ({"Solver type": "CG"}, 10),                      # matrix-based path is not part of this library
    ({"Preconditioner type": "amg"}, 10),
    ({"MF caching": "tensor4_ns", "Formulation": 0}, 10),   # referential variants are formulation 1
    ({"MF caching": "magic"}, 2),                     # Unknown caching (mf_nh_operator.h:441)
    ({"Formulation": 0}, 10),                         # formulation 0 needs scalar caching
    ({"Dimension": 2}, 10),
    ({"Quadrature order": 4}, 10),
    ({"Neumann IDs and expressions": "11:0,t/(16.0e-6"}, 9),   # bad expression
    ({"Neumann IDs and expressions": "11:0,q*2,0"}, 9),        # unknown variable
    ({"Dirichlet IDs and component mask": "2:true,true,true"}, 9),  # no mask for id 1
    ({"Preconditioner relaxation": "abc"}, 9),
    ({"Shear modulus": "-1"}, 9),
    ({"MF scatter": "sometimes"}, 9),
])
def test_prm_rejected(change, status):
    v = dict(BASE)
    v.update(change)
    st, msg = lsmf.prm_validate(prm_text(v))
    assert st == status, (st, msg)
    assert msg


def test_prm_undeclared_entry():
    st, msg = lsmf.prm_validate(prm_text(BASE) + "subsection Geometry\n  set Colour = blue\nend\n")
    assert st == 9 and "undeclared entry" in msg


def test_prm_structure_errors():
    assert lsmf.prm_validate("subsection Geometry\n set Dimension = 3\n")[0] == 9   # missing end
    assert lsmf.prm_validate("end\n")[0] == 9
    assert lsmf.prm_validate("garbage line\n")[0] == 9
