"""Builds reference-format .prm texts (deal.II ParameterHandler syntax) for
the tests from flat {key: value} dictionaries."""

SECTIONS = {
    "Finite element system": ["Polynomial degree", "Quadrature order"],
    "Geometry": ["Elements per edge", "Global refinement", "Grid scale", "Extrusion height", "Extrusion slices",
                 "Dimension", "Type", "Box cells", "Box lower corner", "Box upper corner", "Cook thickness",
                 "Void spheres"],
    "Material properties": ["Poisson's ratio", "Shear modulus", "Formulation"],
    "Linear solver": ["Solver type", "Residual", "Max iteration multiplier", "Preconditioner type",
                      "Preconditioner relaxation", "Preconditioner AMG aggregation threshold",
                      "Condition number CG iterations", "MF caching", "MF Chebyshev number CG iterations",
                      "MF Chebyshev coarse", "MF Chebyshev coarse accurate eigenvalues", "MF level precision",
                      "MF Chebyshev degree", "MF Chebyshev smoothing range", "MF scatter"],
    "Nonlinear solver": ["Max iterations Newton-Raphson", "Tolerance force", "Absolute tolerance force",
                         "Tolerance displacement", "Absolute tolerance displacement"],
    "Time": ["End time", "Time step size"],
    "Misc": ["Output folder", "Output solution", "Always assemble tangent", "Output absolute norms",
             "Output points"],
    "Boundary conditions": ["Dirichlet IDs and expressions", "Dirichlet IDs and component mask",
                            "Neumann IDs and expressions"],
}


def prm_text(values):
    out = []
    used = set()
    for sec, keys in SECTIONS.items():
        lines = ["  set %s = %s" % (k, values[k]) for k in keys if k in values]
        used.update(k for k in keys if k in values)
        if lines:
            out.append("subsection %s" % sec)
            out.extend(lines)
            out.append("end")
    unknown = set(values) - used
    if unknown:
        raise KeyError("no subsection for %s" % sorted(unknown))
    return "\n".join(out) + "\n"
