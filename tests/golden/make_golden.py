"""Generate tests/golden/reference_vectors.json from the reference's own tests.

The reference (Rust) cannot be compiled here, so its known-answer data is read
*as text* from its test sources and quadrature tables and written to a small
JSON fixture that travels with the repository.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/higher_order_embedded_fem

Sources read (paths inside the reference project):
  fenris/tests/unit_tests/assembly.rs   csr_par_assemble_mock_pattern (552-621),
                                        apply_homogeneous_dirichlet_bc_csr_simple_example (318-345)
  fenris/tests/unit_tests/materials.rs  test_deformation_gradients_3d, contraction_test_vectors_3d,
                                        young_poisson_test_parameters (158-259)
  fenris/src/solid/materials.rs         SNH analytic-vs-numerical test matrix (955-989)
  fenris/tests/unit_tests/cg.rs         solve_arbitrary / solve_arbitrary_preconditioned
  simulation_toolbox/src/fem/newton_cg.rs  build_block_preconditioner (827-876)
  hamilton2/tests/unit_tests/newton.rs  newton_converges_in_single_iteration_for_linear_system
  fenris/src/quadrature.rs              tet_quadrature_strength_{1,2,3,5}, hex_quadrature_strength_5
"""
import json
import os
import re
import sys

FLOAT = r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"


def floats(s):
    return [float(x) for x in re.findall(FLOAT, s)]


def float_items(s):
    """The comma-separated items of a vec![...] body (brackets excluded),
    each a literal or a quotient of two literals (e.g. `(4.0 / 3.0)`)."""
    out = []
    for item in s.split(","):
        item = item.strip().strip("()").strip()
        if not item:
            continue
        if "/" in item:
            num, den = item.split("/")
            out.append(float(num) / float(den))
        else:
            out.append(float(item))
    return out


def ints(s):
    return [int(x) for x in re.findall(r"-?\d+", s)]


def body_of(text, signature):
    """Return the text of the brace-delimited item that starts at `signature`."""
    i = text.index(signature)
    j = text.index("{", i)
    depth = 0
    for k in range(j, len(text)):
        if text[k] == "{":
            depth += 1
        elif text[k] == "}":
            depth -= 1
            if depth == 0:
                return text[j : k + 1]
    raise ValueError(signature)


def bracket_groups(s, opener):
    """All groups `opener ... )` / `]` with balanced brackets."""
    out = []
    pos = 0
    close = {"(": ")", "[": "]"}
    while True:
        i = s.find(opener, pos)
        if i < 0:
            return out
        start = i + len(opener) - 1
        ch = s[start]
        depth = 0
        for k in range(start, len(s)):
            if s[k] == ch:
                depth += 1
            elif s[k] == close[ch]:
                depth -= 1
                if depth == 0:
                    out.append(s[start + 1 : k])
                    pos = k + 1
                    break


def strip_comments(s):
    return re.sub(r"//[^\n]*", "", s)


def mock_patterns(ref):
    text = open(os.path.join(ref, "fenris/tests/unit_tests/assembly.rs")).read()
    body = strip_comments(body_of(text, "fn csr_par_assemble_mock_pattern"))
    cases = []
    for blk in re.split(r"\n    \{", body)[1:]:
        sdim = int(re.search(r"solution_dim:\s*(\d+)", blk).group(1))
        nn = int(re.search(r"num_nodes:\s*(\d+)", blk).group(1))
        conn_src = bracket_groups(blk, "element_connectivities: vec![")[0]
        elems = [ints(g) for g in bracket_groups(conn_src, "vec![")]
        pat = bracket_groups(blk, "SparsityPattern::from_offsets_and_indices(")[0]
        m = re.match(r"\s*(\d+),\s*(\d+),\s*(.*)", pat, re.S)
        nrows, ncols, rest = int(m.group(1)), int(m.group(2)), m.group(3)
        if "vec![0; " in rest:
            k = int(re.search(r"vec!\[0;\s*(\d+)\]", rest).group(1))
            offsets = [0] * k
            indices = []
        else:
            groups = bracket_groups(rest, "vec![")
            offsets, indices = ints(groups[0]), ints(groups[1]) if len(groups) > 1 else []
        cases.append(dict(solution_dim=sdim, num_nodes=nn, elements=elems, nrows=nrows, ncols=ncols,
                          row_offsets=offsets, col_indices=indices))
    return cases


def dirichlet_example(ref):
    text = open(os.path.join(ref, "fenris/tests/unit_tests/assembly.rs")).read()
    body = strip_comments(body_of(text, "fn apply_homogeneous_dirichlet_bc_csr_simple_example"))
    rep = re.search(r"DMatrix::repeat\((\d+),\s*(\d+),\s*(" + FLOAT + r")\)", body)
    n = int(rep.group(1))
    fill = float(rep.group(3))
    nodes = ints(re.search(r"&mut matrix,\s*&\[([^\]]*)\]", body).group(1))
    dim = int(re.search(r"apply_homogeneous_dirichlet_bc_csr::<_,\s*U(\d)>", body).group(1))
    cs = bracket_groups(body, "DMatrix::from_column_slice(")[0]
    vals = floats(cs.split("&[", 1)[1])
    return dict(n=n, fill=fill, nodes=nodes, dim=dim, expected_column_major=vals)


def material_vectors(ref):
    text = open(os.path.join(ref, "fenris/tests/unit_tests/materials.rs")).read()
    fb = strip_comments(body_of(text, "fn test_deformation_gradients_3d"))
    Fs = []
    if "Matrix3::identity()" in fb:
        Fs.append([1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0])
    for g in bracket_groups(fb, "Matrix3::new("):
        Fs.append(floats(g))  # nalgebra Matrix3::new takes row-major arguments
    vb = strip_comments(body_of(text, "fn contraction_test_vectors_3d"))
    vecs = [floats(g) for g in bracket_groups(vb, "Vector3::new(")]
    yb = strip_comments(body_of(text, "fn young_poisson_test_parameters"))
    yp = [dict(young=float(y), poisson=float(p)) for y, p in
          re.findall(r"young:\s*(" + FLOAT + r"),\s*poisson:\s*(" + FLOAT + r")", yb)]
    return dict(deformation_gradients_row_major=Fs, vectors=vecs, young_poisson=yp)


def snh_analytic(ref):
    text = open(os.path.join(ref, "fenris/src/solid/materials.rs")).read()
    body = strip_comments(body_of(text, "fn stable_neo_hookean_analytic_decomposition_matches_numerical_3d"))
    young = float(re.search(r"young:\s*(" + FLOAT + r")f64", body).group(1))
    poisson = float(re.search(r"poisson:\s*(" + FLOAT + r")f64", body).group(1))
    F = floats(bracket_groups(body, "Matrix3::new(")[0])
    return dict(young=young, poisson=poisson, F_row_major=F)


def cg_cases(ref):
    text = strip_comments(open(os.path.join(ref, "fenris/tests/unit_tests/cg.rs")).read())
    b1 = body_of(text, "fn solve_arbitrary()")
    diag = float(re.search(r"if r == c \{\s*(" + FLOAT + r")\s*\} else \{\s*(" + FLOAT + r")", b1).group(1))
    off = float(re.search(r"if r == c \{\s*(" + FLOAT + r")\s*\} else \{\s*(" + FLOAT + r")", b1).group(2))
    x0 = floats(bracket_groups(b1, "from_row_slice(&[")[0])
    tol1 = float(re.search(r"RelativeResidualCriterion::new\((" + FLOAT + r")\)", b1).group(1))
    b2 = body_of(text, "fn solve_arbitrary_preconditioned")
    mats = bracket_groups(b2, "DMatrix::from_row_slice(3, 3, &[")
    A = floats(mats[0])
    P = floats(mats[1])
    cols = bracket_groups(b2, "DVector::from_column_slice(&[")
    x0b, guess = floats(cols[0]), floats(cols[1])
    iters = int(re.search(r"assert_eq!\(output\.num_iterations,\s*(\d+)\)", b2).group(1))
    tol2 = float(re.search(r"RelativeResidualCriterion::new\((" + FLOAT + r")\)", b2).group(1))
    return dict(arbitrary=dict(n=3, diag=diag, off=off, x0=x0, tol=tol1),
                preconditioned=dict(A_row_major=A, P_row_major=P, x0=x0b, guess=guess, iterations=iters, tol=tol2))


def block_precond(ref):
    text = strip_comments(open(os.path.join(ref, "simulation_toolbox/src/fem/newton_cg.rs")).read())
    body = body_of(text, "fn build_block_preconditioner()")
    m = floats(bracket_groups(body, "DMatrix::from_row_slice(")[0].split("&[", 1)[1])
    cols = bracket_groups(body, "DVector::from_column_slice(&[")
    return dict(matrix_row_major=m, x=floats(cols[0]), y_initial=floats(cols[1]))


def newton_linear(ref):
    text = strip_comments(open(os.path.join(ref, "hamilton2/tests/unit_tests/newton.rs")).read())
    a = floats(bracket_groups(text, "Matrix3::new(")[0])
    b = floats(bracket_groups(text, "Vector3::new(")[0])
    body = body_of(text, "fn newton_converges_in_single_iteration_for_linear_system")
    expected = floats(bracket_groups(body, "Vector3::new(")[0])
    return dict(A_row_major=a, b=b, expected=expected, iterations=1)


def quadrature(ref):
    text = open(os.path.join(ref, "fenris/src/quadrature.rs")).read()
    out = {}
    for name in ["tet_quadrature_strength_1", "tet_quadrature_strength_2", "tet_quadrature_strength_3",
                 "tet_quadrature_strength_5", "hex_quadrature_strength_5"]:
        body = strip_comments(body_of(text, "pub fn " + name))
        groups = {}
        for key in ["w", "x", "y", "z"]:
            m = re.search(r"let " + key + r"(?::\s*Vec<T>)?\s*=\s*vec!\[", body)
            start = m.end() - 1
            grp = bracket_groups(body[start - 4:], "vec![")[0]
            groups[key] = float_items(grp)
        out[name] = dict(weights=groups["w"], points=[list(p) for p in zip(groups["x"], groups["y"], groups["z"])])
    return out


def main():
    if len(sys.argv) > 1:
        ref = sys.argv[1]
    elif os.environ.get("HOEFEM_REFERENCE_DIR"):
        ref = os.environ["HOEFEM_REFERENCE_DIR"]
    else:
        sys.exit("usage: make_golden.py <reference checkout> (or set HOEFEM_REFERENCE_DIR)")
    data = dict(
        source="InteractiveComputerGraphics/higher_order_embedded_fem (test sources read as text)",
        mock_patterns=mock_patterns(ref),
        dirichlet_example=dirichlet_example(ref),
        materials=material_vectors(ref),
        snh_analytic=snh_analytic(ref),
        cg=cg_cases(ref),
        block_preconditioner=block_precond(ref),
        newton_linear=newton_linear(ref),
        quadrature=quadrature(ref),
    )
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")
    with open(out, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", out)


if __name__ == "__main__":
    main()
