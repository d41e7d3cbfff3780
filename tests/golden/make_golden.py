"""Extract the reference test suite's hard-coded golden vectors into JSON.

Reads FastMultipole.jl's own test files *as text* (the Julia package cannot be
executed here) and writes ``reference_vectors.json`` next to this script.  The
fixture holds, per case, the coefficient vectors in the reference's
"full" ordering (n = 0..p, m = -n..n) as [re, im] pairs, plus the scalar
parameters of the case as they appear in the test file.

Usage:  python tests/golden/make_golden.py path/to/FastMultipole.jl
(the path of a FastMultipole.jl checkout is required).
"""
import json
import os
import re
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_golden.py path/to/FastMultipole.jl")
REF = sys.argv[1]
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")

NUM = r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eE][-+]?\d+)?"
CPLX = re.compile(rf"({NUM})\s*([-+])\s*({NUM})im")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def testset(text, title):
    """Text of one @testset block (up to the next @testset)."""
    i = text.index(f'@testset "{title}"')
    j = text.find("@testset", i + 10)
    return text[i: j if j >= 0 else len(text)]


def cvec(block, name):
    m = re.search(rf"^{name} = (-?)ComplexF64\[(.*)\]\s*$", block, re.M)
    if not m:
        raise KeyError(name)
    sign = -1.0 if m.group(1) == "-" else 1.0
    out = []
    for item in m.group(2).split(","):
        c = CPLX.search(item)
        re_, s, im_ = float(c.group(1)), c.group(2), float(c.group(3))
        out.append([sign * re_, sign * (im_ if s == "+" else -im_)])
    return out


def scalar(block, name):
    m = re.search(rf"^\s*{name} = ({NUM})\s*$", block, re.M)
    return float(m.group(1))


def svec(block, name):
    m = re.search(rf"^\s*{name} = SVector{{3}}\(\[?({NUM}),\s*({NUM}),\s*({NUM})\]?\)", block, re.M)
    return [float(m.group(k)) for k in (1, 2, 3)]


def julia_matrix(block, name):
    """Parse `name = [a b c\n d e f ...]` (real parts only; the matrices are real)."""
    m = re.search(rf"^{name} = \[(.*?)\]", block, re.M | re.S)
    rows = [r for r in re.split(r"[;\n]", m.group(1)) if r.strip()]
    mat = []
    for r in rows:
        vals = re.findall(rf"({NUM})(?:[-+]{NUM}im)?", r.replace("+0.0im", "").replace("-0.0im", ""))
        mat.append([float(v) for v in vals])
    return mat


def main():
    cases = {}

    t = read("test/translate_multipole_to_local_test.jl")
    b = testset(t, "multipole-to-local z translation")
    cases["m2l_z"] = dict(p=10, r=scalar(b, "r"), src=cvec(b, "original_weights_test"),
                          expected=cvec(b, "translated_weights_test"), atol=1e-12,
                          cite="test/translate_multipole_to_local_test.jl:1-40")
    b = testset(t, "multipole-to-local: point-and-shoot")
    cases["m2l_point_and_shoot"] = dict(
        p=10, src=cvec(b, "multipole_expansion_test"), expected=cvec(b, "local_expansion_test"),
        source_center=[0.2, 0.4, -0.15999999999999998], target_center=[2.5, -4.3999999999999995, 0.8],
        atol=1e-12, cite="test/translate_multipole_to_local_test.jl:42-102")

    t = read("test/translate_multipole_test.jl")
    b = testset(t, "multipole-to-multipole z translation")
    lit = re.search(r"vec\(tmp\) \.= vec\(\[(.*?)\]\)", b, re.S).group(1)
    slices = [s.strip() for s in lit.split(";;;")]
    src = []
    for s in slices:  # slice k = [re_phi re_chi; im_phi im_chi]
        (a, bb), (c, d) = [[float(v) for v in row.split()] for row in s.split(";")]
        src.append([a, c])
    cases["m2m_z"] = dict(p=10, r=scalar(b, "r"), src_compressed=src,
                          expected=cvec(b, "translated_weights_test"), atol=1e-12,
                          cite="test/translate_multipole_test.jl:1-34")
    b = testset(t, "multipole-to-multipole: point-and-shoot")
    cases["m2m_point_and_shoot"] = dict(
        p=7, x=[0.1, 0.2, -0.3], offset=[-0.2, 0.07, -0.1], mass=0.7, shift=[0.1, 0.2, 0.14],
        expected=cvec(b, "translated_weights_test"), atol=1e-12,
        cite="test/translate_multipole_test.jl:36-88")

    t = read("test/translate_local_test.jl")
    b = testset(t, "local-to-local z translation")
    cases["l2l_z"] = dict(p=10, r=scalar(b, "r"), src=cvec(b, "original_weights_test"),
                          expected=cvec(b, "translated_weights_test"), atol=1e-12,
                          cite="test/translate_local_test.jl:1-40")
    b = testset(t, "local-to-local: point-and-shoot")
    cases["l2l_point_and_shoot"] = dict(
        p=10, src=cvec(b, "source_weights_test"), expected=cvec(b, "translated_weights_test"),
        source_center=[2.5, -4.3999999999999995, 0.8], target_center=[2.4, -4.199999999999999, 0.5],
        atol=1e-12, cite="test/translate_local_test.jl:42-102")

    t = read("test/evaluate_expansions_test.jl")
    b = testset(t, "evaluate local expansion")
    cases["l2p_point_mass"] = dict(
        p=10, local=cvec(b, "local_weights_test"), x_target=[2.3, -4.1, 0.4],
        center=[2.4, -4.199999999999999, 0.5], source=[0.1 - 0.2, 0.2 + 0.07, -0.3 - 0.1], mass=0.7,
        atol_phi=1e-12, atol_grad=1e-11, atol_hess=1e-9, cite="test/evaluate_expansions_test.jl:1-55")

    t = read("test/lamb_helmholtz_test.jl")
    b = testset(t, "Lamb-Helmholtz transform: multipole")
    cases["lh_multipole"] = dict(p=10, r=scalar(b, "r"), phi=cvec(b, "weights_1"), chi=cvec(b, "weights_2"),
                                 expected_phi=cvec(b, "new_weights_1"), expected_chi=cvec(b, "new_weights_2"),
                                 atol=1e-12, cite="test/lamb_helmholtz_test.jl:1-43")
    b = testset(t, "Lamb-Helmholtz transform: local")
    cases["lh_local"] = dict(p=10, r=scalar(b, "r"), phi=cvec(b, "weights_1"), chi=cvec(b, "weights_2"),
                             expected_phi=cvec(b, "new_weights_1"), expected_chi=cvec(b, "new_weights_2"),
                             atol=1e-12, cite="test/lamb_helmholtz_test.jl:45-85")
    b = testset(t, "Lamb-Helmholtz transform: multipole-to-multipole")
    cases["lh_m2m"] = dict(p=10, phi=cvec(b, "weights_1"), chi=cvec(b, "weights_2"),
                           expected_phi=cvec(b, "translated_weights_1"), expected_chi=cvec(b, "translated_weights_2"),
                           source_center=[0.01, 0.02, -0.03], target_center=[0.04, 0.04, -0.019999999999999997],
                           n_check=10, atol=1e-12, cite="test/lamb_helmholtz_test.jl:87-152")
    b = testset(t, "Lamb-Helmholtz transform: multipole-to-local")
    cases["lh_m2l"] = dict(p=10, phi=cvec(b, "weights_1"), chi=cvec(b, "weights_2"),
                           expected_phi=cvec(b, "translated_weights_1"), expected_chi=cvec(b, "translated_weights_2"),
                           source_center=[0.04, 0.04, -0.019999999999999997], target_center=[0.96, 0.03, -0.02],
                           n_check=7, atol=1e-12, rtol=1e-12, cite="test/lamb_helmholtz_test.jl:154-213")
    b = testset(t, "Lamb-Helmholtz transform: local-to-local")
    cases["lh_l2l"] = dict(p=10, phi=cvec(b, "weights_1"), chi=cvec(b, "weights_2"),
                           expected_phi=cvec(b, "translated_weights_1"), expected_chi=cvec(b, "translated_weights_2"),
                           source_center=[0.96, 0.03, -0.02], target_center=[0.98, 0.01, 0.01],
                           n_check=7, atol=1e-11, rtol=1e-12, cite="test/lamb_helmholtz_test.jl:215-269")
    b = testset(t, "Lamb-Helmholtz: vorton")
    cases["lh_vorton"] = dict(p=10, phi=cvec(b, "multipole_weights_1"), chi=cvec(b, "multipole_weights_2"),
                              x_source=[0.0, 0.0, 0.0], x_target=[1.0, 0.0, 0.0], gamma=[0.0, 0.0, 1.0],
                              source_center=[0.01, 0.02, -0.03], target_center=[1.0 - 0.04, 0.03, -0.02],
                              atol_grad=1e-11, atol_hess=1e-9, cite="test/lamb_helmholtz_test.jl:271-339")

    t = read("test/rotate_test.jl")
    b = testset(t, "y axis rotations by π/2")
    cases["H_pi2"] = dict(p=4, beta="pi/2", mats=[julia_matrix(b, f"H{n}") for n in (1, 2, 3, 4)], atol=1e-6,
                          cite="test/rotate_test.jl:21-76")
    b = testset(t, "y axis rotation matrices")
    cases["T_3pi7"] = dict(p=5, beta="3pi/7", mats=[julia_matrix(b, f"T{n}") for n in (1, 2, 3, 4)], atol=1e-6,
                           cite="test/rotate_test.jl:80-120")

    with open(OUT, "w") as f:
        json.dump({"source": "FastMultipole.jl test suite (v1.0.0)", "cases": cases}, f, indent=1)
    print("wrote", OUT, "with", len(cases), "cases")


if __name__ == "__main__":
    main()
