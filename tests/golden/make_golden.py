"""Extract the reference's literal test vectors into tests/golden/reference_literals.json.

Run once in a container that has the reference tree (its path is the first
argument; there is no default). The GPU box never runs this: the JSON it
writes is committed and is what the tests read.

Sources (stwo_gpu_backend/src, NethermindEth/stwo-gpu):
  poly.rs:291-334   test_interpolate_2: 32 evaluation values (inputs only)
  poly.rs:399-614   test_interpolate_from_fib: domain literal, values, and the full
                    twiddle / itwiddle tree of root coset {8388608, 33554432, log 6}
  fri.rs:142-192    test_fold_line: the algebraic fold identity (parameters)
  fri.rs:313-940    test_fold_circle_into_line_fibonacci: dst/src columns, alpha,
                    domains and the same twiddle tree (inputs only)
  accumulation.rs:110-180  literal sums
Every Coset literal also pins one CirclePointIndex -> CirclePoint pair.
"""
import json
import os
import re
import sys

if len(sys.argv) < 2:
    sys.exit("usage: make_golden.py REFERENCE_TREE  (the NethermindEth/stwo-gpu checkout to read)")
REF = sys.argv[1]
SRC = os.path.join(REF, "stwo_gpu_backend", "src")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_literals.json")

NUM = r"(?:BaseField::from|M31::from|M31)\((\d+)\)"


def read(name):
    with open(os.path.join(SRC, name)) as f:
        return f.read()


def fn_body(text, fn_name):
    start = text.index("fn " + fn_name + "(")
    depth, i = 0, text.index("{", start)
    while True:
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start:i + 1]
        i += 1


def vec_after(text, marker):
    """Numbers inside the first `vec![ ... ]` that follows `marker`."""
    i = text.index(marker)
    j = text.index("vec![", i)
    k = text.index("]", j)
    return [int(x) for x in re.findall(NUM, text[j:k])]


def columns_after(text, marker):
    i = text.index(marker)
    j = text.index("columns: [", i)
    cols, pos = [], j
    for _ in range(4):
        a = text.index("vec![", pos)
        b = text.index("]", a)
        cols.append([int(x) for x in re.findall(NUM, text[a:b])])
        pos = b + 1
    return cols


def cosets(text):
    pat = re.compile(
        r"initial_index:\s*CirclePointIndex\((\d+)\),\s*initial:\s*CirclePoint\s*\{\s*x:\s*"
        + NUM + r",\s*y:\s*" + NUM + r",?\s*\},\s*step_size:\s*CirclePointIndex\((\d+)\),\s*step:\s*"
        r"CirclePoint\s*\{\s*x:\s*" + NUM + r",\s*y:\s*" + NUM + r",?\s*\},\s*log_size:\s*(\d+)",
        re.S)
    out = []
    for m in pat.finditer(text):
        ii, ix, iy, si, sx, sy, lg = (int(v) for v in m.groups())
        out.append({"initial_index": ii, "initial": [ix, iy], "step_size": si, "step": [sx, sy],
                    "log_size": lg})
    return out


def main():
    poly, fri, acc = read("poly.rs"), read("fri.rs"), read("accumulation.rs")
    g = {"source": "NethermindEth/stwo-gpu stwo_gpu_backend/src (test literals)"}

    body = fn_body(poly, "test_interpolate_2")
    g["interpolate_2_values"] = vec_after(body, "let cpu_values")

    body = fn_body(poly, "test_interpolate_from_fib")
    cs = cosets(body)
    g["interpolate_from_fib"] = {
        "domain_half_coset": cs[0],
        "values": vec_after(body, "BaseFieldVec::from_vec"),
        "root_coset": cs[1],
        "twiddles": vec_after(body, "let twiddles"),
        "itwiddles": vec_after(body, "let itwiddles"),
    }

    body = fn_body(fri, "test_fold_circle_into_line_fibonacci")
    cs = cosets(body)
    alpha = re.search(r"let alpha = QM31::from_m31\(\s*" + r",\s*".join([NUM] * 4), body)
    g["fold_circle_into_line_fib"] = {
        "dst": columns_after(body, "let dst_values"),
        "src": columns_after(body, "let src_values"),
        "dst_line_domain": cs[0],
        "src_circle_half_coset": cs[1],
        "alpha": [int(v) for v in alpha.groups()],
        "root_coset": cs[2],
        "twiddles": vec_after(body, "let twiddles"),
        "itwiddles": vec_after(body, "let itwiddles"),
    }

    body = fn_body(fri, "test_fold_line")
    even = re.search(r"even_coeffs: \[SecureField; DEGREE / 2\] = \[([\d,\s]+)\]", body).group(1)
    odd = re.search(r"odd_coeffs: \[SecureField; DEGREE / 2\] = \[([\d,\s]+)\]", body).group(1)
    g["fold_line_identity"] = {
        "degree": int(re.search(r"const DEGREE: usize = (\d+);", body).group(1)),
        "even": [int(x) for x in even.replace(" ", "").split(",") if x],
        "odd": [int(x) for x in odd.replace(" ", "").split(",") if x],
        "alpha": int(re.search(r"BaseField::from_u32_unchecked\((\d+)\)\.into\(\)", body).group(1)),
    }

    cases = []
    for name in ("test_accumulation", "test_accumulation_m31_arithmetic"):
        body = fn_body(acc, name)
        nums = lambda seg: [int(x) if x != "P - 1" else 2147483646
                            for x in re.findall(r"M31::from\((\d+|P - 1)\)", seg)]
        left = nums(body[body.index("left_summand"):body.index("right_summand")])
        right = nums(body[body.index("right_summand"):body.index("let mut left_secure_column")])
        exp = nums(body[body.index("expected_result"):])
        cases.append({"left": left, "right": right, "expected": exp})
    g["accumulation"] = cases

    pts = {}
    for c in cosets(poly) + cosets(fri):
        pts[c["initial_index"]] = c["initial"]
        pts[c["step_size"]] = c["step"]
    g["circle_points"] = [{"index": k, "point": v} for k, v in sorted(pts.items())]

    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
