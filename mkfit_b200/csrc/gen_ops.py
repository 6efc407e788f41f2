#!/usr/bin/env python3
"""Code generator for the register-unrolled small-matrix products of the
Kalman hot path (B200 CUDA device code).

In the spirit of the reference's GenMul (Matriplex/GenMul.pm:482-634 and the
sparsity patterns in mkFit/GenMPlexOps.pl:143-324), each product is written
out element by element with the known zero / one entries of the operands
folded away, so the compiler sees straight-line FMA chains on scalars that
live in registers. The emitted code works on one track per CUDA thread
(scalars, not Matriplex lanes).

Besides the header, the generator counts the floating-point operations of
every product (FMA = 2, MUL/ADD = 1); these counts are the algorithmic FLOPs
used for roofline numbers (written to ops_flops.json).

Run:  python gen_ops.py   (rewrites generated_ops.cuh and ops_flops.json)
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))

# Packed lower-triangle index of a symmetric matrix element (i, j).
def sym_idx(i, j):
    if i < j:
        i, j = j, i
    return i * (i + 1) // 2 + j


def parse_pattern(text):
    return [row.split() for row in text.strip().splitlines()]


class Mat:
    """Operand description: name, shape, pattern ('x' = variable, '0', '1'),
    and whether storage is symmetric-packed or full row-major."""

    def __init__(self, name, rows, cols, pattern=None, sym=False, transpose_of=None):
        self.name, self.rows, self.cols, self.sym = name, rows, cols, sym
        if pattern is None:
            pattern = [["x"] * cols for _ in range(rows)]
        self.pattern = pattern

    def entry(self, i, j):
        p = self.pattern[i][j]
        if p == "0":
            return None
        if p == "1":
            return "1"
        if self.sym:
            return f"{self.name}[{sym_idx(i, j)}]"
        return f"{self.name}[{i * self.cols + j}]"

    def transposed(self, name=None):
        t = Mat(name or self.name, self.cols, self.rows,
                [[self.pattern[j][i] for j in range(self.rows)] for i in range(self.cols)],
                self.sym)
        t._src = self
        return t


class TMat(Mat):
    """Transposed view that reads the original's storage."""

    def __init__(self, base):
        super().__init__(base.name, base.cols, base.rows,
                         [[base.pattern[j][i] for j in range(base.rows)] for i in range(base.cols)],
                         base.sym)
        self.base = base

    def entry(self, i, j):
        return self.base.entry(j, i)


def product(a, b, out_name, out_sym=False, out_pattern=None):
    """Emit out = a * b. Returns (lines, flops, out Mat)."""
    assert a.cols == b.rows
    rows, cols = a.rows, b.cols
    lines, flops = [], 0
    pat = [["0"] * cols for _ in range(rows)]
    for i in range(rows):
        for j in range(cols):
            if out_sym and j > i:
                continue
            terms, consts = [], 0
            for k in range(a.cols):
                ea, eb = a.entry(i, k), b.entry(k, j)
                if ea is None or eb is None:
                    continue
                if ea == "1" and eb == "1":
                    consts += 1
                    terms.append("1.f")
                elif ea == "1":
                    terms.append(eb)
                elif eb == "1":
                    terms.append(ea)
                else:
                    terms.append(f"{ea} * {eb}")
            if out_pattern is not None and out_pattern[i][j] == "0":
                continue
            idx = sym_idx(i, j) if out_sym else i * cols + j
            if not terms:
                lines.append(f"  {out_name}[{idx}] = 0.f;")
                continue
            pat[i][j] = "x"
            if out_sym:
                pat[j][i] = "x"
            # Each product term after the first costs an FMA (2 flops); a first
            # product costs one MUL; plain additions of copies cost one ADD.
            n_mul = sum(1 for t in terms if "*" in t)
            n_copy = len(terms) - n_mul
            if n_mul:
                f = 1 + 2 * (n_mul - 1) + n_copy
            else:
                f = max(0, n_copy - 1)
            flops += f
            lines.append(f"  {out_name}[{idx}] = {' + '.join(terms)};")
    return lines, flops, Mat(out_name, rows, cols, pat, out_sym)


def emit_function(name, doc, params, body, flops):
    head = f"// {doc}\n// Algorithmic FLOPs (FMA = 2): {flops}\n"
    return (head + f"__device__ __forceinline__ void {name}({params})\n{{\n"
            + "\n".join(body) + "\n}\n")


def main():
    funcs, counts = [], {}

    # ---------------------------------------------------------------- barrel
    # Helix propagation Jacobian to a cylinder, CCS coordinates.
    # Pattern as in mkFit/GenMPlexOps.pl:254-265 (errProp for MultHelixProp).
    jb = parse_pattern("""
x x 0 x x 0
x x 0 x x 0
x x 1 x x x
x x 0 x x 0
x x 0 x x 0
0 0 0 0 0 1
""")
    # The barrel Jacobian's row 3 is (0 0 0 1 0 0) in this implementation
    # (1/pT is not changed by the helix step), which removes further terms.
    jb[3] = "0 0 0 1 0 0".split()
    J = Mat("J", 6, 6, jb)
    C = Mat("C", 6, 6, sym=True)
    l1, f1, T = product(J, C, "T")
    l2, f2, _ = product(T, TMat(J), "Cout", out_sym=True)
    funcs.append(emit_function(
        "similarity_barrel",
        "Cout = J * C * J^T for the barrel helix Jacobian (C, Cout packed symmetric)",
        "const float (&J)[36], const float (&C)[21], float (&Cout)[21]",
        ["  float T[36];"] + l1 + l2, f1 + f2))
    counts["similarity_barrel"] = f1 + f2

    # ---------------------------------------------------------------- endcap
    # Pattern as in mkFit/GenMPlexOps.pl:296-303 (errProp, endcap version).
    je = parse_pattern("""
1 0 x x x x
0 1 x x x x
0 0 0 0 0 0
0 0 0 1 0 0
0 0 x x 1 x
0 0 0 0 0 1
""")
    J = Mat("J", 6, 6, je)
    l1, f1, T = product(J, C, "T")
    l2, f2, _ = product(T, TMat(J), "Cout", out_sym=True)
    funcs.append(emit_function(
        "similarity_endcap",
        "Cout = J * C * J^T for the endcap (propagate-to-z) Jacobian",
        "const float (&J)[36], const float (&C)[21], float (&Cout)[21]",
        ["  float T[36];"] + l1 + l2, f1 + f2))
    counts["similarity_endcap"] = f1 + f2

    # ---------------------------------------------------------------- K H C
    # Barrel update: KH has non-zero columns 0..2 (mkFit/GenMPlexOps.pl:168-180),
    # result is symmetric: Out = KH * C (lower triangle).
    kh = parse_pattern("""
x x x 0 0 0
x x x 0 0 0
x x x 0 0 0
x x x 0 0 0
x x x 0 0 0
x x x 0 0 0
""")
    KH = Mat("KH", 6, 6, kh)
    l1, f1, _ = product(KH, C, "Out", out_sym=True)
    funcs.append(emit_function(
        "khc_barrel", "Out = KH * C (KH with three live columns; Out packed symmetric)",
        "const float (&KH)[36], const float (&C)[21], float (&Out)[21]", l1, f1))
    counts["khc_barrel"] = f1

    # Endcap update: K is 6x2 (mkFit/GenMPlexOps.pl:186-200): Out = K * C[0:2,:].
    K2 = Mat("K", 6, 2)
    C2 = Mat("C", 2, 6)
    C2.sym = True  # rows 0..1 of the symmetric C
    l1, f1, _ = product(K2, C2, "Out", out_sym=True)
    funcs.append(emit_function(
        "khc_endcap", "Out = K * C[0:2,:] (K is 6x2; Out packed symmetric)",
        "const float (&K)[12], const float (&C)[21], float (&Out)[21]", l1, f1))
    counts["khc_endcap"] = f1

    header = ("// GENERATED by gen_ops.py -- do not edit by hand.\n"
              "// Register-unrolled small-matrix products for the Kalman hot path.\n"
              "#pragma once\n\nnamespace mkfg {\n\n" + "\n".join(funcs) + "\n}  // namespace mkfg\n")
    with open(os.path.join(HERE, "generated_ops.cuh"), "w") as f:
        f.write(header)
    with open(os.path.join(HERE, "ops_flops.json"), "w") as f:
        json.dump(counts, f, indent=1, sort_keys=True)
    print(json.dumps(counts))


if __name__ == "__main__":
    main()
