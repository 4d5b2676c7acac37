"""Extracts the constants of the lattice model from the reference's Fortran
source into reference_constants.json, a fixture the CPU tests compare the
oracle and the library with (the reference cannot be built here, so its
source text is the record of these values):

  matm rows        solution.f90:17-25   (the MRT transform M)
  e(k,:), w(k)     D2Q9model.f90:5-32   (lattice order and weights, as written)
  mesh%s(1..9)     ini_mesh.f90:59-67   (relaxation rates; 8 and 9 are 1/tau_f)
  kernel branches  boundary_condition.f90 (immersed_boundary_Wu's first kernel block)
  D2Q9feq          D2Q9model.f90:35-46  (the equilibrium)
  colission        solution.f90:605-633 (equilibrium moments, forcing, relaxation)

Run here, where the reference tree is present:
    python tests/golden/make_reference_constants.py <reference dir>
"""
import json
import os
import re
import sys


def read(ref, name):
    with open(os.path.join(ref, name), encoding="utf-8", errors="replace") as fh:
        return fh.read()


def fnum(tok):
    return float(tok.lower().replace("d", "e"))


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_reference_constants.py <reference source directory>")
    ref = sys.argv[1]
    sol = read(ref, "solution.f90")
    rows = {}
    for m in re.finditer(r"matm\((\d)\s*,\s*:\s*\)\s*=\s*\(/([^/]*)/\)", sol):
        rows[int(m.group(1))] = [fnum(t) for t in m.group(2).split(",")]
    assert sorted(rows) == list(range(1, 10)), rows.keys()
    d2q9 = read(ref, "D2Q9model.f90")
    e = {}
    for m in re.finditer(r"\be\((\d)\s*,\s*(\d)\)\s*=\s*(-?\d+)", d2q9):
        e.setdefault(int(m.group(1)), [0, 0])[int(m.group(2)) - 1] = int(m.group(3))
    w = {}
    for m in re.finditer(r"\bw\((\d)\)\s*=\s*([0-9.]+/[0-9.]+)", d2q9):
        w[int(m.group(1))] = m.group(2)
    mesh = read(ref, "ini_mesh.f90")
    s = {}
    for m in re.finditer(r"%s\((\d)\)\s*=\s*([^\s!]+)", mesh):
        k, v = int(m.group(1)), m.group(2)
        s.setdefault(k, v)
    # the discrete delta kernels: the x-axis branches of each smooth variant in
    # the first kernel block of immersed_boundary_Wu, verbatim (condition,
    # expression)
    bc = read(ref, "boundary_condition.f90").splitlines()
    sub = next(i for i, l in enumerate(bc) if re.match(r"(?i)\s*subroutine\s+immersed_boundary_Wu", l))
    i0 = next(i for i in range(sub, len(bc)) if bc[i].strip().lower().startswith("if(smooth.eq.0)"))

    def block(first):
        a = next(i for i in range(first, len(bc)) if "disr=abs((x0" in bc[i].replace(" ", ""))
        b = next(i for i in range(a + 1, len(bc)) if "disr=abs((y0" in bc[i].replace(" ", ""))
        out, cond = [], None
        for line in bc[a + 1:b]:
            t = line.strip()
            m = re.match(r"(?i)(?:else\s*)?if\s*\((.*)\)\s*then$", t)
            if m:
                cond = m.group(1)
            elif t.lower() == "else":
                cond = "else"
            m = re.match(r"kernel1\s*=\s*(.*)$", t)
            if m:
                out.append([cond, m.group(1)])
        return out, b

    kern0, end0 = block(i0)
    kern1, _ = block(end0 + 1)
    kern = {0: kern0, 1: kern1}
    # the equilibrium D2Q9feq (D2Q9model.f90:35-46), its three assignments verbatim
    body = d2q9[d2q9.lower().index("function d2q9feq"):]
    body = body[:body.lower().index("end function")]
    feq = {}
    for name in ("eu", "utwo", "D2Q9feq"):
        m = re.search(r"(?im)^\s*" + name + r"\s*=\s*(.*)$", body)
        feq[name] = m.group(1).strip()
    # colission's per-node equilibrium moments and forcing (solution.f90:605-626), verbatim
    col = sol[sol.lower().index("subroutine colission"):]
    col = col[:col.lower().index("end subroutine")]
    temp = {}
    for m in re.finditer(r"(?m)^\s*temp\((\d)\)\s*=\s*(.*)$", col):
        temp.setdefault(int(m.group(1)), m.group(2).strip())
    fp = {}
    for m in re.finditer(r"(?m)^\s*fp\((\d)\)\s*=\s*(.*)$", col):
        fp.setdefault(int(m.group(1)), m.group(2).strip())
    relax = re.search(r"(?m)^\s*(temp\(k\)\s*=\s*temp1\(k\).*)$", col).group(1).strip()
    pai = None
    for name in ("main.f90", "mode.f90", "solution.f90"):
        m = re.search(r"pai\s*=\s*([0-9.d+-]+)", read(ref, name))
        if m:
            pai = m.group(1)
            break
    out = {
        "source": {"matm": "solution.f90:17-25", "e_w": "D2Q9model.f90:5-32", "s": "ini_mesh.f90:59-67",
                   "kernels": "boundary_condition.f90, first kernel1 block of immersed_boundary_Wu"},
        "kernel_branches": {"0": kern[0], "1": kern[1]},
        "feq": feq,
        "collision": {"temp": [temp[k] for k in range(1, 10)], "fp": [fp[k] for k in range(1, 10)],
                      "relax": relax},
        "pai_literal": pai,
        "matm": [rows[k] for k in range(1, 10)],
        "e": [e[k] for k in range(1, 10)],
        "w_literal": [w[k] for k in range(1, 10)],
        "s_literal": [s[k] for k in range(1, 10)],
    }
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_constants.json")
    with open(path, "w") as fh:
        json.dump(out, fh, indent=1)
    print(path)


if __name__ == "__main__":
    main()
