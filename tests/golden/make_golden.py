"""Build the golden fixtures under tests/golden/ from the reference checkout.

Run once in a container that has the reference sources, with
``FORTFEM_REFERENCE`` set to the reference checkout::

    FORTFEM_REFERENCE=<path to lazy-fortran/fortfem> python tests/golden/make_golden.py

It reads the reference's fortsym-generated Nedelec tables as text and stores
only canonical digests of their exact rational entries (plus entry counts and a
few sample entries), so the tests can pin this repository's own exact
generator without copying the tables:

* ``src/generated/fortfem_tetra_nedelec_coefficients.f90`` (orders 1-4);
* ``src/generated/fortfem_tetra_face_moment_transforms.f90``
  (``basis_to_local_order_{2,3,4}``, six permutations each).
"""
from __future__ import annotations

import hashlib
import json
import os
import re
from fractions import Fraction

REF = os.environ.get("FORTFEM_REFERENCE", "")
HERE = os.path.dirname(os.path.abspath(__file__))

NUM = r"(-?\d+)\.0_real64(?:\s*/\s*(\d+)\.0_real64)?"


def canonical_digest(entries: dict) -> str:
    """sha256 over sorted 'row,col,num/den' lines of the non-zero entries (1-based)."""
    h = hashlib.sha256()
    for (r, c) in sorted(entries):
        v = Fraction(entries[(r, c)])
        if v == 0:
            continue
        h.update(f"{r},{c},{v.numerator}/{v.denominator}\n".encode())
    return h.hexdigest()


def parse_coefficients():
    path = os.path.join(REF, "src/generated/fortfem_tetra_nedelec_coefficients.f90")
    tables, order = {}, None
    case_re = re.compile(r"^\s*case \((\d+)\)")
    ent_re = re.compile(r"^\s*coefficients\((\d+),(\d+)\) = " + NUM)
    for line in open(path):
        m = case_re.match(line)
        if m:
            order = int(m.group(1))
            tables[order] = {}
            continue
        m = ent_re.match(line)
        if m and order is not None:
            num = int(m.group(3))
            den = int(m.group(4)) if m.group(4) else 1
            tables[order][(int(m.group(1)), int(m.group(2)))] = Fraction(num, den)
    return tables


def parse_face_transforms():
    path = os.path.join(REF, "src/generated/fortfem_tetra_face_moment_transforms.f90")
    text = open(path).read()
    out = {}
    for order in (2, 3, 4):
        m = re.search(rf"subroutine basis_to_local_order_{order}\(.*?end subroutine basis_to_local_order_{order}",
                      text, re.S)
        body = m.group(0)
        size = order * (order - 1)
        for case in re.finditer(r"case \((\d)\)\s*transform = reshape\(\[(.*?)\], shape", body, re.S):
            perm = int(case.group(1))
            vals = [Fraction(int(a), int(b) if b else 1) for a, b in re.findall(NUM, case.group(2))]
            assert len(vals) == size * size
            ent = {}
            for idx, v in enumerate(vals):  # Fortran reshape: column-major
                ent[(idx % size + 1, idx // size + 1)] = v
            out[(order, perm)] = ent
    return out


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "src", "generated")):
        raise SystemExit("set FORTFEM_REFERENCE to a lazy-fortran/fortfem checkout "
                         "(the directory holding src/generated)")
    coeffs = parse_coefficients()
    faces = parse_face_transforms()
    fixture = {"source": "reference src/generated (fortsym@ca903547), digests only",
               "coefficients": {}, "face_transforms": {}}
    for order, ent in sorted(coeffs.items()):
        nz = {k: v for k, v in ent.items() if v != 0}
        sample = sorted(nz)[:: max(1, len(nz) // 8)][:8]
        fixture["coefficients"][str(order)] = {
            "digest": canonical_digest(nz), "nonzeros": len(nz),
            "samples": [[r, c, str(nz[(r, c)])] for r, c in sample]}
    for (order, perm), ent in sorted(faces.items()):
        nz = {k: v for k, v in ent.items() if v != 0}
        fixture["face_transforms"][f"{order}/{perm}"] = {
            "digest": canonical_digest(nz), "nonzeros": len(nz)}
    with open(os.path.join(HERE, "nedelec_tables.json"), "w") as fh:
        json.dump(fixture, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "nedelec_tables.json"))


if __name__ == "__main__":
    main()
