"""Regenerate the golden fixtures of this directory from the reference's tests.

The reference (rapidfem) pins its DGTD kernels with sympy-exact tables that
live as Rust `const` arrays in

  crates/rapidfem-td/tests/dg_basis_golden_test.rs   (M, Dr, Ds, Dt, p=1..3)
  crates/rapidfem-td/tests/rhs_curl_golden_test.rs   (element_curl, p=2)
  crates/rapidfem-td/tests/propagator_expm_test.rs   (exp(hA) v0, 6x6 skew A)

This script reads those files as text and writes the numbers into JSON
fixtures, so the tests never need the reference tree at run time.

Usage:  python tests/golden/make_golden.py REFERENCE_ROOT
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CONST_RE = re.compile(r"^const\s+([A-Z0-9_]+)\s*:\s*([^=]+)=\s*(.*);\s*$", re.M)


def parse_consts(path):
    src = open(path).read()
    out = {}
    for name, ty, body in CONST_RE.findall(src):
        nums = [float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", body)]
        if "usize" in ty:
            out[name] = int(nums[0])
        elif ty.strip() == "f64":
            out[name] = nums[0]
        else:
            out[name] = nums
    return out


def main(root):
    tdir = os.path.join(root, "crates", "rapidfem-td", "tests")
    basis = parse_consts(os.path.join(tdir, "dg_basis_golden_test.rs"))
    curl = parse_consts(os.path.join(tdir, "rhs_curl_golden_test.rs"))
    prop = parse_consts(os.path.join(tdir, "propagator_expm_test.rs"))
    fixtures = {
        "dg_basis.json": {
            "source": "crates/rapidfem-td/tests/dg_basis_golden_test.rs",
            "tables": {k: v for k, v in basis.items()},
        },
        "rhs_curl.json": {
            "source": "crates/rapidfem-td/tests/rhs_curl_golden_test.rs",
            "order": 2,
            "tet": curl["TET"],
            "field": curl["FIELD"],
            "curl": curl["CURL"],
        },
        "propagator_expm.json": {
            "source": "crates/rapidfem-td/tests/propagator_expm_test.rs",
            "n": 6,
            "a": prop["A"],
            "v0": prop["V0"],
            "cases": [[prop["H0"], prop["REF0"]], [prop["H1"], prop["REF1"]], [prop["H2"], prop["REF2"]]],
        },
    }
    for name, data in fixtures.items():
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(data, f, indent=0)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <root of the rapidfem source tree>")
    main(sys.argv[1])
