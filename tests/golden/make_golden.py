"""Extracts the reference's golden vectors into small fixtures (run in the
container that has the NanoGW tree; the fixtures are committed).

* lanczos_h_aux.npz  <- shared/test_lanczos/H_aux_v0.txt : the 104x104 auxiliary
  Hamiltonian, the start vector v0 and the golden table
  (z, S(0).real, S(z+0.1i).real, S(z+0.1i).imag) written by the reference's
  notebook with niter = 5 (= 4 Lanczos levels).
* libxc_lda.npz      <- LIB/libxc/testsuite/lda_x.data, lda_c_pz.data :
  (rhoa, rhob, zk, vrhoa, vrhob, v2rhoa2, v2rhoab, v2rhob2) per point.

Usage: python tests/golden/make_golden.py /path/to/NanoGW
"""
import os
import re
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit("usage: make_golden.py /path/to/NanoGW  (the reference source tree)")
REF = sys.argv[1]
OUT = os.path.dirname(os.path.abspath(__file__))


def lanczos_fixture():
    lines = open(os.path.join(REF, "shared/test_lanczos/H_aux_v0.txt")).read().split("\n")
    n = int(lines[0].split()[1])
    H = np.zeros((n, n))
    for k in range(n * n):
        i, j, v = lines[1 + k].split()
        H[int(i), int(j)] = float(v)
    assert lines[1 + n * n].split()[0] == "v0"
    v0 = np.array([float(lines[2 + n * n + k].split()[1]) for k in range(n)])
    header = lines[2 + n * n + n]
    niter = int(header.split("niter=")[1])
    tab = np.array([[float(x) for x in l.split()] for l in lines[3 + n * n + n:] if l.strip()])
    np.savez_compressed(os.path.join(OUT, "lanczos_h_aux.npz"), H=H, v0=v0, table=tab,
                        niter=niter, eta=0.1)


def libxc_fixture():
    out = {}
    for name in ("lda_x", "lda_c_pz"):
        txt = open(os.path.join(REF, "LIB/libxc/testsuite", name + ".data")).read()
        rows = []
        for block in txt.split(" rhoa=")[1:]:
            head = block.split("\n")[0]
            rhoa = float(head.split()[0])
            rhob = float(re.search(r"rhob=\s*(\S+)", head).group(1))
            vals = dict(re.findall(r"(\w+)\s*=\s*(\S+)", block))
            rows.append([rhoa, rhob] + [float(vals[k]) for k in
                                        ("zk", "vrhoa", "vrhob", "v2rhoa2", "v2rhoab", "v2rhob2")])
        out[name] = np.array(rows)
    np.savez_compressed(os.path.join(OUT, "libxc_lda.npz"), **out)


if __name__ == "__main__":
    lanczos_fixture()
    libxc_fixture()
    print("fixtures written to", OUT)
