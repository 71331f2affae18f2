"""Converts the reference's golden OMF fixtures into tests/golden/ref_fields.npz.

Source files (read from the reference tree, which exists only in the build container):
  src/magnum_tests/ref/M1.omf         magnetisation, 200x50x1 cells, 2.5x2.5x3 nm (SP4 state)
  src/magnum_tests/ref/H1_exch.omf    exchange field of M1, A = 13e-12, Ms = 8e5 (exchange_test.py:31-53)
  src/magnum_tests/ref/H1_stray.omf   stray field of M1, PADDING_ROUND_4 (stray_field_test.py:29-50)
  src/magnum_tests/ref/H1_unianiso.omf uniaxial field of M1, axis (1,1,1)/sqrt3, k = 520e3, Ms = 8e5
                                       (anisotropy_test.py:30-47, ref/H1_unianiso.txt)
Run:  python tests/golden/make_golden.py /path/to/src/magnum_tests/ref
      (or set MMB200_REFERENCE to the checkout's root)
The OMF 'Data Text' section lists one vector per line, x fastest, then y, then z.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_omf_text(path):
    header, rows, in_data = {}, [], False
    with open(path) as f:
        for line in f:
            s = line.strip()
            if s.startswith("#"):
                body = s[1:].strip()
                if body.lower().startswith("begin: data text"):
                    in_data = True
                elif body.lower().startswith("end: data"):
                    in_data = False
                elif ":" in body:
                    k, v = body.split(":", 1)
                    header[k.strip().lower()] = v.strip()
                continue
            if in_data and s:
                rows.append([float(t) for t in s.split()])
    nx, ny, nz = (int(header[k]) for k in ("xnodes", "ynodes", "znodes"))
    d = tuple(float(header[k]) for k in ("xstepsize", "ystepsize", "zstepsize"))
    arr = np.asarray(rows, dtype=np.float64)
    assert arr.shape == (nx * ny * nz, 3), (path, arr.shape)
    return arr.T.copy(), (nx, ny, nz), d


def main(refdir):
    out = {}
    for name in ("M1", "H1_exch", "H1_stray", "H1_unianiso"):
        field, dims, delta = read_omf_text(os.path.join(refdir, name + ".omf"))
        out[name] = field
        out["dims"] = np.array(dims)
        out["delta"] = np.array(delta)
    np.savez_compressed(os.path.join(HERE, "ref_fields.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_fields.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("MMB200_REFERENCE"):
        main(os.path.join(os.environ["MMB200_REFERENCE"], "src", "magnum_tests", "ref"))
    else:
        sys.exit("usage: make_golden.py <src/magnum_tests/ref> (or set MMB200_REFERENCE)")
