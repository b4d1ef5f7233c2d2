"""Regenerate ``sensor_tables.csv`` from the reference renderer's CIE data files.

The sensor tables are published standards data, not code: the CIE 1931 2-degree
colour-matching functions and the CIE D65 / illuminant A spectral power
distributions, tabulated at 5 nm from 380 to 730 nm.  The reference renderer
embeds exactly these rows (``spectral-core/data/*.csv``, loaded by
``spectral-core/src/cie.rs:6-8``); parity with its film requires the identical
decimal strings, so this script copies the rows verbatim (no float round trip)
into one table with columns ``nm,xbar,ybar,zbar,d65,a``.

Usage (needs the reference checkout):
    python spectral_b200/data/make_sensor_tables.py <reference-root>
"""
import hashlib
import os
import sys


def _rows(path):
    with open(path) as f:
        return [ln.strip().split(",") for ln in f if ln.strip()]


def main(ref_root):
    data = os.path.join(ref_root, "spectral-core", "data")
    cmf = _rows(os.path.join(data, "cie_1931_2deg.csv"))
    d65 = _rows(os.path.join(data, "illuminant_d65.csv"))
    ill_a = _rows(os.path.join(data, "illuminant_a.csv"))
    assert len(cmf) == len(d65) == len(ill_a) == 71
    digest = hashlib.sha256()
    for name in ("cie_1931_2deg.csv", "illuminant_d65.csv", "illuminant_a.csv"):
        with open(os.path.join(data, name), "rb") as f:
            digest.update(f.read())
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sensor_tables.csv")
    with open(out, "w") as f:
        f.write("# CIE 1931 2deg CMF + D65 + A SPD, 5 nm, 380..730 nm\n")
        f.write("# source sha256 (cmf|d65|a concatenated): %s\n" % digest.hexdigest())
        f.write("nm,xbar,ybar,zbar,d65,a\n")
        for c, d, a in zip(cmf, d65, ill_a):
            assert c[0].strip() == d[0].strip() == a[0].strip()
            f.write(",".join([c[0].strip(), c[1].strip(), c[2].strip(), c[3].strip(),
                              d[1].strip(), a[1].strip()]) + "\n")
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python spectral_b200/data/make_sensor_tables.py <reference-root>")
    main(sys.argv[1])
