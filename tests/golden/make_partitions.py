"""Fixture of the reference's unit-sphere partitions (its data files
unit_sphere_partitions/unit_sphere_partition_<N>.txt), stored as their raw
text, for the tests of the sphere discretisation and of the generated
recursive zonal equal-area points.

Usage: python tests/golden/make_partitions.py [reference_dir]
Writes: tests/golden/unit_sphere_partitions.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("D3Q19_REFERENCE")
    if not ref:
        sys.exit("usage: make_partitions.py <reference_dir> (or set D3Q19_REFERENCE)")
    d = os.path.join(ref, "unit_sphere_partitions")
    out = {}
    for fn in sorted(os.listdir(d)):
        n = int(fn.rsplit("_", 1)[1].split(".")[0])
        with open(os.path.join(d, fn), "rb") as fh:
            out[f"p{n}"] = np.frombuffer(fh.read(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "unit_sphere_partitions.npz"), **out)
    print(sorted(out))


if __name__ == "__main__":
    main()
