"""Regenerates the golden fixtures of tests/golden/.

helper_math_golden.jsonl -- length(), normalize() and cross() evaluated by
    the reference's own src/helper_math_double.h (host build), compiled from
    the reference tree by `make -C oracle probe` (recipe: oracle/Makefile,
    program: oracle/ref_helper_probe.cpp).  Needs the reference checkout, so
    it runs only where the reference is mounted; the output is committed.
oracle_small.npz -- one-step outputs of the CPU oracle on two small scenes
    (regression fixtures for the oracle itself).

Usage: python tests/golden/make_golden.py [--ref /path/to/DVIDE]
"""
import argparse
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def helper_golden(ref):
    subprocess.check_call(["make", "-C", os.path.join(ROOT, "oracle"), "probe", f"REF={ref}"])
    out = subprocess.check_output([os.path.join(ROOT, "oracle", "_ref", "ref_helper_probe")])
    with open(os.path.join(HERE, "helper_math_golden.jsonl"), "wb") as f:
        f.write(out)


def oracle_fixtures():
    from dvide_b200 import scenes
    from oracle import oracle as O
    O.build()
    data = {}
    for name, sc, steps in (("ball", scenes.ball_on_ground(), 3),
                            ("cluster", scenes.random_cluster(7, n=12), 2)):
        o = O.OracleScene(sc)
        o.step(steps)
        p, v = o.state()
        a, b, nP, loc = o.contacts()
        data[f"{name}_p"] = p
        data[f"{name}_v"] = v
        data[f"{name}_gamma"] = o.gamma()
        data[f"{name}_a"] = a
        data[f"{name}_b"] = b
        data[f"{name}_nP"] = nP
        data[f"{name}_iterations"] = np.array([o.stats()["iterations"]])
    np.savez(os.path.join(HERE, "oracle_small.npz"), **data)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None,
                    help="reference source tree (needed for the helper_math golden vectors)")
    args = ap.parse_args()
    if args.ref and os.path.isdir(os.path.join(args.ref, "src")):
        helper_golden(args.ref)
    oracle_fixtures()
