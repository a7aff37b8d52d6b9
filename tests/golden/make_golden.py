"""Regenerates the golden fixtures in this folder from the reference's own test data.

Run from the repository root in a container that has the reference tree, given as the argument or
in the environment variable GPT_REFERENCE_DIR:
    GPT_REFERENCE_DIR=<reference tree> python tests/golden/make_golden.py

It reads the reference's known-answer files (testfiles/0_0_eepos.traj, the
forward kinematics of every row of testfiles/0_0_traj.csv written by
generateeepos.cu:101-107) and the explicit-Euler dt=1/64 trajectories
testfiles/*_traj.csv, and stores them as float32 arrays in reference_testfiles.npz.
Nothing at test time reads the reference tree.
"""
import glob
import os
import sys

import numpy as np


def main(ref_root):
    tf = os.path.join(ref_root, "testfiles")
    out = {}
    out["traj_0_0"] = np.loadtxt(os.path.join(tf, "0_0_traj.csv"), delimiter=",").astype(np.float32)
    out["eepos_0_0"] = np.loadtxt(os.path.join(tf, "0_0_eepos.traj"), delimiter=",").astype(np.float32)
    for f in sorted(glob.glob(os.path.join(tf, "*_traj.csv"))):
        name = os.path.basename(f)[:-len("_traj.csv")]
        if name == "0_0":
            continue
        out[f"traj_{name}"] = np.loadtxt(f, delimiter=",").astype(np.float32)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_testfiles.npz")
    np.savez_compressed(dst, **out)
    print("wrote", dst, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GPT_REFERENCE_DIR")
    if not root or not os.path.isdir(root):
        sys.exit("make_golden.py: give the reference tree as the argument or in GPT_REFERENCE_DIR")
    main(root)
