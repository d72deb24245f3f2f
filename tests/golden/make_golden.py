"""Extract the golden fixture from the reference's only known-answer run.

The FORTRESS sources ship one complete output: OUTPUT/ of the 1D spin-2
spin-orbit-coupled imaginary-time run of INPUT/input1D.dat (NX=2048, DX=0.05,
DT=1.25e-4, STP=400, converged at iteration 399200).  This script copies the
input records and a sample of the output rows (as printed, no re-rounding)
into tests/golden/fortress_1d_spin2.json.  It reads the reference tree, so it
runs where that tree is mounted; the JSON it writes is what the tests use.

    python tests/golden/make_golden.py /path/to/FORTRESS
"""
import json
import os
import sys


def rows(path):
    with open(path) as f:
        return [ln.rstrip("\n") for ln in f if ln.strip()]


def sample(lines, head=12, every=25, tail=4):
    keep = set(range(min(head, len(lines))))
    keep |= set(range(0, len(lines), every))
    keep |= set(range(max(0, len(lines) - tail), len(lines)))
    return [[i, lines[i]] for i in sorted(keep)]


def main(root):
    out_dir = os.path.join(root, "OUTPUT")
    g = {
        "source": "FORTRESS OUTPUT/ for INPUT/input1D.dat (1D spin-2, imaginary time)",
        "input1D": open(os.path.join(root, "INPUT", "input1D.dat")).read(),
        "file1": rows(os.path.join(out_dir, "file1_im_spin2.dat")),
        "file2": sample(rows(os.path.join(out_dir, "file2_im_spin2.dat"))),
        "file3": sample(rows(os.path.join(out_dir, "file3_im_spin2.dat"))),
        "convergence": sample(rows(os.path.join(out_dir, "convergence.dat"))),
        "n_rows": len(rows(os.path.join(out_dir, "file2_im_spin2.dat"))),
        "solution": [[i, ln] for i, ln in enumerate(rows(os.path.join(out_dir, "solution_file_im_spin2.dat")))
                     if i % 8 == 0 or 1016 <= i <= 1032],
    }
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fortress_1d_spin2.json")
    with open(dst, "w") as f:
        json.dump(g, f, indent=0)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/FORTRESS")
    main(sys.argv[1])
