"""Turns the reference program's text outputs (from make_ref_golden.sh) into
small .npz fixtures:

  ey_centre[t]   ey at (NX/2, NY/2, NZ/2) after step t-1, printed by the
                 reference's per-step printf (main.cu:2726), 7 digits
  scatabs_<t>    the 19-column ScatAbs.<t>.txt (Spectral.cu:1157-1174)
  yz_<n>, yz_<n>_N, aux_<n>, aux_<n>_2
                 the snapshot files videofiles/YZ_sim.<n>[_N].txt and
                 aux_sim.<n>[_2].txt (snapshot.cu), when the deck wrote them

    python tests/golden/import_ref_golden.py <directory holding the reference's outputs>
"""
import glob
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_case(d):
    out = {}
    t, ey = [], []
    sp = os.path.join(d, "stdout.txt")
    for line in open(sp) if os.path.exists(sp) else []:
        parts = line.split()
        if len(parts) == 4 and re.fullmatch(r"\d+", parts[0]) and parts[1] == "1":
            t.append(int(parts[0]))
            ey.append(float(parts[2]))
    if t:
        out["ey_t"] = np.array(t, np.int32)
        out["ey_centre"] = np.array(ey)
    files = sorted(glob.glob(os.path.join(d, "ScatAbs.*.txt")),
                   key=lambda p: int(p.split(".")[-2]))
    steps = [int(p.split(".")[-2]) for p in files]
    # keep the last two dumps (the spectra the run converges to)
    for p, s in list(zip(files, steps))[-2:]:
        out[f"scatabs_{s}"] = np.loadtxt(p)
    for p in glob.glob(os.path.join(d, "videofiles", "YZ_sim.*.txt")):
        tag = os.path.basename(p)[len("YZ_sim."):-len(".txt")]
        out[f"yz_{tag}"] = np.loadtxt(p, ndmin=2)
    for p in glob.glob(os.path.join(d, "aux_sim.*.txt")):
        tag = os.path.basename(p)[len("aux_sim."):-len(".txt")]
        out[f"aux_{tag}"] = np.loadtxt(p, ndmin=1)
    return out


def main(src):
    for d in sorted(glob.glob(os.path.join(src, "*"))):
        if not os.path.isdir(d):
            continue
        rc = open(os.path.join(d, "rc.txt")).read()
        if "rc=0" not in rc:
            print("skip", d, rc)
            continue
        name = os.path.basename(d)
        data = load_case(d)
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), **data)
        print(name, {k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main(sys.argv[1])
