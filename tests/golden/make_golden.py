"""Runs the reference's own GPU drivers (compiled unmodified by oracle/Makefile into oracle/_ref/)
on the golden inputs and stores their full-precision outputs as fixtures.  Needs a B200.

    python tests/golden/make_golden.py [--la path/to/LosAngeles.txt]

Writes, next to this file:
  ref_g2k_mhl.txt   BC of g2k.txt by Graph::brandesBCIndexGPU_5 of MHLQBC.cu   ("vid bc", %.17g)
  ref_g2k_qbc.txt   BC of g2k.txt + g2k.order by Graph::brandesBCIndexGPU_5 of QBC.cu
  ref_g2k_rq.txt    BC of the g2k.query vertices by brandesBCIndexGPU_PointBatch of RQ.cu
  ref_la_mhl.npz    BC of the LosAngeles graph by MHLQBC.cu (when --la is given)
  ref_timings.json  wall times of those runs (index build alone, and the whole driver call)
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref")


def run(binary, args, out_path):
    with tempfile.TemporaryDirectory() as wd:  # the drivers write tmpRoadCountIndex into the CWD
        r = subprocess.run([os.path.join(REF, binary), *args, out_path], cwd=wd, capture_output=True, text=True,
                           timeout=1800)
    if r.returncode != 0:
        sys.stderr.write(r.stdout[-4000:] + r.stderr[-4000:])
        raise SystemExit(f"{binary} failed with {r.returncode}")
    last = [ln for ln in r.stdout.splitlines() if ln.startswith("{")][-1]
    return json.loads(last)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--la", default=None)
    a = ap.parse_args()
    if a.la:
        a.la = os.path.abspath(a.la)
    g = os.path.join(HERE, "g2k.txt")
    timings = {}
    timings["g2k_mhl"] = run("ref_mhlqbc", [g], os.path.join(HERE, "ref_g2k_mhl.txt"))
    timings["g2k_qbc"] = run("ref_qbc", [g, os.path.join(HERE, "g2k.order")], os.path.join(HERE, "ref_g2k_qbc.txt"))
    timings["g2k_rq"] = run("ref_rq", [g, os.path.join(HERE, "g2k.query")], os.path.join(HERE, "ref_g2k_rq.txt"))
    if a.la:
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "la.txt")
            timings["la_mhl"] = run("ref_mhlqbc", [a.la], p)
            bc = np.loadtxt(p)[:, 1]
        np.savez_compressed(os.path.join(HERE, "ref_la_mhl.npz"), bc=bc)
    with open(os.path.join(HERE, "ref_timings.json"), "w") as f:
        json.dump(timings, f, indent=1)
    print(json.dumps(timings))


if __name__ == "__main__":
    main()
