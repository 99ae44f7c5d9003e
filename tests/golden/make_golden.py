"""Runs the reference's own GPU drivers (compiled unmodified by oracle/Makefile into oracle/_ref/)
on the golden inputs and stores their full-precision outputs as fixtures.  Needs a B200.

    python tests/golden/make_golden.py [--la path/to/LosAngeles.txt] [--g50k]

Writes, next to this file:
  ref_g2k_mhl.txt   BC of g2k.txt by Graph::brandesBCIndexGPU_5 of MHLQBC.cu   ("vid bc", %.17g)
  ref_g2k_qbc.txt   BC of g2k.txt + g2k.order by Graph::brandesBCIndexGPU_5 of QBC.cu
  ref_g2k_rq.txt    BC of the g2k.query vertices by brandesBCIndexGPU_PointBatch of RQ.cu
  ref_la_mhl.npz    BC of the LosAngeles graph by MHLQBC.cu (when --la is given)
  ref_g50k_mhl.npz  BC of the seeded 50k grid (the benchmark's graph, gpu_betweennesscentrality_b200.synth
                    grid_graph(50000, seed=1)) by MHLQBC.cu (when --g50k is given)
  ref_timings.json  times of those runs: the CPU index build alone, the whole driver call, and the
                    reference kernels' own time (kernel_ms, CUDA events around each launch of the
                    oracle/_ref/ref_mhlqbc_timed build)
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


def mhl(graph_path, out_path):
    """MHL-QBC driver, kernel-timed build when present"""
    timed = os.path.exists(os.path.join(REF, "ref_mhlqbc_timed"))
    return run("ref_mhlqbc_timed" if timed else "ref_mhlqbc", [graph_path], out_path)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--la", default=None)
    ap.add_argument("--g50k", action="store_true")
    a = ap.parse_args()
    if a.la:
        a.la = os.path.abspath(a.la)
    g = os.path.join(HERE, "g2k.txt")
    timings = {}
    timings["g2k_mhl"] = mhl(g, os.path.join(HERE, "ref_g2k_mhl.txt"))
    timings["g2k_qbc"] = run("ref_qbc", [g, os.path.join(HERE, "g2k.order")], os.path.join(HERE, "ref_g2k_qbc.txt"))
    timings["g2k_rq"] = run("ref_rq", [g, os.path.join(HERE, "g2k.query")], os.path.join(HERE, "ref_g2k_rq.txt"))
    if a.la:
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "la.txt")
            timings["la_mhl"] = mhl(a.la, p)
            bc = np.loadtxt(p)[:, 1]
        np.savez_compressed(os.path.join(HERE, "ref_la_mhl.npz"), bc=bc)
    if a.g50k:
        sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
        from gpu_betweennesscentrality_b200 import synth

        with tempfile.TemporaryDirectory() as td:
            gp, p = os.path.join(td, "g50k.txt"), os.path.join(td, "out.txt")
            synth.write_graph(gp, synth.grid_graph(50000, seed=1))
            timings["g50k_mhl"] = mhl(gp, p)
            bc = np.loadtxt(p)[:, 1]
        np.savez_compressed(os.path.join(HERE, "ref_g50k_mhl.npz"), bc=bc)
    with open(os.path.join(HERE, "ref_timings.json"), "w") as f:
        json.dump(timings, f, indent=1)
    print(json.dumps(timings))


if __name__ == "__main__":
    main()
