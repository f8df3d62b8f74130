"""Regenerates the golden fixtures of tests/golden/ from the reference tree.

Run where the reference tree is present (it is not on GPU machines), with
the reference's root directory as the one argument:
    python tests/golden/make_fixtures.py <reference-root>
Writes:
  * Lobatto40.txt, Lobatto10.txt -- the reference's velocity-quadrature files
    (tc/tc1/Lobatto40.txt, tc/tc4/Lobatto10.txt), copied verbatim;
  * tc1_reentry.plt.gz, tc3_nanotubesphere.plt.gz -- the tc1 and tc3 meshes
    (tc/tc1/reentry.plt, tc/tc3/NanoTubeSphere.plt), gzip-compressed;
  * kat.json -- the reference's known answers: SUMWEIGHT printed by the tc1
    run (tc/tc1/output:24) and the mesh / velocity-space counts of its
    FILE.OUT (tc/tc1/FILE.OUT:5,8), plus the tc1 and tc3 namelists' physical
    inputs (tc/tc1/reentry_test.con, tc/tc3/Nanoparticle.con).
"""
import gzip
import json
import os
import re
import shutil
import sys


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    shutil.copyfile(os.path.join(ref, "tc/tc1/Lobatto40.txt"), os.path.join(here, "Lobatto40.txt"))
    shutil.copyfile(os.path.join(ref, "tc/tc4/Lobatto10.txt"), os.path.join(here, "Lobatto10.txt"))
    for src, dst in (("tc/tc1/reentry.plt", "tc1_reentry.plt.gz"), ("tc/tc3/NanoTubeSphere.plt", "tc3_nanotubesphere.plt.gz")):
        with open(os.path.join(ref, src), "rb") as fi, gzip.GzipFile(os.path.join(here, dst), "wb", 9, mtime=0) as fo:
            shutil.copyfileobj(fi, fo)
    out = open(os.path.join(ref, "tc/tc1/output")).read()
    sw = re.search(r"SUMWEIGHT=\s*([0-9.Ee+-]+)", out).group(1)
    fo = open(os.path.join(ref, "tc/tc1/FILE.OUT")).read().split("\n")
    counts = [int(x) for x in fo[4].split()]
    vcounts = [int(x) for x in fo[7].split()]
    times = [float(x) for x in re.findall(r"Iteration time:\s*([0-9.]+)", out)]

    def nml(path):
        d = {}
        for line in open(os.path.join(ref, path)):
            line = line.split("!")[0]
            m = re.match(r"\s*IVD%(\w+(?:\(\d\))?)\s*=\s*([^,]+)", line)
            if m:
                d[m.group(1)] = m.group(2).strip().strip('"')
        return d

    kat = {"sumweight_lobatto40_torder40_fp32": sw, "tc1_nelem_npoin_nboun": counts,
           "tc1_rorder_torder_vnpnt": vcounts, "tc1_iteration_times_s": {"n": len(times), "mean": sum(times) / len(times),
                                                                       "min": min(times), "max": max(times)},
           "tc1_namelist": nml("tc/tc1/reentry_test.con"), "tc3_namelist": nml("tc/tc3/Nanoparticle.con")}
    with open(os.path.join(here, "kat.json"), "w") as fh:
        json.dump(kat, fh, indent=1, sort_keys=True)
    print(json.dumps(kat, indent=1)[:600])


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference-root>")
    main(sys.argv[1])
