"""Variants of the n26 input deck written to a temporary run directory.

Each variant keeps the reference's own tables (n26.u2/.u3/.b/.v/.k) and
changes only which keyword records are present, so the walker path is
exercised with and without backflow, three-body Jastrow, twist and
k-space potential. The fixture files are copied next to the new .sy so the
records keep the bare file names of the original deck (80-column records).
"""
import os
import shutil

from conftest import N26


def write_variant(tmpdir, runid, u2=True, u3=True, backflow=True, v2=True, rhok=True,
                  ntwists=4, extra=()):
    tmpdir = str(tmpdir)
    for f in os.listdir(N26):
        dst = os.path.join(tmpdir, f)
        if not os.path.exists(dst):
            shutil.copyfile(os.path.join(N26, f), dst)
    lines = ["  ndim 2", "  type up 13 1. n26.up.x", "  type down 13 1. n26.down.x"]
    pairs = (("up", "up"), ("down", "down"), ("up", "down"))
    if u2:
        lines += [f"  u2 {a} {b} n26.u2" for a, b in pairs]
    if u3:
        lines += [f"  u3 {a} {b} n26.u3" for a, b in pairs]
    if rhok:
        lines += ["  rhok up", "  rhok down"]
    lines += ["  pbc 9.03777677 9.03777677", "  kspace n26.k"]
    if backflow:
        lines += [f"  backflow {a} {b} 1 n26.b" for a, b in (("up", "up"), ("up", "down"),
                                                            ("down", "down"))]
    if ntwists:
        lines.append(f"  ntwists {ntwists}")
    if v2:
        lines += [f"  v2 {a} {b} n26.v 0. 1 1." for a, b in pairs]
        lines.append("  v0 -69.0949679")
    lines += list(extra)
    lines.append("  end")
    with open(os.path.join(tmpdir, runid + ".sy"), "w") as f:
        f.write("\n".join(lines) + "\n")
    return tmpdir
