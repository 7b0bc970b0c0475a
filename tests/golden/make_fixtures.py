"""Build the committed n26 fixtures from the reference's sample run directory.

The reference (fabioaffinito/2degas) ships one sample working directory,
n26/ (N=26, 13 up + 13 down, r_s=1), with its input files, spline tables and
the outputs of one VMC block: n26.res (block sums, final RNG state, twist)
and n26.{up,down}.x.res.0 (the final configuration of rank 0). The
10,000-configuration start files n26.{up,down}.x.0 are inside n26.tar.gz.
te.vrk is the setup program's intermediate Ewald-breakup file for the same
deck.

This script copies the text inputs and golden outputs verbatim and keeps
only the first NCONF start configurations, so the fixtures stay small. It is
run once, where the reference tree is available:

    python tests/golden/make_fixtures.py /path/to/reference
"""
import os
import shutil
import sys
import tarfile

NCONF = 64
NPER = 13  # electrons per spin in n26

COPY = [
    "n26.sy", "n26.sy_vmc", "n26.in", "n26.u2", "n26.u3", "n26.b", "n26.v", "n26.k",
    "seed", "runid", "n26.res", "n26.up.x.res.0", "n26.down.x.res.0",
    "n26.up.x.res.1", "n26.down.x.res.1", "n26.rhok_up", "n26.rhok_down",
    # the setup program's Ewald breakup for this deck (fitpn's table, from
    # which traduci wrote n26.v)
    "te.vrk",
]


def main(ref):
    src = os.path.join(ref, "n26")
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "n26")
    os.makedirs(dst, exist_ok=True)
    for name in COPY:
        shutil.copyfile(os.path.join(src, name), os.path.join(dst, name))
    with tarfile.open(os.path.join(src, "n26.tar.gz")) as tf:
        for spin in ("up", "down"):
            member = tf.getmember(f"n26.{spin}.x.0")
            lines = tf.extractfile(member).read().decode().splitlines()
            with open(os.path.join(dst, f"n26.{spin}.x.0"), "w") as out:
                out.write("\n".join(lines[: NCONF * NPER]) + "\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <reference tree>")
    main(sys.argv[1])
