"""Copies the reference's own ParaTC input files into tests/golden/ as format
fixtures of the namelist reader (paratc_params_from_namelist and friends).

The reference ships no tests; these input decks are the only files it holds
whose parse is known: the values a Fortran NAMELIST read gives are the ones
written in them.  Run from the repository root with the reference checked
out at REF (default /root/reference); it writes the files below and
reference_inputs.sha256 (their SHA-256 digests).  The copies are verbatim.
"""
import hashlib
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
FILES = {
    "Input/TurbCha0180_4th.standard": "TurbCha0180_4th.standard",
    "Input/GravityFlow/GravityFlow.prm": "GravityFlow.prm",
    "Input/GravityFlow/GravityFlow.small": "GravityFlow.small",
    "Input/StratifiedFlow/SF_Ri000.prm": "SF_Ri000.prm",
    "Input/StratifiedFlow/SF_Ri018.prm": "SF_Ri018.prm",
    "Input/StratifiedFlow/SF_Ri120.prm": "SF_Ri120.prm",
    "Input/StratifiedFlow/SF_Ri480.prm": "SF_Ri480.prm",
}


def main():
    lines = []
    for src, dst in FILES.items():
        out = os.path.join(HERE, dst)
        shutil.copyfile(os.path.join(REF, src), out)
        digest = hashlib.sha256(open(out, "rb").read()).hexdigest()
        lines.append("%s  %s  (reference %s)" % (digest, dst, src))
    with open(os.path.join(HERE, "reference_inputs.sha256"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print("\n".join(lines))


if __name__ == "__main__":
    main()
