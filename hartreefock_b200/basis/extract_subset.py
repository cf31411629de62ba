"""Maintainer helper: copy the H/He/C/N/O/F blocks of the Pople basis sets the
engine's workloads use (STO-3G, 6-31G, 6-31G*, 6-31+G**) out of the NWChem-format
data files that ship with aromanro/HartreeFock (Basis Set Exchange exports),
unchanged, into this directory.  Run once where that tree is available:

    python extract_subset.py /path/to/HartreeFock
"""
import os
import re
import sys

FILES = {"sto3g.txt": "sto-3g.nw", "6-31g.1.nw": "6-31g.nw", "6-31g_st_.1.nw": "6-31g_st.nw",
         "6-31+g_st__st_.1.nw": "6-31+g_st_st.nw"}
KEEP = {"H", "He", "C", "N", "O", "F"}


def main(src_dir):
    here = os.path.dirname(os.path.abspath(__file__))
    shell = re.compile(r"^(\w+)\s+(\w+)\s*$")
    for src, dst in FILES.items():
        out, keep = ["# subset (H, He, C, N, O, F) of " + src + " from the Basis Set Exchange data",
                     'BASIS "ao basis" PRINT'], False
        for line in open(os.path.join(src_dir, src)):
            line = line.rstrip("\r\n")
            m = shell.match(line)
            if m:
                keep = m.group(1) in KEEP
            elif line.strip().startswith(("BASIS", "END")) or line.strip().startswith("#"):
                continue
            if keep and line.strip():
                out.append(line)
        out.append("END")
        with open(os.path.join(here, dst), "w") as fh:
            fh.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main(sys.argv[1])
