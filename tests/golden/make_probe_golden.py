"""Extract the 2-D lines of the reference's variation probe report for the
variations this build implements.

Source: docs/generated/variation-probe.txt of calibas/fflame-rust (the
reference's own committed golden report: class glyphs per output component
at the 27 inputs of src/probe/inputs.rs, and the FNV-1a digest of the
quantised outputs, src/probe/classify.rs).  Run where the reference tree is
mounted; the output, tests/golden/variation_probe_2d.txt, is committed.

    python tests/golden/make_probe_golden.py /path/to/reference
"""

import os
import sys

NAMES = ["linear", "sinusoidal", "spherical", "swirl", "horseshoe", "polar", "disc",
         "ex", "julia", "bubble", "cylinder", "curl"]


def main(ref):
    src = os.path.join(ref, "docs", "generated", "variation-probe.txt")
    header, lines = [], {}
    with open(src, encoding="utf-8") as f:
        for line in f:
            if line.startswith("# adapter") or line.startswith("# backend") or line.startswith("# driver") \
                    or line.startswith("# inputs") or line.startswith("# build"):
                header.append(line.rstrip("\n"))
            parts = line.split()
            if len(parts) == 4 and parts[1] == "2d" and parts[0] in NAMES:
                lines[parts[0]] = (parts[2], parts[3])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "variation_probe_2d.txt")
    with open(out, "w", encoding="utf-8") as f:
        f.write("# 2-D lines of the reference's docs/generated/variation-probe.txt\n")
        f.write("# (generated by tests/golden/make_probe_golden.py; name classes digest)\n")
        for h in header:
            f.write(h + "\n")
        for n in NAMES:
            c, d = lines[n]
            f.write(f"{n} {c} {d}\n")
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
