"""Extract the 2-D lines of the reference's variation probe report for the
variations this build implements, with each one's probe-batch slot.

Source: docs/generated/variation-probe.txt of calibas/fflame-rust (the
reference's own committed golden report: class glyphs per output component
at the 27 inputs of src/probe/inputs.rs, and the FNV-1a digest of the
quantised outputs, src/probe/classify.rs).

The probe seeds each variation's RNG from its transform's index in its
probe batch (main_template.wgsl:1467-1500), so the slot is written beside
the glyphs.  It follows src/probe/batch.rs:94-139: every shipped variation
in registration order (ALL_VARIATIONS, src/variations/defs/mod.rs:446),
first-fit into batches of at most 99 variations and 1600 packed parameter
slots (user parameters + init_param_count, definition.rs:452-454).  A
parameter list given as another definition's (`X.parameters`) counts as
that one's.

Run where the reference tree is mounted; the output,
tests/golden/variation_probe_2d.txt, is committed.

    python tests/golden/make_probe_golden.py /path/to/reference
"""

import glob
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))

from oracle.oracle import REGISTRY  # noqa: E402  (names of this build's variations)

NAMES = sorted(REGISTRY, key=REGISTRY.get)
MAX_PER_FLAME, MAX_SLOTS = 99, 1600


def probe_slots(ref):
    defs = os.path.join(ref, "src", "variations", "defs")
    mod = open(os.path.join(defs, "mod.rs"), encoding="utf-8").read()
    i = mod.index("pub static ALL_VARIATIONS")
    order = re.findall(r"&(\w+),", mod[i:mod.index("];", i)])
    info, nparams, alias = {}, {}, {}
    for p in glob.glob(os.path.join(defs, "*.rs")):
        src = open(p, encoding="utf-8").read()
        for m in re.finditer(r"pub static (\w+): VariationDef = VariationDef \{(.*?)\n\};", src, re.S):
            body = m.group(2)
            name = re.search(r'name: "([^"]+)"', body).group(1)
            plist = re.search(r"parameters: &\[(.*?)\n    \],", body, re.S)
            nparams[m.group(1)] = len(re.findall(r"ParamDef::new\(|param!\(", plist.group(1))) if plist else 0
            other = re.search(r"parameters: (\w+)\.parameters,", body)
            if other:
                alias[m.group(1)] = other.group(1)
            ic = re.search(r"init_param_count: (\d+)", body)
            info[m.group(1)] = (name, int(ic.group(1)) if ic else 0)
    for st, (name, ic) in list(info.items()):
        info[st] = (name, nparams[alias.get(st, st)] + ic)
    slot, count, used = {}, 0, 0
    for st in order:
        name, s = info[st]
        if count > 0 and (count + 1 > MAX_PER_FLAME or used + s > MAX_SLOTS):
            count, used = 0, 0
        slot[name] = count
        count += 1
        used += s
    return slot


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
    slots = probe_slots(ref)
    out = os.path.join(HERE, "variation_probe_2d.txt")
    with open(out, "w", encoding="utf-8") as f:
        f.write("# 2-D lines of the reference's docs/generated/variation-probe.txt\n")
        f.write("# (generated by tests/golden/make_probe_golden.py; name classes digest probe-batch-slot)\n")
        for h in header:
            f.write(h + "\n")
        for n in NAMES:
            c, d = lines[n]
            f.write(f"{n} {c} {d} {slots[n]}\n")
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_probe_golden.py <reference checkout>")
    main(sys.argv[1])
