"""Generates the validation fixtures of tests/golden from the reference checkout (run once, where a
checkout exists):  python tests/golden/make_validation_fixtures.py <path of the reference checkout>

  validation_numbers.json  printed results of validation/reference_full.txt and reference_quick.txt
                           for the hot-path sections (1 linear wake, 2 blowout, 3 betatron, 4 gain,
                           6 displaced analytic driver in mode 1 (linear regime), 7 centroid betatron
                           oscillation with azimuthal mode 1, 13 adaptive sub-slicing)
  decks/*.in               the validation decks those numbers come from (blowout, gain, betatron, linear, and
                           the paper case conv_s1 of section 13)
"""
import json
import os
import re
import shutil
import sys

if len(sys.argv) != 2:
    sys.exit("usage: make_validation_fixtures.py <path of the reference checkout>")
ref = sys.argv[1]
here = os.path.dirname(os.path.abspath(__file__))
out = {}
for tag, fn in (("full", "reference_full.txt"), ("quick", "reference_quick.txt")):
    prev = ""
    for line in open(os.path.join(ref, "validation", fn)):
        if "linear regime (d = 0.01)" in prev and "L2 rel. errors:" in line:
            errs, _, sin = line.split("L2 rel. errors:")[1].partition("|")
            vals = dict(tok.strip().split() for tok in errs.split(","))
            vals["sin_max"] = sin.split(":")[1].strip()
            out["m1_shift_linear_" + tag] = vals
        prev = line
        m = re.match(r"(uniform_dr0\.01_dxi0\.01|stretched_dxi0\.005|stretched_dxi0\.005_PCR)\s+Ez\(-5\)=(\S+) "
                     r"Ez\(-7\)=(\S+) Ez\(-8\)=(\S+) Ezmin=(\S+) @xi=(\S+)\s+Wr/r\(r=\.5,xi=-6\)=(\S+)", line)
        if m:
            out["blowout_" + m.group(1)] = dict(zip(["Ez(-5)", "Ez(-7)", "Ez(-8)", "Ezmin", "xi_min", "Wr/r"],
                                                    m.groups()[1:]))
        m = re.match(r"max \|r_rms - r0 \|cos\(w_b t\)\|\| / r0 = (\S+)", line)
        if m:
            out["betatron_" + tag] = m.group(1)
        m = re.match(r"max \|x_c - x0 cos\(w_b t\)\|/x0 = (\S+),\s+max \|y_c\|/x0 = (\S+)", line)
        if m:
            out["m1_centroid_" + tag] = {"x": m.group(1), "y": m.group(2)}
        m = re.match(r"\s*(out_ss_plain|out_ss_sub)\s+extra sub-slices\s+(\d+) \| behind the spike: Ez (\S+) psi (\S+) \| "
                     r"witness: Ez (\S+) psi (\S+) \| spike integral (\S+)", line)
        if m:
            out["subslice_" + m.group(1)[7:] + "_" + tag] = dict(
                zip(["extra", "behind Ez", "behind psi", "witness Ez", "witness psi", "spike"], m.groups()[1:]))
        m = re.match(r"\s*reference out_ss_ref: integral of Ez over the closure spike \(xi -9\.2\.\.-8\.9\) = (\S+)", line)
        if m:
            out["subslice_ref_" + tag] = {"spike": m.group(1)}
        m = re.match(r"d<gamma>/dt = (\S+)", line)
        if m:
            out["gain_" + tag] = m.group(1)
        m = re.match(r"(uniform dr=0\.01|stretched 0\.002 -> 0\.05)\s*: max\|Ez\|=(\S+)\s+rel\.err Ez\(r=0\)=(\S+)\s+"
                     r"psi\(0\)=(\S+)\s+\(Er-Bth\)\(r=0\.5\)=(\S+)", line)
        if m:
            out["linear_" + m.group(1).split()[0] + "_" + tag] = dict(
                zip(["max|Ez|", "rel.err Ez(r=0)", "psi(0)", "(Er-Bth)(r=0.5)"], m.groups()[1:]))
with open(os.path.join(here, "validation_numbers.json"), "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
os.makedirs(os.path.join(here, "decks"), exist_ok=True)
for d in ("blowout.in", "gain.in", "betatron.in", "linear.in"):
    shutil.copy(os.path.join(ref, "validation", d), os.path.join(here, "decks", d))
shutil.copy(os.path.join(ref, "paper", "inputs", "conv_s1.in"), os.path.join(here, "decks", "conv_s1.in"))
print(json.dumps(out, indent=1, sort_keys=True))
