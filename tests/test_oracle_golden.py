"""The oracle against the reference's own fixtures (CPU).

* docs/generated/variation-probe.txt (tests/golden/variation_probe_2d.txt):
  per variation, the class glyph of each output component at the 27 inputs
  of src/probe/inputs.rs, and the FNV-1a digest of the quantised outputs.
* the pixel-mapping known answers of src/renderer/compute_kernel.rs:6404-6511.
* the firefly downsample of src/export/supersample.rs:132-167.

The reference GPU evaluated sin/cos with the hardware's approximate
functions: at arguments that are multiples of f32(pi)/2 they return
exactly 0 (IEEE gives +-4e-8), and outside about 1e-6 <= |x| <= 1e6 they
return 0.  The oracle calls IEEE-accurate libm, so at those inputs the
class can differ; each such input is listed below with the condition it
must meet, and every other input must match exactly.

The report's draws: the build that wrote it drew from the same PCG as
rng.wgsl but with one increment for every thread (pcg_hash's constant,
2891336453); the current rng.wgsl gives each thread its own.  A
variation's first draw is the same under both; its later draws are not,
so the report is compared with the oracle drawing from the report's
stream (gaussian_blur and pre_blur then match it bit for bit, and no
reordering of the current stream does).
"""

import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
LABELS = ("+0+0 +0-0 -0+0 -0-0 +x -x +y -y q1 q2 q3 q4 mid odd big pi_e unit half_unit tiny normal_min "
          "subnormal large near_threshold past_threshold lopsided y_neg0x neg0y_x").split()

# (variation) -> {input label: why the class may differ}
SFU_SIN = {
    "sinusoidal": {"pi_e": "sin(pi)", "tiny": "tiny", "normal_min": "tiny", "large": "huge",
                   "near_threshold": "huge", "past_threshold": "huge", "lopsided": "huge"},
    "cylinder": {"pi_e": "sin(pi)", "tiny": "tiny", "normal_min": "tiny", "large": "huge",
                 "near_threshold": "huge", "past_threshold": "huge", "lopsided": "huge"},
    "disc": {"+x": "sin(pi)", "-x": "sin(pi)", "-y": "sin(pi)", "unit": "sin(pi)", "y_neg0x": "sin(pi)"},
    "julia": {"-x": "cos(pi/2)", "unit": "sin(pi)", "y_neg0x": "sin(pi)", "lopsided": "inf*sin(pi)"},
    "ex": {"q1": "cancel", "q3": "cancel", "q4": "cancel", "half_unit": "cancel"},
}

# The wider registry.  "zero": ours within a few ulp of 0 where the
# reference's approximate sin/cos/tan gave 0 or a tiny value of either
# sign; "huge": an argument beyond 1e6, where the reference's sin/cos/tan
# return 0; "inf*0": ours +-inf where the reference multiplied its exact 0
# by inf; "pow": the reference evaluates pow(x, y) as exp2(y log2 x), NaN
# at y = 0, x = inf; "branch": a comparison met at equality (ngon's phi
# against pi/sides at the -x input); "signed-zero": the reference's
# compiler folded `0 + 1 * x` to x for the carrier of a Post variation, or
# its sinh ((e^x - e^-x) / 2) gave +0 for -0; "tiny-quotient": the
# reference's sin and sinh return exactly 0 at the 1e-20 input (an absolute
# error bound) where ours return the argument, so a quotient whose zero
# denominator the body replaces by 1e-20 is finite here and 0 there;
# "shared-square": the reference's compiler reused p.x * p.x, infinite at
# these inputs, for `twist * p.x * p.x` (mcarpet; q_ode's `q03 * p.x * p.x`
# and its like), so 0 * inf gave NaN where the
# source order (twist * p.x) * p.x gives a finite value here;
# "zero-divisor": the reference's tan at f32(pi) returned exactly 0, which
# the body replaced by a 1e-30 divisor (infinite there, finite here);
# "reassociated": the reference's compiler grouped `x * x * y * y` as
# (x * x) * (y * y), inf * 0 = NaN, which its max() then replaced, where
# the source order gives inf and a NaN further on;
# "fused": the reference's compiler contracted `x * x - y * y` into one
# fused multiply-add, fma(x, x, -(y * y)) = -inf where x * x and y * y
# both overflow, where the source order's inf - inf is NaN (plusrecip's
# square root of z^2 - a then stays finite here and is infinite there);
# "scaled-zero": the reference's cos(f32(pi) / 2) is exactly 0 where ours
# is -4.4e-8, and the body multiplies it by a large finite factor
# (onion2's p / max(|p|, 1e-30) at the 1e-20 input, whose squares flush to
# zero), finite here and 0 there;
# "tiny-branch": the reference's sin returns exactly 0 at the 1e-20 input,
# which skips a branch the body takes for a nonzero sine (the Jacobi
# functions' back substitution under |sn| > 1e-30); ours takes it, and
# its cos / sin of 1e20 overflows the recurrence to NaN.
HUGE_ARGS = ["large", "near_threshold", "past_threshold", "lopsided"]
# Where the bipolar series' sigma is f32(pi) (sin(sigma) -4.4e-8 here, 0 on
# the reference) and the elliptic series' nu is f32(pi)/2 (cos(nu) -4.4e-8).
BIPOLAR_PI = ["+0+0", "+0-0", "-0+0", "-0-0", "+x", "-x", "unit", "tiny", "normal_min", "subnormal", "y_neg0x"]
# The inputs whose signed zeros a Pre or Post variation's linear carrier
# keeps on the reference (its compiler folded 0 + 1 * p into p).
CARRIER_ZEROS = ["+0-0", "-0+0", "-0-0", "subnormal", "y_neg0x", "neg0y_x"]
# The wf curves' angle atan2(x, y) at multiples of f32(pi)/2.
WF_CURVE = ["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "lopsided", "y_neg0x"]
ELLIPTIC_PI2 = ["+0+0", "+0-0", "-0+0", "-0-0", "+y", "-y", "tiny", "normal_min", "subnormal", "neg0y_x"]
WIDER = {
    "heart": dict.fromkeys(["+x", "-x", "-y", "unit", "y_neg0x"], "zero"),
    "diamond": dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "y_neg0x"], "zero"),
    "flatten": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "julian": {"-x": "zero", "y_neg0x": "zero", "lopsided": "inf*0"},
    "blob": {**dict.fromkeys(["+x", "-x", "-y", "unit", "y_neg0x"], "zero"), "lopsided": "inf*0"},
    "fan2": {**dict.fromkeys(["+x", "+y", "-y", "unit", "y_neg0x", "neg0y_x"], "zero"), "lopsided": "inf*0"},
    "ngon": {"-x": "branch"},
    "wedge": {"-x": "zero"},
    "juliascope": {"+x": "zero", "-x": "zero", "lopsided": "inf*0"},
    "radial_blur": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "tangent": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"),
                **dict.fromkeys(["large", "near_threshold", "past_threshold", "lopsided"], "huge")},
    "cosine": {**dict.fromkeys(["q1", "q2", "q3", "q4", "mid", "big"], "zero"),
               **dict.fromkeys(["large", "near_threshold", "past_threshold", "lopsided"], "huge")},
    "popcorn": {"tiny": "zero", "lopsided": "huge"},
    "split": dict.fromkeys(["large", "near_threshold", "past_threshold"], "huge"),
    "power": dict.fromkeys(["large", "near_threshold", "past_threshold", "lopsided"], "pow"),
    "exponential": {**dict.fromkeys(["+y", "-y", "q1", "q2", "q3", "q4", "big", "tiny", "normal_min", "neg0y_x"], "zero"),
                    **dict.fromkeys(["large", "near_threshold", "past_threshold", "lopsided"], "huge")},
    "foci": dict.fromkeys(["tiny", "normal_min"], "zero"),
    "waves2": {"tiny": "zero"},
    "escher": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "auger": dict.fromkeys(["near_threshold", "lopsided"], "huge"),
    "sin": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "cos": {"pi_e": "zero", **dict.fromkeys(HUGE_ARGS, "huge")},
    "tan": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), "lopsided": "huge"},
    "sec": {"pi_e": "zero", "lopsided": "huge"},
    "csc": {"pi_e": "zero", "tiny": "tiny-quotient", "normal_min": "zero", "lopsided": "huge"},
    "cot": {"pi_e": "zero", "tiny": "tiny-quotient", "normal_min": "zero", "lopsided": "huge"},
    "sinh": {**dict.fromkeys(["-0+0", "-0-0", "neg0y_x"], "signed-zero"), "tiny": "zero", **dict.fromkeys(HUGE_ARGS, "huge")},
    "cosh": dict.fromkeys(HUGE_ARGS, "huge"),
    "tanh": {"tiny": "zero"},
    "coth": {"tiny": "tiny-quotient", "normal_min": "zero"},
    "sech": {"tiny": "tiny-quotient"},
    "csch": {"tiny": "tiny-quotient", "normal_min": "zero"},
    "exp": {**dict.fromkeys(["tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "popcorn2": {"tiny": "zero"},
    "modulus": dict.fromkeys(["past_threshold", "lopsided"], "huge"),
    "whorl": {"lopsided": "inf*0"},
    "flux": dict.fromkeys(["+0+0", "+0-0", "-0+0", "-0-0", "-x", "tiny", "normal_min", "subnormal"], "zero"),
    "rays": dict.fromkeys(["tiny", "normal_min"], "zero"),
    "flower": dict.fromkeys(["+x", "-x", "unit", "y_neg0x"], "zero"),
    "disc2": {"lopsided": "huge"},
    "wedge_julia": {"-y": "zero"},
    "epispiral": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "neg0y_x"], "zero"),
    "cardioid": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "neg0y_x"], "zero"),
    "petal": {"pi_e": "zero", **dict.fromkeys(HUGE_ARGS, "huge")},
    "unpolar": {"pi_e": "zero", "tiny": "zero", "lopsided": "huge"},
    "idisc": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "half_unit", "tiny", "normal_min", "neg0y_x"], "zero"),
    "exp2": {**dict.fromkeys(["+y", "-y", "q1", "q2", "q3", "q4", "tiny", "normal_min", "neg0y_x"], "zero"), "big": "huge",
             **dict.fromkeys(HUGE_ARGS, "huge")},
    "invpolar": {**dict.fromkeys(["+x", "-x", "q1", "q2", "mid", "unit", "tiny", "normal_min", "y_neg0x"], "zero"),
                 "big": "huge", **dict.fromkeys(HUGE_ARGS, "huge")},
    "swirl3": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "wdisc": dict.fromkeys(["-0-0", "-x", "+y", "-y", "half_unit", "tiny", "neg0y_x"], "zero"),
    "sin2_bs": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "cos2_bs": {"pi_e": "zero", **dict.fromkeys(HUGE_ARGS, "huge")},
    "sinh2_bs": {**dict.fromkeys(["tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "cosh2_bs": dict.fromkeys(HUGE_ARGS, "huge"),
    "exp2_bs": {**dict.fromkeys(["tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "layered_spiral": {"tiny": "zero"},
    "circlesplit": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "mcarpet": dict.fromkeys(HUGE_ARGS, "shared-square"),
    "clifford_js": dict.fromkeys(HUGE_ARGS, "huge"),
    "anamorphcyl": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "tan2_bs": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), "lopsided": "huge"},
    "tanh2_bs": dict.fromkeys(["tiny", "normal_min"], "zero"),
    "cot2_bs": {"pi_e": "zero", **dict.fromkeys(["tiny", "normal_min"], "tiny-quotient"), "lopsided": "huge"},
    "coth2_bs": dict.fromkeys(["tiny", "normal_min"], "tiny-quotient"),
    "csc2_bs": {"pi_e": "zero", **dict.fromkeys(["tiny", "normal_min"], "tiny-quotient"), "lopsided": "huge"},
    "csch2_bs": dict.fromkeys(["tiny", "normal_min"], "tiny-quotient"),
    "sec2_bs": {"pi_e": "zero", "lopsided": "huge"},
    "deltaA": dict.fromkeys(["+0+0", "+0-0", "-0+0", "-0-0", "-x", "tiny", "normal_min", "subnormal"], "zero"),
    "epispiral_wf": dict.fromkeys(WF_CURVE, "zero"),
    "hyperbolicellipse": {**dict.fromkeys(["-0+0", "-0-0", "neg0y_x"], "signed-zero"),
                          **dict.fromkeys(["tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    # A Pre variation feeds the probe's linear carrier; the reference's
    # compiler folded that carrier's 0 + 1 * p to p, keeping its -0.
    "pre_disc": {**dict.fromkeys(["-0+0", "-0-0", "+y", "neg0y_x"], "signed-zero"),
                 **dict.fromkeys(["+x", "-x", "-y", "unit", "y_neg0x"], "zero")},
    "pre_sinusoidal": {**dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
                       **dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "pre_spherical": dict.fromkeys(["+0-0", "-0+0", "-0-0", "subnormal", "large", "near_threshold", "past_threshold",
                                    "y_neg0x", "neg0y_x"], "signed-zero"),
    "sintrange": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), "lopsided": "inf*0"},
    "squirrel": dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"),
    "svensson_js": {**dict.fromkeys(["tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "post_curl": {"-0-0": "signed-zero"},
    "sinq": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"),
        **dict.fromkeys(["large", "past_threshold"], "inf*0"),
        **dict.fromkeys(["near_threshold", "lopsided"], "huge")},
    "cosq": {"pi_e": "zero", **dict.fromkeys(["large", "past_threshold"], "inf*0"),
        **dict.fromkeys(["near_threshold", "lopsided"], "huge")},
    "tanq": {**dict.fromkeys(["pi_e", "normal_min"], "zero"), "tiny": "tiny-quotient"},
    "cotq": {**dict.fromkeys(["pi_e", "normal_min"], "zero"), "tiny": "tiny-quotient"},
    "secq": dict.fromkeys(["pi_e", "tiny"], "zero"),
    "cscq": {**dict.fromkeys(["pi_e", "normal_min"], "zero"), "tiny": "tiny-quotient"},
    "sinhq": {**dict.fromkeys(["tiny", "normal_min"], "zero"),
        **dict.fromkeys(["large", "past_threshold", "lopsided"], "inf*0"), "near_threshold": "huge"},
    "coshq": {**dict.fromkeys(["large", "past_threshold", "lopsided"], "inf*0"), "near_threshold": "huge"},
    "tanhq": {"tiny": "tiny-quotient", "normal_min": "zero"},
    "cothq": {"tiny": "tiny-quotient", "normal_min": "zero"},
    "sechq": {"tiny": "zero"},
    "cschq": {"tiny": "tiny-quotient", "normal_min": "zero"},
    "bCollide": dict.fromkeys(BIPOLAR_PI, "zero"),
    "bMod": dict.fromkeys(BIPOLAR_PI, "zero"),
    "bSwirl": dict.fromkeys(BIPOLAR_PI, "zero"),
    "eCollide": {**dict.fromkeys(ELLIPTIC_PI2, "zero"),
        **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "eMod": {**dict.fromkeys(ELLIPTIC_PI2, "zero"),
        **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "eScale": {**dict.fromkeys(ELLIPTIC_PI2, "zero"),
        **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "ePush": {**dict.fromkeys(ELLIPTIC_PI2, "zero"),
        **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "eRotate": {**dict.fromkeys(ELLIPTIC_PI2, "zero"),
        **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "hole2": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "neg0y_x"], "zero"),
    "pTransform": {**dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "y_neg0x"], "zero"),
        "lopsided": "inf*0"},
    # ortho: the reference's cos(pi/2) = 0 meets x >= 0 at equality (+y, -y),
    # and a / (2 theta) rounds to 1 on one side, just below it on the other
    # (half_unit).
    "ortho": {"-x": "zero", **dict.fromkeys(["+y", "-y", "neg0y_x", "half_unit"], "branch")},
    "circlize": dict.fromkeys(["-x", "+y", "-y", "lopsided", "neg0y_x"], "zero"),
    "circlize2": dict.fromkeys(["-x", "+y", "-y", "lopsided", "neg0y_x"], "zero"),
    "fibonacci2": {**dict.fromkeys(["+x", "-x", "unit", "tiny", "normal_min", "y_neg0x"], "zero"),
        **dict.fromkeys(["large", "near_threshold", "past_threshold"], "huge"), "lopsided": "inf*0"},
    "disc3": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "fdisc": dict.fromkeys("+0+0 +0-0 -0+0 -0-0 +x -x +y -y unit half_unit tiny normal_min subnormal y_neg0x "
                           "neg0y_x".split(), "zero"),
    "csc_squared": {"pi_e": "zero-divisor", **dict.fromkeys(HUGE_ARGS, "huge")},
    "atan2_spirals": {"-x": "zero"},
    "eMotion": {**dict.fromkeys(ELLIPTIC_PI2, "zero"), **dict.fromkeys(HUGE_ARGS, "inf*0")},
    "mask": {"pi_e": "zero"},
    "pre_crop": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "post_crop": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "mobiusN": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "sphericalN": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "neg0y_x"], "zero"),
    "murl2": {"-x": "zero"},
    "q_ode": dict.fromkeys(HUGE_ARGS, "shared-square"),
    "heart_wf": {"-y": "zero"},
    "inverted_julia": dict.fromkeys(["+0+0", "+0-0", "-0+0", "-0-0", "-y", "neg0y_x"], "zero"),
    "bTransform": dict.fromkeys(BIPOLAR_PI, "zero"),
    "cannabiscurve_wf": dict.fromkeys("+0+0 +0-0 -0+0 -0-0 +x +y -y unit subnormal lopsided y_neg0x "
                                      "neg0y_x".split(), "zero"),
    "sattractor_js": dict.fromkeys(["q4", "neg0y_x"], "zero"),
    "woggle_js": dict.fromkeys(["+0-0", "-0+0", "subnormal"], "zero"),
    "lace_js": {"-x": "zero", "lopsided": "inf*0"},
    "cloverleaf_wf": dict.fromkeys(WF_CURVE, "zero"),
    "rose_wf": dict.fromkeys(WF_CURVE, "zero"),
    "bwraps": {"lopsided": "zero"},
    "target": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "spligon": dict.fromkeys(["+0-0", "-0-0", "-y", "tiny", "subnormal"], "zero"),
    "circus": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "murl": {"-x": "zero"},
    "shredrad": {**dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "y_neg0x"], "zero"), "lopsided": "inf*0"},
    "xheart": {"normal_min": "zero"},
    "pre_bwraps": {**dict.fromkeys(CARRIER_ZEROS, "signed-zero"), "lopsided": "zero"},
    "post_bwraps": {**dict.fromkeys(CARRIER_ZEROS, "signed-zero"), "lopsided": "zero"},
    "target_sp": {**dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"), "lopsided": "inf*0"},
    "cpow3": dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "y_neg0x"], "zero"),
    "phoenix_julia": dict.fromkeys(["-0+0", "-0-0"], "zero"),
    "pow_block": dict.fromkeys(["+0-0", "-0-0", "-y", "subnormal", "neg0y_x"], "zero"),
    "trade": {"-x": "zero"},
    # checks: i32(round(2e30)) is out of range; the reference's conversion gave the other parity.
    "checks": {"lopsided": "branch"},
    # npolar at parity 0 scales cos(-pi/2) by 0: -0 here (cos -4.4e-8), +0 on the reference (its
    # cos exactly 0); atan2 of the signed zeros then picks the other of +-pi.
    "npolar": dict.fromkeys(["+0+0", "-0+0", "-x", "neg0y_x"], "branch"),
    "eJulia": {"-x": "zero"},
    "ripple": {"lopsided": "reassociated"},
    "bsplit": {**dict.fromkeys(["tiny", "normal_min"], "tiny-quotient"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "pre_rotate_x": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "pre_rotate_y": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "post_rotate_x": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "post_rotate_y": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "pre_zscale": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "pre_ztranslate": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "julia3D": dict.fromkeys(["-x", "unit"], "zero"),
    "post_curl3D": dict.fromkeys(CARRIER_ZEROS, "signed-zero"),
    "tangent3D": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "sinusoidal3d": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "disc3d": dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "tiny",
                             "normal_min", "subnormal", "y_neg0x"], "zero"),
    "waves2_3D": {"tiny": "zero"},
    "blob3D": {**dict.fromkeys(["+x", "-x", "-y", "unit", "y_neg0x"], "zero"), "lopsided": "inf*0"},
    "taurus": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "svf": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "cone": dict.fromkeys(["-0+0", "-0-0", "-x", "y_neg0x"], "zero"),
    "foci_3D": dict.fromkeys(["tiny", "normal_min"], "zero"),
    "estiq": {**dict.fromkeys(["tiny", "normal_min"], "zero"),
        **dict.fromkeys(["large", "past_threshold", "lopsided"], "inf*0"), "near_threshold": "huge"},
    "pre_spin_z": dict.fromkeys(["+x", "-x", "+y", "-y", "unit", "lopsided", "y_neg0x", "neg0y_x"], "zero"),
    "post_spin_z": {**dict.fromkeys(["+0+0", "+0-0", "-0+0", "-0-0", "subnormal"], "signed-zero"),
        **dict.fromkeys(["+x", "-x", "+y", "-y", "unit", "lopsided", "y_neg0x", "neg0y_x"], "zero")},
    "pre_disc3d": dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit",
                                 "tiny", "normal_min", "subnormal", "y_neg0x"], "zero"),
    "pre_sinusoidal3d": {**dict.fromkeys(["pi_e", "tiny", "normal_min"], "zero"), **dict.fromkeys(HUGE_ARGS, "huge")},
    "dinis_surface_wf": {**dict.fromkeys(["pi_e", "tiny", "lopsided"], "zero"),
        **dict.fromkeys(["large", "near_threshold", "past_threshold"], "huge")},
    "popcorn2_3D": {"lopsided": "huge"},
    "ho": {**dict.fromkeys(["tiny", "normal_min"], "zero"), "lopsided": "huge"},
    "flower_db": dict.fromkeys(["-x", "+y", "-y", "q3", "neg0y_x"], "zero"),
    "sphere_nja": {"tiny": "tiny-quotient"},
    "exblur": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "neg0y_x"], "zero"),
    # lazysensen: i32 of an out-of-range floor(c * scale); the reference's conversion gives the other parity.
    "lazysensen": dict.fromkeys(HUGE_ARGS, "branch"),
    "hypercrop": dict.fromkeys(["-x", "-y"], "zero"),
    "post_heat": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "onion2": {"tiny": "scaled-zero", "normal_min": "zero"},
    "waves2_wf": {**dict.fromkeys(["+y", "-y", "neg0y_x"], "zero"), "lopsided": "huge"},
    "waves3_wf": dict.fromkeys(["+y", "-y", "neg0y_x"], "zero"),
    "waves4_wf": dict.fromkeys(["+y", "-y", "neg0y_x"], "zero"),
    "plusrecip": dict.fromkeys(["large", "near_threshold", "past_threshold"], "fused"),
    # gamma: log|Gamma(r)| at r = 1 is 0; ours and the reference's logs round it to a few ulp of either sign.
    "jac_sn": {"tiny": "tiny-branch", **dict.fromkeys(HUGE_ARGS, "huge")},
    "jac_cn": {"tiny": "tiny-branch", **dict.fromkeys(HUGE_ARGS, "huge")},
    "jac_dn": {"tiny": "tiny-branch", **dict.fromkeys(HUGE_ARGS, "huge")},
    "z": dict.fromkeys(["-x", "+y", "-y", "neg0y_x"], "zero"),
    "cpow3_wf": {"half_unit": "zero"},
    # pRose3D: cos(6 th) at multiples of pi / 4 and its reflections; the reference's cos rounds to either sign.
    "pRose3D": dict.fromkeys(["-0+0", "-0-0", "-x", "+y", "-y", "q1", "q2", "q3", "q4", "half_unit", "tiny", "normal_min",
                              "large", "near_threshold", "past_threshold", "neg0y_x"], "zero"),
    "waves2b": dict.fromkeys(["+0+0", "+0-0", "-0+0", "-0-0", "tiny", "normal_min", "subnormal"], "zero"),
    "juliaq": {**dict.fromkeys(["-0+0", "+y", "q4", "tiny", "neg0y_x"], "zero"), "large": "inf*0"},
    "julia3Dq": dict.fromkeys(["+y", "q1", "q2", "half_unit", "tiny"], "zero"),
    "juliac": dict.fromkeys(["-x", "-y", "neg0y_x"], "zero"),
    "cpow2": dict.fromkeys(["+0-0", "-0-0", "+x", "-x", "-y", "unit", "subnormal", "y_neg0x"], "zero"),
    "post_juliaq": {**dict.fromkeys(["-y", "normal_min"], "zero"), "large": "inf*0"},
    "post_julia3Dq": {**dict.fromkeys(["q3", "q4"], "zero"), "normal_min": "signed-zero"},
    "gamma": dict.fromkeys(["+x", "-x", "+y", "-y", "unit", "half_unit", "y_neg0x", "neg0y_x"], "zero"),
    # cut_jigsaw's piece orientation hashes the cell: fract(1e5 sin(27 ix + 57 iy)) takes the sine's last
    # bits 1e5-fold, so the hide branch follows the platform's sine ("large": a cell past 1e6).
    "cut_jigsaw": {"odd": "branch", "large": "huge"},
    # cut_metaballs' jitter: fract(43758.5453 sin(.)) of the neighbouring cells, the same amplification,
    # decides m_dist against its 0.06 step.
    "cut_metaballs": {"+x": "branch"},
    # cut_hextruchetflow's arc orientation: fract(43758.54 sin(37 hx + 39 hz)) of the hex cell, at sine
    # arguments of 72-115 here; every one of these five points takes the reference's side once that
    # orientation is flipped.
    "cut_hextruchetflow": dict.fromkeys(["+0+0", "+x", "tiny", "large", "near_threshold"], "branch"),
    # circular, circular2: the turn adds fract(43758.5453 sin(12.9898 x + 78.233 y)); at sine arguments
    # of tens to hundreds the platform sine's last bits, 43758-fold, set the turn (agreement where the
    # argument is 0: the zero inputs).
    "circular": {**dict.fromkeys(["q1", "q3", "odd", "pi_e", "y_neg0x"], "branch"), "near_threshold": "huge"},
    "circular2": {**dict.fromkeys(["+y", "-y", "q1", "q3", "odd", "big", "pi_e", "unit", "y_neg0x"], "branch"),
                  "near_threshold": "huge"},
    # r_circleblur: the cell's jitter, the same hash of the cell.
    "r_circleblur": {"half_unit": "branch"},
    # hypershift2: the draw picks the rotation by f32(pi), whose sine the reference returns as 0.
    "hypershift2": dict.fromkeys(["+0+0", "+0-0", "normal_min", "subnormal", "lopsided", "y_neg0x"], "zero"),
}
FIRST_TWELVE = {"linear", "sinusoidal", "spherical", "swirl", "horseshoe", "polar", "disc", "ex", "julia", "bubble",
                "cylinder", "curl"}
# Bit for bit with the report (classes and the digest of the quantised values).
EXACT_DIGEST = sorted(["linear", "spherical", "swirl", "horseshoe", "polar", "bubble", "curl", "handkerchief",
                       "spiral", "hyperbolic", "bent", "eyefish", "noise", "blur", "cross", "rings2", "pdj",
                       "rectangles", "splits", "pre_blur", "secant2", "pie", "butterfly", "fan", "fisheye", "stripes",
                       "bent2", "rings", "linear3D", "klein_group", "subflame_wf", "pre_subflame_wf", "loonie",
                       "scry", "elliptic", "bipolar", "lazysusan", "separation", "cell", "edisc", "curve", "square",
                       "blade", "twintrian", "arch", "parabola", "super_shape", "conic", "cpow", "boarders",
                       "oscilloscope", "blur_circle", "blur_zoom", "blur_pixelize", "tancos", "spiralwing",
                       "panorama1", "panorama2", "circleblur", "henon", "cylinder2", "flipcircle", "lozi",
                       "bi_linear", "twoface", "flipy", "rippled", "loonie3", "d_spherical", "acoth", "arcsinh",
                       "arctanh", "ennepers", "post_spherical", "rays2", "rays3", "roundspher", "sech2_bs", "arcsech",
                       "arcsech2", "pre_curl", "barycentroid", "gridout", "bipolar2", "sigmoid", "blocky",
                       "kaleidoscope", "eclipse", "hypershift", "chunk", "rational3", "corners", "atan",
                       "collideoscope", "projective", "shredlin", "stwin", "squircular", "rays1", "fourth",
                       "squarize", "erf", "holesq", "gridout2", "crop", "acosh", "acosech", "sqrt_acoth",
                       "sqrt_acosh", "sqrt_acosech", "sqrt_asech", "sqrt_asinh", "sqrt_atanh", "log_tile2",
                       "tile_log", "glynnia", "glynnia3", "apollony", "tqmirror", "spirograph", "lissajous",
                       "tile_hlp", "tile_reverse", "invsquircular", "stripfit", "dustpoint", "threepoint_js",
                       "wallpaper_js", "hadamard_js", "invtree_js", "apocarpet_js", "siercarpet_js", "hypertile",
                       "hypertile1", "blur_linear", "shift", "glynnSim1", "glynnSim2", "starblur", "yin_yang",
                       "oscilloscope2", "boarders2", "squish", "julian2", "waffle", "sym_ng1", "sym_ng2", "sym_ng3",
                       "sym_ng4", "sym_ng5", "sym_ng6", "sym_ng7", "sym_ng8", "sym_ng9", "sym_ng10", "sym_ng11",
                       "sym_ng12", "sym_ng13", "sym_ng14", "sym_ng15", "sym_ng16", "sym_ng17", "sym_bg1", "sym_bg2",
                       "sym_bg3", "sym_bg4", "sym_bg5", "sym_bg6", "sym_bg7", "pre_circlecrop", "post_circlecrop",
                       "circlecrop", "zcone", "hemisphere", "zscale", "zblur", "blur3D", "ztranslate", "julia3Dz",
                       "curl3D", "helix", "helicoid", "pie3D", "butterfly3D", "pyramid", "whitney_umbrella",
                       "ennepers2", "spherical3D", "square3D", "bubble2", "splits3D", "loonie_3D", "blade3D", "line",
                       "inflateZ_1", "inflateZ_2", "inflateZ_3", "inflateZ_4", "inflateZ_5", "inflateZ_6", "ovoid3d",
                       "sph3D", "pre_blur3D", "extrude", "post_ztranslate_wf", "bubble_wf", "solid_sphere",
                       "matrix3D", "onion", "octagon", "xerf", "erf3D", "spherical3D_wf", "pre_wave3D_wf",
                       "hypertile3D", "voron", "minkQM", "poincare3D", "rosoni", "bwraps7", "curl_sp", "circleLinear",
                       "mobiq", "xheart_blur_wf", "affine3D", "w", "harmonograph_js",
                       "loonie2", "elliptic2", "asteria", "scry2", "pre_bwraps2", "post_bwraps2", "pre_rect_wf",
                       "spliptic_bs", "pointgrid_wf", "truchet2", "bubbleT3D",
                       "hypertile3D1", "hypertile3D2", "julian3Dx",
                       "cut_sqcir", "cut_yuebing", "cut_sincos", "cut_chains", "cut_hexdots",
                       "cut_sqsplits", "cut_btree", "cut_fractal", "cut_glypho", "cut_circdes", "cut_snowflake",
                       "cut_rgrid", "cut_x", "cut_kaleido", "cut_spiral", "cut_swarp",
                       "cut_apollonian", "cut_bricks", "cut_web", "cut_tileillusion", "cut_pattern", "cut_celtic",
                       "spherecrop", "scry_3D", "roundspher3D", "crop3D", "pre_boarders2", "splitbrdr", "minkowskope",
                       "glynnlissa"])


def golden():
    g = {}
    with open(os.path.join(HERE, "golden", "variation_probe_2d.txt"), encoding="utf-8") as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            n, c, d, slot = line.split()
            g[n] = (c, int(d, 16), int(slot))
    return g


GOLDEN = golden()


def probe(oracle, name):
    """The oracle's probe of `name` at its report batch slot, report stream."""
    slot = GOLDEN[name][2]
    return oracle.probe(name, xform_slot=slot, fold_first=slot == 0, report_stream=True)


@pytest.mark.parametrize("name", sorted(n for n in GOLDEN if n not in FIRST_TWELVE))
def test_wider_registry_probe_matches_the_reference(oracle, name):
    classes, digest, out = probe(oracle, name)
    gold, gold_digest, _ = GOLDEN[name]
    allowed = WIDER.get(name, {})
    for i, label in enumerate(LABELS):
        ours, theirs = classes[2 * i:2 * i + 2], gold[2 * i:2 * i + 2]
        if ours == theirs:
            continue
        assert label in allowed, f"{name} at {label}: ours {ours} reference {theirs}"
        vals = [float(v) for v in out[2 * i:2 * i + 2]]
        why = allowed[label]
        for c in range(2):
            if ours[c] == theirs[c]:
                continue
            v = vals[c]
            if why == "zero":
                assert abs(v) <= 2e-6 * max(1.0, max(abs(u) for u in vals if math.isfinite(u))), (name, label, v)
            elif why == "inf*0":
                assert math.isinf(v) and theirs[c] == "n", (name, label, v)
            elif why == "pow":
                assert math.isfinite(v) and theirs[c] == "n", (name, label, v)
            elif why == "signed-zero":
                assert v == 0.0 and theirs[c] in "0o", (name, label, v)
            elif why == "shared-square":
                assert math.isfinite(v) and theirs[c] == "n", (name, label, v)
            elif why == "tiny-quotient":
                assert math.isfinite(v) and theirs[c] in "0o", (name, label, v)
            elif why == "zero-divisor":
                assert math.isfinite(v) and theirs[c] in "iI", (name, label, v)
            elif why == "fused":
                assert math.isfinite(v) and theirs[c] in "iI", (name, label, v)
            elif why == "scaled-zero":
                assert math.isfinite(v) and theirs[c] in "0o", (name, label, v)
            elif why == "tiny-branch":
                assert math.isnan(v) and theirs[c] != "n", (name, label, v)
            elif why == "reassociated":
                assert math.isnan(v) and theirs[c] != "n", (name, label, v)
            else:
                assert why in ("huge", "branch"), why
    if name in EXACT_DIGEST:
        assert digest == gold_digest, f"{name}: digest {digest:016x} vs reference {gold_digest:016x}"


@pytest.mark.parametrize("name", sorted(FIRST_TWELVE))
def test_probe_classes_match_the_reference(oracle, name):
    classes, digest, out = probe(oracle, name)
    gold, gold_digest, _ = GOLDEN[name]
    allowed = SFU_SIN.get(name, {})
    for i, label in enumerate(LABELS):
        ours, theirs = classes[2 * i:2 * i + 2], gold[2 * i:2 * i + 2]
        if ours == theirs:
            continue
        assert label in allowed, f"{name} at {label}: ours {ours} reference {theirs}"
        vals = out[2 * i:2 * i + 2]
        why = allowed[label]
        for c in range(2):
            if ours[c] == theirs[c]:
                continue
            v = float(vals[c])
            if why in ("sin(pi)", "cos(pi/2)"):
                assert abs(v) < 1e-7 and theirs[c] in "0o", (name, label, v)
            elif why == "tiny":
                assert abs(v) < 1e-6 and theirs[c] in "0o", (name, label, v)
            elif why == "huge":
                assert theirs[c] in "0o", (name, label, v)      # the reference's sin(|x| > 1e6) is 0
            elif why == "inf*sin(pi)":
                assert math.isinf(v) and theirs[c] == "n", (name, label, v)   # inf * 0 on the reference
            elif why == "cancel":
                # m0 - m1 with m0 ~ m1: below the last few ulp of r*m0.
                assert abs(v) < 1e-5 * max(1.0, float(np.max(np.abs(vals)))), (name, label, v)
    if not allowed:
        assert digest == gold_digest, f"{name}: digest {digest:016x} vs reference {gold_digest:016x}"


def test_variations_match_the_report_bit_for_bit(oracle):
    assert sorted(n for n in FIRST_TWELVE if n not in SFU_SIN) == \
        sorted(["linear", "spherical", "swirl", "horseshoe", "polar", "bubble", "curl"])
    for n in EXACT_DIGEST:
        c, d, _ = probe(oracle, n)
        assert (c, d) == GOLDEN[n][:2], n


def test_report_slots_are_the_batch_plan():
    """The RNG variations' report slots (src/probe/batch.rs:94-139): ids
    below 99 in the first batch at their id; pie (id 150) the 52nd of the second."""
    for n, want in (("julia", 13), ("julian", 24), ("noise", 29), ("blur", 30), ("gaussian_blur", 31),
                    ("pre_blur", 54), ("juliascope", 69), ("radial_blur", 73), ("pie", 51)):
        assert GOLDEN[n][2] == want, n


def test_later_draws_come_from_the_report_stream(oracle):
    """gaussian_blur's radius sums its 2nd-5th draws: the current per-thread
    stream disagrees with the report at about half the inputs, the report's
    fixed-increment stream nowhere."""
    gold = GOLDEN["gaussian_blur"][0]
    c_now, _, _ = oracle.probe("gaussian_blur", xform_slot=31, fold_first=False)
    c_rep, d_rep, _ = oracle.probe("gaussian_blur", xform_slot=31, fold_first=False, report_stream=True)
    assert c_rep == gold
    assert sum(a != b for a, b in zip(c_now, gold)) >= 10


def test_julia_rng_slot_is_the_reference_batch_slot(oracle):
    """julia's omega draw comes from rng_init(13*27 + point, 0x9E3779B9): the
    signs of its outputs (away from the SFU inputs) pin the draw."""
    c13, _, _ = oracle.probe("julia", xform_slot=13, fold_first=False)
    c0, _, _ = oracle.probe("julia", xform_slot=3, fold_first=False)
    gold = GOLDEN["julia"][0]
    agree13 = sum(a == b for a, b in zip(c13, gold))
    agree0 = sum(a == b for a, b in zip(c0, gold))
    assert agree13 >= 48 and agree13 > agree0


def _flat_point(oracle, x, cfg):
    fl = oracle.Flame(cfg, 64, 64)
    return fl.world_to_pixel(x, 0.0)


def test_pixel_mapping_known_answers(oracle):
    """compute_kernel.rs:6404-6427, 6502-6511: at 64x64, zoom 1, a point at
    x = -1.96875 is pixel 0.5 (column 0); x = -2.03125 is pixel -0.5 (off)."""
    cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": 0, "f": 0, "weight": 1, "color": 0,
                                     "variations": {"linear": 1.0}}]}}
    assert _flat_point(oracle, -1.96875, cfg) == (0, 32)
    px, _ = _flat_point(oracle, -2.03125, cfg)
    assert px == -1


def test_point_render_lights_one_pixel(oracle):
    """The same test through the whole chaos game: every plotted point is
    the affine's constant, so one pixel lights, or none."""
    for x, lit in ((-1.96875, 1), (-2.03125, 0)):
        cfg = {"flame": {"transforms": [{"a": 0, "b": 0, "c": 0, "d": 0, "e": x, "f": 0, "weight": 1, "color": 0,
                                         "variations": {"linear": 1.0}}]}}
        fl = oracle.Flame(cfg, 64, 64)
        plotted, inframe, cnt, _ = fl.render(256, 400, rng="pcg", threads=2)
        assert plotted == 256 * (400 - 20)
        assert int((cnt > 0).sum()) == lit
        if lit:
            assert cnt[32, 0] == inframe == plotted


def test_agx_shape_of_the_reference(oracle):
    """The AgX highlight modes' curve against the reference's own checks of
    it (scene/tonemap.rs:370-397): rising, greys grey, black black, scene
    middle grey 0.18 to 0.35-0.55 display, white from 16, a bright colour's
    channels kept in order; the Punchy look darker below the middle, more
    saturated, greys still grey."""
    grey = lambda x, p=False: oracle.agx_display([x, x, x], p)
    last = -1.0
    for i in range(200):
        x = 1.0e-4 * 1.08 ** i
        g = grey(x)
        assert abs(g[0] - g[1]) < 2e-3 and abs(g[1] - g[2]) < 2e-3, (x, g)
        assert g[0] >= last - 1e-6, x
        last = g[0]
    assert grey(0.0)[0] < 0.01
    assert 0.35 <= grey(0.18)[0] <= 0.55
    assert grey(16.0)[0] > 0.97
    o = oracle.agx_display([8.0, 4.0, 0.5])
    assert o[0] > o[1] > o[2]
    assert grey(0.05, True)[0] < grey(0.05)[0] and abs(grey(0.05, True)[0] - grey(0.05, True)[2]) < 2e-3
    o, p = oracle.agx_display([1.0, 0.3, 0.1]), oracle.agx_display([1.0, 0.3, 0.1], True)
    assert p[0] - p[2] > o[0] - o[2]


def test_firefly_downsample_known_answers(oracle):
    """supersample.rs:132-167: a uniform quad passes; a lone bright sample
    over a dark quad is clamped to 4x the median luminance plus 64."""
    quad = np.array([[[10, 20, 30, 255]] * 2] * 2, np.uint8)
    out = oracle.downsample_firefly(quad, 1, 1)
    assert out[0, 0].tolist() == [10, 20, 30, 255]
    q = np.zeros((2, 2, 4), np.uint8)
    q[..., 3] = 255
    q[0, 0] = [255, 255, 255, 255]
    out = oracle.downsample_firefly(q, 1, 1)
    # lum 1020 over cap 64: scale 64/1020; (255*64/1020)/4 = 4.0
    assert out[0, 0].tolist() == [4, 4, 4, 255]


def test_pcg_matches_rng_wgsl(oracle):
    """rng.wgsl:23-45 restated: pcg_hash(0) and the first draws of a stream,
    against the formula written out in Python."""
    def h(x):
        s = (x * 747796405 + 2891336453) & 0xFFFFFFFF
        w = (((s >> ((s >> 28) + 4)) ^ s) * 277803737) & 0xFFFFFFFF
        return (w >> 22) ^ w
    for x in (0, 1, 12345, 0xFFFFFFFF):
        assert oracle.pcg_hash(x) == h(x)
    st = oracle.rng_init(7, 12345)
    assert st[0] == h(7 ^ 12345)
    assert st[1] == ((h((h(7) + 12345) & 0xFFFFFFFF) << 1) | 1) & 0xFFFFFFFF


def test_philox_known_answer(oracle):
    """Philox4x32-10 known-answer vectors (Random123 kat_vectors)."""
    assert oracle.philox(0, 0, [0, 0, 0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert oracle.philox(0xffffffff, 0xffffffff, [0xffffffff] * 4) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert oracle.philox(0xa4093822, 0x299f31d0, [0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344]) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_palette_f16_and_decode(oracle):
    """buffers.rs:3215-3221: texels are f16(clamp(v,0,1)); utilities.wgsl:143-145 decodes with pow 2.2."""
    assert oracle.f16_round(1.0 / 3.0) == np.float32(0.333251953125)
    assert oracle.f16_round(1.0) == 1.0
    assert oracle.f16_round(1e-6) == np.float32(round(1e-6 * 2 ** 24) / 2 ** 24)
    cfg = {"palette": {"indexed_colors": "000000,FFFFFF"}, "palette_size": 2}
    t = oracle.palette_table(cfg).reshape(-1, 3)
    assert t[0].tolist() == [0.0, 0.0, 0.0] and t[1].tolist() == [1.0, 1.0, 1.0]
