"""ctypes front of the CPU oracle (oracle/flame_oracle.cpp) -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module, and only as the checker.  The product never does.

The oracle restates the reference's render path (see the C++ header for the
file:line of every function).  This module turns a flame description (the
`.fae` JSON subset, as a Python dict) into the oracle's flat arrays: the
local variation order of the reference (src/scene/transforms.rs:40-70,
668-682, 2297-2319), the f32 transform records, the palette table.
"""

import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

# Registry ids: positions in ALL_VARIATIONS (src/variations/defs/mod.rs:446).
REGISTRY = {
    "linear": 0, "sinusoidal": 1, "spherical": 2, "swirl": 3, "horseshoe": 4,
    "polar": 5, "handkerchief": 6, "heart": 7, "disc": 8, "spiral": 9, "hyperbolic": 10,
    "diamond": 11, "ex": 12, "julia": 13, "bent": 14, "waves": 15, "flatten": 17,
    "julian": 24, "blob": 25, "eyefish": 26, "bubble": 27, "cylinder": 28, "noise": 29,
    "blur": 30, "gaussian_blur": 31, "polar2": 32, "cross": 33, "rings2": 44, "fan2": 45,
    "pdj": 46, "curl": 47, "rectangles": 48, "splits": 49, "ngon": 50, "pre_blur": 54,
    "wedge": 66, "juliascope": 69, "radial_blur": 73, "tangent": 141, "secant2": 143,
    "cosine": 144, "pie": 150, "butterfly": 152, "popcorn": 181, "fan": 190, "fisheye": 191,
    "split": 248, "stripes": 250, "bent2": 281, "power": 325, "exponential": 341,
    "perspective": 345, "rings": 379, "klein_group": 501, "subflame_wf": 502, "pre_subflame_wf": 503,
    "linear3D": 533,
    "loonie": 34, "scry": 35, "foci": 37, "elliptic": 38, "waves2": 39, "log": 40, "escher": 41, "bipolar": 42,
    "lazysusan": 43, "auger": 51, "separation": 77, "mobius": 78, "sin": 93, "cos": 94, "tan": 95, "sec": 96,
    "csc": 97, "cot": 98, "sinh": 99, "cosh": 100, "tanh": 101, "coth": 102, "sech": 103, "csch": 104, "exp": 136,
    "cell": 161, "popcorn2": 170, "modulus": 273, "whorl": 302, "flux": 307, "edisc": 337, "curve": 338,
    "cpow": 85, "parabola": 149, "flower": 163, "square": 166, "disc2": 178, "wedge_julia": 210, "wedge_sph": 211,
    "super_shape": 212, "boarders": 229, "oscilloscope": 284, "rays": 308, "arch": 312, "blade": 314,
    "twintrian": 319, "conic": 324,
    "epispiral": 67, "blur_circle": 74, "blur_zoom": 75, "blur_pixelize": 76, "tancos": 140, "petal": 145,
    "cardioid": 146, "spiralwing": 158, "panorama1": 194, "panorama2": 195, "circleblur": 198, "henon": 213,
    "cylinder2": 241,
    "flipcircle": 200, "lozi": 243, "bi_linear": 313, "twoface": 318, "unpolar": 320, "idisc": 323, "exp2": 340,
    "flipy": 342, "invpolar": 344, "swirl3": 374, "wdisc": 375, "rippled": 380,
    "sin2_bs": 123, "cos2_bs": 124, "sinh2_bs": 129, "cosh2_bs": 130, "exp2_bs": 135, "pulse": 244, "linearT": 287,
    "layered_spiral": 363,
    "circlesplit": 199, "loonie3": 217, "mcarpet": 282, "d_spherical": 334, "clifford_js": 435,
    "pre_spherical": 57, "pre_sinusoidal": 58, "pre_disc": 59, "acoth": 86, "arcsinh": 91, "arctanh": 92,
    "tan2_bs": 125, "sec2_bs": 126, "csc2_bs": 127, "cot2_bs": 128, "tanh2_bs": 131, "coth2_bs": 132, "sech2_bs": 133,
    "csch2_bs": 134, "ennepers": 154, "rays2": 156, "rays3": 157, "squirrel": 249, "anamorphcyl": 296, "roundspher": 326,
    "deltaA": 336, "sintrange": 354, "hyperbolicellipse": 362, "post_spherical": 388, "svensson_js": 436,
    "epispiral_wf": 446,
    "post_curl": 83,
    "arcsech": 89,
    "arcsech2": 90,
    "sinq": 105,
    "cosq": 106,
    "tanq": 107,
    "cotq": 108,
    "secq": 109,
    "cscq": 110,
    "sinhq": 111,
    "coshq": 112,
    "tanhq": 113,
    "cothq": 114,
    "sechq": 115,
    "cschq": 116,
    "pre_curl": 221,
    "bCollide": 262,
    "bMod": 263,
    "bSwirl": 264,
    "barycentroid": 265,
    "eCollide": 266,
    "eMod": 267,
    "eSwirl": 268,
    "eScale": 269,
    "ePush": 270,
    "eRotate": 271,
    "gridout": 192,
    "bipolar2": 202,
    "sigmoid": 219,
    "blocky": 220,
    "kaleidoscope": 233,
    "hole2": 235,
    "eclipse": 242,
    "hypershift": 245,
    "chunk": 257,
    "pTransform": 258,
    "rational3": 259,
    "ortho": 261,
    "corners": 272,
    "circlize": 276,
    "circlize2": 277,
    "atan": 278,
    "collideoscope": 280,
    "fibonacci2": 285,
    "disc3": 290,
    "projective": 291,
    "shredlin": 298,
    "stwin": 301,
    "devil_warp": 303,
    "squircular": 306,
    "rays1": 309,
    "fourth": 311,
    "squarize": 316,
    "erf": 332,
    "funnel": 343,
    "holesq": 347,
    "fdisc": 358,
    "csc_squared": 361,
    "atan2_spirals": 364,
    "gridout2": 365,
    "eMotion": 367,
    "mask": 370,
    "pre_crop": 61,
    "falloff2": 65,
    "crop": 79,
    "post_crop": 81,
    "acosh": 87,
    "acosech": 88,
    "sqrt_acoth": 117,
    "sqrt_acosh": 118,
    "sqrt_acosech": 119,
    "sqrt_asech": 120,
    "sqrt_asinh": 121,
    "sqrt_atanh": 122,
    "log_tile2": 138,
    "tile_log": 139,
    "chrysanthemum": 160,
    "mobiusN": 196,
    "glynnia": 205,
    "glynnia3": 206,
    "apollony": 214,
    "tqmirror": 292,
    "sineblur": 226,
    "spirograph": 236,
    "lissajous": 237,
    "sphericalN": 253,
    "tile_hlp": 255,
    "tile_reverse": 260,
    "murl2": 372,
    "invsquircular": 377,
    "stripfit": 382,
    "q_ode": 383,
    "waves2_radial": 390,
    "heart_wf": 429,
    "pre_falloff2": 62,
    "post_falloff2": 82,
    "inverted_julia": 322,
    "dustpoint": 335,
    "bTransform": 359,
    "cannabiscurve_wf": 426,
    "sattractor_js": 437,
    "threepoint_js": 438,
    "woggle_js": 440,
    "lace_js": 441,
    "wallpaper_js": 442,
    "hadamard_js": 443,
    "invtree_js": 444,
    "cloverleaf_wf": 447,
    "rose_wf": 448,
    "apocarpet_js": 458,
    "siercarpet_js": 473,
    "bwraps": 68,
    "hypertile": 184,
    "hypertile1": 185,
    "blur_linear": 201,
    "target": 179,
    "shift": 251,
    "pressure_wave": 252,
    "spligon": 254,
    "circus": 275,
    "murl": 279,
    "shredrad": 299,
    "xheart": 300,
    "pre_bwraps": 60,
    "post_bwraps": 80,
    "hypertile2": 186,
    "glynnSim1": 207,
    "glynnSim2": 208,
    "glynnSim3": 209,
    "target_sp": 216,
    "starblur": 227,
    "vogel": 238,
    "cpow3": 177,
    "yin_yang": 180,
    "oscilloscope2": 286,
    "phoenix_julia": 288,
    "pow_block": 289,
    "trade": 304,
    "checks": 330,
    "boarders2": 230,
    "squish": 317,
    "npolar": 360,
    "eJulia": 366,
    "julian2": 369,
    "waffle": 381,
    "ripple": 384,
    "sym_ng1": 544,
    "sym_ng2": 545,
    "sym_ng3": 546,
    "sym_ng4": 547,
    "sym_ng5": 548,
    "sym_ng6": 549,
    "sym_ng7": 550,
    "sym_ng8": 551,
    "sym_ng9": 552,
    "sym_ng10": 553,
    "sym_ng11": 554,
    "sym_ng12": 555,
    "sym_ng13": 556,
    "sym_ng14": 557,
    "sym_ng15": 558,
    "sym_ng16": 559,
    "sym_ng17": 560,
    "sym_bg1": 561,
    "sym_bg2": 562,
    "sym_bg3": 563,
    "sym_bg4": 564,
    "sym_bg5": 565,
    "sym_bg6": 566,
    "sym_bg7": 567,
    "bsplit": 240,
    "pre_circlecrop": 410,
    "post_circlecrop": 411,
    "circlecrop": 412,
    "zcone": 16,
    "hemisphere": 18,
    "pre_rotate_x": 19,
    "pre_rotate_y": 20,
    "post_rotate_x": 21,
    "post_rotate_y": 22,
    "zscale": 23,
    "zblur": 52,
    "blur3D": 53,
    "pre_zscale": 55,
    "pre_ztranslate": 56,
    "ztranslate": 63,
    "julia3D": 64,
    "julia3Dz": 71,
    "curl3D": 72,
    "post_curl3D": 84,
    "tangent3D": 142,
    "helix": 147,
    "helicoid": 148,
    "pie3D": 151,
    "butterfly3D": 153,
    "pyramid": 155,
    "whitney_umbrella": 159,
    "ennepers2": 162,
    "spherical3D": 164,
    "sinusoidal3d": 165,
    "square3D": 167,
    "disc3d": 168,
    "bubble2": 169,
    "splits3D": 171,
    "waves2_3D": 172,
    "blob3D": 203,
    "loonie_3D": 218,
    "taurus": 234,
    "linearT3D": 283,
    "svf": 297,
    "blade3D": 315,
    "cone": 331,
    "line": 346,
    "inflateZ_1": 348,
    "inflateZ_2": 349,
    "inflateZ_3": 350,
    "inflateZ_4": 351,
    "inflateZ_5": 352,
    "inflateZ_6": 353,
    "foci_3D": 355,
    "estiq": 357,
    "ovoid3d": 371,
    "sph3D": 376,
    "pre_spin_z": 386,
    "post_spin_z": 387,
    "pre_disc3d": 389,
    "pre_sinusoidal3d": 393,
    "pre_blur3D": 394,
    "extrude": 415,
    "post_ztranslate_wf": 430,
    "bubble_wf": 449,
    "dinis_surface_wf": 455,
    "popcorn2_3D": 474,
    "solid_sphere": 605,
    "matrix3D": 643,
    "onion": 215,
    "ho": 256,
    "octagon": 274,
    "xerf": 321,
    "erf3D": 333,
    "flower_db": 368,
    "sphere_nja": 378,
    "loq": 400,
    "seashell3D": 397,
    "exblur": 413,
    "lazysensen": 421,
    "spherical3D_wf": 427,
    "pre_wave3D_wf": 468,
    "hypertile3D": 187,
    "hypercrop": 247,
    "voron": 305,
    "minkQM": 373,
    "poincare3D": 392,
    "rosoni": 396,
    "bwraps7": 399,
    "post_heat": 404,
    "onion2": 406,
    "curl_sp": 414,
    "circleLinear": 425,
    "waves2_wf": 452,
    "waves3_wf": 453,
    "waves4_wf": 454,
    "plusrecip": 476,
    "gamma": 477,
    "mobiq": 197,
    "jac_sn": 407,
    "jac_cn": 408,
    "jac_dn": 409,
    "xheart_blur_wf": 423,
    "affine3D": 464,
    "z": 489,
    "w": 490,
    "harmonograph_js": 496,
    "loonie2": 310,
    "elliptic2": 339,
    "asteria": 356,
    "scry2": 385,
    "pre_bwraps2": 402,
    "post_bwraps2": 403,
    "post_rblur": 405,
    "cpow3_wf": 434,
    "pre_rect_wf": 463,
    "spliptic_bs": 391,
    "pointgrid_wf": 456,
    "truchet2": 465,
    "bubbleT3D": 478,
    "pRose3D": 568,
    "hypertile3D1": 188,
    "hypertile3D2": 189,
    "julian3Dx": 395,
    "waves2b": 479,
    "log_db": 137,
    "juliaq": 173,
    "julia3Dq": 174,
    "juliac": 175,
    "cpow2": 176,
    "post_juliaq": 222,
    "post_julia3Dq": 223,
    "cut_sqcir": 570,
    "cut_yuebing": 571,
    "cut_vasarely": 572,
    "cut_sincos": 573,
    "cut_chains": 574,
    "cut_hexdots": 575,
    "cut_booleans": 576,
    "cut_sqsplits": 577,
    "cut_btree": 578,
    "cut_fractal": 579,
    "cut_glypho": 580,
    "cut_circdes": 581,
    "cut_snowflake": 582,
    "cut_jigsaw": 583,
    "cut_rgrid": 584,
    "cut_x": 585,
    "cut_metaballs": 586,
    "cut_kaleido": 587,
    "cut_spiral": 588,
    "cut_swarp": 589,
    "cut_apollonian": 590,
    "cut_zigzag": 591,
    "cut_bricks": 592,
    "cut_web": 593,
    "cut_tileillusion": 595,
    "cut_pattern": 596,
    "cut_celtic": 597,
    "cut_hextruchetflow": 569,
    "circular": 193,
    "circular2": 204,
    "r_circleblur": 228,
    "hypershift2": 398,
    "spherecrop": 422,
    "scry_3D": 36,
    "roundspher3D": 327,
    "crop3D": 239,
    "pre_boarders2": 231,
    "splitbrdr": 232,
    "minkowskope": 417,
    "glynnlissa": 418,
}
# User parameters and their defaults (the ParamDef lists of
# src/variations/defs/*.rs); derived values come from the C oracle's
# restatement of each `wgsl_init` (of_var_row).
PARAMS = {
    "curl": [("c1", 1.0), ("c2", 0.0)],
    "julian": [("power", 2.0), ("dist", 1.0)],
    "blob": [("high", 1.0), ("low", 1.0), ("waves", 6.0)],
    "rings2": [("val", 1.0)],
    "fan2": [("x", 1.0), ("y", 0.0)],
    "pdj": [("a", 0.0), ("b", 0.0), ("c", 0.0), ("d", 0.0)],
    "rectangles": [("x", 1.0), ("y", 1.0)],
    "splits": [("x", 0.4), ("y", 0.4), ("lshear", 0.0), ("rshear", 0.0), ("ushear", 0.0), ("dshear", 0.0)],
    "ngon": [("sides", 5.0), ("power", 3.0), ("circle", 1.0), ("corners", 2.0)],
    "wedge": [("angle", 90.0), ("hole", 0.0), ("count", 2.0), ("swirl", 0.0)],
    "juliascope": [("power", 2.0), ("dist", 1.0)],
    "radial_blur": [("angle", 0.0)],
    "pie": [("slices", 6.0), ("rotation", 0.0), ("thickness", 0.5)],
    "split": [("xsize", 0.4), ("ysize", 0.6)],
    "stripes": [("space", 0.2), ("warp", 0.6)],
    "bent2": [("x", 1.0), ("y", 1.0)],
    "perspective": [("angle", 0.62), ("dist", 2.2)],
    "klein_group": [("a_re", 2.0), ("a_im", 0.0), ("b_re", 2.0), ("b_im", 0.0), ("recipe", 0.0), ("avoid_reversal", 1.0)],
    "subflame_wf": [("subflame_id", 0.0), ("scale", 1.0), ("angle", 0.0), ("offset_x", 0.0), ("offset_y", 0.0),
                    ("offset_z", 0.0), ("colorscale_z", 0.0), ("color_mode", -1.0)],
}
PARAMS.update({
    "waves2": [("freqx", 2.0), ("scalex", 1.0), ("freqy", 2.0), ("scaley", 1.0), ("freqz", 0.0), ("scalez", 0.0)],
    "log": [("base", 2.718281828)],
    "escher": [("beta", 0.0)],
    "bipolar": [("shift", 0.0)],
    "lazysusan": [("spin", 0.0), ("space", 0.0), ("twist", 0.0), ("x", 0.0), ("y", 0.0)],
    "auger": [("freq", 1.0), ("weight", 0.5), ("scale", 0.5), ("sym", 0.0)],
    "separation": [("x", 1.0), ("y", 1.0), ("xinside", 0.0), ("yinside", 0.0)],
    "mobius": [("re_a", 0.1), ("im_a", 0.2), ("re_b", 0.2), ("im_b", -0.12), ("re_c", -0.15), ("im_c", -0.15),
               ("re_d", 0.21), ("im_d", 0.1)],
    "cell": [("size", 0.6)],
    "popcorn2": [("x", 1.0), ("y", 0.5), ("c", 1.5)],
    "modulus": [("x", 0.2), ("y", 0.5)],
    "whorl": [("inside", 0.1), ("outside", 0.2)],
    "flux": [("spread", 0.3)],
    "curve": [("xamp", 0.25), ("yamp", 0.5), ("xlength", 1.0), ("ylength", 1.0)],
    "parabola": [("width", 1.0), ("height", 0.5)],
    "flower": [("holes", 0.4), ("petals", 7.0)],
    "super_shape": [("rnd", 3.0), ("m", 1.0), ("n1", 1.0), ("n2", 1.0), ("n3", 1.0), ("holes", 0.0)],
    "conic": [("eccentricity", 1.0), ("holes", 0.0)],
    "disc2": [("rot", 2.0), ("twist", 0.5)],
    "cpow": [("r", 1.0), ("i", 0.1), ("power", 1.5)],
    "oscilloscope": [("separation", 1.0), ("frequency", 3.14159265), ("amplitude", 1.0), ("damping", 0.0)],
    "wedge_julia": [("power", 7.0), ("dist", 0.2), ("count", 2.0), ("angle", 0.3)],
    "wedge_sph": [("angle", 0.2), ("hole", 0.2), ("count", 2.0), ("swirl", 0.3)],
    "epispiral": [("n", 6.0), ("thickness", 0.0), ("holes", 1.0)],
    "blur_zoom": [("length", 0.0), ("x", 0.0), ("y", 0.0)],
    "blur_pixelize": [("size", 0.1), ("scale", 1.0)],
    "cardioid": [("a", 1.0)],
    "henon": [("a", 0.5), ("b", 1.0), ("c", 1.0)],
    "lozi": [("a", 0.5), ("b", 1.0), ("c", 1.0)],
    "swirl3": [("shift", 0.5)],
    **{n: [("x1", 1.0), ("x2", 1.0), ("y1", 1.0), ("y2", 1.0)] for n in ("sin2_bs", "cos2_bs", "sinh2_bs", "cosh2_bs")},
    "exp2_bs": [("x1", 1.0), ("y1", 1.0), ("y2", 1.0)],
    "pulse": [("freqx", 2.0), ("freqy", 2.0), ("scalex", 1.0), ("scaley", 1.0)],
    "linearT": [("powX", 1.2), ("powY", 1.2)],
    "layered_spiral": [("radius", 1.0)],
    "circlesplit": [("radius", 1.0), ("split", 0.5)],
    "mcarpet": [("x", 1.0), ("y", 1.0), ("twist", 0.0), ("tilt", 0.0)],
    "d_spherical": [("d_spher_weight", 0.5)],
    "clifford_js": [("a", -1.4), ("b", 1.6), ("c", 1.0), ("d", 0.7)],
    **{n: [("x1", 2.0), ("x2", 2.0), ("y1", 2.0), ("y2", 2.0)] for n in ("tan2_bs", "cot2_bs", "tanh2_bs", "coth2_bs")},
    **{n: [("x1", 1.0), ("x2", 1.0), ("y1", 1.0), ("y2", 1.0)] for n in ("sec2_bs", "csc2_bs", "sech2_bs", "csch2_bs")},
    "epispiral_wf": [("waves", 4.0)],
    "hyperbolicellipse": [("a", 1.0)],
    "sintrange": [("w", 1.0)],
    "squirrel": [("a", 1.0), ("b", 1.0)],
    "anamorphcyl": [("a", 1.0), ("b", 1.3), ("k", 3.0)],
    "svensson_js": [("a", 1.4), ("b", 1.56), ("c", 1.4), ("d", -6.56)],
    "post_curl": [("c1", 0.0), ("c2", 0.0)],
    "pre_curl": [("c1", 0.0), ("c2", 0.0)],
    "bCollide": [("num", 1.0), ("a", 0.0)],
    "bMod": [("radius", 1.0), ("distance", 0.0)],
    "bSwirl": [("in_p", 0.0), ("out_p", 0.0)],
    "barycentroid": [("a", 1.0), ("b", 0.0), ("c", 0.0), ("d", 1.0)],
    "eCollide": [("num", 1.0), ("a", 0.0)],
    "eMod": [("radius", 1.0), ("distance", 0.0)],
    "eSwirl": [("in_p", 1.2), ("out_p", 0.2)],
    "eScale": [("scale", 1.0), ("angle", 0.0)],
    "ePush": [("push", 0.0), ("dist", 1.0), ("rotate", 0.0)],
    "eRotate": [("rotate", 0.0)],
})
PARAMS.update({
    "bipolar2": [("shift", 0.0), ("a", 1.0), ("b", 2.0), ("c", 0.5), ("d", 1.0), ("e", 2.0), ("f1", 0.25), ("g1", 1.0), ("h", 1.0)],
    "sigmoid": [("shiftx", 1.0), ("shifty", 1.0)],
    "blocky": [("x", 1.0), ("y", 1.0), ("mp", 4.0)],
    "kaleidoscope": [("pull", 0.0), ("rotate", 1.0), ("line_up", 1.0), ("x", 0.0), ("y", 0.0)],
    "hole2": [("a", 1.0), ("b", 2.0), ("c", 1.0), ("d", 1.0), ("inside", 0.0), ("shape", 0.0)],
    "eclipse": [("shift", 0.0)],
    "hypershift": [("shift", 2.0), ("stretch", 1.0)],
    "chunk": [("a", 1.0), ("b", 0.0), ("c", 1.0), ("d", 0.0), ("e", 0.0), ("f", -1.0), ("mode", 0.0)],
    "pTransform": [("rotate", 0.0), ("power", 1.0), ("move", 0.0), ("split", 0.0), ("use_log", 1.0)],
    "rational3": [("a", 0.5), ("b", 0.0), ("c", 0.0), ("d", 1.0), ("e", 0.0), ("f", 1.0), ("g", 0.0), ("h", 1.0)],
    "ortho": [("in_p", 0.0), ("out_p", 0.0)],
    "corners": [("xwidth", 1.0), ("ywidth", 1.0), ("multx", 1.0), ("multy", 1.0), ("xpower", 0.75), ("ypower", 0.75), ("xypower", 0.0), ("logmode", 0.0), ("log_base", 2.71828)],
    "circlize": [("hole", 0.4)],
    "circlize2": [("hole", 0.0)],
    "atan": [("mode", 0.0), ("stretch", 1.0)],
    "collideoscope": [("a", 0.2), ("num", 1.0)],
    "fibonacci2": [("sc", 1.0), ("sc2", 1.0)],
    "disc3": [("a", 1.0), ("b", 1.0), ("c", 1.0), ("d", 1.0), ("e", 1.0), ("f", 1.0), ("g", 1.0), ("h", 1.0)],
    "projective": [("a", 0.0), ("b", 0.0), ("c", 1.0), ("a1", 1.0), ("b1", 0.0), ("c1", 0.0), ("a2", 0.0), ("b2", 1.0), ("c2", 0.0)],
})
PARAMS.update({
    "shredlin": [("xdistance", 1.0), ("xwidth", 0.5), ("ydistance", 1.0), ("ywidth", 0.5)],
    "stwin": [("distort", 1.0), ("offset_xy", 0.0), ("offset_x2", 0.0), ("offset_y2", 0.0)],
    "devil_warp": [("a", 2.0), ("b", 1.0), ("effect", 1.0), ("warp", 0.5), ("rmin", -0.24), ("rmax", 100.0)],
    "fourth": [("spin", 3.14159265), ("space", 0.0), ("twist", 0.0), ("x", 0.0), ("y", 0.0)],
    "funnel": [("effect", 8.0)],
    "fdisc": [("ashift", 1.0), ("rshift", 1.0), ("xshift", 0.0), ("yshift", 0.0), ("term1", 1.0), ("term2", 0.0), ("term3", 0.0), ("term4", 0.0)],
    "csc_squared": [("csc_div", 1.0), ("cos_div", 1.0), ("tan_div", 1.0), ("csc_pow", 0.5), ("pi_mult", 0.5), ("csc_add", 0.25), ("scaley", 1.0)],
    "atan2_spirals": [("r_mult", 1.5), ("r_add", 1.0), ("xy2_mult", 1.125), ("xy2_add", 0.132), ("x_mult", 2.0), ("x_add", 0.25), ("yx_div", 1.0), ("yx_add", 0.0), ("yy_div", 1.25), ("yy_add", 0.0), ("sin_add", 0.0), ("y_mult", 1.0), ("r_power", 0.5), ("x2y2_pow", 1.0)],
    "gridout2": [("a", 1.0), ("b", 1.0), ("c", 1.0), ("d", 1.0)],
    "eMotion": [("move", 0.0), ("rotate", 0.0)],
    "mask": [("xshift", 0.0), ("yshift", 0.0), ("ushift", 1.0), ("xscale", 1.0), ("yscale", 1.0)],
})
PARAMS.update({
    "pre_crop": [("left", -1.0), ("top", -1.0), ("right", 1.0), ("bottom", 1.0), ("scatter_area", 0.0), ("zero", 0.0)],
    "falloff2": [("scatter", 1.0), ("mindist", 0.5), ("mul_x", 1.0), ("mul_y", 1.0), ("mul_z", 0.0), ("mul_c", 0.0), ("x0", 0.0), ("y0", 0.0), ("z0", 0.0), ("invert", 0.0), ("type", 0.0)],
    "crop": [("left", -1.0), ("top", -1.0), ("right", 1.0), ("bottom", 1.0), ("scatter_area", 0.0), ("zero", 0.0)],
    "post_crop": [("left", -1.0), ("top", -1.0), ("right", 1.0), ("bottom", 1.0), ("scatter_area", 0.0), ("zero", 0.0)],
    "log_tile2": [("spreadx", 2.0), ("spready", 2.0), ("spreadz", 0.0)],
    "tile_log": [("spread", 1.0)],
})
PARAMS.update({
    "mobiusN": [("re_a", 1.0), ("re_b", 0.0), ("re_c", 0.0), ("re_d", 1.0), ("im_a", 0.0), ("im_b", 0.0), ("im_c", 0.0), ("im_d", 0.0), ("power", 1.0), ("dist", 1.0)],
    "glynnia3": [("rscale", 1.0), ("dscale", 1.0), ("rthresh", 0.0), ("ythresh", 0.0)],
    "tqmirror": [("a", 1.0), ("b", 1.0), ("c", 1.0), ("d", 1.0), ("e", 1.0), ("f", 1.0), ("g", 1.0), ("h", 1.0), ("type", 0.0)],
    "sineblur": [("power", 1.0)],
    "spirograph": [("a", 3.0), ("b", 2.0), ("d", 0.0), ("c1", 0.0), ("c2", 0.0), ("tmin", -1.0), ("tmax", 1.0), ("ymin", -1.0), ("ymax", 1.0)],
    "lissajous": [("tmin", -3.14159265), ("tmax", 3.14159265), ("a", 3.0), ("b", 2.0), ("c", 0.0), ("d", 0.0), ("e", 0.0)],
    "sphericalN": [("power", 1.0), ("dist", 1.0)],
    "tile_hlp": [("width", 1.0)],
    "tile_reverse": [("space", 1.0), ("reversal", 1.0), ("vertical", 0.0)],
    "murl2": [("c", 0.1), ("power", 3.0)],
    "stripfit": [("dx", 1.0)],
    "q_ode": [("q_ode01", 0.0), ("q_ode02", 1.0), ("q_ode03", 0.0), ("q_ode04", 0.0), ("q_ode05", 0.0), ("q_ode06", 0.0), ("q_ode07", 0.0), ("q_ode08", 1.0), ("q_ode09", 0.0), ("q_ode10", 0.0), ("q_ode11", 0.0), ("q_ode12", 0.0)],
    "waves2_radial": [("w2r_scalex", 0.1), ("w2r_scaley", 0.1), ("w2r_freqx", 7.0), ("w2r_freqy", 13.0), ("w2r_null", 2.0), ("w2r_distance", 10.0)],
    "heart_wf": [("scale_x", 1.0), ("scale_t", 1.0), ("shift_t", 0.0), ("scale_r_left", 1.0), ("scale_r_right", 1.0)],
})
PARAMS.update({
    "pre_falloff2": [("scatter", 1.0), ("mindist", 0.5), ("mul_x", 1.0), ("mul_y", 1.0), ("mul_z", 0.0), ("mul_c", 0.0), ("x0", 0.0), ("y0", 0.0), ("z0", 0.0), ("invert", 0.0), ("type", 0.0)],
    "post_falloff2": [("scatter", 1.0), ("mindist", 0.5), ("mul_x", 1.0), ("mul_y", 1.0), ("mul_z", 0.0), ("mul_c", 0.0), ("x0", 0.0), ("y0", 0.0), ("z0", 0.0), ("invert", 0.0), ("type", 0.0)],
    "inverted_julia": [("power", 0.25), ("y2_mult", 1.0), ("a2x_mult", 1.0), ("a2y_mult", 1.0), ("a2y_add", 0.0), ("cos_mult", 0.0), ("y_mult", 1.0), ("center", 3.14), ("x2y2_add", 0.0)],
    "bTransform": [("rotate", 0.0), ("power", 1.0), ("move", 0.0), ("split", 0.0)],
    "cannabiscurve_wf": [("filled", 1.0)],
    "sattractor_js": [("m", 10.0)],
    "woggle_js": [("m", 2.0)],
    "wallpaper_js": [("a", 1.156), ("b", -0.28), ("c", 21.288)],
    "cloverleaf_wf": [("filled", 1.0)],
    "rose_wf": [("amp", 0.5), ("waves", 4.0), ("filled", 0.0)],
    "siercarpet_js": [("m", 3.0)],
})
PARAMS.update({
    "bwraps": [("cellsize", 1.0), ("space", 0.0), ("gain", 1.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "hypertile": [("p", 3.0), ("q", 7.0), ("n", 1.0)],
    "hypertile1": [("p", 3.0), ("q", 7.0)],
    "blur_linear": [("length", 1.0), ("angle", 0.5)],
    "target": [("even", 0.0), ("odd", 0.0), ("size", 1.0)],
    "shift": [("shift_x", 0.0), ("shift_y", 0.0), ("angle", 0.0)],
    "pressure_wave": [("x_freq", 1.0), ("y_freq", 1.0)],
    "spligon": [("sides", 3.0), ("i", 1.0)],
    "circus": [("scale", 1.0)],
    "murl": [("c", 0.1), ("power", 1.0)],
    "shredrad": [("n", 4.0), ("width", 0.5)],
    "xheart": [("angle", 0.0), ("ratio", 0.0)],
})
PARAMS.update({
    "pre_bwraps": [("cellsize", 1.0), ("space", 0.0), ("gain", 1.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "post_bwraps": [("cellsize", 1.0), ("space", 0.0), ("gain", 1.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "hypertile2": [("p", 3.0), ("q", 7.0)],
    "glynnSim1": [("radius", 1.0), ("radius1", 0.1), ("phi1", 110.0), ("thickness", 0.1), ("pow", 1.5), ("contrast", 0.5)],
    "glynnSim2": [("radius", 1.0), ("thickness", 0.1), ("contrast", 0.5), ("pow", 1.5), ("phi1", 110.0), ("phi2", 150.0)],
    "glynnSim3": [("radius", 1.0), ("thickness", 0.1), ("contrast", 0.5), ("pow", 1.5)],
    "target_sp": [("twist", 0.0), ("n_of_sp", 1.0), ("size", 1.0), ("tightness", 0.5)],
    "starblur": [("power", 5.0), ("range", 0.40162283)],
    "vogel": [("n", 20.0), ("scale", 1.0)],
})
PARAMS.update({
    "cpow3": [("r", 1.0), ("d", 1.0), ("divisor", 1.0), ("spread", 1.0)],
    "yin_yang": [("radius", 0.5), ("ang1", 0.0), ("ang2", 0.0), ("dual_t", 1.0), ("outside", 0.0)],
    "oscilloscope2": [("separation", 1.0), ("frequencyx", 3.14159265), ("frequencyy", 3.14159265), ("amplitude", 1.0), ("perturbation", 1.0), ("damping", 0.0)],
    "phoenix_julia": [("power", 3.0), ("dist", 1.0), ("x_distort", -0.5), ("y_distort", 0.0)],
    "pow_block": [("numerator", 3.0), ("denominator", 2.0), ("correctn", 1.0), ("correctd", 1.0), ("root", 1.0)],
    "trade": [("r1", 1.0), ("d1", 1.0), ("r2", 1.0), ("d2", 1.0)],
    "checks": [("x", 0.5), ("y", 0.5), ("size", 0.5), ("rnd", 0.0)],
})
PARAMS.update({
    "boarders2": [("c", 0.4), ("left", 0.65), ("right", 0.35)],
    "squish": [("power", 2.0)],
    "npolar": [("parity", 0.0), ("n", 1.0)],
    "eJulia": [("power", 2.0)],
    "julian2": [("power", 0.0), ("dist", 1.0), ("a", 1.0), ("b", 0.0), ("c", 0.0), ("d", 1.0), ("e", 0.0), ("f", 0.0)],
    "waffle": [("slices", 6.0), ("xthickness", 0.5), ("ythickness", 0.5), ("rotation", 0.0)],
    "ripple": [("frequency", 2.0), ("velocity", 1.0), ("amplitude", 0.5), ("centerx", 0.0), ("centery", 0.0), ("phase", 0.0), ("scale", 1.0), ("fixed_dist_calc", 0.0)],
})
PARAMS.update({
    "sym_ng1": [("stepx", 0.5), ("stepy", 0.5)],
    "sym_ng2": [("stepx", 2.0), ("stepy", 2.0)],
    "sym_ng3": [("sepx", 0.5), ("sepy", 0.0), ("step", 2.0)],
    "sym_ng4": [("sepx", 0.0), ("sepy", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_ng5": [("sepx", 0.0), ("sepy", 0.0), ("stepx", 0.0)],
    "sym_ng6": [("sepy", 0.1), ("stepx", 1.0), ("stepy", 1.0)],
    "sym_ng7": [("sepx", 0.0), ("sepy", 0.0)],
    "sym_ng8": [("sepx", 0.0), ("sepy", 0.0), ("skewx", 0.0), ("skewy", 0.0)],
    "sym_ng9": [("sepx", 0.0), ("sepy", 0.0)],
    "sym_ng10": [("space", 0.0), ("spacex", 0.0), ("spacey", 0.0)],
    "sym_ng11": [("space", 0.0), ("spacex", 0.0), ("spacey", 0.0), ("stepx", 1.5), ("stepy", 1.5)],
    "sym_ng12": [("space", 0.0), ("spacex", 0.0), ("spacey", 0.0)],
    "sym_ng13": [("radius", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_ng14": [("radius", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_ng15": [("radius", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_ng16": [("radius", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_ng17": [("radius", 0.0), ("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg1": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg2": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg3": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg4": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg5": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg6": [("stepx", 0.0), ("stepy", 0.0)],
    "sym_bg7": [("stepx", 0.0), ("stepy", 0.0)],
})
PARAMS.update({
    "bsplit": [("x", 0.0), ("y", 0.0)],
    "pre_circlecrop": [("radius", 1.0), ("x", 0.0), ("y", 0.0), ("scatter_area", 0.0), ("zero", 1.0)],
    "post_circlecrop": [("radius", 1.0), ("x", 0.0), ("y", 0.0), ("scatter_area", 0.0), ("zero", 1.0)],
    "circlecrop": [("radius", 1.0), ("x", 0.0), ("y", 0.0), ("scatter_area", 0.0), ("zero", 1.0)],
})
PARAMS.update({
    "julia3D": [("power", 2.0)],
    "julia3Dz": [("power", 2.0)],
    "curl3D": [("cx", 0.0), ("cy", 0.0), ("cz", 0.0)],
    "post_curl3D": [("cx", 0.0), ("cy", 0.0), ("cz", 0.0)],
    "helix": [("frequency", 1.0), ("width", 0.5)],
    "helicoid": [("frequency", 1.0)],
    "pie3D": [("slices", 7.0), ("rotation", 0.0), ("thickness", 0.5)],
    "ennepers2": [("a", 1.0), ("b", 0.3333), ("c", 0.075)],
    "disc3d": [("pi", 3.14159265358979)],
    "bubble2": [("x", 1.0), ("y", 1.0), ("z", 0.0)],
    "splits3D": [("x", 0.1), ("y", 0.3), ("z", 0.2)],
    "waves2_3D": [("freq", 2.0), ("scale", 1.0)],
    "blob3D": [("low", 0.3), ("high", 1.2), ("waves", 6.0)],
})
PARAMS.update({
    "taurus": [("r", 3.0), ("n", 5.0), ("inv", 1.5), ("sor", 1.0)],
    "linearT3D": [("powX", 1.2), ("powY", 1.2), ("powZ", 1.2)],
    "svf": [("n", 2.0)],
    "cone": [("radius1", 0.5), ("radius2", 1.0), ("size1", 0.5), ("size2", 2.0), ("ywave", 1.0), ("xwave", 1.0), ("height", 1.0), ("warp", 1.0), ("weight", 2.0)],
    "line": [("delta", 0.0), ("phi", 0.0)],
    "ovoid3d": [("x", 1.0), ("y", 1.0), ("z", 1.0)],
    "sph3D": [("x", 1.0), ("y", 1.0), ("z", 1.0)],
    "pre_disc3d": [("pi", 3.141592653589793)],
    "extrude": [("root_face", 0.5)],
    "dinis_surface_wf": [("a", 0.8), ("b", 0.2)],
    "popcorn2_3D": [("popcorn2_3D_x", 0.1), ("popcorn2_3D_y", 0.1), ("popcorn2_3D_z", 0.1), ("popcorn2_3D_c", 3.0)],
    "solid_sphere": [("radius", 1.0), ("thickness", 0.1), ("cx", 0.0), ("cy", 0.0), ("cz", 0.0)],
    "matrix3D": [("xx", 1.0), ("xy", 0.0), ("xz", 0.0), ("yx", 0.0), ("yy", 1.0), ("yz", 0.0), ("zx", 0.0), ("zy", 0.0), ("zz", 1.0), ("tx", 0.0), ("ty", 0.0), ("tz", 0.0)],
})
PARAMS.update({
    "onion": [("centre_x", 0.0), ("centre_y", 0.0)],
    "ho": [("xpow", 3.0), ("ypow", 3.0), ("zpow", 3.0)],
    "octagon": [("x", 0.0), ("y", 0.0), ("z", 0.0)],
    "flower_db": [("petals", 6.0), ("petal_split", 0.0), ("petal_spread", 1.0), ("stem_thickness", 1.0), ("stem_length", 0.0), ("petal_fold_strength", 0.0), ("petal_fold_radius", 1.0)],
    "sphere_nja": [("circle_a", 1.0), ("circle_b", 1.0), ("shift_x", 0.0), ("shift_y", 0.0), ("shift_z", 0.0), ("stretch", 1.0)],
    "loq": [("base", 2.718281828459045)],
})
PARAMS.update({
    "seashell3D": [("final_radius", 0.25), ("height", 3.5), ("inner_radius", 0.4), ("nSpirals", 3.0)],
    "exblur": [("dist", 0.5), ("r", 0.0), ("x_origin", 0.0), ("y_origin", 0.0), ("z_origin", 0.0)],
    "lazysensen": [("scale_x", 1.0), ("scale_y", 1.0), ("scale_z", 0.0)],
    "spherical3D_wf": [("invert", 0.0), ("exponent", 2.0)],
    "pre_wave3D_wf": [("axis", 0.0), ("wavelen", 0.5), ("phase", 0.0), ("damping", 0.01), ("centre_x", 0.0), ("centre_y", 0.0), ("centre_z", 0.0)],
})
PARAMS.update({
    "hypertile3D": [("p", 3.0), ("q", 7.0), ("n", 0.0)],
    "hypercrop": [("n", 4.0), ("rad", 1.0), ("zero", 0.0)],
    "voron": [("k", 0.99), ("step", 0.25), ("num", 1.0), ("xseed", 3.0), ("yseed", 7.0)],
    "minkQM": [("a", 1.0), ("b", 1.0), ("c", 1.0), ("dd", 1.0), ("e", 0.5), ("f", 20.0)],
    "poincare3D": [("r", 0.0), ("a", 0.0), ("b", 0.0)],
    "rosoni": [("maxiter", 25.0), ("sweetiter", 3.0), ("altshapes", 0.0), ("cutoff", 1.0), ("radius", 0.4), ("dx", 0.6), ("dy", 0.0)],
    "bwraps7": [("cellsize", 1.0), ("space", 0.0), ("gain", 2.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "post_heat": [("theta_period", 0.0), ("theta_phase", 0.0), ("theta_amp", 0.0), ("phi_period", 0.0), ("phi_phase", 0.0), ("phi_amp", 0.0), ("r_period", 0.0), ("r_phase", 0.0), ("r_amp", 0.0)],
    "onion2": [("meeting_pt", 0.5), ("circle_a", 1.0), ("circle_b", 1.0), ("shift_x", 0.0), ("shift_y", 0.0), ("shift_z", 0.0), ("top_crop", 0.0), ("stretch", 1.0)],
    "curl_sp": [("pow", 1.0), ("c1", -0.01), ("c2", 0.03), ("sx", 0.0), ("sy", 0.0), ("dc", 0.0)],
    "circleLinear": [("Sc", 1.0), ("K", 0.5), ("Dens1", 0.5), ("Dens2", 0.5), ("Reverse", 1.0), ("X", 10.0), ("Y", 10.0), ("Seed", 0.0)],
    "waves2_wf": [("scalex", 0.25), ("scaley", 0.5), ("freqx", 1.5707963267948966), ("freqy", 0.7853981633974483), ("use_cos_x", 1.0), ("use_cos_y", 0.0), ("dampx", 0.0), ("dampy", 0.0)],
    "waves3_wf": [("scalex", 0.25), ("scaley", 0.5), ("freqx", 1.5707963267948966), ("freqy", 0.7853981633974483), ("use_cos_x", 1.0), ("use_cos_y", 0.0), ("dampx", 0.0), ("dampy", 0.0)],
    "waves4_wf": [("scalex", 0.25), ("scaley", 0.5), ("freqx", 1.5707963267948966), ("freqy", 0.7853981633974483), ("use_cos_x", 1.0), ("use_cos_y", 0.0), ("dampx", 0.0), ("dampy", 0.0)],
    "plusrecip": [("ar", 4.0), ("ai", 0.0)],
})
PARAMS.update({
    "mobiq": [("qat", 1.0), ("qax", 0.0), ("qay", 0.0), ("qaz", 0.0), ("qbt", 0.0), ("qbx", 0.0), ("qby", 0.0), ("qbz", 0.0), ("qct", 0.0), ("qcx", 0.0), ("qcy", 0.0), ("qcz", 0.0), ("qdt", 1.0), ("qdx", 0.0), ("qdy", 0.0), ("qdz", 0.0)],
    "jac_sn": [("jac_sn_k", 0.5)],
    "jac_cn": [("jac_cn_k", 0.5)],
    "jac_dn": [("jac_dn_k", 0.5)],
    "xheart_blur_wf": [("angle", 0.0), ("ratio", 0.0)],
    "affine3D": [("translateX", 0.0), ("translateY", 0.0), ("translateZ", 0.0), ("scaleX", 1.0), ("scaleY", 1.0), ("scaleZ", 1.0), ("rotateX", 0.0), ("rotateY", 0.0), ("rotateZ", 0.0), ("shearXY", 0.0), ("shearXZ", 0.0), ("shearYX", 0.0), ("shearYZ", 0.0), ("shearZX", 0.0), ("shearZY", 0.0)],
    "z": [("hypergon", 0.0), ("hypergon_n", 4.0), ("hypergon_r", 1.0), ("star", 0.0), ("star_n", 5.0), ("star_slope", 2.0), ("lituus", 0.0), ("lituus_a", 1.0), ("super_shape", 0.0), ("super_m", 1.0), ("super_n1", 1.0), ("super_n2", 1.0), ("super_n3", 0.0)],
    "w": [("angle", 0.0), ("hypergon", 0.0), ("hypergon_n", 4.0), ("hypergon_r", 1.0), ("star", 0.0), ("star_n", 5.0), ("star_slope", 2.0), ("lituus", 0.0), ("lituus_a", 1.0), ("super_shape", 0.0), ("super_m", 1.0), ("super_n1", 1.0), ("super_n2", 1.0), ("super_n3", 0.0)],
    "harmonograph_js": [("seed", 1234.0), ("time", 100.0), ("a1", 0.0), ("f1", 0.0), ("p1", 0.0), ("d1", 0.0), ("a2", 0.0), ("f2", 0.0), ("p2", 0.0), ("d2", 0.0), ("a3", 0.0), ("f3", 0.0), ("p3", 0.0), ("d3", 0.0), ("a4", 0.0), ("f4", 0.0), ("p4", 0.0), ("d4", 0.0)],
})
PARAMS.update({
    "loonie2": [("sides", 4.0), ("star", 0.0), ("circle", 0.0)],
    "elliptic2": [("a1", 1.0), ("a2", 1.0), ("a3", 0.0), ("b1", 2.0), ("b2", 1.0), ("c", 0.5), ("d", 1.0), ("e", 0.5), ("f", 1.0), ("g", 1.0), ("h", 2.0)],
    "asteria": [("alpha", 0.0)],
    "scry2": [("sides", 4.0), ("star", 0.0), ("circle", 0.0)],
    "pre_bwraps2": [("cellsize", 1.0), ("space", 0.0), ("gain", 2.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "post_bwraps2": [("cellsize", 1.0), ("space", 0.0), ("gain", 2.0), ("inner_twist", 0.0), ("outer_twist", 0.0)],
    "post_rblur": [("strength", 1.0), ("offset", 1.0), ("center_x", 0.0), ("center_y", 1.0)],
    "cpow3_wf": [("r", 1.0), ("a", 0.1), ("divisor", 1.0), ("spread", 1.0), ("discrete_spread", 1.0), ("spread2", 0.0), ("offset2", 1.0)],
    "pre_rect_wf": [("x0", -0.5), ("x1", 0.5), ("y0", -0.5), ("y1", 0.5)],
})
PARAMS.update({
    "spliptic_bs": [("x", 0.05), ("y", 0.05)],
    "pointgrid_wf": [("xmin", -3.0), ("xmax", 3.0), ("xcount", 32.0), ("ymin", -3.0), ("ymax", 3.0), ("ycount", 32.0), ("distortion", 2.3), ("seed", 1234.0)],
    "truchet2": [("exponent1", 1.0), ("exponent2", 2.0), ("width1", 0.5), ("width2", 0.5), ("scale", 10.0), ("seed", 50.0), ("inverse", 0.0)],
    "bubbleT3D": [("number_of_stripes", 0.0), ("ratio_of_stripes", 1.0), ("angle_of_hole", 0.0), ("exponent_z", 1.0), ("symmetry_z", 0.0), ("modus_blur", 0.0)],
    "pRose3D": [("l", 1.0), ("k", 6.0), ("c", 0.0), ("z1", 1.0), ("z2", 1.0), ("refSc", 1.0), ("opt", 1.0), ("optSc", 1.0), ("opt3", 0.0), ("transp", 0.5), ("dist", 1.0), ("wagsc", 0.0), ("srvsc", 0.0), ("f", 3.0), ("wigsc", 0.0), ("offset", 0.0)],
})
PARAMS.update({
    "hypertile3D1": [("p", 3.0), ("q", 7.0)],
    "hypertile3D2": [("p", 3.0), ("q", 7.0)],
    "julian3Dx": [("power", 0.0), ("dist", 1.0), ("a", 1.0), ("b", 0.0), ("c", 0.0), ("d", 1.0), ("e", 0.0), ("f", 0.0)],
    "waves2b": [("freqx", 2.0), ("freqy", 2.0), ("pwx", 1.0), ("pwy", 1.0), ("scalex", 1.0), ("scaleinfx", 1.0), ("scaley", 1.0), ("scaleinfy", 1.0), ("unity", 1.0), ("jacok", 0.25)],
})
PARAMS.update({
    "log_db": [("base", 1.0), ("fix_period", 1.0)],
    "juliaq": [("power", 3.0), ("divisor", 2.0)],
    "julia3Dq": [("power", 3.0), ("divisor", 2.0)],
    "juliac": [("re", 3.0), ("im", 0.5), ("dist", 1.0)],
    "cpow2": [("r", 1.0), ("a", 0.0), ("divisor", 1.0), ("range", 1.0)],
    "post_juliaq": [("power", 3.0), ("divisor", 2.0)],
    "post_julia3Dq": [("power", 3.0), ("divisor", 2.0)],
})
PARAMS.update({
    "cut_sqcir": [("mode", 1.0), ("zoom", 2.0), ("invert", 0.0), ("power", 2.0)],
    "cut_yuebing": [("mode", 1.0), ("zoom", 0.25), ("invert", 0.0), ("p1", 2.0), ("p2", 25.0)],
    "cut_vasarely": [("mode", 1.0), ("zoom", 1.0), ("invert", 0.0), ("size", 0.5)],
    "cut_sincos": [("seed", 1000.0), ("mode", 1.0), ("time", 0.9), ("zoom", 0.5), ("invert", 0.0)],
    "cut_chains": [("shiftX", 0.0), ("shiftY", 0.0), ("mode", 1.0), ("zoom", 2.5), ("invert", 0.0)],
    "cut_hexdots": [("mode", 1.0), ("size", 0.5), ("zoom", 4.0), ("invert", 0.0)],
    "cut_booleans": [("seed", 1000.0), ("mode", 1.0), ("type", 0.0), ("zoom", 250.0), ("invert", 0.0)],
})
PARAMS.update({
    "cut_sqsplits": [("seed", 1000.0), ("mode", 1.0), ("time", 0.9), ("zoom", 2.0), ("invert", 0.0)],
    "cut_btree": [("seed", 0.0), ("time", 1.0), ("thickness", 5.0), ("zoom", 1.0), ("mode", 1.0), ("invert", 1.0)],
    "cut_fractal": [("seed", 0.0), ("mode", 1.0), ("time", 0.0), ("iters", 30.0), ("zoom", 1.0), ("invert", 0.0)],
    "cut_glypho": [("mode", 1.0), ("zoom", 1.0), ("invert", 0.0), ("f1", 0.115), ("f2", 0.75), ("f3", 1.5)],
    "cut_circdes": [("seed", 1000.0), ("mode", 1.0), ("time", 0.0), ("zoom", 10.0), ("invert", 0.0)],
    "cut_snowflake": [("seed", 1000.0), ("mode", 1.0), ("time", 0.0), ("level", 10.0), ("zoom", 10.0), ("invert", 0.0)],
})
PARAMS.update({
    "cut_jigsaw": [("seed", 1000.0), ("time", 0.0), ("mode", 1.0), ("zoom", 4.0), ("invert", 0.0)],
    "cut_rgrid": [("mode", 1.0), ("zoom", 7.0), ("invert", 0.0), ("angle", 0.0)],
    "cut_x": [("mode", 1.0), ("zoom", 1.0), ("invert", 0.0), ("size", 0.1)],
    "cut_metaballs": [("mode", 1.0), ("zoom", 7.0), ("invert", 0.0), ("time", 0.0)],
    "cut_kaleido": [("seed", 1000.0), ("mode", 1.0), ("time", 0.0), ("n", 6.0), ("zoom", 0.5), ("invert", 0.0)],
    "cut_spiral": [("time", 0.0), ("mode", 1.0), ("zoom", 2.5), ("invert", 0.0)],
    "cut_swarp": [("seed", 1000.0), ("mode", 1.0), ("time", 0.0), ("type", 0.0), ("zoom", 1.0), ("invert", 0.0)],
    "cut_apollonian": [("mode", 1.0), ("levels", 4.0), ("zoom", 2.0), ("invert", 0.0)],
    "cut_zigzag": [("mode", 1.0), ("xpar", 1.0), ("ypar", 2.0), ("zoom", 2.0), ("invert", 0.0)],
    "cut_bricks": [("seed", 1000.0), ("mode", 1.0), ("size", 0.9), ("zoom", 3.0), ("invert", 0.0)],
    "cut_web": [("seed", 1000.0), ("time", 0.0), ("mode", 1.0), ("thick", 0.05), ("invert", 1.0)],
    "cut_tileillusion": [("time", 0.0), ("mode", 1.0), ("zoom", 15.0), ("invert", 0.0)],
    "cut_pattern": [("seed", 1000.0), ("mode", 1.0), ("time", 0.9), ("zoom", 0.5), ("invert", 0.0)],
    "cut_celtic": [("mode", 1.0), ("zoom", 5.0), ("invert", 0.0)],
    "cut_hextruchetflow": [("randomize", 0.0), ("mode", 1.0), ("grid", 0.0), ("zoom", 10.0), ("invert", 0.0)],
    "circular": [("angle", 90.0), ("seed", 0.0)],
    "circular2": [("angle", 90.0), ("seed", 0.0), ("xx", 12.9898), ("yy", 78.233)],
    "r_circleblur": [("n", 1.0), ("seed", 0.0), ("dist", 0.5), ("min", 0.1), ("max", 1.0)],
    "hypershift2": [("p", 3.0), ("q", 7.0)],
    "spherecrop": [("radius", 1.0), ("x", 0.0), ("y", 0.0), ("z", 0.0), ("scatter_area", 0.0), ("zero", 1.0)],
    "crop3D": [("left", -1.0), ("top", -1.0), ("floor", -1.0), ("right", 1.0), ("bottom", 1.0), ("ceiling", 1.0),
               ("scatter_area", 0.0), ("zero", 0.0)],
    "pre_boarders2": [("c", 0.4), ("left", 0.65), ("right", 0.35)],
    "splitbrdr": [("x", 0.25), ("y", 0.25), ("px", 0.0), ("py", 0.0)],
    "minkowskope": [("separation", 0.5), ("frequencyx", 1.5), ("frequencyy", 1.0), ("amplitude", 0.5), ("perturbation", 0.3),
                    ("damping", 0.0)],
    "glynnlissa": [("radius", 1.0), ("radius1", 0.5), ("thickness", 1.0), ("phi1", 0.0), ("a", 3.0), ("b", 2.0), ("width", 0.0),
                   ("phase", 0.0), ("scale", 0.71), ("pow", 1.5), ("contrast", 0.5)],
})
PARAMS["pre_subflame_wf"] = PARAMS["subflame_wf"]
SLOTS = 24         # packed parameter row a variation (user + derived)
WORDS = 64         # draw words an iteration

XF_STRIDE = 18


def var_meta(name):
    """(draws, user parameters, derived values, phase 0 pre / 1 normal / 2 post / 3 normal with Feature::Replace)."""
    out = (ctypes.c_int * 4)()
    lib().of_var_meta(ctypes.c_int(REGISTRY[name]), out)
    return tuple(out)


def var_row(name, user=None):
    """The packed parameter row: user parameters (defaults where not given), then the derived values."""
    if user is None:
        user = [d for _, d in PARAMS.get(name, [])]
    u = np.zeros(SLOTS, np.float32)
    u[:len(user)] = user
    row = np.zeros(SLOTS, np.float32)
    lib().of_var_row(ctypes.c_int(REGISTRY[name]), _fp(u), _fp(row))
    return row


def build():
    """Compile the oracle (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.of_probe.restype = ctypes.c_uint64
        L.of_render_filtered.restype = ctypes.c_uint64
        L.of_probe_digest.restype = ctypes.c_uint64
        L.of_render.restype = ctypes.c_uint64
        L.of_ctx_new.restype = ctypes.c_void_p
        L.of_ctx_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.of_ctx_free.argtypes = [ctypes.c_void_p]
        L.of_ctx_run.restype = ctypes.c_uint64
        L.of_ctx_run.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
        L.of_ctx_merge.restype = ctypes.c_int64
        L.of_ctx_merge.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_double)]
        L.of_pcg_hash.restype = ctypes.c_uint32
        L.of_rng_next.restype = ctypes.c_uint32
        L.of_f16_round.restype = ctypes.c_float
        L.of_f16_round.argtypes = [ctypes.c_float]
        L.of_select.argtypes = [ctypes.c_void_p, ctypes.c_float]
        L.of_world_to_pixel.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        _lib = L
    return _lib


class OFlame(ctypes.Structure):
    _fields_ = [
        ("n_xf", ctypes.c_int), ("n_fin", ctypes.c_int), ("n_var", ctypes.c_int),
        ("var_id", ctypes.POINTER(ctypes.c_int)),
        ("xf", ctypes.POINTER(ctypes.c_float)),
        ("var_w", ctypes.POINTER(ctypes.c_float)),
        ("var_p", ctypes.POINTER(ctypes.c_float)),
        ("zoom", ctypes.c_float), ("pan_x", ctypes.c_float), ("pan_y", ctypes.c_float),
        ("cos_r", ctypes.c_float), ("sin_r", ctypes.c_float),
        ("width", ctypes.c_int), ("height", ctypes.c_int),
        ("palette", ctypes.POINTER(ctypes.c_float)), ("pal_n", ctypes.c_int),
        ("sym_kind", ctypes.c_int), ("sym_order", ctypes.c_int),
        ("sym_cx", ctypes.c_float), ("sym_cy", ctypes.c_float), ("sym_distance", ctypes.c_float),
        ("sym_rotation", ctypes.c_float),
        ("xaos", ctypes.POINTER(ctypes.c_float)),
        ("n_sub", ctypes.c_int),
        ("sub_nxf", ctypes.POINTER(ctypes.c_int)),
        ("sub_nfin", ctypes.POINTER(ctypes.c_int)),
        ("n_lnk", ctypes.c_int),
        ("att", ctypes.POINTER(ctypes.c_int)),
        ("color_mode", ctypes.c_int),
        ("speed_factor", ctypes.c_float),
        ("orbit_refresh", ctypes.c_int),
    ]


def walk_splits_orbits(weights, xaos):
    """xaos.rs:66-123: whether the xaos walk (not the first pick) decides
    which closed group of the chain an orbit ends in.  Transitions go where
    weight x xaos > 0 (a row with none goes to transform 0); a closed group
    is a set the chain never leaves; a start is a transform of positive weight."""
    n = len(weights)
    nxt = []
    for i in range(n):
        row = [j for j in range(n) if max(weights[j], 0.0) * xaos[i][j] > 0.0] or [0]
        nxt.append(row)
    reach = []
    for s0 in range(n):
        seen, stack = {s0}, [s0]
        while stack:
            i = stack.pop()
            for j in nxt[i]:
                if j not in seen:
                    seen.add(j)
                    stack.append(j)
        reach.append(seen)
    starts = [i for i in range(n) if weights[i] > 0.0]
    live = set().union(*(reach[i] for i in starts)) if starts else set()
    closed = [i for i in sorted(live)
              if all(i in reach[j] for j in reach[i]) and not any(j < i and i in reach[j] and j in reach[i] for j in range(n))]
    if len(closed) < 2:
        return False
    return any(sum(1 for c in closed if c in reach[i]) > 1 for i in starts)


ATTACH = 32        # a chain's length at most (MAX_ATTACHMENTS_PER_TRANSFORM)


def attachments(flame):
    """Each normal's (linked, final) chains as pool indices
    (gpu/buffers.rs:621-660): a legacy singular final attached to every
    normal, indices past their pool dropped, at most ATTACH kept."""
    nl, fins = len(flame.get("linked_transforms", [])), finals_of(flame)
    legacy = len(flame.get("final_transforms", [])) if flame.get("final_transform") else None
    out = []
    for t in flame["transforms"]:
        fa = [int(a) for a in t.get("final_attachments", [])]
        if legacy is not None and legacy not in fa:
            fa.append(legacy)
        la = [int(a) for a in t.get("linked_attachments", [])]
        out.append(([a for a in la if 0 <= a < nl][:ATTACH], [a for a in fa if 0 <= a < len(fins)][:ATTACH]))
    return out


class TonemapParams(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int), ("exposure", ctypes.c_double), ("gamma", ctypes.c_double),
        ("density_scale", ctypes.c_double), ("bg", ctypes.c_double * 3),
        ("use_curve", ctypes.c_int), ("curve", ctypes.POINTER(ctypes.c_float)),
        ("vibrancy", ctypes.c_double), ("brightness", ctypes.c_double), ("white_level", ctypes.c_double),
        ("prefilter_white", ctypes.c_double), ("bright_adjust", ctypes.c_double),
        ("area", ctypes.c_double), ("sample_density", ctypes.c_double),
        ("saturation", ctypes.c_double), ("hue_shift", ctypes.c_double), ("gamma_threshold", ctypes.c_double),
        ("alpha_blend_low", ctypes.c_double), ("alpha_blend_high", ctypes.c_double),
        ("transparent_mode", ctypes.c_int), ("highlight_mode", ctypes.c_int), ("levels_enabled", ctypes.c_int),
        ("levels_low", ctypes.c_double), ("levels_high", ctypes.c_double), ("levels_gamma", ctypes.c_double),
        ("levels_density", ctypes.c_double),
    ]


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def f32(x):
    return float(np.float32(x))


# ------------------------------------------------------------------ flames --

def ordered_variation_names(t):
    """transforms.rs:668-682: `variation_order` entries first, then registry order."""
    out = []
    for n in t.get("variation_order", []):
        if n in t["variations"] and n not in out:
            out.append(n)
    for n in sorted(REGISTRY, key=REGISTRY.get):
        if n in t["variations"] and n not in out:
            out.append(n)
    for n in t["variations"]:
        if n not in REGISTRY:
            raise ValueError(f"variation `{n}` is not in this oracle's registry")
    return out


def finals_of(flame):
    fins = list(flame.get("final_transforms", []))
    if flame.get("final_transform"):
        fins.append(flame["final_transform"])
    return fins


def subflame_transforms(flame):
    """Each subflame's (normals, finals) (gpu/buffers.rs:230-253)."""
    return [(list(sf.get("transforms", [])), finals_of(sf)) for sf in flame.get("subflames", [])]


def local_order(flame):
    """transforms.rs:2297-2319: normals, linked, finals, then each subflame's; first appearance wins."""
    out = []
    allx = list(flame["transforms"]) + list(flame.get("linked_transforms", [])) + finals_of(flame)
    for nx, fx in subflame_transforms(flame):
        allx += nx + fx
    for t in allx:
        for n in ordered_variation_names(t):
            if n not in out:
                out.append(n)
    return out


def hex_stops(hexs):
    """palette.rs:453-482: `indexed_colors` -> stops at i/255."""
    pos, col = [], []
    for i, h in enumerate(hexs.split(",")):
        pos.append(f32(f32(i) / f32(255.0)))
        col += [f32(int(h[k:k + 2], 16)) / f32(255.0) for k in (0, 2, 4)]
    return np.array(pos, np.float32), np.array(col, np.float32)


def palette_table(cfg):
    pal = cfg.get("palette")
    size = int(cfg.get("palette_size", 256))
    if pal is None:
        # Palette::fire, the config default (palette.rs:148-174; fractal_config.rs default_palette).
        pos = np.array([0.0, 0.25, 0.5, 0.75, 1.0], np.float32)
        col = np.array([0, 0, 0, 0.5, 0, 0, 1.0, 0.3, 0, 1.0, 0.8, 0, 1.0, 1.0, 0.8], np.float32)
    elif "indexed_colors" in pal:
        pos, col = hex_stops(pal["indexed_colors"])
    else:
        pos = np.array([s["position"] for s in pal["stops"]], np.float32)
        col = np.array([c for s in pal["stops"] for c in s["color"]], np.float32)
    out = np.zeros(size * 3, np.float32)
    mode = {"linear": 0, "Linear": 0, "geometric": 1, "Geometric": 1}[cfg.get("palette_squeeze_mode", "linear")]
    lib().of_palette_table(ctypes.c_int(len(pos)), _fp(pos), _fp(col), ctypes.c_int(size),
                           ctypes.c_float(cfg.get("palette_rotation", 0.0)),
                           ctypes.c_int(1 if cfg.get("palette_reverse") else 0), _fp(out), ctypes.c_int(mode),
                           ctypes.c_float(cfg.get("palette_squeeze", 1.0)), ctypes.c_float(cfg.get("palette_squeeze_falloff", 0.5)),
                           ctypes.c_float(cfg.get("palette_log_strength", 0.0)))
    return out


class Flame:
    """A config (dict) flattened for the oracle; keeps its arrays alive."""

    def __init__(self, cfg, width, height):
        flame = cfg["flame"]
        self.names = local_order(flame)
        normals = flame["transforms"]
        links = list(flame.get("linked_transforms", []))
        fins = finals_of(flame)
        subs = subflame_transforms(flame)
        allx = list(normals) + links + fins
        for nx, fx in subs:
            allx += nx + fx
        nv = len(self.names)
        self.var_id = np.array([REGISTRY[n] for n in self.names], np.int32)
        self.xf = np.zeros(len(allx) * XF_STRIDE, np.float32)
        self.var_w = np.zeros(len(allx) * max(nv, 1), np.float32)
        self.var_p = np.zeros(len(allx) * max(nv, 1) * SLOTS, np.float32)
        solo = flame.get("solo_transform")
        for i, t in enumerate(allx):
            post = bool(t.get("post_affine_enabled", False))      # transforms.rs:1542; buffers.rs:467
            # The solo transform (buffers.rs:523-536): the other normals plot nothing.
            opacity = 0.0 if solo is not None and i < len(normals) and i != solo else t.get("opacity", 1.0)
            rec = [t["a"], t["b"], t["c"], t["d"], t["e"], t["f"],
                   t.get("post_a", 1.0), t.get("post_b", 0.0), t.get("post_c", 0.0),
                   t.get("post_d", 1.0), t.get("post_e", 0.0), t.get("post_f", 0.0),
                   1.0 if post else 0.0, t.get("weight", 1.0), t.get("color", 0.5),
                   t.get("color_speed", 0.0), opacity, t.get("direct_color", 0.0)]
            self.xf[i * XF_STRIDE:(i + 1) * XF_STRIDE] = rec
            for v, n in enumerate(self.names):
                self.var_w[i * nv + v] = t["variations"].get(n, 0.0)
                user = [t.get("variation_params", {}).get(f"{n}.{pn}", dflt) for pn, dflt in PARAMS.get(n, [])]
                self.var_p[(i * nv + v) * SLOTS:(i * nv + v + 1) * SLOTS] = var_row(n, user)
        self.palette = palette_table(cfg)
        rot = float(cfg.get("rotation", 0.0))
        s = OFlame()
        s.n_xf, s.n_fin, s.n_var = len(normals), len(fins), nv
        s.var_id = self.var_id.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        s.xf, s.var_w, s.var_p = _fp(self.xf), _fp(self.var_w), _fp(self.var_p)
        s.zoom = cfg.get("zoom", 1.0)
        s.pan_x, s.pan_y = cfg.get("pan_x", 0.0), cfg.get("pan_y", 0.0)
        s.cos_r, s.sin_r = math.cos(rot), math.sin(rot)
        s.width, s.height = width, height
        s.palette, s.pal_n = _fp(self.palette), len(self.palette) // 3
        self.sub_nxf = np.array([len(nx) for nx, _ in subs] or [0], np.int32)
        self.sub_nfin = np.array([len(fx) for _, fx in subs] or [0], np.int32)
        s.n_sub = len(subs)
        s.sub_nxf = self.sub_nxf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        s.sub_nfin = self.sub_nfin.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        att = np.zeros((max(len(normals), 1), 2 + 2 * ATTACH), np.int32)
        for k, (la, fa) in enumerate(attachments(flame)):
            att[k, 0], att[k, 1:1 + len(la)] = len(la), la
            att[k, 1 + ATTACH], att[k, 2 + ATTACH:2 + ATTACH + len(fa)] = len(fa), fa
        self.att = np.ascontiguousarray(att.ravel())
        s.n_lnk = len(links)
        s.color_mode = {"palette": 0, "Palette": 0, "speed": 1, "Speed": 1}[cfg.get("color_mode", "palette")]
        s.speed_factor = cfg.get("speed_factor", 0.5)
        s.att = self.att.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        # Xaos (xaos.rs:29-40, 128-135): read when some weight differs from 1; missing entries are 1.
        self.xaos = None
        if flame.get("xaos"):
            n = len(normals)
            m = np.ones((n, n), np.float32)
            for i, row in enumerate(flame["xaos"]):
                for j, v in enumerate(row):
                    if i < n and j < n:
                        m[i, j] = v
            if any(abs(f32(v) - 1.0) > 1e-6 for row in flame["xaos"] for v in row):
                self.xaos = np.ascontiguousarray(m.ravel())
                s.xaos = _fp(self.xaos)
                if walk_splits_orbits([f32(t.get("weight", 1.0)) for t in normals], m.tolist()):
                    s.orbit_refresh = 4                                    # ORBIT_REFRESH_PERIOD
        ps = flame.get("post_symmetry")
        if ps:
            s.sym_kind = {"none": 0, "xaxis": 1, "yaxis": 2, "point": 3}[ps.get("ty", "none")]
            s.sym_order = int(ps["order"])
            s.sym_cx, s.sym_cy, s.sym_distance = ps["center_x"], ps["center_y"], ps["distance"]
            # f32::to_radians: deg * f32(f32(pi) / 180)
            s.sym_rotation = f32(f32(ps["rotation_deg"]) * f32(f32(math.pi) / f32(180.0)))
        self.s = s
        self.width, self.height = width, height

    @property
    def ptr(self):
        return ctypes.byref(self.s)

    def render(self, walkers, iters, *, seed=12345, seed_hi=0, rng="philox", burn_in=20, ipt=1024,
               threads=1, walker0=0, hist=True, f64=False):
        """The chaos game: (plotted, inframe, counts[h,w] u32, rgb sums[h,w,3] f64)."""
        n = self.width * self.height
        cnt = np.zeros(n, np.uint32) if hist else None
        rgb = np.zeros(n * 3, np.float64) if hist else None
        inframe = ctypes.c_int64(0)
        plotted = lib().of_render(
            self.ptr, ctypes.c_int(0 if rng == "pcg" else 1), ctypes.c_uint32(seed & 0xFFFFFFFF),
            ctypes.c_uint32(seed_hi & 0xFFFFFFFF), ctypes.c_uint32(burn_in), ctypes.c_uint32(ipt),
            ctypes.c_uint32(walker0), ctypes.c_uint32(walkers), ctypes.c_uint64(iters), ctypes.c_int(threads),
            cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)) if hist else None,
            rgb.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if hist else None,
            ctypes.byref(inframe), ctypes.c_int(1 if f64 else 0))
        if not hist:
            return plotted, inframe.value, None, None
        return plotted, inframe.value, cnt.reshape(self.height, self.width), rgb.reshape(self.height, self.width, 3)

    def cpu_render(self, threads):
        """A persistent host render of this flame (CpuRender)."""
        return CpuRender(self, threads)

    def render_filtered(self, walkers, iters, sigma, blur_edges=0.0, *, seed=12345, seed_hi=0, rng="philox", burn_in=20,
                        ipt=1024, threads=1, walker0=0):
        """The chaos game in batches of `ipt` iterations, each batch's
        histogram spatially filtered and summed: (plotted, inframe, [h, w, 4] r, g, b, count)."""
        out = np.zeros((self.height, self.width, 4), np.float32)
        inframe = ctypes.c_int64(0)
        plotted = lib().of_render_filtered(
            self.ptr, ctypes.c_int(0 if rng == "pcg" else 1), ctypes.c_uint32(seed & 0xFFFFFFFF),
            ctypes.c_uint32(seed_hi & 0xFFFFFFFF), ctypes.c_uint32(burn_in), ctypes.c_uint32(ipt),
            ctypes.c_uint32(walker0), ctypes.c_uint32(walkers), ctypes.c_uint64(iters), ctypes.c_int(threads),
            ctypes.c_float(sigma), ctypes.c_float(blur_edges), _fp(out), ctypes.byref(inframe))
        return plotted, inframe.value, out

    def apply_xform(self, xi, xs, ys, draws=None, with_affine=True, scales=False):
        """One step of transform xi; with `scales`, also the magnitude of the
        terms each output component sums (f64), for cancellation-aware tolerances."""
        xs = np.ascontiguousarray(xs, np.float32)
        ys = np.ascontiguousarray(ys, np.float32)
        n = len(xs)
        d = np.zeros(n * WORDS, np.float32) if draws is None else np.ascontiguousarray(draws, np.float32)
        assert d.size == n * WORDS, "draws: WORDS words a point"
        xo, yo = np.zeros(n, np.float32), np.zeros(n, np.float32)
        sx, sy = np.zeros(n, np.float64), np.zeros(n, np.float64)
        P = ctypes.POINTER(ctypes.c_double)
        lib().of_apply_xform(self.ptr, ctypes.c_int(xi), ctypes.c_int(n), _fp(xs), _fp(ys), _fp(d), _fp(xo), _fp(yo),
                             ctypes.c_int(1 if with_affine else 0),
                             sx.ctypes.data_as(P) if scales else None, sy.ctypes.data_as(P) if scales else None)
        return (xo, yo, sx, sy) if scales else (xo, yo)

    def select(self, u):
        return lib().of_select(self.ptr, ctypes.c_float(u))

    def draw_slots(self):
        return lib().of_draw_slots(self.ptr)

    def world_to_pixel(self, x, y):
        px, py = ctypes.c_int(), ctypes.c_int()
        lib().of_world_to_pixel(self.ptr, ctypes.c_float(x), ctypes.c_float(y), ctypes.byref(px), ctypes.byref(py))
        return px.value, py.value


# ------------------------------------------------------------ variations --

def _draws8(draws, n):
    """Draws as 8 words a point: [n] (one draw) or [n, k] (k <= 8)."""
    if draws is None:
        return None
    d = np.asarray(draws, np.float32)
    if d.ndim == 1:
        d = d[:, None]
    out = np.zeros((n, 8), np.float32)
    out[:, :d.shape[1]] = d
    return out


def variation(name, xs, ys, draws=None, params=None, f64=False, ftz=True, w=1.0, xf=None):
    """One variation at n points.  `params` its user parameters (defaults
    if None), `draws` [n] or [n, k] its draws in order, `w` its weight and
    `xf` an affine (a..f) for the bodies that read them."""
    xs = np.ascontiguousarray(xs, np.float32)
    ys = np.ascontiguousarray(ys, np.float32)
    n = len(xs)
    row = var_row(name, params)
    d = _draws8(draws, n)
    x6 = None if xf is None else np.asarray(xf, np.float32)
    xo, yo = np.zeros(n, np.float32), np.zeros(n, np.float32)
    lib().of_variation(ctypes.c_int(REGISTRY[name]), _fp(row), ctypes.c_int(n), _fp(xs), _fp(ys),
                       _fp(d) if d is not None else None, ctypes.c_float(w), _fp(x6) if x6 is not None else None,
                       _fp(xo), _fp(yo), ctypes.c_int(1 if f64 else 0), ctypes.c_int(1 if ftz else 0))
    return xo, yo


def variation_scale(name, xs, ys, draws=None, params=None, w=1.0, xf=None):
    """Per-component tolerance scale of one variation (f64): the magnitude
    of its terms, or its numeric conditioning (variations beyond the first
    twelve)."""
    xs = np.ascontiguousarray(xs, np.float32)
    ys = np.ascontiguousarray(ys, np.float32)
    n = len(xs)
    row = var_row(name, params)
    d = _draws8(draws, n)
    x6 = None if xf is None else np.asarray(xf, np.float32)
    sx, sy = np.zeros(n, np.float64), np.zeros(n, np.float64)
    P = ctypes.POINTER(ctypes.c_double)
    lib().of_variation_scale(ctypes.c_int(REGISTRY[name]), _fp(row), ctypes.c_int(n), _fp(xs), _fp(ys),
                             _fp(d) if d is not None else None, ctypes.c_float(w), _fp(x6) if x6 is not None else None,
                             sx.ctypes.data_as(P), sy.ctypes.data_as(P))
    return sx, sy


def probe(name, xform_slot=None, fold_first=None, report_stream=False):
    """(classes, digest, raw outputs) as src/probe/ reports them.  With
    `report_stream`, the draws come from the stream of the build that wrote
    the reference's committed report (one PCG increment for every thread)."""
    vid = REGISTRY[name]
    slot = vid if xform_slot is None else xform_slot
    fold = (slot == 0) if fold_first is None else fold_first
    prm = var_row(name)
    cls = ctypes.create_string_buffer(64)
    out = np.zeros(54, np.float32)
    dig = lib().of_probe(ctypes.c_int(vid), _fp(prm), ctypes.c_int(slot), ctypes.c_int(1 if fold else 0), cls, _fp(out),
                         ctypes.c_int(1 if report_stream else 0))
    return cls.value.decode(), dig, out


def hist_filter(rgbc, sigma, sigma_d):
    """The spatial filter of one batch ([h, w, 4] r, g, b, count) -> [h, w, 4]."""
    rgbc = np.ascontiguousarray(rgbc, np.float32)
    h, w, _ = rgbc.shape
    out = np.zeros_like(rgbc)
    lib().of_hist_filter(_fp(rgbc), ctypes.c_int(w), ctypes.c_int(h), ctypes.c_float(sigma), ctypes.c_float(sigma_d), _fp(out))
    return out


def probe_draws(slot, k, seed=0x9E3779B9):
    """The first k draws of rng_init(slot, seed) as rng_nextf returns them (the current stream)."""
    st = rng_init(slot, seed)
    return [f32((rng_next(st) >> 8) / 16777216.0) for _ in range(k)]


def probe_draw(slot, seed=0x9E3779B9):
    """The first draw of rng_init(slot, seed) as rng_nextf returns it."""
    st = rng_init(slot, seed)
    return (rng_next(st) >> 8) * (1.0 / 16777216.0)


def probe_digest(vals):
    v = np.ascontiguousarray(vals, np.float32)
    cls = ctypes.create_string_buffer(64)
    dig = lib().of_probe_digest(_fp(v), cls)
    return cls.value.decode(), dig


# ------------------------------------------------------------------- RNG --

def pcg_hash(x):
    return lib().of_pcg_hash(ctypes.c_uint32(x))


def rng_init(tid, seed):
    st = (ctypes.c_uint32 * 2)()
    lib().of_rng_init(ctypes.c_uint32(tid), ctypes.c_uint32(seed), st)
    return st


def rng_next(st):
    return lib().of_rng_next(st)


def philox(k0, k1, ctr):
    c = (ctypes.c_uint32 * 4)(*ctr)
    o = (ctypes.c_uint32 * 4)()
    lib().of_philox(ctypes.c_uint32(k0), ctypes.c_uint32(k1), c, o)
    return list(o)


def f16_round(v):
    return lib().of_f16_round(ctypes.c_float(v))


# ------------------------------------------------------------ tone map ----

def curve_lut_identity():
    """tonemap.rs:289-304 for the linear (identity) curve: f16(i/255)."""
    return np.array([f16_round(f32(i) / f32(255.0)) for i in range(256)], np.float32)


def tonemap_params_for(cfg, w, h, sd, transparent=0):
    """The oracle's tone-map parameters from a config.  The reference's config
    fields are f32 (src/config/fractal_config.rs), so each is rounded to f32
    first, as the product's parser does; everything after is f64."""
    import ctypes
    f = lambda key, d: float(np.float32(cfg.get(key, d)))
    tm = TonemapParams()
    modes = {"linear": 0, "Linear": 0, "logarithmic": 1, "Logarithmic": 1, "density": 2, "DensityVisualization": 2}
    highs = {"clip": 0, "Clip": 0, "max_norm": 1, "MaxNorm": 1, "reinhard": 2, "Reinhard": 2, "filmic": 3, "Filmic": 3,
             "agx": 4, "AgX": 4, "agx_punchy": 5, "AgXPunchy": 5}
    tm.mode = modes[cfg.get("tonemap_mode", "logarithmic")]
    tm.highlight_mode = highs[cfg.get("highlight_mode", "clip")]
    tm.exposure = f("exposure", 1.0)
    tm.gamma = f("gamma", 4.0)
    tm.density_scale = f("density_scale", 1.0)
    bg = cfg.get("background_color", [0, 0, 0])
    for k in range(3):
        tm.bg[k] = float(np.float32(bg[k]))
    tm.use_curve = 1 if cfg.get("use_curve", True) else 0
    lut = curve_lut_identity()
    tm._lut = lut
    tm.curve = lut.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    tm.vibrancy = f("vibrancy", 1.0)
    tm.brightness = f("brightness", 4.0)
    tm.white_level = f("white_level", 200.0)
    tm.prefilter_white = 67108864.0
    tm.bright_adjust = 2.3
    ppu = min(w, h) * 0.25 * f("zoom", 1.0)
    tm.area = w * h / (ppu * ppu)
    tm.sample_density = sd
    tm.saturation = f("saturation", 1.0)
    tm.hue_shift = f("hue_shift", 0.0)
    tm.gamma_threshold = f("gamma_threshold", 5.0)
    tm.alpha_blend_low = f("alpha_blend_low", 0.3)
    tm.alpha_blend_high = f("alpha_blend_high", 0.8)
    tm.transparent_mode = transparent
    tm.levels_enabled = 1 if cfg.get("levels_enabled", True) else 0
    tm.levels_low = f("levels_low", 0.0)
    tm.levels_high = f("levels_high", 10.0)
    tm.levels_gamma = f("levels_gamma", 0.5)
    tm.levels_density = float(np.float32(sd))
    return tm


def tonemap(params, cnt, rgb):
    """Double-precision tone map: (float RGBA [n,4], RGBA8 [n,4])."""
    cnt = np.ascontiguousarray(cnt, np.float64).ravel()
    rgb = np.ascontiguousarray(rgb, np.float64).ravel()
    n = len(cnt)
    of = np.zeros(n * 4, np.float64)
    ou = np.zeros(n * 4, np.uint8)
    lib().of_tonemap(ctypes.byref(params), cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                     rgb.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.c_int(n),
                     of.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ou.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return of.reshape(n, 4), ou.reshape(n, 4)


def agx_display(rgb, punchy=False):
    """AgX as the tone map's highlight modes 4 / 5 apply it, display-referred."""
    a = np.ascontiguousarray(rgb, np.float64)
    out = np.zeros(3, np.float64)
    P = ctypes.POINTER(ctypes.c_double)
    lib().of_agx_display(a.ctypes.data_as(P), ctypes.c_int(1 if punchy else 0), out.ctypes.data_as(P))
    return out


def downsample_firefly(rgba, ow, oh):
    src = np.ascontiguousarray(rgba, np.uint8).ravel()
    out = np.zeros(ow * oh * 4, np.uint8)
    lib().of_downsample_firefly(src.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), ctypes.c_int(ow), ctypes.c_int(oh),
                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return out.reshape(oh, ow, 4)


def density_estimate(cnt, rgb, w, h, r_max, r_min=0.0, curve=0.4):
    cnt = np.ascontiguousarray(cnt, np.float64).ravel()
    rgb = np.ascontiguousarray(rgb, np.float64).ravel()
    oc = np.zeros(w * h, np.float64)
    orgb = np.zeros(w * h * 3, np.float64)
    P = ctypes.POINTER(ctypes.c_double)
    lib().of_density_estimate(cnt.ctypes.data_as(P), rgb.ctypes.data_as(P), ctypes.c_int(w), ctypes.c_int(h),
                              ctypes.c_double(r_max), ctypes.c_double(r_min), ctypes.c_double(curve),
                              oc.ctypes.data_as(P), orgb.ctypes.data_as(P))
    return oc.reshape(h, w), orgb.reshape(h, w, 3)


# ------------------------------------------------------------ gradients --

class DiffCfg(ctypes.Structure):
    _fields_ = [
        ("seed_lo", ctypes.c_uint32), ("seed_hi", ctypes.c_uint32), ("burn_in", ctypes.c_uint32),
        ("walker0", ctypes.c_uint32), ("walkers", ctypes.c_uint32), ("iters", ctypes.c_uint64),
        ("window", ctypes.c_int), ("use_f64", ctypes.c_int), ("threads", ctypes.c_int),
    ]


_DP = ctypes.POINTER(ctypes.c_double)


def theta_layout(cfg):
    """(n_xf, variation names) of the differentiable render's theta:
    [n_xf*6 affine | n_xf*n_var weights, transform-major | n_xf colours]."""
    return len(cfg["flame"]["transforms"]), local_order(cfg["flame"])


def theta_of(cfg):
    n, names = theta_layout(cfg)
    t = cfg["flame"]["transforms"]
    aff = [f32(x[k]) for x in t for k in "abcdef"]
    w = [f32(x["variations"].get(v, 0.0)) for x in t for v in names]
    col = [f32(x.get("color", 0.5)) for x in t]
    return np.array(aff + w + col, np.float32)


def with_theta(cfg, theta):
    """A copy of the config with theta's values in place (f32-exact)."""
    import copy
    n, names = theta_layout(cfg)
    out = copy.deepcopy(cfg)
    theta = np.asarray(theta, np.float64)
    for k, x in enumerate(out["flame"]["transforms"]):
        for i, key in enumerate("abcdef"):
            x[key] = float(theta[k * 6 + i])
        x["variations"] = {v: float(theta[n * 6 + k * len(names) + j]) for j, v in enumerate(names)}
        x["color"] = float(theta[n * (6 + len(names)) + k])
    return out


class DiffFlame(Flame):
    """The differentiable render's oracle for one config at one theta."""

    def _cfg(self, walkers, iters, seed, burn_in, window, f64, threads, walker0=0):
        c = DiffCfg()
        c.seed_lo, c.seed_hi, c.burn_in = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF, burn_in
        c.walker0, c.walkers, c.iters = walker0, walkers, iters
        c.window, c.use_f64, c.threads = window, 1 if f64 else 0, threads
        return c

    def render(self, walkers, iters, *, seed=12345, burn_in=20, f64=False, threads=8):
        """(bilinear histogram [h, w, 4] f64, plotted samples)."""
        hist = np.zeros(self.width * self.height * 4, np.float64)
        c = self._cfg(walkers, iters, seed, burn_in, 0, f64, threads)
        lib().of_diff_render.restype = ctypes.c_uint64
        n = lib().of_diff_render(self.ptr, ctypes.byref(c), hist.ctypes.data_as(_DP))
        return hist.reshape(self.height, self.width, 4), n

    def grad(self, dh, walkers, iters, *, seed=12345, burn_in=20, window=16, f64=False, threads=8):
        """dL/dtheta given dL/dhistogram [h, w, 4]."""
        dh = np.ascontiguousarray(dh, np.float64).ravel()
        n_xf = self.s.n_xf
        g = np.zeros(n_xf * (7 + self.s.n_var), np.float64)
        c = self._cfg(walkers, iters, seed, burn_in, window, f64, threads)
        lib().of_diff_grad(self.ptr, ctypes.byref(c), dh.ctypes.data_as(_DP), g.ctypes.data_as(_DP))
        return g


def diff_tonemap(params, hist):
    """Linear-light tone map of a bilinear histogram [..., 4] -> [..., 4]."""
    h = np.ascontiguousarray(hist, np.float64)
    out = np.zeros_like(h)
    lib().of_diff_tonemap(ctypes.byref(params), h.ctypes.data_as(_DP), ctypes.c_int(h.size // 4), out.ctypes.data_as(_DP))
    return out


def diff_tonemap_vjp(params, hist, dimg):
    h = np.ascontiguousarray(hist, np.float64)
    d = np.ascontiguousarray(dimg, np.float64)
    out = np.zeros_like(h)
    lib().of_diff_tonemap_vjp(ctypes.byref(params), h.ctypes.data_as(_DP), d.ctypes.data_as(_DP), ctypes.c_int(h.size // 4),
                              out.ctypes.data_as(_DP))
    return out


def variation_jacobian(name, xs, ys, draws=None, params=None):
    """(vx, vy, J00, J01, J10, J11) [n, 6] by central differences in double."""
    xs = np.ascontiguousarray(xs, np.float32)
    ys = np.ascontiguousarray(ys, np.float32)
    prm = var_row(name, params)
    d = None if draws is None else np.ascontiguousarray(draws, np.float32)
    out = np.zeros(len(xs) * 6, np.float64)
    lib().of_variation_jacobian(ctypes.c_int(REGISTRY[name]), _fp(prm), ctypes.c_int(len(xs)), _fp(xs), _fp(ys),
                                _fp(d) if d is not None else None, out.ctypes.data_as(_DP))
    return out.reshape(-1, 6)


class CpuRender:
    """One frame rendered on the host cores over several calls: a private
    histogram a thread, allocated and zeroed when this is made; `run` adds
    a batch of walkers' samples (the chaos game and its splats, nothing
    else); `merge` sums the threads' histograms.  The benchmark's CPU legs
    time `run` alone."""

    def __init__(self, flame, threads):
        self.flame = flame                       # keeps the flat arrays alive
        self.threads = int(threads)
        self.ptr = lib().of_ctx_new(flame.ptr, self.threads)

    def run(self, walker0, walkers, iters, *, seed=12345, seed_hi=0, rng="philox", burn_in=20, ipt=1024):
        """Plotted samples of walkers [walker0, walker0 + walkers), `iters` iterations each."""
        return lib().of_ctx_run(self.ptr, 0 if rng == "pcg" else 1, seed & 0xFFFFFFFF, seed_hi & 0xFFFFFFFF, burn_in, ipt,
                                walker0, walkers, iters)

    def merge(self):
        """(in-frame splats, counts[h, w] u32, rgb sums[h, w, 3] f64) of every run so far."""
        n = self.flame.width * self.flame.height
        cnt = np.zeros(n, np.uint32)
        rgb = np.zeros(n * 3, np.float64)
        inf = lib().of_ctx_merge(self.ptr, cnt.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                 rgb.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return inf, cnt.reshape(self.flame.height, self.flame.width), rgb.reshape(self.flame.height, self.flame.width, 3)

    def close(self):
        if self.ptr:
            lib().of_ctx_free(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
