"""Writes the golden fixtures of this directory from the reference's own sources.

Run where a NumericDream checkout exists (default /root/reference, or ND_REFERENCE):

    python tests/golden/make_golden.py

* de_reference_fp64.json: FP64 distance estimates of every translatable formula of
  the reference (its formula files and built-in Mandelbulb, with the DE helpers of
  its shader template), evaluated by oracle/_ref (the reference WGSL translated
  mechanically and compiled on the host, see oracle/build_ref.py) at 32 seeded points
  in [-2, 2]^3 per parameter set: the formula's @param defaults, plus the benchmark
  parameter sets for the Mandelbulb, Mandelbox, Menger sponge and pseudo-Kleinian.
* template_consts.json: the values of the shader-template constants that formula
  files may name (template.wgsl module constants).
* march_reference_fp64.json: the reference's own fs_simple primary pass (march_to,
  march_epsilon and tetra_gradient of its shader template, run by oracle/_ref in FP64)
  on 16x16 rays of one view per formula of the benchmarks and per march mode (sphere
  tracing with bisection; high quality with 20 refinements; verify each step): per
  ray hit, t, probe steps, march evaluations and the tetrahedral normal.
* shade_reference_fp64.json: simple_geometry's Lambert level (camera key light) and
  the opaque shadow ray (visibility_march with shadow_factor's parameters) of the
  reference, FP64, on 16x16 rays of four benchmark formulas, with and without a light.
* trap_reference_fp64.json: the reference's generated formula wrapper (formula_N,
  fractal_renderer.zig:490-512, distance LOD off) with its orbit-trap functions
  (template.wgsl:1227-1289), FP64, at 32 seeded points per formula of the benchmarks
  for every trap shape (closest approach) and every trap mode (box shell).
* lite_reference.json: pieces of the reference's lite shading: calc_ao (FP64) at the
  hits of the march fixture's sphere-tracing cases, orbit_trap_to_strip and
  fresnel_schlick (f32) at 600 seeded inputs.
* combine_reference_f32.json: the reference's combine_de (instance combine modes,
  template.wgsl:1708-1730, with smin ... smix) in f32 at 2,800 seeded inputs.
"""

import ctypes as C
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from numericdream_b200 import workloads  # noqa: E402
from numericdream_b200.formula import pack_params, parse_formula_params  # noqa: E402
from numericdream_b200.translator.wgsl import TEMPLATE_CONSTS  # noqa: E402
from oracle import build_ref  # noqa: E402

EXTRA_SETS = {
    "mandelbrot": [workloads.mandelbulb_params(8.0, 12), workloads.mandelbulb_params(5.3, 6)],
    "amazingbox_box": [workloads.mandelbox_params(-1.5, 15), workloads.mandelbox_params(-1.7, 12),
                       [2.0, 0.5, 1.0, 1.0, 12.0, 30.0, -20.0, 10.0, 1.0, 0.1, 0.2, 0.3]],
    "menger3_ifs": [workloads.menger_params(3), workloads.menger_params(6)],
    "pseudokleinian_kleinian": [workloads.pseudo_kleinian_params(0.8), workloads.pseudo_kleinian_params(1.2)],
    "sphere_primitive": [[1.3]],
    "cube_primitive": [[0.7]],
}


MARCH_CASES = [("mandelbrot", workloads.mandelbulb_params(8.0, 12), (0.3, 0.8, -2.4)),
               ("amazingbox_box", workloads.mandelbox_params(-1.5, 15), (0.5, 0.9, -4.0)),
               ("menger3_ifs", workloads.menger_params(4), (0.6, 0.9, -2.7)),
               ("pseudokleinian_kleinian", workloads.pseudo_kleinian_params(1.0), (0.2, 0.3, -2.0)),
               ("sphere_primitive", [1.0], (0.2, 0.3, -3.0)),
               ("cube_primitive", [0.7], (0.6, 0.9, -3.0))]
MARCH_MODES = [{}, {"high_quality": 1, "refine_budget": 20}, {"march_verify": 1, "refine_budget": 3}]


def march_view(params, cam, mode):
    from numericdream_b200 import abi

    return abi.make_view(0, 16, 16, cam, fov_y_deg=60.0, params=params, max_steps=256, **mode)


def write_march(lib):
    lib.ref_trace.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int64, C.c_int64, C.c_void_p]
    cases = []
    for name, params, cam in MARCH_CASES:
        for mode in MARCH_MODES:
            v = march_view(params, cam, mode)
            out = np.zeros((256, 12))
            assert lib.ref_trace(C.addressof(v), name.encode(), 64, 0, 256, out.ctypes.data) == 0
            cases.append({"formula": name, "params": [float(x) for x in params], "camera": list(cam), "mode": mode,
                          "hit": [int(x) for x in out[:, 0]], "t": out[:, 1].tolist(),
                          "steps": [int(x) for x in out[:, 2]], "evals": [int(x) for x in out[:, 3]],
                          "normal": np.round(out[:, 4:7], 8).tolist()})
    with open(os.path.join(HERE, "march_reference_fp64.json"), "w") as fh:
        json.dump({"view": "16x16, fov 60, max_steps 256, make_view defaults otherwise", "cases": cases}, fh,
                  separators=(",", ":"))
    # the Lambert level (simple_geometry's camera key light, which takes the camera's
    # up and right as they are: a 90 degree field of view keeps them unit) and the
    # shadow ray toward a directional light
    from numericdream_b200 import abi

    shade_cases = []
    for name, params, cam in MARCH_CASES[:4]:
        for shadow in (0, 1):
            v = abi.make_view(0, 16, 16, cam, fov_y_deg=90.0, params=params, max_steps=256, shadow=shadow,
                              light_dir=(0.4, 0.8, -0.45) if shadow else (0.0, 0.0, 0.0))
            out = np.zeros((256, 12))
            assert lib.ref_trace(C.addressof(v), name.encode(), 64, 0, 256, out.ctypes.data) == 0
            shade_cases.append({"formula": name, "params": [float(x) for x in params], "camera": list(cam),
                                "shadow": shadow, "hit": [int(x) for x in out[:, 0]],
                                "shade": out[:, 8].tolist(), "visibility": out[:, 9].tolist()})
    with open(os.path.join(HERE, "shade_reference_fp64.json"), "w") as fh:
        json.dump({"view": "16x16, fov 90, max_steps 256; light_dir (0.4, 0.8, -0.45) with a shadow ray",
                   "cases": shade_cases}, fh, separators=(",", ":"))


TRAP_SPECS = [dict(shape=sh, mode=0) for sh in range(5)] + [dict(shape=2, mode=md) for md in range(1, 5)]


def write_trap(lib):
    lib.ref_de_trap.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(7)
    cases = []
    for name, params, _ in MARCH_CASES:
        for spec in TRAP_SPECS:
            trap = np.array([0.1, -0.2, 0.15, spec["shape"], 0.6, 0.5, 0.7, spec["mode"], 0.9, 0.25], np.float32)
            pts = rng.uniform(-1.5, 1.5, (32, 3))
            prm = np.zeros(16, np.float32)
            prm[:len(params)] = params
            out = np.zeros((32, 2))
            assert lib.ref_de_trap(name.encode(), prm.ctypes.data, trap.ctypes.data, 64, 32,
                                   np.ascontiguousarray(pts).ctypes.data, out.ctypes.data) == 0
            cases.append({"formula": name, "params": [float(x) for x in prm], "trap": [float(x) for x in trap],
                          "points": pts.tolist(), "de": out[:, 0].tolist(), "trap_value": out[:, 1].tolist()})
    with open(os.path.join(HERE, "trap_reference_fp64.json"), "w") as fh:
        json.dump({"trap_fields": "center xyz, shape, box xyz, mode, radius, tube", "cases": cases}, fh,
                  separators=(",", ":"))


def write_lite(lib):
    """calc_ao at the hits of the march fixture's default-mode cases; strip and Fresnel
    at seeded inputs."""
    from numericdream_b200 import abi

    lib.ref_ao.argtypes = [C.c_void_p, C.c_char_p, C.c_int64] + [C.c_void_p] * 4
    lib.ref_strip_fresnel.argtypes = [C.c_int64] + [C.c_void_p] * 6
    with open(os.path.join(HERE, "march_reference_fp64.json")) as fh:
        march = json.load(fh)["cases"]
    ao_cases = []
    for c in march:
        if c["mode"]:
            continue
        v = march_view(c["params"], c["camera"], c["mode"])
        hit = np.where(np.array(c["hit"]) == 1)[0][:64]
        idx = np.arange(256)
        px, py = idx % 16, idx // 16
        ux = (2.0 * (px + 0.5) / 16 - 1.0) * 1.0
        uy = -(1.0 - 2.0 * (py + 0.5) / 16)
        d = np.array(v.fwd[:])[None] + np.array(v.right[:])[None] * ux[:, None] + np.array(v.up[:])[None] * uy[:, None]
        d /= np.linalg.norm(d, axis=1)[:, None]
        t = np.array(c["t"])[hit]
        pos = np.array(v.cam_pos[:])[None] + d[hit] * t[:, None]
        nrm = np.array(c["normal"])[hit]
        nrm /= np.linalg.norm(nrm, axis=1)[:, None]
        out = np.zeros(len(hit))
        assert lib.ref_ao(C.addressof(v), c["formula"].encode(), len(hit), np.ascontiguousarray(pos).ctypes.data,
                          np.ascontiguousarray(nrm).ctypes.data, np.ascontiguousarray(t).ctypes.data,
                          out.ctypes.data) == 0
        ao_cases.append({"formula": c["formula"], "params": c["params"], "camera": c["camera"],
                         "pos": pos.tolist(), "normal": nrm.tolist(), "t": t.tolist(), "ao": out.tolist()})
    rng = np.random.default_rng(9)
    n = 600
    sor = np.stack([rng.uniform(0.0, 3.0, n), rng.uniform(-1.0, 1.0, n), rng.integers(0, 3, n)], 1).astype(np.float32)
    sor[::25, 0] = 0.0  # spans below TRAP_MIN_SPAN
    val = rng.uniform(-3.0, 5.0, n).astype(np.float32)
    cosv = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    ior = rng.uniform(1.0, 2.5, n).astype(np.float32)
    st, fr = np.zeros(n, np.float32), np.zeros(n, np.float32)
    lib.ref_strip_fresnel(n, sor.ctypes.data, val.ctypes.data, cosv.ctypes.data, ior.ctypes.data, st.ctypes.data,
                          fr.ctypes.data)
    with open(os.path.join(HERE, "lite_reference.json"), "w") as fh:
        json.dump({"ao": ao_cases, "strip_fresnel": {"span_offset_repeat": sor.tolist(), "v": val.tolist(),
                                                    "cos": cosv.tolist(), "ior": ior.tolist(), "strip": st.tolist(),
                                                    "fresnel": fr.tolist()}}, fh, separators=(",", ":"))


def write_combine(lib):
    lib.ref_combine.argtypes = [C.c_int64] + [C.c_void_p] * 5
    rng = np.random.default_rng(5)
    n = 7 * 400
    mode = np.repeat(np.arange(7, dtype=np.int32), 400)
    d = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    di = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    k = rng.uniform(0.0, 0.6, n).astype(np.float32)
    k[::10] = 0.0        # the hard operations
    k[5::10] = 1e-4      # SMOOTH_K_MIN itself
    out = np.zeros(2 * n, np.float32)
    lib.ref_combine(n, mode.ctypes.data, d.ctypes.data, di.ctypes.data, k.ctypes.data, out.ctypes.data)
    rec = {"mode": mode.tolist(), "d": d.tolist(), "di": di.tolist(), "k": k.tolist(),
           "de": out[0::2].tolist(), "weight": out[1::2].tolist()}
    with open(os.path.join(HERE, "combine_reference_f32.json"), "w") as fh:
        json.dump(rec, fh, separators=(",", ":"))


def main():
    ref = build_ref.reference_root()
    if ref is None:
        raise SystemExit("no reference checkout")
    lib = C.CDLL(build_ref.build())
    lib.ref_formula_name.restype = C.c_char_p
    lib.ref_de.argtypes = [C.c_char_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int]
    names = [lib.ref_formula_name(i).decode() for i in range(lib.ref_formula_count())]
    rng = np.random.default_rng(20261203)
    out = {"points_per_set": 32, "formulas": {}}
    for name in names:
        path = (os.path.join(ref, "src", "gpu", "shaders", "mandelbrot.wgsl") if name == "mandelbrot"
                else os.path.join(ref, "formulas", name + ".wgsl"))
        with open(path, encoding="utf-8") as fh:
            src = fh.read()
        sets = [pack_params(parse_formula_params(src))] + [list(s) + [0.0] * (16 - len(s)) for s in EXTRA_SETS.get(name, [])]
        entries = []
        for prm in sets:
            pts = rng.uniform(-2.0, 2.0, (32, 3))
            p32 = np.asarray(prm, np.float32)
            de = np.zeros(32)
            assert lib.ref_de(name.encode(), p32.ctypes.data, 32, np.ascontiguousarray(pts).ctypes.data,
                              de.ctypes.data, 64) == 0
            entries.append({"params": [float(x) for x in p32], "points": pts.tolist(), "de": de.tolist()})
        out["formulas"][name] = entries
    with open(os.path.join(HERE, "de_reference_fp64.json"), "w") as fh:
        json.dump(out, fh, separators=(",", ":"))
    # template constants a formula may name, as the template defines them
    with open(os.path.join(ref, "src", "gpu", "shaders", "template.wgsl"), encoding="utf-8") as fh:
        tpl = fh.read()
    consts = {}
    for name in TEMPLATE_CONSTS:
        m = re.search(r"^const\s+" + name + r"(?:\s*:\s*\w+)?\s*=\s*([^;]+);", tpl, re.M)
        if m:
            consts[name] = m.group(1).strip()
    with open(os.path.join(HERE, "template_consts.json"), "w") as fh:
        json.dump(consts, fh, indent=1, sort_keys=True)
    write_march(lib)
    write_combine(lib)
    write_trap(lib)
    write_lite(lib)
    print(f"{len(names)} formulas, {sum(len(v) for v in out['formulas'].values())} parameter sets, "
          f"{len(MARCH_CASES) * len(MARCH_MODES)} march cases")


if __name__ == "__main__":
    main()
