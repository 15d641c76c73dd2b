"""Generate the golden images used by the parity tests.

Cases on a dump run the reference's iharm build; cases whose "dump" is the
name of a known-answer model (analytic, sphere) run the reference built with
that model (oracle/_ref/ipole_<model>, no dump; ``make -C oracle plugins REF=<checkout>``)
and take their noise floor from its FMA build (ipole_<model>_fma).

Each case runs the reference ipole itself (oracle/_ref/ipole_nofma: the
reference sources built with -O2 -ffp-contract=off, see oracle/Makefile) on a
seeded synthetic iharm FMKS dump and stores its image arrays in
tests/golden/<case>.npz together with the command-line arguments and the
sha256 of the dump's primitives (the dump is regenerated on demand from its
seed, so the tests check the hash before comparing) and the reference's own
noise floor: how far its other legal builds (oracle/Makefile targets ref and
noise) land from this one, per test metric.  The other builds are sampled
as NOISE_RUNS lists them: the makefile's -O3 build, -O2 with FMA
contraction, -O3 for AVX-512, and three independent "other libms" (the ulp
shim with IPG_ULP_SALT 0, 1, 2), each without and with FMA contraction.

    python tests/golden/make_golden.py [case ...]
    python tests/golden/make_golden.py --floor [case ...]   # floors only: runs
        the realizations a stored golden's floor lacks and merges them in
    python tests/golden/make_golden.py --refloor [case ...]  # floors only,
        every realization again (after a change of the metrics)

Needs the reference builds (``make -C oracle ref noise REF=<checkout>``), i.e. the reference tree.
"""
from __future__ import annotations

import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ipole_b200 import ipgc, synthdump  # noqa: E402

# dump name -> (n1, n2, n3, seed)
DUMPS = {"c1": (128, 64, 64, 1), "c2": (288, 128, 128, 1)}

BASE = ["--freqcgs=230.e9", "--thetacam=163", "--phicam=0", "--rotcam=0", "--MBH=6.5e9", "--dsource=16.8e6",
        "--fov=160", "--trat_large=20", "--trat_small=1"]

# case -> (dump, extra args).  Sizes are small so the reference finishes in seconds.
CASES = {
    "c1_thin_32": ("c1", ["--M_unit=1e25", "--nx=32", "--ny=32"]),
    "c1_bright_32": ("c1", ["--M_unit=3e27", "--nx=32", "--ny=32"]),
    "c1_thick_24": ("c1", ["--M_unit=9e28", "--nx=24", "--ny=24"]),
    "c1_faraday_24": ("c1", ["--M_unit=3e27", "--trat_large=160", "--nx=24", "--ny=24"]),
    "c1_pandya_24": ("c1", ["--M_unit=3e27", "--emission_type=1", "--nx=24", "--ny=24"]),
    "c1_unpol_24": ("c1", ["--M_unit=3e27", "-unpol", "--nx=24", "--ny=24"]),
    "c1_refine_32": ("c1", ["--M_unit=3e27", "--nx=32", "--ny=32", "--nx_min=8", "--ny_min=8",
                            "--refine_abs=2e-2", "--refine_rel=1e-2"]),
    "c1_refine_odd_33": ("c1", ["--M_unit=3e27", "--nx=33", "--ny=33", "--nx_min=9", "--ny_min=9"]),
    "c1_incl17_rot_24": ("c1", ["--M_unit=3e27", "--thetacam=17", "--rotcam=30", "--qu_conv=1", "--nx=24",
                                "--ny=24"]),
    "c1_subring1_16": ("c1", ["--M_unit=3e27", "--target_nturns=1", "--nx=16", "--ny=16"]),
    "c1_counterjet_16": ("c1", ["--M_unit=3e27", "--counterjet=1", "--nx=16", "--ny=16"]),
    "c1_xoff_floors_16": ("c1", ["--M_unit=3e27", "--xoff=0.3", "--yoff=-0.2", "--stokes_floors=1",
                                 "--eps=0.02", "--nx=16", "--ny=20"]),
    # the production dump shape (288x128x128, seed 1) at both inclinations and
    # both R_high of the 400x400 workload, on small images
    "c2_rhigh1_incl17_24": ("c2", ["--M_unit=7.5e27", "--trat_large=1", "--thetacam=17", "--nx=24", "--ny=24"]),
    "c2_rhigh160_incl163_24": ("c2", ["--M_unit=7.5e27", "--trat_large=160", "--nx=24", "--ny=24"]),
    # the full-size workloads: the 128x64x64 dump's own 128x128 image, and the
    # production dump at its four (inclination, R_high) pairs with M_unit set
    # for a total flux of 0.6 Jy (tests/golden/tune_munit.py) -- the 400x400
    # bench image itself and the other three at 128x128
    "c1_full_128": ("c1", ["--M_unit=1e25", "--nx=128", "--ny=128"]),
    "c2_rhigh160_incl163_400": ("c2", ["--M_unit=7.96e27", "--trat_large=160", "--nx=400", "--ny=400"]),
    "c2_rhigh1_incl163_128": ("c2", ["--M_unit=3.05e26", "--trat_large=1", "--nx=128", "--ny=128"]),
    "c2_rhigh160_incl17_128": ("c2", ["--M_unit=7.97e27", "--trat_large=160", "--thetacam=17", "--nx=128",
                                      "--ny=128"]),
    "c2_rhigh1_incl17_128": ("c2", ["--M_unit=3.05e26", "--trat_large=1", "--thetacam=17", "--nx=128",
                                    "--ny=128"]),
}
# cases stored without tau and the tauF channel (the parity metrics use
# neither), to keep the 400x400 fixture at 6.4 MB
SLIM = {"c2_rhigh160_incl163_400"}


# known-answer models: the reference test's parameters (tests/analytic/analytic.par,
# tests/isothermal_sphere/info) at sizes the reference finishes in seconds
ANALYTIC = ["--plugin=analytic", "--emission_type=10", "--rcam=1000", "--thetacam=60", "--phicam=0", "--dx=30",
            "--dy=30", "--dsource=7778", "--freqcgs=230.e9", "--MBH=4.063e6"]
SPHERE = ["--plugin=sphere", "--dsource=8000", "--fov=1200"]
PLUGIN_CASES = {
    **{f"analytic_m{m}_32": ("analytic", [*ANALYTIC, f"--model={m}", "--nx=32", "--ny=32"]) for m in range(1, 6)},
    "sphere_f223_i90_32": ("sphere", [*SPHERE, "--freqcgs=223005000000.0", "--thetacam=90", "--nx=32", "--ny=32"]),
    "sphere_f49_i90_32": ("sphere", [*SPHERE, "--freqcgs=49731200000.0", "--thetacam=90", "--nx=32", "--ny=32"]),
    "sphere_f223_i30_32": ("sphere", [*SPHERE, "--freqcgs=223005000000.0", "--thetacam=30", "--nx=32", "--ny=32"]),
    "sphere_pandya_24": ("sphere", [*SPHERE, "--freqcgs=106682000000.0", "--thetacam=60", "--emission_type=1",
                                    "--nx=24", "--ny=24"]),
}
PLUGINS = ("analytic", "sphere")
CASES.update(PLUGIN_CASES)

# check mode (-check, src/main.c:538-575, src/io.c:193-227): the reference
# writes the image, then a -check run appends the check/recheck blocks to it
CHECK_CASES = {
    "check_c1_48": ("c1", ["--M_unit=3e27", "--nx=48", "--ny=44"]),
    "check_c1_unpol_40": ("c1", ["--M_unit=3e27", "-unpol", "--nx=40", "--ny=40"]),
}
CASES.update(CHECK_CASES)
CHECK_KEYS = ("unpol", "tau", "pol")

# trace output (dump_var_along, src/io.c:279-543) of one pixel; the arrays
# kept are the ray's rows 0..nstep of each per-step dataset
TRACE_CASES = {
    "trace_c1_32_p14_17": ("c1", ["--M_unit=3e27", "--nx=32", "--ny=32", "--trace=1", "--trace_i=14",
                                  "--trace_j=17"]),
    "trace_c1_unpol_24_p11_12": ("c1", ["--M_unit=3e27", "-unpol", "--nx=24", "--ny=24", "--trace=1",
                                        "--trace_i=11", "--trace_j=12"]),
}
CASES.update(TRACE_CASES)


# the realizations of the reference's noise floor: (name recorded in the
# golden, binary in oracle/_ref, IPG_ULP_SALT or None)
NOISE_RUNS = [("ipole", "ipole", None), ("ipole_o2fma", "ipole_o2fma", None), ("ipole_v4", "ipole_v4", None),
              ("ipole_ulp", "ipole_ulp", None), ("ipole_ulpfma", "ipole_ulpfma", None),
              ("ipole_ulp:1", "ipole_ulp", "1"), ("ipole_ulpfma:1", "ipole_ulpfma", "1"),
              ("ipole_ulp:2", "ipole_ulp", "2"), ("ipole_ulpfma:2", "ipole_ulpfma", "2")]


def run_env(salt):
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))
    env.pop("IPG_ULP_SALT", None)
    if salt is not None:
        env["IPG_ULP_SALT"] = salt
    return env


REDO = False  # --refloor: recompute floors from every realization


def make_trace_case(case, binary, tmpdir, dumps, skip=()):
    dname, extra = CASES[case]
    dpath, dhash = dumps[dname]
    env = dict(os.environ, OMP_NUM_THREADS=os.environ.get("OMP_NUM_THREADS", "8"))

    def run(bin_name, salt=None):
        tr = os.path.join(tmpdir, f"{case}_{bin_name}_{salt}_trace.ipgc")
        out = os.path.join(tmpdir, f"{case}_{bin_name}_{salt}.ipgc")
        if os.path.exists(tr):
            os.remove(tr)
        r = subprocess.run([os.path.join(os.path.dirname(binary), bin_name), f"--dump={dpath}", *BASE, *extra,
                            f"--trace_outf={tr}", f"--outfile={out}"], capture_output=True, text=True,
                           env=run_env(salt))
        if r.returncode != 0:
            raise RuntimeError(f"{case}: {bin_name} exited {r.returncode}\n{r.stderr[-2000:]}")
        t = ipgc.read(tr)
        n = int(t["/nstep"][0, 0])
        return n, {k[1:]: v[0, 0, :n + 1] for k, v in t.items() if isinstance(v, np.ndarray) and v.ndim >= 3}

    if skip:
        # floors only: the stored golden is the no-FMA build's output
        meta0, rec = load_stored(case)
        n = meta0["nstep"]
        floor, used = dict(meta0["ref_noise_floor"]), list(meta0["ref_noise_builds"])
    else:
        n, rec = run("ipole_nofma")
        floor, used = {}, []
    # per dataset: the largest deviation of the other builds, relative to the
    # dataset's largest magnitude along the ray
    for name, other, salt in NOISE_RUNS:
        if name in used or not os.path.exists(os.path.join(os.path.dirname(binary), other)):
            continue
        n2, rec2 = run(other, salt)
        if n2 != n:
            floor["nstep_differs"] = 1.0
            continue
        for k, v in rec.items():
            sc = float(np.max(np.abs(v))) or 1.0
            floor[k] = max(floor.get(k, 0.0), float(np.max(np.abs(rec2[k] - v))) / sc)
        used.append(name)
    meta = {"case": case, "dump": dname, "dump_shape_seed": DUMPS[dname], "dump_sha256": dhash,
            "args": [*BASE, *extra], "nstep": n, "trace": True,
            "generator": "oracle/_ref/ipole_nofma (reference sources, -O2 -ffp-contract=off)",
            "ref_noise_floor": floor, "ref_noise_builds": used}
    np.savez_compressed(os.path.join(HERE, f"{case}.npz"), meta=json.dumps(meta), **rec)
    print(case, "nstep", n, "floor", {k: f"{v:.1e}" for k, v in floor.items()})


def run_checked(binary, args, out, env):
    """the reference's check run: normal image first, then -check appends"""
    r = subprocess.run([binary, *args], capture_output=True, text=True, env=env)
    if r.returncode != 0:
        return r
    return subprocess.run([binary, *args, "-check"], capture_output=True, text=True, env=env)


def dump_path(name: str, tmpdir: str) -> tuple[str, str]:
    n1, n2, n3, seed = DUMPS[name]
    path = os.path.join(tmpdir, f"dump_{name}.ipgc")
    h = synthdump.write_iharm_dump(path, n1, n2, n3, seed=seed)
    return path, h


def load_stored(case):
    z = np.load(os.path.join(HERE, f"{case}.npz"))
    return json.loads(str(z["meta"])), {k: z[k] for k in z.files if k != "meta"}


def make_case(case: str, binary: str, tmpdir: str, dumps: dict, floor_only: bool = False) -> None:
    dname, extra = CASES[case]
    out = os.path.join(tmpdir, f"{case}.ipgc")
    if dname in PLUGINS:
        binary = os.path.join(os.path.dirname(binary), f"ipole_{dname}")
        base, dhash, others = [], None, [(f"ipole_{dname}_fma", f"ipole_{dname}_fma", None)]
        args = [*extra, f"--outfile={out}"]
    else:
        dpath, dhash = dumps[dname]
        base, others = BASE, NOISE_RUNS
        args = [f"--dump={dpath}", *BASE, *extra, f"--outfile={out}"]
    env = run_env(None)
    check = case in CHECK_CASES
    if floor_only:
        # the stored golden is the no-FMA build's output; only the missing
        # realizations of the floor run
        meta0, rec = load_stored(case)
        img = None
    else:
        r = run_checked(binary, args, out, env) if check else subprocess.run([binary, *args], capture_output=True,
                                                                              text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"{case}: reference exited {r.returncode}\n{r.stderr[-2000:]}")
        img = ipgc.read(out)
        if check:
            # the check block is compared like an image; the recheck block rides along
            img = {**img, "/unpol": img["/unpol_check"], "/tau": img["/tau_check"],
                   **({"/pol": img["/pol_check"]} if "/pol_check" in img else {})}
        rec = {"unpol": img["/unpol"], "tau": img["/tau"]}
        if "/pol" in img:
            rec["pol"] = img["/pol"]
        if case in SLIM:
            del rec["tau"]
            rec["pol"] = np.ascontiguousarray(rec["pol"][..., :4])
        if check:
            for k in CHECK_KEYS:
                if f"/{k}_recheck" in img:
                    rec[f"{k}_recheck"] = img[f"/{k}_recheck"]
    # the reference's own noise floor: the largest deviation from this
    # -ffp-contract=off build among the other legal builds of the same sources
    # (NOISE_RUNS; oracle/Makefile targets ref and noise), in the metrics the
    # tests use
    from tests.common import image_errors
    floor, used = None, []
    if floor_only and not REDO:
        floor, used = dict(meta0["ref_noise_floor"]), list(meta0["ref_noise_builds"])
    for name, other_bin, salt in others:
        path = os.path.join(os.path.dirname(binary), other_bin)
        if name in used or not os.path.exists(path):
            continue
        out2 = os.path.join(tmpdir, f"{case}_{other_bin}_{salt}.ipgc")
        oargs = [*args[:-1], f"--outfile={out2}"]
        oenv = run_env(salt)
        r = run_checked(path, oargs, out2, oenv) if check else subprocess.run([path, *oargs], capture_output=True,
                                                                              text=True, env=oenv)
        if r.returncode != 0:
            continue
        other = ipgc.read(out2)
        if check:
            other = {"/unpol": other["/unpol_check"], "/pol": other.get("/pol_check")}

        class _Img:
            unpol = other["/unpol"]
            pol = other.get("/pol")
        e = image_errors(_Img, rec)
        floor = e if floor is None else {k: max(floor.get(k, 0.0), e[k]) for k in e}
        used.append(name)
        print(f"  {case} {name}: " + " ".join(f"{k} {e[k]:.1e}" for k in ("Ftot", "totQ", "EVPA_deg") if k in e),
              flush=True)
    if floor_only:
        if not used:
            print(case, "no other build available: floor unchanged")
            return
        meta0.update(ref_noise_floor=floor, ref_noise_builds=used)
        np.savez_compressed(os.path.join(HERE, f"{case}.npz"), meta=json.dumps(meta0), **rec)
        print(case, "floor updated from", len(used), "builds")
        return
    meta = {"case": case, "dump": dname, "dump_shape_seed": DUMPS.get(dname), "dump_sha256": dhash,
            "args": [*base, *extra], "Ftot_unpol": float(img["/Ftot_unpol"]),
            "Ftot": float(img["/Ftot"]) if "/Ftot" in img else None, "scale": float(img["/header/scale"]),
            "check": check,
            "generator": f"oracle/_ref/{os.path.basename(binary)} (reference sources, -O2 -ffp-contract=off)",
            "ref_noise_floor": floor, "ref_noise_builds": used}
    np.savez_compressed(os.path.join(HERE, f"{case}.npz"), meta=json.dumps(meta), **rec)
    print(case, "Ftot", meta["Ftot"], "Ftot_unpol", meta["Ftot_unpol"])


def main(cases, floor_only=False):
    binary = os.path.join(ROOT, "oracle", "_ref", "ipole_nofma")
    if not os.path.exists(binary):
        raise SystemExit("build the reference first: make -C oracle ref REF=<reference checkout>")
    with tempfile.TemporaryDirectory() as td:
        dumps = {}
        for c in cases:
            d = CASES[c][0]
            if d not in dumps and d not in PLUGINS:
                dumps[d] = dump_path(d, td)
            if c in TRACE_CASES:
                make_trace_case(c, binary, td, dumps, skip=floor_only)
            else:
                make_case(c, binary, td, dumps, floor_only=floor_only)


if __name__ == "__main__":
    argv = sys.argv[1:]
    fo = "--floor" in argv or "--refloor" in argv
    REDO = "--refloor" in argv
    argv = [a for a in argv if a not in ("--floor", "--refloor")]
    main(argv or list(CASES), floor_only=fo)
