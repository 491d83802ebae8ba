"""Generate the golden fixtures of the parity tests from the reference itself.

Each case writes a seeded synthetic field (barbie_b200.synth) in the reference's
input format, runs the reference estimator program oracle/_ref/barbie_ref --
compiled by oracle/Makefile from the reference's own barbie.c/funcs.c with the
FFTW-API shim, printing %.17e instead of %e/%f -- in a scratch directory, and
stores its 16 output files as one small .npz:

  rows   float64[n, 7]: ii, k1 bin, t bin, mu bin, multipole value (column 4),
         normalisation / NN^2 (column 6), analytic bispectrum (column 5)
  field_sha256, and the configuration.

Column 5 accumulates the analytic bispectrum (barbie.c:300-305,361,391) in an
array the reference never initialises (barbie.c:87); in a fresh process the
stack pages under it are zero, so its values are reproducible run to run, and
the oracle's zero-initialised restatement is checked against them.

pk_<case>.npz holds the reference's power-spectrum multipoles of the same field
(calpow_mom.c with funcs.c:860-1074, built as oracle/_ref/calpow_ref, printing
%.17e): pk float64[n, 6] = k, P0, P2, P4, P6, mode count of the printed bins.

field_<case>.npz holds the r2c buffer written by the reference's field
generator (generate_field.c + ngrf_2d_funcs.c, built unmodified as
oracle/_ref/field_ref against the FFTW shim and the GSL stand-in, whose normal
deviates are the Philox stream of oracle/philox_normal.h): r2c
float64[NN][NN][NN+2] and the printed sigma.

oracle_<case>.npz holds the raw bin sums of cases at the benchmark's and the
serving form's sizes, where the reference program would need its 9-21 GB disk
cache and hours of its single-threaded loop: the oracle's restatement
(oracle/beam_oracle.c, orc_estimate_ex, pixel sums over the plane-ring
transforms as barbie.c:315-337 in pixel order, each accumulated in long double
so that the oracle's own rounding stays far below the 1e-10 bar where bins
cancel by ~1e5, threaded over triangles) -- pinned to the reference program
on the cases above -- gives
  bs, norm, ana  float64[n_k1bin][n_mtbin][n_mtbin][16]: bin_BS_real,
                 bin_normalization and the analytic sum before barbie.c:390
  counts         int64[n_k1bin][n_mtbin][n_mtbin]: closed triangles with B != 0
  field_sha256, the configuration and the oracle's wall time.

Usage: python tests/golden/make_golden.py [--pk | --field | --oracle] [case ...]
(default: all reference cases; --pk makes only the pk_<case>.npz files, --field
only the field ones, --oracle the oracle_<case>.npz ones). Needs the reference
sources (to build oracle/_ref) -- run where they exist; --oracle needs only the
oracle library, RAM for the plane-ring arrays (9.4 GB at NN=384, 21 GB at
NN=512) and takes minutes per case on 8 cores.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from barbie_b200.synth import realization_seed, synth_field, write_field  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "barbie_ref")
PK_BIN = os.path.join(ROOT, "oracle", "_ref", "calpow_ref")
FIELD_BIN = os.path.join(ROOT, "oracle", "_ref", "field_ref")

# name: (NN, realization) of the generator fixtures; 24 = 2^3 * 3 takes a radix-3 stage
FIELD_CASES = {"n16_r1": (16, 1), "n24_r3": (24, 3)}

# name: (NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, realization)
CASES = {
    # the CPU-runnable case: NN=64, Nmax=16, Nr=10, bins 1..11 width 1
    "nn64_cfg1": (64, 16, 10, 11, 1, 1, 1),
    # same geometry, other realization, wider bins and an offset k1 range
    "nn64_bw2": (64, 16, 10, 13, 3, 2, 2),
    # radix-3 grid, 20 rings in two blocks of widths 1 and 2
    "nn96_r20": (96, 32, 20, 21, 1, 1, 3),
    # the drop-in comparison case: NN=256, Nmax=64, Nr=30, bins 1..31 width 1
    "nn256_cfg2": (256, 64, 30, 31, 1, 1, 1),
}

# name: (NN, Nmax, Nr, UL_k1, LL_k1, BW_k1, realization) of the oracle fixtures
ORACLE_CASES = {
    # the benchmark workload `barbie 384 1 51 1 1` on the benchmark's first field
    "nn384_cfg3": (384, 100, 40, 51, 1, 1, 1),
    # served shapes: NN=192 with 30 rings to 60 and k1 bins of width 2 over
    # 1..61; NN=512 with 40 rings to 128, k1 bins 1..31 (of 1..129)
    "nn192_serve": (192, 60, 30, 61, 1, 2, 4),
    "nn512_serve": (512, 128, 40, 31, 1, 1, 5),
}


def run_case(name: str, scratch: str) -> str:
    NN, Nmax, Nr, UL, LL, BW, r = CASES[name]
    work = os.path.join(scratch, name)
    shutil.rmtree(work, ignore_errors=True)
    os.makedirs(os.path.join(work, f"ResFiles_N{NN}", "data_files"))
    field = synth_field(NN, realization_seed(r))
    write_field(os.path.join(work, f"field_N{NN}_R{r}.txt"), field)
    env = dict(os.environ, BEAM_REF_NMAX=str(Nmax), BEAM_REF_NR=str(Nr))
    t = time.time()
    with open(os.path.join(work, "run.log"), "w") as log:
        subprocess.run(["bash", "-c", f"ulimit -s unlimited; exec {REF_BIN} {NN} {r} {UL} {LL} {BW}"],
                       cwd=work, env=env, stdout=log, stderr=subprocess.STDOUT, check=True)
    rows = []
    for ii in range(16):
        path = os.path.join(work, f"ResFiles_N{NN}", f"BS_test_ii{ii}_N{NN}_R{r}.txt")
        with open(path) as fh:
            for line in fh:
                f = line.split()
                rows.append([ii, int(f[0]), int(f[1]), int(f[2]), float(f[3]), float(f[5]), float(f[4])])
    out = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(out, rows=np.array(rows, dtype=np.float64),
                        field_sha256=hashlib.sha256(field.tobytes()).hexdigest(),
                        config=np.array([NN, Nmax, Nr, UL, LL, BW, r], dtype=np.int64))
    shutil.rmtree(work, ignore_errors=True)
    print(f"{name}: {len(rows)} rows in {time.time() - t:.1f} s -> {out}")
    return out


def run_pk_case(name: str, scratch: str) -> str:
    NN, r = CASES[name][0], CASES[name][6]
    work = os.path.join(scratch, "pk_" + name)
    shutil.rmtree(work, ignore_errors=True)
    os.makedirs(os.path.join(work, f"ResFiles_N{NN}", "data_files"))
    field = synth_field(NN, realization_seed(r))
    write_field(os.path.join(work, f"ResFiles_N{NN}", "data_files", f"field_N{NN}_R{r}.txt"), field)
    with open(os.path.join(work, "run.log"), "w") as log:
        subprocess.run([PK_BIN, str(NN), str(r)], cwd=work, stdout=log, stderr=subprocess.STDOUT, check=True)
    pk = np.loadtxt(os.path.join(work, f"ResFiles_N{NN}", f"psoutN{NN}_R{r}.dat"), ndmin=2)
    out = os.path.join(HERE, f"pk_{name}.npz")
    np.savez_compressed(out, pk=pk, field_sha256=hashlib.sha256(field.tobytes()).hexdigest(),
                        config=np.array([NN, r], dtype=np.int64))
    shutil.rmtree(work, ignore_errors=True)
    print(f"pk_{name}: {len(pk)} bins -> {out}")
    return out


def run_field_case(name: str, scratch: str) -> str:
    NN, r = FIELD_CASES[name]
    work = os.path.join(scratch, "field_" + name)
    shutil.rmtree(work, ignore_errors=True)
    os.makedirs(os.path.join(work, f"ResFiles_N{NN}", "data_files"))
    res = subprocess.run([FIELD_BIN, str(NN), str(r)], cwd=work, capture_output=True, text=True, check=True)
    sigma = float(res.stdout.split("sigma =")[1].split()[0])
    r2c = np.fromfile(os.path.join(work, f"ResFiles_N{NN}", "data_files", f"field_N{NN}_R{r}.txt"))
    out = os.path.join(HERE, f"field_{name}.npz")
    np.savez_compressed(out, r2c=r2c.reshape(NN, NN, NN + 2), sigma=sigma, config=np.array([NN, r], dtype=np.int64))
    shutil.rmtree(work, ignore_errors=True)
    print(f"field_{name}: sigma {sigma} -> {out}")
    return out


def run_oracle_case(name: str, save_B: str | None = None) -> str:
    from oracle import oracle_py
    NN, Nmax, Nr, UL, LL, BW, r = ORACLE_CASES[name]
    field = synth_field(NN, realization_seed(r))
    t = time.time()
    res = oracle_py.estimate(field, NN, Nmax, Nr, UL, LL, BW, want_B=save_B is not None, wide=True)
    secs = time.time() - t
    out = os.path.join(HERE, f"oracle_{name}.npz")
    np.savez_compressed(out, bs=res["bs"], norm=res["norm"], ana=res["ana"], counts=res["counts"],
                        field_sha256=hashlib.sha256(field.tobytes()).hexdigest(),
                        config=np.array([NN, Nmax, Nr, UL, LL, BW, r], dtype=np.int64), seconds=secs)
    if save_B:  # per-triangle sums in loop order (large; not a committed fixture)
        np.save(save_B, res["B"])
    print(f"oracle_{name}: {int((res['norm'][..., 0] > 0.1).sum())} printed bins in {secs:.1f} s -> {out}")
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*")
    ap.add_argument("--pk", action="store_true", help="only the power-spectrum multipole fixtures")
    ap.add_argument("--field", action="store_true", help="only the field generator fixtures")
    ap.add_argument("--oracle", action="store_true", help="the oracle fixtures of large cases")
    ap.add_argument("--save-B", default=None, help="with --oracle and one case: .npy path for its per-triangle B")
    ap.add_argument("--scratch", default=os.path.join(HERE, ".scratch"))
    args = ap.parse_args()
    if args.oracle:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "oracle"], check=True)
        for c in args.cases or list(ORACLE_CASES):
            run_oracle_case(c, args.save_B)
        return
    args.cases = args.cases or list(CASES)
    sys.path.insert(0, ROOT)
    from __graft_entry__ import reference_dir
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "all", f"REF={reference_dir()}"], check=True)
    if not os.path.exists(REF_BIN):
        sys.exit("oracle/_ref/barbie_ref is missing: the reference sources are needed to build it")
    if args.field:
        for c in (args.cases if args.cases != list(CASES) else list(FIELD_CASES)):
            run_field_case(c, args.scratch)
        shutil.rmtree(args.scratch, ignore_errors=True)
        return
    for c in args.cases:
        if args.pk:
            run_pk_case(c, args.scratch)
        else:
            run_case(c, args.scratch)
            run_pk_case(c, args.scratch)
    shutil.rmtree(args.scratch, ignore_errors=True)


if __name__ == "__main__":
    main()
