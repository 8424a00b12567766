"""Dataset profiling harness with the reference's CSV contract.

Restates the behaviour of the reference's scripts/AE_test.py for any set of
programs that take the reference flags (-m1 A.mtx -m2 B.mtx -o C.mtx -l
log.txt, one ms number in the log, exit code 0 on success):

* datasets: every `NAME.mtx` or `NAME/NAME.mtx` under --data-dir
  (AE_test.py:41-47, 161-167); square ones run C = A*A, rectangular ones
  C = A*A^T with the transpose written beside the results (the reference
  stops there with a TODO, AE_test.py:165-171, 216-217);
* each program runs --runs times per dataset (default 20, AE_test.py:57);
  every run appends `program, dataset, run<i>, <ms>` to all_result.csv
  (header `Software,DataSet,Scenario,Runtime(ms)`, AE_test.py:151-152,
  207-220);
* when a program fails on a dataset, the dataset is reduced to its top-left
  quarter and all programs rerun on it, until the quarter would have fewer
  than 1,000 rows or no entries (AE_test.py:77-113, 247-257);
* avg_result.csv = mean runtime per (program, dataset) (AE_test.py:59-71);
  final_result.csv = datasets x programs plus one
  `Speedup (<baseline> / <program>)` column per other program
  (AE_test.py:124-142; the reference has one such column, cuSparse over
  optixSpMSpM).

    python -m rtspmspm_b200.ae_harness --data-dir DATA --out-dir RESULT \\
        [--runs 20] [--program NAME=COMMAND ...] [--baseline cuSparse]

Without --program the engine's own CLI runs twice: `cuSparse` (--algo
cusparse, the reference's cuSPARSE SpGEMM sequence on the same GPU) and
`spgemm` (--algo learned).
"""
from __future__ import annotations

import argparse
import csv
import os
import shlex
import subprocess
import sys
from collections import OrderedDict

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CLI = os.path.join(HERE, "spgemm")


def discover(data_dir: str) -> "OrderedDict[str, str]":
    """Dataset name -> path: NAME/NAME.mtx when present, else NAME.mtx."""
    found: "OrderedDict[str, str]" = OrderedDict()
    for root, _, files in sorted(os.walk(data_dir)):
        for f in sorted(files):
            if not f.endswith(".mtx") or f.endswith("_transpose.mtx") or f.endswith("_small.mtx"):
                continue
            name = f[:-4]
            path = os.path.join(root, f)
            nested = os.path.basename(root) == name
            if name not in found or nested:
                found[name] = path
    return found


def _read(path):
    from .engine import read_mtx

    return read_mtx(path)


def _write(path, m):
    from .engine import write_mtx

    write_mtx(path, m)


def transpose(m):
    from .gen import coo_to_csr

    r = np.repeat(np.arange(m.rows, dtype=np.int64), np.diff(m.row_ptr))
    return coo_to_csr(m.cols, m.rows, m.col_idx.astype(np.int64), r, m.val)


def top_left_quarter(m):
    """Rows [0, rows/2) x cols [0, cols/2) (AE_test.py:77-104)."""
    from .gen import coo_to_csr

    rr, cc = m.rows // 2, m.cols // 2
    r = np.repeat(np.arange(m.rows, dtype=np.int64), np.diff(m.row_ptr))
    keep = (r < rr) & (m.col_idx < cc)
    return coo_to_csr(rr, cc, r[keep], m.col_idx[keep].astype(np.int64), m.val[keep])


def default_programs():
    return OrderedDict([("cuSparse", [CLI, "--algo", "cusparse"]), ("spgemm", [CLI, "--algo", "learned"])])


def run_once(cmd, a_path, b_path, out_path, log_path, timeout):
    if os.path.exists(log_path):
        os.remove(log_path)
    subprocess.run(cmd + ["-m1", a_path, "-m2", b_path, "-o", out_path, "-l", log_path], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL, timeout=timeout)
    with open(log_path) as f:
        return f.read().strip()


def profile(data_dir, out_dir, programs, runs=20, timeout=3600.0, log=print):
    """Runs every program on every dataset; writes the three CSV files and
    returns {dataset: path actually used} (reduced datasets included)."""
    os.makedirs(out_dir, exist_ok=True)
    all_path = os.path.join(out_dir, "all_result.csv")
    with open(all_path, "w") as f:
        f.write("Software,DataSet,Scenario,Runtime(ms)\n")
    used = OrderedDict()
    failed = []
    for name, path in discover(data_dir).items():
        res_dir = os.path.join(out_dir, name, "result")
        os.makedirs(res_dir, exist_ok=True)
        a_path = path
        while True:
            A = _read(a_path)
            if A.rows == A.cols:
                b_path = a_path
            else:
                b_path = os.path.join(res_dir, f"{name}_transpose.mtx")
                _write(b_path, transpose(A))
            buf = []
            ok = True
            for prog, cmd in programs.items():
                out_path = os.path.join(res_dir, f"{prog}.mtx")
                log_path = os.path.join(res_dir, f"{prog}.log")
                for i in range(runs):
                    try:
                        ms = run_once(cmd, a_path, b_path, out_path, log_path, timeout)
                        buf.append(f"{prog}, {name}, run{i}, {ms}\n")
                    except (subprocess.CalledProcessError, subprocess.TimeoutExpired, OSError):
                        buf.append(f"{prog}, {name}, run{i}, \n")
                        ok = False
            if ok:
                with open(all_path, "a") as f:
                    f.writelines(buf)
                used[name] = a_path
                log(f"all programs succeeded for {name}")
                break
            # reduce to the top-left quarter and retry (the reference's sampling)
            small = top_left_quarter(A)
            if small.rows < 1000 or small.nnz == 0:
                log(f"{name}: a program failed and the matrix cannot be reduced further")
                failed.append(name)
                break
            a_path = os.path.join(res_dir, f"{name}_small.mtx")
            _write(a_path, small)
            log(f"{name}: a program failed; reduced to {small.rows} x {small.cols} and retrying")
    averages(all_path, os.path.join(out_dir, "avg_result.csv"))
    speedups(os.path.join(out_dir, "avg_result.csv"), os.path.join(out_dir, "final_result.csv"),
             list(programs), baseline=next(iter(programs)) if programs else None)
    return used, failed


def averages(all_path, out_path):
    """Mean runtime per (program, dataset), blank runs ignored."""
    sums: "OrderedDict[tuple, list]" = OrderedDict()
    with open(all_path) as f:
        rd = csv.reader(f)
        next(rd)
        for row in rd:
            if len(row) < 4:
                continue
            key = (row[0].strip(), row[1].strip())
            sums.setdefault(key, [])
            try:
                sums[key].append(float(row[3]))
            except ValueError:
                pass
    with open(out_path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["Software", "DataSet", "Runtime(ms)"])
        for (prog, ds), v in sums.items():
            w.writerow([prog, ds, repr(sum(v) / len(v)) if v else ""])


def speedups(avg_path, out_path, programs, baseline):
    """Datasets x programs, plus `Speedup (<baseline> / <program>)` columns."""
    table: "OrderedDict[str, dict]" = OrderedDict()
    with open(avg_path) as f:
        rd = csv.DictReader(f)
        for row in rd:
            table.setdefault(row["DataSet"], {})[row["Software"]] = row["Runtime(ms)"]
    others = [p for p in programs if p != baseline]
    with open(out_path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(["DataSet"] + list(programs) + [f"Speedup ({baseline} / {p})" for p in others])
        for ds in sorted(table):
            vals = [table[ds].get(p, "") for p in programs]
            sp = []
            for p in others:
                try:
                    sp.append(repr(float(table[ds][baseline]) / float(table[ds][p])))
                except (KeyError, ValueError, ZeroDivisionError):
                    sp.append("")
            w.writerow([ds] + vals + sp)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--data-dir", required=True)
    ap.add_argument("--out-dir", required=True)
    ap.add_argument("--runs", type=int, default=20)
    ap.add_argument("--timeout", type=float, default=3600.0, help="seconds per program run")
    ap.add_argument("--program", action="append", default=[],
                    help="NAME=COMMAND (the command gets -m1 -m2 -o -l appended); repeatable")
    ap.add_argument("--baseline", default=None, help="program the speedups divide (default: the first)")
    args = ap.parse_args(argv)
    programs = OrderedDict()
    for spec in args.program:
        name, _, cmd = spec.partition("=")
        if not name or not cmd:
            ap.error(f"--program wants NAME=COMMAND, got {spec!r}")
        programs[name] = shlex.split(cmd)
    if not programs:
        programs = default_programs()
    if args.baseline:
        if args.baseline not in programs:
            ap.error(f"--baseline {args.baseline!r} is not a program")
        programs.move_to_end(args.baseline, last=False)
    used, failed = profile(args.data_dir, args.out_dir, programs, runs=args.runs, timeout=args.timeout)
    print(f"datasets: {len(used)} profiled, {len(failed)} failed {failed if failed else ''}".rstrip())
    return 0 if used or not failed else 1


if __name__ == "__main__":
    sys.exit(main())
