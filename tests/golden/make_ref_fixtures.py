"""Record golden fixtures from the reference (sg0/nido) itself.

Runs on a machine with a B200 and the prebuilt reference programs in
oracle/_ref/ (built from the reference sources by `make -f Makefile.ref` in
oracle/):
  * ref_harness  - the reference's GraphGPU / LouvainGPU objects driven step
                   by step (move, coarsen, whole run)
  * run_1_100    - the reference's own command-line program
For every case it writes <out>/<case>.npz holding the input graph, the
assignments used and the reference's outputs.  Inputs come from this
library's seeded generators, so the script regenerates exactly the same
graphs everywhere.

    python tests/golden/make_ref_fixtures.py --out tests/golden
    python tests/golden/make_ref_fixtures.py --configs c1,c2 --out tests/golden

--configs records whole reference runs on the benchmark configurations at
their full size (c1: planted partition, 65,536 vertices, U[0.5,1.5] weights,
-b 1; c2: R-MAT scale 22, unit weights, -b 2) into <out>/configs/<name>.json:
every phase's final Q and every loop's Q (17 digits), loop counts, the
number of communities and the sha256 of the partition file; c1 also keeps
the whole partition (<name>_partition.npz).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import zlib

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from nido_b200 import capi  # noqa: E402

HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
REFBIN = os.path.join(ROOT, "oracle", "_ref", "run_1_100")


def coarse_of(g: capi.Csr, labels: np.ndarray) -> capi.Csr:
    """A graph with self-loops: the quotient graph of `g` by `labels` (edge
    weights summed), vertex ids in label order."""
    nv = int(labels.max()) + 1
    src = np.repeat(np.arange(g.nv), np.diff(g.off))
    key = labels[src] * nv + labels[g.adj]
    uk, inv = np.unique(key, return_inverse=True)
    w = np.zeros(len(uk))
    np.add.at(w, inv, g.w)
    s, d = uk // nv, uk % nv
    off = np.zeros(nv + 1, np.int64)
    np.add.at(off, s + 1, 1)
    return capi.Csr(np.cumsum(off), d.astype(np.int64), w)


def cases():
    out = {}
    out["planted_int"] = capi.gen_planted(16, 32, 12.0, 0.8, capi.W_INT8, 11)
    out["rmat_unit"] = capi.gen_rmat(1024, 8192, wmode=capi.W_ONE, seed=12)
    out["rmat_int"] = capi.gen_rmat(4096, 65536, wmode=capi.W_INT8, seed=13)
    out["sbm_lognormal"] = capi.gen_sbm(3000, cmin=8, cmax=200, avg_degree=10.0, wmode=capi.W_LOGNORMAL, seed=14)
    out["sparse_isolated"] = capi.gen_planted(64, 16, 1.5, 0.7, capi.W_INT8, 15)
    base = out["rmat_int"]
    rng = np.random.default_rng(16)
    out["selfloop_int"] = coarse_of(base, rng.integers(0, 600, base.nv))
    return out


def assignments(g: capi.Csr, name: str):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    k = max(2, g.nv // 8)
    return {"singleton": np.arange(g.nv, dtype=np.int64),
            "random": rng.integers(0, k, g.nv).astype(np.int64)}


def run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{cmd} failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
    return r.stdout


def read_scalars(d):
    vals = {}
    for line in open(os.path.join(d, "scalars.txt")):
        p = line.split()
        vals[p[0]] = int(p[2], 16) if len(p) > 2 else int(p[1])
    return vals


# benchmark configurations recorded at full size: (workload, -b)
CONFIGS = {"c1": ("planted", 1), "c2": ("rmat22", 2)}


def parse_run(out: str):
    """Per-phase final Q, per-phase loop Q lists and loop counts from the
    reference's stdout (louvain_gpu.cpp:30-131 with 17-digit printing)."""
    phases = []
    for block in out.split("PHASE #")[1:]:
        loops = re.findall(r"^(\d+) \t(\S+) \t(\S+)$", block, flags=re.M)
        fq = re.search(r"Final Q: (\S+)", block)
        phases.append({"loop_q": [q for i, q, _ in loops if int(i) > 0],
                       "start_q": next((q for i, q, _ in loops if int(i) == 0), None),
                       "final_q": fq.group(1) if fq else None})
    return phases


def record_configs(out_dir: str, names: list[str]):
    from nido_b200 import workloads
    os.makedirs(os.path.join(out_dir, "configs"), exist_ok=True)
    tmp = tempfile.mkdtemp()
    for name in names:
        wl, nb = CONFIGS[name]
        g = workloads.single_graph(wl)
        path = os.path.join(tmp, name + ".bin")
        capi.write_vite(path, g)
        part = os.path.join(tmp, name + "_part.txt")
        out = run([HARNESS, "run", path, str(nb), "1e-06", "500", part])
        raw = open(part, "rb").read()
        labels = np.array(raw.split(), dtype=np.int64)
        rec = {"config": name, "workload": wl, "nv": g.nv, "ne": g.ne, "nbatches": nb, "tau": 1e-6,
               "max_iter": 500, "phases": parse_run(out), "ncommunities": int(labels.max()) + 1 if len(labels) else 0,
               "partition_sha256": hashlib.sha256(raw).hexdigest(),
               "recorded_with": "oracle/_ref/ref_harness run (the unmodified reference's GraphGPU + LouvainGPU)"}
        with open(os.path.join(out_dir, "configs", name + ".json"), "w") as f:
            json.dump(rec, f, indent=1)
        if name == "c1":
            np.savez_compressed(os.path.join(out_dir, "configs", name + "_partition.npz"), partition=labels)
        os.remove(path)
        print(name, g.nv, g.ne, "phases", len(rec["phases"]), "final Q", rec["phases"][-1]["final_q"], flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--configs", default="", help="comma-separated: record whole runs of these configurations")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    if args.configs:
        record_configs(args.out, [c for c in args.configs.split(",") if c])
        return
    tmp = tempfile.mkdtemp()
    for name, g in cases().items():
        path = os.path.join(tmp, name + ".bin")
        capi.write_vite(path, g)
        rec = {"off": g.off, "adj": g.adj, "w": g.w}
        for an, assign in assignments(g, name).items():
            rec[f"assign_{an}"] = assign
            ap_ = os.path.join(tmp, f"{name}_{an}.i64")
            assign.tofile(ap_)
            for nb, batch in ((1, 0), (3, 1)):
                d = tempfile.mkdtemp(dir=tmp)
                run([HARNESS, "move", path, ap_, str(nb), str(batch), d])
                tag = f"move_{an}_b{nb}_{batch}"
                rec[tag + "_newcomm"] = np.fromfile(os.path.join(d, "newcomm.i64"), np.int64)
                rec[tag + "_a"] = np.fromfile(os.path.join(d, "a.f64"), np.float64)
                rec[tag + "_cuts"] = np.fromfile(os.path.join(d, "cuts.i64"), np.int64)
                sc = read_scalars(d)
                rec[tag + "_mbits"] = np.array([sc["m"]], np.uint64)
                rec[tag + "_qbits"] = np.array([sc["Q"]], np.uint64)
                rec["k"] = np.fromfile(os.path.join(d, "k.f64"), np.float64)
            d = tempfile.mkdtemp(dir=tmp)
            run([HARNESS, "coarsen", path, ap_, d])
            sc = read_scalars(d)
            rec[f"coarsen_{an}_done"] = np.array([sc["extra"]], np.int64)
            rec[f"coarsen_{an}_newid"] = np.fromfile(os.path.join(d, "newid.i64"), np.int64)
            if not sc["extra"]:
                rec[f"coarsen_{an}_off"] = np.fromfile(os.path.join(d, "coff.i64"), np.int64)
                rec[f"coarsen_{an}_adj"] = np.fromfile(os.path.join(d, "cadj.i64"), np.int64)
                rec[f"coarsen_{an}_w"] = np.fromfile(os.path.join(d, "cw.f64"), np.float64)
        for nb in (1, 2):
            part = os.path.join(tmp, f"{name}_run{nb}.txt")
            out = run([HARNESS, "run", path, str(nb), "1e-06", "500", part])
            finals = [float(x) for x in re.findall(r"Final Q: (\S+)", out)]
            loops = re.findall(r"^(\d+) \t(\S+) \t(\S+)$", out, flags=re.M)
            rec[f"run_b{nb}_final_q"] = np.array(finals)
            rec[f"run_b{nb}_loop_q"] = np.array([float(q) for _, q, _ in loops])
            rec[f"run_b{nb}_partition"] = np.loadtxt(part, dtype=np.int64).reshape(-1)
        # the reference's own program, default -b 2, with -o
        part = os.path.join(tmp, f"{name}_bin.txt")
        out = run([REFBIN, "-f", path, "-o", part])
        rec["refbin_partition"] = np.loadtxt(part, dtype=np.int64).reshape(-1)
        rec["refbin_stdout"] = np.array(out)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), **rec)
        print(name, g.nv, g.ne, "phases", len(rec["run_b1_final_q"]), "Q", rec["run_b1_final_q"][-1:], flush=True)


if __name__ == "__main__":
    main()
