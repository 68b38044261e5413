"""Regenerates the committed parity fixtures under tests/golden/ from the
reference's own golden files and benchmark instances.

    python tests/golden/make_golden.py [--ref REFERENCE_TREE]

The reference tree comes from --ref, else the SIDR_REF environment variable, else
the tree oracle/Makefile compiled oracle/_ref from (oracle/_ref/reference_tree.txt).

Reads (never copies) the reference tree:
  verify/golden/sim.txt        12 cases (c101/r101/rc101/pr01 x ns11/ext29/full61):
                               tree, mask, zp, 20 scenarios of sampled durations,
                               20 expected route scores (hex doubles)
  verify/golden/gp.txt         c101 x {ns11, ext29rmod} x 3 generations: 1024
                               rules (prefix), 1 scenario, 1024 expected fitnesses
  verify/golden/durations.txt  duration sampling, 3 instances x 3 base seeds x 5
  verify/golden/compile.txt    46 rules with their post-order ops/args
  instances/{solomon,cordeau}  the benchmark instances those cases run on
  results/ga40/results/trace_<inst>_Sga.json
                               the campaign's generation traces (c101, r101,
                               rc101, pr01): per-generation bests and the 30
                               finals with their held-out gains
  results/baseline/cap2-results.csv
                               the NS-GP mean-30 (km) the gains are taken over
  results/ga40/logs/c101_search.log
                               the vocabulary GA's stdout on c101 (the lines
                               up to the third generation, timings dropped)

and writes them as numpy archives (doubles kept bit-exact):
  sim_cases.npz, gp_cases.npz, durations.npz, compile.npz, campaign.npz.
Rules are compiled here by sidr.rules.compile_rule; the compile fixture pins
that compiler against the reference's own compile_rmod output.
"""
from __future__ import annotations

import argparse
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "solver-informed-dispatching-rules_b200"))

from sidr.instance import load_instance_file  # noqa: E402
from sidr.rules import compile_rule, pack  # noqa: E402


def hexd(h: str) -> float:
    return struct.unpack("<d", struct.pack("<Q", int(h, 16)))[0]


def inst_arrays(ref: str, name: str):
    sub = "cordeau" if name.startswith("pr") else "solomon"
    inst = load_instance_file(os.path.join(ref, "instances", sub, name + ".txt"))
    P = inst.pois
    return {
        "x": np.array([p.x for p in P]), "y": np.array([p.y for p in P]),
        "score": np.array([p.score for p in P]), "open": np.array([p.open_time for p in P]),
        "close": np.array([p.close_time for p in P]), "dur": np.array([p.duration for p in P]),
        "tmax": np.array([inst.tmax]),
    }


def put_inst(out: dict, key: str, arrs: dict) -> None:
    for k, v in arrs.items():
        out[f"{key}/inst_{k}"] = v


def make_sim(ref: str) -> dict:
    out = {}
    names = []
    cur = None
    with open(os.path.join(ref, "verify", "golden", "sim.txt")) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            if line.startswith("# case "):
                inst, kind = line[7:].split()
                cur = f"{inst}_{kind}"
                names.append(cur)
                put_inst(out, cur, inst_arrays(ref, inst))
                out[f"{cur}/sampled"] = []
            elif line.startswith("tree "):
                ops, args = compile_rule(line[5:])
                out[f"{cur}/ops"] = np.array(ops, dtype=np.int32)
                out[f"{cur}/args"] = np.array(args, dtype=np.int32)
            elif line.startswith("mask "):
                out[f"{cur}/mask"] = np.array([int(v) for v in line[5:].split()], dtype=np.int64)
            elif line.startswith("zp "):
                out[f"{cur}/zp"] = np.array([hexd(h) for h in line[3:].split()])
            elif line.startswith("sampled "):
                out[f"{cur}/sampled"].append([hexd(h) for h in line[8:].split()])
            elif line.startswith("scores "):
                out[f"{cur}/expected"] = np.array([hexd(h) for h in line[7:].split()])
    for k in names:
        out[f"{k}/sampled"] = np.array(out[f"{k}/sampled"])
    out["cases"] = np.array(names)
    return out


def make_gp(ref: str) -> dict:
    out = {}
    put_inst(out, "c101", inst_arrays(ref, "c101"))
    blocks = []
    case = None
    trees = []
    with open(os.path.join(ref, "verify", "golden", "gp.txt")) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            if line.startswith("# case "):
                case = line.split()[-1]
                trees = []
            elif line[0] == "p" and line[2] == " ":
                trees.append(line[3:])
            elif line.startswith("sampled "):
                parts = line[8:].split()
                gen = int(parts[0])
                key = f"{case}_g{gen}"
                pk = pack(trees)
                out[f"{key}/ops"] = pk.ops
                out[f"{key}/args"] = pk.args
                out[f"{key}/offsets"] = pk.offsets
                out[f"{key}/lengths"] = pk.lengths
                out[f"{key}/sampled"] = np.array([[hexd(h) for h in parts[1:]]])
                trees = []
            elif line.startswith("fits "):
                parts = line[5:].split()
                key = f"{case}_g{int(parts[0])}"
                out[f"{key}/expected"] = np.array([hexd(h) for h in parts[1:]])
                blocks.append(key)
    out["blocks"] = np.array(blocks)
    return out


def make_durations(ref: str) -> dict:
    out = {}
    blocks = []
    cur = None
    with open(os.path.join(ref, "verify", "golden", "durations.txt")) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if not line:
                continue
            if line.startswith("# inst "):
                nm, _, seed = line[7:].split()
                cur = f"{nm}_{seed}"
                blocks.append(cur)
                a = inst_arrays(ref, nm)
                out[f"{cur}/durations"] = a["dur"][1:]
                out[f"{cur}/base_seed"] = np.array([int(seed)])
                out[f"{cur}/expected"] = []
            elif line.startswith("dur "):
                out[f"{cur}/expected"].append([hexd(h) for h in line[4:].split()])
    for b in blocks:
        out[f"{b}/expected"] = np.array(out[f"{b}/expected"])
    out["blocks"] = np.array(blocks)
    return out


def make_compile(ref: str) -> dict:
    trees, ops, args = [], [], []
    with open(os.path.join(ref, "verify", "golden", "compile.txt")) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if line.startswith("tree "):
                trees.append(line[5:])
            elif line.startswith("ops "):
                ops.append(np.array([int(v) for v in line[4:].split()], dtype=np.int32))
            elif line.startswith("args "):
                args.append(np.array([int(v) for v in line[5:].split()], dtype=np.int32))
    out = {"trees": np.array(trees)}
    for i, (o, a) in enumerate(zip(ops, args)):
        out[f"{i}/ops"] = o
        out[f"{i}/args"] = a
    return out


CAMPAIGN_INSTANCES = ("c101", "r101", "rc101", "pr01")


def baseline_km(ref: str, name: str) -> float:
    import csv
    with open(os.path.join(ref, "results", "baseline", "cap2-results.csv")) as f:
        for row in csv.DictReader(f):
            if row["instance"] == name:
                return float(row["baseline_nsgp_mean30"])
    raise KeyError(name)


def make_campaign(ref: str) -> dict:
    out = {}
    for nm in CAMPAIGN_INSTANCES:
        put_inst(out, nm, inst_arrays(ref, nm))
        out[f"{nm}/km"] = np.array([baseline_km(ref, nm)])
        with open(os.path.join(ref, "results", "ga40", "results", f"trace_{nm}_Sga.json")) as f:
            out[f"{nm}/trace"] = np.array(f.read())
    lines = []
    with open(os.path.join(ref, "results", "ga40", "logs", "c101_search.log")) as f:
        for line in f:
            line = line.rstrip("\r\n")
            if line.startswith("  batch "):
                continue
            lines.append(line)
            if line.startswith("gen 2 "):
                break
    out["c101/search_head"] = np.array(lines)
    out["instances"] = np.array(CAMPAIGN_INSTANCES)
    return out


def recorded_reference_tree():
    """SIDR_REF, else the tree oracle/Makefile built oracle/_ref from."""
    if os.environ.get("SIDR_REF"):
        return os.environ["SIDR_REF"]
    rec = os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle", "_ref",
                       "reference_tree.txt")
    if os.path.exists(rec):
        with open(rec) as f:
            return f.read().strip() or None
    return None


MAKERS = {"sim_cases": make_sim, "gp_cases": make_gp, "durations": make_durations,
          "compile": make_compile, "campaign": make_campaign}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None, help="the reference source tree")
    ap.add_argument("--only", nargs="*", choices=sorted(MAKERS), help="regenerate these only")
    a = ap.parse_args()
    if a.ref is None:
        a.ref = recorded_reference_tree()
    if not a.ref or not os.path.isdir(a.ref):
        raise SystemExit("reference tree unknown: pass --ref or set SIDR_REF")
    for name in a.only or list(MAKERS):
        fn = MAKERS[name]
        data = fn(a.ref)
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **data)
        print(f"wrote {path} ({os.path.getsize(path)} bytes)")


if __name__ == "__main__":
    main()
