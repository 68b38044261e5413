"""Python front end of the campaign drivers (include/sidr_campaign.h).

The reference's stage-3/4 programs on the B200 evaluator:

  batch_score / seq_score / gate   s4_selection/ga.cu:111-286 (lockstep
                                   retraining of genomes in one grouped-masks
                                   launch per generation, its sequential twin,
                                   and the --gate equality check)
  run_ga                           s4_selection/ga.cu:288-523 (the tree-13
                                   vocabulary GA with its evaluation cache)
  gen_trace                        s3_generation/gen_trace.cu (trace JSON)
  redeploy                         s4_selection/redeploy.cu (sealing)
  choice                           s4_selection/choice.cu (cross-validatory
                                   choice on the TRAIN block)

Command line (instances are Solomon/Cordeau files; km is the instance's NS-GP
mean-30 from the baseline table):

  python -m sidr.campaign ga <instance> --universe A,B,... [--gate] [...]
  python -m sidr.campaign trace <instance> --terms A,B --tag T --km K [--seeds 30]
  python -m sidr.campaign redeploy <instance> <trace.json> --km K
  python -m sidr.campaign choice <instance> <trace.json>...
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys
from dataclasses import dataclass
from typing import Callable, Optional, Sequence

import numpy as np

from . import Context, _Inst, _Keep, _check, load, zstats
from .gp import _Cfg, _Result, config
from .instance import SimData, load_instance_file
from .rules import NS_TERMINALS

TRAIN_SEED, TRAIN_N = 2000000, 64
TEST_SEED, TEST_N = 1000000, 500

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_FITNESS = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_uint32), C.c_int32, C.c_int32,
                       C.c_int32, _dp)


class GaConfig(C.Structure):
    _fields_ = [("pgens", C.c_int32), ("proxy", C.c_int32), ("confirm", C.c_int32),
                ("gens", C.c_int32), ("stag", C.c_int32), ("bmax", C.c_int32), ("top", C.c_int32),
                ("pm", C.c_double), ("seeds_neutral", C.c_int32), ("nofull", C.c_int32),
                ("ga_seed", C.c_int64)]


STRUCTS = {"sidr_vocab_ga_config": GaConfig}


def _lib():
    L = load()
    if not getattr(L, "_campaign_ready", False):
        pi = C.POINTER(_Inst)
        pc = C.POINTER(_Cfg)
        L.sidr_vocab_batch_score.argtypes = [C.c_void_p, pi, pc, C.c_char_p, C.c_char_p,
                                             C.POINTER(C.c_uint32), C.c_int32, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_int64, C.c_int32, _dp,
                                             C.POINTER(_Result)]
        L.sidr_vocab_seq_score.argtypes = [C.c_void_p, pi, pc, C.c_char_p, C.c_char_p, C.c_uint32,
                                           C.c_int32, C.c_int32, C.c_int64, C.c_int32, _dp]
        L.sidr_vocab_gate.argtypes = [C.c_void_p, pi, pc, C.c_char_p, C.c_char_p, C.c_int32,
                                      C.c_int32, C.c_int32, C.c_int64, C.c_int32,
                                      C.POINTER(C.c_int64), C.POINTER(C.c_int64), _dp]
        L.sidr_vocab_ga_default_config.argtypes = [C.POINTER(GaConfig)]
        L.sidr_vocab_ga.argtypes = [C.c_void_p, pi, pc, C.POINTER(GaConfig), C.c_char_p,
                                    C.c_char_p, C.c_char_p, C.c_char_p, _FITNESS, C.c_void_p,
                                    C.POINTER(C.c_uint32), _dp, C.POINTER(C.c_int64), C.c_char_p,
                                    C.c_int64, C.POINTER(C.c_int64)]
        L.sidr_gen_trace.argtypes = [C.c_void_p, pi, pc, C.c_char_p, C.c_char_p, C.c_char_p,
                                     C.c_int32, C.c_double, C.c_int64, C.c_int32, C.c_char_p,
                                     C.c_int64, C.POINTER(C.c_int64), _dp]
        L.sidr_redeploy.argtypes = [C.c_void_p, pi, C.c_char_p, C.c_char_p, C.c_char_p, C.c_double,
                                    C.c_int64, C.c_int32, _dp, _dp, _dp, _ip]
        L.sidr_trace_mean_train.argtypes = [C.c_void_p, pi, C.c_char_p, C.c_char_p, C.c_int64,
                                            C.c_int32, _dp, _dp]
        L.sidr_rule_compile_prefix.argtypes = [C.c_char_p, _ip, _ip, _ip]
        L._campaign_ready = True
    return L


def _csv(names: Sequence[str]) -> bytes:
    return ",".join(names).encode()


def ga_config(**kw) -> GaConfig:
    """The GA's command-line defaults (s4_selection/ga.cu:52-55) with overrides."""
    c = GaConfig()
    _lib().sidr_vocab_ga_default_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def batch_score(ctx: Context, universe: Sequence[str], genomes: Sequence[int], n_seeds: int,
                n_gens: int, bmax: int = 10, base: Sequence[str] = NS_TERMINALS,
                block_seed: int = TRAIN_SEED, block_n: int = TRAIN_N, **cfg):
    """Per-genome, per-seed block means [K, n_seeds] and the run's timings."""
    c = config(**cfg)
    k = _Keep()
    inst = k.inst(ctx.sd)
    g = np.ascontiguousarray(genomes, dtype=np.uint32)
    out = np.zeros((len(g), n_seeds))
    res = _Result()
    _check(_lib().sidr_vocab_batch_score(ctx.h, C.byref(inst), C.byref(c), _csv(base),
                                         _csv(universe), g.ctypes.data_as(C.POINTER(C.c_uint32)),
                                         len(g), n_seeds, n_gens, bmax, block_seed, block_n,
                                         out.ctypes.data_as(_dp), C.byref(res)))
    return out, res


def seq_score(ctx: Context, universe: Sequence[str], genome: int, n_seeds: int, n_gens: int,
              base: Sequence[str] = NS_TERMINALS, block_seed: int = TRAIN_SEED,
              block_n: int = TRAIN_N, **cfg) -> np.ndarray:
    c = config(**cfg)
    k = _Keep()
    inst = k.inst(ctx.sd)
    out = np.zeros(n_seeds)
    _check(_lib().sidr_vocab_seq_score(ctx.h, C.byref(inst), C.byref(c), _csv(base),
                                       _csv(universe), genome, n_seeds, n_gens, block_seed,
                                       block_n, out.ctypes.data_as(_dp)))
    return out


def gate(ctx: Context, universe: Sequence[str], n_seeds: int = 4, n_gens: int = 5, bmax: int = 10,
         base: Sequence[str] = NS_TERMINALS, block_seed: int = TRAIN_SEED,
         block_n: int = TRAIN_N, **cfg):
    """(compared, mismatches, max |diff|) of batch_score vs seq_score on the
    five gate genomes (s4_selection/ga.cu:260-286)."""
    c = config(**cfg)
    k = _Keep()
    inst = k.inst(ctx.sd)
    cmp_, bad, mx = C.c_int64(), C.c_int64(), C.c_double()
    _check(_lib().sidr_vocab_gate(ctx.h, C.byref(inst), C.byref(c), _csv(base), _csv(universe),
                                  n_seeds, n_gens, bmax, block_seed, block_n, C.byref(cmp_),
                                  C.byref(bad), C.byref(mx)))
    return cmp_.value, bad.value, mx.value


@dataclass
class GaResult:
    champion: int
    champion_mean: float
    evals: int
    log: str


def run_ga(universe: Sequence[str], instance_name: str, ctx: Optional[Context] = None,
           fitness: Optional[Callable] = None, cache_path: Optional[str] = None,
           base: Sequence[str] = NS_TERMINALS, gp: Optional[dict] = None, **ga_kw) -> GaResult:
    """The vocabulary GA.  fitness(genomes, n_seeds, n_gens) -> [K, n_seeds]
    replaces batch_score on the evaluator when given."""
    L = _lib()
    c = config(**(gp or {}))
    g = ga_config(**ga_kw)
    k = _Keep()
    inst = k.inst(ctx.sd) if ctx is not None else None
    err = []

    def _cb(user, gs, K, n, ng, out):
        try:
            arr = np.asarray(fitness([gs[i] for i in range(K)], n, ng), dtype=np.float64).reshape(-1)
            for i in range(K * n):
                out[i] = float(arr[i])
            return 0
        except Exception as e:  # raised again after the native call returns
            err.append(e)
            return 1

    cb = _FITNESS(_cb) if fitness is not None else _FITNESS()
    champ, mean, evals, need = C.c_uint32(), C.c_double(), C.c_int64(), C.c_int64()
    cap = 1 << 20
    buf = C.create_string_buffer(cap)
    st = L.sidr_vocab_ga(ctx.h if ctx is not None else None,
                         C.byref(inst) if inst is not None else None, C.byref(c), C.byref(g),
                         instance_name.encode(), _csv(base), _csv(universe),
                         cache_path.encode() if cache_path else None, cb, None, C.byref(champ),
                         C.byref(mean), C.byref(evals), buf, cap, C.byref(need))
    if err:
        raise err[0]
    _check(st)
    return GaResult(champ.value, mean.value, evals.value, buf.value.decode())


def gen_trace(ctx: Context, instance_name: str, extra: Sequence[str], km: float, n_seeds: int = 30,
              base: Sequence[str] = NS_TERMINALS, test_seed: int = TEST_SEED,
              n_test: int = TEST_N, **cfg):
    """The trace JSON text (as s3_generation/gen_trace.cu writes it) and the
    mean gain."""
    c = config(**cfg)
    k = _Keep()
    inst = k.inst(ctx.sd)
    need, mg = C.c_int64(), C.c_double()
    cap = 1 << 24
    buf = C.create_string_buffer(cap)
    _check(_lib().sidr_gen_trace(ctx.h, C.byref(inst), C.byref(c), instance_name.encode(),
                                 _csv(base), _csv(extra), n_seeds, km, test_seed, n_test, buf, cap,
                                 C.byref(need), C.byref(mg)))
    return buf.value.decode(), mg.value


def redeploy(ctx: Context, instance_name: str, trace_text: str, km: float,
             base: Sequence[str] = NS_TERMINALS, test_seed: int = TEST_SEED,
             n_test: int = TEST_N) -> dict:
    k = _Keep()
    inst = k.inst(ctx.sd)
    tg, g, d, s = C.c_double(), C.c_double(), C.c_double(), C.c_int32()
    _check(_lib().sidr_redeploy(ctx.h, C.byref(inst), instance_name.encode(), trace_text.encode(),
                                _csv(base), km, test_seed, n_test, C.byref(tg), C.byref(g),
                                C.byref(d), C.byref(s)))
    return {"trace_gain": tg.value, "gain": g.value, "delta": d.value, "sealed": bool(s.value)}


def trace_mean_train(ctx: Context, trace_text: str, base: Sequence[str] = NS_TERMINALS,
                     train_seed: int = TRAIN_SEED, n_train: int = TRAIN_N):
    k = _Keep()
    inst = k.inst(ctx.sd)
    mt, ho = C.c_double(), C.c_double()
    _check(_lib().sidr_trace_mean_train(ctx.h, C.byref(inst), trace_text.encode(), _csv(base),
                                        train_seed, n_train, C.byref(mt), C.byref(ho)))
    return mt.value, ho.value


def compile_prefix(text: str):
    """(ops, args) of one prefix rule, the evaluator's post-order encoding."""
    L = _lib()
    n = C.c_int32()
    _check(L.sidr_rule_compile_prefix(text.encode(), None, None, C.byref(n)))
    ops = np.zeros(n.value, np.int32)
    args = np.zeros(2 * n.value, np.int32)
    _check(L.sidr_rule_compile_prefix(text.encode(), ops.ctypes.data_as(_ip),
                                      args.ctypes.data_as(_ip), C.byref(n)))
    return ops, args


def choice(ctx: Context, instance_name: str, traces: Sequence[str], labels: Sequence[str],
           train_seed: int = TRAIN_SEED, n_train: int = TRAIN_N) -> str:
    """The cross-validatory choice report (s4_selection/choice.cu:32-99,
    without the NS-GP backup column): each trace's mean TRAIN score of its
    finals, the choice by TRAIN and the virtual best by held-out gain."""
    out = [f"# choice {instance_name} | train block 2M x {n_train} | columns: {len(traces)}"]
    rows = []
    for text, label in zip(traces, labels):
        mt, ho = trace_mean_train(ctx, text, train_seed=train_seed, n_train=n_train)
        rows.append((label, mt, ho))
        out.append(f"  {label:<24s} mean-TRAIN {mt:8.2f} | held-out {ho:+.2f}")
    ch = rows[0]
    for r in rows:
        if r[1] > ch[1]:
            ch = r
    out.append("")
    out.append(f"CROSS-VALIDATORY CHOICE (train-side): {ch[0]} (train {ch[1]:.2f}) -> "
               f"held-out {ch[2]:+.2f}")
    vbs = rows[0]
    for r in rows:
        if r[2] > vbs[2]:
            vbs = r
    out.append(f"virtual best (labeled): {vbs[0]} -> {vbs[2]:+.2f} | choice==VBS? "
               f"{'True' if ch[0] == vbs[0] else 'False'}")
    return "\n".join(out) + "\n"


# ------------------------------------------------------------- command line

def _context(path: str, m: int = 3):
    sd = SimData.from_instance(load_instance_file(path), m=m)
    return Context(sd, zstats(sd))


def _stem(path: str) -> str:
    return os.path.splitext(os.path.basename(path))[0]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m sidr.campaign")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("ga")
    g.add_argument("instance")
    g.add_argument("--universe", required=True)
    g.add_argument("--seeds", default="random", choices=["random", "neutral"])
    for name, d in (("pgens", 51), ("proxy", 16), ("confirm", 30), ("gens", 50), ("stag", 5),
                    ("bmax", 10), ("top", 4)):
        g.add_argument(f"--{name}", type=int, default=d)
    g.add_argument("--pm", type=float, default=0.5)
    g.add_argument("--nofull", action="store_true")
    g.add_argument("--gate", action="store_true")
    g.add_argument("--cache")
    t = sub.add_parser("trace")
    t.add_argument("instance")
    t.add_argument("--terms", required=True)
    t.add_argument("--tag", required=True)
    t.add_argument("--km", type=float, required=True)
    t.add_argument("--seeds", type=int, default=30)
    t.add_argument("--out", default="results")
    r = sub.add_parser("redeploy")
    r.add_argument("instance")
    r.add_argument("trace")
    r.add_argument("--km", type=float, required=True)
    c = sub.add_parser("choice")
    c.add_argument("instance")
    c.add_argument("traces", nargs="+")
    a = ap.parse_args(argv)
    name = _stem(a.instance)
    ctx = _context(a.instance)
    if a.cmd == "ga":
        uni = [x.strip() for x in a.universe.split(",") if x.strip()]
        if a.gate:
            cmp_, bad, mx = gate(ctx, uni, bmax=a.bmax)
            print(f"GATE compared {cmp_} | mismatches {bad} | max|diff| {mx:.3e} | "
                  f"{'GATE_PASS' if bad == 0 else 'GATE_FAIL'}")
            return 0 if bad == 0 else 1
        res = run_ga(uni, name, ctx=ctx, cache_path=a.cache, pgens=a.pgens, proxy=a.proxy,
                     confirm=a.confirm, gens=a.gens, stag=a.stag, bmax=a.bmax, top=a.top, pm=a.pm,
                     seeds_neutral=int(a.seeds == "neutral"), nofull=int(a.nofull))
        sys.stdout.write(res.log)
        return 0
    if a.cmd == "trace":
        extra = [x.strip() for x in a.terms.split(",") if x.strip()]
        text, mg = gen_trace(ctx, name, extra, a.km, n_seeds=a.seeds)
        os.makedirs(a.out, exist_ok=True)
        path = os.path.join(a.out, f"trace_{name}_{a.tag}.json")
        with open(path, "w") as f:
            f.write(text)
        print(f"  {name} 11+[{','.join(extra)}] | mean gain {mg:+.2f}% -> {path}")
        print("TRACE_DONE")
        return 0
    if a.cmd == "redeploy":
        with open(a.trace) as f:
            text = f.read()
        r_ = redeploy(ctx, name, text, a.km)
        print(f"redeploy {name} {a.trace}: trace-gain {r_['trace_gain']:+.2f} | re-deploy CUDA "
              f"{r_['gain']:+.2f} | delta {r_['delta']:.4f}pp -> "
              f"{'SEALED' if r_['sealed'] else 'FAILED'}")
        return 0
    texts = []
    for p in a.traces:
        with open(p) as f:
            texts.append(f.read())
    sys.stdout.write(choice(ctx, name, texts, [_stem(p) for p in a.traces]))
    return 0


if __name__ == "__main__":
    sys.exit(main())
