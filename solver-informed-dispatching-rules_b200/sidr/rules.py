"""Dispatching rules: expression trees, prefix text, the post-order compiler
and the packed flat layout the evaluator consumes, plus ramped half-and-half
rule generation and scenario sampling.

Mirrors the reference's rule encoding exactly:
  * slot map and aliases -- engine/vocab.hpp:21-62; the 11 NS-GP terminals and
    the 18-terminal constructed menu -- :64-71;
  * ``compile_rule`` -- engine/vocab.hpp:99-126 (post-order; terminal -> op -1
    with args (slot, 0); numeric label -> op -2 with args
    (llround(value*1000), 0); operator -> opcode 0..6 with args (left, right)
    = indices of the two children's last nodes);
  * ``pack`` -- engine/factory.cuh:20-40 (``ops``, flat ``args`` with two ints
    per node, ``offsets``, ``lengths``);
  * prefix text -- engine/tree.hpp:62-96;
  * ``ramped_half_and_half`` -- engine/gp.hpp:36-77 (ERC labels "%.3f");
  * ``gen_durations`` -- engine/sim_host.hpp:43-58 with the MT19937 generator
    of engine/rng.hpp, which draws the same stream as Python's ``random``
    module (seeding by init_by_array, 53-bit doubles, Box-Muller ``gauss``
    with the spare value cached).
"""
from __future__ import annotations

import math
import random
from dataclasses import dataclass
from typing import List, Sequence, Tuple, Union

import numpy as np

N_TERMS = 61
MAX_N = 512
MAX_TREE = 1024
MAX_STACK = 32

TERM_NAMES = [
    "SCORE", "DUR", "TO", "TC", "TA", "TR", "TSV", "TFV", "SL", "RemT", "NS", "REGRET",
    "NSROB", "MAXN", "REACH2", "NSTW", "RAND", "FRAGCNT", "FRAGSCORE", "DOWNSLACK", "PBUST",
    "REACH1", "REACH3", "REACH5", "SAT", "VFRAC", "NFEAS", "VEH", "HARVEST", "BOLSAO",
    "ATRISK", "ZTC", "ZREACH", "ZWLOSS", "ZATRISK", "ZD2D", "C1", "C2", "C3", "C4", "C5",
    "REACH2ROB", "RELCOST", "NETREACH", "SKIPLOSS", "FRAGILITY", "SROB", "REACH3ROB",
    "REACH5ROB", "NSA2", "NSA05", "FEASCORE", "NFEASROB", "NSROB05", "NSROB2", "NNFWD",
    "NNK3", "NNCHAIN3", "SAVINGS", "DETOUR", "SCORERANK",
]
assert len(TERM_NAMES) == N_TERMS
TERM_ALIASES = {"D2D": 5, "SLACK": 8, "WLOSS": 11}
NS_TERMINALS = ["SCORE", "DUR", "TO", "TC", "TA", "TR", "TSV", "TFV", "SL", "RemT", "NS"]
EXTRA = ["REGRET", "NSROB", "MAXN", "REACH2", "NSTW", "FRAGCNT", "FRAGSCORE", "PBUST",
         "REACH1", "REACH3", "REACH5", "SAT", "VFRAC", "NFEAS", "HARVEST", "BOLSAO",
         "ATRISK", "REACH2ROB"]
FUNCTIONS = ["+", "-", "*", "/", "min", "max"]
FUNCS_RMOD = FUNCTIONS + ["rmod"]
OPCODES = {"+": 0, "-": 1, "*": 2, "/": 3, "min": 4, "max": 5, "rmod": 6}

_TERM_INDEX = {nm: i for i, nm in enumerate(TERM_NAMES)}


def term_index(label: str) -> int:
    if label in _TERM_INDEX:
        return _TERM_INDEX[label]
    return TERM_ALIASES.get(label, -1)


def term_mask_from(names: Sequence[str]) -> np.ndarray:
    """engine/sim_host.hpp:85-94 (``ERC`` is skipped)."""
    m = np.zeros(N_TERMS, dtype=np.int64)
    for nm in names:
        if nm == "ERC":
            continue
        i = term_index(nm)
        if i < 0:
            raise ValueError(f"unknown terminal {nm}")
        m[i] = 1
    return m


# ------------------------------------------------------------------ trees

Node = Tuple[str, tuple]  # (label, children)


def leaf(label: str) -> Node:
    return (label, ())


def to_prefix(nd: Node) -> str:
    label, ch = nd
    if not ch:
        return label
    return "(" + label + "".join(" " + to_prefix(c) for c in ch) + ")"


def parse_prefix(s: str) -> Node:
    toks = s.replace("(", " ( ").replace(")", " ) ").split()
    pos = 0

    def at() -> Node:
        nonlocal pos
        tok = toks[pos]
        if tok == "(":
            pos += 1
            sym = toks[pos]
            pos += 1
            kids = []
            while toks[pos] != ")":
                kids.append(at())
            pos += 1
            return (sym, tuple(kids))
        pos += 1
        return (tok, ())

    return at()


def tree_depth(nd: Node) -> int:
    return 0 if not nd[1] else 1 + max(tree_depth(c) for c in nd[1])


def _llround(v: float) -> int:
    a = abs(v)
    r = math.floor(a)
    if a - r >= 0.5:
        r += 1
    return int(-r if v < 0 else r)


def compile_rule(tree: Union[Node, str]) -> Tuple[List[int], List[int]]:
    """Post-order flatten -> (ops, args) with two args per node."""
    if isinstance(tree, str):
        tree = parse_prefix(tree)
    ops: List[int] = []
    args: List[int] = []

    def visit(nd: Node) -> None:
        label, ch = nd
        if not ch:
            ti = term_index(label)
            if ti >= 0:
                ops.append(-1)
                args.extend((ti, 0))
            else:
                ops.append(-2)
                args.extend((_llround(float(label) * 1000.0), 0))
            return
        visit(ch[0])
        left = len(ops) - 1
        visit(ch[1])
        right = len(ops) - 1
        if label not in OPCODES:
            raise ValueError(f"unknown operator {label}")
        ops.append(OPCODES[label])
        args.extend((left, right))

    visit(tree)
    return ops, args


@dataclass
class PackedRules:
    """The reference's PackedTrees (engine/factory.cuh:20-24) as int32 arrays."""
    ops: np.ndarray
    args: np.ndarray
    offsets: np.ndarray
    lengths: np.ndarray

    @property
    def P(self) -> int:
        return int(self.offsets.shape[0])

    def rule(self, p: int) -> Tuple[np.ndarray, np.ndarray]:
        o, L = int(self.offsets[p]), int(self.lengths[p])
        return self.ops[o:o + L], self.args[2 * o:2 * (o + L)]

    def subset(self, idx: Sequence[int]) -> "PackedRules":
        return pack_compiled([self.rule(int(p)) for p in idx])


def pack_compiled(compiled: Sequence[Tuple[Sequence[int], Sequence[int]]]) -> PackedRules:
    ops, args, offs, lens = [], [], [], []
    off = 0
    for o, a in compiled:
        offs.append(off)
        lens.append(len(o))
        ops.extend(int(v) for v in o)
        args.extend(int(v) for v in a)
        off += len(o)
    return PackedRules(np.asarray(ops, dtype=np.int32), np.asarray(args, dtype=np.int32),
                       np.asarray(offs, dtype=np.int32), np.asarray(lens, dtype=np.int32))


def pack(trees: Sequence[Union[Node, str]]) -> PackedRules:
    return pack_compiled([compile_rule(t) for t in trees])


# ------------------------------------------------------- rule generation

class _TreeConfig:
    def __init__(self, terminals, functions, min_depth, max_depth):
        self.terminals = list(terminals)
        self.functions = list(functions)
        self.min_depth = min_depth
        self.max_depth = max_depth


def _pick_terminal(cfg: _TreeConfig, rng: random.Random) -> Node:
    t = cfg.terminals[rng._randbelow(len(cfg.terminals))]
    if t == "ERC":
        return leaf("%.3f" % rng.random())
    return leaf(t)


def _full(cfg, rng, depth) -> Node:
    if depth <= 0:
        return _pick_terminal(cfg, rng)
    sym = cfg.functions[rng._randbelow(len(cfg.functions))]
    a = _full(cfg, rng, depth - 1)
    b = _full(cfg, rng, depth - 1)
    return (sym, (a, b))


def _grow(cfg, rng, depth) -> Node:
    if depth <= 0:
        return _pick_terminal(cfg, rng)
    nt, nf = float(len(cfg.terminals)), float(len(cfg.functions))
    if rng.random() < nt / (nt + nf):
        return _pick_terminal(cfg, rng)
    sym = cfg.functions[rng._randbelow(len(cfg.functions))]
    a = _grow(cfg, rng, depth - 1)
    b = _grow(cfg, rng, depth - 1)
    return (sym, (a, b))


def ramped_half_and_half(terminals: Sequence[str], functions: Sequence[str], min_depth: int,
                         max_depth: int, seed: int, pop: int) -> List[Node]:
    """engine/gp.hpp:67-77 driven by Mt19937(seed)."""
    cfg = _TreeConfig(terminals, functions, min_depth, max_depth)
    rng = random.Random(seed)
    nd = max_depth - min_depth + 1
    out = []
    for i in range(pop):
        d = min_depth + i % nd
        out.append(_full(cfg, rng, d) if (i // nd) % 2 == 0 else _grow(cfg, rng, d))
    return out


def gen_durations(durations: np.ndarray, sigma: float, S: int, base_seed: int) -> np.ndarray:
    """[S][n] sampled service times; scenario s draws from Mt19937(base_seed + s),
    one N(d, sigma*d) draw per customer with d > 0, clipped at 0."""
    n = len(durations)
    out = np.zeros((S, n), dtype=np.float64)
    dl = [float(d) for d in durations]
    for s in range(S):
        rng = random.Random(base_seed + s)
        row = out[s]
        for i, d in enumerate(dl):
            if d <= 0.0:
                continue
            v = rng.gauss(d, sigma * d)
            row[i] = v if v > 0.0 else 0.0
    return out
