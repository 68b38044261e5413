"""Oracle: a pure-Python restatement of the reference's vocabulary GA
(s4_selection/ga.cu:288-523), with the fitness source left to the caller.

Test infrastructure only -- the product path is the C++ driver
(sidr_vocab_ga); this file exists so that tests can check its host logic
(pool seeding, the tree-13 hierarchy and its swaps, uniform crossover and
mutation, re-injection, stagnation, the evaluation cache, finalist
confirmation) against an independent statement of the same steps.  The GA's
generator is random.Random(seed): CPython's Mersenne Twister seeded from an
int and its 53-bit random(), the stream the reference's Mt19937 reproduces
(engine/rng.hpp).

run_ga(universe, fitness, ...) returns (champion, champion_mean, evals,
lines, cache_text): lines are the program's stdout lines without the timing
lines ("  batch ...", "PERF ..."); cache_text is what the cache file holds at
the end (when cache=True or preload is given).
"""
from __future__ import annotations

import random


def c_hexfloat(x: float) -> str:
    """printf's %a text of x (glibc: mantissa digits without trailing zeros)."""
    m, e = float.hex(x).split("p")
    if "." in m:
        m = m.rstrip("0").rstrip(".")
    return m + "p" + e


def run_ga(universe, fitness, instance="inst", pgens=51, proxy=16, confirm=30, gens=50, stag_k=5,
           bmax=10, top_n=4, pm_mult=0.5, seed_mode="random", nofull=False, cgens=51,
           ga_seed=20260714, cache=False, preload=None):
    nb = len(universe)
    rng = random.Random(ga_seed)
    lines = []
    cache_p, cache_c = {}, {}
    evals = 0
    hdr = (f"# gacache v1 {instance} uni={','.join(universe)} proxy={proxy} pgens={pgens} "
           f"confirm={confirm} cgens={cgens}")
    cache_lines = []
    if preload is not None:  # the cache file of an earlier run (ga.cu:334-351)
        rows = preload.split("\n")
        hits = 0
        if rows and rows[0] == hdr:
            for ln in rows[1:]:
                parts = ln.split()
                if len(parts) < 3 or parts[0] not in ("P", "C"):
                    continue
                g, n = int(parts[1], 16), int(parts[2])
                v = [float.fromhex(x) for x in parts[3:3 + n]]
                if len(v) != n:
                    continue
                (cache_p if parts[0] == "P" else cache_c)[g] = v
                hits += 1
        if hits > 0:
            cache_lines = [r for r in rows if r]
            lines.append(f"# cache CACHE | {hits} entries loaded")
        else:
            cache_lines = [hdr]
    elif cache:
        cache_lines = [hdr]

    def name_of(g):
        s = ",".join(universe[b] for b in range(nb) if g >> b & 1)
        return s if s else "(base)"

    def nbits(g):
        return bin(g).count("1")

    def mean_of(v):
        a = 0.0
        for x in v:
            a += x
        return a / len(v)

    def batch_score(gs, n, ng):
        nonlocal evals
        res = []
        for k0 in range(0, len(gs), bmax):
            chunk = gs[k0:k0 + bmax]
            res.extend(fitness(chunk, n, ng))
            evals += len(chunk)
        return res

    def append(kind, g, v):
        if cache or preload is not None:
            cache_lines.append(f"{kind} {g:x} {len(v)} " + " ".join(c_hexfloat(x) for x in v))

    def ensure(want):
        want = sorted(set(want))
        miss = [g for g in want if g not in cache_p]
        if not miss:
            return
        res = batch_score(miss, proxy, pgens)
        for g, r in zip(miss, res):
            cache_p[g] = list(r)
            append("P", g, list(r))

    def mean_c(g):
        return mean_of(cache_p[g])

    full = (1 << nb) - 1
    seeds = []
    if seed_mode == "neutral":
        seeds.append(0)
        if not nofull:
            seeds.append(full)
        seeds.extend(1 << b for b in range(nb))
    seeds = sorted(set(seeds))
    NP = 13

    def random_genome():
        g = 0
        for b in range(nb):
            if rng.random() < 0.35:
                g |= 1 << b
        return g

    pool = list(seeds)
    while len(pool) < NP:
        pool.append(random_genome())
    lines.append(f"# ga {instance} | universe {nb} | seeds {seed_mode} ({len(seeds)})"
                 f"{' nofull' if nofull else ''} | tree-13 uniform-x pm {pm_mult:.2f} | "
                 f"gens {gens} stag {stag_k}")
    ensure(pool)
    key = lambda g: (-mean_c(g), nbits(g))  # noqa: E731 (sorted() is stable: ties keep order)
    pool = sorted(pool, key=key)[:NP]
    tree = list(pool)

    def restore():
        for _ in range(NP):
            moved = False
            for c in range(3, -1, -1):
                lead = 0 if c == 0 else c
                base = 1 if c == 0 else 4 + 3 * (c - 1)
                best = -1
                for j in range(3):
                    idx = base + j
                    if mean_c(tree[idx]) > mean_c(tree[lead]):
                        if best < 0 or mean_c(tree[idx]) > mean_c(tree[best]):
                            best = idx
                if best >= 0:
                    tree[lead], tree[best] = tree[best], tree[lead]
                    moved = True
            if not moved:
                break

    restore()

    def cross_mut(a, b):
        child = 0
        for k in range(nb):
            child |= (a if rng.random() < 0.5 else b) & (1 << k)
        for k in range(nb):
            if rng.random() < pm_mult / nb:
                child ^= 1 << k
        return child

    best_seen = mean_c(tree[0])
    stag = 0
    for gen in range(gens):
        uniq = set(tree)
        pmean = 0.0
        for i in range(NP):
            pmean += mean_c(tree[i])
        pmean /= NP
        lines.append(f"gen {gen} | best {mean_c(tree[0]):.2f} [{name_of(tree[0])}] | mean "
                     f"{pmean:.2f} | unique {len(uniq)} | evals {evals}")
        if len(uniq) <= 6:
            fresh = []
            for r in range(2):
                g = random_genome()
                tree[12 - r] = g
                fresh.append(g)
            ensure(fresh)
            lines.append("  reinject 2")
        children, pairs = [], []
        for c in range(4):
            lead = 0 if c == 0 else c
            base = 1 if c == 0 else 4 + 3 * (c - 1)
            for j in range(3):
                sup = base + j
                children.append(cross_mut(tree[lead], tree[sup]))
                pairs.append((lead, sup))
        ensure(children)
        for ch, (lead, sup) in zip(children, pairs):
            wp = sup if mean_c(tree[sup]) <= mean_c(tree[lead]) else lead
            if mean_c(ch) > mean_c(tree[wp]):
                tree[wp] = ch
        restore()
        cur = mean_c(tree[0])
        if cur > best_seen:
            best_seen, stag = cur, 0
        else:
            stag += 1
        if stag >= stag_k:
            lines.append(f"stop: stagnant {stag} gens")
            break
    pmean = 0.0
    for i in range(NP):
        pmean += mean_c(tree[i])
    pmean /= NP
    lines.append(f"gen end | best {mean_c(tree[0]):.2f} [{name_of(tree[0])}] | mean {pmean:.2f} | "
                 f"evals {evals}")
    fin = sorted(sorted(set(tree)), key=key)[:top_n]  # sort + unique, then stable order
    lines.append("")
    lines.append(f"confirming top-{len(fin)} at {confirm} seeds:")
    cmiss = [g for g in fin if g not in cache_c]
    if cmiss:
        res = batch_score(cmiss, confirm, cgens)
        for g, r in zip(cmiss, res):
            cache_c[g] = list(r)
            append("C", g, list(r))
    conf = [cache_c[g] for g in fin]
    bi = 0
    for i in range(1, len(fin)):
        a, b = mean_of(conf[i]), mean_of(conf[bi])
        if a > b or (a == b and nbits(fin[i]) < nbits(fin[bi])):
            bi = i
    for g, cv in zip(fin, conf):
        lines.append(f"  {mean_of(cv):.2f} (proxy {mean_c(g):.2f}) [{name_of(g)}]")
    lines.append("")
    lines.append(f"CHAMPION train-{confirm} {mean_of(conf[bi]):.2f} | evals {evals} | terms: "
                 f"{name_of(fin[bi])}")
    cache_text = "\n".join(cache_lines) + "\n" if cache_lines else ""
    return fin[bi], mean_of(conf[bi]), evals, lines, cache_text
