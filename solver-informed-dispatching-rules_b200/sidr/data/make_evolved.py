"""Writes evolved_gp_generation.npz: populations of the benchmark GP run.

    python solver-informed-dispatching-rules_b200/sidr/data/make_evolved.py   (needs a CUDA device)

The run is the plain GP behind the gp_generation workload (engine/gp.hpp's
GP with the benchmark's settings): seed 0, population 1024, the 29-terminal
menu, 500 training scenarios per generation from base seed 0*10000 + g
(engine/gp_engine.cu:179), fitness = per-rule mean over the block.  The GP is
deterministic (bit-exact fitness), so the file is a pure function of the code.
Saved: the prefix text of generations 25 and 49 and every generation's best
training fitness.  Evolved rules keep routes alive longer and lean on ATRISK,
so these populations cost several times generation 0 per evaluation; the
benchmark times generation 49 beside the initial population.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

KEEP = (25, 49)


def main():
    import sidr
    from sidr import gp, workload
    from sidr.rules import to_prefix

    w = workload.gp_generation(P=1024, S=1)
    zp = sidr.zstats(w.sd)
    ctx = sidr.Context(w.sd, zp)
    sess = gp.Session(workload.MENU29, 0, population=1024, generations=50, train_samples=500,
                      test_samples=500)
    # the session's initial population is the workload's (the same RHH stream)
    assert sess.text() == [to_prefix(t) for t in w.trees]
    pops, best = {}, []
    for g in range(max(KEEP) + 1):
        if g in KEEP:
            pops[f"gen{g}"] = np.array("\n".join(sess.text()))
        smp = gp.gen_durations(w.sd.durations, w.sd.sigma, 500, g)
        out = ctx.evaluate(sess.packed(), smp, 500, w.mask)
        fit = out.sum(axis=1) / 500.0  # integer-valued scores: exact in any order
        best.append(float(fit.max()))
        if g < max(KEEP):
            sess.step(fit)
        print(f"gen {g:2d} best train {best[-1]:.3f}", flush=True)
    ctx.close()
    np.savez_compressed(os.path.join(HERE, "evolved_gp_generation.npz"),
                        best_train=np.array(best), **pops)


if __name__ == "__main__":
    main()
