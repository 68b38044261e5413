"""The host GP loop (include/sidr_gp.h) against the reference: the golden
populations and fitnesses of verify/golden/gp.txt, and the reference's own
gp_step replayed over many generations."""
import numpy as np
import pytest

from sidr import gp
from sidr import rules as R
from sidr import workload


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def test_gp_reproduces_golden_generations():
    """c101 golden GP (seed 0): populations of generations 0-2 step by step,
    driven by the golden fitness of each generation."""
    from test_oracle import load_gp_blocks
    blocks = {b: (rules, exp) for b, sd, rules, mask, sampled, exp in load_gp_blocks()}
    for case, terms, rmod in (("ns11", R.NS_TERMINALS, 0), ("ext29rmod", R.NS_TERMINALS + R.EXTRA, 1)):
        s = gp.Session(terms, 0, with_rmod=rmod)
        for g in range(3):
            want, fits = blocks[f"{case}_g{g}"]
            got = s.packed()
            assert np.array_equal(got.ops, want.ops) and np.array_equal(got.args, want.args), (case, g)
            assert np.array_equal(got.offsets, want.offsets), (case, g)
            s.step(fits)
        s.close()


@pytest.mark.parametrize("terms,rmod,seed", [(workload.MENU29, 0, 3),
                                             (R.NS_TERMINALS + ["ERC"], 1, 11)])
def test_gp_matches_reference_over_generations(reference, terms, rmod, seed):
    """Random fitness with many ties (stable sort, tournament ties): six
    generations of 256 rules equal the reference's gp_step text."""
    rng = np.random.default_rng(seed)
    fits = rng.integers(0, 40, size=(6, 256)).astype(np.float64)
    want = reference.gp_replay(terms, rmod, seed, 256, fits)
    s = gp.Session(terms, seed, population=256, with_rmod=rmod)
    for g in range(7):
        assert s.text() == want[g], g
        if g < 6:
            s.step(fits[g])
    s.close()


def test_gen_durations_capi_matches_golden():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "durations.npz"))
    for b in z["blocks"]:
        exp = z[f"{b}/expected"]
        got = gp.gen_durations(z[f"{b}/durations"], 0.2, exp.shape[0], int(z[f"{b}/base_seed"][0]))
        assert np.array_equal(bits(got), bits(exp)), b


def test_gp_rejects_bad_config():
    import sidr
    with pytest.raises(sidr.SidrError):
        gp.Session(["SCORE", "NOPE"], 0)
    with pytest.raises(sidr.SidrError):
        gp.Session(["SCORE"], 0, max_depth=9)


def test_run_multi_rejects_bad_arguments():
    """Argument checks of the many-instance driver come before any device work."""
    import sidr
    from sidr import workload
    w = workload.plain_eval(P=1, S=1)
    zp = sidr.zstats(w.sd)
    for kw in (dict(shape=7), dict(shape=-2)):
        with pytest.raises(sidr.SidrError):
            gp.run_multi([w.sd], [zp], workload.MENU29, [w.mask], 2, **kw)
    with pytest.raises(sidr.SidrError):
        gp.run_multi([w.sd], [zp], ["SCORE", "NOPE"], [w.mask], 2)
    with pytest.raises(sidr.SidrError):
        gp.run_multi([w.sd], [zp], workload.MENU29, [w.mask], 0)
    with pytest.raises(sidr.SidrError):  # more populations than one launch's entries
        gp.run_multi([w.sd] * 2, [zp] * 2, workload.MENU29, [w.mask] * 2, 20000, generations=1)


def _fitness_of(sess):
    """A deterministic stand-in fitness: a hash of each rule's text."""
    import zlib
    return np.array([zlib.crc32(t.encode()) % 1000 / 7.0 for t in sess.text()])


@pytest.mark.parametrize("terms,rmod", [(["SCORE", "TA", "NS", "ATRISK", "ERC"], 1),
                                        (["SCORE", "DUR", "TC", "REACH2"], 0)])
def test_checkpoint_resume_continues_identically(terms, rmod):
    """Three steps, a checkpoint, three more steps; a session restored from the
    checkpoint takes the same three steps to the same populations, with ERC
    constants and the generator state carried over."""
    cfg = dict(population=40, max_depth=6, with_rmod=rmod)
    a = gp.Session(terms, 9, **cfg)
    for _ in range(3):
        a.step(_fitness_of(a))
    text = a.checkpoint()
    b = gp.Session.restore(text)
    assert b.generation == a.generation == 3
    assert b.text() == a.text() and b.checkpoint() == text
    for _ in range(3):
        fa, fb = _fitness_of(a), _fitness_of(b)
        a.step(fa)
        b.step(fb)
        assert b.text() == a.text()
    pa, pb = a.packed(), b.packed()
    assert np.array_equal(pa.ops, pb.ops) and np.array_equal(pa.args, pb.args)
    assert b.generation == 6 and b.checkpoint() == a.checkpoint()


def test_restore_refuses_malformed_checkpoints():
    import sidr
    a = gp.Session(["SCORE", "TA", "ERC"], 1, population=12, max_depth=4)
    text = a.checkpoint()
    lines = text.splitlines()
    bad = [
        "not a checkpoint",
        text.replace("sidr-gp-checkpoint 1", "sidr-gp-checkpoint 2"),
        "\n".join(lines[:-3]) + "\n",                                   # truncated population
        "\n".join(lines[:-1] + ["2 0 -1"]) + "\n",                      # not one tree
        "\n".join(lines[:-1] + ["3 0 -1 -1 -1"]) + "\n",                # codes beyond its length
        "\n".join(lines[:-1] + ["1 -999"]) + "\n",                      # unknown leaf label
        "\n".join(l if not l.startswith("rng ") else "rng 5 0 0x0p+0 1 2" for l in lines) + "\n",
        "\n".join(l if not l.startswith("config ") else l.replace("config 12", "config 13", 1)
                  for l in lines) + "\n",                               # population count differs
    ]
    for t in bad:
        with pytest.raises(sidr.SidrError):
            gp.Session.restore(t)
