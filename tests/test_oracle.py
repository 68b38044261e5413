"""The CPU oracle against the reference's own golden vectors (fixtures in
tests/golden/, generated by tests/golden/make_golden.py from the reference's
verify/golden files), and against the reference compiled from its headers."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

from sidr.instance import SimData
from sidr import rules as R
from sidr.rules import EXTRA, NS_TERMINALS, PackedRules, pack_compiled, term_mask_from


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


def load_sim_cases():
    z = np.load(os.path.join(GOLDEN, "sim_cases.npz"))
    out = []
    for c in z["cases"]:
        g = lambda k: z[f"{c}/{k}"]  # noqa: E731
        sd = SimData.from_arrays(g("inst_x"), g("inst_y"), g("inst_score"), g("inst_open"),
                                 g("inst_close"), g("inst_dur"), g("inst_tmax"), m=3)
        out.append((str(c), sd, pack_compiled([(g("ops"), g("args"))]), g("mask"), g("zp"),
                    g("sampled"), g("expected")))
    return out


def load_gp_blocks():
    z = np.load(os.path.join(GOLDEN, "gp_cases.npz"))
    sd = SimData.from_arrays(*[z[f"c101/inst_{k}"] for k in
                               ("x", "y", "score", "open", "close", "dur", "tmax")], m=3)
    out = []
    for b in z["blocks"]:
        b = str(b)
        rules = PackedRules(z[f"{b}/ops"], z[f"{b}/args"], z[f"{b}/offsets"], z[f"{b}/lengths"])
        mask = term_mask_from(NS_TERMINALS + (EXTRA if "ext29" in b else []))
        out.append((b, sd, rules, mask, z[f"{b}/sampled"], z[f"{b}/expected"]))
    return out


SIM_CASES = load_sim_cases()


@pytest.mark.parametrize("case", SIM_CASES, ids=[c[0] for c in SIM_CASES])
def test_oracle_sim_golden(oracle, case):
    name, sd, rules, mask, zp, sampled, expected = case
    out = oracle.eval_pairs(sd, zp, rules, sampled, sampled.shape[0], mask)
    assert np.array_equal(bits(out[0]), bits(expected)), name


@pytest.mark.parametrize("case", SIM_CASES[::3], ids=[c[0] for c in SIM_CASES[::3]])
def test_oracle_zstats_golden(oracle, case):
    name, sd, rules, mask, zp, sampled, expected = case
    assert np.array_equal(bits(oracle.zstats(sd)), bits(zp)), name


def test_oracle_gp_golden(oracle):
    """6144 per-rule fitnesses of 3 GP generations on c101 (ns11 and
    ext29+rmod), 1 scenario each (verify/golden/gp.txt)."""
    for b, sd, rules, mask, sampled, expected in load_gp_blocks():
        zp = oracle.zstats(sd)
        out = oracle.eval_pairs(sd, zp, rules, sampled, 1, mask)
        assert np.array_equal(bits(out[:, 0]), bits(expected)), b


def test_oracle_durations_golden(oracle):
    from sidr.rules import gen_durations
    z = np.load(os.path.join(GOLDEN, "durations.npz"))
    for b in z["blocks"]:
        d = z[f"{b}/durations"]
        seed = int(z[f"{b}/base_seed"][0])
        exp = z[f"{b}/expected"]
        got_c = oracle.gen_durations(d, 0.2, exp.shape[0], seed)
        got_py = gen_durations(d, 0.2, exp.shape[0], seed)
        assert np.array_equal(bits(got_c), bits(exp)), b
        assert np.array_equal(bits(got_py), bits(exp)), b


def test_oracle_catches_a_planted_change(oracle):
    """The golden comparison is sharp: planting a change in the oracle's inputs
    (service times 30% longer, or the z-statistics shifted) moves golden
    scores."""
    hits = 0
    for name, sd, rules, mask, zp, sampled, expected in SIM_CASES:
        a = oracle.eval_pairs(sd, zp, rules, sampled * 1.3, sampled.shape[0], mask)
        hits += int(not np.array_equal(bits(a[0]), bits(expected)))
    assert hits >= 6
    name, sd, rules, mask, zp, sampled, expected = [c for c in SIM_CASES if c[0] == "r101_full61"][0]
    zp2 = zp.copy()
    zp2[5:] *= 0.01  # a uniform shift would not move the argmax; a rescale does
    a = oracle.eval_pairs(sd, zp2, rules, sampled, sampled.shape[0], mask)
    assert not np.array_equal(bits(a[0]), bits(expected))


def test_rng_matches_reference_golden_stream(reference_tree):
    """Python's MT19937 (used for rules and scenarios) replays the reference's
    verify/golden/rng.txt random/gauss draws."""
    import random
    import struct
    path = os.path.join(reference_tree, "verify", "golden", "rng.txt")
    rng = None
    checked = 0
    for line in open(path):
        p = line.split()
        if not p:
            continue
        if p[0] == "#":
            rng = random.Random(int(p[2]))
            continue
        if p[0] == "random":
            want = struct.unpack("<d", struct.pack("<Q", int(p[1], 16)))[0]
            assert rng.random() == want
            checked += 1
        elif p[0] == "gauss":
            want = struct.unpack("<d", struct.pack("<Q", int(p[1], 16)))[0]
            assert rng.gauss(10.0, 2.0) == want
            checked += 1
        elif p[0].startswith("getrandbits_"):
            assert rng.getrandbits(int(p[0][12:])) == int(p[1])
        elif p[0] in ("randint_2_8", "mix_randint"):
            assert rng.randint(2, 8) == int(p[1])
        elif p[0] == "choice29":
            assert rng._randbelow(29) == int(p[1])
        elif p[0] == "mix_choice":
            assert rng._randbelow(61) == int(p[1])
        elif p[0] in ("sample1024_7", "sample50_7"):
            n = 1024 if p[0] == "sample1024_7" else 50
            assert rng.sample(range(n), 7) == [int(v) for v in p[1:]]
        elif p[0] == "mix_random":
            want = struct.unpack("<d", struct.pack("<Q", int(p[1], 16)))[0]
            assert rng.random() == want
        elif p[0] == "mix_gauss":
            want = struct.unpack("<d", struct.pack("<Q", int(p[1], 16)))[0]
            assert rng.gauss(5.0, 1.5) == want
    assert checked > 1000


def test_reference_rmod_calls_pow_at_run_time(reference, oracle):
    """rmod with the regime clipped to 1 is pow(x, 2.0), which a compiler may
    fold into x * x; the C library's pow differs from x * x in the last bit for
    a few arguments.  Rules that subtract x * x from rmod(x, 1.5) make that bit
    decide: the reference's compiled simulator scores them differently from an
    all-zero priority (so it calls pow at run time, as the evaluator's restated
    pow does), and the oracle gives the reference's scores bit for bit."""
    from sidr import workload
    w = workload.gp_generation(P=1, S=300)
    mask = R.term_mask_from(workload.MENU29 + ["ERC"])
    terms = ["NSTW", "TFV", "BOLSAO"]
    rules = R.pack([f"(- (rmod {t} 1.5) (* {t} {t}))" for t in terms] +
                   [f"(- (* {t} {t}) (* {t} {t}))" for t in terms])
    ref = reference.eval_pairs(w.sd, reference.zp_of(w.sd), rules, w.sampled, 300, mask)
    ora = oracle.eval_pairs(w.sd, oracle.zstats(w.sd), rules, w.sampled, 300, mask)
    assert np.array_equal(ref.view(np.uint64), ora.view(np.uint64))
    assert all(not np.array_equal(ref[k], ref[k + 3]) for k in range(3))
