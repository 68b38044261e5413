"""Host-side pieces on the CPU: the C-ABI library loads and exports every
symbol include/sidr.h declares, its host computations (z-statistics, rule
validation) behave like the reference, and the Python plumbing (parsers,
compiler, rule generator, scenario sampler, instance generator) reproduces
the reference's own outputs."""
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, REPO

import sidr
from sidr import rules as R
from sidr import workload
from sidr.instance import SimData, generate_instance, load_instance_file, parse_solomon_text


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


# ------------------------------------------------------------ the C-ABI .so

HEADERS = ("sidr.h", "sidr_gp.h", "sidr_campaign.h", "sidr_surrogate.h")


def header_symbols():
    text = "".join(open(os.path.join(REPO, "include", h)).read() for h in HEADERS)
    return sorted(set(re.findall(r"\b(sidr_[a-z0-9_]+)\s*\(", text)))


def all_structs():
    from sidr import campaign, gp, surrogate
    return {**sidr.STRUCTS, "sidr_gp_config": gp._Cfg, "sidr_gp_result": gp._Result,
            **campaign.STRUCTS, **surrogate.STRUCTS}


def test_library_exports_every_declared_symbol():
    L = sidr.load()
    declared = header_symbols()
    assert len(declared) >= 19
    for name in declared:
        assert hasattr(L, name), name
    assert set(sidr.EXPORTS) <= set(declared)


def test_ctypes_structs_match_header(tmp_path):
    """Every ctypes mirror has the C struct's size and member offsets (a
    mismatch lets the library write past a Python-owned buffer)."""
    import ctypes
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>'] + [f'#include "{h}"' for h in HEADERS]
    lines.append("int main(void){")
    for cname, py in all_structs().items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = {}
    for ln in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n"):
        if ln:
            a, b, c = ln.split()
            got[(a, b)] = int(c)
    for cname, py in all_structs().items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert got[(cname, f)] == getattr(py, f).offset, (cname, f)


def test_capi_zstats_matches_golden():
    from test_oracle import SIM_CASES
    for name, sd, rules, mask, zp, sampled, expected in SIM_CASES[::3]:
        assert np.array_equal(bits(sidr.zstats(sd)), bits(zp)), name


def test_capi_zstats_rejects_bad_instances():
    w = workload.plain_eval(P=2, S=1)
    sd = w.sd
    bad = SimData(**{**sd.__dict__, "scores": sd.scores.copy()})
    bad.scores[3] = np.nan
    with pytest.raises(sidr.SidrError) as e:
        sidr.zstats(bad)
    assert e.value.status == 7


def test_ctx_without_device_fails_cleanly():
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a device is present")
    w = workload.plain_eval(P=2, S=1)
    with pytest.raises(sidr.SidrError) as e:
        sidr.Context(w.sd)
    assert e.value.status == 5


def _one(ops, args):
    return R.pack_compiled([(ops, args)])


ALL = np.ones(61, dtype=np.int64)


@pytest.mark.parametrize("ops,args,status", [
    ([-1, -1, 9], [0, 0, 1, 0, 0, 1], 2),           # unknown opcode
    ([-1, -1, 0], [0, 0, 61, 0, 0, 1], 2),          # slot out of range
    ([-1, 0], [0, 0, 0, 0], 2),                     # operator with one operand
    ([-1, -1], [0, 0, 1, 0], 2),                    # two values left
])
def test_rules_check_rejects_malformed(ops, args, status):
    with pytest.raises(sidr.SidrError) as e:
        sidr.rules_check(_one(ops, args), ALL)
    assert e.value.status == status


def test_rules_check_limits():
    deep = [-1] * 33 + [0] * 32
    args = [0, 0] * 33 + [0, 0] * 32
    with pytest.raises(sidr.SidrError) as e:
        sidr.rules_check(_one(deep, args), ALL)
    assert e.value.status == 3  # stack deeper than 32
    ok = [-1] * 32 + [0] * 31
    assert sidr.rules_check(_one(ok, [0, 0] * 63), ALL) >= 32
    long_rule = [-1] + [-1, 0] * 512
    with pytest.raises(sidr.SidrError) as e:
        sidr.rules_check(_one(long_rule, [0, 0] * len(long_rule)), ALL)
    assert e.value.status == 3  # longer than MAX_TREE


def test_rules_check_offsets_bounds():
    r = _one([-1], [0, 0])
    r.offsets[0] = 5
    with pytest.raises(sidr.SidrError) as e:
        sidr.rules_check(r, ALL)
    assert e.value.status == 1


def test_rules_check_accepts_generated_populations():
    w = workload.gp_generation(P=256, S=1)
    rows = sidr.rules_check(w.rules, w.mask)
    assert 1 <= rows <= 93


# ---------------------------------------------------------- Python plumbing

def test_compiler_matches_golden_compile():
    z = np.load(os.path.join(GOLDEN, "compile.npz"))
    for k, t in enumerate(z["trees"]):
        ops, args = R.compile_rule(str(t))
        assert ops == list(z[f"{k}/ops"]), t
        assert args == list(z[f"{k}/args"]), t
        assert R.to_prefix(R.parse_prefix(str(t))) == str(t)


def test_compiler_matches_reference_on_constants(reference):
    for pref in ["(+ 0.123 (* -2.5 SCORE))", "(rmod 0.999 (/ NS 1.0005))", "(- D2D WLOSS)",
                 "(max 12.3456 SLACK)", "0.0005", "(min -0.0015 TA)"]:
        o, a = reference.compile(pref)
        ops, args = R.compile_rule(pref)
        assert ops == list(o) and args == list(a), pref


def test_rhh_matches_reference(reference):
    for terms, lo, hi, seed, pop, rmod in [(workload.MENU29, 2, 6, 1, 200, False),
                                          (R.NS_TERMINALS + ["ERC"], 2, 8, 7, 120, True)]:
        funcs = R.FUNCS_RMOD if rmod else R.FUNCTIONS
        ours = [R.to_prefix(t) for t in R.ramped_half_and_half(terms, funcs, lo, hi, seed, pop)]
        assert ours == reference.rhh(terms, rmod, lo, hi, seed, pop)


def test_gen_durations_matches_reference(reference):
    w = workload.gp_generation(P=2, S=1)
    for seed in (1, 1000000, 123456789):
        got = R.gen_durations(w.sd.durations, 0.2, 16, seed)
        assert np.array_equal(bits(got), bits(reference.gen_durations(w.sd.durations, 0.2, 16, seed)))


def test_parsers_and_dist_match_reference(reference, reference_tree):
    for sub in ("solomon", "cordeau"):
        d = os.path.join(reference_tree, "instances", sub)
        for fn in sorted(os.listdir(d)):
            path = os.path.join(d, fn)
            inst = load_instance_file(path)
            arrs, tmax = reference.parse_instance(path, cordeau=(sub == "cordeau"))
            mine = [np.array([getattr(p, k) for p in inst.pois]) for k in
                    ("x", "y", "score", "open_time", "close_time", "duration")]
            for a, b in zip(mine, arrs):
                assert np.array_equal(bits(a), bits(b)), fn
            assert inst.tmax == tmax
            sd = SimData.from_instance(inst)
            dist, d2d = reference.build_dist(mine[0], mine[1])
            assert np.array_equal(bits(sd.dist), bits(dist)), fn
            assert np.array_equal(bits(sd.dist_to_depot), bits(d2d)), fn


def test_generator_shapes_and_ranges():
    for layout in ("uniform", "clustered", "mixed"):
        for n, H in ((25, 230.0), (288, 1000.0)):
            text = generate_instance(n, layout, H, seed=5)
            inst = parse_solomon_text(text)
            assert inst.n_customers == n and inst.tmax == H
            xs = [p.x for p in inst.pois[1:]]
            assert min(xs) >= 0 and max(xs) <= 100
            sc = [p.score for p in inst.pois[1:]]
            assert min(sc) >= 1 and max(sc) <= 50
            for p in inst.pois[1:]:
                assert 0 <= p.open_time <= p.close_time <= H
                assert p.duration == 10.0
    assert generate_instance(50, "uniform", 230.0, 9) == generate_instance(50, "uniform", 230.0, 9)


def test_workload_oracle_equals_reference(oracle, reference):
    """Config-sized sample: the oracle and the reference agree bit for bit on a
    synthetic instance with the 29-terminal menu."""
    w = workload.plain_eval(P=24, S=6)
    zp = oracle.zstats(w.sd)
    assert np.array_equal(bits(zp), bits(reference.zp_of(w.sd)))
    a = oracle.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    b = reference.eval_pairs(w.sd, zp, w.rules, w.sampled, w.S, w.mask)
    assert np.array_equal(bits(a), bits(b))


def test_large_combined_oracle_equals_reference(oracle, reference):
    """The large combined run's instance shape (288 customers around 12
    cluster centres, m = 4, H = 1000) with initial populations of two GP seeds:
    the oracle and the reference agree bit for bit."""
    mw = workload.large_combined(K=1, seeds=2, rules_per_seed=4, S=2)
    sd = mw.sds[0]
    assert sd.n == 288 and sd.m == 4 and sd.tmax == 1000.0 and mw.rules[0].P == 8
    zp = oracle.zstats(sd)
    assert np.array_equal(bits(zp), bits(reference.zp_of(sd)))
    a = oracle.eval_pairs(sd, zp, mw.rules[0], mw.sampled[0], mw.S, mw.masks[0])
    b = reference.eval_pairs(sd, zp, mw.rules[0], mw.sampled[0], mw.S, mw.masks[0])
    assert np.array_equal(bits(a), bits(b))
