"""ctypes front end of the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Two checkers live under oracle/:
  * ``Oracle``     -- the plain-C restatement in sidr_oracle.c
                      (_build/libsidr_oracle.so);
  * ``Reference``  -- the reference's own engine headers compiled in place
                      through ref_shim.cpp (_ref/libsidr_ref.so), present only
                      where the reference tree was available at build time.

Only tests/, __graft_entry__.smoke() and the cpu_baseline / reference legs of
bench.py may import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libsidr_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libsidr_ref.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


def build(quiet: bool = True) -> None:
    """make -C oracle (the reference part is skipped when its tree is absent)."""
    r = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    if not quiet:
        print(r.stdout)


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(_ip)


def _l(a):
    return np.ascontiguousarray(a, dtype=np.int64).ctypes.data_as(_lp)


class _SoSim(C.Structure):
    _fields_ = [("n", C.c_int), ("m", C.c_int), ("ld", C.c_int), ("tmax", C.c_double),
                ("scores", _dp), ("durations", _dp), ("open_t", _dp), ("close_t", _dp),
                ("dist", _dp), ("dist_to_depot", _dp)]


class _SoCounts(C.Structure):
    _fields_ = [("decisions", C.c_int64), ("candidates", C.c_int64), ("tokens", C.c_int64)]


def _keep(sd):
    arrs = [np.ascontiguousarray(getattr(sd, k), dtype=np.float64)
            for k in ("scores", "durations", "open_t", "close_t", "dist", "dist_to_depot")]
    s = _SoSim(sd.n, sd.m, sd.n + 1, float(sd.tmax), *[a.ctypes.data_as(_dp) for a in arrs])
    return s, arrs


def _grouping(P, sampled, T, group_size, masks, mask_group):
    sampled = np.ascontiguousarray(sampled, dtype=np.float64)
    masks = np.ascontiguousarray(masks, dtype=np.int64).reshape(-1)
    if group_size is None:
        group_size = P
    if mask_group is None:
        mask_group = P
    return sampled, group_size, masks, mask_group


class Oracle:
    """The C restatement."""

    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        self.lib = C.CDLL(ORACLE_SO)
        L = self.lib
        L.so_zstats.argtypes = [C.POINTER(_SoSim), _dp]
        L.so_gen_durations.argtypes = [C.c_int, _dp, C.c_double, C.c_int, C.c_longlong, _dp]
        L.so_eval_pairs.argtypes = [C.POINTER(_SoSim), _dp, _ip, _ip, _ip, _ip, C.c_int, _dp,
                                    C.c_int, C.c_int, _lp, C.c_int, _dp, C.c_int,
                                    C.POINTER(_SoCounts)]
        L.so_build_dist.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        L.so_mt_seed.argtypes = [C.c_void_p, C.c_uint64]
        L.so_mt_random.argtypes = [C.c_void_p]
        L.so_mt_random.restype = C.c_double
        L.so_mt_gauss.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.so_mt_gauss.restype = C.c_double

    def zstats(self, sd) -> np.ndarray:
        s, keep = _keep(sd)
        zp = np.zeros(10)
        self.lib.so_zstats(C.byref(s), _d(zp))
        return zp

    def gen_durations(self, durations, sigma, S, base_seed) -> np.ndarray:
        d = np.ascontiguousarray(durations, dtype=np.float64)
        out = np.zeros((S, len(d)))
        self.lib.so_gen_durations(len(d), _d(d), sigma, S, base_seed, _d(out))
        return out

    def build_dist(self, x, y):
        n = len(x) - 1
        dist = np.zeros((n + 1) * (n + 1))
        d2d = np.zeros(n)
        self.lib.so_build_dist(n, _d(x), _d(y), _d(dist), _d(d2d))
        return dist, d2d

    def eval_pairs(self, sd, zp, rules, sampled, T, masks, group_size=None, mask_group=None,
                   nthreads=None, counts=False):
        """out[P, T]; see so_eval_pairs."""
        P = rules.P
        sampled, group_size, masks, mask_group = _grouping(P, sampled, T, group_size, masks,
                                                          mask_group)
        s, keep = _keep(sd)
        zp = np.ascontiguousarray(zp, dtype=np.float64)
        out = np.zeros((P, T))
        cnt = _SoCounts()
        self.lib.so_eval_pairs(C.byref(s), _d(zp), _i(rules.ops), _i(rules.args),
                               _i(rules.offsets), _i(rules.lengths), P, _d(sampled), T,
                               group_size, _l(masks), mask_group, _d(out),
                               nthreads or os.cpu_count() or 1, C.byref(cnt))
        if counts:
            return out, {"decisions": cnt.decisions, "candidates": cnt.candidates,
                         "tokens": cnt.tokens}
        return out

    def mt_draws(self, seed, count, kind="random"):
        st = (C.c_uint8 * 4096)()
        self.lib.so_mt_seed(st, seed)
        if kind == "random":
            return np.array([self.lib.so_mt_random(st) for _ in range(count)])
        return np.array([self.lib.so_mt_gauss(st, 0.0, 1.0) for _ in range(count)])


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class Reference:
    """The reference's own engine, compiled from its headers (oracle/_ref)."""

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        self.lib = C.CDLL(REF_SO)
        L = self.lib
        L.ref_parse_instance.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp,
                                         _dp, _dp]
        L.ref_build_dist.argtypes = [C.c_int, _dp, _dp, _dp, _dp]
        L.ref_zp_of.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_gen_durations.argtypes = [C.c_int, _dp, C.c_double, C.c_int, C.c_longlong, _dp]
        L.ref_compile.argtypes = [C.c_char_p, C.c_int, _ip, _ip]
        L.ref_rhh.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int,
                              C.c_char_p, C.c_long]
        L.ref_rhh.restype = C.c_long
        L.ref_eval_pairs.argtypes = [C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp,
                                     _dp, _ip, _ip, _ip, _ip, C.c_int, _dp, C.c_int, C.c_int,
                                     _lp, C.c_int, _dp, C.c_int]
        L.ref_mt_draws.argtypes = [C.c_ulonglong, C.c_int, C.c_longlong, C.c_int, _dp]

    def parse_instance(self, path, cordeau=False):
        cap = 2048
        arrs = [np.zeros(cap) for _ in range(6)]
        tmax = C.c_double()
        np_ = self.lib.ref_parse_instance(path.encode(), int(cordeau), cap,
                                          *[a.ctypes.data_as(_dp) for a in arrs], C.byref(tmax))
        if np_ < 0:
            raise RuntimeError("reference parser failed on " + path)
        return [a[:np_] for a in arrs], tmax.value

    def build_dist(self, x, y):
        n = len(x) - 1
        dist = np.zeros((n + 1) * (n + 1))
        d2d = np.zeros(n)
        self.lib.ref_build_dist(n, _d(x), _d(y), _d(dist), _d(d2d))
        return dist, d2d

    def zp_of(self, sd):
        zp = np.zeros(10)
        self.lib.ref_zp_of(sd.n, sd.tmax, _d(sd.scores), _d(sd.durations), _d(sd.open_t),
                           _d(sd.close_t), _d(sd.dist), _d(sd.dist_to_depot), _d(zp))
        return zp

    def gen_durations(self, durations, sigma, S, base_seed):
        d = np.ascontiguousarray(durations, dtype=np.float64)
        out = np.zeros((S, len(d)))
        self.lib.ref_gen_durations(len(d), _d(d), sigma, S, base_seed, _d(out))
        return out

    def compile(self, prefix):
        ops = np.zeros(4096, dtype=np.int32)
        args = np.zeros(8192, dtype=np.int32)
        L = self.lib.ref_compile(prefix.encode(), 4096, _i(ops), _i(args))
        if L < 0:
            raise RuntimeError("reference compile failed")
        return ops[:L].copy(), args[:2 * L].copy()

    def rhh(self, terminals, with_rmod, min_depth, max_depth, seed, pop):
        cap = 1 << 26
        buf = C.create_string_buffer(cap)
        n = self.lib.ref_rhh(",".join(terminals).encode(), int(with_rmod), min_depth, max_depth,
                             seed, pop, buf, cap)
        if n < 0:
            raise RuntimeError("rhh buffer too small")
        return buf.value.decode().splitlines()

    def eval_pairs(self, sd, zp, rules, sampled, T, masks, group_size=None, mask_group=None,
                   nthreads=None):
        P = rules.P
        sampled, group_size, masks, mask_group = _grouping(P, sampled, T, group_size, masks,
                                                          mask_group)
        out = np.zeros((P, T))
        self.lib.ref_eval_pairs(sd.n, sd.m, sd.tmax, _d(sd.scores), _d(sd.durations),
                                _d(sd.open_t), _d(sd.close_t), _d(sd.dist),
                                _d(sd.dist_to_depot), _d(np.asarray(zp, dtype=np.float64)),
                                _i(rules.ops), _i(rules.args), _i(rules.offsets),
                                _i(rules.lengths), P, _d(sampled), T, group_size, _l(masks),
                                mask_group, _d(out), nthreads or os.cpu_count() or 1)
        return out

    def mt_draws(self, seed, kind, arg, count):
        out = np.zeros(count)
        self.lib.ref_mt_draws(seed, kind, arg, count, _d(out))
        return out


def _ref_gp_replay(self, terminals, with_rmod, seed, pop, fits):
    """The reference's RHH + gp_step over len(fits) generations; returns the
    populations (prefix text) of generations 0..len(fits)."""
    L = self.lib
    L.ref_gp_replay.argtypes = [C.c_char_p, C.c_int, C.c_ulonglong, C.c_int, C.c_int, _dp,
                                C.c_char_p, C.c_long]
    L.ref_gp_replay.restype = C.c_long
    fits = np.ascontiguousarray(fits, dtype=np.float64)
    cap = 1 << 27
    buf = C.create_string_buffer(cap)
    n = L.ref_gp_replay(",".join(terminals).encode(), int(with_rmod), seed, pop, len(fits),
                        fits.ctypes.data_as(_dp), buf, cap)
    if n < 0:
        raise RuntimeError("replay buffer too small")
    out, cur = [], []
    for line in buf.value.decode().splitlines():
        if line == "#":
            out.append(cur)
            cur = []
        else:
            cur.append(line)
    return out


Reference.gp_replay = _ref_gp_replay


REF_GPU_SO = os.path.join(HERE, "_ref", "libsidr_ref_gpu.so")


class ReferenceGPU:
    """The reference's own GPU evaluator (engine/factory.cuh) as its Makefile
    builds it (oracle/_ref/libsidr_ref_gpu.so): used to show where that build
    and the CPU simulator differ.  Needs a CUDA device."""

    def __init__(self):
        if not os.path.exists(REF_GPU_SO):
            raise FileNotFoundError(REF_GPU_SO)
        self.lib = C.CDLL(REF_GPU_SO)
        self.lib.ref_gpu_evaluate_grouped_masks.argtypes = (
            [C.c_int, C.c_int, C.c_double] + [_dp] * 7 + [_ip] * 4 +
            [C.c_int, _dp, C.c_int, C.c_int, C.c_int, C.c_int, _lp, _dp])

    def evaluate_grouped_masks(self, sd, zp, rules, grouped, G, T, group_size, mask_group,
                               masks):
        keep = [np.ascontiguousarray(a, dtype=np.float64) for a in
                (sd.scores, sd.durations, sd.open_t, sd.close_t, sd.dist, sd.dist_to_depot, zp,
                 grouped)]
        ints = [np.ascontiguousarray(a, dtype=np.int32) for a in
                (rules.ops, rules.args, rules.offsets, rules.lengths)]
        mk = np.ascontiguousarray(masks, dtype=np.int64).reshape(-1)
        out = np.zeros((rules.P, T))
        st = self.lib.ref_gpu_evaluate_grouped_masks(
            sd.n, sd.m, sd.tmax, *[_d(a) for a in keep[:7]], *[a.ctypes.data_as(_ip) for a in ints],
            rules.P, _d(keep[7]), G, T, group_size, mask_group, mk.ctypes.data_as(_lp), _d(out))
        if st != 0:
            raise ValueError("input outside the reference kernel's bounds")
        return out

    def evaluate(self, sd, zp, rules, sampled, N, mask):
        return self.evaluate_grouped_masks(sd, zp, rules, sampled, 1, N, max(rules.P, 1),
                                           max(rules.P, 1), mask)
