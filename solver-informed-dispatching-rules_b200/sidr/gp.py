"""Python front end of the host GP loop (include/sidr_gp.h): the reference's
GP (engine/gp.hpp) on flat prefix-order rules in C++, evaluated by the B200
evaluator."""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import _Keep, _check, load
from .rules import PackedRules


class _Cfg(C.Structure):
    _fields_ = [("population", C.c_int32), ("generations", C.c_int32), ("max_depth", C.c_int32),
                ("min_depth", C.c_int32), ("tournament", C.c_int32), ("elitism", C.c_int32),
                ("crossover_rate", C.c_double), ("mutation_rate", C.c_double),
                ("reproduction_rate", C.c_double), ("train_samples", C.c_int32),
                ("test_samples", C.c_int32), ("with_rmod", C.c_int32)]


class _Result(C.Structure):
    _fields_ = [("eval_seconds", C.c_double), ("host_seconds", C.c_double),
                ("evaluations", C.c_int64)]


class _SampleStats(C.Structure):
    _fields_ = [("pairs", C.c_int64), ("host_pairs", C.c_int64)]


def _lib():
    L = load()
    if not getattr(L, "_gp_ready", False):
        L.sidr_gp_default_config.argtypes = [C.POINTER(_Cfg)]
        L.sidr_gp_create.argtypes = [C.POINTER(_Cfg), C.c_char_p, C.c_uint64, C.POINTER(C.c_void_p)]
        L.sidr_gp_destroy.argtypes = [C.c_void_p]
        L.sidr_gp_population_text.argtypes = [C.c_void_p, C.c_char_p, C.c_int64]
        L.sidr_gp_population_text.restype = C.c_int64
        ip = C.POINTER(C.c_int32)
        L.sidr_gp_population_packed.argtypes = [C.c_void_p, ip, ip, ip, ip, C.POINTER(C.c_int64)]
        L.sidr_gp_step.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        L.sidr_gp_generation.argtypes = [C.c_void_p]
        L.sidr_gp_generation.restype = C.c_int64
        L.sidr_gp_checkpoint.argtypes = [C.c_void_p, C.c_char_p, C.c_int64]
        L.sidr_gp_checkpoint.restype = C.c_int64
        L.sidr_gp_restore.argtypes = [C.c_char_p, C.POINTER(C.c_void_p)]
        dp = C.POINTER(C.c_double)
        L.sidr_gen_durations.argtypes = [C.c_int32, dp, C.c_double, C.c_int32, C.c_int64, dp]
        from . import _Inst
        L.sidr_gp_run_batched.argtypes = [C.c_void_p, C.POINTER(_Inst), C.POINTER(_Cfg), C.c_char_p,
                                          C.POINTER(C.c_int64), C.c_int32, C.c_int64, C.c_int64,
                                          dp, dp, C.c_char_p, C.c_int64, C.POINTER(_Result)]
        L.sidr_gp_run_multi.argtypes = [C.POINTER(_Inst), dp, C.c_int32, C.POINTER(_Cfg), C.c_char_p,
                                        C.POINTER(C.c_int64), C.c_int32, C.c_int64, C.c_int64,
                                        C.c_int32, C.c_int32, dp, dp, C.c_char_p, C.c_int64,
                                        C.POINTER(_Result)]
        L.sidr_gen_durations_device.argtypes = [C.c_int32, C.c_int32, dp, C.c_double, C.c_int32,
                                                C.c_int64, C.c_void_p, C.c_int32,
                                                C.POINTER(_SampleStats)]
        L.sidr_sample_dd_eval.argtypes = [C.c_int32, dp, dp, C.c_int32, C.c_int32, dp]
        vp = C.c_void_p
        L.sidr_gp_batched_create.argtypes = [vp, C.POINTER(_Inst), C.POINTER(_Cfg), C.c_char_p,
                                             C.POINTER(C.c_int64), C.c_int32, C.c_int64, C.c_int64,
                                             C.POINTER(vp)]
        L.sidr_gp_batched_step.argtypes = [vp, C.c_int32]
        L.sidr_gp_batched_generation.argtypes = [vp]
        L.sidr_gp_batched_generation.restype = C.c_int64
        L.sidr_gp_batched_checkpoint.argtypes = [vp, C.c_char_p, C.c_int64]
        L.sidr_gp_batched_checkpoint.restype = C.c_int64
        L.sidr_gp_batched_restore.argtypes = [vp, C.POINTER(_Inst), C.c_char_p, C.POINTER(vp)]
        L.sidr_gp_batched_finish.argtypes = [vp, dp, dp, C.c_char_p, C.c_int64, C.POINTER(_Result)]
        L.sidr_gp_batched_destroy.argtypes = [vp]
        L._gp_ready = True
    return L


def config(**kw) -> _Cfg:
    """EvolutionConfig defaults (engine/gp.hpp:20-34) with overrides."""
    c = _Cfg()
    _lib().sidr_gp_default_config(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Session:
    """One seed's population (ramped half-and-half with Mt19937(seed))."""

    def __init__(self, terminals: Sequence[str], seed: int, **cfg):
        self.cfg = config(**cfg)
        h = C.c_void_p()
        _check(_lib().sidr_gp_create(C.byref(self.cfg), ",".join(terminals).encode(), seed,
                                     C.byref(h)))
        self.h = h.value

    def text(self) -> List[str]:
        L = _lib()
        n = L.sidr_gp_population_text(self.h, None, 0)
        buf = C.create_string_buffer(int(n))
        L.sidr_gp_population_text(self.h, buf, n)
        return buf.value.decode().splitlines()

    def packed(self) -> PackedRules:
        L = _lib()
        nn = C.c_int64()
        _check(L.sidr_gp_population_packed(self.h, None, None, None, None, C.byref(nn)))
        P = self.cfg.population
        ops = np.zeros(nn.value, np.int32)
        args = np.zeros(2 * nn.value, np.int32)
        off = np.zeros(P, np.int32)
        ln = np.zeros(P, np.int32)
        ip = C.POINTER(C.c_int32)
        _check(L.sidr_gp_population_packed(self.h, ops.ctypes.data_as(ip), args.ctypes.data_as(ip),
                                           off.ctypes.data_as(ip), ln.ctypes.data_as(ip),
                                           C.byref(nn)))
        return PackedRules(ops, args, off, ln)

    def step(self, fitness) -> None:
        f = np.ascontiguousarray(fitness, dtype=np.float64)
        _check(_lib().sidr_gp_step(self.h, f.ctypes.data_as(C.POINTER(C.c_double))))

    @property
    def generation(self) -> int:
        """gp_step calls so far."""
        return int(_lib().sidr_gp_generation(self.h))

    def checkpoint(self) -> str:
        """The session's whole state as text (sidr_gp_checkpoint)."""
        L = _lib()
        n = L.sidr_gp_checkpoint(self.h, None, 0)
        buf = C.create_string_buffer(int(n))
        L.sidr_gp_checkpoint(self.h, buf, n)
        return buf.value.decode()

    @classmethod
    def restore(cls, text: str) -> "Session":
        """A session that continues exactly as the checkpointed one would."""
        h = C.c_void_p()
        _check(_lib().sidr_gp_restore(text.encode(), C.byref(h)))
        s = cls.__new__(cls)
        s.h = h.value
        v = text.splitlines()[1].split()[1:]
        s.cfg = config(population=int(v[0]), generations=int(v[1]), max_depth=int(v[2]),
                       min_depth=int(v[3]), tournament=int(v[4]), elitism=int(v[5]),
                       crossover_rate=float.fromhex(v[6]), mutation_rate=float.fromhex(v[7]),
                       reproduction_rate=float.fromhex(v[8]), train_samples=int(v[9]),
                       test_samples=int(v[10]), with_rmod=int(v[11]))
        return s

    def close(self):
        if getattr(self, "h", None):
            _lib().sidr_gp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_durations(durations, sigma: float, S: int, base_seed: int) -> np.ndarray:
    d = np.ascontiguousarray(durations, dtype=np.float64)
    out = np.zeros((S, len(d)))
    dp = C.POINTER(C.c_double)
    _check(_lib().sidr_gen_durations(len(d), d.ctypes.data_as(dp), sigma, S, base_seed,
                                     out.ctypes.data_as(dp)))
    return out


def gen_durations_device(durations, sigma: float, S: int, base_seed: int, device: int = 0,
                         out_ptr: int = 0):
    """sidr_gen_durations_device: gen_durations on the GPU, bit-identical to
    gen_durations.  Returns ([S, n] array, stats dict); with out_ptr (a device
    pointer to S * n doubles on `device`) the durations are written there and
    the array is None."""
    d = np.ascontiguousarray(durations, dtype=np.float64)
    st = _SampleStats()
    dp = C.POINTER(C.c_double)
    if out_ptr:
        _check(_lib().sidr_gen_durations_device(device, len(d), d.ctypes.data_as(dp), sigma, S, base_seed,
                                                C.c_void_p(out_ptr), 1, C.byref(st)))
        out = None
    else:
        out = np.zeros((S, len(d)))
        _check(_lib().sidr_gen_durations_device(device, len(d), d.ctypes.data_as(dp), sigma, S, base_seed,
                                                C.c_void_p(out.ctypes.data), 0, C.byref(st)))
    return out, {"pairs": st.pairs, "host_pairs": st.host_pairs}


def sample_dd_eval(u1, u2, on_device: bool = True, device: int = 0) -> np.ndarray:
    """sidr_sample_dd_eval: [k, 9] = log hi, lo, second candidate, sin hi, lo,
    second, cos hi, lo, second of the sampler's double-double evaluation, by
    the device or the host build."""
    a = np.ascontiguousarray(u1, dtype=np.float64)
    b = np.ascontiguousarray(u2, dtype=np.float64)
    out = np.zeros((len(a), 9))
    dp = C.POINTER(C.c_double)
    _check(_lib().sidr_sample_dd_eval(device, a.ctypes.data_as(dp), b.ctypes.data_as(dp), len(a),
                                      int(on_device), out.ctypes.data_as(dp)))
    return out


@dataclass
class RunResult:
    best_test: np.ndarray
    best_train: np.ndarray  # [generations, n_seeds]
    best_rules: List[str]
    eval_seconds: float
    host_seconds: float
    evaluations: int


def run_batched(ctx, terminals: Sequence[str], mask, n_seeds: int, first_seed: int = 0,
                test_seed: int = 1000000, **cfg) -> RunResult:
    """exhaust_batched (engine/gp_engine.cu:131-203) on the B200 evaluator."""
    c = config(**cfg)
    k = _Keep()
    inst = k.inst(ctx.sd)
    bt = np.zeros(n_seeds)
    btr = np.zeros((c.generations, n_seeds))
    buf = C.create_string_buffer(1 << 22)
    res = _Result()
    dp = C.POINTER(C.c_double)
    _check(_lib().sidr_gp_run_batched(ctx.h, C.byref(inst), C.byref(c),
                                      ",".join(terminals).encode(), k.i64(mask), n_seeds,
                                      first_seed, test_seed, bt.ctypes.data_as(dp),
                                      btr.ctypes.data_as(dp), buf, 1 << 22, C.byref(res)))
    return RunResult(bt, btr, buf.value.decode().splitlines(), res.eval_seconds,
                     res.host_seconds, res.evaluations)


class Batched:
    """The seed-batched run one generation at a time (sidr_gp_batched_*):
    step, checkpoint to text, restore from it and finish with the results of
    run_batched.  The context must hold the instance the run evolves on."""

    def __init__(self, ctx, terminals: Sequence[str] = (), mask=None, n_seeds: int = 1,
                 first_seed: int = 0, test_seed: int = 1000000, _restore: str = None, **cfg):
        L = _lib()
        self.ctx = ctx
        k = _Keep()
        inst = k.inst(ctx.sd)
        h = C.c_void_p()
        if _restore is not None:
            _check(L.sidr_gp_batched_restore(ctx.h, C.byref(inst), _restore.encode(), C.byref(h)))
            lines = _restore.splitlines()
            self.n_seeds = int(lines[1].split()[1])
            self.generations = int(next(x for x in lines if x.startswith("config ")).split()[2])
        else:
            c = config(**cfg)
            _check(L.sidr_gp_batched_create(ctx.h, C.byref(inst), C.byref(c),
                                            ",".join(terminals).encode(), k.i64(mask), n_seeds,
                                            first_seed, test_seed, C.byref(h)))
            self.n_seeds, self.generations = n_seeds, c.generations
        self.h = h.value

    @classmethod
    def restore(cls, ctx, checkpoint: str) -> "Batched":
        """sidr_gp_batched_restore: a run that continues as the checkpointed one."""
        return cls(ctx, _restore=checkpoint)

    def step(self, generations: int = 1) -> None:
        _check(_lib().sidr_gp_batched_step(self.h, generations))

    @property
    def generation(self) -> int:
        return int(_lib().sidr_gp_batched_generation(self.h))

    def checkpoint(self) -> str:
        L = _lib()
        n = L.sidr_gp_batched_checkpoint(self.h, None, 0)
        buf = C.create_string_buffer(int(n))
        L.sidr_gp_batched_checkpoint(self.h, buf, n)
        return buf.value.decode()

    def finish(self) -> RunResult:
        bt = np.zeros(self.n_seeds)
        btr = np.zeros((self.generations, self.n_seeds))
        buf = C.create_string_buffer(1 << 22)
        res = _Result()
        dp = C.POINTER(C.c_double)
        _check(_lib().sidr_gp_batched_finish(self.h, bt.ctypes.data_as(dp), btr.ctypes.data_as(dp),
                                             buf, 1 << 22, C.byref(res)))
        return RunResult(bt, btr, buf.value.decode().splitlines(), res.eval_seconds,
                         res.host_seconds, res.evaluations)

    def close(self) -> None:
        if self.h:
            _lib().sidr_gp_batched_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_multi(sds, zps, terminals: Sequence[str], masks, n_seeds: int, first_seed: int = 0,
              test_seed: int = 1000000, shape: int = 1, device: int = 0, **cfg) -> RunResult:
    """Seed-batched GP runs on many instances at once, one multi-instance launch
    per generation (sidr_gp_run_multi): best_test [K, n_seeds], best_train
    [generations, K, n_seeds], best_rules in (instance, seed) order."""
    c = config(**cfg)
    k = _Keep()
    K = len(sds)
    from . import _Inst
    insts = (_Inst * K)(*[k.inst(sd) for sd in sds])
    z = np.ascontiguousarray(np.stack([np.asarray(v, dtype=np.float64) for v in zps]))
    m = np.ascontiguousarray(np.stack([np.asarray(v, dtype=np.int64) for v in masks]))
    bt = np.zeros((K, n_seeds))
    btr = np.zeros((c.generations, K, n_seeds))
    buf = C.create_string_buffer(1 << 22)
    res = _Result()
    dp = C.POINTER(C.c_double)
    _check(_lib().sidr_gp_run_multi(insts, z.ctypes.data_as(dp), K, C.byref(c),
                                    ",".join(terminals).encode(),
                                    m.ctypes.data_as(C.POINTER(C.c_int64)), n_seeds, first_seed,
                                    test_seed, shape, device, bt.ctypes.data_as(dp),
                                    btr.ctypes.data_as(dp), buf, 1 << 22, C.byref(res)))
    return RunResult(bt, btr, buf.value.decode().splitlines(), res.eval_seconds,
                     res.host_seconds, res.evaluations)
