"""Python front end of the surrogate model (include/sidr_surrogate.h): the
tensor-core GEMM and the 40 -> 256 -> 256 -> 1 MLP trained with Adam on the
device."""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _check, load

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_u16 = C.POINTER(C.c_uint16)

INPUTS, HIDDEN = 40, 256
PARAM_NAMES = ["W1", "b1", "W2", "b2", "w3", "b3"]
PARAM_SHAPES = {"W1": (HIDDEN, 48), "b1": (HIDDEN,), "W2": (HIDDEN, HIDDEN), "b2": (HIDDEN,),
                "w3": (HIDDEN,), "b3": (1,)}


def _lib():
    L = load()
    if not getattr(L, "_surrogate_ready", False):
        L.sidr_gemm_bf16.argtypes = [_u16, _u16, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                     _fp]
        L.sidr_mlp_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]
        L.sidr_mlp_destroy.argtypes = [C.c_void_p]
        L.sidr_mlp_param.argtypes = [C.c_void_p, C.c_int32, C.c_int32, _fp, _fp, C.POINTER(C.c_int64)]
        L.sidr_mlp_predict.argtypes = [C.c_void_p, _fp, C.c_int32, _fp]
        L.sidr_mlp_gradients.argtypes = [C.c_void_p, _fp, _fp, C.c_int32, _fp]
        L.sidr_mlp_train.argtypes = [C.c_void_p, _fp, _fp, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                     C.c_uint64, _fp]
        L.sidr_gemm_wait_check.argtypes = [C.c_int, C.c_uint32]
        L._surrogate_ready = True
    return L


def to_bf16_bits(x) -> np.ndarray:
    """Round-to-nearest-even FP32 -> BF16, as 16-bit patterns."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def gemm_wait_check(device: int = 0, wait_limit: int = 1000) -> int:
    """sidr_gemm_wait_check's status: SIDR_ERR_KERNEL (6) when the GEMM kernel,
    with its MMAs withheld, gave up its bounded waits and said so."""
    return int(_lib().sidr_gemm_wait_check(device, wait_limit))


def gemm_bf16(A_bits, B_bits, splits: int = 1, device: int = 0) -> np.ndarray:
    """C = A B^T on the tensor-core kernel; A [M x K], B [N x K] BF16 bits."""
    A = np.ascontiguousarray(A_bits, dtype=np.uint16)
    B = np.ascontiguousarray(B_bits, dtype=np.uint16)
    M, K = A.shape
    N = B.shape[0]
    out = np.zeros((M, N), np.float32)
    _check(_lib().sidr_gemm_bf16(A.ctypes.data_as(_u16), B.ctypes.data_as(_u16), M, N, K, splits,
                                 device, out.ctypes.data_as(_fp)))
    return out


class MLP:
    def __init__(self, seed: int = 0, device: int = 0):
        h = C.c_void_p()
        _check(_lib().sidr_mlp_create(device, seed, C.byref(h)))
        self.h = h.value

    def param(self, name: str):
        L = _lib()
        i = PARAM_NAMES.index(name)
        v = np.zeros(PARAM_SHAPES[name], np.float32)
        g = np.zeros(PARAM_SHAPES[name], np.float32)
        n = C.c_int64()
        _check(L.sidr_mlp_param(self.h, i, 0, v.ctypes.data_as(_fp), g.ctypes.data_as(_fp),
                                C.byref(n)))
        return v, g

    def set_param(self, name: str, values) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(PARAM_SHAPES[name])
        _check(_lib().sidr_mlp_param(self.h, PARAM_NAMES.index(name), 1, v.ctypes.data_as(_fp), None,
                                     None))

    def predict(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros(x.shape[0], np.float32)
        _check(_lib().sidr_mlp_predict(self.h, x.ctypes.data_as(_fp), x.shape[0],
                                       y.ctypes.data_as(_fp)))
        return y

    def gradients(self, x, t) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(_lib().sidr_mlp_gradients(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                         x.shape[0], C.byref(loss)))
        return loss.value

    def train(self, x, t, steps: int, batch: int = 1024, lr: float = 1e-3, seed: int = 0) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        loss = C.c_float()
        _check(_lib().sidr_mlp_train(self.h, x.ctypes.data_as(_fp), t.ctypes.data_as(_fp),
                                     x.shape[0], steps, batch, lr, seed, C.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None):
            _lib().sidr_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------ situations, phenotype

class _SgpCfg(C.Structure):
    _fields_ = [("screen", C.c_int32), ("train_steps", C.c_int32), ("batch", C.c_int32),
                ("lr", C.c_float), ("audit", C.c_int32), ("rho_min", C.c_double),
                ("history", C.c_int32), ("n_situations", C.c_int32),
                ("capture_scenarios", C.c_int32), ("max_cand", C.c_int32),
                ("model_seed", C.c_uint64), ("use_surrogate", C.c_int32), ("device", C.c_int32),
                ("selection", C.c_int32), ("target", C.c_int32), ("screen_fraction", C.c_double),
                ("distinct", C.c_int32)]


class _SgpResult(C.Structure):
    _fields_ = [("eval_seconds", C.c_double), ("model_seconds", C.c_double),
                ("host_seconds", C.c_double), ("evaluations", C.c_int64),
                ("generations_screened", C.c_int32), ("generations_fallback", C.c_int32)]


STRUCTS = {"sidr_sgp_config": _SgpCfg, "sidr_sgp_result": _SgpResult}


def _lib2():
    L = _lib()
    if not getattr(L, "_sgp_ready", False):
        from . import _Inst, _Rules
        from .gp import _Cfg
        L.sidr_capture_situations.argtypes = [C.c_void_p, C.POINTER(_Rules), _dp, C.c_int32,
                                              C.POINTER(C.c_int64), C.c_int32, C.c_int32, _dp, _ip, _ip]
        L.sidr_phenotype.argtypes = [C.POINTER(_Rules), _dp, _ip, _ip, C.c_int32, C.c_int32, C.c_int,
                                     _fp]
        L.sidr_sgp_default_config.argtypes = [C.POINTER(_SgpCfg)]
        L.sidr_sgp_run.argtypes = [C.c_void_p, C.POINTER(_Inst), C.POINTER(_Cfg), C.POINTER(_SgpCfg),
                                   C.c_char_p, C.POINTER(C.c_int64), C.c_uint64, C.c_int64, _dp, _dp,
                                   _dp, _dp, C.c_char_p, C.c_int64, C.POINTER(_SgpResult)]
        L.sidr_sgp_run_resumable.argtypes = [
            C.c_void_p, C.POINTER(_Inst), C.POINTER(_Cfg), C.POINTER(_SgpCfg), C.c_char_p,
            C.POINTER(C.c_int64), C.c_uint64, C.c_int64, C.c_char_p, C.c_int32, C.c_int32,
            C.POINTER(C.c_int32), _dp, _dp, _dp, _dp, C.c_char_p, C.c_int64, C.POINTER(_SgpResult)]
        L.sidr_mlp_state.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_float),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        L.sidr_sgp_run_multi.argtypes = [C.POINTER(_Inst), _dp, C.c_int32, C.POINTER(_Cfg),
                                         C.POINTER(_SgpCfg), C.c_char_p, C.POINTER(C.c_int64),
                                         C.c_int32, C.c_int64, C.c_int64, C.c_int32, _dp, _dp, _dp,
                                         C.c_char_p, C.c_int64, C.POINTER(_SgpResult)]
        L.sidr_sgp_run_multi_resumable.argtypes = [
            C.POINTER(_Inst), _dp, C.c_int32, C.POINTER(_Cfg), C.POINTER(_SgpCfg), C.c_char_p,
            C.POINTER(C.c_int64), C.c_int32, C.c_int64, C.c_int64, C.c_int32, C.c_char_p, C.c_int32,
            C.c_int32, C.POINTER(C.c_int32), _dp, _dp, _dp, C.c_char_p, C.c_int64, C.POINTER(_SgpResult)]
        L._sgp_ready = True
    return L


def capture_situations(ctx, rule, sampled, mask, max_decisions: int = 64, max_cand: int = 64):
    """Terminal tables of every decision of `rule` (PackedRules with P = 1) on
    the scenarios: terms [S, D, C, 61], cust [S, D, C], info [S, D, 2]."""
    from . import _Keep
    L = _lib2()
    k = _Keep()
    smp = np.ascontiguousarray(sampled, dtype=np.float64)
    S = smp.shape[0]
    terms = np.zeros((S, max_decisions, max_cand, 61))
    cust = np.zeros((S, max_decisions, max_cand), np.int32)
    info = np.zeros((S, max_decisions, 2), np.int32)
    r = k.rules(rule)
    _check(L.sidr_capture_situations(ctx.h, C.byref(r), smp.ctypes.data_as(_dp), S, k.i64(mask),
                                     max_decisions, max_cand, terms.ctypes.data_as(_dp),
                                     cust.ctypes.data_as(_ip), info.ctypes.data_as(_ip)))
    return terms, cust, info


def phenotype(rules, terms, ncand, ref, device: int = 0) -> np.ndarray:
    """features [P, n_sit + 8] of the rules on situations terms [n_sit, C, 61]."""
    from . import _Keep
    L = _lib2()
    k = _Keep()
    t = np.ascontiguousarray(terms, dtype=np.float64)
    n_sit, max_cand = t.shape[0], t.shape[1]
    nc = np.ascontiguousarray(ncand, dtype=np.int32)
    rf = np.ascontiguousarray(ref, dtype=np.int32)
    out = np.zeros((rules.P, n_sit + 8), np.float32)
    r = k.rules(rules)
    _check(L.sidr_phenotype(C.byref(r), t.ctypes.data_as(_dp), nc.ctypes.data_as(_ip),
                            rf.ctypes.data_as(_ip), n_sit, max_cand, device,
                            out.ctypes.data_as(_fp)))
    return out


def sgp_config(**kw) -> _SgpCfg:
    c = _SgpCfg()
    _lib2().sidr_sgp_default_config(C.byref(c))
    for k_, v in kw.items():
        setattr(c, k_, v)
    return c


def sgp_run(ctx, terminals, mask, seed: int = 0, test_seed: int = 1000000,
            gp: Optional[dict] = None, checkpoint: Optional[str] = None, every: int = 1,
            stop_after: int = -1, **sgp_kw) -> dict:
    """The surrogate-assisted GP (use_surrogate=0: the same driver breeding
    plainly); per-generation best train fitness, held-out score, audit rho and
    wall clock.  checkpoint: a file path (sidr_sgp_run_resumable) the run's
    state is written to every `every` generations and resumed from when it
    exists; stop_after >= 0 returns after that many generations of this call
    ("finished" False, outputs of the generations so far filled)."""
    from . import _Keep
    from .gp import config
    L = _lib2()
    c = config(**(gp or {}))
    s = sgp_config(**sgp_kw)
    k = _Keep()
    inst = k.inst(ctx.sd)
    G = c.generations
    bt, ho, rho, secs = np.zeros(G), np.zeros(G), np.zeros(G), np.zeros(G)
    buf = C.create_string_buffer(1 << 16)
    res = _SgpResult()
    fin = C.c_int32(1)
    if checkpoint is None:
        _check(L.sidr_sgp_run(ctx.h, C.byref(inst), C.byref(c), C.byref(s),
                              ",".join(terminals).encode(), k.i64(mask), seed, test_seed,
                              bt.ctypes.data_as(_dp), ho.ctypes.data_as(_dp), rho.ctypes.data_as(_dp),
                              secs.ctypes.data_as(_dp), buf, 1 << 16, C.byref(res)))
    else:
        _check(L.sidr_sgp_run_resumable(ctx.h, C.byref(inst), C.byref(c), C.byref(s),
                                        ",".join(terminals).encode(), k.i64(mask), seed, test_seed,
                                        str(checkpoint).encode(), every, stop_after, C.byref(fin),
                                        bt.ctypes.data_as(_dp), ho.ctypes.data_as(_dp),
                                        rho.ctypes.data_as(_dp), secs.ctypes.data_as(_dp), buf,
                                        1 << 16, C.byref(res)))
    return {"finished": bool(fin.value), "best_train": bt, "held_out": ho, "rho": rho, "seconds": secs,
            "best_rule": buf.value.decode(), "eval_seconds": res.eval_seconds,
            "model_seconds": res.model_seconds, "host_seconds": res.host_seconds,
            "evaluations": res.evaluations, "screened": res.generations_screened,
            "fallback": res.generations_fallback}


def sgp_run_multi(sds, zps, terminals, masks, n_seeds: int, first_seed: int = 0,
                  test_seed: int = 1000000, shape: int = -1, gp: Optional[dict] = None,
                  checkpoint: Optional[str] = None, every: int = 1, stop_after: int = -1,
                  **sgp_kw) -> dict:
    """sidr_sgp_run_multi: K instances x n_seeds surrogate-screened GP runs,
    one multi-instance launch per generation; per generation and population
    (e = k * n_seeds + s) the best train fitness, held-out score and audit
    rho, shaped [G, K, n_seeds].  checkpoint / every / stop_after: as in
    sgp_run (sidr_sgp_run_multi_resumable)."""
    from . import _Inst, _Keep
    from .gp import config
    L = _lib2()
    c = config(**(gp or {}))
    s = sgp_config(**sgp_kw)
    k = _Keep()
    K = len(sds)
    insts = (_Inst * K)(*[k.inst(sd) for sd in sds])
    z = np.ascontiguousarray(np.stack([np.asarray(v, dtype=np.float64) for v in zps]))
    m = np.ascontiguousarray(np.stack([np.asarray(v, dtype=np.int64) for v in masks]))
    G = c.generations
    bt, ho, rho = (np.zeros((G, K, n_seeds)) for _ in range(3))
    res = _SgpResult()
    cap = 1 << 24
    buf = C.create_string_buffer(cap)
    fin = C.c_int32(1)
    if checkpoint is None:
        _check(L.sidr_sgp_run_multi(insts, z.ctypes.data_as(_dp), K, C.byref(c), C.byref(s),
                                    ",".join(terminals).encode(), m.ctypes.data_as(C.POINTER(C.c_int64)),
                                    n_seeds, first_seed, test_seed, shape, bt.ctypes.data_as(_dp),
                                    ho.ctypes.data_as(_dp), rho.ctypes.data_as(_dp), buf, cap,
                                    C.byref(res)))
    else:
        _check(L.sidr_sgp_run_multi_resumable(
            insts, z.ctypes.data_as(_dp), K, C.byref(c), C.byref(s), ",".join(terminals).encode(),
            m.ctypes.data_as(C.POINTER(C.c_int64)), n_seeds, first_seed, test_seed, shape,
            str(checkpoint).encode(), every, stop_after, C.byref(fin), bt.ctypes.data_as(_dp),
            ho.ctypes.data_as(_dp), rho.ctypes.data_as(_dp), buf, cap, C.byref(res)))
    return {"finished": bool(fin.value), "best_train": bt, "held_out": ho, "rho": rho,
            "best_rules": buf.value.decode().splitlines(), "eval_seconds": res.eval_seconds,
            "model_seconds": res.model_seconds, "host_seconds": res.host_seconds,
            "evaluations": res.evaluations, "screened": res.generations_screened,
            "fallback": res.generations_fallback}


def _main(argv=None) -> int:
    """python -m sidr.surrogate [--rows R] [--steps K] [--batch B]: trains the
    model on R random 40-feature rows for K Adam steps of B rows and prints
    the step rate and the tensor-core GEMM throughput it implies."""
    import argparse
    import json
    import time
    ap = argparse.ArgumentParser(prog="python -m sidr.surrogate")
    ap.add_argument("--rows", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--batch", type=int, default=1024)
    a = ap.parse_args(argv)
    rng = np.random.default_rng(0)
    x = rng.random((a.rows, INPUTS), dtype=np.float32)
    t = (x[:, :8].sum(axis=1) - 4.0).astype(np.float32)
    m = MLP(seed=1)
    m.train(x, t, steps=3, batch=a.batch)  # warm-up
    t0 = time.perf_counter()
    loss = m.train(x, t, steps=a.steps, batch=a.batch)
    dt = time.perf_counter() - t0
    # GEMM FLOPs per step: forward 2B(48*256 + 256*256), backward dW2, dH1, dW1
    flops = 2.0 * a.batch * (48 * 256 + 256 * 256) + 2.0 * a.batch * (256 * 256 * 2 + 256 * 48)
    print(json.dumps({"steps": a.steps, "batch": a.batch, "seconds": dt,
                      "steps_per_s": a.steps / dt, "gemm_tflops": flops * a.steps / dt / 1e12,
                      "final_loss": loss}))
    m.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(_main())
