"""Python front end of the B200 rule x scenario evaluator (libsidr_b200.so).

A thin ctypes layer over the C-ABI declared in include/sidr.h, shaped like the
reference's evaluator API (augustompm/solver-informed-dispatching-rules,
engine/factory.cuh:124-217):

    ctx = Context(simdata, zp, device=0)            # FactoryContext(sd, zp)
    ctx.evaluate(rules, sampled, N, mask)            # -> [P, N]
    ctx.evaluate_grouped(rules, grouped, G, T, group_size, mask)
    ctx.evaluate_grouped_masks(rules, grouped, T, group_size, mask_group, masks)

plus device-resident batches (``ctx.batch(...)``) for repeated launches.
There is no CPU fallback: if the native library is missing, importing the
evaluator raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .instance import SimData  # noqa: F401
from .rules import N_TERMS, PackedRules  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "libsidr_b200.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class SidrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"sidr status {status}: {msg}")
        self.status = status


class _Inst(C.Structure):
    _fields_ = [("n", C.c_int32), ("m", C.c_int32), ("tmax", C.c_double), ("scores", _dp),
                ("durations", _dp), ("open_t", _dp), ("close_t", _dp), ("dist", _dp),
                ("dist_to_depot", _dp)]


class _Rules(C.Structure):
    _fields_ = [("ops", _ip), ("args", _ip), ("offsets", _ip), ("lengths", _ip), ("P", C.c_int32),
                ("n_nodes", C.c_int64)]


class _Counts(C.Structure):
    _fields_ = [("decisions", C.c_int64), ("candidates", C.c_int64), ("scan_iters", C.c_int64),
                ("heavy_iters", C.c_int64), ("hop_iters", C.c_int64), ("fp64_ops", C.c_int64)]


# ctypes mirrors of the C structs, checked against include/sidr.h by the tests.
STRUCTS = {"sidr_instance_desc": _Inst, "sidr_rules_desc": _Rules, "sidr_counts": _Counts}


EXPORTS = [
    "sidr_last_error", "sidr_status_string", "sidr_version", "sidr_zstats", "sidr_ctx_create",
    "sidr_ctx_destroy", "sidr_evaluate", "sidr_evaluate_grouped", "sidr_evaluate_grouped_masks",
    "sidr_batch_create", "sidr_batch_run", "sidr_batch_read", "sidr_batch_fitness",
    "sidr_batch_device_out", "sidr_batch_destroy", "sidr_batch_set_counting", "sidr_batch_counts",
    "sidr_kernel_launches", "sidr_rules_check", "sidr_last_transfer_bytes", "sidr_fp64_peak",
    "sidr_evaluate_static", "sidr_multi_create", "sidr_multi_autotune", "sidr_multi_set_shape",
    "sidr_multi_capture", "sidr_multi_run", "sidr_multi_read", "sidr_multi_destroy",
    "sidr_libm_eval", "sidr_batch_guard_check", "sidr_libm_pow", "sidr_multi_autotune_sampled",
    "sidr_batch_set_shape", "sidr_batch_autotune_sampled", "sidr_ctx_set_shape",
    "sidr_multi_autotune_classes", "sidr_multi_set_class_shape", "sidr_multi_shapes",
    "sidr_atrisk_table_check",
]

_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    """Loads libsidr_b200.so; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run solver-informed-dispatching-rules_b200/"
                          "build.py (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.sidr_last_error.restype = C.c_char_p
    L.sidr_status_string.restype = C.c_char_p
    L.sidr_status_string.argtypes = [C.c_int]
    L.sidr_zstats.argtypes = [C.POINTER(_Inst), _dp]
    L.sidr_ctx_create.argtypes = [C.POINTER(_Inst), _dp, C.c_int, C.POINTER(C.c_void_p)]
    L.sidr_ctx_destroy.argtypes = [C.c_void_p]
    L.sidr_evaluate.argtypes = [C.c_void_p, C.POINTER(_Rules), _dp, C.c_int32, _lp, _dp]
    L.sidr_evaluate_grouped.argtypes = [C.c_void_p, C.POINTER(_Rules), _dp, C.c_int32, C.c_int32,
                                        C.c_int32, _lp, _dp]
    L.sidr_evaluate_grouped_masks.argtypes = [C.c_void_p, C.POINTER(_Rules), _dp, C.c_int32,
                                              C.c_int32, C.c_int32, C.c_int32, _lp, _dp]
    L.sidr_batch_create.argtypes = [C.c_void_p, C.POINTER(_Rules), _dp, C.c_int32, C.c_int32,
                                    C.c_int32, C.c_int32, _lp, C.POINTER(C.c_void_p)]
    L.sidr_batch_run.argtypes = [C.c_void_p, C.c_void_p]
    L.sidr_batch_read.argtypes = [C.c_void_p, _dp]
    L.sidr_batch_fitness.argtypes = [C.c_void_p, _dp]
    L.sidr_batch_device_out.argtypes = [C.c_void_p]
    L.sidr_batch_device_out.restype = C.c_void_p
    L.sidr_batch_destroy.argtypes = [C.c_void_p]
    L.sidr_batch_set_counting.argtypes = [C.c_void_p, C.c_int]
    L.sidr_batch_counts.argtypes = [C.c_void_p, C.POINTER(_Counts)]
    L.sidr_batch_guard_check.argtypes = [C.c_void_p]
    L.sidr_batch_set_shape.argtypes = [C.c_void_p, C.c_int32]
    L.sidr_ctx_set_shape.argtypes = [C.c_void_p, C.c_int32]
    L.sidr_batch_autotune_sampled.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                              C.POINTER(C.c_float)]
    L.sidr_libm_pow.argtypes = [_dp, _dp, C.c_int64, C.c_int, _dp]
    L.sidr_kernel_launches.restype = C.c_int64
    L.sidr_rules_check.argtypes = [C.POINTER(_Rules), _lp, C.c_int32, C.POINTER(C.c_int32)]
    L.sidr_last_transfer_bytes.argtypes = [_lp, _lp]
    L.sidr_fp64_peak.argtypes = [C.c_int, C.c_int, _dp]
    L.sidr_evaluate_static.argtypes = [C.POINTER(_Inst), _dp, C.POINTER(_Rules), _dp, C.c_int32,
                                       C.c_int32, C.c_int32, C.c_int32, _lp, C.c_int32, _dp]
    _lib = L
    return L


def _check(st: int) -> None:
    if st != 0:
        L = load()
        raise SidrError(st, L.sidr_last_error().decode())


def _d(a):
    return a.ctypes.data_as(_dp)


class _Keep:
    """Holds contiguous copies alive for the duration of a native call."""

    def __init__(self):
        self.refs = []

    def f64(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.refs.append(a)
        return a.ctypes.data_as(_dp)

    def i32(self, a):
        a = np.ascontiguousarray(a, dtype=np.int32)
        self.refs.append(a)
        return a.ctypes.data_as(_ip)

    def i64(self, a):
        a = np.ascontiguousarray(a, dtype=np.int64)
        self.refs.append(a)
        return a.ctypes.data_as(_lp)

    def inst(self, sd) -> _Inst:
        return _Inst(sd.n, sd.m, float(sd.tmax), self.f64(sd.scores), self.f64(sd.durations),
                     self.f64(sd.open_t), self.f64(sd.close_t), self.f64(sd.dist),
                     self.f64(sd.dist_to_depot))

    def rules(self, r) -> _Rules:
        return _Rules(self.i32(r.ops), self.i32(r.args), self.i32(r.offsets), self.i32(r.lengths),
                      r.P, int(len(r.ops)))


def zstats(sd) -> np.ndarray:
    """zp_of(sd): host computation through the C-ABI."""
    L = load()
    k = _Keep()
    zp = np.zeros(10)
    inst = k.inst(sd)
    _check(L.sidr_zstats(C.byref(inst), _d(zp)))
    return zp


def atrisk_table_check(sd, seed: int = 0):
    """sidr_atrisk_table_check: (points checked, mismatches) of ATRISK's
    per-pair step functions against the classification they stand for."""
    L = load()
    L.sidr_atrisk_table_check.argtypes = [C.POINTER(_Inst), C.c_int32, C.POINTER(C.c_int64),
                                          C.POINTER(C.c_int64)]
    k = _Keep()
    inst = k.inst(sd)
    a, b = C.c_int64(), C.c_int64()
    _check(L.sidr_atrisk_table_check(C.byref(inst), seed, C.byref(a), C.byref(b)))
    return a.value, b.value


def rules_check(rules, masks, mask_group=None) -> int:
    """Validates and compiles rules on the host; returns the per-lane value
    rows the largest program needs."""
    L = load()
    k = _Keep()
    masks = np.ascontiguousarray(masks, dtype=np.int64).reshape(-1)
    r = k.rules(rules)
    rows = C.c_int32()
    _check(L.sidr_rules_check(C.byref(r), k.i64(masks), mask_group or max(rules.P, 1),
                              C.byref(rows)))
    return rows.value


def kernel_launches() -> int:
    return int(load().sidr_kernel_launches())


def last_transfer_bytes():
    """(h2d, d2h) bytes of this thread's last evaluate* call."""
    a, b = C.c_int64(), C.c_int64()
    _check(load().sidr_last_transfer_bytes(C.byref(a), C.byref(b)))
    return a.value, b.value


def fp64_peak(device: int = 0, reps: int = 5) -> float:
    """Measured FP64 pipe throughput of the device (operations/s)."""
    v = C.c_double()
    _check(load().sidr_fp64_peak(device, reps, C.byref(v)))
    return v.value


LIBM_FUNCS = {"erf": 0, "erfc": 1, "exp": 2}


def libm_eval(fn: str, x, device: int = 0) -> np.ndarray:
    """The evaluator's device erf / erfc / exp on an array (diagnostic)."""
    L = load()
    L.sidr_libm_eval.argtypes = [C.c_int32, _dp, C.c_int64, C.c_int, _dp]
    a = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(a)
    _check(L.sidr_libm_eval(LIBM_FUNCS[fn], _d(a), a.size, device, _d(out)))
    return out


def libm_pow(x, y, device: int = 0) -> np.ndarray:
    """The evaluator's device pow (glibc's, restated) on host arrays."""
    a = np.ascontiguousarray(x, dtype=np.float64)
    b = np.ascontiguousarray(y, dtype=np.float64)
    if a.shape != b.shape:
        raise ValueError("x and y differ in shape")
    out = np.zeros_like(a)
    _check(load().sidr_libm_pow(_d(a), _d(b), a.size, device, _d(out)))
    return out


STATIC_SCRATCH_BYTES = 16 << 20  # SIDR_STATIC_SCRATCH_BYTES
STATIC_MAX_N = 128               # SIDR_STATIC_MAX_N


def evaluate_static(sd, zp, rules, grouped_sampled, G, T, group_size, mask_group, masks,
                    device: int = 0) -> np.ndarray:
    """sidr_evaluate_static: the grouped, multi-mask evaluation with no device
    allocation (all device data in the library's fixed static array); every
    argument is a host array.  Returns [P, T] scores."""
    k = _Keep()
    inst = k.inst(sd)
    r = k.rules(rules)
    out = np.zeros((rules.P, T))
    _check(load().sidr_evaluate_static(C.byref(inst), k.f64(zp), C.byref(r),
                                       k.f64(grouped_sampled), G, T, group_size, mask_group,
                                       k.i64(masks), device, _d(out)))
    return out


class Batch:
    """Rules, scenarios and masks resident in HBM (sidr_batch_*)."""

    def __init__(self, ctx: "Context", handle: int, P: int, T: int):
        self.ctx, self.h, self.P, self.T = ctx, handle, P, T

    def run(self, stream: int = 0) -> None:
        _check(load().sidr_batch_run(self.h, C.c_void_p(stream)))

    def read(self) -> np.ndarray:
        out = np.zeros((self.P, self.T))
        _check(load().sidr_batch_read(self.h, _d(out)))
        return out

    def fitness(self) -> np.ndarray:
        out = np.zeros(self.P)
        _check(load().sidr_batch_fitness(self.h, _d(out)))
        return out

    def device_out(self) -> int:
        return int(load().sidr_batch_device_out(self.h) or 0)

    def set_counting(self, on: bool) -> None:
        _check(load().sidr_batch_set_counting(self.h, int(on)))

    # warps per block, resident blocks per SM, lanes per (rule, scenario) pair
    SHAPES = ((4, 4, 32), (4, 5, 32), (4, 4, 16), (4, 5, 16))

    def set_shape(self, shape: int) -> None:
        """sidr_batch_set_shape: the block shape of the following runs."""
        _check(load().sidr_batch_set_shape(self.h, shape))

    def autotune_sampled(self, stride: int = 16, reps: int = 1):
        """sidr_batch_autotune_sampled: times each block shape on every
        stride-th rule and keeps the faster; returns (shape, [ms per shape]).
        The sampled rules' scores are overwritten: run the batch afterwards."""
        ch = C.c_int32()
        ms = (C.c_float * len(self.SHAPES))()
        _check(load().sidr_batch_autotune_sampled(self.h, reps, stride, C.byref(ch), ms))
        return ch.value, [float(x) for x in ms]

    def guard_check(self) -> int:
        """sidr_batch_guard_check: the kernel's rule-record guard, tripped on
        purpose; returns the status (SIDR_ERR_KERNEL expected)."""
        return int(load().sidr_batch_guard_check(self.h))

    def counts(self) -> dict:
        c = _Counts()
        _check(load().sidr_batch_counts(self.h, C.byref(c)))
        return {k: int(getattr(c, k)) for k, _ in _Counts._fields_}

    def close(self) -> None:
        if self.h:
            load().sidr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """FactoryContext(sd, zp) on one device."""

    def __init__(self, sd, zp=None, device: int = 0):
        L = load()
        self.sd = sd
        self.zp = np.ascontiguousarray(zstats(sd) if zp is None else zp, dtype=np.float64)
        k = _Keep()
        inst = k.inst(sd)
        h = C.c_void_p()
        _check(L.sidr_ctx_create(C.byref(inst), _d(self.zp), device, C.byref(h)))
        self.h = h.value

    def close(self) -> None:
        if getattr(self, "h", None):
            load().sidr_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_shape(self, shape: int) -> None:
        """sidr_ctx_set_shape: the block shape of this context's evaluate*
        calls (Batch.SHAPES)."""
        _check(load().sidr_ctx_set_shape(self.h, shape))

    # -- the reference-shaped calls (host buffers, synchronous)
    def evaluate(self, rules, sampled, N, term_mask) -> np.ndarray:
        k = _Keep()
        r = k.rules(rules)
        out = np.zeros((rules.P, N))
        _check(load().sidr_evaluate(self.h, C.byref(r), k.f64(sampled), N, k.i64(term_mask),
                                    _d(out)))
        return out

    def evaluate_grouped(self, rules, grouped_sampled, G, T, group_size, term_mask):
        k = _Keep()
        r = k.rules(rules)
        out = np.zeros((rules.P, T))
        _check(load().sidr_evaluate_grouped(self.h, C.byref(r), k.f64(grouped_sampled), G, T,
                                            group_size, k.i64(term_mask), _d(out)))
        return out

    def evaluate_grouped_masks(self, rules, grouped_sampled, G, T, group_size, mask_group, masks):
        k = _Keep()
        r = k.rules(rules)
        out = np.zeros((rules.P, T))
        _check(load().sidr_evaluate_grouped_masks(self.h, C.byref(r), k.f64(grouped_sampled), G,
                                                  T, group_size, mask_group, k.i64(masks),
                                                  _d(out)))
        return out

    def batch(self, rules, grouped_sampled, T, masks, G=1, group_size=None,
              mask_group=None) -> Batch:
        k = _Keep()
        r = k.rules(rules)
        h = C.c_void_p()
        _check(load().sidr_batch_create(self.h, C.byref(r), k.f64(grouped_sampled), G, T,
                                        group_size or max(rules.P, 1),
                                        mask_group or max(rules.P, 1), k.i64(masks),
                                        C.byref(h)))
        return Batch(self, h.value, rules.P, T)


class Multi:
    """A multi-instance batch (sidr_multi_*): several instances of uneven size,
    each with its own rules, scenarios and mask, in one persistent launch."""

    # warps per block, min blocks per SM, lanes per (rule, scenario) pair
    SHAPES = ((4, 3, 32), (8, 2, 32), (2, 6, 32), (4, 3, 16), (4, 3, 8))
    # size classes of instances (customers): each class runs in a launch of its own
    CLASSES = ((0, 32), (33, 64), (65, 128), (129, 512))

    def __init__(self, sds, zps, rules_per_instance, sampled_per_instance, T, masks,
                 device: int = 0):
        L = load()
        if not getattr(L, "_multi_ready", False):
            vp = C.c_void_p
            L.sidr_multi_create.argtypes = [C.POINTER(_Inst), _dp, C.c_int32, C.POINTER(_Rules),
                                            _ip, _dp, C.c_int64, _lp, C.c_int32, _lp, C.c_int32,
                                            C.POINTER(vp)]
            L.sidr_multi_autotune.argtypes = [vp, C.c_int32, C.POINTER(C.c_int32),
                                              C.POINTER(C.c_float)]
            L.sidr_multi_autotune_sampled.argtypes = [vp, C.c_int32, C.c_int32,
                                                      C.POINTER(C.c_int32), C.POINTER(C.c_float)]
            L.sidr_multi_set_shape.argtypes = [vp, C.c_int32]
            L.sidr_multi_autotune_classes.argtypes = [vp, C.c_int32, C.c_int32,
                                                      C.POINTER(C.c_int32), C.POINTER(C.c_float)]
            L.sidr_multi_set_class_shape.argtypes = [vp, C.c_int32, C.c_int32]
            L.sidr_multi_shapes.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
            L.sidr_multi_capture.argtypes = [vp]
            L.sidr_multi_run.argtypes = [vp, vp]
            L.sidr_multi_read.argtypes = [vp, _dp]
            L.sidr_multi_destroy.argtypes = [vp]
            L._multi_ready = True
        from .rules import pack_compiled
        K = len(sds)
        k = _Keep()
        insts = (_Inst * K)(*[k.inst(sd) for sd in sds])
        zp = np.ascontiguousarray(np.stack([np.asarray(z, dtype=np.float64) for z in zps]))
        compiled, owner = [], []
        for i, r in enumerate(rules_per_instance):
            for p in range(r.P):
                compiled.append(r.rule(p))
                owner.append(i)
        allr = pack_compiled(compiled)
        self.P, self.T, self.counts = allr.P, T, [r.P for r in rules_per_instance]
        offs, blocks, at = [], [], 0
        for sd, smp in zip(sds, sampled_per_instance):
            a = np.ascontiguousarray(smp, dtype=np.float64).reshape(-1)[:T * sd.n]
            offs.append(at)
            blocks.append(a)
            at += a.size
        flat = np.concatenate(blocks) if blocks else np.zeros(1)
        m = np.ascontiguousarray(np.stack([np.asarray(x, dtype=np.int64) for x in masks]))
        rr = k.rules(allr)
        h = C.c_void_p()
        _check(L.sidr_multi_create(insts, zp.ctypes.data_as(_dp), K, C.byref(rr),
                                   k.i32(np.asarray(owner, dtype=np.int32)), k.f64(flat),
                                   int(flat.size), k.i64(np.asarray(offs, dtype=np.int64)), T,
                                   m.ctypes.data_as(_lp), device, C.byref(h)))
        self.h = h.value

    def autotune(self, reps: int = 1):
        ch = C.c_int32()
        ms = (C.c_float * len(self.SHAPES))()
        _check(load().sidr_multi_autotune(self.h, reps, C.byref(ch), ms))
        return ch.value, [float(x) for x in ms]

    def autotune_sampled(self, stride: int = 16, reps: int = 1):
        """sidr_multi_autotune_sampled: the block shape chosen on every
        stride-th rule of the longest-first order."""
        ch = C.c_int32()
        ms = (C.c_float * len(self.SHAPES))()
        _check(load().sidr_multi_autotune_sampled(self.h, reps, stride, C.byref(ch), ms))
        return ch.value, [float(x) for x in ms]

    def autotune_classes(self, stride: int = 16, reps: int = 1):
        """sidr_multi_autotune_classes: a block shape per size class, each
        timed on every stride-th rule of the class.  Returns ([shape per class,
        -1 for classes without rules], [[ms per shape] per class, -1 where not
        timed])."""
        nc, ns = len(self.CLASSES), len(self.SHAPES)
        ch = (C.c_int32 * nc)()
        ms = (C.c_float * (nc * ns))()
        _check(load().sidr_multi_autotune_classes(self.h, reps, stride, ch, ms))
        return list(ch), [[float(ms[c * ns + s]) for s in range(ns)] for c in range(nc)]

    def set_shape(self, shape: int):
        """The same block shape for every size class."""
        _check(load().sidr_multi_set_shape(self.h, shape))

    def set_class_shape(self, cls: int, shape: int):
        _check(load().sidr_multi_set_class_shape(self.h, cls, shape))

    def shapes(self):
        """(shape per size class, rules per size class)."""
        nc = len(self.CLASSES)
        sh, cnt = (C.c_int32 * nc)(), (C.c_int32 * nc)()
        _check(load().sidr_multi_shapes(self.h, sh, cnt))
        return list(sh), list(cnt)

    def capture(self):
        _check(load().sidr_multi_capture(self.h))

    def run(self, stream: int = 0):
        _check(load().sidr_multi_run(self.h, C.c_void_p(stream)))

    def read(self):
        """Scores split per instance: a list of [P_k, T] arrays."""
        out = np.zeros((self.P, self.T))
        _check(load().sidr_multi_read(self.h, _d(out)))
        res, at = [], 0
        for c in self.counts:
            res.append(out[at:at + c])
            at += c
        return res

    def close(self):
        if getattr(self, "h", None):
            load().sidr_multi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
