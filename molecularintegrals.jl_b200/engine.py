"""Python host side of libmolints_cuda.so (ctypes over the C ABI of include/molints.h).

The public calls mirror the reference's drivers (MolecularIntegrals.jl):

    all_twoe_ints(shells)        ~ all_twoe_ints(bfs, ERI=coulomb)   src/ERI.jl:104-112
    all_twoe_ints_chrr(shells)   ~ all_twoe_ints_chrr(bfs)           src/HGP.jl:22-34
    all_twoe_ints_rys(shells)    ~ all_twoe_ints_rys(bfs)            src/Rys.jl:16-24

Both return the packed vector of unique normalised integrals in iindex order
(src/Utils.jl:14-19), 0-based.  ``Engine`` exposes the context/plan API for callers that
keep inputs and outputs on the device.  There is no CPU fallback: if the library is
missing or no CUDA device is present, these calls raise.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libmolints_cuda.so"

FP64, MIXED = 0, 1
BOYS_REFERENCE, BOYS_EXACT = 0, 1
METHOD_AUTO, METHOD_HGP, METHOD_RYS = 0, 1, 2
CLASS_NO_FP32 = 4   # flag in a set_class_methods entry: MIXED plans run the FP64 kernel
LMAX = 4  # g shells: generic Rys kernel (molints.h MOLINTS_LMAX)
# shell-pair classes in the engine's order (la+lb, then la): index -> (la, lb)
PAIR_CLASSES = [(0, 0), (1, 0), (1, 1), (2, 0), (2, 1), (3, 0), (2, 2), (3, 1), (2, 3), (3, 2), (3, 3)]
NUM_PAIR_CLASSES = len(PAIR_CLASSES)

_STATUS = {0: "OK", -1: "invalid argument", -2: "unsupported", -3: "HBM budget exceeded",
           -4: "CUDA error", -5: "timeout", -6: "out of host memory"}

EXPORTED_SYMBOLS = [
    "molints_abi_version", "molints_default_options", "molints_nbf", "molints_npacked",
    "molints_create", "molints_destroy", "molints_last_error", "molints_set_stream",
    "molints_eri_packed", "molints_plan_create", "molints_plan_execute", "molints_plan_stats",
    "molints_plan_destroy", "molints_plan_schwarz", "molints_boys_eval",
    "molints_plan_set_profiling", "molints_plan_launch_times", "molints_eri_packed_noalloc",
    "molints_plan_create_batch", "molints_plan_npacked", "molints_set_class_methods",
    "molints_serve_start", "molints_serve_stop", "molints_submit", "molints_poll",
    "molints_result", "molints_result_copy", "molints_request_info", "molints_request_error",
    "molints_release", "molints_serve_stats", "molints_shard_range", "molints_plan_create_shard",
    "molints_plan_set_graph", "molints_plan_jk", "molints_jk", "molints_one_e",
    "molints_get_class_methods", "molints_plan_class_work", "molints_set_schedule",
    "molints_get_schedule",
]


class MolintsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


class Basis(ctypes.Structure):
    _fields_ = [("nshell", ctypes.c_int32), ("xyz", ctypes.c_void_p), ("L", ctypes.c_void_p),
                ("nprim", ctypes.c_void_p), ("prim_off", ctypes.c_void_p),
                ("expn", ctypes.c_void_p), ("coef", ctypes.c_void_p)]


class Options(ctypes.Structure):
    _fields_ = [("method", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("boys", ctypes.c_int32), ("output", ctypes.c_int32),
                ("fp32_cutoff", ctypes.c_double), ("screen_cutoff", ctypes.c_double),
                ("prim_cutoff", ctypes.c_double)]


PRIM_CUTOFF = 1e-18
# enum molints_output: how the class kernels reach the packed vector
OUTPUT_AUTO, OUTPUT_DIRECT, OUTPUT_TWO_PHASE = 0, 1, 2


class Stats(ctypes.Structure):
    _fields_ = [("n_eri", ctypes.c_int64), ("n_shell_quartets", ctypes.c_int64),
                ("n_prim_quartets", ctypes.c_int64), ("n_fp32_quartets", ctypes.c_int64),
                ("n_screened", ctypes.c_int64), ("n_kernel_launches", ctypes.c_int32),
                ("n_fp32_launches", ctypes.c_int32), ("device_ms", ctypes.c_double),
                ("n_prim_pairs", ctypes.c_int64), ("n_prim_pairs_kept", ctypes.c_int64),
                ("plan_ms", ctypes.c_double * 4)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "plan_ms"}
        d["plan_ms"] = list(self.plan_ms)
        return d


class Schedule(ctypes.Structure):
    """molints_schedule: the work-queue knobs of the plans a context creates."""
    _fields_ = [("lane_cost", ctypes.c_double), ("hgp_widen", ctypes.c_int32),
                ("rys_chunks", ctypes.c_int32), ("rys_max_width", ctypes.c_int32),
                ("gather_blocks", ctypes.c_int32)]
    KEYS = ("lane_cost", "hgp_widen", "rys_chunks", "rys_max_width", "gather_blocks")

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k in self.KEYS}


_lib = None


def load_library(path: Path | str | None = None):
    """Load libmolints_cuda.so (built in-tree by build.py); raise if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} is missing: run molecularintegrals.jl_b200/build.py")
    L = ctypes.CDLL(str(p))
    P, I32, I64, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "molints_abi_version": (ctypes.c_int, []),
        "molints_default_options": (None, [P]),
        "molints_nbf": (I64, [P]),
        "molints_npacked": (I64, [I64]),
        "molints_create": (ctypes.c_int, [P, ctypes.c_int, I64, ctypes.c_uint32]),
        "molints_destroy": (ctypes.c_int, [P]),
        "molints_last_error": (ctypes.c_char_p, [P]),
        "molints_set_stream": (ctypes.c_int, [P, P]),
        "molints_eri_packed": (ctypes.c_int, [P, P, P, P, ctypes.c_int, P]),
        "molints_plan_create": (ctypes.c_int, [P, P, P, P]),
        "molints_plan_execute": (ctypes.c_int, [P, P]),
        "molints_plan_stats": (ctypes.c_int, [P, P]),
        "molints_plan_destroy": (ctypes.c_int, [P]),
        "molints_plan_schwarz": (ctypes.c_int, [P, P]),
        "molints_boys_eval": (ctypes.c_int, [P, I32, I32, P, I64, P]),
        "molints_plan_set_profiling": (ctypes.c_int, [P, ctypes.c_int]),
        "molints_plan_launch_times": (ctypes.c_int, [P, P, P, ctypes.c_int]),
        "molints_eri_packed_noalloc": (ctypes.c_int, [P, P, P, P, ctypes.c_char_p, ctypes.c_size_t]),
        "molints_plan_create_batch": (ctypes.c_int, [P, I32, P, P, P]),
        "molints_plan_npacked": (I64, [P]),
        "molints_set_class_methods": (ctypes.c_int, [P, P, I32]),
        "molints_get_class_methods": (ctypes.c_int, [P, P, I32]),
        "molints_set_schedule": (ctypes.c_int, [P, P]),
        "molints_get_schedule": (ctypes.c_int, [P, P]),
        "molints_plan_class_work": (ctypes.c_int, [P, P, P, I32]),
        "molints_serve_start": (ctypes.c_int, [P, I32, I64]),
        "molints_serve_stop": (ctypes.c_int, [P]),
        "molints_submit": (ctypes.c_int, [P, P, P, P]),
        "molints_poll": (ctypes.c_int, [P, I32]),
        "molints_result": (ctypes.c_int, [P, P, P]),
        "molints_result_copy": (ctypes.c_int, [P, P, I64]),
        "molints_request_info": (ctypes.c_int, [P, P, P, P, P]),
        "molints_request_error": (ctypes.c_char_p, [P]),
        "molints_release": (ctypes.c_int, [P]),
        "molints_serve_stats": (ctypes.c_int, [P, P, P, P, P]),
        "molints_shard_range": (ctypes.c_int, [P, I32, I32, P, P]),
        "molints_plan_create_shard": (ctypes.c_int, [P, P, P, I32, I32, P]),
        "molints_plan_set_graph": (ctypes.c_int, [P, ctypes.c_int]),
        "molints_plan_jk": (ctypes.c_int, [P, P, P, P]),
        "molints_jk": (ctypes.c_int, [P, P, P, P, P, P]),
        "molints_one_e": (ctypes.c_int, [P, P, I32, P, P, P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = L
    return L


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class _BasisArrays:
    """Keeps the contiguous arrays a molints_basis points into alive."""

    def __init__(self, shells):
        self.xyz = np.ascontiguousarray(shells.xyz, dtype=np.float64).reshape(-1)
        self.L = np.ascontiguousarray(shells.L, dtype=np.int32)
        self.nprim = np.ascontiguousarray(shells.nprim, dtype=np.int32)
        self.prim_off = np.ascontiguousarray(shells.prim_off, dtype=np.int32)
        self.expn = np.ascontiguousarray(shells.expn, dtype=np.float64)
        self.coef = np.ascontiguousarray(shells.coef, dtype=np.float64)
        self.c = Basis(len(self.L), _ptr(self.xyz), _ptr(self.L), _ptr(self.nprim),
                       _ptr(self.prim_off), _ptr(self.expn), _ptr(self.coef))


def make_options(precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0, screen_cutoff=0.0,
                 method=METHOD_AUTO, prim_cutoff=PRIM_CUTOFF, output=OUTPUT_AUTO) -> Options:
    return Options(method, precision, boys, int(output), float(fp32_cutoff), float(screen_cutoff),
                   float(prim_cutoff))


class Plan:
    """One basis (or a batch of them) resident on the device; ``execute`` runs the whole
    device path.  For a batch, molecule m's packed vector starts at ``offsets[m]``."""

    def __init__(self, engine: "Engine", shells, opts: Options, shard=None):
        self.engine = engine
        batch = isinstance(shells, (list, tuple))
        mols = list(shells) if batch else [shells]
        self._arrs = [_BasisArrays(sh) for sh in mols]
        self.nbf = [sh.nbf for sh in mols] if batch else shells.nbf
        self.offsets = np.concatenate([[0], np.cumsum([sh.npacked for sh in mols])]).astype(np.int64)
        self.npacked = int(self.offsets[-1])
        self.nshell = sum(sh.nshell for sh in mols)
        self._nshells = [sh.nshell for sh in mols]
        h = ctypes.c_void_p()
        if batch:
            arr = (Basis * len(mols))(*[a.c for a in self._arrs])
            self._carr = arr
            engine._check(engine.lib.molints_plan_create_batch(engine.ctx, len(mols), arr,
                                                               ctypes.byref(opts), ctypes.byref(h)))
        elif shard is not None:
            r, n = shard
            engine._check(engine.lib.molints_plan_create_shard(engine.ctx, ctypes.byref(self._arrs[0].c),
                                                               ctypes.byref(opts), int(r), int(n),
                                                               ctypes.byref(h)))
            self.slice = shard_range(shells, r, n)
            self.npacked = self.slice[1] - self.slice[0]
        else:
            engine._check(engine.lib.molints_plan_create(engine.ctx, ctypes.byref(self._arrs[0].c),
                                                         ctypes.byref(opts), ctypes.byref(h)))
        self.h = h
        assert engine.lib.molints_plan_npacked(h) == self.npacked

    def execute(self, out_device_ptr: int) -> None:
        """Queue the device path on the engine's stream, writing npacked doubles."""
        self.engine._check(self.engine.lib.molints_plan_execute(self.h, ctypes.c_void_p(out_device_ptr)))

    def stats(self) -> dict:
        st = Stats()
        self.engine._check(self.engine.lib.molints_plan_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def class_work(self) -> dict:
        """{tag: (shell quartets, evaluated primitive quartets)} per class pair of the plan,
        tags as 'ppps' (bra class then ket class, PAIR_CLASSES order)."""
        n = NUM_PAIR_CLASSES * NUM_PAIR_CLASSES
        q = np.zeros(n, dtype=np.int64)
        k = np.zeros(n, dtype=np.float64)
        self.engine._check(self.engine.lib.molints_plan_class_work(self.h, _ptr(q), _ptr(k), n))
        L = "spdf"
        out = {}
        for x in range(NUM_PAIR_CLASSES):
            for y in range(x + 1):
                if q[x * NUM_PAIR_CLASSES + y]:
                    (a, b), (c, d) = PAIR_CLASSES[x], PAIR_CLASSES[y]
                    out[L[a] + L[b] + L[c] + L[d]] = (int(q[x * NUM_PAIR_CLASSES + y]),
                                                      float(k[x * NUM_PAIR_CLASSES + y]))
        return out

    def jk(self, D_ptr: int, J_ptr: int, K_ptr: int) -> None:
        """Queue J and K (n x n device arrays) for the symmetric device density at D_ptr."""
        self.engine._check(self.engine.lib.molints_plan_jk(self.h, ctypes.c_void_p(D_ptr),
                                                           ctypes.c_void_p(J_ptr), ctypes.c_void_p(K_ptr)))

    def set_graph(self, enable: bool = True) -> None:
        """Launch executes as one captured CUDA graph (recaptured for a new output pointer)."""
        self.engine._check(self.engine.lib.molints_plan_set_graph(self.h, int(enable)))

    def set_profiling(self, enable: bool = True) -> None:
        self.engine._check(self.engine.lib.molints_plan_set_profiling(self.h, int(enable)))

    def launch_times(self, cap: int = 256):
        """[(kernel name, ms)] of the last execute (profiling must be on)."""
        names = (ctypes.c_char_p * cap)()
        ms = (ctypes.c_float * cap)()
        n = self.engine.lib.molints_plan_launch_times(self.h, names, ms, cap)
        if n < 0:
            self.engine._check(n)
        return [(names[k].decode(), float(ms[k])) for k in range(min(n, cap))]

    def schwarz(self) -> np.ndarray:
        out = np.zeros(sum(n * (n + 1) // 2 for n in self._nshells))
        self.engine._check(self.engine.lib.molints_plan_schwarz(self.h, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "h", None):
            self.engine.lib.molints_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Request:
    """One submitted molecule of the serving API (molints_submit)."""

    def __init__(self, engine: "Engine", handle: ctypes.c_void_p, npacked: int):
        self.engine = engine
        self.h = handle
        self.npacked = npacked

    def poll(self, timeout_ms: int = 0) -> bool:
        """True once the result is ready, False on timeout; raises the request's error."""
        rc = self.engine.lib.molints_poll(self.h, int(timeout_ms))
        if rc == -5:
            return False
        if rc != 0:
            msg = self.engine.lib.molints_request_error(self.h)
            raise MolintsError(rc, msg.decode() if msg else "")
        return True

    def device_ptr(self) -> int:
        ptr, n = ctypes.c_void_p(), ctypes.c_int64()
        self.engine._check_req(self.engine.lib.molints_result(self.h, ctypes.byref(ptr), ctypes.byref(n)), self)
        return ptr.value or 0

    def result(self) -> np.ndarray:
        out = np.empty(self.npacked, dtype=np.float64)
        self.engine._check_req(self.engine.lib.molints_result_copy(self.h, _ptr(out), out.size), self)
        return out

    def info(self) -> dict:
        t = [ctypes.c_double() for _ in range(3)]
        slot = ctypes.c_int32()
        self.engine.lib.molints_request_info(self.h, *[ctypes.byref(x) for x in t], ctypes.byref(slot))
        return {"t_submit": t[0].value, "t_admit": t[1].value, "t_done": t[2].value, "slot": slot.value}

    def release(self):
        if self.h is not None:
            self.engine.lib.molints_release(self.h)
            self.h = None


class Engine:
    """One molints context on one CUDA device."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        rc = self.lib.molints_create(ctypes.byref(h), device, int(hbm_budget_bytes), 0)
        if rc != 0:
            raise MolintsError(rc, f"molints_create on device {device}")
        self.ctx = h
        self.device = device

    def _check(self, rc: int):
        if rc != 0:
            msg = self.lib.molints_last_error(self.ctx) if self.ctx else b"context closed"
            raise MolintsError(rc, msg.decode() if msg else "")

    def set_stream(self, stream_handle: int | None):
        """Launch on a cudaStream_t handle (e.g. torch's ``Stream.cuda_stream``); handle 0, the
        legacy default stream, is passed as cudaStreamLegacy; None selects the own stream."""
        if stream_handle is None:
            h = None
        elif stream_handle == 0:
            h = ctypes.c_void_p(1)  # cudaStreamLegacy
        else:
            h = ctypes.c_void_p(stream_handle)
        self._check(self.lib.molints_set_stream(self.ctx, h))

    def eri_packed(self, shells, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
                   screen_cutoff=0.0, out: np.ndarray | None = None, with_stats=False,
                   prim_cutoff=PRIM_CUTOFF, method=METHOD_AUTO, output=OUTPUT_AUTO):
        """The packed iindex vector of all unique integrals, into a host array."""
        arrs = _BasisArrays(shells)
        if out is None:
            out = np.empty(shells.npacked, dtype=np.float64)
        if shells.npacked == 0:
            st = Stats()
            self._check(self.lib.molints_eri_packed(self.ctx, ctypes.byref(arrs.c), None, None, 0,
                                                    ctypes.byref(st)))
            return (out, st.as_dict()) if with_stats else out
        if out.dtype != np.float64 or out.size != shells.npacked or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of npacked elements")
        opts = make_options(precision, boys, fp32_cutoff, screen_cutoff, method, prim_cutoff, output)
        st = Stats()
        self._check(self.lib.molints_eri_packed(self.ctx, ctypes.byref(arrs.c), ctypes.byref(opts),
                                                _ptr(out), 0, ctypes.byref(st) if with_stats else None))
        return (out, st.as_dict()) if with_stats else out

    def eri_packed_device(self, shells, out_device_ptr: int, precision=FP64, boys=BOYS_REFERENCE,
                          fp32_cutoff=0.0, screen_cutoff=0.0, prim_cutoff=PRIM_CUTOFF,
                          method=METHOD_AUTO, output=OUTPUT_AUTO):
        arrs = _BasisArrays(shells)
        opts = make_options(precision, boys, fp32_cutoff, screen_cutoff, method, prim_cutoff, output)
        st = Stats()
        self._check(self.lib.molints_eri_packed(self.ctx, ctypes.byref(arrs.c), ctypes.byref(opts),
                                                ctypes.c_void_p(out_device_ptr), 1, ctypes.byref(st)))
        return st.as_dict()

    def plan(self, shells, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
             screen_cutoff=0.0, prim_cutoff=PRIM_CUTOFF, method=METHOD_AUTO,
             output=OUTPUT_AUTO) -> Plan:
        return Plan(self, shells, make_options(precision, boys, fp32_cutoff, screen_cutoff,
                                               method, prim_cutoff, output))

    def plan_shard(self, shells, shard: int, nshards: int, precision=FP64, boys=BOYS_REFERENCE,
                   fp32_cutoff=0.0, screen_cutoff=0.0, prim_cutoff=PRIM_CUTOFF,
                   method=METHOD_AUTO) -> Plan:
        """Plan of shard `shard` of `nshards`: its execute writes the packed slice
        ``shard_range(shells, shard, nshards)`` (offsets relative to the slice start)."""
        return Plan(self, shells, make_options(precision, boys, fp32_cutoff, screen_cutoff,
                                               method, prim_cutoff), shard=(shard, nshards))

    def plan_batch(self, shells_list, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
                   screen_cutoff=0.0, prim_cutoff=PRIM_CUTOFF, method=METHOD_AUTO,
                   output=OUTPUT_AUTO) -> Plan:
        """One plan over several molecules: a single execute computes all of them."""
        return Plan(self, list(shells_list), make_options(precision, boys, fp32_cutoff,
                                                          screen_cutoff, method, prim_cutoff, output))

    def set_class_methods(self, table=None):
        """Per class pair method for METHOD_AUTO plans: ``table[(x, y)] = METHOD_HGP or
        METHOD_RYS`` (optionally | CLASS_NO_FP32) for pair-class indices x >= y (PAIR_CLASSES
        order); missing entries are AUTO (HGP).  None restores the library's default table (the
        tuned one on a B200)."""
        if table is None:
            self._check(self.lib.molints_set_class_methods(self.ctx, None, 0))
            return
        arr = np.zeros(NUM_PAIR_CLASSES * NUM_PAIR_CLASSES, dtype=np.int32)
        for (x, y), m in dict(table).items():
            arr[x * NUM_PAIR_CLASSES + y] = m
        self._check(self.lib.molints_set_class_methods(self.ctx, _ptr(arr), arr.size))

    def set_schedule(self, sched: dict | None = None):
        """Work-queue schedule of the plans created afterwards: a dict with any of lane_cost,
        hgp_widen, rys_chunks, rys_max_width, gather_blocks (the others keep their current
        values); None
        restores the library's default (the tuned one on a B200)."""
        if sched is None:
            self._check(self.lib.molints_set_schedule(self.ctx, None))
            return
        cur = self.schedule()
        cur.update(sched)
        sc = Schedule(**{k: cur[k] for k in Schedule.KEYS})
        self._check(self.lib.molints_set_schedule(self.ctx, ctypes.byref(sc)))

    def schedule(self) -> dict:
        """The context's current work-queue schedule."""
        sc = Schedule()
        self._check(self.lib.molints_get_schedule(self.ctx, ctypes.byref(sc)))
        return sc.as_dict()

    def class_methods(self) -> dict:
        """The context's current table as {(x, y): entry} for x >= y."""
        arr = np.zeros(NUM_PAIR_CLASSES * NUM_PAIR_CLASSES, dtype=np.int32)
        self._check(self.lib.molints_get_class_methods(self.ctx, _ptr(arr), arr.size))
        return {(x, y): int(arr[x * NUM_PAIR_CLASSES + y])
                for x in range(NUM_PAIR_CLASSES) for y in range(x + 1)}

    # ---- serving
    def serve_start(self, nslots: int = 4, hbm_budget_bytes: int = 0):
        """Start this context's server: nslots concurrent slots, admission by HBM budget."""
        self._check(self.lib.molints_serve_start(self.ctx, int(nslots), int(hbm_budget_bytes)))

    def serve_stop(self):
        self._check(self.lib.molints_serve_stop(self.ctx))

    def submit(self, shells, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
               screen_cutoff=0.0, prim_cutoff=PRIM_CUTOFF, method=METHOD_AUTO) -> Request:
        arrs = _BasisArrays(shells)
        opts = make_options(precision, boys, fp32_cutoff, screen_cutoff, method, prim_cutoff)
        h = ctypes.c_void_p()
        self._check(self.lib.molints_submit(self.ctx, ctypes.byref(arrs.c), ctypes.byref(opts),
                                            ctypes.byref(h)))
        return Request(self, h, shells.npacked)

    def serve_stats(self) -> dict:
        v = [ctypes.c_int64() for _ in range(4)]
        self._check(self.lib.molints_serve_stats(self.ctx, *[ctypes.byref(x) for x in v]))
        return dict(zip(("ledger_bytes", "queued", "done", "failed"), [x.value for x in v]))

    def _check_req(self, rc: int, req: Request):
        if rc != 0:
            msg = self.lib.molints_request_error(req.h)
            raise MolintsError(rc, msg.decode() if msg else "")

    def jk(self, shells, D, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
           method=METHOD_AUTO):
        """(J, K) for the symmetric density D (n x n host array), digested on the device
        without storing the integrals."""
        arrs = _BasisArrays(shells)
        n = shells.nbf
        D = np.ascontiguousarray(D, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError(f"D must be {n} x {n}")
        J = np.empty((n, n))
        K = np.empty((n, n))
        opts = make_options(precision, boys, fp32_cutoff, 0.0, method)
        self._check(self.lib.molints_jk(self.ctx, ctypes.byref(arrs.c), ctypes.byref(opts),
                                        _ptr(D), _ptr(J), _ptr(K)))
        return J, K

    def one_e(self, shells, atom_xyz, atom_charge):
        """(S, T, V): overlap, kinetic energy and nuclear attraction (point charges
        atom_charge at atom_xyz, bohr) of the basis, n x n each."""
        arrs = _BasisArrays(shells)
        n = shells.nbf
        xyz = np.ascontiguousarray(atom_xyz, dtype=np.float64).reshape(-1)
        z = np.ascontiguousarray(atom_charge, dtype=np.float64).reshape(-1)
        if xyz.size != 3 * z.size:
            raise ValueError("atom_xyz must hold 3 coordinates per charge")
        S, T, V = (np.zeros((n, n)) for _ in range(3))
        self._check(self.lib.molints_one_e(self.ctx, ctypes.byref(arrs.c), z.size, _ptr(xyz), _ptr(z),
                                           _ptr(S), _ptr(T), _ptr(V)))
        return S, T, V

    def boys(self, mmax: int, T, mode=BOYS_REFERENCE) -> np.ndarray:
        T = np.ascontiguousarray(T, dtype=np.float64)
        out = np.empty((T.size, mmax))
        self._check(self.lib.molints_boys_eval(self.ctx, mode, mmax, _ptr(T), T.size, _ptr(out)))
        return out

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.molints_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def shard_range(shells, shard: int, nshards: int):
    """(lo, hi): the contiguous packed slice shard `shard` of `nshards` owns (host only)."""
    lib = load_library()
    arrs = _BasisArrays(shells)
    lo, hi = ctypes.c_int64(), ctypes.c_int64()
    rc = lib.molints_shard_range(ctypes.byref(arrs.c), int(shard), int(nshards), ctypes.byref(lo),
                                 ctypes.byref(hi))
    if rc != 0:
        raise MolintsError(rc, "molints_shard_range")
    return lo.value, hi.value


_default_engine: Engine | None = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine(0)
    return _default_engine


def all_twoe_ints(shells, precision=FP64, boys=BOYS_REFERENCE, fp32_cutoff=0.0,
                  screen_cutoff=0.0) -> np.ndarray:
    """Drop-in for all_twoe_ints(bfs) (src/ERI.jl:104-112): packed normalised ERIs."""
    return default_engine().eri_packed(shells, precision, boys, fp32_cutoff, screen_cutoff)


def all_twoe_ints_chrr(shells) -> np.ndarray:
    """Drop-in for all_twoe_ints_chrr(bfs) (src/HGP.jl:22-34), with its layout and
    normalisation defects fixed: the same vector as all_twoe_ints."""
    return default_engine().eri_packed(shells, method=METHOD_HGP)


def all_1e_ints(shells, atoms):
    """Drop-in for all_1e_ints(bfs, mol) (src/OneInts.jl:267-290): (S, T, V) for the basis and
    the atoms (objects with ``atno`` and ``xyz`` in bohr, as ``basis.atom`` makes)."""
    xyz = np.array([a.xyz for a in atoms], dtype=np.float64).reshape(-1, 3)
    z = np.array([a.atno for a in atoms], dtype=np.float64)
    return default_engine().one_e(shells, xyz, z)


def make2JmK(D, shells) -> np.ndarray:
    """2J - K for the density D (make2JmK(D, Ints), src/ERI.jl:114-128), with the integrals
    digested on the device instead of read from a packed vector."""
    J, K = default_engine().jk(shells, D)
    return 2.0 * J - K


def all_twoe_ints_rys(shells) -> np.ndarray:
    """Drop-in for all_twoe_ints_rys(bfs) (src/Rys.jl:16-24): Rys quadrature for every class
    pair, with the contracted-function norms the reference driver leaves out applied."""
    return default_engine().eri_packed(shells, method=METHOD_RYS, boys=BOYS_EXACT)
