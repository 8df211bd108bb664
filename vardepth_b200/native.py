"""ctypes bindings of libvardepth_pairhmm.so (include/vardepth_pairhmm.h).

The library is the only compute path: there is no CPU fallback.  Loading
fails with an ImportError-style RuntimeError when the shared library has not
been built, and engine creation raises RuntimeError when no CUDA device is
usable, mirroring caller/native/caller/accelerator.py:91-96.
"""
from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvardepth_pairhmm.so"

VD_OK, VD_EINVAL, VD_ECUDA, VD_ENODEV, VD_ENOMEM, VD_EOVERFLOW = range(6)
VD_PRECISION_MIXED, VD_PRECISION_FLOAT64 = 0, 1
VD_SCHEDULE_BATCHED, VD_SCHEDULE_PLAIN = 0, 1
VD_CHECKPOINT_SQRT, VD_CHECKPOINT_ALL = 0, 1
VD_LONG_WARP, VD_LONG_SINGLE, VD_LONG_BLOCK = 0, 1, 2
LONG_GROUP_MAX = 8  # haplotypes of one long-read warp item (kLongGroupMax)

c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_u8p = ctypes.POINTER(ctypes.c_ubyte)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_i32p = ctypes.POINTER(ctypes.c_int32)
c_dp = ctypes.POINTER(ctypes.c_double)


class VdParams(ctypes.Structure):
    _fields_ = [("gap", ctypes.c_double), ("ext", ctypes.c_double), ("anchored", ctypes.c_int),
                ("precision", ctypes.c_int), ("quality_offsets", c_dp), ("schedule", ctypes.c_int),
                ("reserved", ctypes.c_int * 3)]


class VdBatch(ctypes.Structure):
    _fields_ = [("read_bases", c_u8p), ("read_quals", c_u8p), ("read_off", c_i64p), ("n_reads", c_i64),
                ("hap_bases", c_u8p), ("hap_off", c_i64p), ("n_haps", c_i64),
                ("region_read_off", c_i64p), ("region_hap_off", c_i64p), ("n_regions", c_i64),
                ("pair_read", c_i32p), ("pair_hap", c_i32p), ("n_pairs", c_i64)]


class VdStats(ctypes.Structure):
    _fields_ = [("pairs", c_i64), ("dp_cells", c_i64), ("work_items", c_i64), ("batches", c_i64),
                ("rescued_fp64", c_i64), ("rescued_robust", c_i64), ("h2d_bytes", c_i64), ("d2h_bytes", c_i64),
                ("kernel_launches", c_i64), ("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("host_ms", ctypes.c_double), ("live_bytes", c_i64), ("primary_ms", ctypes.c_double),
                ("rescue_ms", ctypes.c_double), ("shared_cells", c_i64), ("rescued_fp32", c_i64),
                ("long_strips", c_i64), ("long_strip_runs", c_i64)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class VdTuning(ctypes.Structure):
    _fields_ = [("long_read_rows", ctypes.c_int), ("pair_mask", ctypes.c_int), ("max_item_columns", ctypes.c_int),
                ("pipeline_gcells", ctypes.c_int), ("long_mode", ctypes.c_int), ("pair_split", ctypes.c_int),
                ("long_group", ctypes.c_int), ("reserved", ctypes.c_int * 1)]

    def as_dict(self) -> dict:
        return {"long_read_rows": self.long_read_rows, "pair_mask": self.pair_mask,
                "max_item_columns": self.max_item_columns, "pipeline_gcells": self.pipeline_gcells,
                "long_mode": self.long_mode, "pair_split": self.pair_split or 6,
                "long_group": self.long_group or LONG_GROUP_MAX}


class VdGenotypeOptions(ctypes.Structure):
    _fields_ = [("artifact_prior", ctypes.c_double), ("near_tie_guard", ctypes.c_int), ("reserved", ctypes.c_int * 3)]


class VdGradStats(ctypes.Structure):
    _fields_ = [("pairs", c_i64), ("dp_cells", c_i64), ("fp64_pairs", c_i64), ("failed_pairs", c_i64),
                ("scratch_bytes", c_i64), ("kernel_launches", c_i64), ("kernel_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every symbol include/vardepth_pairhmm.h declares, with its ctypes signature.
SIGNATURES = {
    "vd_engine_create": (ctypes.c_int, [ctypes.c_int, c_i64, ctypes.POINTER(ctypes.c_void_p)]),
    "vd_engine_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "vd_engine_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                      ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "vd_region_genotypes": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdBatch), ctypes.POINTER(VdParams),
                                           c_u8p, ctypes.POINTER(VdGenotypeOptions), c_dp, c_dp, c_dp, c_dp,
                                           ctypes.POINTER(ctypes.c_int), ctypes.POINTER(VdStats)]),
    "vd_engine_set_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdTuning)]),
    "vd_engine_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdTuning)]),
    "vd_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdBatch), ctypes.POINTER(VdParams), c_dp,
                                  ctypes.POINTER(VdStats)]),
    "vd_batch_outputs": (c_i64, [ctypes.POINTER(VdBatch)]),
    "vd_prefix_plan": (ctypes.c_int, [c_u8p, c_i64p, c_i64, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.POINTER(ctypes.c_int32)]),
    "vd_plan_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdBatch), ctypes.POINTER(VdParams),
                                      ctypes.POINTER(ctypes.c_void_p)]),
    "vd_plan_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdStats)]),
    "vd_plan_fetch": (ctypes.c_int, [ctypes.c_void_p, c_dp]),
    "vd_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "vd_forward_backward": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(VdBatch), ctypes.POINTER(VdParams),
                                           ctypes.c_int, c_dp, c_dp, ctypes.POINTER(VdGradStats)]),
    "vd_pairhmm_pairs": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(c_u8p),
                                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_char_p),
                                        ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp]),
    "vd_trie_many": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(c_u8p),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(ctypes.c_char_p),
                                    ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int, c_dp,
                                    ctypes.POINTER(ctypes.c_uint64)]),
    "vd_read_haplotype_batch_mode": (ctypes.c_int, [ctypes.c_char_p, c_u8p, ctypes.c_int,
                                                    ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int),
                                                    ctypes.c_int, ctypes.c_double, ctypes.c_double, c_dp,
                                                    ctypes.c_int]),
    "vd_read_haplotype": (ctypes.c_double, [ctypes.c_char_p, c_u8p, ctypes.c_int, ctypes.c_char_p, ctypes.c_int,
                                            ctypes.c_double, ctypes.c_double]),
    "vd_anchored_pairhmm": (ctypes.c_double, [ctypes.c_char_p, c_u8p, ctypes.c_int, ctypes.c_char_p,
                                              ctypes.c_int, ctypes.c_double, ctypes.c_double]),
    # device pointers in and out; scratch in a fixed static device array
    "vd_forward_region_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 c_i64, ctypes.c_void_p, ctypes.c_void_p, c_i64,
                                                 ctypes.POINTER(VdParams), ctypes.c_void_p, ctypes.c_void_p]),
    # pointer arrays of the Python pair list (vardepth_b200._pairlist.gather)
    "vd_score_pair_list": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, c_i64, ctypes.POINTER(VdParams), c_dp,
                                          ctypes.POINTER(VdStats)]),
    "vd_pair_list_plan": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p, c_i64, c_i64p, c_i32p, c_i32p, c_i32p, c_i64p]),
    "vd_last_error": (ctypes.c_char_p, []),
    "vd_device_count": (ctypes.c_int, []),
    "vd_version": (ctypes.c_char_p, []),
    "vd_measure_fp32_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
}

_LIB = None
_LOCK = threading.Lock()


def library() -> ctypes.CDLL:
    """Load the shared library (built by vardepth_b200.build) exactly once."""
    global _LIB
    with _LOCK:
        if _LIB is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH.name} is not built: run `python -m vardepth_b200.build` "
                    "(the PairHMM has no CPU fallback)")
            lib = ctypes.CDLL(str(LIB_PATH))
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _LIB = lib
        return _LIB


def last_error() -> str:
    msg = library().vd_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str) -> None:
    if rc == VD_OK:
        return
    msg = f"{what} failed ({rc}): {last_error()}"
    if rc == VD_EINVAL:
        raise ValueError(msg)
    if rc == VD_ENOMEM and "budget" in msg:
        raise ValueError(msg)
    raise RuntimeError(msg)


def _ptr(a: np.ndarray | None, ctype):
    if a is None:
        return ctypes.cast(None, ctypes.POINTER(ctype))
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class Packed:
    """Reads and haplotypes in the packed layout of vd_batch.

    Holds references to every array so the pointers stay valid for the call.
    """

    def __init__(self, read_bases, read_quals, read_off, hap_bases, hap_off, *,
                 region_read_off=None, region_hap_off=None, pair_read=None, pair_hap=None):
        self.read_bases = np.ascontiguousarray(read_bases, dtype=np.uint8)
        self.read_quals = np.ascontiguousarray(read_quals, dtype=np.uint8)
        self.read_off = np.ascontiguousarray(read_off, dtype=np.int64)
        self.hap_bases = np.ascontiguousarray(hap_bases, dtype=np.uint8)
        self.hap_off = np.ascontiguousarray(hap_off, dtype=np.int64)
        self.region_read_off = None if region_read_off is None else np.ascontiguousarray(region_read_off, np.int64)
        self.region_hap_off = None if region_hap_off is None else np.ascontiguousarray(region_hap_off, np.int64)
        self.pair_read = None if pair_read is None else np.ascontiguousarray(pair_read, np.int32)
        self.pair_hap = None if pair_hap is None else np.ascontiguousarray(pair_hap, np.int32)
        if self.read_bases.shape != self.read_quals.shape:
            raise ValueError("read bases and qualities differ in length")
        b = VdBatch()
        b.read_bases = _ptr(self.read_bases, ctypes.c_ubyte)
        b.read_quals = _ptr(self.read_quals, ctypes.c_ubyte)
        b.read_off = _ptr(self.read_off, ctypes.c_int64)
        b.n_reads = len(self.read_off) - 1
        b.hap_bases = _ptr(self.hap_bases, ctypes.c_ubyte)
        b.hap_off = _ptr(self.hap_off, ctypes.c_int64)
        b.n_haps = len(self.hap_off) - 1
        if self.pair_read is not None:
            b.pair_read = _ptr(self.pair_read, ctypes.c_int32)
            b.pair_hap = _ptr(self.pair_hap, ctypes.c_int32)
            b.n_pairs = len(self.pair_read)
        else:
            b.region_read_off = _ptr(self.region_read_off, ctypes.c_int64)
            b.region_hap_off = _ptr(self.region_hap_off, ctypes.c_int64)
            b.n_regions = len(self.region_read_off) - 1
        self.batch = b

    def n_outputs(self) -> int:
        if self.pair_read is not None:
            return len(self.pair_read)
        rr = np.diff(self.region_read_off)
        hh = np.diff(self.region_hap_off)
        return int(np.sum(rr * hh))


def prefix_plan(hap_bases: np.ndarray, hap_off: np.ndarray):
    """(order, share) of one region's haplotypes as the two-read kernels stream them
    (vd_prefix_plan; host only)."""
    hb = np.ascontiguousarray(hap_bases, dtype=np.uint8)
    ho = np.ascontiguousarray(hap_off, dtype=np.int64)
    n = len(ho) - 1
    order = np.empty(max(n, 0), np.int32)
    share = np.empty(max(n, 0), np.int32)
    i32p = ctypes.POINTER(ctypes.c_int32)
    check(library().vd_prefix_plan(hb.ctypes.data_as(c_u8p), ho.ctypes.data_as(c_i64p), n,
                                   order.ctypes.data_as(i32p), share.ctypes.data_as(i32p)), "vd_prefix_plan")
    return order, share


class PairList:
    """A Python list of (read, qualities, haplotype) triples as the pointer arrays of the
    reference's pair-list calling convention (batch_hmm.cpp:192), pointing into the Python
    objects themselves (vardepth_b200._pairlist.gather).  Raises ValueError with the
    reference's messages for reads or haplotypes that are not ASCII str, qualities that are
    not integer Phred scores in [0, 255], and read/quality length mismatches; the ACGTN check
    runs in the library."""

    def __init__(self, pairs):
        try:
            from . import _pairlist
        except ImportError as e:  # the helper is built with the library
            raise RuntimeError("vardepth_b200._pairlist is not built: run `python -m vardepth_b200.build`") from e
        self.pairs = pairs if isinstance(pairs, (list, tuple)) else list(pairs)
        (self.count, self._reads, self._quals, self._rn, self._haps, self._hn,
         self._keep) = _pairlist.gather(self.pairs)
        addr = lambda b: np.frombuffer(b, np.uint8).ctypes.data if len(b) else None
        self.args = tuple(addr(b) for b in (self._reads, self._quals, self._rn, self._haps, self._hn))

    def cells(self) -> int:
        return int(np.dot(np.frombuffer(self._rn, np.int32).astype(np.int64),
                          np.frombuffer(self._hn, np.int32).astype(np.int64)))


def pair_list_plan(pairs) -> dict:
    """The regrouping vd_score_pair_list applies to a pair list (vd_pair_list_plan; host only)."""
    pl = pairs if isinstance(pairs, PairList) else PairList(pairs)
    n = pl.count
    counts = np.zeros(4, np.int64)
    out = {k: np.empty(n, dt) for k, dt in (("read", np.int32), ("hap", np.int32), ("region", np.int32),
                                               ("slot", np.int64))}
    check(library().vd_pair_list_plan(*pl.args, n, counts.ctypes.data_as(c_i64p),
                                      out["read"].ctypes.data_as(c_i32p), out["hap"].ctypes.data_as(c_i32p),
                                      out["region"].ctypes.data_as(c_i32p), out["slot"].ctypes.data_as(c_i64p)),
          "vd_pair_list_plan")
    out.update(n_reads=int(counts[0]), n_haps=int(counts[1]), n_regions=int(counts[2]), n_slots=int(counts[3]))
    return out


def make_params(gap: float, ext: float, anchored: bool, precision: int, quality_offsets=None,
                schedule: int = VD_SCHEDULE_BATCHED):
    p = VdParams()
    p.gap = float(gap)
    p.ext = float(ext)
    p.anchored = 1 if anchored else 0
    p.precision = int(precision)
    p.schedule = int(schedule)
    keep = None
    if quality_offsets is not None:
        keep = np.ascontiguousarray(quality_offsets, dtype=np.float64)
        if keep.shape != (4,):
            raise ValueError("quality_offsets must hold 4 values")
        p.quality_offsets = keep.ctypes.data_as(c_dp)
    return p, keep


class Engine:
    """One vd_engine (device, stream, cached buffers)."""

    def __init__(self, device: int = 0, memory_mb: int = 4096):
        lib = library()
        h = ctypes.c_void_p()
        rc = lib.vd_engine_create(int(device), int(memory_mb), ctypes.byref(h))
        if rc == VD_ENODEV:
            raise RuntimeError("CUDA PairHMM requires an accessible NVIDIA GPU: " + last_error())
        check(rc, "vd_engine_create")
        self.handle = h
        self.device = device
        self.memory_mb = memory_mb
        import weakref
        self._plans = weakref.WeakSet()

    def info(self) -> dict:
        name = ctypes.create_string_buffer(256)
        major, minor, sms = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check(library().vd_engine_info(self.handle, name, 256, ctypes.byref(major), ctypes.byref(minor),
                                       ctypes.byref(sms)), "vd_engine_info")
        return {"gpu": name.value.decode(), "compute_capability": [major.value, minor.value], "sm_count": sms.value}

    def tuning(self) -> dict:
        t = VdTuning()
        check(library().vd_engine_get_tuning(self.handle, ctypes.byref(t)), "vd_engine_get_tuning")
        return t.as_dict()

    def set_tuning(self, long_read_rows: int = 256, pair_mask: int = 0x1FE, max_item_columns: int = 0,
                   pipeline_gcells: int = 0, long_mode: int = VD_LONG_WARP, pair_split: int = 6,
                   long_group: int = 0) -> None:
        t = VdTuning()
        t.long_read_rows, t.pair_mask, t.max_item_columns = int(long_read_rows), int(pair_mask), int(max_item_columns)
        t.pipeline_gcells = int(pipeline_gcells)
        t.long_mode = int(long_mode)
        t.pair_split = int(pair_split)
        t.long_group = int(long_group)
        check(library().vd_engine_set_tuning(self.handle, ctypes.byref(t)), "vd_engine_set_tuning")

    def forward(self, packed: Packed, params: VdParams, out: np.ndarray | None = None):
        n = packed.n_outputs()
        if out is None:
            out = np.empty(n, np.float64)
        stats = VdStats()
        check(library().vd_forward(self.handle, ctypes.byref(packed.batch), ctypes.byref(params),
                                   out.ctypes.data_as(c_dp), ctypes.byref(stats)), "vd_forward")
        return out, stats

    def score_pair_list(self, pairs, params: VdParams, out: np.ndarray | None = None):
        """ln L of a list of (read, qualities, haplotype) triples in input order, through
        vd_score_pair_list (validation, dedupe and regrouping into regions in native code)."""
        pl = pairs if isinstance(pairs, PairList) else PairList(pairs)
        if out is None:
            out = np.empty(pl.count, np.float64)
        stats = VdStats()
        check(library().vd_score_pair_list(self.handle, *pl.args, pl.count, ctypes.byref(params),
                                           out.ctypes.data_as(c_dp), ctypes.byref(stats)), "vd_score_pair_list")
        return out, stats

    def forward_backward(self, packed: Packed, params: VdParams, checkpoint: int = VD_CHECKPOINT_SQRT):
        """ln L per output and d ln L / d(Qg, Qx, o0..o3) as an (outputs, 6) array."""
        n = packed.n_outputs()
        ln = np.empty(n, np.float64)
        jac = np.empty((n, 6), np.float64)
        stats = VdGradStats()
        check(library().vd_forward_backward(self.handle, ctypes.byref(packed.batch), ctypes.byref(params),
                                            int(checkpoint), ln.ctypes.data_as(c_dp), jac.ctypes.data_as(c_dp),
                                            ctypes.byref(stats)), "vd_forward_backward")
        return ln, jac, stats

    def region_genotypes(self, packed: Packed, params: VdParams, mapping_quality=None, artifact_prior=None,
                         values: bool = True, certainty: bool = True, ln: bool = True,
                         near_tie_guard: bool = False) -> dict:
        """Forward pass plus on-device normalised rows and diploid genotype log-likelihoods of
        every region (vd_region_genotypes); ``gl`` is a list with one array per region."""
        if packed.pair_read is not None:
            raise ValueError("genotypes need the region form of the batch")
        rr = np.diff(packed.region_read_off)
        hh = np.diff(packed.region_hap_off)
        n_out = int(np.sum(rr * hh))
        P = hh * (hh + 1) // 2
        gl = np.empty(int(P.sum()), np.float64)
        out = {"ln": np.empty(n_out) if ln else None, "values": np.empty(n_out) if values else None,
               "certainty": np.full(len(packed.read_off) - 1, np.nan) if certainty else None}
        mq = None if mapping_quality is None else np.ascontiguousarray(mapping_quality, np.uint8)
        if mq is not None and len(mq) != len(packed.read_off) - 1:
            raise ValueError("one mapping quality per read")
        options = VdGenotypeOptions()
        options.artifact_prior = -1.0 if artifact_prior is None else float(artifact_prior)
        options.near_tie_guard = 1 if near_tie_guard else 0
        guarded = np.zeros(len(P), np.int32)
        stats = VdStats()
        opt = lambda a: a.ctypes.data_as(c_dp) if a is not None else ctypes.cast(None, c_dp)
        check(library().vd_region_genotypes(self.handle, ctypes.byref(packed.batch), ctypes.byref(params),
                                            _ptr(mq, ctypes.c_ubyte), ctypes.byref(options), opt(out["ln"]),
                                            opt(out["values"]), opt(out["certainty"]), gl.ctypes.data_as(c_dp),
                                            guarded.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                            ctypes.byref(stats)),
              "vd_region_genotypes")
        offs = np.concatenate([[0], np.cumsum(P)])
        out["gl"] = [gl[offs[g]:offs[g + 1]] for g in range(len(P))]
        out["guarded"] = guarded.astype(bool)
        out["stats"] = stats
        return out

    def plan(self, packed: Packed, params: VdParams) -> "Plan":
        return Plan(self, packed, params)

    def close(self):
        if getattr(self, "handle", None):
            for plan in list(self._plans):
                plan.close()
            library().vd_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A device-resident batch (vd_plan_*)."""

    def __init__(self, engine: Engine, packed: Packed, params: VdParams):
        self.engine = engine
        self.packed = packed
        self.n_out = packed.n_outputs()
        h = ctypes.c_void_p()
        check(library().vd_plan_create(engine.handle, ctypes.byref(packed.batch), ctypes.byref(params),
                                       ctypes.byref(h)), "vd_plan_create")
        self.handle = h
        engine._plans.add(self)

    def run(self) -> VdStats:
        st = VdStats()
        check(library().vd_plan_run(self.handle, ctypes.byref(st)), "vd_plan_run")
        return st

    def fetch(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.n_out, np.float64)
        check(library().vd_plan_fetch(self.handle, out.ctypes.data_as(c_dp)), "vd_plan_fetch")
        return out

    def close(self):
        if getattr(self, "handle", None):
            library().vd_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
