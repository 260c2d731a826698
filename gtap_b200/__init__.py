"""Python host binding of libgtap_b200.so (the B200 GTaP runtime).

The library is the product; this module is a thin ctypes layer that mirrors
the reference's host interface (gtap_initialize / gtap_finalize / gtap_reset /
gtap_synchronize / gtap_check_runtime_error / gtap_visualize_profile, see
runtime/detail/thread/gtap_runtime_thread.cuh:338-441 and
runtime/detail/common/gtap_runtime_error.cuh:38-249 in the reference) plus the
batch / serve entry points and the seeded generators.

Importing never needs a GPU.  Loading the library fails loudly if it has not
been built (``python -m gtap_b200.build``); there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgtap_b200.so")
if os.environ.get("GTAP_LIB_PATH"):
    LIB_PATH = os.environ["GTAP_LIB_PATH"]   # an alternative build of the same library
elif os.environ.get("GTAP_LIB_VARIANT") == "debug":
    # same library built with per-id live checks (python -m gtap_b200.build --debug)
    LIB_PATH = os.path.join(HERE, "libgtap_b200_debug.so")

# ---- constants mirrored from include/gtap.h --------------------------------
MODE_THREAD, MODE_BLOCK = 0, 1
VICTIM_RANDOM, VICTIM_LAST_SUCCESS, VICTIM_PROBE_MAX = 0, 1, 2
ADMIT_AS_GIVEN, ADMIT_BY_KIND, ADMIT_SPLIT = 0, 1, 2
KIND_FIB, KIND_NQ, KIND_CILKSORT, KIND_MERGESORT, KIND_BFS, KIND_TREESUM = 1, 2, 3, 4, 5, 6
ROOT_PENDING, ROOT_RUNNING, ROOT_DONE = 0, 1, 2

ERROR_NAMES = {
    0: "NONE", 1: "INVALID_QUEUE_IDX", 2: "INVALID_QUEUE_IDX_AFTER_JOIN", 3: "QUEUE_OVERFLOW",
    4: "RESULT_HANDLE_OVERFLOW", 5: "TASK_ID_POOL_SLOT_BUSY", 6: "TASK_ID_POOL_LOW_HEADROOM",
    7: "GENERATED_TASK_ID_BUFFER_OVERFLOW", 8: "INVALID_TASKWAIT", 9: "TIMEOUT", 10: "INVALID_KIND",
    11: "INVALID_ARGUMENT", 12: "NOT_INITIALIZED", 13: "BUSY",
}
ERROR_QUEUE_OVERFLOW = 3
ERROR_TIMEOUT = 9
ERROR_INVALID_ARGUMENT = 11
ERROR_NOT_INITIALIZED = 12

STAT_NAMES = ["tasks", "executions", "rounds", "steal_attempts", "steal_successes", "stolen_tasks", "pops",
              "published", "idle_polls", "overflow_pushes", "join_finishes", "idle_ns"]
STAT_COUNT = 16


class Config(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32), ("grid", ctypes.c_int32), ("block", ctypes.c_int32),
        ("num_queues", ctypes.c_int32), ("deque_capacity", ctypes.c_int32), ("steal_batch", ctypes.c_int32),
        ("victim_policy", ctypes.c_int32), ("probe_width", ctypes.c_int32), ("spawn_capacity", ctypes.c_int32),
        ("ids_per_worker", ctypes.c_int32), ("total_ids", ctypes.c_int64), ("frame_bytes", ctypes.c_int32),
        ("admit_batch", ctypes.c_int32), ("watchdog_ms", ctypes.c_int64), ("profile_samples", ctypes.c_int32),
        ("result_handles", ctypes.c_int32), ("publish_lazy", ctypes.c_int32), ("max_inflight_roots", ctypes.c_int32),
        ("admit_order", ctypes.c_int32), ("leaf_batch", ctypes.c_int32),
        ("join_walk", ctypes.c_int32), ("sub_rounds", ctypes.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Root(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32), ("i0", ctypes.c_int32), ("i1", ctypes.c_int32), ("i2", ctypes.c_int32),
        ("n", ctypes.c_int64), ("p0", ctypes.c_void_p), ("p1", ctypes.c_void_p), ("p2", ctypes.c_void_p),
        ("p3", ctypes.c_void_p),
    ]


class RootResult(ctypes.Structure):
    _fields_ = [
        ("value", ctypes.c_int64), ("tasks", ctypes.c_int64), ("t_admit_ns", ctypes.c_uint64),
        ("t_done_ns", ctypes.c_uint64), ("status", ctypes.c_int32), ("index", ctypes.c_int32),
    ]


class RunStats(ctypes.Structure):
    _fields_ = [
        ("counters", ctypes.c_uint64 * STAT_COUNT), ("kernel_ms", ctypes.c_double), ("grid", ctypes.c_int32),
        ("block", ctypes.c_int32), ("workers", ctypes.c_int32), ("status", ctypes.c_int32),
        ("launches", ctypes.c_int32), ("light_workers", ctypes.c_int32), ("light_kernel_ms", ctypes.c_double),
    ]

    def as_dict(self):
        d = {name: int(self.counters[i]) for i, name in enumerate(STAT_NAMES)}
        d.update(kernel_ms=self.kernel_ms, grid=self.grid, block=self.block, workers=self.workers,
                 status=self.status, launches=self.launches, light_workers=self.light_workers,
                 light_kernel_ms=self.light_kernel_ms)
        return d

    def worker_ms(self):
        """Workers x milliseconds over the launches (the idle fraction's denominator)."""
        full_ms = self.kernel_ms - self.light_kernel_ms
        full_workers = self.workers if full_ms > 0 else 0
        return self.light_workers * self.light_kernel_ms + full_workers * full_ms


class ErrorReport(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("valid", "code", "src_line", "block_idx", "thread_idx", "tid", "queue_idx", "value", "limit")]


class GtapError(RuntimeError):
    def __init__(self, code, where=""):
        self.code = code
        name = ERROR_NAMES.get(code, "CUDA_ERROR_%d" % (-code) if code < 0 else str(code))
        super().__init__("%s failed: %s (%d)" % (where, name, code))


_lib = None

# C signatures: (name, restype, argtypes)
_SIGS = [
    ("gtap_version", ctypes.c_char_p, []),
    ("gtap_default_config", ctypes.c_int, [ctypes.POINTER(Config)]),
    ("gtap_initialize", ctypes.c_int, [ctypes.POINTER(Config)]),
    ("gtap_finalize", ctypes.c_int, []),
    ("gtap_reset", ctypes.c_int, []),
    ("gtap_synchronize", ctypes.c_int, []),
    ("gtap_get_runtime_error_code", ctypes.c_int, [ctypes.POINTER(ctypes.c_int)]),
    ("gtap_check_runtime_error", ctypes.c_int, []),
    ("gtap_get_runtime_error_string", ctypes.c_char_p, [ctypes.c_int]),
    ("gtap_get_error_report", ctypes.c_int, [ctypes.POINTER(ErrorReport)]),
    ("gtap_get_config", ctypes.c_int, [ctypes.POINTER(Config)]),
    ("gtap_launch", ctypes.c_int,
     [ctypes.POINTER(Root), ctypes.c_int32, ctypes.POINTER(RootResult), ctypes.POINTER(RunStats), ctypes.c_void_p]),
    ("gtap_launch_per_root", ctypes.c_int,
     [ctypes.POINTER(Root), ctypes.c_int32, ctypes.POINTER(RootResult), ctypes.POINTER(RunStats), ctypes.c_void_p]),
    ("gtap_run_host", ctypes.c_int,
     [ctypes.POINTER(Root), ctypes.c_int32, ctypes.POINTER(RootResult), ctypes.POINTER(RunStats),
      ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    ("gtap_serve_start", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32]),
    ("gtap_serve_enqueue", ctypes.c_int, [ctypes.POINTER(Root), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    ("gtap_serve_poll", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    ("gtap_serve_results", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32), ctypes.c_int32, ctypes.POINTER(RootResult)]),
    ("gtap_serve_shutdown", ctypes.c_int, [ctypes.POINTER(RunStats)]),
    ("gtap_visualize_profile", ctypes.c_int, [ctypes.c_char_p]),
    ("gtap_write_profile", ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p]),
    ("gtap_selftest_queues", ctypes.c_int,
     [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32] + [ctypes.POINTER(ctypes.c_int64)] * 4),
    ("gtap_get_arena_counters", ctypes.c_int, [ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]),
    ("gtap_debug_set_ring_position", ctypes.c_int, [ctypes.c_int32, ctypes.c_uint32]),
    ("gtap_debug_admission_order", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    ("gtap_measure_atomic_rate", ctypes.c_int, [ctypes.c_int32, ctypes.c_int64, ctypes.POINTER(ctypes.c_double)]),
    ("gtap_launch_noalloc", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]),
    # support of the drop-in task-ABI header for caller-launched kernels
    ("gtap_external_initialize", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32]),
    ("gtap_external_prepare", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    ("gtap_external_finalize", ctypes.c_int, []),
    ("gtap_external_error_code", ctypes.c_int, [ctypes.POINTER(ctypes.c_int32)]),
    ("gtap_external_check", ctypes.c_int, []),
    ("gtap_gen_keys", ctypes.c_int, [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_int64]),
    ("gtap_gen_mix", ctypes.c_int, [ctypes.c_uint64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    ("gtap_gen_rmat", ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]),
    ("gtap_read_array_file", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    ("gtap_write_array_file", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64]),
    ("gtap_read_csr_file", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]),
    ("gtap_write_csr_file", ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]),
    ("gtap_gen_tree", ctypes.c_int,
     [ctypes.c_int32, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
]
EXPORTED = [s[0] for s in _SIGS]


def lib():
    """Load libgtap_b200.so (raises if it is missing: no fallback path)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libgtap_b200.so is not built; run `python -m gtap_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(rc, where):
    if rc != 0:
        raise GtapError(rc, where)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


# ---- reference-named host API ----------------------------------------------
def default_config(**overrides):
    c = Config()
    _check(lib().gtap_default_config(ctypes.byref(c)), "gtap_default_config")
    for k, v in overrides.items():
        setattr(c, k, v)
    return c


def gtap_initialize(config=None, **overrides):
    c = config if config is not None else default_config(**overrides)
    _check(lib().gtap_initialize(ctypes.byref(c)), "gtap_initialize")
    return current_config()


def gtap_finalize():
    _check(lib().gtap_finalize(), "gtap_finalize")


def gtap_reset():
    _check(lib().gtap_reset(), "gtap_reset")


def gtap_synchronize():
    return lib().gtap_synchronize()


def gtap_get_runtime_error_code():
    code = ctypes.c_int(0)
    _check(lib().gtap_get_runtime_error_code(ctypes.byref(code)), "gtap_get_runtime_error_code")
    return code.value


def gtap_check_runtime_error():
    return lib().gtap_check_runtime_error()


def gtap_get_runtime_error_string(code):
    return lib().gtap_get_runtime_error_string(code).decode()


def gtap_get_error_report():
    r = ErrorReport()
    _check(lib().gtap_get_error_report(ctypes.byref(r)), "gtap_get_error_report")
    return {n: getattr(r, n) for n, _ in ErrorReport._fields_}


def gtap_visualize_profile(app_name, directory=None):
    if directory is None:
        _check(lib().gtap_visualize_profile(app_name.encode()), "gtap_visualize_profile")
    else:
        _check(lib().gtap_write_profile(directory.encode(), app_name.encode()), "gtap_write_profile")


def current_config():
    c = Config()
    _check(lib().gtap_get_config(ctypes.byref(c)), "gtap_get_config")
    return c


# ---- roots -------------------------------------------------------------------
def fib_root(n, cutoff=0, epaq=False):
    return Root(kind=KIND_FIB, i0=n, i1=cutoff, i2=1 if epaq else 0)


def nq_root(n, cutoff_depth=None):
    """cutoff_depth None = one task per row (rows 0..n-1 fork)."""
    return Root(kind=KIND_NQ, i0=n, i1=(n - 1) if cutoff_depth is None else cutoff_depth)


def cilksort_root(src, arr, tmp, n, sort_cutoff=64, merge_cutoff=256):
    """src/arr/tmp: device (or, for run_host, host) int32 buffer addresses."""
    return Root(kind=KIND_CILKSORT, i0=sort_cutoff, i1=merge_cutoff, n=n, p0=src, p1=arr, p2=tmp)


def mergesort_root(src, out, tmp, n, cutoff=128, merge_cutoff=256):
    return Root(kind=KIND_MERGESORT, i0=cutoff, i1=merge_cutoff, n=n, p0=src, p1=out, p2=tmp)


def bfs_root(row, col, depth, nv, source, split=32):
    return Root(kind=KIND_BFS, i0=source, i1=split, n=nv, p0=row, p1=col, p2=depth)


def treesum_root(left, right, value, size, n, root_node=0, cutoff=32):
    return Root(kind=KIND_TREESUM, i0=root_node, i1=cutoff, n=n, p0=left, p1=right, p2=value, p3=size)


def _root_array(roots):
    arr = (Root * len(roots))()
    for i, r in enumerate(roots):
        arr[i] = r
    return arr


def launch(roots, stream=None, per_root=False):
    """One persistent launch over device-resident roots; returns (results, stats)."""
    arr = _root_array(roots)
    res = (RootResult * len(roots))()
    st = RunStats()
    f = lib().gtap_launch_per_root if per_root else lib().gtap_launch
    rc = f(arr, len(roots), res, ctypes.byref(st), ctypes.c_void_p(stream or 0))
    _check(rc, "gtap_launch_per_root" if per_root else "gtap_launch")
    return list(res), st


def run_host(roots):
    """Roots whose pointers are HOST buffers: copies in, one launch, copies out."""
    arr = _root_array(roots)
    res = (RootResult * len(roots))()
    st = RunStats()
    hin, hout = ctypes.c_int64(0), ctypes.c_int64(0)
    rc = lib().gtap_run_host(arr, len(roots), res, ctypes.byref(st), ctypes.byref(hin), ctypes.byref(hout))
    _check(rc, "gtap_run_host")
    return list(res), st, hin.value, hout.value


# ---- serve -------------------------------------------------------------------
def serve_start(ring_capacity=4096, admit_watermark=0):
    _check(lib().gtap_serve_start(ring_capacity, admit_watermark), "gtap_serve_start")


def serve_enqueue(roots):
    arr = _root_array(roots)
    first = ctypes.c_int32(0)
    _check(lib().gtap_serve_enqueue(arr, len(roots), ctypes.byref(first)), "gtap_serve_enqueue")
    return first.value


def serve_poll(max_n=4096):
    buf = (ctypes.c_int32 * max_n)()
    n = ctypes.c_int32(0)
    _check(lib().gtap_serve_poll(buf, max_n, ctypes.byref(n)), "gtap_serve_poll")
    return [buf[i] for i in range(n.value)]


def serve_results(indices):
    idx = (ctypes.c_int32 * len(indices))(*indices)
    out = (RootResult * len(indices))()
    _check(lib().gtap_serve_results(idx, len(indices), out), "gtap_serve_results")
    return list(out)


def serve_shutdown():
    st = RunStats()
    rc = lib().gtap_serve_shutdown(ctypes.byref(st))
    _check(rc, "gtap_serve_shutdown")
    return st


def arena_counters():
    out = (ctypes.c_int64 * 8)()
    _check(lib().gtap_get_arena_counters(out, 8), "gtap_get_arena_counters")
    keys = ("fresh_next", "fresh_base", "pool", "overflow_left", "completed", "total_ids", "workers", "status")
    return dict(zip(keys, list(out)))


def set_ring_position(position, target=0):
    """Testing aid: both global rings empty, cursors at `position` (0..2^32-1).
    target 0 = the gtap_initialize arena, 1 = gtap_launch_noalloc's scratch."""
    _check(lib().gtap_debug_set_ring_position(target, position & 0xFFFFFFFF), "gtap_debug_set_ring_position")


def admission_order(roots):
    """(order, n_light): the order a grouped batch launch admits roots in (host only)."""
    arr = _root_array(roots)
    order = (ctypes.c_int32 * max(1, len(roots)))()
    n_light = ctypes.c_int32(0)
    _check(lib().gtap_debug_admission_order(arr, len(roots), order, ctypes.byref(n_light)),
           "gtap_debug_admission_order")
    return [order[i] for i in range(len(roots))], n_light.value


def measure_atomic_rate(mode=0, ops=1 << 28):
    """Peak scattered 32-bit atomic adds per second (mode 0: atom.add with a
    return value; 1: red.add)."""
    v = ctypes.c_double(0.0)
    _check(lib().gtap_measure_atomic_rate(mode, ops, ctypes.byref(v)), "gtap_measure_atomic_rate")
    return v.value


def selftest_queues(rounds=60, per_round_max=32, mode=7):
    """Device exactly-once test of the deques and the overflow queue."""
    v = [ctypes.c_int64(0) for _ in range(4)]
    rc = lib().gtap_selftest_queues(rounds, per_round_max, mode, *[ctypes.byref(x) for x in v])
    return rc, dict(zip(("produced", "consumed", "duplicates", "lost"), [x.value for x in v]))


# ---- generators ----------------------------------------------------------------
def gen_keys(seed, n):
    out = np.empty(n, dtype=np.int32)
    _check(lib().gtap_gen_keys(seed, _ptr(out), n), "gtap_gen_keys")
    return out


def gen_mix(seed, n_roots):
    kind = np.empty(n_roots, np.int32)
    param = np.empty(n_roots, np.int32)
    key_seed = np.empty(n_roots, np.uint64)
    _check(lib().gtap_gen_mix(seed, n_roots, _ptr(kind), _ptr(param), _ptr(key_seed)), "gtap_gen_mix")
    return kind, param, key_seed


def gen_rmat(scale, edge_factor=16, seed=42):
    nv = 1 << scale
    row = np.empty(nv + 1, np.int32)
    col = np.empty(nv * edge_factor, np.int32)
    _check(lib().gtap_gen_rmat(scale, edge_factor, seed, _ptr(row), _ptr(col)), "gtap_gen_rmat")
    return row, col


def gen_tree(n, seed=42):
    left = np.empty(n, np.int32)
    right = np.empty(n, np.int32)
    value = np.empty(n, np.int32)
    size = np.empty(n, np.int32)
    _check(lib().gtap_gen_tree(n, seed, _ptr(left), _ptr(right), _ptr(value), _ptr(size)), "gtap_gen_tree")
    return left, right, value, size


# ---- the reference's input files ------------------------------------------------
def read_array(path):
    """An int32 array in the reference's gen_vector format (size_t n, int32[n])."""
    n = ctypes.c_int64(0)
    _check(lib().gtap_read_array_file(str(path).encode(), None, 0, ctypes.byref(n)), "gtap_read_array_file")
    out = np.empty(n.value, np.int32)
    _check(lib().gtap_read_array_file(str(path).encode(), _ptr(out), n.value, ctypes.byref(n)), "gtap_read_array_file")
    return out


def write_array(path, a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    _check(lib().gtap_write_array_file(str(path).encode(), _ptr(a), len(a)), "gtap_write_array_file")


def read_csr(path):
    """(row, col) from the reference's CSR binary (int N, int M, row[N+1], col[M])."""
    n, m = ctypes.c_int32(0), ctypes.c_int32(0)
    _check(lib().gtap_read_csr_file(str(path).encode(), None, 0, None, 0, ctypes.byref(n), ctypes.byref(m)),
           "gtap_read_csr_file")
    row = np.empty(n.value + 1, np.int32)
    col = np.empty(m.value, np.int32)
    _check(lib().gtap_read_csr_file(str(path).encode(), _ptr(row), len(row), _ptr(col), len(col), ctypes.byref(n),
                                    ctypes.byref(m)), "gtap_read_csr_file")
    return row, col


def write_csr(path, row, col):
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    _check(lib().gtap_write_csr_file(str(path).encode(), _ptr(row), _ptr(col), len(row) - 1, len(col)),
           "gtap_write_csr_file")


def max_degree_vertex(row):
    deg = np.diff(row)
    return int(np.argmax(deg))
