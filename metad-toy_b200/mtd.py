"""Python binding of libmetad_b200.so (the C ABI declared in include/metad_b200.h).

This mirrors the reference plugin's interface for one `fix metad` instance:
the constructor takes the fix arguments (the tokens after ``fix ID group metad``),
``post_force`` is ``FixMetadynamics::post_force``, ``compute_scalar`` /
``compute_vector`` are the thermo outputs and ``extract`` is
``Fix::extract("colvar_peratom:<CAL>.<prop>")``.  Errors raise ``MetadError``
with the library's message, the way the reference stops on ``error->all``.

There is no CPU fallback: if the shared library is missing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmetad_b200.so")
HEADER = os.path.join(HERE, "..", "include", "metad_b200.h")

MTD_OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "PARSE", 3: "CUDA", 4: "OOM", 5: "NEIGH_OVERFLOW",
                6: "TIMEOUT", 7: "NAN", 8: "IO", 9: "UNSUPPORTED"}
PREC = {"mixed": 0, "fp64": 1}

# Every entry point declared in include/metad_b200.h.
EXPORTS = ["mtd_options_default", "mtd_create", "mtd_destroy", "mtd_parse_args", "mtd_eval_expression", "mtd_set_box", "mtd_init", "mtd_post_force",
           "mtd_post_force_device", "mtd_sync", "mtd_compute_scalar", "mtd_compute_vector", "mtd_cv_dim",
           "mtd_extract_peratom", "mtd_get_neighbors", "mtd_neighbor_stats", "mtd_neighbor_set_wait", "mtd_set_host_copy_mode", "mtd_host_copy_mode_in_use", "mtd_sk_tiles", "mtd_set_sk_tiles", "mtd_get_tuning", "mtd_set_tuning_all", "mtd_hills_replay", "mtd_get_grid", "mtd_last_launch_count",
           "mtd_set_stream", "mtd_profile_enable", "mtd_profile_report",
           "mtd_max_neighbors", "mtd_last_error", "mtd_abi_version", "mtd_sk_noalloc", "mtd_nn_state",
           "mtd_nnbias_create", "mtd_nnbias_destroy", "mtd_nnbias_last_error", "mtd_nnbias_add_hills",
           "mtd_nnbias_num_hills", "mtd_nnbias_exact", "mtd_nnbias_eval", "mtd_nnbias_fit", "mtd_nnbias_validate",
           "mtd_nnbias_usable", "mtd_nnbias_point_device", "mtd_nnbias_eval_device", "mtd_nnbias_get_params", "mtd_nnbias_set_params",
           "mtd_nnbias_vscale", "mtd_nnbias_loss_grad", "mtd_nnbias_set_wait", "mtd_nnbias_sync",
           "mtd_walkers_create", "mtd_walkers_destroy", "mtd_walkers_last_error", "mtd_walkers_count",
           "mtd_walkers_set_box", "mtd_walkers_init", "mtd_walkers_enable_graph", "mtd_walkers_step_device",
           "mtd_walkers_sync", "mtd_walkers_cv", "mtd_walkers_bias", "mtd_walkers_get_grid",
           "mtd_walkers_last_launch_count", "mtd_walkers_enable_persistent", "mtd_walkers_persistent_active",
           "mtd_walkers_set_wait", "mtd_autotune", "mtd_set_tuning", "mtd_walkers_autotune", "mtd_set_types", "mtd_needs_types",
           "mtd_set_domain", "mtd_set_nlocal", "mtd_ghost_cutoff",
           "mtd_set_positions_f64", "mtd_step", "mtd_get_peratom", "mtd_create_from_config",
           "mtd_set_domain_device", "mtd_walkers_set_ranks", "mtd_walkers_set_ranks_device"]


class MetadError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("device", C.c_int), ("boltz", C.c_double), ("n_groups", C.c_int),
                ("group_names", C.POINTER(C.c_char_p)), ("group_bits", C.POINTER(C.c_int)),
                ("hills_path", C.c_char_p), ("work_dir", C.c_char_p)]


class Config(C.Structure):
    _fields_ = [("narg", C.c_int), ("arg", C.POINTER(C.c_char_p)), ("opt", Options)]


_lib = None

# int (*)(double *buf, int count, void *user): in-place sum of buf over the ranks
ALLREDUCE_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int, C.c_void_p)
# int (*)(double *d_buf, int count, void *stream, void *user): enqueue that sum on the stream
ALLREDUCE_DEVICE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p)
# int (*)(const double *send, int count, double *recv, void *user): every rank's send, in rank order
ALLGATHER_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_void_p)
# int (*)(const double *d_send, int count, double *d_recv, void *stream, void *user)
ALLGATHER_DEVICE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p)
WALK_REC = 8   # doubles per walker in the exchange: s[4], height, deposit flag, overflow flag, 0


def build(jobs=8):
    """Compile libmetad_b200.so for sm_100a with the package Makefile."""
    subprocess.check_call(["make", "-s", "-j%d" % jobs, "-C", HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libmetad_b200.so is not built (run `make -C metad-toy_b200` or "
                              "__graft_entry__.build()); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.mtd_options_default.argtypes = [C.POINTER(Options)]
        L.mtd_create.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(Options), C.POINTER(vp)]
        L.mtd_destroy.argtypes = [vp]
        L.mtd_set_box.argtypes = [vp, dp, dp, ip]
        L.mtd_init.argtypes = [vp]
        L.mtd_post_force.argtypes = [vp, C.c_int64, C.c_int, vp, vp, vp, vp, vp]
        L.mtd_post_force_device.argtypes = [vp, C.c_int64, C.c_int, vp, vp, vp, vp, vp]
        L.mtd_sync.argtypes = [vp]
        L.mtd_compute_scalar.argtypes = [vp]
        L.mtd_compute_scalar.restype = C.c_double
        L.mtd_compute_vector.argtypes = [vp, C.c_int]
        L.mtd_compute_vector.restype = C.c_double
        L.mtd_cv_dim.argtypes = [vp]
        L.mtd_extract_peratom.argtypes = [vp, C.c_char_p, dp, C.c_int]
        L.mtd_hills_replay.argtypes = [vp, C.c_char_p]
        L.mtd_get_grid.argtypes = [vp, dp, C.c_int64]
        L.mtd_last_launch_count.argtypes = [vp]
        L.mtd_max_neighbors.argtypes = [vp, C.c_char_p]
        L.mtd_get_neighbors.argtypes = [vp, C.c_char_p, C.c_int, ip, ip, C.c_int]
        L.mtd_neighbor_stats.argtypes = [vp, C.POINTER(C.c_int64), ip]
        L.mtd_neighbor_set_wait.argtypes = [vp, C.c_int, C.c_int]
        L.mtd_set_host_copy_mode.argtypes = [vp, C.c_int]
        L.mtd_host_copy_mode_in_use.argtypes = [vp, C.POINTER(C.c_int)]
        L.mtd_sk_tiles.argtypes = [vp, ip, ip]
        L.mtd_get_tuning.argtypes = [vp, ip]
        L.mtd_set_tuning_all.argtypes = [vp, ip]
        L.mtd_set_sk_tiles.argtypes = [vp, C.c_int, C.c_int]
        L.mtd_set_types.argtypes = [vp, C.c_int, C.POINTER(C.c_int)]
        L.mtd_needs_types.argtypes = [vp]
        L.mtd_set_domain.argtypes = [vp, C.c_int, C.c_int, ALLREDUCE_FN, vp]
        L.mtd_set_domain_device.argtypes = [vp, C.c_int, C.c_int, ALLREDUCE_DEVICE_FN, vp]
        L.mtd_set_nlocal.argtypes = [vp, C.c_int]
        L.mtd_walkers_set_ranks.argtypes = [vp, C.c_int, C.c_int, ALLGATHER_FN, vp]
        L.mtd_walkers_set_ranks_device.argtypes = [vp, C.c_int, C.c_int, ALLGATHER_DEVICE_FN, vp]
        L.mtd_ghost_cutoff.argtypes = [vp]
        L.mtd_ghost_cutoff.restype = C.c_double
        L.mtd_set_positions_f64.argtypes = [vp, dp, ip, ip, C.c_int, C.c_int]
        L.mtd_step.argtypes = [vp, C.c_int64, dp, dp, dp, dp]
        L.mtd_get_peratom.argtypes = [vp, C.c_char_p, dp]
        L.mtd_create_from_config.argtypes = [C.POINTER(Config), C.POINTER(vp)]
        L.mtd_autotune.argtypes = [vp, C.c_int, vp, vp, C.c_int, C.POINTER(C.c_int)]
        L.mtd_set_tuning.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.mtd_walkers_autotune.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_void_p), C.c_int,
                                           C.POINTER(C.c_int)]
        L.mtd_last_error.argtypes = [vp]
        L.mtd_last_error.restype = C.c_char_p
        L.mtd_abi_version.restype = C.c_int
        L.mtd_set_stream.argtypes = [vp, vp]
        L.mtd_profile_enable.argtypes = [vp, C.c_int]
        L.mtd_profile_report.argtypes = [vp, C.c_char_p, C.c_int]
        L.mtd_parse_args.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.POINTER(Options), C.c_char_p, C.c_int]
        L.mtd_eval_expression.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), dp, dp, dp]
        L.mtd_nn_state.argtypes = [vp, ip, ip, ip]
        L.mtd_walkers_create.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_char_p), C.POINTER(Options), C.POINTER(vp)]
        L.mtd_walkers_destroy.argtypes = [vp]
        L.mtd_walkers_last_error.argtypes = [vp]
        L.mtd_walkers_last_error.restype = C.c_char_p
        L.mtd_walkers_count.argtypes = [vp]
        L.mtd_walkers_set_box.argtypes = [vp, C.c_int, dp, dp, ip]
        L.mtd_walkers_init.argtypes = [vp]
        L.mtd_walkers_enable_graph.argtypes = [vp, C.c_int]
        L.mtd_walkers_step_device.argtypes = [vp, C.c_int64, ip, C.POINTER(vp), C.POINTER(vp)]
        L.mtd_walkers_sync.argtypes = [vp]
        L.mtd_walkers_cv.argtypes = [vp, C.c_int, C.c_int]
        L.mtd_walkers_cv.restype = C.c_double
        L.mtd_walkers_bias.argtypes = [vp, C.c_int]
        L.mtd_walkers_bias.restype = C.c_double
        L.mtd_walkers_get_grid.argtypes = [vp, dp, C.c_int64]
        L.mtd_walkers_last_launch_count.argtypes = [vp]
        L.mtd_walkers_enable_persistent.argtypes = [vp, C.c_int]
        L.mtd_walkers_persistent_active.argtypes = [vp]
        L.mtd_walkers_set_wait.argtypes = [vp, C.c_int, C.c_int]
        L.mtd_nnbias_create.argtypes = [C.c_int, dp, dp, C.c_uint64, C.POINTER(vp)]
        L.mtd_nnbias_destroy.argtypes = [vp]
        L.mtd_nnbias_last_error.argtypes = [vp]
        L.mtd_nnbias_last_error.restype = C.c_char_p
        L.mtd_nnbias_add_hills.argtypes = [vp, C.c_int, dp, dp, dp]
        L.mtd_nnbias_num_hills.argtypes = [vp]
        L.mtd_nnbias_exact.argtypes = [vp, C.c_int, dp, dp, dp]
        L.mtd_nnbias_eval.argtypes = [vp, C.c_int, dp, dp, dp]
        L.mtd_nnbias_fit.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_uint64, dp]
        L.mtd_nnbias_validate.argtypes = [vp, C.c_int, C.c_uint64, C.c_double, dp, dp]
        L.mtd_nnbias_usable.argtypes = [vp]
        L.mtd_nnbias_point_device.argtypes = [vp, vp, vp, vp, C.c_int, vp]
        L.mtd_nnbias_eval_device.argtypes = [vp, C.c_int, vp, vp, vp, C.c_int, vp]
        L.mtd_nnbias_get_params.argtypes = [vp, C.POINTER(C.c_float)]
        L.mtd_nnbias_set_params.argtypes = [vp, C.POINTER(C.c_float), C.c_double]
        L.mtd_nnbias_vscale.argtypes = [vp]
        L.mtd_nnbias_vscale.restype = C.c_double
        L.mtd_nnbias_loss_grad.argtypes = [vp, C.c_int, dp, dp, C.c_double, C.POINTER(C.c_float), dp]
        L.mtd_nnbias_set_wait.argtypes = [vp, C.c_int, C.c_int]
        L.mtd_nnbias_sync.argtypes = [vp]
        L.mtd_sk_noalloc.argtypes = [C.c_int, vp, vp, C.c_int, C.c_int, vp, C.c_int, vp, vp, vp, C.c_char_p,
                                     C.c_int]
        _lib = L
    return _lib


def _options(precision="mixed", device=0, boltz=8.617343e-5, groups=None, hills_path="", work_dir=None):
    groups = groups or {"all": 1}
    names = (C.c_char_p * len(groups))(*[g.encode() for g in groups])
    bits = (C.c_int * len(groups))(*[int(b) for b in groups.values()])
    opt = Options()
    lib().mtd_options_default(C.byref(opt))
    opt.precision = PREC[precision]
    opt.device = int(device)
    opt.boltz = float(boltz)
    opt.n_groups = len(groups)
    opt.group_names = C.cast(names, C.POINTER(C.c_char_p))
    opt.group_bits = C.cast(bits, C.POINTER(C.c_int))
    opt.hills_path = hills_path.encode() if hills_path is not None else None
    opt.work_dir = work_dir.encode() if work_dir else None
    return opt, (names, bits)


def parse_args(args, groups=None):
    """Host-only grammar check: returns "" when `args` would build a context, else the message."""
    opt, keep = _options(groups=groups)
    toks = [str(a).encode() for a in args]
    argv = (C.c_char_p * max(1, len(toks)))(*toks)
    buf = C.create_string_buffer(1024)
    lib().mtd_parse_args(len(toks), argv, C.byref(opt), buf, 1024)
    return buf.value.decode()


def sk_noalloc(n, x_ptr, k_ptr, nk, s_ptr, rho_ptr=0, mask_ptr=0, groupbit=1, precision="mixed", stream=0):
    """Allocation-free k-vector S(k) on device buffers (integer device pointers);
    enqueues on `stream` (a cudaStream_t handle, 0 = default) and returns."""
    buf = C.create_string_buffer(256)
    st = lib().mtd_sk_noalloc(int(n), C.c_void_p(x_ptr or None), C.c_void_p(mask_ptr or None), int(groupbit),
                              int(nk), C.c_void_p(k_ptr or None), PREC[precision], C.c_void_p(rho_ptr or None),
                              C.c_void_p(s_ptr or None), C.c_void_p(stream or None), buf, 256)
    if st != 0:
        raise MetadError(st, buf.value.decode())


def eval_expression(expr, values):
    """Host evaluation of a DIM expression: (value, {symbol: derivative})."""
    names = list(values)
    n = len(names)
    carr = (C.c_char_p * max(1, n))(*[k.encode() for k in names])
    vals = np.ascontiguousarray([values[k] for k in names], dtype=np.float64)
    out = np.zeros(1)
    grad = np.zeros(max(1, n))
    st = lib().mtd_eval_expression(expr.encode(), n, carr, vals.ctypes.data_as(C.POINTER(C.c_double)),
                                   out.ctypes.data_as(C.POINTER(C.c_double)),
                                   grad.ctypes.data_as(C.POINTER(C.c_double)))
    if st != MTD_OK:
        raise MetadError(st, "cannot evaluate expression %r" % expr)
    return out[0], dict(zip(names, grad[:n]))


def _ptr(a):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Metad:
    """One `fix metad` instance on one GPU."""

    def __init__(self, args, precision="mixed", device=0, boltz=8.617343e-5, groups=None,
                 hills_path="", work_dir=None):
        L = lib()
        opt, self._keep = _options(precision, device, boltz, groups, hills_path, work_dir)
        toks = [str(a).encode() for a in args]
        argv = (C.c_char_p * max(1, len(toks)))(*toks)
        h = C.c_void_p()
        st = L.mtd_create(len(toks), argv, C.byref(opt), C.byref(h))
        self._h = h
        if st != MTD_OK:
            msg = L.mtd_last_error(h).decode() if h else "mtd_create failed"
            if h:
                L.mtd_destroy(h)
            self._h = None
            raise MetadError(st, msg)
        self.cv_dim = L.mtd_cv_dim(h)

    def _check(self, st):
        if st != MTD_OK:
            raise MetadError(st, lib().mtd_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().mtd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_box(self, lo, hi, periodic=(1, 1, 1)):
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        hi = np.ascontiguousarray(hi, dtype=np.float64)
        pe = np.ascontiguousarray(periodic, dtype=np.int32)
        self._check(lib().mtd_set_box(self._h, lo.ctypes.data_as(C.POINTER(C.c_double)),
                                      hi.ctypes.data_as(C.POINTER(C.c_double)),
                                      pe.ctypes.data_as(C.POINTER(C.c_int))))

    def init(self):
        self._check(lib().mtd_init(self._h))

    def post_force(self, step, x, f, mask=None, image=None, virial=False):
        """f (n x 3, float64, C order) is updated in place: f -= bias force."""
        assert x.dtype == np.float64 and x.flags.c_contiguous and f.dtype == np.float64 and f.flags.c_contiguous
        n = x.shape[0]
        v = np.zeros(6) if virial else None
        m = np.ascontiguousarray(mask, dtype=np.int32) if mask is not None else None
        im = np.ascontiguousarray(image, dtype=np.int32) if image is not None else None
        self._check(lib().mtd_post_force(self._h, int(step), n, _ptr(x), _ptr(m), _ptr(im), _ptr(f), _ptr(v)))
        return v

    def post_force_device(self, step, n, x_ptr, f_in_ptr, f_out_ptr, mask_ptr=0, image_ptr=0):
        """Device pointers (ints); asynchronous on the context stream."""
        self._check(lib().mtd_post_force_device(self._h, int(step), int(n), C.c_void_p(x_ptr),
                                                C.c_void_p(mask_ptr or None), C.c_void_p(image_ptr or None),
                                                C.c_void_p(f_in_ptr), C.c_void_p(f_out_ptr)))

    def sync(self):
        self._check(lib().mtd_sync(self._h))

    def compute_scalar(self):
        return lib().mtd_compute_scalar(self._h)

    def compute_vector(self, k):
        return lib().mtd_compute_vector(self._h, int(k))

    @property
    def cv(self):
        return np.array([self.compute_vector(k) for k in range(self.cv_dim)])

    def extract(self, key, n):
        out = np.zeros(n)
        self._check(lib().mtd_extract_peratom(self._h, key.encode(), out.ctypes.data_as(C.POINTER(C.c_double)), n))
        return out

    def hills_replay(self, path):
        self._check(lib().mtd_hills_replay(self._h, path.encode()))

    def grid(self, size):
        out = np.zeros(size)
        self._check(lib().mtd_get_grid(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), size))
        return out

    def launch_count(self):
        return lib().mtd_last_launch_count(self._h)

    def max_neighbors(self, cal):
        return lib().mtd_max_neighbors(self._h, cal.encode())

    def neighbor_stats(self):
        """(rebuilds so far, whether the last step used skin lists)."""
        r, a = C.c_int64(), C.c_int()
        self._check(lib().mtd_neighbor_stats(self._h, C.byref(r), C.byref(a)))
        return r.value, bool(a.value)

    def tuning(self):
        """{name: value} of every tuned shape (results never depend on them)."""
        a = (C.c_int * 6)()
        self._check(lib().mtd_get_tuning(self._h, a))
        keys = ["neighbors", "q_block", "lambda_block", "q_filter_split", "sk_q_values", "sk_force_unroll"]
        return dict(zip(keys, list(a)))

    def set_tuning_all(self, neighbors, q_block, lambda_block, q_filter_split, sk_q_values, sk_force_unroll):
        a = (C.c_int * 6)(neighbors, q_block, lambda_block, q_filter_split, sk_q_values, sk_force_unroll)
        self._check(lib().mtd_set_tuning_all(self._h, a))

    def sk_tiles(self):
        """S(k) shapes: (k-vectors per value pass, unroll depth of the force pass)."""
        a, b = C.c_int(), C.c_int()
        self._check(lib().mtd_sk_tiles(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_sk_tiles(self, q_values, q_force):
        self._check(lib().mtd_set_sk_tiles(self._h, int(q_values), int(q_force)))

    def set_host_copy_mode(self, mode):
        """f over the host link for mtd_post_force: 1 copies, 2 upload + zero-copy write, 3 zero copy;
        0 (default): the first calls time modes 1-3 and the fastest is kept."""
        self._check(lib().mtd_set_host_copy_mode(self._h, int(mode)))

    def host_copy_mode_in_use(self):
        """The caller's mode, or the one the timing trial of mode 0 picked (0 while it runs)."""
        m = C.c_int()
        self._check(lib().mtd_host_copy_mode_in_use(self._h, C.byref(m)))
        return m.value

    def neighbor_set_wait(self, limit=0, stall=False):
        """Grid-barrier wait limit of the one-launch skin-list rebuild (0: default);
        stall=True makes the next rebuild's waits run out (MTD_ERR_TIMEOUT)."""
        self._check(lib().mtd_neighbor_set_wait(self._h, int(limit), 1 if stall else 0))

    def neighbors(self, cal, n, max_per_atom=None):
        """Last step's neighbour lists of CAL `cal`: (counts[n], lists) with
        lists an (n, max_per_atom) array of ascending caller indices, -1
        padded (None when max_per_atom is None)."""
        counts = np.zeros(n, dtype=np.int32)
        ip = C.POINTER(C.c_int)
        if max_per_atom is None:
            self._check(lib().mtd_get_neighbors(self._h, cal.encode(), int(n), counts.ctypes.data_as(ip), None, 0))
            return counts, None
        idx = np.zeros((n, max_per_atom), dtype=np.int32)
        self._check(lib().mtd_get_neighbors(self._h, cal.encode(), int(n), counts.ctypes.data_as(ip),
                                            idx.ctypes.data_as(ip), int(max_per_atom)))
        return counts, idx

    def autotune(self, n, x_ptr, mask_ptr=0, reps=5):
        """Device pointers (ints); returns (neighbour shape, q block, lambda block)."""
        ch = (C.c_int * 3)()
        self._check(lib().mtd_autotune(self._h, int(n), C.c_void_p(x_ptr), C.c_void_p(mask_ptr or None), int(reps),
                                       ch))
        return tuple(ch)

    def set_types(self, types):
        """Atom types (caller order) for STRU_FACTOR Chemical."""
        t = np.ascontiguousarray(types, dtype=np.int32)
        self._check(lib().mtd_set_types(self._h, int(t.shape[0]), t.ctypes.data_as(C.POINTER(C.c_int))))

    @property
    def needs_types(self):
        return bool(lib().mtd_needs_types(self._h))

    def set_positions(self, x, types=None, mask=None, groupbit=1):
        """First call of the two-call step: x (n x 3 float64) and optional
        types / mask, copied to the device before returning."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        t = np.ascontiguousarray(types, dtype=np.int32) if types is not None else None
        m = np.ascontiguousarray(mask, dtype=np.int32) if mask is not None else None
        ip = C.POINTER(C.c_int)
        self._check(lib().mtd_set_positions_f64(self._h, x.ctypes.data_as(C.POINTER(C.c_double)),
                                                t.ctypes.data_as(ip) if t is not None else None,
                                                m.ctypes.data_as(ip) if m is not None else None,
                                                int(x.shape[0]), int(groupbit)))

    def step(self, step, f, virial=False):
        """Second call: f (n x 3 float64) -= bias force in place; returns
        (cv, bias energy, virial or None)."""
        assert f.dtype == np.float64 and f.flags.c_contiguous
        cv = np.zeros(self.cv_dim)
        b = np.zeros(1)
        v = np.zeros(6) if virial else None
        dp = C.POINTER(C.c_double)
        self._check(lib().mtd_step(self._h, int(step), f.ctypes.data_as(dp), cv.ctypes.data_as(dp),
                                   b.ctypes.data_as(dp), v.ctypes.data_as(dp) if v is not None else None))
        return cv, b[0], v

    def get_peratom(self, key, n):
        out = np.zeros(n)
        self._check(lib().mtd_get_peratom(self._h, key.encode(), out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def set_domain(self, nlocal, rank, allreduce):
        """Domain decomposition: the first nlocal atoms of each step are owned,
        the rest ghosts.  allreduce(buf) must replace the float64 array buf, in
        place, with its element-wise sum over all ranks (identical on every
        rank); it is called once per step from inside post_force."""
        def cb(ptr, count, _user):
            try:
                allreduce(np.ctypeslib.as_array(ptr, shape=(count,)))
                return 0
            except Exception as e:  # reported through the step's status
                self._domain_error = e
                return 1
        self._domain_error = None
        self._domain_cb = ALLREDUCE_FN(cb)   # kept alive as long as the context
        self._check(lib().mtd_set_domain(self._h, int(nlocal), int(rank), self._domain_cb, None))

    def set_domain_device(self, nlocal, rank, allreduce):
        """Domain decomposition with the exchange on the device:
        allreduce(ptr, count, stream) gets the device address of count float64
        totals and the context's cudaStream_t (ints) and must enqueue their
        in-place sum over all ranks on that stream (domain.TorchDeviceAllreduce
        does it with torch.distributed / NCCL)."""
        def cb(ptr, count, stream, _user):
            try:
                allreduce(int(ptr or 0), int(count), int(stream or 0))
                return 0
            except Exception as e:  # reported through the step's status
                self._domain_error = e
                return 1
        self._domain_error = None
        self._domain_cb = ALLREDUCE_DEVICE_FN(cb)
        self._check(lib().mtd_set_domain_device(self._h, int(nlocal), int(rank), self._domain_cb, None))

    def set_nlocal(self, nlocal):
        self._check(lib().mtd_set_nlocal(self._h, int(nlocal)))

    @property
    def ghost_cutoff(self):
        return lib().mtd_ghost_cutoff(self._h)

    def set_tuning(self, neighbor_shape=0, q_block=0, lambda_block=0):
        self._check(lib().mtd_set_tuning(self._h, int(neighbor_shape), int(q_block), int(lambda_block)))

    def nn_state(self):
        """(hills, hills fitted, network in use) of the hill-list bias."""
        h, f, u = C.c_int(), C.c_int(), C.c_int()
        self._check(lib().mtd_nn_state(self._h, C.byref(h), C.byref(f), C.byref(u)))
        return h.value, f.value, bool(u.value)

    def set_stream(self, stream_ptr):
        """Run on an external cudaStream_t (an int handle, e.g. torch's cuda_stream); 0 = own stream."""
        self._check(lib().mtd_set_stream(self._h, C.c_void_p(stream_ptr or None)))

    def profile(self, enable=True):
        self._check(lib().mtd_profile_enable(self._h, 1 if enable else 0))

    def profile_report(self):
        """{kernel name: (calls, total ms)} accumulated since profile(True)."""
        need = lib().mtd_profile_report(self._h, None, 0)
        buf = C.create_string_buffer(max(need, 1))
        lib().mtd_profile_report(self._h, buf, need)
        out = {}
        for line in buf.value.decode().splitlines():
            name, calls, ms = line.split()
            out[name] = (int(calls), float(ms))
        return out


NN_PARAMS = 17281


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class NNBias:
    """Learned bias V_theta(s) (MLP D -> 128 -> 128 -> 1, BF16 weights, trained
    on the device on the FP64 hill sum, which stays its check and fallback)."""

    def __init__(self, lo, hi, seed=1):
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        hi = np.ascontiguousarray(hi, dtype=np.float64)
        self.D = lo.shape[0]
        h = C.c_void_p()
        st = lib().mtd_nnbias_create(self.D, _dp(lo), _dp(hi), int(seed), C.byref(h))
        self._h = h
        if st != 0:
            msg = lib().mtd_nnbias_last_error(h).decode() if h else ""
            lib().mtd_nnbias_destroy(h)
            self._h = None
            raise MetadError(st, msg)

    def _check(self, st):
        if st != 0:
            raise MetadError(st, lib().mtd_nnbias_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().mtd_nnbias_destroy(self._h)
            self._h = None

    def sync_device(self):
        """Waits for the object's stream; raises TIMEOUT if a network tile gave up a wait."""
        self._check(lib().mtd_nnbias_sync(self._h))

    def set_wait(self, tries=0, stall=False):
        """Limit of the tile kernel's tensor-core waits (0: default); stall=True
        makes the next batched call take the timeout path (MTD_ERR_TIMEOUT)."""
        self._check(lib().mtd_nnbias_set_wait(self._h, int(tries), 1 if stall else 0))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_hills(self, centers, heights, sigmas):
        c = np.ascontiguousarray(centers, dtype=np.float64).reshape(-1, self.D)
        h = np.ascontiguousarray(heights, dtype=np.float64).reshape(-1)
        s = np.ascontiguousarray(sigmas, dtype=np.float64).reshape(-1)
        self._check(lib().mtd_nnbias_add_hills(self._h, c.shape[0], _dp(c), _dp(h), _dp(s)))

    @property
    def num_hills(self):
        return lib().mtd_nnbias_num_hills(self._h)

    def exact(self, pts):
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, self.D)
        V = np.zeros(p.shape[0])
        dV = np.zeros_like(p)
        self._check(lib().mtd_nnbias_exact(self._h, p.shape[0], _dp(p), _dp(V), _dp(dV)))
        return V, dV

    def eval(self, pts):
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, self.D)
        V = np.zeros(p.shape[0])
        dV = np.zeros_like(p)
        self._check(lib().mtd_nnbias_eval(self._h, p.shape[0], _dp(p), _dp(V), _dp(dV)))
        return V, dV

    def fit(self, ntrain=262144, iters=2000, batch=4096, lr=2e-3, seed=1):
        loss = C.c_double()
        self._check(lib().mtd_nnbias_fit(self._h, int(ntrain), int(iters), int(batch), float(lr), int(seed),
                                         C.byref(loss)))
        return loss.value

    def validate(self, npts=65536, seed=7, tol=1e-3):
        mx, rms = C.c_double(), C.c_double()
        self._check(lib().mtd_nnbias_validate(self._h, int(npts), int(seed), float(tol), C.byref(mx), C.byref(rms)))
        return mx.value, rms.value

    @property
    def usable(self):
        return bool(lib().mtd_nnbias_usable(self._h))

    def point_device(self, s_ptr, v_ptr, dv_ptr, use_nn=-1, stream=0):
        self._check(lib().mtd_nnbias_point_device(self._h, C.c_void_p(s_ptr), C.c_void_p(v_ptr),
                                                  C.c_void_p(dv_ptr), int(use_nn), C.c_void_p(stream or None)))

    def eval_device(self, npts, pts_ptr, v_ptr, dv_ptr=0, use_nn=-1, stream=0):
        """Device pointers (ints): npts rows of D doubles in, V (and dV/ds rows) out."""
        self._check(lib().mtd_nnbias_eval_device(self._h, int(npts), C.c_void_p(pts_ptr), C.c_void_p(v_ptr),
                                                 C.c_void_p(dv_ptr or None), int(use_nn), C.c_void_p(stream or None)))

    def get_params(self):
        w = np.zeros(NN_PARAMS, dtype=np.float32)
        self._check(lib().mtd_nnbias_get_params(self._h, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def set_params(self, w, vscale):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(lib().mtd_nnbias_set_params(self._h, w.ctypes.data_as(C.POINTER(C.c_float)), float(vscale)))

    @property
    def vscale(self):
        return lib().mtd_nnbias_vscale(self._h)

    def loss_grad(self, pts, targets, vscale):
        p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, self.D)
        t = np.ascontiguousarray(targets, dtype=np.float64)
        g = np.zeros(NN_PARAMS, dtype=np.float32)
        loss = C.c_double()
        self._check(lib().mtd_nnbias_loss_grad(self._h, p.shape[0], _dp(p), _dp(t), float(vscale),
                                               g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return g, loss.value


class Walkers:
    """nwalk walkers sharing one bias grid (mtd_walkers_*); every walker is a
    context built from the same `fix metad` arguments."""

    def __init__(self, nwalk, args, precision="mixed", device=0, groups=None, hills_path="", work_dir=None):
        opt, self._keep = _options(precision, device, groups=groups, hills_path=hills_path, work_dir=work_dir)
        toks = [str(a).encode() for a in args]
        argv = (C.c_char_p * max(1, len(toks)))(*toks)
        h = C.c_void_p()
        st = lib().mtd_walkers_create(int(nwalk), len(toks), argv, C.byref(opt), C.byref(h))
        self._h = h
        self.n = int(nwalk)
        if st != 0:
            msg = lib().mtd_walkers_last_error(h).decode() if h else ""
            lib().mtd_walkers_destroy(h)
            self._h = None
            raise MetadError(st, msg)

    def _check(self, st):
        if st != 0:
            raise MetadError(st, lib().mtd_walkers_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().mtd_walkers_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_box(self, k, lo, hi, periodic=(1, 1, 1)):
        lo = np.ascontiguousarray(lo, dtype=np.float64)
        hi = np.ascontiguousarray(hi, dtype=np.float64)
        per = (C.c_int * 3)(*[int(p) for p in periodic])
        self._check(lib().mtd_walkers_set_box(self._h, int(k), _dp(lo), _dp(hi), per))

    def init(self):
        self._check(lib().mtd_walkers_init(self._h))

    def enable_graph(self, on=True):
        self._check(lib().mtd_walkers_enable_graph(self._h, 1 if on else 0))

    def set_ranks(self, rank, nranks, allgather):
        """Shard walkers over ranks: allgather(send, recv) fills the float64
        array recv (nranks * len(send)) with every rank's send in rank order."""
        def cb(sp, count, rp, _user):
            try:
                allgather(np.ctypeslib.as_array(sp, shape=(count,)),
                          np.ctypeslib.as_array(rp, shape=(count * nranks,)))
                return 0
            except Exception as e:
                self._rank_error = e
                return 1
        self._rank_error = None
        self._rank_cb = ALLGATHER_FN(cb)
        self._check(lib().mtd_walkers_set_ranks(self._h, int(rank), int(nranks), self._rank_cb, None))

    def set_ranks_device(self, rank, nranks, allgather):
        """Device variant: allgather(send_ptr, count, recv_ptr, stream) enqueues
        the gather on the walkers' stream (ints: device addresses, cudaStream_t)."""
        def cb(sp, count, rp, stream, _user):
            try:
                allgather(int(sp or 0), int(count), int(rp or 0), int(stream or 0))
                return 0
            except Exception as e:
                self._rank_error = e
                return 1
        self._rank_error = None
        self._rank_cb = ALLGATHER_DEVICE_FN(cb)
        self._check(lib().mtd_walkers_set_ranks_device(self._h, int(rank), int(nranks), self._rank_cb, None))

    def step_device(self, step, ns, x_ptrs, f_ptrs):
        n = (C.c_int * self.n)(*[int(v) for v in ns])
        xp = (C.c_void_p * self.n)(*[int(p) for p in x_ptrs])
        fp = (C.c_void_p * self.n)(*[int(p) for p in f_ptrs])
        self._check(lib().mtd_walkers_step_device(self._h, int(step), n, xp, fp))

    def sync(self):
        self._check(lib().mtd_walkers_sync(self._h))

    def cv(self, k, dim):
        return np.array([lib().mtd_walkers_cv(self._h, int(k), d) for d in range(dim)])

    def bias(self, k):
        return lib().mtd_walkers_bias(self._h, int(k))

    def grid(self, size):
        out = np.zeros(size)
        self._check(lib().mtd_walkers_get_grid(self._h, out.ctypes.data_as(C.POINTER(C.c_double)), int(size)))
        return out

    def launch_count(self):
        return lib().mtd_walkers_last_launch_count(self._h)

    def enable_persistent(self, on=True):
        """One persistent kernel launch per step where the deck allows it (default on)."""
        self._check(lib().mtd_walkers_enable_persistent(self._h, 1 if on else 0))

    @property
    def persistent_active(self):
        return bool(lib().mtd_walkers_persistent_active(self._h))

    def set_wait(self, limit=0, stall=False):
        """Grid-barrier wait limit of the persistent step (0: default); stall=True
        makes the next step's waits run out (MTD_ERR_TIMEOUT from sync)."""
        self._check(lib().mtd_walkers_set_wait(self._h, int(limit), 1 if stall else 0))

    def autotune(self, ns, x_ptrs, reps=5):
        """Per walker (neighbour shape, q block, lambda block), tuned on its own device positions."""
        k = len(ns)
        na = (C.c_int * k)(*[int(v) for v in ns])
        xa = (C.c_void_p * k)(*[C.c_void_p(p) for p in x_ptrs])
        ch = (C.c_int * (3 * k))()
        self._check(lib().mtd_walkers_autotune(self._h, na, xa, int(reps), ch))
        return [tuple(ch[3 * i:3 * i + 3]) for i in range(k)]
