"""Python binding of the engine's C ABI (include/vmc_b200.h) via ctypes.

The shared library is built in-tree (vmachine_b200/libvmc_b200.so, see build.py).
There is no fallback: if the library or a CUDA device is missing, calls raise.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvmc_b200.so")

_lib = None


class VmcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"vmc error {code}: {msg}")
        self.code = code


class Options(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int),
                ("num_walkers", ctypes.c_int), ("walkers_per_block", ctypes.c_int),
                ("refresh_interval", ctypes.c_int), ("compat", ctypes.c_int)]


class Info(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "n_particles", "n_dimensions", "n_coords", "n_elements", "p_max", "n_walkers",
        "precision", "sampling", "steps_per_walker", "burn_in", "batches", "n_iterations",
        "compat", "n_accumulators", "walkers_per_block", "refresh_interval")] + [
        ("element_kind", ctypes.c_int * 8), ("kernel_variant", ctypes.c_int), ("walkers_per_warp", ctypes.c_int),
        ("sweep_form", ctypes.c_int)]

KERNEL_RUNTIME_FLAGS, KERNEL_DOT, KERNEL_GENERAL = 0, 1, 2
SWEEP_STAGED, SWEEP_OWNER = 1, 2


class Sums(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "energy", "energy2", "kinetic", "kinetic2", "external", "external2", "interaction",
        "interaction2", "accepts", "n_samples", "n_window", "seconds", "sweep_seconds",
        "sweep_launches", "max_drift", "q99_drift")] + [
        ("status", ctypes.c_uint32)]


class Averages(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "energy", "std_error", "kinetic", "external", "interaction", "acceptance",
        "walker_std_error")]


class Block(ctypes.Structure):
    _fields_ = [("mean", ctypes.c_double), ("std_error", ctypes.c_double), ("mse_mean", ctypes.c_double),
                ("mse_std_error", ctypes.c_double), ("n_k", ctypes.c_longlong)]


class BlockingResult(ctypes.Structure):
    _fields_ = [("energy", Block), ("kinetic", Block), ("external", Block), ("interaction", Block),
                ("energy_walkers", Block), ("samples_per_walker", ctypes.c_longlong)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("n_systems", ctypes.c_int), ("n_general", ctypes.c_int), ("n_walkers", ctypes.c_longlong),
                ("precision", ctypes.c_int), ("walkers_per_block", ctypes.c_int),
                ("walkers_per_item", ctypes.c_int), ("grid", ctypes.c_int), ("tuned", ctypes.c_int),
                ("graph_captures", ctypes.c_int), ("graph_replay", ctypes.c_int), ("rounds", ctypes.c_int),
                ("seconds", ctypes.c_double), ("sweep_seconds", ctypes.c_double),
                ("walker_moves", ctypes.c_double)]


class BatchCandidate(ctypes.Structure):
    _fields_ = [("walkers_per_block", ctypes.c_int), ("walkers_per_item", ctypes.c_int),
                ("grid", ctypes.c_int), ("ns_per_walker_move", ctypes.c_double)]


EXPORTS = ["vmc_abi_version", "vmc_create", "vmc_destroy", "vmc_get_info", "vmc_last_error",
           "vmc_set_parameters", "vmc_get_parameters", "vmc_init_walkers", "vmc_get_positions",
           "vmc_sample", "vmc_run_iteration", "vmc_get_walker_energies", "vmc_eval",
           "vmc_probe_move", "vmc_replay", "vmc_set_replay", "vmc_get_status",
           "vmc_run_simulation", "vmc_stopwatch", "vmc_measure_fma_peak", "vmc_apply_sums",
           "vmc_batch_create", "vmc_batch_destroy", "vmc_batch_get_info", "vmc_batch_system",
           "vmc_batch_init_walkers", "vmc_batch_set_tile", "vmc_batch_run_iteration",
           "vmc_batch_last_sums", "vmc_batch_tuning", "vmc_block_series", "vmc_blocking",
           "vmc_format_weights", "vmc_write_weights", "vmc_read_weights", "vmc_save_state", "vmc_load_state",
           "vmc_last_blocking", "vmc_densities", "vmc_set_refresh_interval"]


def library():
    """Load libvmc_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m vmachine_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    L.vmc_abi_version.restype = ip
    L.vmc_last_error.restype = ctypes.c_char_p
    L.vmc_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(Options), ctypes.POINTER(vp)]
    L.vmc_destroy.argtypes = [vp]
    L.vmc_destroy.restype = None
    L.vmc_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.vmc_set_parameters.argtypes = [vp, vp, ip, ip]
    L.vmc_get_parameters.argtypes = [vp, vp, ip, ip]
    L.vmc_init_walkers.argtypes = [vp, vp, ctypes.c_uint64]
    L.vmc_get_positions.argtypes = [vp, vp]
    L.vmc_sample.argtypes = [vp, ip, ip, ip, ctypes.POINTER(Sums), vp, vp]
    L.vmc_run_iteration.argtypes = [vp, ip, ctypes.POINTER(Averages)]
    L.vmc_apply_sums.argtypes = [vp, ctypes.POINTER(Sums), vp, vp, ctypes.POINTER(Averages)]
    L.vmc_get_walker_energies.argtypes = [vp, vp]
    L.vmc_eval.argtypes = [vp, vp, vp, vp, vp]
    L.vmc_probe_move.argtypes = [vp, vp, vp, vp]
    L.vmc_replay.argtypes = [vp, vp, ip, vp, vp]
    L.vmc_set_replay.argtypes = [vp, vp, ip]
    L.vmc_get_status.argtypes = [vp, vp]
    L.vmc_run_simulation.argtypes = [vp, ctypes.POINTER(Averages), ip]
    L.vmc_stopwatch.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_double)]
    L.vmc_set_refresh_interval.argtypes = [vp, ip]
    L.vmc_measure_fma_peak.argtypes = [ip, ip, ctypes.POINTER(ctypes.c_double)]
    L.vmc_format_weights.argtypes = [vp, ip, ip, ip, ctypes.c_char_p, ctypes.c_longlong]
    L.vmc_write_weights.argtypes = [vp, ctypes.c_char_p, ip]
    L.vmc_read_weights.argtypes = [vp, ctypes.c_char_p]
    L.vmc_save_state.argtypes = [vp, ctypes.c_char_p]
    L.vmc_load_state.argtypes = [vp, ctypes.c_char_p]
    L.vmc_last_blocking.argtypes = [vp, ctypes.POINTER(BlockingResult)]
    L.vmc_densities.argtypes = [vp, ip, ip, ip, dp, vp, vp, vp]
    L.vmc_block_series.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(Block)]
    L.vmc_blocking.argtypes = [vp, ip, ip, ctypes.POINTER(BlockingResult)]
    L.vmc_batch_create.argtypes = [ctypes.POINTER(ctypes.c_char_p), ip, ctypes.POINTER(Options), ctypes.POINTER(vp)]
    L.vmc_batch_destroy.argtypes = [vp]
    L.vmc_batch_destroy.restype = None
    L.vmc_batch_get_info.argtypes = [vp, ctypes.POINTER(BatchInfo)]
    L.vmc_batch_system.argtypes = [vp, ip, ctypes.POINTER(vp)]
    L.vmc_batch_init_walkers.argtypes = [vp, vp]
    L.vmc_batch_set_tile.argtypes = [vp, ip, ip]
    L.vmc_batch_run_iteration.argtypes = [vp, ip, vp]
    L.vmc_batch_last_sums.argtypes = [vp, vp]
    L.vmc_batch_tuning.argtypes = [vp, vp, ip]
    for name in EXPORTS:
        if name not in ("vmc_destroy", "vmc_last_error", "vmc_batch_destroy"):
            getattr(L, name).restype = ip
    L.vmc_format_weights.restype = ctypes.c_longlong
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class Engine:
    """One walker population on one GPU, built from input.in text."""

    def __init__(self, input_in, *, device=0, precision=None, walkers=None,
                 walkers_per_block=None, refresh_interval=None, compat=None):
        L = library()
        o = Options(device, -1 if precision is None else int(precision),
                    0 if walkers is None else int(walkers),
                    0 if walkers_per_block is None else int(walkers_per_block),
                    -1 if refresh_interval is None else int(refresh_interval),
                    -1 if compat is None else int(compat))
        h = ctypes.c_void_p()
        self._check(L.vmc_create(input_in.encode(), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        info = Info()
        self._check(L.vmc_get_info(self._h, ctypes.byref(info)))
        self.info = info
        self.W, self.D, self.E, self.P = info.n_walkers, info.n_coords, info.n_elements, info.p_max

    @staticmethod
    def _check(rc):
        if rc != 0:
            raise VmcError(rc, library().vmc_last_error().decode())

    def close(self):
        if getattr(self, "_h", None):
            library().vmc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- parameters and walkers
    def set_parameters(self, theta):
        th = np.ascontiguousarray(theta, np.float64).reshape(self.E, self.P)
        self._check(library().vmc_set_parameters(self._h, _p(th), self.E, self.P))

    def parameters(self):
        th = np.zeros((self.E, self.P))
        self._check(library().vmc_get_parameters(self._h, _p(th), self.E, self.P))
        return th

    def init_walkers(self, positions=None, seed=0):
        pos = None if positions is None else np.ascontiguousarray(positions, np.float64).reshape(
            self.W, self.D)
        self._check(library().vmc_init_walkers(self._h, _p(pos), int(seed)))

    def positions(self, out=None):
        """Walker positions (W x D, FP64), into `out` when given (a C-contiguous float64
        array of that shape, e.g. a pinned host buffer)."""
        if out is None:
            out = np.zeros((self.W, self.D))
        elif out.shape != (self.W, self.D) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("positions: out must be a C-contiguous float64 array of shape (W, D)")
        self._check(library().vmc_get_positions(self._h, _p(out)))
        return out

    # --- sampling
    def sample(self, iteration, steps, burn_in):
        s = Sums()
        g = np.zeros((self.E, self.P))
        ge = np.zeros((self.E, self.P))
        self._check(library().vmc_sample(self._h, iteration, steps, burn_in, ctypes.byref(s),
                                         _p(g), _p(ge)))
        return s, g, ge

    def apply_sums(self, sums, grad_sum, egrad_sum):
        """Averages + optimiser step from (possibly all-reduced) totals."""
        a = Averages()
        g = np.ascontiguousarray(grad_sum, np.float64).reshape(self.E, self.P)
        ge = np.ascontiguousarray(egrad_sum, np.float64).reshape(self.E, self.P)
        self._check(library().vmc_apply_sums(self._h, ctypes.byref(sums), _p(g), _p(ge),
                                             ctypes.byref(a)))
        return a

    def run_iteration(self, iteration):
        a = Averages()
        self._check(library().vmc_run_iteration(self._h, iteration, ctypes.byref(a)))
        return a

    def run_simulation(self):
        """System::runSimulation: the per-iteration averages of the iterations run."""
        n = self.info.n_iterations
        hist = (Averages * n)()
        rc = library().vmc_run_simulation(self._h, hist, n)
        if rc < 0:
            self._check(rc)
        return list(hist)[:rc]

    def last_blocking(self):
        r = BlockingResult()
        self._check(library().vmc_last_blocking(self._h, ctypes.byref(r)))
        return r

    def densities(self, steps, burn_in=0, bins=1000, max_radius=5.0, radial=True, spatial=False, two_body=False):
        """Electron-density counts over `steps` moves per walker (vmc_densities)."""
        r = np.zeros(bins, np.uint64) if radial else None
        sp = np.zeros((bins, bins), np.uint64) if spatial else None
        tb = np.zeros((bins, bins), np.uint64) if two_body else None
        self._check(library().vmc_densities(self._h, int(steps), int(burn_in), int(bins), float(max_radius),
                                            _p(r), _p(sp), _p(tb)))
        return r, sp, tb

    def walker_energies(self):
        out = np.zeros(self.W)
        self._check(library().vmc_get_walker_energies(self._h, _p(out)))
        return out

    # --- oracle entries
    def eval(self):
        g = np.zeros((self.W, self.E, self.D))
        lap = np.zeros((self.W, self.E))
        pg = np.zeros((self.W, self.E, self.P))
        en = np.zeros((self.W, 3))
        self._check(library().vmc_eval(self._h, _p(g), _p(lap), _p(pg), _p(en)))
        return g, lap, pg, en

    def probe_move(self, k, xnew):
        k = np.ascontiguousarray(k, np.int32).reshape(self.W)
        x = np.ascontiguousarray(xnew, np.float64).reshape(self.W)
        r = np.zeros((self.W, self.E))
        self._check(library().vmc_probe_move(self._h, _p(k), _p(x), _p(r)))
        return r

    def set_replay(self, stream):
        """stream: (W, length, 3) consumed by later sample/run_iteration calls; None clears."""
        if stream is None:
            self._check(library().vmc_set_replay(self._h, None, 0))
            return
        st = np.ascontiguousarray(stream, np.float64)
        self._keep_replay = st
        self._check(library().vmc_set_replay(self._h, _p(st), st.shape[1]))

    def replay(self, stream, steps=None):
        """Record `steps` moves per walker; stream (W, steps, 3) or None for Philox."""
        st = None if stream is None else np.ascontiguousarray(stream, np.float64)
        steps = st.shape[1] if st is not None else int(steps)
        acc = np.zeros((self.W, steps), np.uint8)
        en = np.zeros((self.W, steps, 3))
        self._check(library().vmc_replay(self._h, _p(st), steps, _p(acc), _p(en)))
        return acc, en

    def stopwatch_start(self):
        self._check(library().vmc_stopwatch(self._h, 0, None))

    def stopwatch_stop(self):
        ms = ctypes.c_double()
        self._check(library().vmc_stopwatch(self._h, 1, ctypes.byref(ms)))
        return ms.value

    def refresh_interval(self):
        """Current FP64 rebuild cadence in steps (autotuned for `refreshInterval: auto`)."""
        info = Info()
        self._check(library().vmc_get_info(self._h, ctypes.byref(info)))
        return info.refresh_interval

    def set_refresh_interval(self, steps):
        """Set the FP64 rebuild cadence (mixed precision; vmc_set_refresh_interval)."""
        self._check(library().vmc_set_refresh_interval(self._h, int(steps)))

    # --- checkpoints
    def write_weights(self, path, digits=0):
        """Parameter file in the reference's format (digits <= 0: its 6 digits)."""
        self._check(library().vmc_write_weights(self._h, os.fspath(path).encode(), int(digits)))

    def read_weights(self, path):
        self._check(library().vmc_read_weights(self._h, os.fspath(path).encode()))

    def save_state(self, path):
        """Walkers, parameters and optimiser state for an exact restart."""
        self._check(library().vmc_save_state(self._h, os.fspath(path).encode()))

    def load_state(self, path):
        self._check(library().vmc_load_state(self._h, os.fspath(path).encode()))

    def blocking(self, steps, burn_in=0):
        """Sample `steps` moves per walker with the current parameters and block the
        energy series on the device (vmc_blocking)."""
        r = BlockingResult()
        self._check(library().vmc_blocking(self._h, int(steps), int(burn_in), ctypes.byref(r)))
        return r

    def status(self):
        out = np.zeros(self.W, np.uint32)
        self._check(library().vmc_get_status(self._h, _p(out)))
        return out


def block_series(x):
    """The reference's Blocker on a host series (vmc_block_series)."""
    a = np.ascontiguousarray(x, np.float64)
    b = Block()
    Engine._check(library().vmc_block_series(_p(a), len(a), ctypes.byref(b)))
    return b


def measure_fma_peak(device=0, precision=1):
    """Device FMA throughput in TFLOP/s (precision 1: FP32, 0: FP64)."""
    t = ctypes.c_double()
    Engine._check(library().vmc_measure_fma_peak(device, precision, ctypes.byref(t)))
    return t.value


class _Member(Engine):
    """A system's engine inside a Batch (owned by the batch: closing it is a no-op)."""

    def __init__(self, handle):
        self._h = handle
        self._owned = False
        info = Info()
        self._check(library().vmc_get_info(self._h, ctypes.byref(info)))
        self.info = info
        self.W, self.D, self.E, self.P = info.n_walkers, info.n_coords, info.n_elements, info.p_max

    def close(self):
        self._h = None


class Batch:
    """Many systems (input.in texts), each with its own walkers and parameters,
    iterated together by the persistent multi-system kernel and a captured graph."""

    def __init__(self, texts, *, device=0, precision=None, refresh_interval=None, compat=None):
        L = library()
        arr = (ctypes.c_char_p * len(texts))(*[t.encode() for t in texts])
        o = Options(device, -1 if precision is None else int(precision), 0, 0,
                    -1 if refresh_interval is None else int(refresh_interval),
                    -1 if compat is None else int(compat))
        h = ctypes.c_void_p()
        Engine._check(L.vmc_batch_create(arr, len(texts), ctypes.byref(o), ctypes.byref(h)))
        self._h = h
        self.n = len(texts)
        self.systems = []
        for s in range(self.n):
            eh = ctypes.c_void_p()
            Engine._check(L.vmc_batch_system(self._h, s, ctypes.byref(eh)))
            self.systems.append(_Member(eh))

    def close(self):
        if getattr(self, "_h", None):
            for m in self.systems:
                m.close()
            library().vmc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def info(self):
        i = BatchInfo()
        Engine._check(library().vmc_batch_get_info(self._h, ctypes.byref(i)))
        return i

    def init_walkers(self, seeds=None):
        sd = None if seeds is None else np.ascontiguousarray(seeds, np.uint64)
        Engine._check(library().vmc_batch_init_walkers(self._h, _p(sd)))

    def set_tile(self, walkers_per_block, walkers_per_item):
        Engine._check(library().vmc_batch_set_tile(self._h, int(walkers_per_block), int(walkers_per_item)))

    def run_iteration(self, iteration):
        out = (Averages * self.n)()
        Engine._check(library().vmc_batch_run_iteration(self._h, int(iteration), out))
        return list(out)

    def last_sums(self):
        out = (Sums * self.n)()
        Engine._check(library().vmc_batch_last_sums(self._h, out))
        return list(out)

    def tuning(self):
        n = library().vmc_batch_tuning(self._h, None, 0)
        out = (BatchCandidate * max(n, 1))()
        library().vmc_batch_tuning(self._h, out, n)
        return [(c.walkers_per_block, c.walkers_per_item, c.grid, c.ns_per_walker_move) for c in out[:n]]
