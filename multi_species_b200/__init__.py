"""B200 (sm_100a) implementation of the FARRSIGHT per-step hot path.

Python mirror of the reference's operator interfaces over the C ABI of
``libfs_b200.so`` (declared in ``include/fs_b200.h``):

* ``E_MQ_DirectSum_B200`` / ``E_MQ_Treecode_B200`` -- drop-ins for the
  reference's ``ElectricField`` subclasses (``inc/FieldStructure.hpp:87-198``):
  ``field(es, targets, nt, sources, q_ws, ns)`` fills ``es`` exactly like
  ``ElectricField::operator()``; ``field.evaluate(targets, sources, q_ws)``
  returns a new array.
* ``Simulation`` -- the device-resident ``AMRSimulation``
  (``inc/AMRSimulation.hpp:63-131``): ``step()``, ``run()``, ``state()``.
* ``mesh(...)`` -- the host panel mesh of ``create_prerefined_mesh``.

There is no CPU fallback: if the CUDA library is missing, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfs_b200.so")

FS_FIELD_DIRECT64 = 0
FS_FIELD_DIRECT32C = 1
FS_FIELD_TREECODE64 = 2
FS_FIELD_TREECODE32C = 3
FS_FIELD_DIRECT64_OPEN = 4
PANEL_INTS = 18

STATUS = {0: "FS_OK", 1: "FS_ERR_ARG", 2: "FS_ERR_CUDA", 3: "FS_ERR_NOMEM", 4: "FS_ERR_WALK",
          5: "FS_ERR_SHIFT", 6: "FS_ERR_TIMEOUT", 7: "FS_ERR_STATE", 8: "FS_ERR_UNSUPPORTED",
          9: "FS_ERR_TREE"}

# Every symbol include/fs_b200.h declares (checked by the tests).
EXPORTS = ["fs_field_create", "fs_field_destroy", "fs_field_eval", "fs_field_eval_device", "fs_field_eval_noalloc",
           "fs_sim_create", "fs_sim_destroy", "fs_sim_step", "fs_sim_remesh", "fs_sim_num_points", "fs_sim_export",
           "fs_sim_import_xp", "fs_sim_iter", "fs_sim_pair_count", "fs_sim_work", "fs_sim_step_times", "fs_mesh_sizes",
           "fs_mesh_fill", "fs_profile_enable", "fs_profile_read", "fs_profile_reset", "fs_last_error",
           "fs_version", "fs_kernel_launches", "fs_batch_create", "fs_batch_destroy", "fs_batch_add",
           "fs_batch_remove", "fs_batch_step", "fs_batch_export", "fs_batch_info", "fs_batch_step_times",
           "fs_batch_work", "fs_batch_stats", "fs_batch_band_pairs", "fs_batch_set_tuning", "fs_batch_set_graphs", "fs_pool_create",
           "fs_pool_destroy", "fs_pool_submit", "fs_pool_cancel", "fs_pool_poll", "fs_pool_wait", "fs_pool_result",
           "fs_pool_release", "fs_pool_step_times", "fs_pool_stats", "fs_pool_estimate_bytes", "fs_sim_set_output",
           "fs_sim_flush_output", "fs_sim_restart", "fs_initial_f0", "fs_debug_set_wait_limits"]


class FsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class FieldParams(C.Structure):
    _fields_ = [("L", C.c_double), ("epsilon", C.c_double), ("kind", C.c_int), ("mac", C.c_double),
                ("degree", C.c_int), ("max_source", C.c_int), ("max_target", C.c_int), ("device", C.c_int)]


class SpeciesParams(C.Structure):
    _fields_ = [("q", C.c_double), ("m", C.c_double), ("initial_height", C.c_int), ("p_height", C.c_int),
                ("pmin", C.c_double), ("pmax", C.c_double), ("ics_type", C.c_int), ("pth", C.c_double),
                ("pstr", C.c_double), ("amp", C.c_double), ("normalized_wavenumber", C.c_double),
                ("do_adaptively_refine", C.c_int), ("max_height", C.c_int), ("n_amr_eps", C.c_int),
                ("amr_eps", C.c_double * 5), ("mu", C.c_double), ("wave_beta", C.c_double)]


class SimParams(C.Structure):
    _fields_ = [("xmin", C.c_double), ("xmax", C.c_double), ("quadrature", C.c_int), ("dt", C.c_double),
                ("remesh_period", C.c_int), ("greens_epsilon", C.c_double), ("field_kind", C.c_int),
                ("mac", C.c_double), ("degree", C.c_int), ("max_source", C.c_int), ("num_species", C.c_int),
                ("species", SpeciesParams * 8), ("device", C.c_int), ("use_external_field", C.c_int),
                ("external_type", C.c_int), ("external_Am", C.c_double), ("external_k", C.c_double),
                ("external_omega", C.c_double), ("relativistic_push", C.c_int)]


class PoolParams(C.Structure):
    _fields_ = [("device", C.c_int), ("hbm_budget_bytes", C.c_double), ("max_live", C.c_int),
                ("targets_per_thread", C.c_int), ("tiles_per_item", C.c_int)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("steps_done", C.c_int), ("nsteps", C.c_int), ("npoints", C.c_int),
                ("pairs", C.c_double), ("step_ms_p50", C.c_double), ("step_ms_p99", C.c_double),
                ("queue_ms", C.c_double), ("total_ms", C.c_double), ("error", C.c_char * 256)]


class PoolStats(C.Structure):
    _fields_ = [(n, C.c_longlong) for n in ("submitted", "admitted", "completed", "failed", "cancelled", "queued",
                                           "live", "iterations")] + \
               [(n, C.c_double) for n in ("hbm_in_use_bytes", "pairs", "busy_ms", "step_ms_p50", "step_ms_p99")]


REQUEST_STATES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}

_lib = None
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def lib():
    """Load libfs_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m multi_species_b200.build` "
                              "(the CUDA library is required; there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        st = C.c_int
        L.fs_field_create.argtypes = [C.POINTER(FieldParams), C.POINTER(C.c_void_p)]
        L.fs_field_destroy.argtypes = [C.c_void_p]
        L.fs_field_eval.argtypes = [C.c_void_p, _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        L.fs_field_eval_device.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                           C.c_int, C.c_void_p]
        L.fs_field_eval_noalloc.argtypes = [C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                            C.c_void_p]
        L.fs_debug_set_wait_limits.argtypes = [C.c_int, C.c_longlong, C.c_int]
        L.fs_sim_create.argtypes = [C.POINTER(SimParams), C.POINTER(C.c_void_p)]
        L.fs_sim_destroy.argtypes = [C.c_void_p]
        L.fs_sim_step.argtypes = [C.c_void_p, C.c_int]
        L.fs_sim_remesh.argtypes = [C.c_void_p]
        L.fs_sim_num_points.argtypes = [C.c_void_p, C.c_int, _ip]
        L.fs_sim_export.argtypes = [C.c_void_p, _dp, _dp, _dp, _dp, _dp]
        L.fs_sim_import_xp.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.fs_sim_iter.argtypes = [C.c_void_p, _ip, _dp]
        L.fs_sim_pair_count.argtypes = [C.c_void_p, _dp]
        L.fs_sim_step_times.argtypes = [C.c_void_p, _dp, C.c_int, _ip]
        L.fs_sim_work.argtypes = [C.c_void_p, _dp, _dp]
        L.fs_sim_set_output.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int, C.c_int]
        L.fs_sim_set_output.restype = st
        L.fs_sim_flush_output.argtypes = [C.c_void_p]
        L.fs_sim_restart.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_char_p), C.c_int]
        L.fs_sim_restart.restype = st
        L.fs_sim_flush_output.restype = st
        L.fs_initial_f0.argtypes = [C.POINTER(SimParams), C.c_int, C.c_int, _dp, _dp, _dp]
        L.fs_initial_f0.restype = st
        L.fs_profile_enable.argtypes = [C.c_int]
        L.fs_profile_read.argtypes = [C.c_char_p, C.POINTER(C.c_longlong), _dp, _dp]
        L.fs_profile_reset.argtypes = []
        L.fs_mesh_sizes.argtypes = [C.c_int, C.c_int, _ip, _ip, _ip]
        L.fs_mesh_fill.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_int, _dp, _dp, _ip, _ip, _dp]
        L.fs_batch_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        L.fs_batch_destroy.argtypes = [C.c_void_p]
        L.fs_batch_add.argtypes = [C.c_void_p, C.POINTER(SimParams), _ip]
        L.fs_batch_remove.argtypes = [C.c_void_p, C.c_int]
        L.fs_batch_step.argtypes = [C.c_void_p, C.c_int]
        L.fs_batch_export.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp, _dp, _dp]
        L.fs_batch_info.argtypes = [C.c_void_p, C.c_int, _ip, _ip, _dp, _dp]
        L.fs_batch_step_times.argtypes = [C.c_void_p, _dp, C.c_int, _ip]
        L.fs_batch_work.argtypes = [C.c_void_p, _dp]
        L.fs_batch_stats.argtypes = [C.c_void_p, _ip, _ip, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        L.fs_batch_band_pairs.argtypes = [C.c_void_p, _dp, _dp]
        L.fs_batch_set_graphs.argtypes = [C.c_void_p, C.c_int]
        L.fs_batch_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _llp = C.POINTER(C.c_longlong)
        L.fs_pool_create.argtypes = [C.POINTER(PoolParams), C.POINTER(C.c_void_p)]
        L.fs_pool_destroy.argtypes = [C.c_void_p]
        L.fs_pool_submit.argtypes = [C.c_void_p, C.POINTER(SimParams), C.c_int, _llp]
        L.fs_pool_cancel.argtypes = [C.c_void_p, C.c_longlong]
        L.fs_pool_poll.argtypes = [C.c_void_p, C.c_longlong, C.POINTER(RequestInfo)]
        L.fs_pool_wait.argtypes = [C.c_void_p, C.c_longlong, C.c_double, _ip]
        L.fs_pool_result.argtypes = [C.c_void_p, C.c_longlong, _dp, _dp, _dp, _dp, _dp]
        L.fs_pool_release.argtypes = [C.c_void_p, C.c_longlong]
        L.fs_pool_step_times.argtypes = [C.c_void_p, C.c_longlong, _dp, C.c_int, _ip]
        L.fs_pool_stats.argtypes = [C.c_void_p, C.POINTER(PoolStats)]
        L.fs_pool_estimate_bytes.argtypes = [C.POINTER(SimParams), _dp]
        for n in ("fs_pool_create", "fs_pool_destroy", "fs_pool_submit", "fs_pool_cancel", "fs_pool_poll",
                  "fs_pool_wait", "fs_pool_result", "fs_pool_release", "fs_pool_step_times", "fs_pool_stats",
                  "fs_pool_estimate_bytes"):
            getattr(L, n).restype = st
        for n in ("fs_batch_create", "fs_batch_destroy", "fs_batch_add", "fs_batch_remove", "fs_batch_step",
                  "fs_batch_export", "fs_batch_info", "fs_batch_step_times", "fs_batch_work", "fs_batch_stats",
                  "fs_batch_band_pairs", "fs_batch_set_tuning", "fs_batch_set_graphs"):
            getattr(L, n).restype = st
        for n in ("fs_field_create", "fs_field_destroy", "fs_field_eval", "fs_field_eval_device",
                  "fs_field_eval_noalloc", "fs_sim_create",
                  "fs_sim_destroy", "fs_sim_step", "fs_sim_remesh", "fs_sim_num_points", "fs_sim_export", "fs_sim_import_xp",
                  "fs_sim_iter", "fs_sim_pair_count", "fs_sim_work", "fs_sim_step_times", "fs_mesh_sizes",
                  "fs_mesh_fill",
                  "fs_profile_enable", "fs_profile_read", "fs_profile_reset"):
            getattr(L, n).restype = st
        L.fs_last_error.restype = C.c_char_p
        L.fs_version.restype = C.c_int
        L.fs_kernel_launches.restype = C.c_longlong
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise FsError(rc, lib().fs_last_error().decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def kernel_launches() -> int:
    return int(lib().fs_kernel_launches())


def profile_enable(on: bool = True) -> None:
    _check(lib().fs_profile_enable(1 if on else 0))


def profile_reset() -> None:
    _check(lib().fs_profile_reset())


def profile_read(kernel: str):
    """(launches, total device ms, total work) of the named kernel since the last reset."""
    n, ms, w = C.c_longlong(), C.c_double(), C.c_double()
    _check(lib().fs_profile_read(kernel.encode(), C.byref(n), C.byref(ms), C.byref(w)))
    return n.value, ms.value, w.value


# --------------------------------------------------------------------- field
class _Field:
    kind = FS_FIELD_DIRECT64

    def __init__(self, L: float, epsilon: float, kind: int, mac=-1.0, degree=-1, max_source=2000,
                 max_target=2000, device=0):
        self.L, self.epsilon = float(L), float(epsilon)
        p = FieldParams(float(L), float(epsilon), int(kind), float(mac), int(degree), int(max_source),
                        int(max_target), int(device))
        h = C.c_void_p()
        _check(lib().fs_field_create(C.byref(p), C.byref(h)))
        self._h = h

    def __call__(self, es, targets, nt, sources, q_ws, ns):
        """ElectricField::operator()(es, targets, nt, sources, q_ws, ns): fills es in place."""
        for a in (es, targets, sources, q_ws):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TypeError("arrays must be C-contiguous float64 numpy arrays")
        _check(lib().fs_field_eval(self._h, _ptr(es), _ptr(targets), int(nt), _ptr(sources), _ptr(q_ws), int(ns)))

    def evaluate(self, targets, sources, q_ws):
        t, s, q = _f64(targets), _f64(sources), _f64(q_ws)
        es = np.zeros(len(t))
        self(es, t, len(t), s, q, len(s))
        return es

    def evaluate_device(self, d_es, d_targets, nt, d_sources, d_q, ns, stream=None):
        """Device-pointer variant (integers: CUDA device addresses)."""
        _check(lib().fs_field_eval_device(self._h, d_es, d_targets, nt, d_sources, d_q, ns, stream))

    def close(self):
        if getattr(self, "_h", None):
            lib().fs_field_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class E_MQ_DirectSum_B200(_Field):
    """E_MQ_DirectSum(L, epsilon) (src/FieldStructure.cpp:102-164) on the GPU.

    precision="fp64": the reference arithmetic, bit-identical results.
    precision="fp32c": FP32 pair kernel with compensation + FP64 background.
    """

    def __init__(self, L, epsilon, precision="fp64", device=0):
        kind = {"fp64": FS_FIELD_DIRECT64, "fp32c": FS_FIELD_DIRECT32C}[precision]
        super().__init__(L, epsilon, kind, device=device)


class E_MQ_DirectSum_openbcs_B200(_Field):
    """E_MQ_DirectSum_openbcs(epsilon) (src/FieldStructure.cpp:166-192) on the
    GPU: open boundaries, FP64, bit-identical to the reference."""

    def __init__(self, epsilon, device=0):
        super().__init__(1.0, epsilon, FS_FIELD_DIRECT64_OPEN, device=device)


class E_MQ_Treecode_B200(_Field):
    """E_MQ_Treecode(L, epsilon, mac, degree, max_source, max_target, verbosity)
    (src/FieldStructure.cpp:210-503) on the GPU.  Like the reference it ignores
    the targets and evaluates at the sources."""

    def __init__(self, L, epsilon, mac, degree, max_source, max_target=2000, verbosity=0, precision="fp64",
                 device=0):
        kind = {"fp64": FS_FIELD_TREECODE64, "fp32c": FS_FIELD_TREECODE32C}[precision]
        super().__init__(L, epsilon, kind, mac, degree, max_source, max_target, device=device)


def debug_set_wait_limits(device: int = 0, mbar_polls: int = -1, walk_panels: int = 0) -> None:
    """Test hook: bounds of the device waits on `device` (fs_debug_set_wait_limits).
    mbar_polls: polls of a pair kernel's tile wait before FS_ERR_TIMEOUT (0 = at
    once, < 0 = default); walk_panels: panels a remesh walk may visit before
    FS_ERR_WALK (<= 0 = default).  Call with no limits to restore the defaults."""
    _check(lib().fs_debug_set_wait_limits(int(device), int(mbar_polls), int(walk_panels)))


def field_eval_noalloc(L, epsilon, d_es, d_x, d_q_ws, n, stream=None):
    """fs_field_eval_noalloc: self-field of n <= 32768 points on device pointers
    (integers), with all scratch in the library's static device array -- for
    callers that cannot allocate device memory at call time."""
    _check(lib().fs_field_eval_noalloc(float(L), float(epsilon), d_es, d_x, d_q_ws, int(n), stream))


# --------------------------------------------------------------------- simulation
FIELD_KINDS = {"direct64": FS_FIELD_DIRECT64, "direct32c": FS_FIELD_DIRECT32C, "treecode64": FS_FIELD_TREECODE64,
               "treecode32c": FS_FIELD_TREECODE32C, "direct64_open": FS_FIELD_DIRECT64_OPEN}


def sim_params(deck: dict, field_backend: str | None = None, device: int = 0) -> SimParams:
    """deck.json keys (src/simulation_files/AMRSimulation_load.cpp:14-270) -> SimParams.
    `field_backend` (or the deck's optional "field_backend" key) picks the solver;
    the default follows use_treecode like make_field_return_ptr."""
    if int(deck.get("bcs", 0)) != 0:
        raise FsError(8, "only periodic boundary conditions (bcs=0) are implemented")
    P = SimParams()
    P.xmin, P.xmax = float(deck.get("xmin", 0.0)), float(deck.get("xmax", 0.0))
    P.quadrature = int(deck.get("quadrature", 1))
    P.dt = float(deck.get("dt", 0.5))
    P.remesh_period = int(deck.get("remesh_period", 1))
    P.greens_epsilon = float(deck.get("greens_epsilon", 0.2))
    backend = field_backend or deck.get("field_backend")
    if backend is None:
        backend = "treecode64" if int(deck.get("use_treecode", 0)) > 0 else "direct64"
    P.field_kind = FIELD_KINDS[backend]
    P.mac = float(deck.get("mac", -1.0))
    P.degree = int(deck.get("degree", -1))
    P.max_source = int(deck.get("max_source", 2000))
    sl = deck["species_list"]
    if not 1 <= len(sl) <= 8:
        raise FsError(1, "species_list must hold 1..8 species")
    P.num_species = len(sl)
    for i, sp in enumerate(sl):
        S = P.species[i]
        S.q, S.m = float(sp.get("q", -1.0)), float(sp.get("m", 1.0))
        S.initial_height, S.p_height = int(sp.get("initial_height", 6)), int(sp.get("p_height", 0))
        S.pmin, S.pmax = float(sp.get("pmin", -1.0)), float(sp.get("pmax", 1.0))
        S.ics_type = int(sp.get("ics_type", 1))
        S.pth, S.pstr, S.amp = float(sp.get("pth", 1.0)), float(sp.get("pstr", 0.0)), float(sp.get("amp", 0.0))
        S.normalized_wavenumber = float(sp.get("normalized_wavenumber", 1.0))
        # adaptive refinement: off unless do_adaptively_refine and amr_epsilons
        # are given (AMRSimulation_load.cpp:246-258)
        eps = sp.get("amr_epsilons")
        S.do_adaptively_refine = 1 if (bool(sp.get("do_adaptively_refine", False)) and eps is not None) else 0
        S.max_height = int(sp.get("max_height", sp.get("initial_height", 6)))
        eps = [float(e) for e in (eps or [])][:5]
        S.n_amr_eps = len(eps)
        for k, e in enumerate(eps):
            S.amr_eps[k] = e
        # relativistic initial conditions: the reference's defaults when the
        # keys are absent (AMRSimulation_load.cpp:169-207)
        S.mu, S.wave_beta = float(sp.get("mu", 1.0)), float(sp.get("wave_beta", 0.8))
    P.device = int(device)
    # opt-in relativistic position push; the reference's own "relativistic"
    # key has no effect on its RK4 step and is ignored here too
    P.relativistic_push = 1 if int(deck.get("relativistic_push", 0)) > 0 else 0
    # "external_field" block (AMRSimulation_load.cpp:98-136); absent = off
    ext = deck.get("external_field") or {}
    if int(ext.get("use_external_field", 0)) > 0:
        P.use_external_field = 1
        P.external_type = int(ext.get("external_type", 0))
        P.external_Am, P.external_k, P.external_omega = float(ext["Am"]), float(ext["k"]), float(ext["omega"])
    return P


class Simulation:
    """Device-resident AMRSimulation (inc/AMRSimulation.hpp:63-131)."""

    def __init__(self, deck: dict, field_backend: str | None = None, device: int = 0):
        self.deck = deck
        self._p = sim_params(deck, field_backend, device)
        h = C.c_void_p()
        _check(lib().fs_sim_create(C.byref(self._p), C.byref(h)))
        self._h = h
        n = C.c_int()
        _check(lib().fs_sim_num_points(self._h, -1, C.byref(n)))
        self.n = n.value
        self.species_points = []
        for s in range(self._p.num_species):
            _check(lib().fs_sim_num_points(self._h, s, C.byref(n)))
            self.species_points.append(n.value)
        self.num_steps = int(deck.get("num_steps", 10))

    def set_output(self, sim_dir: str, diag_period: int | None = None,
                   diag_phase_space_period: int | None = None) -> None:
        """Write the reference's diagnostic files (xs/ps/fs, leaf_point_inds,
        full_tree, reduce_xs/reduced_es) under sim_dir/simulation_output/,
        species directories named by the deck; periods default to the deck's
        diag_period / diag_phase_space_period (AMRSimulation_load.cpp:38-39)."""
        dp = int(diag_period if diag_period is not None else self.deck.get("diag_period", 1))
        pp = int(diag_phase_space_period if diag_phase_space_period is not None
                 else self.deck.get("diag_phase_space_period", 1))
        names = [str(sp.get("name", f"species{i}")).encode() for i, sp in enumerate(self.deck["species_list"])]
        arr = (C.c_char_p * len(names))(*names)
        _check(lib().fs_sim_set_output(self._h, str(sim_dir).encode(), arr, dp, pp))

    def flush_output(self) -> None:
        _check(lib().fs_sim_flush_output(self._h))

    def restart(self, sim_dir: str, iteration: int) -> None:
        """Load the dump of `iteration` under sim_dir/simulation_output/ (the
        reference's restart): the state, the panel trees, t = iteration * dt,
        and the reduced-grid field on the loaded state."""
        names = [str(sp.get("name", f"species{i}")).encode() for i, sp in enumerate(self.deck["species_list"])]
        arr = (C.c_char_p * len(names))(*names)
        _check(lib().fs_sim_restart(self._h, str(sim_dir).encode(), arr, int(iteration)))

    def step(self, n: int = 1) -> None:
        """n x AMRSimulation::step (AMRSimulation_step.cpp:5-99)."""
        _check(lib().fs_sim_step(self._h, int(n)))

    def remesh(self) -> None:
        """AMRSimulation::remesh (AMRSimulation_remesh.cpp:3-48) on the current state."""
        _check(lib().fs_sim_remesh(self._h))

    def run(self) -> None:
        """AMRSimulation::run (AMRSimulation_run.cpp:3-10)."""
        it, _ = self.iteration()
        if it < self.num_steps:
            self.step(self.num_steps - it)

    def iteration(self):
        i, t = C.c_int(), C.c_double()
        _check(lib().fs_sim_iter(self._h, C.byref(i), C.byref(t)))
        return i.value, t.value

    def work(self):
        """(direct-equivalent pairs, kernel-level evaluations) so far."""
        a, b = C.c_double(), C.c_double()
        _check(lib().fs_sim_work(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def step_times(self):
        """Device ms of each step of the last step() call (CUDA events on the sim stream)."""
        buf = np.zeros(4096)
        n = C.c_int()
        _check(lib().fs_sim_step_times(self._h, _ptr(buf), len(buf), C.byref(n)))
        return buf[: n.value].copy()

    def pair_count(self) -> float:
        v = C.c_double()
        _check(lib().fs_sim_pair_count(self._h, C.byref(v)))
        return v.value

    def state(self) -> dict:
        n = C.c_int()
        _check(lib().fs_sim_num_points(self._h, -1, C.byref(n)))  # adaptive meshes change it at remesh
        self.n = n.value
        self.species_points = []
        for s in range(self._p.num_species):
            _check(lib().fs_sim_num_points(self._h, s, C.byref(n)))
            self.species_points.append(n.value)
        a = {k: np.zeros(self.n) for k in ("xs", "ps", "fs", "q_ws", "es")}
        _check(lib().fs_sim_export(self._h, *(_ptr(a[k]) for k in ("xs", "ps", "fs", "q_ws", "es"))))
        return a

    def import_xp(self, xs=None, ps=None, es=None) -> None:
        arrs = [None if v is None else _f64(v) for v in (xs, ps, es)]
        for v in arrs:
            if v is not None and len(v) != self.n:
                raise ValueError("length mismatch")
        _check(lib().fs_sim_import_xp(self._h, *(_ptr(v) for v in arrs)))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fs_sim_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------- batch
class Batch:
    """Many independent simulations stepped together on one GPU (fs_batch_*).

    Members are decks as for Simulation; their FP32 pair work shares one
    persistent launch per field evaluation, and steps are replayed from CUDA
    graphs once captured.  No counterpart in the reference (one deck per run).
    """

    def __init__(self, device: int = 0, graphs: bool = True, tuning=None):
        h = C.c_void_p()
        _check(lib().fs_batch_create(int(device), C.byref(h)))
        self._h = h
        self.device = int(device)
        self.members = {}
        if not graphs:
            _check(lib().fs_batch_set_graphs(self._h, 0))
        if tuning is not None:
            self.set_tuning(*tuning)

    def set_tuning(self, targets_per_thread: int, tiles_per_item: int) -> None:
        """Fix the item shape (skips the autotuner)."""
        _check(lib().fs_batch_set_tuning(self._h, int(targets_per_thread), int(tiles_per_item)))

    def add(self, deck: dict, field_backend: str | None = None) -> int:
        p = sim_params(deck, field_backend, self.device)
        i = C.c_int()
        _check(lib().fs_batch_add(self._h, C.byref(p), C.byref(i)))
        self.members[i.value] = deck
        return i.value

    def remove(self, sim_id: int) -> None:
        _check(lib().fs_batch_remove(self._h, int(sim_id)))
        self.members.pop(sim_id, None)

    def step(self, n: int = 1) -> None:
        _check(lib().fs_batch_step(self._h, int(n)))

    def info(self, sim_id: int) -> dict:
        n, it, t, w = C.c_int(), C.c_int(), C.c_double(), C.c_double()
        _check(lib().fs_batch_info(self._h, int(sim_id), C.byref(n), C.byref(it), C.byref(t), C.byref(w)))
        return {"n": n.value, "iter": it.value, "t": t.value, "pairs": w.value}

    def state(self, sim_id: int) -> dict:
        n = self.info(sim_id)["n"]
        a = {k: np.zeros(n) for k in ("xs", "ps", "fs", "q_ws", "es")}
        _check(lib().fs_batch_export(self._h, int(sim_id), *(_ptr(a[k]) for k in ("xs", "ps", "fs", "q_ws", "es"))))
        return a

    def step_times(self):
        buf = np.zeros(4096)
        n = C.c_int()
        _check(lib().fs_batch_step_times(self._h, _ptr(buf), len(buf), C.byref(n)))
        return buf[: n.value].copy()

    def pair_count(self) -> float:
        v = C.c_double()
        _check(lib().fs_batch_work(self._h, C.byref(v)))
        return v.value

    def stats(self) -> dict:
        r, t, g, pl = C.c_int(), C.c_int(), C.c_longlong(), C.c_longlong()
        _check(lib().fs_batch_stats(self._h, C.byref(r), C.byref(t), C.byref(g), C.byref(pl)))
        return {"targets_per_thread": r.value, "tiles_per_item": t.value, "graph_steps": g.value,
                "plain_steps": pl.value}

    def band_pairs(self) -> tuple:
        """(band pairs, all pairs) of the FP32c members' last field evaluation:
        the band pairs (|d| <= 16 eps) are the ones evaluated in FP64."""
        b, a = C.c_double(), C.c_double()
        _check(lib().fs_batch_band_pairs(self._h, C.byref(b), C.byref(a)))
        return b.value, a.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------- serving
def initial_f0(deck: dict, species: int, x, p) -> np.ndarray:
    """f0 of species `species` of `deck` at the points (x, p): the
    distribution make_f0_return_ptr builds (AMRSimulation_load.cpp:139-225).
    Host code only; needs no device."""
    P = sim_params(deck)
    x = np.ascontiguousarray(x, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    if x.shape != p.shape:
        raise FsError(1, "x and p differ in shape")
    f = np.empty_like(x)
    _check(lib().fs_initial_f0(C.byref(P), int(species), int(x.size), _ptr(x), _ptr(p), _ptr(f)))
    return f


def estimate_bytes(deck: dict, field_backend: str | None = None) -> float:
    """Device bytes a Pool reserves for this deck (host-only computation)."""
    p = sim_params(deck, field_backend)
    v = C.c_double()
    _check(lib().fs_pool_estimate_bytes(C.byref(p), C.byref(v)))
    return v.value


class Pool:
    """Request loop serving many simulations on one GPU (fs_pool_*).

    submit() queues a (deck, steps) request and returns its id at once; a
    device-owner thread in the library admits requests in arrival order under
    the HBM budget and slot count, steps all live requests together (their pair
    work shares one launch per field evaluation) and retires finished ones.
    Thread-safe.  No counterpart in the reference.
    """

    def __init__(self, device: int = 0, hbm_budget: float = 150e9, max_live: int = 64, tuning=None):
        tpt, tpi = tuning if tuning is not None else (0, 0)
        p = PoolParams(int(device), float(hbm_budget), int(max_live), int(tpt), int(tpi))
        h = C.c_void_p()
        _check(lib().fs_pool_create(C.byref(p), C.byref(h)))
        self._h = h
        self.device = int(device)

    def submit(self, deck: dict, steps: int, field_backend: str | None = None) -> int:
        p = sim_params(deck, field_backend, self.device)
        i = C.c_longlong()
        _check(lib().fs_pool_submit(self._h, C.byref(p), int(steps), C.byref(i)))
        return i.value

    def cancel(self, rid: int) -> None:
        _check(lib().fs_pool_cancel(self._h, int(rid)))

    def poll(self, rid: int) -> dict:
        r = RequestInfo()
        _check(lib().fs_pool_poll(self._h, int(rid), C.byref(r)))
        d = {f: getattr(r, f) for f, _ in RequestInfo._fields_ if f != "error"}
        d["state"] = REQUEST_STATES[r.state]
        d["error"] = r.error.decode(errors="replace")
        return d

    def wait(self, rid: int, timeout: float | None = None) -> str:
        s = C.c_int()
        _check(lib().fs_pool_wait(self._h, int(rid), -1.0 if timeout is None else 1e3 * timeout, C.byref(s)))
        return REQUEST_STATES[s.value]

    def result(self, rid: int) -> dict:
        n = self.poll(rid)["npoints"]
        a = {k: np.zeros(n) for k in ("xs", "ps", "fs", "q_ws", "es")}
        _check(lib().fs_pool_result(self._h, int(rid), *(_ptr(a[k]) for k in ("xs", "ps", "fs", "q_ws", "es"))))
        return a

    def release(self, rid: int) -> None:
        _check(lib().fs_pool_release(self._h, int(rid)))

    def step_times(self, rid: int):
        buf = np.zeros(100000)
        n = C.c_int()
        _check(lib().fs_pool_step_times(self._h, int(rid), _ptr(buf), len(buf), C.byref(n)))
        return buf[: n.value].copy()

    def stats(self) -> dict:
        s = PoolStats()
        _check(lib().fs_pool_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in PoolStats._fields_}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().fs_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------- host mesh
def mesh(initial_height, p_height, xmin, xmax, pmin, pmax, q=-1.0, quadrature=0):
    """Uniform periodic panel mesh (create_prerefined_mesh, AMRStructure_amr.cpp:127-230),
    built by the library's host code.  Returns dict of xs, ps, panels (n x 18), leaves, base_weights."""
    npts, npan, nlv = C.c_int(), C.c_int(), C.c_int()
    _check(lib().fs_mesh_sizes(initial_height, p_height, C.byref(npts), C.byref(npan), C.byref(nlv)))
    xs, ps, w = np.zeros(npts.value), np.zeros(npts.value), np.zeros(npts.value)
    panels = np.zeros((npan.value, PANEL_INTS), dtype=np.int32)
    leaves = np.zeros(nlv.value, dtype=np.int32)
    _check(lib().fs_mesh_fill(initial_height, p_height, xmin, xmax, pmin, pmax, q, quadrature, _ptr(xs), _ptr(ps),
                              panels.ctypes.data_as(_ip), leaves.ctypes.data_as(_ip), _ptr(w)))
    return {"xs": xs, "ps": ps, "panels": panels, "leaves": leaves, "base_weights": w}


def field_energy(xs, es, L: float) -> float:
    """Electrostatic field energy W = 1/2 sum dx E^2 of a state, the potential
    energy of the reference's diagnostics (standard_interface/diagnostic_plot.py:122-130):
    E at the unique positions inside [0, L), each weighted by half the distance
    between its periodic neighbours.  Host arithmetic on exported arrays."""
    xs = np.asarray(xs, dtype=np.float64)
    es = np.asarray(es, dtype=np.float64)
    x_sort, idx = np.unique(xs, return_index=True)
    e_sort = es[idx]
    keep = np.nonzero((x_sort >= 0) * (x_sort < L))
    mx, me = x_sort[keep], e_sort[keep]
    dxs = 0.5 * np.hstack([mx[1] + L - mx[-1], mx[2:] - mx[:-2], mx[0] + L - mx[-2]])
    if np.any(dxs <= 0):
        raise ValueError("field_energy: positions need at least three distinct values in [0, L)")
    return 0.5 * float(np.dot(dxs, me ** 2))
