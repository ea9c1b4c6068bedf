"""CPU oracle for the FARRSIGHT per-step hot path -- TEST INFRASTRUCTURE ONLY.

Three libraries, all built by ``oracle/Makefile``:

* ``oracle/_ref/libfs_ref.so`` -- the reference's own ``src/FieldStructure.cpp``
  compiled unmodified (direct sum ``src/FieldStructure.cpp:102-156`` and treecode
  ``:230-1020``).  This is the pin for the field.
* ``oracle/_ref/libamr_ref.so`` -- every source of the reference's simulation
  (``src/structure_files``, ``src/simulation_files``, ``src/FieldStructure.cpp``)
  compiled unmodified, with stand-ins for the Eigen / Boost calls it makes
  (``oracle/refshim``), driven through ``amr_harness.cpp``.  This is the pin for
  the mesh, RK4, step control, remesh, reduced grid, adaptive refinement and
  initial conditions.
* ``oracle/liboracle.so`` -- ``fs_oracle.c``, a plain C restatement of the whole
  hot path (field, treecode, panel mesh, remesh, RK4 step control), checked bit
  for bit against both reference libraries.  Its 9x9 solve and the Eigen
  stand-in share the same partial-pivot LU; against Eigen itself the remesh fit
  agrees to rounding.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline / reference arm
of ``bench.py`` may import this package.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libfs_ref.so")
_AMR_REF = os.path.join(HERE, "_ref", "libamr_ref.so")
PANEL_INTS = 18

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build(ref_dir: str | None = None) -> None:
    """Compile the oracle (and the reference library when its sources exist)."""
    cmd = ["make", "-s", "-C", HERE]
    if ref_dir:
        cmd.append(f"REF={ref_dir}")
    subprocess.run(cmd, check=True)


class FsoSpecies(C.Structure):
    _fields_ = [("q", C.c_double), ("m", C.c_double), ("initial_height", C.c_int),
                ("p_height", C.c_int), ("pmin", C.c_double), ("pmax", C.c_double),
                ("ics_type", C.c_int), ("pth", C.c_double), ("pstr", C.c_double),
                ("amp", C.c_double), ("normalized_wavenumber", C.c_double),
                ("do_adaptively_refine", C.c_int), ("max_height", C.c_int), ("n_amr_eps", C.c_int),
                ("amr_eps", C.c_double * 5), ("mu", C.c_double), ("wave_beta", C.c_double)]


class FsoSim(C.Structure):
    _fields_ = [("xmin", C.c_double), ("xmax", C.c_double), ("quadrature", C.c_int),
                ("dt", C.c_double), ("remesh_period", C.c_int), ("greens_epsilon", C.c_double),
                ("use_treecode", C.c_int), ("mac", C.c_double), ("degree", C.c_int),
                ("max_source", C.c_int), ("num_species", C.c_int), ("species", FsoSpecies * 8),
                ("use_external_field", C.c_int), ("external_type", C.c_int), ("ext_Am", C.c_double),
                ("ext_k", C.c_double), ("ext_omega", C.c_double), ("relativistic_push", C.c_int)]


_lib = None
_ref = None
_amr_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        L.fso_direct_sum.argtypes = [C.c_double, C.c_double, _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        L.fso_treecode.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp, C.c_int]
        L.fso_treecode.restype = C.c_int
        L.fso_mesh_build.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
        L.fso_mesh_build.restype = C.c_void_p
        L.fso_mesh_destroy.argtypes = [C.c_void_p]
        for n in ("fso_mesh_npoints", "fso_mesh_npanels", "fso_mesh_nleaves"):
            getattr(L, n).argtypes = [C.c_void_p]
            getattr(L, n).restype = C.c_int
        L.fso_mesh_points.argtypes = [C.c_void_p, _dp, _dp]
        L.fso_mesh_panels.argtypes = [C.c_void_p, _ip]
        L.fso_mesh_leaves.argtypes = [C.c_void_p, _ip]
        L.fso_mesh_base_weights.argtypes = [C.c_void_p, C.c_double, C.c_int, _dp]
        L.fso_f0.argtypes = [C.c_int] + [C.c_double] * 6
        L.fso_f0.restype = C.c_double
        L.fso_dist_create.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.fso_dist_create.restype = C.c_void_p
        L.fso_dist_eval.argtypes = [C.c_void_p, C.c_double, C.c_double, C.POINTER(C.c_int)]
        L.fso_dist_eval.restype = C.c_double
        L.fso_dist_destroy.argtypes = [C.c_void_p]
        for n in ("fso_bessel_k1",):
            getattr(L, n).argtypes = [C.c_double]
            getattr(L, n).restype = C.c_double
        for n in ("fso_ellint_1", "fso_ellint_2"):
            getattr(L, n).argtypes = [C.c_double, C.c_double]
            getattr(L, n).restype = C.c_double
        L.fso_remesh_interp.argtypes = [C.c_void_p, _dp, _dp, _dp, C.c_double, _dp, _ip, _dp]
        L.fso_remesh_interp.restype = C.c_int
        L.fso_reduce.argtypes = [_dp, _dp, C.c_int, _dp, _dp, _ip]
        L.fso_reduce.restype = C.c_int
        L.fso_direct_sum_open.argtypes = [C.c_double, _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        L.fso_external_amplitude.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double]
        L.fso_external_amplitude.restype = C.c_double
        L.fso_external_field.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, C.c_int,
                                         C.c_double]
        L.fso_sim_create.argtypes = [C.POINTER(FsoSim)]
        L.fso_sim_create.restype = C.c_void_p
        L.fso_sim_destroy.argtypes = [C.c_void_p]
        L.fso_sim_step.argtypes = [C.c_void_p]
        L.fso_sim_step.restype = C.c_int
        L.fso_sim_total_points.argtypes = [C.c_void_p]
        L.fso_sim_total_points.restype = C.c_int
        L.fso_sim_species_points.argtypes = [C.c_void_p, C.c_int]
        L.fso_sim_species_points.restype = C.c_int
        L.fso_sim_iter.argtypes = [C.c_void_p]
        L.fso_sim_iter.restype = C.c_int
        L.fso_sim_state.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        L.fso_sim_counters.argtypes = [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    """The reference's own field solvers (oracle/_ref/libfs_ref.so)."""
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise FileNotFoundError(f"{_REF} missing: run `make -C oracle` where the reference sources exist")
        R = C.CDLL(_REF)
        R.fsref_set_threads.argtypes = [C.c_int]
        R.fsref_set_threads.restype = C.c_int
        R.fsref_direct_sum.argtypes = [C.c_double, C.c_double, _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        R.fsref_direct_sum.restype = C.c_int
        R.fsref_direct_sum_open.argtypes = [C.c_double, _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        R.fsref_direct_sum_open.restype = C.c_int
        R.fsref_external.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, _dp, _dp, C.c_int, C.c_double]
        R.fsref_external.restype = C.c_int
        R.fsref_treecode.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                     _dp, _dp, C.c_int, _dp, _dp, C.c_int]
        R.fsref_treecode.restype = C.c_int
        _ref = R
    return _ref


def amr_ref_available() -> bool:
    return os.path.exists(_AMR_REF)


def amr_ref():
    """The reference's own simulation code (oracle/_ref/libamr_ref.so: every
    source of src/structure_files, src/simulation_files and src/FieldStructure.cpp
    with amr_harness.cpp)."""
    global _amr_ref
    if _amr_ref is None:
        if not os.path.exists(_AMR_REF):
            raise FileNotFoundError(f"{_AMR_REF} missing: run `make -C oracle REF=<reference checkout>`")
        R = C.CDLL(_AMR_REF)
        R.amrref_sim_create.argtypes = [C.c_char_p, C.c_char_p]
        R.amrref_sim_create.restype = C.c_void_p
        R.amrref_sim_destroy.argtypes = [C.c_void_p]
        R.amrref_sim_step.argtypes = [C.c_void_p, C.c_int]
        R.amrref_sim_step.restype = C.c_int
        for n in ("amrref_sim_remesh", "amrref_sim_nspecies"):
            getattr(R, n).argtypes = [C.c_void_p]
            getattr(R, n).restype = C.c_int
        for n in ("amrref_sim_species_points", "amrref_sim_npanels", "amrref_sim_nleaves", "amrref_sim_nreduced"):
            getattr(R, n).argtypes = [C.c_void_p, C.c_int]
            getattr(R, n).restype = C.c_int
        R.amrref_sim_iter.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        R.amrref_sim_iter.restype = C.c_int
        R.amrref_sim_state.argtypes = [C.c_void_p] + [C.c_void_p] * 5
        R.amrref_sim_state.restype = C.c_int
        R.amrref_sim_set_xp.argtypes = [C.c_void_p, _dp, _dp]
        R.amrref_sim_set_xp.restype = C.c_int
        R.amrref_sim_panels.argtypes = [C.c_void_p, C.c_int, _ip]
        R.amrref_sim_panels.restype = C.c_int
        R.amrref_sim_leaves.argtypes = [C.c_void_p, C.c_int, _ip]
        R.amrref_sim_leaves.restype = C.c_int
        R.amrref_sim_reduced.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        R.amrref_sim_reduced.restype = C.c_int
        R.amrref_sim_f_beyond.argtypes = [C.c_void_p, C.c_int]
        R.amrref_sim_f_beyond.restype = C.c_double
        R.amrref_sim_f0.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, _dp]
        R.amrref_sim_f0.restype = C.c_int
        _amr_ref = R
    return _amr_ref


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# ---------------------------------------------------------------- field
def direct_sum(L, eps, targets, sources, q):
    t, s, q = _f64(targets), _f64(sources), _f64(q)
    es = np.zeros(len(t))
    lib().fso_direct_sum(L, eps, es, t, len(t), s, q, len(s))
    return es


def adaptive_mesh(h, ph, xmin, xmax, pmin, pmax, f0_params, amr_eps, max_height, L=None):
    """Initial adaptive mesh: the uniform mesh, f0 at its points, then
    generate_mesh's refinement with f0 at the new points.  f0_params =
    (ics_type, pth, pstr, amp, normalized_wavenumber).  Returns (xs, ps, f,
    panels (n x 18), leaves)."""
    m = Mesh(h, ph, xmin, xmax, pmin, pmax)
    ics, pth, pstr, amp, nk = f0_params
    _stateless_ics(ics)
    kx = 2 * np.pi / ((xmax - xmin) if L is None else L) * nk
    n = m.npoints
    f = np.array([lib().fso_f0(ics, pth, pstr, kx, amp, x, p) for x, p in zip(m.xs, m.ps)])
    fbuf = lib().fso_f0  # keep a reference while the callback runs
    CB = C.CFUNCTYPE(None, C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int,
                     C.POINTER(C.c_double))

    def cb(ctx, xp, pp, k, out):
        for i in range(k):
            out[i] = fbuf(ics, pth, pstr, kx, amp, xp[i], pp[i])

    ccb = CB(cb)
    L_ = lib()
    L_.fso_mesh_adapt.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_double), C.c_int, C.c_int, CB, C.c_void_p]
    L_.fso_mesh_adapt.restype = C.c_void_p
    L_.malloc_double = None
    import ctypes.util
    libc = C.CDLL(ctypes.util.find_library("c"))
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.free.argtypes = [C.c_void_p]
    buf = libc.malloc(8 * n)
    C.memmove(buf, f.ctypes.data, 8 * n)
    e = (C.c_double * 5)(*amr_eps[:5])
    fp = L_.fso_mesh_adapt(m._m, buf, e, len(amr_eps[:5]), max_height, ccb, None)
    m.npoints = L_.fso_mesh_npoints(m._m)
    m.npanels = L_.fso_mesh_npanels(m._m)
    m.nleaves = L_.fso_mesh_nleaves(m._m)
    xs, ps = np.zeros(m.npoints), np.zeros(m.npoints)
    L_.fso_mesh_points(m._m, xs, ps)
    panels = np.zeros((m.npanels, PANEL_INTS), dtype=np.int32)
    L_.fso_mesh_panels(m._m, panels)
    leaves = np.zeros(m.nleaves, dtype=np.int32)
    L_.fso_mesh_leaves(m._m, leaves)
    fo = np.ctypeslib.as_array((C.c_double * m.npoints).from_address(fp)).copy()
    libc.free(fp)
    return xs, ps, fo, panels, leaves


def direct_sum_open(eps, targets, sources, q):
    """E_MQ_DirectSum_openbcs (src/FieldStructure.cpp:170-192), restated."""
    t, s, q = _f64(targets), _f64(sources), _f64(q)
    es = np.zeros(len(t))
    lib().fso_direct_sum_open(eps, es, t, len(t), s, q, len(s))
    return es


def external_field(kind, Am, k, omega, es, x, t):
    """Drive field added into es in place (src/FieldStructure.cpp:15-96), restated;
    kind 0 tanh, 1 sine, 2 logistic."""
    x = _f64(x)
    lib().fso_external_field(int(kind), Am, k, omega, es, x, len(x), t)
    return es


def ref_direct_sum_open(eps, targets, sources, q):
    t, s, q = _f64(targets), _f64(sources), _f64(q)
    es = np.zeros(len(t))
    ref().fsref_direct_sum_open(eps, es, t, len(t), s, q, len(s))
    return es


def ref_external_field(kind, Am, k, omega, es, x, t):
    x = _f64(x)
    ref().fsref_external(int(kind), Am, k, omega, es, x, len(x), t)
    return es


def treecode(L, eps, mac, degree, max_source, sources, q):
    s, q = _f64(sources), _f64(q)
    es = np.zeros(len(s))
    rc = lib().fso_treecode(L, eps, mac, degree, max_source, es, s, q, len(s))
    if rc < 0:
        raise RuntimeError("treecode: unbounded tree recursion")
    return es


def ref_direct_sum(L, eps, targets, sources, q, threads=0):
    t, s, q = _f64(targets), _f64(sources), _f64(q)
    es = np.zeros(len(t))
    R = ref()
    R.fsref_set_threads(threads)
    R.fsref_direct_sum(L, eps, es, t, len(t), s, q, len(s))
    return es


def ref_treecode(L, eps, mac, degree, max_source, sources, q, max_target=2000):
    s, q = _f64(sources), _f64(q)
    es = np.zeros(len(s))
    ref().fsref_treecode(L, eps, mac, degree, max_source, max_target, es, s, len(s), s, q, len(s))
    return es


# ---------------------------------------------------------------- mesh
class Mesh:
    """create_prerefined_mesh + uniform refinement (AMRStructure_amr.cpp:127-230)."""

    def __init__(self, h, ph, xmin, xmax, pmin, pmax):
        self.h, self.ph = h, ph
        self.xmin, self.xmax, self.pmin, self.pmax = xmin, xmax, pmin, pmax
        self._m = lib().fso_mesh_build(h, ph, xmin, xmax, pmin, pmax)
        if not self._m:
            raise ValueError("bad mesh parameters")
        L = lib()
        self.npoints = L.fso_mesh_npoints(self._m)
        self.npanels = L.fso_mesh_npanels(self._m)
        self.nleaves = L.fso_mesh_nleaves(self._m)
        self.xs = np.zeros(self.npoints)
        self.ps = np.zeros(self.npoints)
        L.fso_mesh_points(self._m, self.xs, self.ps)
        self.panels = np.zeros((self.npanels, PANEL_INTS), dtype=np.int32)
        L.fso_mesh_panels(self._m, self.panels)
        self.leaves = np.zeros(self.nleaves, dtype=np.int32)
        L.fso_mesh_leaves(self._m, self.leaves)

    def base_weights(self, q, quad):
        w = np.zeros(self.npoints)
        lib().fso_mesh_base_weights(self._m, q, quad, w)
        return w

    def remesh(self, old_xs, old_ps, old_fs, f_beyond):
        nf = np.zeros(self.npoints)
        leaf = np.zeros(self.npoints, dtype=np.int32)
        fx = np.zeros(self.npoints)
        rc = lib().fso_remesh_interp(self._m, _f64(old_xs), _f64(old_ps), _f64(old_fs), f_beyond, nf, leaf, fx)
        if rc:
            raise RuntimeError("too many shifts!")
        return nf, leaf, fx

    def __del__(self):
        if getattr(self, "_m", None):
            lib().fso_mesh_destroy(self._m)
            self._m = None


def _stateless_ics(ics):
    """fso_f0 holds the closed forms (ics 1-4, 9, 10 and the Landau default);
    the tabulated and Bessel-normalised forms need initial_f0's parameters."""
    if int(ics) in (5, 6, 7, 8):
        raise ValueError(f"ics_type {ics} needs initial_f0(deck, species, x, p)")


def f0(ics, pth, pstr, k, amp, x, p):
    _stateless_ics(ics)
    fn = lib().fso_f0
    return np.array([fn(ics, pth, pstr, k, amp, float(a), float(b)) for a, b in zip(x, p)])


def initial_f0(deck: dict, species: int, x, p):
    """f0 of one species of a deck at the points (x, p): the distribution
    make_f0_return_ptr builds (AMRSimulation_load.cpp:139-225), every ics_type.
    Raises ValueError for invalid parameters or points beyond the
    Friedman-beam / travelling-wave tables."""
    P = sim_params(deck)
    rc = C.c_int(0)
    d = lib().fso_dist_create(C.byref(P.species[species]), P.xmin, P.xmax, C.byref(rc))
    if not d:
        raise ValueError("invalid initial-condition parameters")
    try:
        out = np.empty(len(x))
        for i, (a, b) in enumerate(zip(np.asarray(x, dtype=np.float64), np.asarray(p, dtype=np.float64))):
            out[i] = lib().fso_dist_eval(d, float(a), float(b), C.byref(rc))
        if rc.value:
            raise ValueError("point beyond the tabulated initial condition")
        return out
    finally:
        lib().fso_dist_destroy(d)


def bessel_k1(x):
    return lib().fso_bessel_k1(float(x))


def ellint_1(k, phi):
    return lib().fso_ellint_1(float(k), float(phi))


def ellint_2(k, phi):
    return lib().fso_ellint_2(float(k), float(phi))


def reduce(xs, q):
    xs, q = _f64(xs), _f64(q)
    n = len(xs)
    rx, rw, inv = np.zeros(n), np.zeros(n), np.zeros(n, dtype=np.int32)
    u = lib().fso_reduce(xs, q, n, rx, rw, inv)
    return rx[:u].copy(), rw[:u].copy(), inv


# ---------------------------------------------------------------- simulation
def _amr_params(sp: dict):
    """(do_adaptively_refine, max_height, amr_epsilons) as AMRSimulation_load.cpp:246-258
    reads them: without amr_epsilons the refinement is disabled."""
    eps = sp.get("amr_epsilons")
    on = bool(sp.get("do_adaptively_refine", False)) and eps is not None
    eps = [float(e) for e in (eps or [])][:5]
    return (1 if on else 0), int(sp.get("max_height", sp.get("initial_height", 6))), eps


def sim_params(deck: dict) -> FsoSim:
    """Deck dict (deck.json keys) -> oracle simulation parameters."""
    P = FsoSim()
    P.xmin, P.xmax = deck.get("xmin", 0.0), deck.get("xmax", 0.0)
    P.quadrature = int(deck.get("quadrature", 1))
    P.dt = deck.get("dt", 0.5)
    P.remesh_period = int(deck.get("remesh_period", 1))
    P.greens_epsilon = deck.get("greens_epsilon", 0.2)
    P.use_treecode = int(deck.get("use_treecode", 0))
    P.mac = deck.get("mac", -1.0)
    P.degree = int(deck.get("degree", -1))
    P.max_source = int(deck.get("max_source", 2000))
    sl = deck["species_list"]
    P.num_species = len(sl)
    for i, sp in enumerate(sl):
        S = P.species[i]
        S.q, S.m = sp.get("q", -1.0), sp.get("m", 1.0)
        S.initial_height, S.p_height = int(sp.get("initial_height", 6)), int(sp.get("p_height", 0))
        S.pmin, S.pmax = sp.get("pmin", -1.0), sp.get("pmax", 1.0)
        S.ics_type = int(sp.get("ics_type", 1))
        S.pth, S.pstr, S.amp = sp.get("pth", 1.0), sp.get("pstr", 0.0), sp.get("amp", 0.0)
        S.normalized_wavenumber = sp.get("normalized_wavenumber", 1.0)
        amr = _amr_params(sp)
        S.do_adaptively_refine, S.max_height, S.n_amr_eps = amr[0], amr[1], len(amr[2])
        for k, e in enumerate(amr[2]):
            S.amr_eps[k] = e
        S.mu, S.wave_beta = float(sp.get("mu", 1.0)), float(sp.get("wave_beta", 0.8))
    P.relativistic_push = 1 if int(deck.get("relativistic_push", 0)) > 0 else 0
    ext = deck.get("external_field") or {}
    P.use_external_field = 1 if int(ext.get("use_external_field", 0)) > 0 else 0
    if P.use_external_field:
        P.external_type = int(ext.get("external_type", 0))
        P.ext_Am, P.ext_k, P.ext_omega = float(ext["Am"]), float(ext["k"]), float(ext["omega"])
    return P


class Sim:
    """Oracle AMRSimulation (AMRSimulation.cpp:5-91, AMRSimulation_step.cpp:5-99)."""

    def __init__(self, deck: dict):
        self._p = sim_params(deck)
        self._s = lib().fso_sim_create(C.byref(self._p))
        if not self._s:
            raise ValueError("bad deck")
        self.n = lib().fso_sim_total_points(self._s)
        self.species_points = [lib().fso_sim_species_points(self._s, i) for i in range(self._p.num_species)]

    def step(self, n=1):
        for _ in range(n):
            rc = lib().fso_sim_step(self._s)
            if rc:
                raise RuntimeError("oracle step failed (too many shifts)")

    @property
    def iter(self):
        return lib().fso_sim_iter(self._s)

    def state(self):
        self.n = lib().fso_sim_total_points(self._s)  # adaptive meshes change it at remesh
        a = {k: np.zeros(self.n) for k in ("xs", "ps", "fs", "q_ws", "es")}
        lib().fso_sim_state(self._s, *(a[k].ctypes.data for k in ("xs", "ps", "fs", "q_ws", "es")))
        return a

    def counters(self):
        f, r = C.c_longlong(), C.c_longlong()
        lib().fso_sim_counters(self._s, C.byref(f), C.byref(r))
        return f.value, r.value

    def __del__(self):
        if getattr(self, "_s", None):
            lib().fso_sim_destroy(self._s)
            self._s = None


# ---------------------------------------------------------------- diagnostics
def field_energy(xs, es, L):
    """Field energy 0.5 * sum dx * E^2 over the unique x in [0, L) with periodic
    centred spacing (standard_interface/diagnostic_plot.py:119-129)."""
    xs = np.asarray(xs, dtype=np.float64)
    es = np.asarray(es, dtype=np.float64)
    x_sort, idx = np.unique(xs, return_index=True)
    e_sort = es[idx]
    keep = np.nonzero((x_sort >= 0) * (x_sort < L))
    mx, me = x_sort[keep], e_sort[keep]
    dxs = 0.5 * np.hstack([mx[1] + L - mx[-1], mx[2:] - mx[:-2], mx[0] + L - mx[-2]])
    return 0.5 * float(np.dot(dxs, me ** 2))


# ---------------------------------------------------------------- the reference simulation
class RefSim:
    """The reference's AMRSimulation (oracle/_ref/libamr_ref.so), built from a
    deck dict exactly as run_FARRSIGHT2.cpp builds it from deck.json: the deck
    is written as JSON into a fresh simulation directory holding the output
    folders the reference writes to (simulation_output/<species>/{xs,ps,fs,
    panels} and simulation_output/{reduce_xs,reduced_es}), then stepped with
    AMRSimulation::step.  `sim_dir` keeps the reference's dump files for
    comparisons; by default a temporary directory removed on close."""

    def __init__(self, deck: dict, sim_dir: str | None = None):
        import json
        import tempfile
        self._s = None
        self._tmp = None
        if sim_dir is None:
            self._tmp = tempfile.TemporaryDirectory(prefix="amrref_")
            sim_dir = self._tmp.name
        self.sim_dir = os.path.join(os.path.abspath(sim_dir), "")
        out = os.path.join(self.sim_dir, "simulation_output")
        for sp in deck["species_list"]:
            for sub in ("xs", "ps", "fs", "panels"):
                os.makedirs(os.path.join(out, sp["name"], sub), exist_ok=True)
        for sub in ("reduce_xs", "reduced_es"):
            os.makedirs(os.path.join(out, sub), exist_ok=True)
        self.deck_path = os.path.join(self.sim_dir, "deck.json")
        with open(self.deck_path, "w") as f:
            json.dump(deck, f)
        R = amr_ref()
        self._s = R.amrref_sim_create(self.sim_dir.encode(), self.deck_path.encode())
        if not self._s:
            raise ValueError("the reference rejected the deck")
        self.nspecies = R.amrref_sim_nspecies(self._s)

    @property
    def species_points(self):
        return [amr_ref().amrref_sim_species_points(self._s, i) for i in range(self.nspecies)]

    @property
    def n(self):
        return int(sum(self.species_points))

    def step(self, n=1):
        if amr_ref().amrref_sim_step(self._s, int(n)):
            raise RuntimeError("reference step raised")

    def remesh(self):
        if amr_ref().amrref_sim_remesh(self._s):
            raise RuntimeError("reference remesh raised")

    @property
    def iter(self):
        return amr_ref().amrref_sim_iter(self._s, None)

    @property
    def t(self):
        t = C.c_double()
        amr_ref().amrref_sim_iter(self._s, C.byref(t))
        return t.value

    def state(self):
        a = {k: np.zeros(self.n) for k in ("xs", "ps", "fs", "q_ws", "es")}
        amr_ref().amrref_sim_state(self._s, *(a[k].ctypes.data for k in ("xs", "ps", "fs", "q_ws", "es")))
        return a

    def set_xp(self, xs, ps):
        amr_ref().amrref_sim_set_xp(self._s, _f64(xs), _f64(ps))

    def panels(self, species):
        R = amr_ref()
        out = np.zeros((R.amrref_sim_npanels(self._s, species), PANEL_INTS), dtype=np.int32)
        R.amrref_sim_panels(self._s, species, out)
        return out

    def leaves(self, species):
        R = amr_ref()
        out = np.zeros(R.amrref_sim_nleaves(self._s, species), dtype=np.int32)
        R.amrref_sim_leaves(self._s, species, out)
        return out

    def reduced(self, species):
        """(unique x, summed weights, reduced E) of the species' last reduced grid."""
        R = amr_ref()
        u = R.amrref_sim_nreduced(self._s, species)
        rx, rw, re = np.zeros(u), np.zeros(u), np.zeros(u)
        R.amrref_sim_reduced(self._s, species, rx.ctypes.data, rw.ctypes.data, re.ctypes.data)
        return rx, rw, re

    def f_beyond_boundary(self, species):
        return amr_ref().amrref_sim_f_beyond(self._s, species)

    def f0(self, species, x, p):
        x, p = _f64(x), _f64(p)
        out = np.zeros(len(x))
        if amr_ref().amrref_sim_f0(self._s, species, len(x), x, p, out):
            raise RuntimeError("reference initial condition raised")
        return out

    def close(self):
        if getattr(self, "_s", None):
            amr_ref().amrref_sim_destroy(self._s)
            self._s = None
        if getattr(self, "_tmp", None):
            self._tmp.cleanup()
            self._tmp = None

    def __del__(self):
        self.close()
