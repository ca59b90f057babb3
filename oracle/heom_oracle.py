"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module, always as the checker or the timed CPU baseline.

Two libraries are wrapped:
  * oracle/_build/libheom_oracle.so -- the plain-C restatement (heom_oracle.c)
  * oracle/_ref/libheom_refcl.so    -- the reference's own heom_ode.cl /
    rk_weighted_add.cl compiled unmodified as C++ (present when the reference
    sources were available at build time)

Physical set-up helpers follow the reference:
  * config SI conversion      dm-heom/src/heom/config.cpp:182-191
  * hierarchy graph           dm-heom/src/heom/hierarchy_graph.cpp:30-181
  * bath precompute           dm-heom/src/heom/instance.cpp:155-273
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HBAR = 1.05457148e-34
KB = 1.380650239684840458953781387048428305608616777679979316e-23
INVCM_TO_JOULE = 1.986456217327470903861498336971100097137908380913187891e-23
INVALID_UID = -2

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class _Graph(C.Structure):
    _fields_ = [("width", C.c_int32), ("depth", C.c_int32), ("nodes", C.c_int64),
                ("first_non_plus", C.c_int32), ("tuples", C.POINTER(C.c_int32)),
                ("plus", C.POINTER(C.c_int32)), ("minus", C.POINTER(C.c_int32)),
                ("nodes_per_depth", C.POINTER(C.c_int64))]


class _System(C.Structure):
    _fields_ = [("states", C.c_int32), ("baths", C.c_int32), ("matsubaras", C.c_int32),
                ("baths_per_state", C.c_int32), ("coupling", C.c_void_p),
                ("temperature", C.c_double), ("lambda_", C.c_void_p), ("invnu", C.c_void_p),
                ("omega", C.c_void_p)]


class _Problem(C.Structure):
    _fields_ = [("states", C.c_int32), ("matsubaras", C.c_int32), ("baths_per_state", C.c_int32),
                ("ado_width", C.c_int32), ("nodes", C.c_int64), ("first_non_plus", C.c_int32),
                ("coupling", C.c_void_p), ("hamiltonian", C.c_void_p), ("tuples", C.c_void_p),
                ("plus", C.c_void_p), ("minus", C.c_void_p), ("pf_same_sum", C.c_void_p),
                ("pf_same", C.c_void_p), ("pf_circ", C.c_void_p), ("cbk", C.c_void_p),
                ("cbk_sqrt", C.c_void_p), ("mask", C.c_void_p)]


_lib = None
_ref = {}


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "_build", "libheom_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"oracle library missing: {path} (run __graft_entry__.build())")
        L = C.CDLL(path)
        L.ho_binomial.restype = C.c_int64
        L.ho_binomial.argtypes = [C.c_int64, C.c_int64]
        L.ho_integer_partitions.restype = C.c_int64
        L.ho_integer_partitions.argtypes = [C.c_int32, C.c_int32, _i32p, C.c_int64]
        L.ho_graph_build.restype = C.c_int
        L.ho_graph_build.argtypes = [C.c_int32, C.c_int32, C.POINTER(_Graph)]
        L.ho_graph_free.argtypes = [C.POINTER(_Graph)]
        L.ho_precompute_baths.argtypes = [C.POINTER(_System), C.POINTER(_Graph), _f64p, _f64p,
                                          _f64p, _f64p, _f64p]
        L.ho_derivative.argtypes = [C.POINTER(_Problem), _f64p, _f64p, C.c_int]
        L.ho_derivative_ld.argtypes = [C.POINTER(_Problem), C.c_void_p, C.c_void_p, C.c_int]
        L.ho_rk4_step.argtypes = [C.POINTER(_Problem), C.c_double, _f64p, _f64p, _f64p, C.c_int]
        L.ho_propagate.restype = C.c_int64
        L.ho_propagate.argtypes = [C.POINTER(_Problem), C.c_double, C.c_int64, C.c_int64, _f64p,
                                   _f64p, C.c_int]
        L.ho_propagate_ld.restype = C.c_int64
        L.ho_propagate_ld.argtypes = L.ho_propagate.argtypes
        _lib = L
    return _lib


def _cpu_has_x86_64_v3():
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
        return {"avx2", "fma", "bmi2", "movbe"} <= flags
    except OSError:
        return False


def ref_lib(fast=False):
    """The reference's own kernels compiled for the host, or None.  fast=True:
    the build for timing (-O3, x86-64-v3, contraction allowed) when this CPU
    runs it, else the parity build (-O2, no contraction)."""
    key = "fast" if fast and _cpu_has_x86_64_v3() else "parity"
    if key not in _ref:
        name = "libheom_refcl_fast.so" if key == "fast" else "libheom_refcl.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            return None if key == "parity" else ref_lib(False)
        R = C.CDLL(path)
        R.refcl_heom_ode.restype = C.c_int
        R.refcl_heom_ode.argtypes = [
            C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_int, _i32p,
            C.c_double, C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_int, _f64p, _f64p,
            _i32p, _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, _f64p, _u8p, C.c_int]
        R.refcl_rk_weighted_add.restype = C.c_int
        R.refcl_rk_weighted_add.argtypes = [C.c_int, C.c_int64, C.c_int, C.c_double, _f64p, _f64p,
                                            _f64p, C.POINTER(C.c_void_p), C.c_int]
        _ref[key] = R
    return _ref[key]


def ref_ip_lib():
    path = os.path.join(HERE, "_ref", "libheom_refip.so")
    if not os.path.exists(path):
        return None
    R = C.CDLL(path)
    R.refip_integer_partitions.restype = C.c_int64
    R.refip_integer_partitions.argtypes = [C.c_int32, C.c_int32, _i64p, C.c_int64]
    return R


def default_threads():
    return max(1, os.cpu_count() or 1)


# --------------------------------------------------------------------------
# graph / system
# --------------------------------------------------------------------------

@dataclass
class Graph:
    width: int
    depth: int
    nodes: int
    first_non_plus: int
    tuples: np.ndarray
    plus: np.ndarray
    minus: np.ndarray
    nodes_per_depth: np.ndarray


def build_graph(width: int, depth: int) -> Graph:
    g = _Graph()
    rc = lib().ho_graph_build(width, depth, C.byref(g))
    if rc != 0:
        raise RuntimeError(f"ho_graph_build failed: {rc}")
    n = g.nodes
    t = np.ctypeslib.as_array(g.tuples, shape=(n, width)).copy()
    p = np.ctypeslib.as_array(g.plus, shape=(n, width)).copy()
    m = np.ctypeslib.as_array(g.minus, shape=(n, width)).copy()
    npd = np.ctypeslib.as_array(g.nodes_per_depth, shape=(depth + 1,)).copy()
    res = Graph(width, depth, n, g.first_non_plus, t, p, m, npd)
    lib().ho_graph_free(C.byref(g))
    return res


def integer_partitions(n: int, s: int) -> np.ndarray:
    cap = int(lib().ho_binomial(n + s - 1, s - 1)) + 1
    out = np.zeros(cap * s, np.int32)
    cnt = lib().ho_integer_partitions(n, s, out, cap)
    if cnt < 0:
        raise RuntimeError("partition buffer too small")
    return out[: cnt * s].reshape(cnt, s)


@dataclass
class System:
    """A population-dynamics system in SI units (after config post_process)."""
    hamiltonian: np.ndarray          # complex (N, N), J
    coupling: np.ndarray             # int32 (N, baths_per_state)
    lambda_: np.ndarray              # (B,) J
    invnu: np.ndarray                # (B,) s
    omega: np.ndarray                # (B,) rad/s
    matsubaras: int
    temperature: float
    depth: int
    rho_init: np.ndarray = field(default=None)  # complex (N, N)

    @property
    def states(self):
        return self.hamiltonian.shape[0]

    @property
    def baths(self):
        return self.lambda_.shape[0]

    @property
    def width(self):
        return self.baths * self.matsubaras


def make_system(h_invcm, lambda_invcm, invnu_fs, omega_invcm, matsubaras, temperature, depth,
                coupling=None, rho_init=None) -> System:
    """Build a System from config units (cm^-1, fs) with config.cpp:182-191's scaling."""
    h = np.asarray(h_invcm, dtype=np.complex128)
    n = h.shape[0]
    lam = np.asarray(lambda_invcm, dtype=np.float64)
    b = lam.shape[0]
    if coupling is None:
        coupling = np.arange(n, dtype=np.int32).reshape(n, 1)
    coupling = np.ascontiguousarray(np.asarray(coupling, dtype=np.int32))
    if rho_init is None:
        rho_init = np.zeros((n, n), np.complex128)
        rho_init[0, 0] = 1.0
    # std::valarray scale: element-wise multiply in double
    hs = np.empty_like(h)
    hs.real = h.real * INVCM_TO_JOULE
    hs.imag = h.imag * INVCM_TO_JOULE
    return System(hamiltonian=hs, coupling=coupling,
                  lambda_=lam * INVCM_TO_JOULE,
                  invnu=np.asarray(invnu_fs, np.float64) * 1.0e-15,
                  omega=np.asarray(omega_invcm, np.float64) * (INVCM_TO_JOULE / HBAR),
                  matsubaras=int(matsubaras), temperature=float(temperature), depth=int(depth),
                  rho_init=np.asarray(rho_init, np.complex128))


@dataclass
class Problem:
    system: System
    graph: Graph
    hamiltonian: np.ndarray   # float64 [N*N*2]
    pf_same_sum: np.ndarray
    pf_same: np.ndarray
    pf_circ: np.ndarray
    cbk: np.ndarray
    cbk_sqrt: np.ndarray
    mask: np.ndarray
    coupling_flat: np.ndarray
    _keep: list = field(default_factory=list)

    @property
    def states(self):
        return self.system.states

    @property
    def state_len(self):
        return self.graph.nodes * self.states * self.states * 2

    def initial_state(self) -> np.ndarray:
        y = np.zeros(self.state_len, np.float64)
        top = self.system.rho_init.reshape(-1)
        y[0:2 * top.size:2] = top.real
        y[1:2 * top.size:2] = top.imag
        return y

    def cstruct(self) -> _Problem:
        s = self.system
        g = self.graph
        p = _Problem()
        p.states = s.states
        p.matsubaras = s.matsubaras
        p.baths_per_state = s.coupling.shape[1]
        p.ado_width = g.width
        p.nodes = g.nodes
        p.first_non_plus = g.first_non_plus
        arrs = [self.coupling_flat, self.hamiltonian, g.tuples, g.plus, g.minus, self.pf_same_sum,
                self.pf_same, self.pf_circ, self.cbk, self.cbk_sqrt, self.mask]
        names = ["coupling", "hamiltonian", "tuples", "plus", "minus", "pf_same_sum", "pf_same",
                 "pf_circ", "cbk", "cbk_sqrt", "mask"]
        for nm, a in zip(names, arrs):
            assert a.flags["C_CONTIGUOUS"]
            setattr(p, nm, a.ctypes.data)
        self._keep = arrs
        return p


def build_problem(system: System, graph: Graph | None = None, mask=None) -> Problem:
    if graph is None:
        graph = build_graph(system.width, system.depth)
    n_b = system.baths
    m = system.matsubaras
    pss = np.zeros(graph.nodes * 2)
    pfs = np.zeros(n_b * 2)
    pfc = np.zeros(n_b * 2)
    cbk = np.zeros(n_b * m * 2)
    cbs = np.zeros(n_b * m)
    coup = np.ascontiguousarray(system.coupling.reshape(-1).astype(np.int32))
    lam = np.ascontiguousarray(system.lambda_)
    inv = np.ascontiguousarray(system.invnu)
    om = np.ascontiguousarray(system.omega)
    sy = _System(system.states, n_b, m, system.coupling.shape[1], coup.ctypes.data,
                 system.temperature, lam.ctypes.data, inv.ctypes.data, om.ctypes.data)
    g = _Graph()
    g.width = graph.width
    g.depth = graph.depth
    g.nodes = graph.nodes
    g.first_non_plus = graph.first_non_plus
    g.tuples = graph.tuples.ctypes.data_as(C.POINTER(C.c_int32))
    lib().ho_precompute_baths(C.byref(sy), C.byref(g), pss, pfs, pfc, cbk, cbs)
    h = np.empty(system.states * system.states * 2)
    hf = system.hamiltonian.reshape(-1)
    h[0::2] = hf.real
    h[1::2] = hf.imag
    if mask is None:
        mask = np.ones(graph.nodes, np.uint8)
    return Problem(system, graph, h, pss, pfs, pfc, cbk, cbs,
                   np.ascontiguousarray(np.asarray(mask, np.uint8)), coup)


# --------------------------------------------------------------------------
# derivative / propagation
# --------------------------------------------------------------------------

def derivative(prob: Problem, y: np.ndarray, threads=None) -> np.ndarray:
    out = np.zeros_like(y)
    ps = prob.cstruct()
    lib().ho_derivative(C.byref(ps), np.ascontiguousarray(y), out, threads or default_threads())
    return out


def derivative_ld(prob: Problem, y: np.ndarray, threads=None) -> np.ndarray:
    yl = np.ascontiguousarray(y.astype(np.longdouble))
    out = np.zeros_like(yl)
    ps = prob.cstruct()
    lib().ho_derivative_ld(C.byref(ps), yl.ctypes.data, out.ctypes.data, threads or default_threads())
    return out


def rk4_step(prob: Problem, h: float, y: np.ndarray, threads=None) -> np.ndarray:
    out = np.zeros_like(y)
    work = np.zeros(5 * y.size)
    ps = prob.cstruct()
    lib().ho_rk4_step(C.byref(ps), h, np.ascontiguousarray(y), out, work, threads or default_threads())
    return out


def propagate(prob: Problem, h: float, steps: int, observe_every: int, y=None, threads=None,
              long_double=False):
    """RK4 propagation; returns (final state, populations [rows, N])."""
    if y is None:
        y = prob.initial_state()
    y = np.ascontiguousarray(y.copy())
    rows = steps // observe_every + 1
    pops = np.zeros(rows * prob.states)
    fn = lib().ho_propagate_ld if long_double else lib().ho_propagate
    ps = prob.cstruct()
    got = fn(C.byref(ps), h, steps, observe_every, y, pops, threads or default_threads())
    if got < 0:
        raise RuntimeError("propagate failed")
    return y, pops[: got * prob.states].reshape(got, prob.states)


def ref_derivative(prob: Problem, y: np.ndarray, threads=None, mode=0, out_coeff=1.0,
                   acc=None, acc_coeff=1.0, acc_init=False, fast=False):
    """One call of the reference's own heom_ode kernel (compiled for the host).

    mode 0 = pure evaluation, 1 = NOMA_NUM_ODE_ACCUMULATE, 2 = NOMA_NUM_ODE_SUBDIAGONAL.
    Returns (out, acc)."""
    R = ref_lib(fast)
    if R is None:
        raise RuntimeError("reference kernels not built (oracle/_ref)")
    s = prob.system
    g = prob.graph
    out = np.zeros_like(y)
    accb = np.zeros_like(y) if acc is None else np.ascontiguousarray(acc.copy())
    rc = R.refcl_heom_ode(mode, s.states, s.matsubaras, s.coupling.shape[1], g.width, g.nodes,
                          g.first_non_plus, prob.coupling_flat, 0.0, out.ctypes.data, out_coeff,
                          accb.ctypes.data, acc_coeff, int(acc_init), np.ascontiguousarray(y),
                          prob.hamiltonian, np.ascontiguousarray(g.tuples.reshape(-1)),
                          np.ascontiguousarray(g.plus.reshape(-1)),
                          np.ascontiguousarray(g.minus.reshape(-1)), prob.pf_same_sum,
                          prob.pf_same, prob.pf_circ, prob.cbk, prob.cbk_sqrt, prob.mask,
                          threads or default_threads())
    if rc != 0:
        raise RuntimeError("refcl_heom_ode failed")
    return out, accb


def ref_weighted_add(prob: Problem, h, y, coeffs, ks, threads=None, fast=False):
    R = ref_lib(fast)
    out = np.zeros_like(y)
    c = np.ascontiguousarray(np.asarray(coeffs, np.float64))
    kp = (C.c_void_p * len(ks))(*[k.ctypes.data for k in ks])
    R.refcl_rk_weighted_add(prob.states, prob.graph.nodes, len(ks), h, out, y, c, kp,
                            threads or default_threads())
    return out


def ref_rk4_step(prob: Problem, h, y, threads=None, fast=False):
    """Classical RK4 step built from the reference's own kernels: pure heom_ode
    evaluations and rk_weighted_add for the stage inputs and the result
    (fast=True: the timing build of the same sources)."""
    k1, _ = ref_derivative(prob, y, threads, fast=fast)
    s = ref_weighted_add(prob, h, y, [0.5], [k1], threads, fast=fast)
    k2, _ = ref_derivative(prob, s, threads, fast=fast)
    s = ref_weighted_add(prob, h, y, [0.0, 0.5], [k1, k2], threads, fast=fast)
    k3, _ = ref_derivative(prob, s, threads, fast=fast)
    s = ref_weighted_add(prob, h, y, [0.0, 0.0, 1.0], [k1, k2, k3], threads, fast=fast)
    k4, _ = ref_derivative(prob, s, threads, fast=fast)
    return ref_weighted_add(prob, h, y, [1.0 / 6, 1.0 / 3, 1.0 / 3, 1.0 / 6], [k1, k2, k3, k4], threads,
                            fast=fast)


def populations(prob: Problem, y: np.ndarray) -> np.ndarray:
    n = prob.states
    return np.array([y[(n + 1) * 2 * i] for i in range(n)])


# --------------------------------------------------------------------------
# synthetic workloads (seeded; all configs of the benchmark plan)
# --------------------------------------------------------------------------

def synthetic_hamiltonian(n: int, seed: int, disorder_invcm: float = 0.0, rng=None):
    """Real-symmetric H in cm^-1: diagonal ~ U[12100, 12700], off-diagonal ~ N(0, 50)."""
    rng = np.random.default_rng(seed) if rng is None else rng
    h = np.zeros((n, n))
    diag = rng.uniform(12100.0, 12700.0, size=n)
    iu = np.triu_indices(n, 1)
    off = rng.normal(0.0, 50.0, size=len(iu[0]))
    h[iu] = off
    h = h + h.T
    h[np.diag_indices(n)] = diag
    if disorder_invcm:
        h[np.diag_indices(n)] += rng.normal(0.0, disorder_invcm, size=n)
    return h


def drude_system(n: int, depth: int, matsubaras: int, seed: int, temperature=300.0,
                 lam=35.0, invnu=50.0, h_invcm=None) -> System:
    h = synthetic_hamiltonian(n, seed) if h_invcm is None else h_invcm
    return make_system(h, [lam] * n, [invnu] * n, [0.0] * n, matsubaras, temperature, depth)
