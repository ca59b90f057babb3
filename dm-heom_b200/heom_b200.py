"""ctypes binding of the C ABI in include/heom_b200.h.

Used by the parity tests, the gradient-check harness and bench.py.  It loads
lib/libheom_b200.so from this directory and fails loudly when it is missing:
there is no CPU fallback.

The host-side arrays follow the reference layouts
(dm-heom/include/heom/instance.hpp:202-214): a hierarchy state is a float64
vector of length matrices * states * states * 2 (interleaved re/im, row-major
ADO tiles in uid order).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libheom_b200.so")

ORDER_LEX, ORDER_REFERENCE = 0, 1
RK4_REFERENCE, RK4_HORNER, RK4_PRODUCT = 0, 1, 2
SOLVE_PURE, SOLVE_ACCUMULATE, SOLVE_SUBDIAGONAL = 0, 1, 2
SCHEMES = {"reference": RK4_REFERENCE, "horner": RK4_HORNER, "product": RK4_PRODUCT}
ORDERS = {"lex": ORDER_LEX, "reference": ORDER_REFERENCE}

# every symbol declared in include/heom_b200.h
EXPORTS = [
    "heom_last_error", "heom_default_options", "heom_create", "heom_destroy",
    "heom_set_hamiltonian", "heom_set_mask", "heom_buffer_create", "heom_buffer_destroy",
    "heom_buffer_write", "heom_buffer_read", "heom_buffer_size_byte", "heom_solve",
    "heom_weighted_add", "heom_set_state", "heom_get_state", "heom_set_top", "heom_get_top",
    "heom_state_buffer", "heom_rk4_steps", "heom_propagate", "heom_rk4_steps_async",
    "heom_synchronize", "heom_stream", "heom_matrices", "heom_states", "heom_kernel_launches",
    "heom_tables_build", "heom_tables_view", "heom_tables_free", "heom_create_from_system",
    "heom_config_load", "heom_config_free", "heom_config_system", "heom_config_rho_init",
    "heom_config_get", "heom_tables_mask", "heom_rk4_steps_noalloc",
    "heom_create_batch", "heom_instances", "heom_instance_matrices", "heom_instance_offset",
    "heom_set_instance_hamiltonian", "heom_set_instance_top", "heom_get_instance_top",
    "heom_ensemble_footprint", "heom_ensemble_create", "heom_ensemble_destroy",
    "heom_ensemble_instances", "heom_ensemble_classes", "heom_ensemble_locate",
    "heom_ensemble_class", "heom_ensemble_set_hamiltonian", "heom_ensemble_set_top",
    "heom_ensemble_get_top", "heom_ensemble_autotune", "heom_ensemble_rk4_steps",
    "heom_ensemble_propagate", "heom_ensemble_top_row_len", "heom_ensemble_top_offset",
    "heom_ensemble_kernel_launches", "heom_ensemble_stream", "heom_ensemble_clear",
    "heom_adjoint_create", "heom_adjoint_destroy", "heom_adjoint_handle", "heom_adjoint_gradient",
    "heom_adjoint_kernel_launches", "heom_bath_derivatives", "heom_adjoint_create_batch",
    "heom_adjoint_instances", "heom_set_mask_compact", "heom_active_matrices", "heom_get_mask",
    "heom_hierarchy_norm", "heom_set_field", "heom_clear_field", "heom_set_time", "heom_time",
    "heom_set_flow_buffers", "heom_add_pre_evaluate_action", "heom_clear_pre_evaluate_actions",
    "heom_hierarchy_add", "heom_hierarchy_subtract", "heom_hierarchy_dot_product", "heom_hierarchy_scale",
    "heom_hierarchy_mmult_left", "heom_hierarchy_mmult_right", "heom_instance_write", "heom_instance_read",
    "heom_tables_state", "heom_adjoint_set_memory_limit", "heom_adjoint_recursive_slots",
    "heom_ensemble_adjoint_create", "heom_ensemble_adjoint_destroy", "heom_ensemble_adjoint_set_memory_limit",
    "heom_ensemble_adjoint_gradient", "heom_ensemble_adjoint_groups", "heom_ensemble_adjoint_group_of",
    "heom_ensemble_adjoint_offset", "heom_ensemble_adjoint_kernel_launches", "heom_buffer_hierarchy_norm",
]

PRE_EVALUATE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_void_p, C.c_void_p)


class HeomError(RuntimeError):
    pass


class InstanceDesc(C.Structure):
    _fields_ = [("states", C.c_int32), ("matsubaras", C.c_int32), ("baths", C.c_int32),
                ("baths_per_state", C.c_int32), ("ado_width", C.c_int32), ("ado_depth", C.c_int32),
                ("matrices", C.c_int64), ("first_non_plus_id", C.c_int32),
                ("baths_coupling", C.c_void_p), ("hamiltonian", C.c_void_p),
                ("ado_tuples", C.c_void_p), ("ado_plus", C.c_void_p), ("ado_minus", C.c_void_p),
                ("pf_same_sum", C.c_void_p), ("pf_same", C.c_void_p), ("pf_circ", C.c_void_p),
                ("cbk", C.c_void_p), ("cbk_sqrt", C.c_void_p)]


class SystemDesc(C.Structure):
    _fields_ = [("sites", C.c_int32), ("ado_depth", C.c_int32), ("hamiltonian", C.c_void_p),
                ("baths", C.c_int32), ("baths_max_per_site", C.c_int32),
                ("baths_coupling", C.c_void_p), ("lambda_", C.c_void_p), ("invnu", C.c_void_p),
                ("omega", C.c_void_p), ("matsubaras", C.c_int32), ("temperature", C.c_double)]


class Pulse(C.Structure):
    _fields_ = [("efield", C.c_double), ("time_center", C.c_double), ("time_width", C.c_double),
                ("frequency", C.c_double), ("phase", C.c_double)]


class Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("ado_order", C.c_int32), ("rk4_scheme", C.c_int32),
                ("use_graphs", C.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HeomError(f"CUDA library not built: {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.heom_last_error.restype = C.c_char_p
        L.heom_default_options.argtypes = [C.POINTER(Options)]
        L.heom_create.argtypes = [C.POINTER(InstanceDesc), C.POINTER(Options), C.POINTER(vp)]
        for name in ["heom_destroy", "heom_synchronize"]:
            getattr(L, name).argtypes = [vp]
        L.heom_set_hamiltonian.argtypes = [vp, vp]
        L.heom_set_mask.argtypes = [vp, vp]
        L.heom_set_mask_compact.argtypes = [vp, vp]
        L.heom_active_matrices.restype = i64
        L.heom_active_matrices.argtypes = [vp]
        L.heom_get_mask.argtypes = [vp, vp]
        L.heom_hierarchy_norm.argtypes = [vp, dbl, vp]
        L.heom_set_field.argtypes = [vp, vp, vp, C.POINTER(Pulse), C.POINTER(Pulse)]
        L.heom_clear_field.argtypes = [vp]
        L.heom_set_time.argtypes = [vp, dbl]
        L.heom_set_flow_buffers.argtypes = [vp, vp, vp]
        L.heom_buffer_hierarchy_norm.argtypes = [vp, vp, vp]
        L.heom_add_pre_evaluate_action.argtypes = [vp, PRE_EVALUATE_FN, vp]
        L.heom_clear_pre_evaluate_actions.argtypes = [vp]
        for name in ["heom_hierarchy_add", "heom_hierarchy_subtract", "heom_hierarchy_dot_product"]:
            getattr(L, name).argtypes = [vp, vp, vp, vp]
        L.heom_hierarchy_scale.argtypes = [vp, vp, dbl, dbl, vp]
        L.heom_hierarchy_mmult_left.argtypes = [vp, vp, vp, vp]
        L.heom_hierarchy_mmult_right.argtypes = [vp, vp, vp, vp]
        L.heom_time.restype = dbl
        L.heom_time.argtypes = [vp]
        L.heom_buffer_create.argtypes = [vp, C.POINTER(vp)]
        L.heom_buffer_destroy.argtypes = [vp]
        L.heom_buffer_write.argtypes = [vp, vp, vp]
        L.heom_buffer_read.argtypes = [vp, vp, vp]
        L.heom_buffer_size_byte.restype = C.c_size_t
        L.heom_buffer_size_byte.argtypes = [vp]
        L.heom_solve.argtypes = [vp, dbl, dbl, vp, vp, dbl, vp, dbl, C.c_int, C.c_int]
        L.heom_weighted_add.argtypes = [vp, C.c_int, dbl, vp, vp, vp, vp]
        for name in ["heom_set_state", "heom_get_state", "heom_set_top", "heom_get_top"]:
            getattr(L, name).argtypes = [vp, vp]
        L.heom_state_buffer.argtypes = [vp, C.POINTER(vp)]
        L.heom_rk4_steps.argtypes = [vp, dbl, i64]
        L.heom_rk4_steps_async.argtypes = [vp, dbl, i64]
        L.heom_propagate.argtypes = [vp, dbl, i64, i64, vp]
        L.heom_stream.restype = vp
        L.heom_stream.argtypes = [vp]
        L.heom_matrices.restype = i64
        L.heom_matrices.argtypes = [vp]
        L.heom_states.restype = i32
        L.heom_states.argtypes = [vp]
        L.heom_kernel_launches.restype = i64
        L.heom_kernel_launches.argtypes = [vp]
        L.heom_tables_build.argtypes = [C.POINTER(SystemDesc), C.POINTER(vp)]
        L.heom_tables_view.argtypes = [vp, C.POINTER(InstanceDesc)]
        L.heom_tables_free.argtypes = [vp]
        L.heom_instance_write.argtypes = [vp, vp, i32, dbl, C.c_char_p]
        L.heom_instance_read.argtypes = [C.c_char_p, vp, C.POINTER(vp)]
        L.heom_tables_state.argtypes = [vp, vp, C.POINTER(dbl)]
        L.heom_tables_free.restype = None
        L.heom_tables_mask.argtypes = [vp, C.c_char_p, i64, vp]
        L.heom_create_from_system.argtypes = [C.POINTER(SystemDesc), C.POINTER(Options), C.POINTER(vp)]
        L.heom_config_load.argtypes = [C.c_char_p, C.POINTER(vp)]
        L.heom_config_free.argtypes = [vp]
        L.heom_config_free.restype = None
        L.heom_config_system.argtypes = [vp, C.POINTER(SystemDesc)]
        L.heom_config_rho_init.argtypes = [vp, vp]
        L.heom_config_get.argtypes = [vp, C.c_char_p, C.c_char_p, C.c_size_t]
        L.heom_rk4_steps_noalloc.argtypes = [vp, vp, dbl, i64]
        L.heom_create_batch.argtypes = [C.POINTER(InstanceDesc), i32, C.POINTER(Options), C.POINTER(vp)]
        L.heom_instances.restype = i32
        L.heom_instances.argtypes = [vp]
        for name in ["heom_instance_matrices", "heom_instance_offset"]:
            getattr(L, name).restype = i64
            getattr(L, name).argtypes = [vp, i32]
        for name in ["heom_set_instance_hamiltonian", "heom_set_instance_top", "heom_get_instance_top",
                     "heom_ensemble_set_hamiltonian", "heom_ensemble_set_top", "heom_ensemble_get_top"]:
            getattr(L, name).argtypes = [vp, i32, vp]
        L.heom_ensemble_footprint.argtypes = [C.POINTER(InstanceDesc), i32, C.POINTER(Options),
                                              C.POINTER(C.c_size_t)]
        L.heom_ensemble_create.argtypes = [C.POINTER(InstanceDesc), i32, C.POINTER(Options), C.POINTER(vp)]
        L.heom_ensemble_destroy.argtypes = [vp]
        for name in ["heom_ensemble_instances", "heom_ensemble_classes"]:
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [vp]
        L.heom_ensemble_locate.argtypes = [vp, i32, C.POINTER(i32), C.POINTER(i32)]
        L.heom_ensemble_class.restype = vp
        L.heom_ensemble_class.argtypes = [vp, i32]
        L.heom_ensemble_autotune.argtypes = [vp, C.POINTER(dbl)]
        L.heom_ensemble_rk4_steps.argtypes = [vp, dbl, i64]
        L.heom_ensemble_propagate.argtypes = [vp, dbl, i64, i64, vp]
        L.heom_ensemble_top_row_len.restype = i64
        L.heom_ensemble_top_row_len.argtypes = [vp]
        L.heom_ensemble_top_offset.restype = i64
        L.heom_ensemble_top_offset.argtypes = [vp, i32]
        L.heom_ensemble_kernel_launches.restype = i64
        L.heom_ensemble_kernel_launches.argtypes = [vp]
        L.heom_ensemble_stream.restype = vp
        L.heom_ensemble_stream.argtypes = [vp]
        L.heom_ensemble_clear.argtypes = [vp]
        L.heom_adjoint_create.argtypes = [C.POINTER(SystemDesc), C.POINTER(Options), C.POINTER(vp)]
        L.heom_adjoint_destroy.argtypes = [vp]
        L.heom_adjoint_handle.restype = vp
        L.heom_adjoint_handle.argtypes = [vp]
        L.heom_adjoint_gradient.argtypes = [vp, vp, vp, vp, dbl, i64, vp, vp, vp, vp, vp]
        L.heom_adjoint_kernel_launches.restype = i64
        L.heom_adjoint_kernel_launches.argtypes = [vp]
        L.heom_bath_derivatives.argtypes = [C.POINTER(SystemDesc), i32, vp, vp, vp]
        L.heom_adjoint_create_batch.argtypes = [C.POINTER(SystemDesc), i32, C.POINTER(Options), C.POINTER(vp)]
        L.heom_adjoint_instances.restype = i32
        L.heom_adjoint_instances.argtypes = [vp]
        L.heom_adjoint_set_memory_limit.argtypes = [vp, i64]
        L.heom_adjoint_recursive_slots.restype = i64
        L.heom_adjoint_recursive_slots.argtypes = [vp]
        L.heom_ensemble_adjoint_create.argtypes = [C.POINTER(SystemDesc), i32, C.POINTER(Options), C.POINTER(vp)]
        L.heom_ensemble_adjoint_destroy.argtypes = [vp]
        L.heom_ensemble_adjoint_set_memory_limit.argtypes = [vp, i64]
        L.heom_ensemble_adjoint_gradient.argtypes = [vp, vp, vp, vp, dbl, i64, vp, vp, vp, vp, vp]
        L.heom_ensemble_adjoint_groups.restype = i32
        L.heom_ensemble_adjoint_groups.argtypes = [vp]
        L.heom_ensemble_adjoint_group_of.argtypes = [vp, i32, vp, vp]
        L.heom_ensemble_adjoint_offset.restype = i64
        L.heom_ensemble_adjoint_offset.argtypes = [vp, i32]
        L.heom_ensemble_adjoint_kernel_launches.restype = i64
        L.heom_ensemble_adjoint_kernel_launches.argtypes = [vp]
        _lib = L
    return _lib


def _need(ok, what):
    """Array sizes are checked before a pointer goes to the library (not with
    assert, which python -O removes)."""
    if not ok:
        raise ValueError(f"array size does not match the handle: {what}")


def _check(rc):
    if rc != 0:
        msg = lib().heom_last_error().decode(errors="replace")
        raise HeomError(f"heom error {rc}: {msg}")


def _ptr(a):
    return a.ctypes.data


class Buffer:
    def __init__(self, owner: "Heom"):
        self.owner = owner
        self.h = C.c_void_p()
        _check(lib().heom_buffer_create(owner.h, C.byref(self.h)))

    def write(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        _need(y.size == self.owner.state_len, "y.size == self.owner.state_len")
        _check(lib().heom_buffer_write(self.owner.h, self.h, _ptr(y)))

    def read(self):
        y = np.empty(self.owner.state_len)
        _check(lib().heom_buffer_read(self.owner.h, self.h, _ptr(y)))
        return y

    def close(self):
        if self.h:
            lib().heom_buffer_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


TABLE_KEYS = ("states", "matsubaras", "baths", "baths_per_state", "ado_width", "ado_depth", "matrices",
              "first_non_plus_id", "baths_coupling", "hamiltonian", "ado_tuples", "ado_plus", "ado_minus",
              "pf_same_sum", "pf_same", "pf_circ", "cbk", "cbk_sqrt")


def make_desc(tables: dict, keep: list) -> InstanceDesc:
    """InstanceDesc over numpy copies of the tables (kept alive in `keep`)."""
    def arr(a, dt):
        a = np.ascontiguousarray(np.asarray(a, dtype=dt).reshape(-1))
        keep.append(a)
        return a.ctypes.data

    t = tables
    return InstanceDesc(t["states"], t["matsubaras"], t["baths"], t["baths_per_state"], t["ado_width"],
                        t["ado_depth"], t["matrices"], t["first_non_plus_id"],
                        arr(t["baths_coupling"], np.int32), arr(t["hamiltonian"], np.float64),
                        arr(t["ado_tuples"], np.int32), arr(t["ado_plus"], np.int32),
                        arr(t["ado_minus"], np.int32), arr(t["pf_same_sum"], np.float64),
                        arr(t["pf_same"], np.float64), arr(t["pf_circ"], np.float64),
                        arr(t["cbk"], np.float64), arr(t["cbk_sqrt"], np.float64))


def make_options(device=0, order="lex", scheme="product", graphs=True) -> Options:
    o = Options()
    lib().heom_default_options(C.byref(o))
    o.device = device
    o.ado_order = ORDERS[order] if isinstance(order, str) else order
    o.rk4_scheme = SCHEMES[scheme] if isinstance(scheme, str) else scheme
    o.use_graphs = 1 if graphs else 0
    return o


class Heom:
    """Hierarchy instances on one GPU (a heom_handle): one instance, or a batch
    of instances that share states and baths (Heom.batch).  For a batch every
    state / top / Hamiltonian array holds the instances back to back."""

    def __init__(self, *, device=0, order="lex", scheme="product", graphs=True, _batch=None, **tables):
        keep = []
        tabs = _batch if _batch is not None else [tables]
        descs = (InstanceDesc * len(tabs))(*[make_desc(t, keep) for t in tabs])
        o = make_options(device, order, scheme, graphs)
        self.h = C.c_void_p()
        _check(lib().heom_create_batch(descs, len(tabs), C.byref(o), C.byref(self.h)))
        self.states = tabs[0]["states"]
        self.instances = len(tabs)
        self.instance_matrices = [int(t["matrices"]) for t in tabs]
        self.matrices = sum(self.instance_matrices)
        self.state_len = self.matrices * self.states * self.states * 2

    @classmethod
    def batch(cls, tables_list, **kw):
        """One handle over several instances (dicts of build_tables)."""
        return cls(_batch=list(tables_list), **kw)

    def instance_offset(self, k):
        """First ADO of instance k in the concatenated state."""
        return lib().heom_instance_offset(self.h, k)

    @staticmethod
    def tables_of(prob) -> dict:
        """Tables (reference layout) of a problem object with the attributes
        system, graph, hamiltonian, pf_* and cbk* (the test oracle's Problem)."""
        s = prob.system
        g = prob.graph
        return dict(states=s.states, matsubaras=s.matsubaras, baths=s.baths,
                    baths_per_state=s.coupling.shape[1], ado_width=g.width, ado_depth=g.depth,
                    matrices=g.nodes, first_non_plus_id=g.first_non_plus,
                    baths_coupling=prob.coupling_flat, hamiltonian=prob.hamiltonian,
                    ado_tuples=g.tuples, ado_plus=g.plus, ado_minus=g.minus,
                    pf_same_sum=prob.pf_same_sum, pf_same=prob.pf_same, pf_circ=prob.pf_circ,
                    cbk=prob.cbk, cbk_sqrt=prob.cbk_sqrt)

    @classmethod
    def from_problem(cls, prob, **kw):
        """Build from an oracle Problem (tables in reference layout)."""
        return cls(**cls.tables_of(prob), **kw)

    def close(self):
        if self.h:
            lib().heom_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- state ---------------------------------------------------------------
    def set_state(self, y):
        y = np.ascontiguousarray(y, dtype=np.float64)
        _need(y.size == self.state_len, "y.size == self.state_len")
        _check(lib().heom_set_state(self.h, _ptr(y)))

    def get_state(self):
        y = np.empty(self.state_len)
        _check(lib().heom_get_state(self.h, _ptr(y)))
        return y

    def set_top(self, top):
        top = np.ascontiguousarray(top, dtype=np.float64)
        _check(lib().heom_set_top(self.h, _ptr(top)))

    def get_top(self):
        t = np.empty(self.instances * self.states * self.states * 2)
        _check(lib().heom_get_top(self.h, _ptr(t)))
        return t

    def set_instance_top(self, k, top):
        top = np.ascontiguousarray(top, dtype=np.float64)
        _need(top.size == self.states * self.states * 2, "top.size == self.states * self.states * 2")
        _check(lib().heom_set_instance_top(self.h, k, _ptr(top)))

    def get_instance_top(self, k):
        t = np.empty(self.states * self.states * 2)
        _check(lib().heom_get_instance_top(self.h, k, _ptr(t)))
        return t

    def set_hamiltonian(self, ham):
        ham = np.ascontiguousarray(ham, dtype=np.float64)
        _need(ham.size == self.instances * self.states * self.states * 2, "ham.size == self.instances * self.states * self.states * 2")
        _check(lib().heom_set_hamiltonian(self.h, _ptr(ham)))

    def set_instance_hamiltonian(self, k, ham):
        ham = np.ascontiguousarray(ham, dtype=np.float64)
        _need(ham.size == self.states * self.states * 2, "ham.size == self.states * self.states * 2")
        _check(lib().heom_set_instance_hamiltonian(self.h, k, _ptr(ham)))

    def set_mask(self, mask, compact=False):
        """compact: masked ADOs are not swept (heom_set_mask_compact)."""
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        fn = lib().heom_set_mask_compact if compact else lib().heom_set_mask
        _check(fn(self.h, _ptr(mask)))

    def active_matrices(self):
        return lib().heom_active_matrices(self.h)

    def get_mask(self):
        m = np.zeros(self.matrices, np.uint8)
        _check(lib().heom_get_mask(self.h, _ptr(m)))
        return m

    def set_field(self, dipole_plus, dipole_minus, pump, probe):
        """Time-dependent H(t) = H - E(t) D- - conj(E(t)) D+ (SI; pump/probe:
        dicts or tuples of efield, time_center, time_width, frequency, phase)."""
        n = self.states
        dp = np.ascontiguousarray(np.asarray(dipole_plus, np.complex128).reshape(n, n)).view(np.float64)
        dm = np.ascontiguousarray(np.asarray(dipole_minus, np.complex128).reshape(n, n)).view(np.float64)
        mk = lambda x: Pulse(**x) if isinstance(x, dict) else Pulse(*x)
        _check(lib().heom_set_field(self.h, _ptr(dp), _ptr(dm), C.byref(mk(pump)), C.byref(mk(probe))))

    def clear_field(self):
        _check(lib().heom_clear_field(self.h))

    def set_time(self, t):
        _check(lib().heom_set_time(self.h, t))

    def time(self):
        return lib().heom_time(self.h)

    def hierarchy_norm(self, threshold=-1.0):
        """Per-ADO sum |sigma_ij|^2 (uid order); threshold >= 0 also filters the mask."""
        v = np.empty(self.matrices)
        _check(lib().heom_hierarchy_norm(self.h, threshold, _ptr(v)))
        return v

    # -- stepping ------------------------------------------------------------
    def rk4_steps(self, dt, steps):
        _check(lib().heom_rk4_steps(self.h, dt, steps))

    def rk4_steps_noalloc(self, d_state_ptr, dt, steps):
        """heom_rk4_steps_noalloc on a caller-owned device buffer (reference layout)."""
        _check(lib().heom_rk4_steps_noalloc(self.h, C.c_void_p(d_state_ptr), dt, steps))

    def rk4_steps_async(self, dt, steps):
        _check(lib().heom_rk4_steps_async(self.h, dt, steps))

    def synchronize(self):
        _check(lib().heom_synchronize(self.h))

    def propagate(self, dt, steps, observe_every):
        """Tops at every observation: [rows, states^2 * 2] for one instance,
        [rows, instances, states^2 * 2] for a batch."""
        rows = steps // observe_every + 1
        nn2 = self.states * self.states * 2
        tops = np.empty(rows * self.instances * nn2)
        _check(lib().heom_propagate(self.h, dt, steps, observe_every, _ptr(tops)))
        if self.instances == 1:
            return tops.reshape(rows, nn2)
        return tops.reshape(rows, self.instances, nn2)

    def populations_from_tops(self, tops):
        n = self.states
        return tops[..., [(n + 1) * 2 * i for i in range(n)]]

    def stream(self):
        return lib().heom_stream(self.h)

    def kernel_launches(self):
        return lib().heom_kernel_launches(self.h)

    # -- reference solve() interface -------------------------------------------
    def buffer(self):
        return Buffer(self)

    def solve(self, inb: Buffer, out: Buffer | None, mode=SOLVE_PURE, out_coeff=1.0,
              acc: Buffer | None = None, acc_coeff=1.0, acc_init=False, time=0.0, step_size=0.0):
        _check(lib().heom_solve(self.h, time, step_size, inb.h, out.h if out else None, out_coeff,
                                acc.h if acc else None, acc_coeff, int(acc_init), mode))

    def add_pre_evaluate_action(self, fn):
        """fn(handle, time, step_size) before every solve(); return 0 to continue."""
        cb = PRE_EVALUATE_FN(lambda user, h, t, dt, i, o: int(fn(self, t, dt) or 0))
        self._actions = getattr(self, "_actions", []) + [cb]  # keep the callbacks alive
        _check(lib().heom_add_pre_evaluate_action(self.h, cb, None))

    def clear_pre_evaluate_actions(self):
        _check(lib().heom_clear_pre_evaluate_actions(self.h))
        self._actions = []

    def hierarchy_op(self, op, a: Buffer, b: Buffer | None, out: Buffer, factor=1.0 + 0j, matrix=None):
        """op: add | subtract | dot_product | scale | mmult_left | mmult_right."""
        L = lib()
        if op in ("add", "subtract", "dot_product"):
            _check(getattr(L, "heom_hierarchy_" + op)(self.h, a.h, b.h, out.h))
        elif op == "scale":
            _check(L.heom_hierarchy_scale(self.h, a.h, float(np.real(factor)), float(np.imag(factor)), out.h))
        else:
            n = self.states
            m = np.ascontiguousarray(np.asarray(matrix, np.complex128).reshape(n, n)).view(np.float64)
            _check(getattr(L, "heom_hierarchy_" + op)(self.h, a.h, _ptr(m), out.h))

    def set_flow_buffers(self, above: Buffer | None, below: Buffer | None):
        _check(lib().heom_set_flow_buffers(self.h, above.h if above else None, below.h if below else None))

    def buffer_norm(self, b: Buffer):
        """Per-ADO sum |sigma_ij|^2 of a buffer (uid order)."""
        v = np.empty(self.matrices)
        _check(lib().heom_buffer_hierarchy_norm(self.h, b.h, _ptr(v)))
        return v

    def weighted_add(self, step, out: Buffer, y: Buffer, coeffs, ks):
        c = np.ascontiguousarray(np.asarray(coeffs, np.float64))
        kp = (C.c_void_p * max(1, len(ks)))(*[k.h.value for k in ks])
        _check(lib().heom_weighted_add(self.h, len(ks), step, out.h, y.h, _ptr(c), kp))


class Ensemble:
    """Instances of any sizes on one GPU (a heom_ensemble): grouped into
    classes of batch handles, one graph launch per RK4 step with the classes
    as concurrent branches, stage grids picked by the autotuner."""

    def __init__(self, tables_list, device=0, order="lex", scheme="product", graphs=True):
        keep = []
        tabs = list(tables_list)
        descs = (InstanceDesc * len(tabs))(*[make_desc(t, keep) for t in tabs])
        o = make_options(device, order, scheme, graphs)
        self.h = C.c_void_p()
        _check(lib().heom_ensemble_create(descs, len(tabs), C.byref(o), C.byref(self.h)))
        self.instances = len(tabs)
        self.states = [int(t["states"]) for t in tabs]
        self.row_len = lib().heom_ensemble_top_row_len(self.h)
        self.top_offsets = [lib().heom_ensemble_top_offset(self.h, k) for k in range(len(tabs))]

    @staticmethod
    def footprint(tables_list, scheme="product"):
        keep = []
        tabs = list(tables_list)
        descs = (InstanceDesc * len(tabs))(*[make_desc(t, keep) for t in tabs])
        o = make_options(0, "lex", scheme, True)
        b = C.c_size_t()
        _check(lib().heom_ensemble_footprint(descs, len(tabs), C.byref(o), C.byref(b)))
        return b.value

    def close(self):
        if self.h:
            lib().heom_ensemble_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def classes(self):
        return lib().heom_ensemble_classes(self.h)

    def locate(self, k):
        c, i = C.c_int32(), C.c_int32()
        _check(lib().heom_ensemble_locate(self.h, k, C.byref(c), C.byref(i)))
        return c.value, i.value

    def clear(self):
        """Zero every instance's hierarchy state (set the tops afterwards)."""
        _check(lib().heom_ensemble_clear(self.h))

    def set_top(self, k, top):
        top = np.ascontiguousarray(top, dtype=np.float64)
        _need(top.size == self.states[k] ** 2 * 2, "top.size == self.states[k] ** 2 * 2")
        _check(lib().heom_ensemble_set_top(self.h, k, _ptr(top)))

    def get_top(self, k):
        t = np.empty(self.states[k] ** 2 * 2)
        _check(lib().heom_ensemble_get_top(self.h, k, _ptr(t)))
        return t

    def set_hamiltonian(self, k, ham):
        ham = np.ascontiguousarray(ham, dtype=np.float64)
        _need(ham.size == self.states[k] ** 2 * 2, "ham.size == self.states[k] ** 2 * 2")
        _check(lib().heom_ensemble_set_hamiltonian(self.h, k, _ptr(ham)))

    def autotune(self):
        us = C.c_double()
        _check(lib().heom_ensemble_autotune(self.h, C.byref(us)))
        return us.value

    def rk4_steps(self, dt, steps):
        _check(lib().heom_ensemble_rk4_steps(self.h, dt, steps))

    def propagate(self, dt, steps, observe_every):
        """Per-instance tops: a list of [rows, states_k^2 * 2] arrays."""
        rows = steps // observe_every + 1
        buf = np.empty(rows * self.row_len)
        _check(lib().heom_ensemble_propagate(self.h, dt, steps, observe_every, _ptr(buf)))
        buf = buf.reshape(rows, self.row_len)
        return [buf[:, o:o + 2 * n * n].copy() for o, n in zip(self.top_offsets, self.states)]

    def populations(self, tops, k):
        n = self.states[k]
        return tops[:, [(n + 1) * 2 * i for i in range(n)]]

    def kernel_launches(self):
        return lib().heom_ensemble_kernel_launches(self.h)

    def stream(self):
        return lib().heom_ensemble_stream(self.h)


# --------------------------------------------------------------------------
# host set-up (graph, tables, config)
# --------------------------------------------------------------------------

class System:
    """A system in the reference's config units (cm^-1, fs, K)."""

    def __init__(self, hamiltonian, lambda_, invnu, omega, matsubaras, temperature, depth,
                 coupling=None):
        h = np.asarray(hamiltonian, dtype=np.complex128)
        self.sites = h.shape[0]
        self.depth = int(depth)
        self.h = np.empty(self.sites * self.sites * 2)
        self.h[0::2] = h.reshape(-1).real
        self.h[1::2] = h.reshape(-1).imag
        self.lambda_ = np.ascontiguousarray(np.asarray(lambda_, np.float64))
        self.invnu = np.ascontiguousarray(np.asarray(invnu, np.float64))
        self.omega = np.ascontiguousarray(np.asarray(omega, np.float64))
        self.baths = self.lambda_.size
        if coupling is None:
            coupling = np.arange(self.sites, dtype=np.int32).reshape(self.sites, 1)
        self.coupling = np.ascontiguousarray(np.asarray(coupling, np.int32))
        self.matsubaras = int(matsubaras)
        self.temperature = float(temperature)

    def desc(self):
        return SystemDesc(self.sites, self.depth, self.h.ctypes.data, self.baths,
                          self.coupling.shape[1], self.coupling.ctypes.data,
                          self.lambda_.ctypes.data, self.invnu.ctypes.data, self.omega.ctypes.data,
                          self.matsubaras, self.temperature)


def build_tables(system: System) -> dict:
    """Host tables built by the library (reference layouts), copied to numpy."""
    t = C.c_void_p()
    d = system.desc()
    _check(lib().heom_tables_build(C.byref(d), C.byref(t)))
    try:
        v = InstanceDesc()
        _check(lib().heom_tables_view(t, C.byref(v)))
        n, w, b, m, s = v.matrices, v.ado_width, v.baths, v.matsubaras, v.states

        def get(ptr, count, ct, dt):
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).astype(dt).copy()

        out = dict(states=s, matsubaras=m, baths=b, baths_per_state=v.baths_per_state,
                   ado_width=w, ado_depth=v.ado_depth, matrices=n,
                   first_non_plus_id=v.first_non_plus_id,
                   baths_coupling=get(v.baths_coupling, s * v.baths_per_state, C.c_int32, np.int32),
                   hamiltonian=get(v.hamiltonian, s * s * 2, C.c_double, np.float64),
                   ado_tuples=get(v.ado_tuples, n * w, C.c_int32, np.int32),
                   ado_plus=get(v.ado_plus, n * w, C.c_int32, np.int32),
                   ado_minus=get(v.ado_minus, n * w, C.c_int32, np.int32),
                   pf_same_sum=get(v.pf_same_sum, n * 2, C.c_double, np.float64),
                   pf_same=get(v.pf_same, b * 2, C.c_double, np.float64),
                   pf_circ=get(v.pf_circ, b * 2, C.c_double, np.float64),
                   cbk=get(v.cbk, b * m * 2, C.c_double, np.float64),
                   cbk_sqrt=get(v.cbk_sqrt, b * m, C.c_double, np.float64))
        return out
    finally:
        lib().heom_tables_free(t)


def bath_derivatives(system: System, theta: int):
    """d(pf_same, pf_circ, cbk)/d theta, theta 0 = lambda of every bath (per J),
    1 = gamma = 1/invnu of every bath (per 1/s); SI tables as build_tables."""
    d = system.desc()
    b, m = system.baths, system.matsubaras
    ps, pc, cb = np.zeros(2 * b), np.zeros(2 * b), np.zeros(2 * b * m)
    _check(lib().heom_bath_derivatives(C.byref(d), theta, _ptr(ps), _ptr(pc), _ptr(cb)))
    return ps, pc, cb


class Adjoint:
    """Adjoint gradients of a time-integrated observable (heom_adjoint_*):
    J = sum_n weights[n] Re(sum_ij conj(O_ij) rho_n(i,j)).  Given a list of
    systems (shared states and baths) it sweeps the whole batch at once and
    returns per-instance results with a leading instance axis."""

    def __init__(self, system, device=0, graphs=True):
        self.batch = isinstance(system, (list, tuple))
        systems = list(system) if self.batch else [system]
        self.systems = systems
        ds = (SystemDesc * len(systems))(*[x.desc() for x in systems])
        o = make_options(device, "lex", "product", graphs)
        self.h = C.c_void_p()
        _check(lib().heom_adjoint_create_batch(ds, len(systems), C.byref(o), C.byref(self.h)))
        self.states = systems[0].sites
        self.instances = len(systems)

    def gradient(self, rho0, observable, weights, dt, steps, outputs=("h", "lambda", "gamma", "rho0")):
        """Loss and gradients; `outputs` names the gradients to compute (the
        others are skipped by the sweep and returned as None)."""
        n, K = self.states, self.instances

        def per_instance(a):
            a = np.asarray(a, np.complex128)
            if a.size == n * n:
                a = np.broadcast_to(a.reshape(1, n, n), (K, n, n))
            return np.ascontiguousarray(a.reshape(K, n, n)).view(np.float64).reshape(-1)

        rho0 = per_instance(rho0)
        obs = per_instance(observable)
        w = np.ascontiguousarray(np.asarray(weights, np.float64))
        _need(w.size == steps + 1, "w.size == steps + 1")
        loss, gl, gg = np.zeros(K), np.zeros(K), np.zeros(K)
        gh = np.zeros(2 * K * n * n)
        gr = np.zeros(2 * K * n * n)
        def opt(name, a):
            return _ptr(a) if name in outputs else None
        _check(lib().heom_adjoint_gradient(self.h, _ptr(rho0), _ptr(obs), _ptr(w), dt, steps, _ptr(loss),
                                           opt("h", gh), opt("lambda", gl), opt("gamma", gg), opt("rho0", gr)))
        out = {"loss": loss, "h": gh.view(np.complex128).reshape(K, n, n),  # dJ/dRe H + i dJ/dIm H, per cm^-1
               "lambda": gl, "gamma": gg, "rho0": gr.view(np.complex128).reshape(K, n, n)}
        out = {k: (v if k == "loss" or k in outputs else None) for k, v in out.items()}
        if not self.batch:
            out = {k: (None if v is None else v[0] if k not in ("loss", "lambda", "gamma") else float(v[0]))
                   for k, v in out.items()}
        return out

    def kernel_launches(self):
        return lib().heom_adjoint_kernel_launches(self.h)

    def set_memory_limit(self, nbytes):
        """Device bytes the sweep may hold for its states (0: free memory)."""
        _check(lib().heom_adjoint_set_memory_limit(self.h, int(nbytes)))

    def recursive_slots(self):
        """Slots of the last sweep's recursive checkpointing (0: sqrt layout)."""
        return lib().heom_adjoint_recursive_slots(self.h)

    def close(self):
        if self.h:
            lib().heom_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class EnsembleAdjoint:
    """Adjoint gradients for systems of any sizes (heom_ensemble_adjoint_*):
    the library groups them into batch adjoints by class and memory and
    sweeps the groups one after another.  rho0 / observable: one (n, n)
    matrix for all instances or a list of per-instance matrices; results are
    per-instance lists (matrices) and arrays (loss, lambda, gamma)."""

    def __init__(self, systems, device=0, graphs=True):
        self.systems = list(systems)
        ds = (SystemDesc * len(self.systems))(*[x.desc() for x in self.systems])
        o = make_options(device, "lex", "product", graphs)
        self.h = C.c_void_p()
        _check(lib().heom_ensemble_adjoint_create(ds, len(self.systems), C.byref(o), C.byref(self.h)))
        self.instances = len(self.systems)
        self.offsets = [lib().heom_ensemble_adjoint_offset(self.h, k) for k in range(self.instances + 1)]

    def set_memory_limit(self, nbytes):
        _check(lib().heom_ensemble_adjoint_set_memory_limit(self.h, int(nbytes)))

    def _pack(self, mats):
        out = np.zeros(2 * self.offsets[-1])
        for k, sysd in enumerate(self.systems):
            n = sysd.sites
            m = mats[k] if isinstance(mats, (list, tuple)) else mats
            m = np.asarray(m, np.complex128).reshape(n, n)
            out[2 * self.offsets[k]:2 * self.offsets[k + 1]] = m.reshape(-1).view(np.float64)
        return out

    def _unpack(self, flat):
        res = []
        for k, sysd in enumerate(self.systems):
            n = sysd.sites
            res.append(flat[2 * self.offsets[k]:2 * self.offsets[k + 1]].view(np.complex128).reshape(n, n).copy())
        return res

    def gradient(self, rho0, observable, weights, dt, steps, outputs=("h", "lambda", "gamma", "rho0")):
        K = self.instances
        r0, ob = self._pack(rho0), self._pack(observable)
        w = np.ascontiguousarray(np.asarray(weights, np.float64))
        _need(w.size == steps + 1, "w.size == steps + 1")
        loss, gl, gg = np.zeros(K), np.zeros(K), np.zeros(K)
        gh, gr = np.zeros(2 * self.offsets[-1]), np.zeros(2 * self.offsets[-1])

        def opt(name, a):
            return _ptr(a) if name in outputs else None
        _check(lib().heom_ensemble_adjoint_gradient(self.h, _ptr(r0), _ptr(ob), _ptr(w), dt, steps, _ptr(loss),
                                                    opt("h", gh), opt("lambda", gl), opt("gamma", gg),
                                                    opt("rho0", gr)))
        return {"loss": loss,
                "h": self._unpack(gh) if "h" in outputs else None,
                "lambda": gl if "lambda" in outputs else None,
                "gamma": gg if "gamma" in outputs else None,
                "rho0": self._unpack(gr) if "rho0" in outputs else None}

    def groups(self):
        """(group, recursive-checkpointing slots) of every instance in the last call."""
        out = []
        for k in range(self.instances):
            g, sl = C.c_int32(), C.c_int64()
            _check(lib().heom_ensemble_adjoint_group_of(self.h, k, C.byref(g), C.byref(sl)))
            out.append((g.value, sl.value))
        return out

    def kernel_launches(self):
        return lib().heom_ensemble_adjoint_kernel_launches(self.h)

    def close(self):
        if self.h:
            lib().heom_ensemble_adjoint_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def shard_instances(sizes, world, rank):
    """Instances of rank `rank` when independent instances are spread over
    `world` GPUs: greedy by bytes, largest first (no data exchange)."""
    load = [0] * world
    mine = []
    for k in sorted(range(len(sizes)), key=lambda q: -sizes[q]):
        r = min(range(world), key=lambda q: load[q])
        load[r] += sizes[k]
        if r == rank:
            mine.append(k)
    return sorted(mine)


def reduce_throughput(dist, ados_steps, secs, device):
    """Whole-job ADO-updates and the slowest rank's time of a sharded run: one
    sum and one max all-reduce (the only collectives of a sharded ensemble)."""
    import torch
    a = torch.tensor([float(ados_steps)], dtype=torch.float64, device=device)
    t = torch.tensor([float(secs)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(a)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(a.item()), float(t.item())


def trapezoid_weights(steps, dt_fs):
    """Weights of the trapezoid rule over t_n = n dt (fs), n = 0..steps."""
    w = np.full(steps + 1, float(dt_fs))
    w[0] = w[-1] = 0.5 * dt_fs
    return w


def _tables_dict(t):
    v = InstanceDesc()
    _check(lib().heom_tables_view(t, C.byref(v)))
    n, w, b, m, s = v.matrices, v.ado_width, v.baths, v.matsubaras, v.states

    def get(ptr, count, ct, dt):
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ct)), shape=(count,)).astype(dt).copy()

    return dict(states=s, matsubaras=m, baths=b, baths_per_state=v.baths_per_state,
                ado_width=w, ado_depth=v.ado_depth, matrices=n, first_non_plus_id=v.first_non_plus_id,
                baths_coupling=get(v.baths_coupling, s * v.baths_per_state, C.c_int32, np.int32),
                hamiltonian=get(v.hamiltonian, s * s * 2, C.c_double, np.float64),
                ado_tuples=get(v.ado_tuples, n * w, C.c_int32, np.int32),
                ado_plus=get(v.ado_plus, n * w, C.c_int32, np.int32),
                ado_minus=get(v.ado_minus, n * w, C.c_int32, np.int32),
                pf_same_sum=get(v.pf_same_sum, n * 2, C.c_double, np.float64),
                pf_same=get(v.pf_same, b * 2, C.c_double, np.float64),
                pf_circ=get(v.pf_circ, b * 2, C.c_double, np.float64),
                cbk=get(v.cbk, b * m * 2, C.c_double, np.float64),
                cbk_sqrt=get(v.cbk_sqrt, b * m, C.c_double, np.float64))


def write_instance(system: System, path, state=None, top_only=False, time=0.0):
    """The reference's binary instance file of a system (and a state)."""
    t = C.c_void_p()
    d = system.desc()
    _check(lib().heom_tables_build(C.byref(d), C.byref(t)))
    try:
        st = None if state is None else np.ascontiguousarray(state, np.float64)
        _check(lib().heom_instance_write(t, _ptr(st) if st is not None else None, int(top_only), time,
                                         str(path).encode()))
    finally:
        lib().heom_tables_free(t)


def read_instance(path, coupling=None):
    """(tables dict, state, time) of a reference instance file."""
    t = C.c_void_p()
    cp = None if coupling is None else np.ascontiguousarray(np.asarray(coupling, np.int32).reshape(-1))
    _check(lib().heom_instance_read(str(path).encode(), _ptr(cp) if cp is not None else None, C.byref(t)))
    try:
        tabs = _tables_dict(t)
        state = np.empty(tabs["matrices"] * tabs["states"] ** 2 * 2)
        tm = C.c_double()
        _check(lib().heom_tables_state(t, _ptr(state), C.byref(tm)))
        return tabs, state, tm.value
    finally:
        lib().heom_tables_free(t)


def tables_mask(system: System, strategy="none", first_layer=-1):
    t = C.c_void_p()
    d = system.desc()
    _check(lib().heom_tables_build(C.byref(d), C.byref(t)))
    try:
        v = InstanceDesc()
        _check(lib().heom_tables_view(t, C.byref(v)))
        mask = np.zeros(v.matrices, np.uint8)
        _check(lib().heom_tables_mask(t, strategy.encode(), first_layer, mask.ctypes.data))
        return mask
    finally:
        lib().heom_tables_free(t)


def from_system(system: System, **kw) -> Heom:
    """Build the tables with the library's host code and create a handle."""
    return Heom(**build_tables(system), **kw)


class Config:
    """A parsed population_dynamics or linear_absorption .cfg file (heom_config_*)."""

    def __init__(self, path):
        self.h = C.c_void_p()
        _check(lib().heom_config_load(str(path).encode(), C.byref(self.h)))

    def get(self, key):
        buf = C.create_string_buffer(1 << 16)
        _check(lib().heom_config_get(self.h, key.encode(), buf, len(buf)))
        return buf.value.decode()

    def system_desc(self):
        d = SystemDesc()
        _check(lib().heom_config_system(self.h, C.byref(d)))
        return d

    def rho_init(self):
        d = self.system_desc()
        out = np.zeros(d.sites * d.sites * 2)
        _check(lib().heom_config_rho_init(self.h, out.ctypes.data))
        return out

    def close(self):
        if self.h:
            lib().heom_config_free(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
