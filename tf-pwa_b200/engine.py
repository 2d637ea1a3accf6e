"""Python side of the engine: ctypes binding of ``libpwa_b200.so``, the
per-evaluation constant block, and the chain rule from the kernel's FP64
sums to the NLL and its gradient.

NLL (``tf_pwa/model/model.py:407-449``)::

    NLL = -sum_data w clip_log(f) + (sum_data w) * ln( sum_MC w~ f )

with data weights alpha-scaled (``model.py:603-641``) and MC weights
normalised to 1 (``model.py:1155-1161``).  The kernel returns, per event set,
S0 = sum w t(f), Gk = sum fac * G_k and the lineshape sums; the derivative of
f with respect to a real parameter theta is

    df/dtheta = 2 Re sum_k J_k(theta) G_k + (lineshape term),

J_k = dc_k/dtheta + c_k * kappa_k(theta), c_k the product of the column's
complex couplings (chain total and one g_ls per vertex) and kappa_k the
derivative of the column's log barrier factors through q0 (nominal masses).
"""
import cmath
import ctypes
import os

import numpy as np

from .codegen import ModelCode
from .particles import bprime_coeff

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpwa_b200.so")

PLAIN_F64 = 0
MIXED_F32 = 1

# Compiled model modules are kept on disk across processes: in the directory
# PWA_CUBIN_CACHE names when it is set (set and empty: no disk cache), else in
# the package's own _cubins directory, where the build step stores the
# shipped models ahead of time (Engine.precompile).
CUBIN_DIR = os.path.join(HERE, "_cubins")

_lib = None


def _default_cubin_cache():
    if "PWA_CUBIN_CACHE" in os.environ:
        return
    try:
        os.makedirs(CUBIN_DIR, exist_ok=True)
    except OSError:
        return
    if os.access(CUBIN_DIR, os.W_OK | os.X_OK):
        os.environ["PWA_CUBIN_CACHE"] = CUBIN_DIR


def load_library(path=LIB_PATH):
    """Load the native library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    _default_cubin_cache()
    if not os.path.exists(path):
        raise RuntimeError(
            f"{path} not found: build it first (python -c 'import __graft_entry__ as g; g.build()')")
    lib = ctypes.CDLL(path)
    vp, cp, i, ll, dp, sz = (ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_longlong,
                             ctypes.POINTER(ctypes.c_double), ctypes.c_size_t)
    lib.pwa_plan_create.argtypes = [cp, sz, i, i, i, i, i, i, i, i, ctypes.POINTER(vp)]
    ip = ctypes.POINTER(ctypes.c_int)
    lib.pwa_cache_data.argtypes = [vp, dp, vp]
    lib.pwa_eval_cached_enqueue.argtypes = [vp, dp, vp]
    lib.pwa_set_param_layout.argtypes = [vp, i, i, ip, ip, ip, i, ip, i, ip]
    lib.pwa_pieces_cached.argtypes = [vp, dp, ctypes.c_double, ctypes.c_double, vp, dp]
    lib.pwa_nll_grad_cached.argtypes = [vp, vp, ctypes.c_double, vp, vp, vp]
    lib.pwa_set_cached_variant.argtypes = [vp, i]
    lib.pwa_set_gram_method.argtypes = [vp, i]
    lib.pwa_wait_check.argtypes = [vp, i, ctypes.c_uint, ctypes.c_double, vp]
    lib.pwa_fma_peak.argtypes = [vp, i, ll, vp, dp]
    lib.pwa_pieces_points.argtypes = [vp, i, dp, ctypes.c_double, ctypes.c_double, vp, dp]
    lib.pwa_autotune_cached.argtypes = [vp, dp, i, vp, ip, dp]
    lib.pwa_cached_config.argtypes = [vp, ip]
    lib.pwa_set_cached_config.argtypes = [vp, i, i, i]
    llp = ctypes.POINTER(ll)
    lib.pwa_pool_reserve.argtypes = [vp, ll]
    lib.pwa_pool_alloc.argtypes = [vp, ll, llp, llp]
    lib.pwa_pool_free.argtypes = [vp, ll]
    lib.pwa_pool_fill.argtypes = [vp, ll, dp, vp, vp, vp, ll, ll, vp]
    lib.pwa_pieces_multi.argtypes = [vp, i, llp, llp, dp, dp, ctypes.c_double, vp, dp]
    lib.pwa_eval_noalloc.argtypes = [vp, dp, vp, vp, vp, ll, ll, ll, vp, vp]
    ull = ctypes.c_ulonglong
    lib.pwa_fields_from_p4.argtypes = [vp, vp, ll, ll, vp, ll, vp]
    lib.pwa_toy_select.argtypes = [vp, dp, ull, ll, ll, ctypes.c_double, i, vp, vp]
    lib.pwa_toy_fields.argtypes = [vp, ull, vp, ll, vp, ll, vp, ll, vp]
    lib.pwa_hessian_cached.argtypes = [vp, dp, ctypes.c_double, ctypes.c_double, vp, dp, dp, dp]
    lib.pwa_hessian_cached_exact.argtypes = [vp, dp, ctypes.c_double, vp, dp, dp, dp]
    lib.pwa_hess_sums_cached.argtypes = [vp, dp, vp, dp]
    lib.pwa_shape_cache.argtypes = [vp, dp, vp]
    lib.pwa_eval_shapecache.argtypes = [vp, dp, dp, vp, dp]
    lib.pwa_eval_shapecache_enqueue.argtypes = [vp, dp, dp, vp]
    lib.pwa_read_dat.argtypes = [cp, vp, ll, ctypes.POINTER(ll)]
    lib.pwa_hostprog_create.argtypes = [ip, ll, dp, ll, ctypes.POINTER(vp)]
    lib.pwa_hostprog_destroy.argtypes = [vp]
    lib.pwa_hostprog_consts.argtypes = [vp, dp, dp]
    lib.pwa_hostprog_jacobian.argtypes = [vp, dp, dp, dp, dp]
    lib.pwa_hostprog_pieces.argtypes = [vp, dp, dp, dp, ctypes.c_double, ctypes.c_double, dp]
    lib.pwa_hostprog_column_rho.argtypes = [vp, dp, dp]
    lib.pwa_set_host_program.argtypes = [vp, vp]
    lib.pwa_pieces_vars.argtypes = [vp, vp, i, ctypes.c_double, ctypes.c_double, vp, vp]
    lib.pwa_nll_grad_vars.argtypes = [vp, vp, i, ctypes.c_double, vp, vp, vp]
    lib.pwa_server_create.argtypes = [vp, dp, dp, i, ctypes.c_double, i, ctypes.POINTER(vp)]
    lib.pwa_server_submit.argtypes = [vp, dp, vp, vp, vp, ll, ll, ctypes.POINTER(ll)]
    ip_ = ctypes.POINTER(ctypes.c_int)
    lib.pwa_server_result.argtypes = [vp, ll, i, ip_, dp, dp, ip_, ip_, dp]
    lib.pwa_server_stats.argtypes = [vp, dp]
    lib.pwa_server_tuning.argtypes = [vp, dp]
    lib.pwa_server_destroy.argtypes = [vp]
    lib.pwa_plan_destroy.argtypes = [vp]
    lib.pwa_compile_only.argtypes = [cp, sz, i, cp, cp, sz]
    lib.pwa_precompile.argtypes = [cp, sz, i, cp, cp, sz]
    lib.pwa_upload_events.argtypes = [vp, vp, vp, vp, ll, ll, i, vp]
    lib.pwa_eval.argtypes = [vp, dp, i, i, vp, dp]
    lib.pwa_eval_enqueue.argtypes = [vp, dp, i, i, vp]
    lib.pwa_eval_pdf.argtypes = [vp, dp, i, ll, ll, vp, vp]
    lib.pwa_build_gram.argtypes = [vp, dp, vp, dp]
    lib.pwa_plan_info.argtypes = [vp, ctypes.POINTER(ll)]
    lib.pwa_last_error.argtypes = [vp]
    lib.pwa_last_error.restype = cp
    for f in EXPORTED:
        if f == "pwa_last_error":
            continue
        getattr(lib, f).restype = i
    _lib = lib
    return lib


EXPORTED = ("pwa_plan_create", "pwa_plan_destroy", "pwa_compile_only", "pwa_precompile",
            "pwa_upload_events",
            "pwa_eval", "pwa_eval_enqueue", "pwa_eval_pdf", "pwa_build_gram", "pwa_cache_data",
            "pwa_eval_cached_enqueue", "pwa_set_param_layout", "pwa_pieces_cached",
            "pwa_nll_grad_cached", "pwa_set_cached_variant", "pwa_pool_reserve",
            "pwa_pool_alloc", "pwa_pool_free", "pwa_pool_fill", "pwa_pieces_multi",
            "pwa_eval_noalloc", "pwa_fields_from_p4", "pwa_toy_select", "pwa_toy_fields",
            "pwa_hessian_cached", "pwa_hessian_cached_exact", "pwa_hess_sums_cached",
            "pwa_shape_cache", "pwa_eval_shapecache", "pwa_eval_shapecache_enqueue",
            "pwa_read_dat", "pwa_hostprog_create", "pwa_hostprog_destroy",
            "pwa_hostprog_consts", "pwa_hostprog_jacobian", "pwa_hostprog_pieces",
            "pwa_hostprog_column_rho", "pwa_set_host_program", "pwa_pieces_vars",
            "pwa_nll_grad_vars", "pwa_server_create", "pwa_server_submit",
            "pwa_server_result", "pwa_server_stats", "pwa_server_destroy",
            "pwa_plan_info", "pwa_last_error")


class PWAError(RuntimeError):
    pass


HOSTPROG_MAGIC = 0x50574850
FORM_PLAIN_F64, FORM_MIXED_F32, FORM_SHAPE_CACHE = 0, 1, 2


class HostProgram:
    """A host program (pwa_hostprog_*): the constant block, the Jacobian of
    the column couplings and the chain rule of one model and variable
    layout in native code, from the flat arrays of
    :meth:`Engine.host_program_arrays`.  Needs no device."""

    def __init__(self, ip, dp, ncol, nconst, nshape, n_train, n_cpc=0):
        self.ip = np.ascontiguousarray(ip, np.int32)
        self.dp = np.ascontiguousarray(dp, np.float64)
        self.ncol, self.nconst, self.nshape, self.n_train = ncol, nconst, nshape, n_train
        self.n_cpc = n_cpc
        lib = load_library()
        h = ctypes.c_void_p()
        rc = lib.pwa_hostprog_create(self.ip.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     len(self.ip), _dptr(self.dp), len(self.dp), ctypes.byref(h))
        if rc:
            raise PWAError(f"pwa_hostprog_create failed ({rc}): "
                           f"{lib.pwa_last_error(None).decode()}")
        self.h = h

    def _check(self, rc, what):
        if rc:
            raise PWAError(f"{what} failed ({rc}): {load_library().pwa_last_error(None).decode()}")

    def consts(self, var_values):
        v = np.ascontiguousarray(var_values, np.float64)
        out = np.zeros(self.nconst)
        self._check(load_library().pwa_hostprog_consts(self.h, _dptr(v), _dptr(out)),
                    "pwa_hostprog_consts")
        return out

    def jacobian(self, var_values):
        """(J, D, Jm): column-coupling Jacobian (n_train x ncol), selectors
        of the extra sums (n_train x nshape), charge -1 Jacobian of the CP
        columns (n_train x n_cpc)."""
        v = np.ascontiguousarray(var_values, np.float64)
        J = np.zeros(2 * self.n_train * self.ncol)
        D = np.zeros(max(self.n_train * self.nshape, 1))
        Jm = np.zeros(max(2 * self.n_train * self.n_cpc, 1))
        self._check(load_library().pwa_hostprog_jacobian(self.h, _dptr(v), _dptr(J), _dptr(D),
                                                         _dptr(Jm)), "pwa_hostprog_jacobian")
        J = (J[0::2] + 1j * J[1::2]).reshape(self.n_train, self.ncol)
        Jm = (Jm[0::2] + 1j * Jm[1::2])[:self.n_train * self.n_cpc].reshape(self.n_train,
                                                                            self.n_cpc)
        return J, D[:self.n_train * self.nshape].reshape(self.n_train, self.nshape), Jm

    def pieces(self, var_values, sd, sm, sw, mc_share=1.0):
        v = np.ascontiguousarray(var_values, np.float64)
        sd = np.ascontiguousarray(sd, np.float64)
        sm = np.ascontiguousarray(sm, np.float64)
        out = np.zeros(3 + 2 * self.n_train)
        self._check(load_library().pwa_hostprog_pieces(self.h, _dptr(v), _dptr(sd), _dptr(sm),
                                                       float(sw), float(mc_share), _dptr(out)),
                    "pwa_hostprog_pieces")
        return out

    def column_rho(self, C):
        C = np.ascontiguousarray(C, np.float64)
        out = np.zeros(self.ncol)
        self._check(load_library().pwa_hostprog_column_rho(self.h, _dptr(C), _dptr(out)),
                    "pwa_hostprog_column_rho")
        return out

    def close(self):
        if getattr(self, "h", None):
            load_library().pwa_hostprog_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


# ----------------------------------------------------------- host formulae
def rel_p2(m0, m1, m2):
    s, d = m1 + m2, m1 - m2
    return (m0 - s) * (m0 + s) * (m0 - d) * (m0 + d) / (2 * m0) ** 2


def rel_p(m0, m1, m2):
    s, d = m1 + m2, m1 - m2
    me = m0 if np.real(m0) > np.real(s) else s
    p = (me - s) * (me + s) * (me - d) * (me + d)
    return np.sqrt(p) / (2 * me)


def poly(l, z):
    r = 0.0
    for c in bprime_coeff(l):
        r = r * z + c
    return r


def density_matrix(J, p):
    """(rho, [d rho / d p_k]) of a vector-polarised parent
    (``tf_pwa/amp/core.py:1965-2000``): spin 1/2, rho = (1 + p . sigma) / 2;
    spin 1, rho = 1 + sum_k p_k G_k with the eight Hermitian generators G_k
    of the reference (in the parent's helicity order)."""
    p = np.asarray(p, np.float64)
    if J == 0.5:
        px, py, pz = p
        rho = 0.5 * np.array([[1 + pz, px - 1j * py], [px + 1j * py, 1 - pz]])
        d = [0.5 * np.array([[0, 1], [1, 0]], complex),
             0.5 * np.array([[0, -1j], [1j, 0]]),
             0.5 * np.array([[1, 0], [0, -1]], complex)]
        return rho, d
    if J == 1:
        s3 = 1.0 / np.sqrt(3.0)
        G = np.zeros((8, 3, 3), complex)
        G[0][0, 1], G[0][1, 0] = 1, 1
        G[1][0, 1], G[1][1, 0] = -1j, 1j
        G[2][0, 0], G[2][1, 1] = 1, -1
        G[3][0, 2], G[3][2, 0] = 1, 1
        G[4][0, 2], G[4][2, 0] = -1j, 1j
        G[5][1, 2], G[5][2, 1] = 1, 1
        G[6][1, 2], G[6][2, 1] = -1j, 1j
        G[7] = np.diag([s3, s3, -2 * s3])
        return np.eye(3) + np.tensordot(p, G, 1), list(G)
    raise NotImplementedError("vector polarisation of a parent with spin other than 1/2 or 1")


def combine_pieces(vec, P):
    """NLL and gradient from the summed piece vector of
    :meth:`Engine.local_pieces` (model.py:433-449):
    NLL = -S_d + sw ln S_m, grad = -g_d + sw g_m / S_m."""
    vec = np.asarray(vec, np.float64)
    sd, sm, sw = vec[0], vec[1], vec[2]
    gd, gm = vec[3:3 + P], vec[3 + P:3 + 2 * P]
    return float(-sd + sw * np.log(sm)), -gd + sw * gm / sm


class Engine:
    """A compiled model bound to a device: events, constants, evaluation."""

    def __init__(self, group, plan, vm, tpb=128, compile=True, order=None):
        self.group = group
        self.plan = plan
        self.vm = vm
        self.code = ModelCode(group, plan, order)
        self.src = self.code.source()
        self.tpb = tpb
        self.h = None
        self._n_data = self._n_mc = 0
        self._sw = None
        self._gram = None
        self.mc_share = 1.0      # this device's fraction of the total MC weight
        self.use_shape_cache = False  # evaluations from the floating-shape column cache
        self._sc_rho = None
        self.dist_reduce = None  # vector sum over devices (multi-GPU)
        self.device = "cuda"     # where the engine's tensors live
        self.toy_chunk = 1 << 24  # generator candidates per toy-kernel launch
        self._prepare_structure()
        if compile:
            self._create()

    # ------------------------------------------------------------- native
    def _create(self):
        lib = load_library()
        c = self.code
        h = ctypes.c_void_p()
        src = self.src.encode()
        rc = lib.pwa_plan_create(src, len(src), len(c.mass_fields), len(c.angle_fields), c.ncol,
                                 c.nout, c.nshape + c.nrho + c.ncp, len(c.consts), c.nf, self.tpb,
                                 ctypes.byref(h))
        if rc != 0:
            msg = lib.pwa_last_error(h).decode(errors="replace")
            lib.pwa_plan_destroy(h)
            raise PWAError(f"pwa_plan_create failed ({rc}): {msg}")
        self.h = h

    def close(self):
        if self.h is not None:
            load_library().pwa_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = load_library().pwa_last_error(self.h).decode(errors="replace")
            raise PWAError(f"{what} failed ({rc}): {msg}")

    def info(self):
        arr = (ctypes.c_longlong * 8)()
        self._check(load_library().pwa_plan_info(self.h, arr), "pwa_plan_info")
        keys = ("regs_f64", "regs_f32", "local_f64", "local_f32", "blocks", "blocks_data",
                "nacc", "tpb")
        return dict(zip(keys, list(arr)))

    def compile_check(self, arch="sm_100a"):
        """NVRTC compile without a device; returns the ptxas log."""
        buf = ctypes.create_string_buffer(1 << 16)
        src = self.src.encode()
        rc = load_library().pwa_compile_only(src, len(src), self.tpb, arch.encode(), buf, len(buf))
        log = buf.value.decode(errors="replace")
        if rc != 0:
            raise PWAError(f"compile failed: {log}")
        return log

    def precompile(self, arch="sm_100a"):
        """Compile this model's module without a device into the on-disk
        cubin cache (pwa_precompile), so that a later process on a device
        of ``arch`` loads it instead of compiling."""
        load_library()
        buf = ctypes.create_string_buffer(1 << 12)
        src = self.src.encode()
        rc = load_library().pwa_precompile(src, len(src), self.tpb, arch.encode(), buf, len(buf))
        if rc != 0:
            raise PWAError(f"precompile failed: {buf.value.decode(errors='replace')}")

    # ------------------------------------------------------------- events
    def split_fields(self, x):
        """(n_fields, N) plan-ordered columns -> (mass columns, angle columns)."""
        c = self.code
        x = np.asarray(x, np.float64)
        xm = np.ascontiguousarray(x[c.mass_fields]) if c.mass_fields else np.zeros((0, x.shape[1]))
        xa = np.ascontiguousarray(x[c.angle_fields]) if c.angle_fields else np.zeros((0, x.shape[1]))
        return xm, xa

    def upload(self, x_data, w_data, x_mc=None, w_mc=None, stream=None):
        """Make data (+ MC) events resident.  x_*: (n_fields, N) columns in
        plan order; w_data: final data weights; w_mc: raw MC weights
        (normalised here to sum 1)."""
        xd = np.asarray(x_data, np.float64)
        wd = np.asarray(w_data, np.float64)
        nd = xd.shape[1]
        if x_mc is None:
            x = xd
            w = wd
            nm = 0
        else:
            xmc = np.asarray(x_mc, np.float64)
            nm = xmc.shape[1]
            wm = np.ones(nm) if w_mc is None else np.asarray(w_mc, np.float64)
            wm = wm / wm.sum()
            x = np.concatenate([xd, xmc], axis=1)
            w = np.concatenate([wd, wm])
        xm, xa = self.split_fields(x)
        w = np.ascontiguousarray(w)
        self._check(load_library().pwa_upload_events(
            self.h, xm.ctypes.data, xa.ctypes.data, w.ctypes.data, nd, nm, 0,
            stream or 0), "pwa_upload_events")
        self._n_data, self._n_mc = nd, nm
        self._sw = float(wd.sum())
        self._gram = None

    def upload_device(self, xm_ptr, xa_ptr, w_ptr, n_data, n_mc, sw, stream=None):
        """Events already on the device (pointers to FP64 row-major columns)."""
        self._check(load_library().pwa_upload_events(
            self.h, xm_ptr, xa_ptr, w_ptr, n_data, n_mc, 1, stream or 0), "pwa_upload_events")
        self._n_data, self._n_mc = n_data, n_mc
        self._sw = float(sw)
        self._gram = None

    # ---------------------------------------------------------- structure
    def _prepare_structure(self):
        g = self.group
        self.coupling_names = []   # complex names per column factor
        self.col_factors = []
        for ci, lsi in self.code.columns:
            c = g[ci]
            names = [c.params_head + "_total_0"]
            for vi, d in enumerate(c):
                names.append(f"{d.params_head}_g_ls_{lsi[vi]}")
            self.col_factors.append(names)
            for n in names:
                if n not in self.coupling_names:
                    self.coupling_names.append(n)
        # membership tests on particles/decays compare keys; precompute them
        self._inner_keys = {id(c): {p.key() for p in c.inner} for c in g}
        self._vertex_chain = {}
        for c in g:
            for d in c:
                self._vertex_chain.setdefault(d.key(), c)
        self.res_info = {}
        for p in g.resonances:
            chains = [c for c in g if p in c.inner]
            dp = chains[0].decay_of(p)
            self.res_info[p] = (dp, chains[0])
        self.shape_index = {}
        for si, p in enumerate(self.code.shape_res):
            self.shape_index[(p, "m")] = 2 * si
            self.shape_index[(p, "g")] = 2 * si + 1
        # column k = product of coupling_names[fac_idx[k, :]] (padded with -1)
        nf = max(len(f) for f in self.col_factors)
        self._fac_idx = np.full((len(self.col_factors), nf), -1, np.int64)
        for k, f in enumerate(self.col_factors):
            self._fac_idx[k, :len(f)] = [self.coupling_names.index(n) for n in f]
        # per coupling: the columns it enters and how often
        self._coup_cols = {}
        for n in self.coupling_names:
            ks = [k for k, f in enumerate(self.col_factors) if n in f]
            cnt = [self.col_factors[k].count(n) for k in ks]
            self._coup_cols[n] = (np.array(ks, np.int64), np.array(cnt))
        self._shape_cache = (None, None)
        self._jac_cache = {}
        self._cn_index = {n: i for i, n in enumerate(self.coupling_names)}
        self._cn_r = [n + "r" for n in self.coupling_names]
        self._cn_i = [n + "i" for n in self.coupling_names]
        self._cn_polar = np.array([self.vm.complex_vars.get(n, True) for n in self.coupling_names])
        # incidence of couplings in columns; True where every coupling enters
        # each of its columns once (then dc_k/dz = c_k / z)
        self._inc = np.zeros((len(self.coupling_names), len(self.col_factors)))
        for k, f in enumerate(self.col_factors):
            for n in f:
                self._inc[self._cn_index[n], k] += 1
        self._inc_linear = bool(np.all(self._inc <= 1))
        cidx = self.code.consts.index
        self._slot_vg = []          # (coupling index, re slot, im slot) of vertex g's and totals
        for d in self.code.vertices:
            for i in range(len(d.get_ls_list())):
                n = f"{d.params_head}_g_ls_{i}"
                if n in self._cn_index:
                    self._slot_vg.append((self._cn_index[n], cidx[f"{d}.g{i}.re"], cidx[f"{d}.g{i}.im"]))
        for ci, ch in enumerate(self.group):
            n = ch.params_head + "_total_0"
            self._slot_vg.append((self._cn_index[n], cidx[f"t{ci}.re"], cidx[f"t{ci}.im"]))
        a = np.array(self._slot_vg, np.int64).reshape(-1, 3)
        self._vg_src, self._vg_re, self._vg_im = a[:, 0], a[:, 1], a[:, 2]
        # constant-block slots of the lineshape and barrier constants
        self._res_slots = []
        for p, kind in self.code.res:
            if kind == "one":
                continue
            self._res_slots.append((p, kind, cidx[f"{p}.m0sq"],
                                    cidx.get(f"{p}.K"), cidx.get(f"{p}.useq"), cidx.get(f"{p}.y"),
                                    cidx.get(f"{p}.iq02"), cidx.get(f"{p}.wn")))
        self._vtx_slots = []
        for d in self.code.vertices:
            sl = {}
            for l in sorted(set(d.get_l_list())):
                sl[l] = (cidx.get(f"{d}.Pz0_{l}") if d.has_barrier_factor and d.has_bprime else None,
                         cidx.get(f"{d}.norm_{l}") if d.has_barrier_factor and d.barrier_factor_norm
                         else None)
            self._vtx_slots.append((d, self._vertex_chain[d.key()], sl))
        self._shape_slots = [(p, cidx[f"{p}.kappa_m"], cidx[f"{p}.inv_g0"])
                             for p in self.code.shape_res]
        # CP-violating chain totals: coupling index, their delta parameters,
        # the minus-charge constant slots, and per parameter its role
        code = self.code
        cp_tot = {ci: self.group[ci].params_head + "_total_0" for ci in code.cp_chains}
        self._cp_coup = np.array([self._cn_index[cp_tot[ci]] for ci in code.cp_chains], np.int64)
        self._cp_dr = [cp_tot[ci] + "deltar" for ci in code.cp_chains]
        self._cp_di = [cp_tot[ci] + "deltai" for ci in code.cp_chains]
        self._cp_t_re = np.array([cidx[f"t{ci}m.re"] for ci in code.cp_chains], np.int64)
        self._cp_t_im = np.array([cidx[f"t{ci}m.im"] for ci in code.cp_chains], np.int64)
        self._cp_cols = np.array(code.cp_cols, np.int64)
        self._cp_c_re = np.array([cidx[f"c{k}m.re"] for k in code.cp_cols], np.int64)
        self._cp_c_im = np.array([cidx[f"c{k}m.im"] for k in code.cp_cols], np.int64)
        self._cp_param = {}
        for ci in code.cp_chains:
            cols = np.array([j for j, k in enumerate(code.cp_cols)
                             if code.columns[k][0] == ci], np.int64)
            for suf in ("r", "i", "deltar", "deltai"):
                self._cp_param[cp_tot[ci] + suf] = (self._cn_index[cp_tot[ci]], suf, cols)
        self._Jm = None
        self._pol_names = list(self.code.pol_names)
        self._pol_index = {n: i for i, n in enumerate(self._pol_names)}
        if self._pol_names:
            na = self.code.na
            self._rho_re = np.array([cidx[f"rho{a}_{b}.re"] for a in range(na) for b in range(na)])
            self._rho_im = np.array([cidx[f"rho{a}_{b}.im"] for a in range(na) for b in range(na)])
            _, self._drho = density_matrix(self.group.top.J, np.zeros(len(self._pol_names)))
        self._mass_names = {f"{p.params_head}_mass": p for p in self.group.resonances}
        self._width_names = {f"{p.params_head}_width": p for p in self.group.resonances}
        self._build_vertex_tables()

    # ------------------------------------------- vectorised barrier constants
    def _build_vertex_tables(self):
        """Rows for the barrier and lineshape constants, built once: nominal
        masses gathered in one list (resonance masses from the parameters,
        the others fixed), one row per vertex with its (l, slot) entries, one
        row per lineshape, and for the Jacobian the (column, vertex entry)
        pairs through which each resonance mass acts.  Evaluated with scalar
        arithmetic (a few dozen rows: cheaper than array calls)."""
        parts = {}
        plist = []

        def pidx(q):
            k = q.key()
            if k not in parts:
                parts[k] = len(plist)
                plist.append(q)
            return parts[k]

        for q in self.group.resonances:
            dq, _ = self.res_info[q]
            for x in (q,) + tuple(dq.outs):
                pidx(x)
        res_keys = {q.key() for q in self.group.resonances}
        self._vt_rows = []
        vindex = {}
        for d, chain, sl in self._vtx_slots:
            a, (b, cc) = d.core, d.outs
            entries = []
            for l in sorted(sl):
                s_pz, s_norm = sl[l]
                entries.append((l, tuple(bprime_coeff(l)), bool(d.has_bprime),
                                bool(d.barrier_factor_norm),
                                -1 if s_pz is None else s_pz, -1 if s_norm is None else s_norm))
            vindex[d.key()] = len(self._vt_rows)
            self._vt_rows.append((pidx(a), pidx(b), pidx(cc), bool(d.no_q0), float(d.d),
                                  bool(d.has_barrier_factor), entries))
        self._m_base = [q.mass if q.mass is not None else 0.0 for q in plist]
        self._m_res = [(i, f"{q.params_head}_mass", q.mass) for i, q in enumerate(plist)
                       if q.key() in res_keys]
        # Jacobian rows of a resonance mass: the vertices it enters (with a
        # barrier factor) and per column the (vertex, l) entries summed
        self._jac_pairs = {}
        for q in self.group.resonances:
            contrib, verts = [], []
            for k, (ci, lsi) in enumerate(self.code.columns):
                chain = self.group[ci]
                if q.key() not in self._inner_keys[id(chain)]:
                    continue
                for vi, d in enumerate(chain):
                    if q not in (d.core,) + d.outs or not d.has_barrier_factor:
                        continue
                    v = vindex[d.key()]
                    if v not in verts:
                        verts.append(v)
                    contrib.append((k, v, d.get_ls_list()[lsi[vi]][0]))
            if contrib:
                self._jac_pairs[q.key()] = (parts[q.key()], verts, contrib)
        # lineshape rows
        shape_pos = {q.key(): j for j, (q, _, _) in enumerate(self._shape_slots)}
        self._ls_rows = []
        for p, kind, s_m0sq, s_k, s_useq, s_y, s_iq, s_wn in self._res_slots:
            dp, chain = self.res_info[p]
            b, cc = dp.outs
            L = p.bw_l if p.bw_l is not None else min(dp.get_l_list())
            j = shape_pos.get(p.key())
            sh = (-1, -1) if j is None else self._shape_slots[j][1:]
            self._ls_rows.append((kind, parts[p.key()], parts[b.key()], parts[cc.key()], L,
                                  float(p.d), f"{p.params_head}_width", p.width,
                                  tuple(bprime_coeff(L)), s_m0sq, s_k, s_useq, s_y, s_iq, s_wn,
                                  sh[0], sh[1]))

    def _mass_list(self, vals):
        M = list(self._m_base)
        for i, n, dflt in self._m_res:
            M[i] = vals.get(n, dflt)
        return M

    @staticmethod
    def _vertex_entry_values(q02, d, entries):
        """[(Pz0_l, norm_l)] of one vertex: ``poly(l, q02 d d)`` and
        ``1 / |q02|^(l/2)`` (``1 / sqrt(q02 q02)^(l/2)`` when complex)."""
        out = []
        z = q02 * d * d
        cplx = isinstance(q02, complex)
        for l, coef, bp, bn, _, _ in entries:
            if bp:
                r = 0.0
                for c_ in coef:
                    r = r * z + c_
            else:
                r = 1.0
            if bn:
                nrm = 1.0 / (cmath.sqrt(q02 * q02) if cplx else abs(q02)) ** (l / 2)
            else:
                nrm = 1.0
            out.append((r, nrm))
        return out

    @staticmethod
    def _vertex_q02(M, row):
        ia, ib, ic, noq0 = row[0], row[1], row[2], row[3]
        if noq0:
            return 1.0
        return rel_p2(M[ia], M[ib], M[ic])

    @staticmethod
    def _lineshape_row_values(kind, m0, g0, mb, mc, L, d, coef):
        """(K, useq, q0^2) of one lineshape at parent mass ``m0`` (real or
        complex): BWR K = m0^2 Gamma0 B_L(q0 d) / q0^(2L+1) (q0 clamped at
        threshold; without the q0 power and useq = 0 below it), BWR2
        K = m0^2 Gamma0 B_L(q0^2 d^2) with q0^2 unclamped, BW K = m0 Gamma0."""
        if kind == "BW":
            return m0 * g0, 1.0, None
        if kind == "BWR2":
            q02 = rel_p2(m0, mb, mc)
            z = q02 * d * d
            r = 0.0
            for c_ in coef:
                r = r * z + c_
            return m0 * m0 * g0 * r, 1.0, q02
        q0 = rel_p(m0, mb, mc)
        z = (q0 * d) ** 2
        r = 0.0
        for c_ in coef:
            r = r * z + c_
        if q0.real > 1e-15:
            return m0 * m0 * g0 * r / q0 ** (2 * L + 1), 1.0, None
        return m0 * m0 * g0 * r, 0.0, None

    def _shape_consts(self, C, vals):
        """Lineshape and barrier constants of the constant block at ``vals``."""
        M = self._mass_list(vals)
        for row in self._vt_rows:
            entries = row[6]
            vals_e = self._vertex_entry_values(self._vertex_q02(M, row), row[4], entries)
            for (_, _, _, _, s_pz, s_norm), (pz, nrm) in zip(entries, vals_e):
                if s_pz >= 0:
                    C[s_pz] = pz
                if s_norm >= 0:
                    C[s_norm] = nrm
        h = 1e-20
        for (kind, im, ib, ic, L, d, gname, gdef, coef, s_m0sq, s_k, s_useq, s_y, s_iq, s_wn,
             s_kap, s_ig) in self._ls_rows:
            m0, mb, mc = M[im], M[ib], M[ic]
            g0 = vals.get(gname, gdef)
            C[s_m0sq] = m0 * m0
            K, useq, q02 = self._lineshape_row_values(kind, m0, g0, mb, mc, L, d, coef)
            if kind == "BWR":
                C[s_k] = K
                C[s_useq] = useq
            elif kind == "BWR2":
                C[s_k] = K
                C[s_iq] = 1.0 / q02
            else:
                C[s_y] = K
            if s_wn is not None:
                C[s_wn] = g0
            if s_kap >= 0:
                # kappa = dlog(m0 Gamma) / dm0 by a complex step; for BWR2
                # m0 Gamma2 = K r^(L+1/2) / (m B): dlog K - (L + 1/2) dlog q0^2
                Kc, _, qc = self._lineshape_row_values(kind, complex(m0, h), g0, mb, mc, L, d,
                                                       coef)
                kap = Kc.imag / h / K.real if K.real != 0 else 0.0
                if kind == "BWR2":
                    kap -= (L + 0.5) * qc.imag / h / q02.real
                C[s_kap] = kap
                C[s_ig] = 1.0 / g0 if g0 else 0.0

    def _mass_dlog(self, vals, key):
        """{column: d ln(prod of its barrier factors) / d m} of a resonance
        mass, by a complex step through the vertices it enters."""
        qi, verts, contrib = self._jac_pairs[key]
        M = self._mass_list(vals)
        Mc = list(M)
        Mc[qi] = complex(M[qi], 1e-20)
        dlog = {}
        for v in verts:
            row = self._vt_rows[v]
            e0 = self._vertex_entry_values(self._vertex_q02(M, row), row[4], row[6])
            ec = self._vertex_entry_values(self._vertex_q02(Mc, row), row[4], row[6])
            for (l, _, bp, bn, _, _), (pz0, n0), (pzc, nc) in zip(row[6], e0, ec):
                t = 0.0
                # bf_l ~ sqrt(Pz0_l) * norm_l
                if bp:
                    t += 0.5 * complex(pzc).imag / 1e-20 / complex(pz0).real
                if bn:
                    t += complex(nc).imag / 1e-20 / complex(n0).real
                dlog[(v, l)] = t
        kap = {}
        for k, v, l in contrib:
            kap[k] = kap.get(k, 0.0) + dlog[(v, l)]
        return kap

    def _shape_key(self, vals):
        return tuple(vals.get(k) for k in self._shape_names)

    def consts(self, vals):
        """Constant block of one evaluation from the parameter dict.  The
        part that depends only on masses and widths (lineshape and barrier
        constants) is cached per mass/width setting."""
        if not hasattr(self, "_shape_names"):
            self._shape_names = sorted(k for k in vals if k.endswith(("_mass", "_width")))
        key = self._shape_key(vals)
        if self._shape_cache[0] == key:
            C = self._shape_cache[1].copy()
        else:
            C = np.zeros(len(self.code.consts))
            self._shape_consts(C, vals)
            self._shape_cache = (key, C.copy())
        self._coupling_consts(C, vals)
        self._fill_rho(C, vals)
        return C

    def _coupling_consts(self, C, vals):
        """Column couplings c_k (products of the complex couplings), vertex
        couplings and chain totals into the constant block."""
        c = self.code
        r = np.fromiter((vals[n] for n in self._cn_r), float, len(self._cn_r))
        ph = np.fromiter((vals[n] for n in self._cn_i), float, len(self._cn_i))
        cp = self._cp_coup
        if len(cp):
            # CP-violating totals: charge +1 takes (r + dr, i + di), -1 (r - dr, i - di)
            dr = np.array([vals[n] for n in self._cp_dr])
            di = np.array([vals[n] for n in self._cp_di])
            rm, phm = r[cp] - dr, ph[cp] - di
            r[cp] += dr
            ph[cp] += di
        z = np.where(self._cn_polar, r * np.exp(1j * ph), r + 1j * ph)
        self._cvec, self._cr, self._cph = z, r, ph
        self._cv = dict(zip(self.coupling_names, z))
        self._ck = np.prod(np.append(z, 1.0 + 0j)[self._fac_idx], axis=1)
        C[0:2 * c.ncol:2] = self._ck.real
        C[1:2 * c.ncol:2] = self._ck.imag
        C[self._vg_re] = z[self._vg_src].real
        C[self._vg_im] = z[self._vg_src].imag
        if len(cp):
            zm = z.copy()
            zm[cp] = np.where(self._cn_polar[cp], rm * np.exp(1j * phm), rm + 1j * phm)
            self._cvec_m, self._cr_m, self._cph_m = zm, rm, phm
            # column couplings without their CP total (the total's factor set to 1)
            zr = z.copy()
            zr[cp] = 1.0
            self._ck_rest = np.prod(np.append(zr, 1.0 + 0j)[self._fac_idx], axis=1)
            self._ck_m = np.prod(np.append(zm, 1.0 + 0j)[self._fac_idx], axis=1)
            C[self._cp_t_re] = zm[cp].real
            C[self._cp_t_im] = zm[cp].imag
            C[self._cp_c_re] = self._ck_m[self._cp_cols].real
            C[self._cp_c_im] = self._ck_m[self._cp_cols].imag

    def _fill_rho(self, C, vals):
        """Parent spin density matrix (polarised models) into its slots."""
        if not self._pol_names:
            return
        rho, _ = density_matrix(self.group.top.J, [vals[n] for n in self._pol_names])
        C[self._rho_re] = rho.real.reshape(-1)
        C[self._rho_im] = rho.imag.reshape(-1)

    # ------------------------------------------------------------ jacobian
    def _jac_layout(self, names):
        """Index arrays of the coupling parameters among ``names`` (None if
        a coupling enters a column more than once)."""
        key = tuple(names)
        lay = getattr(self, "_jac_lay", {}).get(key, 0)
        if lay != 0:
            return lay
        if not self._inc_linear:
            lay = None
        else:
            rows = [pi for pi, n in enumerate(names) if n[:-1] in self._cn_index]
            ci = np.array([self._cn_index[names[pi][:-1]] for pi in rows], np.int64)
            is_r = np.array([names[pi].endswith("r") for pi in rows])
            lay = (ci, is_r, self._cn_polar[ci], np.array(rows, np.int64))
        self._jac_lay = {key: lay}
        return lay

    def jacobian(self, vals, names):
        """J[p, k] (complex) and shape selectors D[p, s] for parameters
        ``names`` at ``vals`` (call after consts())."""
        c = self.code
        P = len(names)
        J = np.zeros((P, c.ncol), np.complex128)
        D = np.zeros((P, max(c.nshape + c.nrho, 1)))
        cv = self._cv
        key = (tuple(names), self._shape_key(vals) if hasattr(self, "_shape_names") else None)
        cached = self._jac_cache.get(key)
        lay = self._jac_layout(names)
        if lay is not None and np.all(self._cr[lay[0]] != 0):
            # every coupling enters its columns linearly: dc_k/dtheta = c_k * f
            ci, is_r, polar, rows = lay
            z, r = self._cvec[ci], self._cr[ci]
            f = np.where(polar, np.where(is_r, 1.0 / r, 1j), np.where(is_r, 1.0 / z, 1j / z))
            J[rows] = self._inc[ci] * self._ck[None, :] * f[:, None]
            names_left = [(pi, n) for pi, n in enumerate(names) if n[:-1] not in cv]
        else:
            names_left = list(enumerate(names))
        for pi, n in names_left:
            if n in self._cp_param:
                continue  # CP-total parameters: _cp_jacobian
            if n in self._pol_index:
                # polarisation: d f / d p = Re sum_ab T_ab d rho_ab / d p, T_ab
                # the (a, b) parent-helicity product sums after the shape sums
                dr = self._drho[self._pol_index[n]]
                D[pi, c.nshape:c.nshape + c.nrho:2] = dr.real.reshape(-1)
                D[pi, c.nshape + 1:c.nshape + c.nrho:2] = -dr.imag.reshape(-1)
                continue
            base = n[:-1]
            if base in cv:
                r, ph = vals[base + "r"], vals[base + "i"]
                polar = self.vm.complex_vars.get(base, True)
                if polar:
                    dz = np.exp(1j * ph) if n.endswith("r") else 1j * cv[base]
                else:
                    dz = 1.0 if n.endswith("r") else 1j
                ks, cnt = self._coup_cols[base]
                z = cv[base]
                if np.all(cnt == 1) and z != 0:
                    # c_k is linear in this coupling: dc_k = c_k / z * dz
                    J[pi, ks] = self._ck[ks] / z * dz
                    continue
                for k in ks:
                    f = self.col_factors[k]
                    m = f.count(base)
                    others = np.prod([cv[x] for x in f if x != base]) if len(f) > m else 1.0
                    J[pi, k] += m * others * z ** (m - 1) * dz
                continue
            if cached is not None:
                J[pi] = cached[0][pi] * self._ck
                D[pi] = cached[1][pi]
                continue
            # masses / widths
            if n in self._mass_names:
                p, kind = self._mass_names[n], "m"
            elif n in self._width_names:
                p, kind = self._width_names[n], "g"
            else:
                raise KeyError(f"unknown parameter {n}")
            if (p, kind) in self.shape_index:
                D[pi, self.shape_index[(p, kind)]] = 1.0
            if kind == "m" and p.key() in self._jac_pairs:
                # barrier factors through q0^2 of every vertex touching p
                for k, kap in self._mass_dlog(vals, p.key()).items():
                    J[pi, k] += self._ck[k] * kap
        if len(self._cp_coup):
            J = self._cp_jacobian(J, names)
        if cached is None and key[1] is not None:
            # mass/width rows: J = kappa_k * c_k with kappa fixed per shape setting
            kap = np.zeros((P, c.ncol), np.complex128)
            for pi, n in enumerate(names):
                if n[:-1] not in cv:
                    kap[pi] = np.divide(J[pi], self._ck, out=np.zeros(c.ncol, np.complex128),
                                        where=self._ck != 0)
            self._jac_cache = {key: (kap, D.copy())}
        return J, D

    def _cp_jacobian(self, J, names):
        """Rows of the CP-violating totals' parameters (r, i, deltar,
        deltai) for both charges, and ``self._Jm``: derivatives of the
        minus-charge column couplings c_k^- of the CP columns.  A parameter
        other than a CP total's enters c_k^- as it enters c_k^+, so its row
        is the plus row times z^-/z^+ of the column's total."""
        cp_cols = self._cp_cols
        tot_of_col = np.empty(len(cp_cols), np.int64)  # coupling index of each CP column's total
        for i, suf_cols in {v[0]: v[2] for v in self._cp_param.values()}.items():
            tot_of_col[suf_cols] = i
        zp_c, zm_c = self._cvec[tot_of_col], self._cvec_m[tot_of_col]
        # (a chain switched off, z^+ = z^- = 0, has zero rows either way)
        ratio = np.divide(zm_c, zp_c, out=np.zeros(len(zp_c), np.complex128), where=zp_c != 0)
        Jm = J[:, cp_cols] * ratio[None, :]
        for pi, n in enumerate(names):
            if n not in self._cp_param:
                continue
            i, suf, cols = self._cp_param[n]
            ks, _ = self._coup_cols[self.coupling_names[i]]
            polar = bool(self._cn_polar[i])
            j = list(self._cp_coup).index(i)
            zp, zm = self._cvec[i], self._cvec_m[i]
            sgn = -1.0 if suf.startswith("delta") else 1.0
            # z = a e^{i phi}: dz/da = e^{i phi}, dz/dphi = i z (polar); 1, i (Cartesian)
            if suf.endswith("r"):
                dp = np.exp(1j * self._cph[i]) if polar else 1.0
                dm = np.exp(1j * self._cph_m[j]) if polar else 1.0
            else:
                dp = 1j * zp if polar else 1j
                dm = 1j * zm if polar else 1j
            J[pi, :] = 0.0
            J[pi, ks] = self._ck_rest[ks] * dp
            Jm[pi, :] = 0.0
            Jm[pi, cols] = self._ck_rest[cp_cols[cols]] * (sgn * dm)
        self._Jm = Jm
        return J

    def grad_from_sums(self, J, D, s):
        """d(sum)/d(parameters) from one event set's kernel sums ``s``:
        2 Re J G over the columns, the lineshape/polarisation selectors D,
        and for CP-violating totals 2 Re J^- G^- over the charge -1 sums."""
        c = self.code
        K = c.ncol
        g = 2 * np.real(J @ (s[1:1 + 2 * K:2] + 1j * s[2:2 + 2 * K:2]))
        ns = c.nshape + c.nrho
        if ns:
            g = g + D[:, :ns] @ s[1 + 2 * K:1 + 2 * K + ns]
        if c.ncp and self._Jm is not None:
            o = 1 + 2 * K + ns
            g = g + 2 * np.real(self._Jm @ (s[o:o + c.ncp:2] + 1j * s[o + 1:o + c.ncp:2]))
        return g

    # ------------------------------------------------------------ evaluate
    def eval_sums(self, C, precision=PLAIN_F64, mc=True, stream=None):
        nacc = self.code.nacc
        out = np.zeros(2 * nacc)
        C = np.ascontiguousarray(C, np.float64)
        self._check(load_library().pwa_eval(self.h, _dptr(C), precision, 1 if mc else 0,
                                            stream or 0, _dptr(out)), "pwa_eval")
        return out[:nacc], out[nacc:]

    # ------------------------------------ floating shapes: shape-free columns
    def _column_rho(self, C):
        """Per column, the product of its barrier normalisations in the
        constant block (sqrt(Pz0_l) per B' vertex, norm_l per normalised
        one): the columns' only dependence on the shapes besides the
        lineshapes themselves."""
        if not hasattr(self, "_rho_terms"):
            idx = self.code.consts.index
            t = [(k, idx[name], kind == "sqrt") for k in range(self.code.ncol)
                 for kind, name in self.code.column_barrier_consts(k)]
            self._rho_terms = (np.array([x[0] for x in t], np.int64),
                               np.array([x[1] for x in t], np.int64),
                               np.array([x[2] for x in t], bool))
        cols, slots, sq = self._rho_terms
        v = np.asarray(C)[slots]
        if not np.all(v > 0.0):  # B' normalisations and 1 / |q0^2|^(l/2) are positive
            raise PWAError("non-positive barrier normalisation: the columns do not factorise "
                           "at this shape setting")
        # product per column as exp of the summed logs (sqrt terms at half weight)
        return np.exp(np.bincount(cols, weights=np.where(sq, 0.5, 1.0) * np.log(v),
                                  minlength=self.code.ncol))

    def shape_cache(self, vals, stream=None):
        """Build the floating-shape column cache (pwa_shape_cache): every
        event's columns without their lineshapes, at the shapes in vals."""
        if not self.code.shape_cache_ok:
            raise PWAError("the floating-shape column cache needs one pass, no polarised "
                           "parent and no CP-violating totals")
        C = np.ascontiguousarray(self.consts(vals), np.float64)
        rho = self._column_rho(C)
        self._check(load_library().pwa_shape_cache(self.h, _dptr(C), stream or 0),
                    "pwa_shape_cache")
        self._sc_rho = rho

    def _sc_ratio(self, C):
        """The columns' barrier-normalisation ratios to the cache's setting
        (kept in self._ratio), or None where a normalisation is not positive
        (the columns do not factorise there: the evaluation recomputes)."""
        try:
            self._ratio = np.ascontiguousarray(self._column_rho(C) / self._sc_rho)
        except PWAError:
            self._ratio = None
        return self._ratio

    def eval_sums_shapecache(self, C, stream=None, ratio=None):
        """Sums of one evaluation from the floating-shape column cache (the
        layout of eval_sums: data and MC rows of nacc)."""
        nacc = self.code.nacc
        C = np.ascontiguousarray(C, np.float64)
        if ratio is None:
            ratio = np.ascontiguousarray(self._column_rho(C) / self._sc_rho)
        out = np.zeros(2 * nacc)
        self._check(load_library().pwa_eval_shapecache(self.h, _dptr(C), _dptr(ratio),
                                                       stream or 0, _dptr(out)),
                    "pwa_eval_shapecache")
        return out[:nacc], out[nacc:]

    def eval_shapecache_enqueue(self, C, stream=None):
        """Launch one floating-shape-cache evaluation without waiting."""
        C = np.ascontiguousarray(C, np.float64)
        ratio = np.ascontiguousarray(self._column_rho(C) / self._sc_rho)
        self._check(load_library().pwa_eval_shapecache_enqueue(self.h, _dptr(C), _dptr(ratio),
                                                               stream or 0),
                    "pwa_eval_shapecache_enqueue")

    def eval_enqueue(self, C, precision=PLAIN_F64, mc=True, stream=None):
        """Launch the evaluation kernels without waiting (for timing)."""
        C = np.ascontiguousarray(C, np.float64)
        self._check(load_library().pwa_eval_enqueue(self.h, _dptr(C), precision, 1 if mc else 0,
                                                    stream or 0), "pwa_eval_enqueue")

    def build_gram(self, C, stream=None):
        if self.code.nrho or self.code.cp_chains:
            raise PWAError("the column cache / Gram form does not apply to a polarised parent "
                           "or CP-violating totals")
        K = self.code.ncol
        out = np.zeros(2 * K * K)
        C = np.ascontiguousarray(C, np.float64)
        self._check(load_library().pwa_build_gram(self.h, _dptr(C), stream or 0, _dptr(out)),
                    "pwa_build_gram")
        M = out[0::2] + 1j * out[1::2]
        return M.reshape(K, K)

    def pdf_device(self, C, beg, end, out_ptr, precision=PLAIN_F64, stream=None):
        C = np.ascontiguousarray(C, np.float64)
        self._check(load_library().pwa_eval_pdf(self.h, _dptr(C), precision, beg, end, out_ptr,
                                                stream or 0), "pwa_eval_pdf")

    def local_pieces(self, vals, names, precision=PLAIN_F64, use_gram=False, stream=None):
        """This device's share of the NLL as the vector
        [S_data, S_mc * f, sw, g_data (P), g_mc * f (P)] with S the summed
        data log term / MC integral, g their gradients, sw the data weight
        sum and f = this device's share of the total MC weight.  Summing the
        vectors of all devices and calling :func:`combine_pieces` gives the
        NLL and gradient of the union of all devices' events."""
        C = self.consts(vals)
        J, D = self.jacobian(vals, names)
        nacc = self.code.nacc
        K = self.code.ncol
        if use_gram:
            if self._gram is None:
                raise PWAError("gram matrix not built")
            sd, _ = self.eval_sums(C, precision, mc=False, stream=stream)
            ck = self._ck
            M = self._gram
            # I = c^H M c; G^mc_k = sum_i w conj(A_i) F_ik = sum_l conj(c_l) M_lk
            Gm = np.conj(ck) @ M
            sm = np.zeros(nacc)
            sm[0] = float(np.real(Gm @ ck))
            sm[1:1 + 2 * K:2] = Gm.real
            sm[2:2 + 2 * K:2] = Gm.imag
        elif self.use_shape_cache and precision != PLAIN_F64 and self._sc_ratio(C) is not None:
            sd, sm = self.eval_sums_shapecache(C, stream=stream, ratio=self._ratio)
        else:
            sd, sm = self.eval_sums(C, precision, mc=True, stream=stream)
        gd = self.grad_from_sums(J, D, sd)
        gm = self.grad_from_sums(J, D, sm)
        f = self.mc_share
        return np.concatenate([[sd[0], sm[0] * f, self._sw], gd, gm * f])

    def nll_grad(self, vals, names, precision=PLAIN_F64, use_gram=False, stream=None):
        """NLL and gradient w.r.t. ``names`` (real parameter names)."""
        vec = self.local_pieces(vals, names, precision, use_gram, stream)
        if self.dist_reduce is not None:
            vec = self.dist_reduce(vec)
        return combine_pieces(vec, len(names))

    # -------------------------------------------------- cached (fixed shapes)
    def _ivec(self, a):
        a = np.ascontiguousarray(np.asarray(a, np.int32))
        return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))

    def set_param_layout(self, var_names, train_names):
        """Hand the coupling structure to the library for its chain rule."""
        idx = {n: i for i, n in enumerate(var_names)}
        r = [idx[n + "r"] for n in self.coupling_names]
        im = [idx[n + "i"] for n in self.coupling_names]
        pol = [1 if self.vm.complex_vars.get(n, True) else 0 for n in self.coupling_names]
        cidx = {n: j for j, n in enumerate(self.coupling_names)}
        nfac = max(len(f) for f in self.col_factors)
        cf = -np.ones((self.code.ncol, nfac), np.int32)
        for k, f in enumerate(self.col_factors):
            for q, n in enumerate(f):
                cf[k, q] = cidx[n]
        tr = [idx[n] for n in train_names]
        self._layout = [self._ivec(x) for x in (r, im, pol, cf.reshape(-1), tr)]
        self._var_names = list(var_names)
        self._n_train = len(tr)
        # per-call buffers of the cached evaluation, addresses taken once
        self._vbuf = np.zeros(len(var_names))
        self._gbuf = np.zeros(len(tr))
        self._nbuf = np.zeros(1)
        self._vbuf_p, self._gbuf_p, self._nbuf_p = (
            self._vbuf.ctypes.data, self._gbuf.ctypes.data, self._nbuf.ctypes.data)
        (a, pa), (b, pb), (c, pc), (d, pd), (e, pe) = self._layout
        self._check(load_library().pwa_set_param_layout(
            self.h, len(var_names), len(r), pa, pb, pc, nfac, pd, len(tr), pe),
            "pwa_set_param_layout")

    # ------------------------------------- native host side (host program)
    def host_program_arrays(self, var_names, train_names):
        """The flat (int, double) arrays of this model's host program for
        the variable layout ``var_names`` (all variables, in order) and the
        gradient w.r.t. ``train_names`` (format in include/pwa_b200.h).
        PWAError for a trainable name with no role."""
        c = self.code
        idx = {n: i for i, n in enumerate(var_names)}
        cp_names = set(self._cp_dr) | set(self._cp_di)
        for n in train_names:
            ok = (n[:-1] in self._cn_index and n[-1] in "ri") or n in self._mass_names \
                or n in self._width_names or n in cp_names or n in self._pol_index
            if not ok or n not in idx:
                raise PWAError(f"trainable variable {n} has no role in the host program")
        try:
            cr = [idx[n + "r"] for n in self.coupling_names]
            ci = [idx[n + "i"] for n in self.coupling_names]
        except KeyError as e:
            raise PWAError(f"coupling variable {e} missing from the layout") from None
        nfac = self._fac_idx.shape[1]
        n_extra = c.nshape + c.nrho + c.ncp
        ip = [HOSTPROG_MAGIC, 2, c.ncol, len(c.consts), n_extra, len(var_names),
              len(train_names), len(self.coupling_names), nfac]
        ip += cr + ci + [int(bool(x)) for x in self._cn_polar]
        ip += [int(x) for x in self._fac_idx.reshape(-1)]
        ip += [idx[n] for n in train_names]
        ip += [len(self._vg_src)]
        for a, b, d in zip(self._vg_src, self._vg_re, self._vg_im):
            ip += [int(a), int(b), int(d)]
        m_var = [-1] * len(self._m_base)
        m_base = [float(x) for x in self._m_base]
        for i, n, dflt in self._m_res:
            if n in idx:
                m_var[i] = idx[n]
            elif dflt is None:
                raise PWAError(f"resonance mass {n} has neither a variable nor a value")
        ip += [len(m_var)] + m_var
        dp = list(m_base)
        ip += [len(self._vt_rows)]
        for ia, ib, ic_, noq0, d, _, entries in self._vt_rows:
            ip += [ia, ib, ic_, int(noq0), len(entries)]
            dp += [float(d)]
            for l, coef, bp, bn, s_pz, s_norm in entries:
                ip += [int(l), int(bp), int(bn), int(s_pz), int(s_norm), len(coef)]
                dp += [float(x) for x in coef]
        kinds = {"BW": 0, "BWR": 1, "BWR2": 2}
        opt = (lambda x: -1 if x is None else int(x))
        ip += [len(self._ls_rows)]
        for (kind, im, ib, ic_, L, d, gname, gdef, coef, s_m0sq, s_k, s_useq, s_y, s_iq, s_wn,
             s_kap, s_ig) in self._ls_rows:
            if kind not in kinds:
                raise PWAError(f"lineshape kind {kind} not in the host program")
            if gname not in idx and gdef is None:
                raise PWAError(f"width {gname} has neither a variable nor a value")
            ip += [kinds[kind], im, ib, ic_, int(L), idx.get(gname, -1), int(s_m0sq), opt(s_k),
                   opt(s_useq), opt(s_y), opt(s_iq), opt(s_wn), opt(s_kap), opt(s_ig), len(coef)]
            dp += [float(d), float(gdef or 0.0)] + [float(x) for x in coef]
        sel = []
        for n in var_names:
            for names, kind in ((self._mass_names, "m"), (self._width_names, "g")):
                if n in names and (names[n], kind) in self.shape_index:
                    sel.append((idx[n], self.shape_index[(names[n], kind)]))
        ip += [len(sel)]
        for a, b in sel:
            ip += [a, b]
        mj = []
        for n, p in self._mass_names.items():
            if n in idx and p.key() in self._jac_pairs:
                qi, verts, contrib = self._jac_pairs[p.key()]
                trip = []
                for k, v, l in contrib:
                    ls_ = [e[0] for e in self._vt_rows[v][6]]
                    trip += [k, v, ls_.index(l)]
                mj.append([idx[n], qi, len(verts)] + list(verts) + [len(contrib)] + trip)
        ip += [len(mj)]
        for row in mj:
            ip += row
        cidx = c.consts.index
        rt = [(k, cidx[name], int(kind == "sqrt")) for k in range(c.ncol)
              for kind, name in c.column_barrier_consts(k)]
        ip += [len(rt)]
        for t in rt:
            ip += list(t)
        # polarised parent: rho = rho0 + sum_q p_q G_q (density_matrix is
        # linear in the polarisation)
        if self._pol_names:
            try:
                pv = [idx[n] for n in self._pol_names]
            except KeyError as e:
                raise PWAError(f"polarisation variable {e} missing from the layout") from None
            rho0, G = density_matrix(self.group.top.J, np.zeros(len(self._pol_names)))
            ne = rho0.size
            ip += [ne] + [int(x) for x in self._rho_re] + [int(x) for x in self._rho_im]
            ip += [c.nshape, len(pv)] + pv
            for m in [rho0] + list(G):
                dp += [float(x) for pair in zip(m.real.reshape(-1), m.imag.reshape(-1))
                       for x in pair]
        else:
            ip += [0, 0, 0]
        # CP-violating totals and the CP columns' charge -1 couplings
        ip += [len(self._cp_coup)]
        for j, ndr, ndi, sre, sim in zip(self._cp_coup, self._cp_dr, self._cp_di,
                                         self._cp_t_re, self._cp_t_im):
            if ndr not in idx or ndi not in idx:
                raise PWAError(f"CP variables of {self.coupling_names[j]} missing from the layout")
            ip += [int(j), idx[ndr], idx[ndi], int(sre), int(sim)]
        ip += [len(self._cp_cols)]
        for k, sre, sim in zip(self._cp_cols, self._cp_c_re, self._cp_c_im):
            ip += [int(k), int(sre), int(sim)]
        ip += [c.nshape + c.nrho if c.ncp else -1]
        ip += [HOSTPROG_MAGIC]
        return np.array(ip, np.int32), np.array(dp, np.float64)

    def host_program(self, var_names, train_names):
        """:class:`HostProgram` of this model for the given layout."""
        ip, dp = self.host_program_arrays(var_names, train_names)
        c = self.code
        return HostProgram(ip, dp, c.ncol, len(c.consts), c.nshape + c.nrho + c.ncp,
                           len(train_names), len(c.cp_cols))

    def set_host_program(self, var_names, train_names):
        """Give the plan its host program: evaluations from the variable
        vector (pieces_vars / nll_grad_vars) then run the host side in
        native code."""
        hp = self.host_program(var_names, train_names)
        try:
            self._check(load_library().pwa_set_host_program(self.h, hp.h), "pwa_set_host_program")
        finally:
            hp.close()
        self._hp_train = len(train_names)
        self._hp_vbuf = np.zeros(len(var_names))
        self._hp_gbuf = np.zeros(len(train_names))
        self._hp_nbuf = np.zeros(1)
        self._hp_ptrs = (self._hp_vbuf.ctypes.data, self._hp_gbuf.ctypes.data,
                         self._hp_nbuf.ctypes.data)

    def pieces_vars(self, var_values, form, mc_share=None, stream=None):
        """This device's piece vector (layout of :meth:`local_pieces`) of
        one evaluation at ``var_values`` (pwa_pieces_vars)."""
        v = np.ascontiguousarray(var_values, np.float64)
        out = np.zeros(3 + 2 * self._hp_train)
        share = self.mc_share if mc_share is None else mc_share
        self._check(load_library().pwa_pieces_vars(self.h, v.ctypes.data, int(form), self._sw,
                                                   share, stream or 0, out.ctypes.data),
                    "pwa_pieces_vars")
        return out

    def nll_grad_vars(self, var_values, form, stream=None):
        """NLL and gradient at ``var_values`` with the host side in native
        code (pwa_nll_grad_vars; over all devices through dist_reduce)."""
        if self.dist_reduce is not None:
            vec = self.dist_reduce(self.pieces_vars(var_values, form, stream=stream))
            return combine_pieces(vec, self._hp_train)
        self._hp_vbuf[:] = var_values
        pv, pg, pn = self._hp_ptrs
        self._check(load_library().pwa_nll_grad_vars(self.h, pv, int(form), self._sw,
                                                     stream or 0, pn, pg), "pwa_nll_grad_vars")
        return float(self._hp_nbuf[0]), self._hp_gbuf.copy()

    def cache_data(self, vals):
        if self.code.nrho or self.code.cp_chains:
            raise PWAError("the column cache / Gram form does not apply to a polarised parent "
                           "or CP-violating totals")
        """Evaluate and keep the data events' partial-wave columns."""
        C = np.ascontiguousarray(self.consts(vals))
        self._check(load_library().pwa_cache_data(self.h, _dptr(C), 0), "pwa_cache_data")

    def pieces_cached(self, var_values, mc_share=None, stream=None):
        v = np.ascontiguousarray(var_values, np.float64)
        out = np.zeros(3 + 2 * self._n_train)
        share = self.mc_share if mc_share is None else mc_share
        self._check(load_library().pwa_pieces_cached(self.h, _dptr(v), self._sw, share,
                                                     stream or 0, _dptr(out)),
                    "pwa_pieces_cached")
        return out

    def nll_grad_cached(self, var_values, stream=None):
        """NLL and gradient from the column cache + Gram matrix (C++ path)."""
        if self.dist_reduce is not None:
            vec = self.dist_reduce(self.pieces_cached(var_values, stream=stream))
            return combine_pieces(vec, self._n_train)
        self._vbuf[:] = var_values
        self._check(load_library().pwa_nll_grad_cached(self.h, self._vbuf_p, self._sw,
                                                       stream or 0, self._nbuf_p, self._gbuf_p),
                    "pwa_nll_grad_cached")
        return float(self._nbuf[0]), self._gbuf.copy()

    def pieces_points(self, var_rows, mc_share=None, stream=None):
        """Piece vectors of many parameter points (rows of all variables) in
        one pass over the column cache (FP32 amplitudes; pwa_pieces_points)."""
        V = np.ascontiguousarray(var_rows, np.float64)
        out = np.zeros((V.shape[0], 3 + 2 * self._n_train))
        share = self.mc_share if mc_share is None else mc_share
        self._check(load_library().pwa_pieces_points(self.h, V.shape[0], _dptr(V), self._sw,
                                                     share, stream or 0, _dptr(out)),
                    "pwa_pieces_points")
        return out

    def hessian_cached(self, var_values, step=1e-4, stream=None):
        """(nll, grad, Hessian) of the cached form, the Hessian by 4-point
        differences of the adjoint gradient (C++ loop, pwa_hessian_cached)."""
        v = np.ascontiguousarray(var_values, np.float64)
        P = self._n_train
        nll = ctypes.c_double()
        g = np.zeros(P)
        H = np.zeros((P, P))
        self._check(load_library().pwa_hessian_cached(self.h, _dptr(v), self._sw, float(step),
                                                      stream or 0, ctypes.byref(nll), _dptr(g),
                                                      _dptr(H)), "pwa_hessian_cached")
        return nll.value, g, H

    def hessian_cached_exact(self, var_values, stream=None):
        """(nll, grad, Hessian) of the cached form with the exact Hessian in
        the coupling parts: one pass of the Hessian-sums kernel over the
        column cache, then the MC term and the coupling derivatives on the
        host (pwa_hessian_cached_exact)."""
        v = np.ascontiguousarray(var_values, np.float64)
        P = self._n_train
        nll = ctypes.c_double()
        g = np.zeros(P)
        H = np.zeros((P, P))
        self._check(load_library().pwa_hessian_cached_exact(self.h, _dptr(v), self._sw,
                                                            stream or 0, ctypes.byref(nll),
                                                            _dptr(g), _dptr(H)),
                    "pwa_hessian_cached_exact")
        return nll.value, g, H

    def hess_sums_cached(self, var_values, stream=None):
        """The data sums of the exact Hessian (pwa_hess_sums_cached):
        S0, S1 (re, im per column), upper triangles of the two 2K x 2K sums."""
        v = np.ascontiguousarray(var_values, np.float64)
        W = 2 * self.code.ncol
        out = np.zeros(1 + W + W * (W + 1))
        self._check(load_library().pwa_hess_sums_cached(self.h, _dptr(v), stream or 0,
                                                        _dptr(out)), "pwa_hess_sums_cached")
        return out

    # ------------------------------------------------------------ dataset step
    def fields_from_p4(self, p4, charge=None):
        """Event fields (n_fields, N) on the device from final-state momenta
        ``p4``: CUDA tensor (N, n_final, 4), finals in the plan's order.
        For data with charges, ``charge`` (default all +1) fills the charge
        field, or with cp_trans parity-transforms the charge < 0 events first
        (``tf_pwa/cal_angle.py:569-573``)."""
        import torch

        n = p4.shape[0]
        p4 = p4.to(torch.float64)
        ci = self.plan.charge_index
        ch = None
        if self.plan.use_charge and charge is not None:
            ch = torch.as_tensor(charge, dtype=torch.float64, device=p4.device)
            if self.plan.cp_trans:
                sgn = torch.where(ch > 0, 1.0, -1.0).to(torch.float64)[:, None, None]
                p4 = torch.cat([p4[:, :, :1], p4[:, :, 1:] * sgn], 2)
        soa = p4.permute(1, 2, 0).reshape(-1, n).contiguous()
        out = torch.empty((self.plan.n_fields, n), dtype=torch.float64, device=p4.device)
        self._check(load_library().pwa_fields_from_p4(self.h, soa.data_ptr(), n, n,
                                                      out.data_ptr(), n, 0),
                    "pwa_fields_from_p4")
        if ch is not None and ci is not None:
            out[ci] = ch
        return out

    def toy_select(self, C, seed, first, n, fmax, flat, out):
        """Accept flags / |A|^2 of candidates first..first+n into the CUDA
        tensor ``out`` (see pwa_toy_select)."""
        Cp = None if C is None else _dptr(np.ascontiguousarray(C, np.float64))
        self._check(load_library().pwa_toy_select(self.h, Cp, int(seed), int(first), int(n),
                                                  float(fmax), int(flat), out.data_ptr(),
                                                  0), "pwa_toy_select")

    def toy_fields(self, seed, idx, with_p4=False):
        """Fields (n_fields, len(idx)) and optionally momenta (len, n_final, 4)
        of candidates ``idx`` (int64 CUDA tensor)."""
        import torch

        n = idx.shape[0]
        idx = idx.to(torch.int64).contiguous()
        out = torch.empty((self.plan.n_fields, n), dtype=torch.float64, device=idx.device)
        p4 = None
        if with_p4:
            p4 = torch.empty((4 * self.code.kin.nfin, n), dtype=torch.float64, device=idx.device)
        self._check(load_library().pwa_toy_fields(self.h, int(seed), idx.data_ptr(), n,
                                                  out.data_ptr(), n,
                                                  None if p4 is None else p4.data_ptr(), n,
                                                  0), "pwa_toy_fields")
        if with_p4:
            return out, p4.reshape(self.code.kin.nfin, 4, n).permute(2, 0, 1)
        return out

    def fma_peak(self, precision=PLAIN_F64, iters=1 << 16):
        """Measured peak FMA throughput (flop/s) of the CUDA cores in FP64
        (PLAIN_F64) or FP32 (MIXED_F32)."""
        out = ctypes.c_double()
        self._check(load_library().pwa_fma_peak(self.h, precision, int(iters), 0,
                                                ctypes.byref(out)), "pwa_fma_peak")
        return out.value

    def autotune_cached(self, reps=8):
        """Time every configuration of the cached data-term kernel on this
        plan's column cache and keep the fastest (pwa_autotune_cached).
        Returns the per-configuration microseconds and the choice
        (variant, ring depth, blocks per SM).  The choice is remembered per
        model source and tile count for the process, and across processes
        in PWA_CUBIN_CACHE when that directory is set."""
        key = self._tune_key()
        hit = _TUNED.get(key) or _tune_disk_read(key)
        if hit is not None:
            self.set_cached_config(*hit)
            _TUNED[key] = hit
            return None, tuple(hit)
        ck = np.ascontiguousarray(np.stack([self._ck.real, self._ck.imag], 1).reshape(-1))
        n = ctypes.c_int()
        out = np.zeros(32)
        self._check(load_library().pwa_autotune_cached(self.h, _dptr(ck), int(reps), 0,
                                                       ctypes.byref(n), _dptr(out)),
                    "pwa_autotune_cached")
        cfg = self.cached_config()
        _TUNED[key] = cfg
        _tune_disk_write(key, cfg)
        return out[:n.value].copy(), cfg

    def _tune_key(self):
        import hashlib

        ntiles = (self._n_data + self.tpb - 1) // self.tpb
        return hashlib.sha1(self.src.encode()).hexdigest()[:20] + f"_{ntiles}"

    def cached_config(self):
        out = (ctypes.c_int * 3)()
        self._check(load_library().pwa_cached_config(self.h, out), "pwa_cached_config")
        return tuple(out)

    def set_cached_config(self, variant, stages=0, bps=0):
        self._check(load_library().pwa_set_cached_config(self.h, int(variant), int(stages),
                                                         int(bps)), "pwa_set_cached_config")

    def set_gram_method(self, method):
        """0: FP64 Gram on the CUDA cores; 1: tensor cores (int8 slices,
        exact integer accumulation); -1: automatic."""
        self._check(load_library().pwa_set_gram_method(self.h, int(method)),
                    "pwa_set_gram_method")

    def set_cached_variant(self, variant):
        self._check(load_library().pwa_set_cached_variant(self.h, int(variant)),
                    "pwa_set_cached_variant")

    def eval_cached_enqueue(self, ck, stream=None):
        ck = np.ascontiguousarray(ck, np.float64)
        self._check(load_library().pwa_eval_cached_enqueue(self.h, _dptr(ck), stream or 0),
                    "pwa_eval_cached_enqueue")

    # ----------------------------------------------------- serving (pool)
    def pool_reserve(self, n_tiles):
        self._check(load_library().pwa_pool_reserve(self.h, int(n_tiles)), "pwa_pool_reserve")

    def pool_alloc(self, n_events):
        """(first_tile, n_tiles), or None when the pool has no free run."""
        a, b = ctypes.c_longlong(), ctypes.c_longlong()
        rc = load_library().pwa_pool_alloc(self.h, int(n_events), ctypes.byref(a), ctypes.byref(b))
        if rc == 5:  # PWA_ERR_OOM
            return None
        self._check(rc, "pwa_pool_alloc")
        return a.value, b.value

    def pool_free(self, first_tile):
        self._check(load_library().pwa_pool_free(self.h, int(first_tile)), "pwa_pool_free")

    def pool_fill(self, first_tile, C, xm_ptr, xa_ptr, w_ptr, n, ld, stream=None):
        C = np.ascontiguousarray(C, np.float64)
        self._check(load_library().pwa_pool_fill(self.h, int(first_tile), _dptr(C), xm_ptr,
                                                 xa_ptr, w_ptr, int(n), int(ld), stream or 0),
                    "pwa_pool_fill")

    def pieces_multi(self, first_tiles, n_tiles, var_rows, sws, mc_share=1.0, stream=None):
        ft = np.ascontiguousarray(first_tiles, np.int64)
        nt = np.ascontiguousarray(n_tiles, np.int64)
        V = np.ascontiguousarray(var_rows, np.float64)
        sw = np.ascontiguousarray(sws, np.float64)
        out = np.zeros((len(ft), 3 + 2 * self._n_train))
        llp = ctypes.POINTER(ctypes.c_longlong)
        self._check(load_library().pwa_pieces_multi(
            self.h, len(ft), ft.ctypes.data_as(llp), nt.ctypes.data_as(llp), _dptr(V), _dptr(sw),
            mc_share, stream or 0, _dptr(out)), "pwa_pieces_multi")
        return out

    def set_gram(self, vals):
        """Build the MC Gram matrix at the current masses/widths."""
        C = self.consts(vals)
        self._gram = self.build_gram(C)
        return self._gram


# cached-kernel configurations chosen by Engine.autotune_cached, per model
# source and tile count
_TUNED = {}


def _tune_path(key):
    d = os.environ.get("PWA_CUBIN_CACHE")
    return os.path.join(d, f"pwa_tune_{key}.txt") if d else None


def _tune_disk_read(key):
    p = _tune_path(key)
    try:
        with open(p) as f:
            v = tuple(int(x) for x in f.read().split())
        return v if len(v) == 3 else None
    except (OSError, TypeError, ValueError):
        return None


def _tune_disk_write(key, cfg):
    p = _tune_path(key)
    if p:
        try:
            with open(p + ".tmp", "w") as f:
                f.write(" ".join(str(int(x)) for x in cfg))
            os.replace(p + ".tmp", p)
        except OSError:
            pass


def read_dat(path):
    """All numbers of a text momentum file, parsed by the native library on
    all host cores (pwa_read_dat); a flat FP64 array in file order."""
    lib = load_library()
    n = ctypes.c_longlong()
    fn = os.fsencode(path)
    if lib.pwa_read_dat(fn, None, 0, ctypes.byref(n)) != 0:
        raise PWAError(lib.pwa_last_error(None).decode(errors="replace"))
    out = np.empty(n.value, np.float64)
    if lib.pwa_read_dat(fn, out.ctypes.data, n.value, ctypes.byref(n)) != 0:
        raise PWAError(lib.pwa_last_error(None).decode(errors="replace"))
    return out
