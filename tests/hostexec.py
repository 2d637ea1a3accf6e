"""Build and call the generated model code on the host (test infrastructure).

The model source that the library compiles with NVRTC for the GPU is
compiled here with g++, after host stand-ins of the CUDA built-ins
(``tests/hostcode/shim.h``) and the library's device header, with the loops
of ``tests/hostcode/harness.cpp`` around it.  The tests run it on the golden
events: the code generator's arithmetic (forward amplitude, adjoint,
columns, kinematics, generator) is checked against the reference's numbers
on CPU, one event at a time in FP64 (or FP32 where the kernel uses FP32).
Compiled without optimisation: the straight-line model code builds in
seconds that way, and x86-64 double arithmetic is the same at any level.
"""
import ctypes
import hashlib
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOSTCODE = os.path.join(ROOT, "tests", "hostcode")
DEVICE_HEADER = os.path.join(ROOT, "tf-pwa_b200", "csrc", "pwa_device.cuh")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class HostModel:
    """The generated functions of one ModelCode, compiled for the host."""

    def __init__(self, code, build_dir):
        self.code = code
        parts = []
        for path in (os.path.join(HOSTCODE, "shim.h"), DEVICE_HEADER):
            with open(path) as f:
                parts.append(f.read())
        parts.append(f"#define PWA_NANGLE_ROWS {max(len(code.angle_fields), 1)}")
        parts.append(code.source())
        with open(os.path.join(HOSTCODE, "harness.cpp")) as f:
            parts.append(f.read())
        text = "\n".join(parts)
        tag = hashlib.sha1(text.encode()).hexdigest()[:16]
        os.makedirs(build_dir, exist_ok=True)
        src = os.path.join(build_dir, f"hx_{tag}.cpp")
        so = os.path.join(build_dir, f"hx_{tag}.so")
        if not os.path.exists(so):
            with open(src, "w") as f:
                f.write(text)
            r = subprocess.run(["g++", "-std=c++17", "-O0", "-fPIC", "-shared",
                                "-Wno-unknown-pragmas", "-Wno-pragma-once-outside-header",
                                src, "-o", so + ".tmp"], capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError("host build of the generated model failed:\n" + r.stderr[-4000:])
            os.replace(so + ".tmp", so)
        lib = ctypes.CDLL(so)
        ll, i, dp = ctypes.c_longlong, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
        lib.hx_sums.argtypes = [dp, dp, dp, dp, ll, ll, ll, i, i, dp]
        lib.hx_amp.argtypes = [dp, dp, dp, ll, ll, i, dp]
        lib.hx_columns.argtypes = [dp, dp, dp, ll, ll, dp]
        lib.hx_columns_ns.argtypes = [dp, dp, dp, ll, ll, dp]
        lib.hx_shapes.argtypes = [dp, dp, ll, ll, dp]
        lib.hx_kin.argtypes = [dp, ll, dp]
        self.has_toy = hasattr(lib, "hx_toy")
        if self.has_toy:
            lib.hx_toy.argtypes = [dp, ctypes.c_ulonglong, ll, ll, dp, dp, dp, dp, dp, dp]
        self.lib = lib

    def _split(self, x):
        c = self.code
        x = np.asarray(x, np.float64)
        n = x.shape[1]
        xm = np.ascontiguousarray(x[c.mass_fields]) if c.mass_fields else np.zeros((1, n))
        xa = np.ascontiguousarray(x[c.angle_fields]) if c.angle_fields else np.zeros((1, n))
        return xm, xa

    def sums(self, C, x, w, n_data, f32=False, stash=False):
        """(data sums, MC sums) of the plain kernel's accumulators over the
        events x[:, :n_data] (data, weights w) and x[:, n_data:] (MC)."""
        C = np.ascontiguousarray(C, np.float64)
        xm, xa = self._split(x)
        w = np.ascontiguousarray(w, np.float64)
        n = xm.shape[1]
        nacc = self.code.nacc
        out = np.zeros(2 * nacc)
        self.lib.hx_sums(_dp(C), _dp(xm), _dp(xa), _dp(w), n_data, n, n, int(f32), int(stash),
                         _dp(out))
        return out[:nacc], out[nacc:]

    def amp(self, C, x, f32=False):
        C = np.ascontiguousarray(C, np.float64)
        xm, xa = self._split(x)
        n = xm.shape[1]
        out = np.zeros(2 * n * self.code.nout)
        self.lib.hx_amp(_dp(C), _dp(xm), _dp(xa), n, n, int(f32), _dp(out))
        return (out[0::2] + 1j * out[1::2]).reshape(n, self.code.nout)

    def pdf(self, C, x, f32=False):
        """sum |A|^2, or with a polarised parent sum_l A_al rho_ab A_bl^*
        with rho taken from the constant block."""
        a = self.amp(C, x, f32)
        c = self.code
        if not c.pol_names:
            return np.sum(np.abs(a) ** 2, axis=1)
        na = c.na
        rho = np.array([[C[c.consts.index[f"rho{i}_{j}.re"]] + 1j * C[c.consts.index[f"rho{i}_{j}.im"]]
                         for j in range(na)] for i in range(na)])
        a = a.reshape(a.shape[0], na, -1)
        return np.real(np.einsum("nal,ab,nbl->n", a, rho, np.conj(a)))

    def columns(self, C, x):
        C = np.ascontiguousarray(C, np.float64)
        xm, xa = self._split(x)
        n = xm.shape[1]
        K, O = self.code.ncol, self.code.nout
        out = np.zeros(2 * n * K * O)
        self.lib.hx_columns(_dp(C), _dp(xm), _dp(xa), n, n, _dp(out))
        return (out[0::2] + 1j * out[1::2]).reshape(n, K, O)

    def columns_ns(self, C, x):
        """Columns without their chains' lineshapes (model_columns_ns)."""
        C = np.ascontiguousarray(C, np.float64)
        xm, xa = self._split(x)
        n = xm.shape[1]
        K, O = self.code.ncol, self.code.nout
        out = np.zeros(2 * n * K * O)
        self.lib.hx_columns_ns(_dp(C), _dp(xm), _dp(xa), n, n, _dp(out))
        return (out[0::2] + 1j * out[1::2]).reshape(n, K, O)

    def shapes(self, C, x):
        """(BW (n, n_chain), DM (n, n_sres), DG (n, n_sres)) of model_shapes."""
        C = np.ascontiguousarray(C, np.float64)
        xm, _ = self._split(x)
        n = xm.shape[1]
        nch, ns = len(self.code.group), max(len(self.code.shape_res), 1)
        W = nch + 2 * ns
        out = np.zeros(2 * n * W)
        self.lib.hx_shapes(_dp(C), _dp(xm), n, n, _dp(out))
        z = (out[0::2] + 1j * out[1::2]).reshape(n, W)
        return z[:, :nch], z[:, nch:nch + ns], z[:, nch + ns:]

    def kin(self, p4):
        """(N, n_final, 4) momenta in dat_order -> (n_fields, N) fields."""
        p4 = np.asarray(p4, np.float64)
        n, nf = p4.shape[0], p4.shape[1]
        rows = np.ascontiguousarray(p4.transpose(1, 2, 0).reshape(4 * nf, n))
        out = np.zeros((self.code.plan.n_fields, n))
        self.lib.hx_kin(_dp(rows), n, _dp(out))
        return out

    def toy(self, C, seed, first, n):
        """Candidates first .. first + n - 1: dict of the phase-space weight,
        the acceptance uniforms, sum |A|^2, momenta (N, n_final, 4) and fields."""
        C = np.ascontiguousarray(C, np.float64)
        out = {k: np.zeros(n) for k in ("wps", "u_ps", "u_amp", "f")}
        nf = self.code.plan.n_fields
        nfin = self.code.kin.nfin
        p4 = np.zeros(4 * nfin * n)
        fields = np.zeros(nf * n)
        self.lib.hx_toy(_dp(C), seed, first, n, _dp(out["wps"]), _dp(out["u_ps"]),
                        _dp(out["u_amp"]), _dp(out["f"]), _dp(p4), _dp(fields))
        out["p4"] = p4.reshape(nfin, 4, n).transpose(2, 0, 1)
        out["fields"] = fields.reshape(nf, n)
        return out
