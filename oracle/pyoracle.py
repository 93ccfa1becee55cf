"""ctypes wrapper around liboracle.so (the C restatement in ddamg_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA library.  Imported by tests/,
__graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the library.
All complex arrays are numpy complex128, layout [site][dof] with site = x*Nt + t.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_c_dp = ctypes.POINTER(ctypes.c_double)
_c_ip = ctypes.POINTER(ctypes.c_int)


class OracleConstants(ctypes.Structure):
    _fields_ = [
        ("sap_gmres_m", ctypes.c_int),
        ("sap_gmres_restarts", ctypes.c_int),
        ("sap_gmres_tol", ctypes.c_double),
        ("sap_tv_iters", ctypes.c_int),
        ("coarse_m", ctypes.c_int),
        ("coarse_restarts", ctypes.c_int),
        ("coarse_tol", ctypes.c_double),
        ("nu1", ctypes.c_int),
        ("nu2", ctypes.c_int),
        ("kc_m", ctypes.c_int),
        ("kc_restarts", ctypes.c_int),
        ("kc_tol", ctypes.c_double),
        ("smoother_tol", ctypes.c_double),
    ]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _c_ip, _c_dp,
                                 ctypes.POINTER(OracleConstants)]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for f in ("orc_level_sites", "orc_level_dof", "orc_level_ntest"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_int
        L.orc_dirac.argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dp, _c_dp]
        for f in ("orc_level_op", "orc_restrict", "orc_prolong"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dp, _c_dp]
        L.orc_set_tvec.argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dp]
        L.orc_get_tvec.argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dp]
        L.orc_orthonormalize.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_make_coarse_links.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_get_links.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_dp]
        L.orc_set_links.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_dp]
        L.orc_setup.argtypes = [ctypes.c_void_p, _c_dp, ctypes.c_long]
        L.orc_setup.restype = ctypes.c_int
        L.orc_setup_random_count.argtypes = [ctypes.c_void_p]
        L.orc_setup_random_count.restype = ctypes.c_long
        L.orc_sap.argtypes = [ctypes.c_void_p, ctypes.c_int, _c_dp, _c_dp, ctypes.c_int, ctypes.c_double]
        L.orc_sap.restype = ctypes.c_int
        L.orc_coarse_gmres.argtypes = [ctypes.c_void_p, _c_dp, _c_dp]
        L.orc_coarse_gmres.restype = ctypes.c_int
        L.orc_vcycle.argtypes = [ctypes.c_void_p, _c_dp, _c_dp]
        L.orc_kcycle.argtypes = [ctypes.c_void_p, _c_dp, _c_dp]
        L.orc_solve.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _c_dp,
                                _c_dp]
        L.orc_solve.restype = ctypes.c_int
        L.orc_gmres_plain.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _c_dp, _c_dp]
        L.orc_gmres_plain.restype = ctypes.c_int
        L.orc_link_gradient.argtypes = [ctypes.c_void_p, _c_dp, _c_dp, _c_dp]
        L.orc_apply_multilevel.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, _c_dp, _c_dp,
                                           _c_dp]
        L.orc_apply_multilevel.restype = ctypes.c_int
        L.orc_fgmres_sap.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_double, _c_dp, _c_dp]
        L.orc_fgmres_sap.restype = ctypes.c_int
        L.orc_sap_fine.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _c_dp, _c_dp, ctypes.c_int,
                                   ctypes.c_double]
        L.orc_sap_fine.restype = ctypes.c_int
        L.orc_dirac_plain.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _c_dp, ctypes.c_int, _c_dp, _c_dp]
        L.orc_bicgstab.argtypes = [ctypes.c_void_p, _c_dp, _c_dp, _c_dp, ctypes.c_int, ctypes.c_double]
        L.orc_bicgstab.restype = ctypes.c_int
        L.orc_cg_normal.argtypes = [ctypes.c_void_p, _c_dp, _c_dp, ctypes.c_int, ctypes.c_double]
        L.orc_cg_normal.restype = ctypes.c_int
        L.orc_rng.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64]
        L.orc_rng.restype = ctypes.c_uint64
        L.orc_metropolis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_uint64,
                                     ctypes.c_double, _c_dp]
        L.orc_metropolis.restype = ctypes.c_double
        L.orc_plaquette.argtypes = [ctypes.c_int, ctypes.c_int, _c_dp]
        L.orc_plaquette.restype = ctypes.c_double
        L.orc_gaussian.argtypes = [ctypes.c_long, ctypes.c_uint64, _c_dp]
        L.orc_uniform.argtypes = [ctypes.c_long, ctypes.c_uint64, _c_dp]
        L.orc_write_binary.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _c_dp]
        L.orc_read_binary.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _c_dp]
        L.orc_read_binary.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_c_dp)


def default_constants():
    c = OracleConstants()
    c.sap_gmres_m, c.sap_gmres_restarts, c.sap_gmres_tol = 5, 5, 1e-3
    c.sap_tv_iters = 4
    c.coarse_m, c.coarse_restarts, c.coarse_tol = 400, 10, 0.1
    c.nu1, c.nu2 = 0, 2
    c.kc_m, c.kc_restarts, c.kc_tol = 5, 2, 0.1
    c.smoother_tol = 1e-10
    return c


# ---------------------------------------------------------------- inputs
def dirac(Nx, Nt, m0, U, phi, dagger=False):
    """D_phi / D_dagger_phi (src/dirac_operator.cpp:24-85) without building a hierarchy."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    phi = np.ascontiguousarray(phi, dtype=np.complex128)
    out = np.zeros_like(phi)
    lib().orc_dirac_plain(Nx, Nt, m0, _p(U), int(bool(dagger)), _p(phi), _p(out))
    return out


def metropolis(Nx, Nt, beta, sweeps, seed, delta=1.0):
    th = np.zeros(2 * Nx * Nt)
    acc = lib().orc_metropolis(Nx, Nt, beta, sweeps, seed, delta, _p(th))
    return th, acc


def plaquette(Nx, Nt, theta):
    return lib().orc_plaquette(Nx, Nt, _p(np.ascontiguousarray(theta, dtype=np.float64)))


def links_from_theta(theta):
    return np.exp(1j * np.asarray(theta, dtype=np.float64))


def gaussian(n, seed):
    out = np.zeros(2 * n)
    lib().orc_gaussian(n, seed, _p(out))
    return out.view(np.complex128)


def uniform(n, seed):
    out = np.zeros(2 * n)
    lib().orc_uniform(n, seed, _p(out))
    return out.view(np.complex128)


def write_binary(path, Nx, Nt, field):
    f = np.ascontiguousarray(field, dtype=np.complex128)
    return lib().orc_write_binary(path.encode(), Nx, Nt, f.ctypes.data_as(_c_dp))


def read_binary(path, Nx, Nt):
    f = np.zeros(2 * Nx * Nt, dtype=np.complex128)
    rc = lib().orc_read_binary(path.encode(), Nx, Nt, f.ctypes.data_as(_c_dp))
    if rc != 0:
        raise IOError(f"read_binary({path}) failed: {rc}")
    return f


def parse_params_text(text):
    rows = []
    for line in text.splitlines():
        toks = line.split()
        if not toks:
            continue
        rows.append([int(v) for v in toks[:6]])
    return rows


class Oracle:
    """One multigrid hierarchy of the CPU restatement."""

    def __init__(self, Nx, Nt, levels, m0, rows, U, constants=None):
        self.Nx, self.Nt, self.levels, self.m0 = Nx, Nt, levels, m0
        r = np.ascontiguousarray(np.array(rows, dtype=np.int32).reshape(-1))
        self._U = np.ascontiguousarray(U, dtype=np.complex128)
        self.constants = constants or default_constants()
        self.h = lib().orc_create(levels, m0, Nx, Nt, r.ctypes.data_as(_c_ip), self._U.ctypes.data_as(_c_dp),
                                  ctypes.byref(self.constants))
        if not self.h:
            raise ValueError("orc_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def sites(self, l):
        return lib().orc_level_sites(self.h, l)

    def dof(self, l):
        return lib().orc_level_dof(self.h, l)

    def ntest(self, l):
        return lib().orc_level_ntest(self.h, l)

    def size(self, l):
        return self.sites(l) * self.dof(l)

    def _out(self, n):
        return np.zeros(n, dtype=np.complex128)

    def dirac(self, phi, dagger=False):
        phi = np.ascontiguousarray(phi, dtype=np.complex128)
        out = self._out(phi.size)
        lib().orc_dirac(self.h, int(dagger), _p(phi), _p(out))
        return out

    def level_op(self, l, v):
        v = np.ascontiguousarray(v, dtype=np.complex128)
        out = self._out(self.size(l))
        lib().orc_level_op(self.h, l, _p(v), _p(out))
        return out

    def restrict(self, l, v):
        v = np.ascontiguousarray(v, dtype=np.complex128)
        out = self._out(self.size(l + 1))
        lib().orc_restrict(self.h, l, _p(v), _p(out))
        return out

    def prolong(self, l, vc):
        vc = np.ascontiguousarray(vc, dtype=np.complex128)
        out = self._out(self.size(l))
        lib().orc_prolong(self.h, l, _p(vc), _p(out))
        return out

    def setup_random_count(self):
        return lib().orc_setup_random_count(self.h)

    def setup(self, rnd):
        rnd = np.ascontiguousarray(rnd, dtype=np.complex128)
        rc = lib().orc_setup(self.h, _p(rnd), rnd.size)
        if rc != 0:
            raise ValueError("random stream too short")

    def get_tvec(self, l):
        out = self._out(self.ntest(l) * self.size(l))
        lib().orc_get_tvec(self.h, l, _p(out))
        return out

    def set_tvec(self, l, tv):
        tv = np.ascontiguousarray(tv, dtype=np.complex128)
        lib().orc_set_tvec(self.h, l, _p(tv))

    def orthonormalize(self, l):
        lib().orc_orthonormalize(self.h, l)

    def make_coarse_links(self, l):
        lib().orc_make_coarse_links(self.h, l)

    def get_links(self, l, which):
        C = self.dof(l) // 2
        n = self.sites(l) * 4 * C * C * (1 if which == 1 else 2)
        out = self._out(n)
        lib().orc_get_links(self.h, l, which, _p(out))
        return out

    def set_links(self, l, which, arr):
        arr = np.ascontiguousarray(arr, dtype=np.complex128)
        lib().orc_set_links(self.h, l, which, _p(arr))

    def sap(self, l, v, x0=None, nu=2, tol=1e-10):
        v = np.ascontiguousarray(v, dtype=np.complex128)
        x = self._out(self.size(l)) if x0 is None else np.array(x0, dtype=np.complex128)
        it = lib().orc_sap(self.h, l, _p(v), _p(x), nu, tol)
        return x, it

    def coarse_gmres(self, b):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = self._out(b.size)
        it = lib().orc_coarse_gmres(self.h, _p(b), _p(x))
        return x, it

    def vcycle(self, eta):
        eta = np.ascontiguousarray(eta, dtype=np.complex128)
        psi = self._out(eta.size)
        lib().orc_vcycle(self.h, _p(eta), _p(psi))
        return psi

    def kcycle(self, eta):
        eta = np.ascontiguousarray(eta, dtype=np.complex128)
        psi = self._out(eta.size)
        lib().orc_kcycle(self.h, _p(eta), _p(psi))
        return psi

    def solve(self, b, cycle=0, m=20, restarts=50, tol=1e-10):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = self._out(b.size)
        it = lib().orc_solve(self.h, cycle, m, restarts, tol, _p(b), _p(x))
        return x, it

    def gmres_plain(self, b, m=50, restarts=200, tol=1e-10):
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = self._out(b.size)
        it = lib().orc_gmres_plain(self.h, m, restarts, tol, _p(b), _p(x))
        return x, it

    def bicgstab(self, b, x0=None, max_iter=10000, tol=1e-10):
        """bi_cgstab (src/conjugate_gradient.cpp:87-176); returns (x, k+1 or max_iter)."""
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x0 = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.complex128)
        x = self._out(b.size)
        it = lib().orc_bicgstab(self.h, _p(b), _p(x0), _p(x), max_iter, tol)
        return x, it

    def cg_normal(self, phi, max_iter=10000, tol=1e-10):
        """conjugate_gradient (src/conjugate_gradient.cpp:4-83) on D^dagger D x = phi from x0 = phi;
        returns (x, k+1 or 0)."""
        phi = np.ascontiguousarray(phi, dtype=np.complex128)
        x = self._out(phi.size)
        it = lib().orc_cg_normal(self.h, _p(phi), _p(x), max_iter, tol)
        return x, it

    def apply_multilevel(self, rhs, cycle=0, it=100, tol=1e-10, x0=None):
        """AlgebraicMG::applyMultilevel (src/amg.cpp:177-243); returns (x, cycles run, rel. residual)."""
        rhs = np.ascontiguousarray(rhs, dtype=np.complex128)
        x = self._out(rhs.size) if x0 is None else np.array(x0, dtype=np.complex128)
        rel = ctypes.c_double(0)
        n = lib().orc_apply_multilevel(self.h, cycle, it, tol, _p(rhs), _p(x), ctypes.byref(rel))
        return x, n, rel.value

    def fgmres_sap(self, b, sap_x=4, sap_t=4, m=20, restarts=50, tol=1e-10):
        """FGMRES_SAP (include/sap.h:236-333); returns (x, iterations)."""
        b = np.ascontiguousarray(b, dtype=np.complex128)
        x = self._out(b.size)
        it = lib().orc_fgmres_sap(self.h, sap_x, sap_t, m, restarts, tol, _p(b), _p(x))
        return x, it

    def sap_fine(self, v, sap_x, sap_t, x0=None, nu=2, tol=1e-10):
        """SAP_C::SAP of SAP_fine_level over sap_x x sap_t blocks; returns (x, SAP's value)."""
        v = np.ascontiguousarray(v, dtype=np.complex128)
        x = self._out(v.size) if x0 is None else np.array(x0, dtype=np.complex128)
        it = lib().orc_sap_fine(self.h, sap_x, sap_t, _p(v), _p(x), nu, tol)
        return x, it

    def link_gradient(self, psi, lam):
        psi = np.ascontiguousarray(psi, dtype=np.complex128)
        lam = np.ascontiguousarray(lam, dtype=np.complex128)
        out = np.zeros(2 * self.Nx * self.Nt)
        lib().orc_link_gradient(self.h, _p(psi), _p(lam), _p(out))
        return out
