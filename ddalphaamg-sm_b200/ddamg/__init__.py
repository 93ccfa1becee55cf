"""Python host API of the B200 DD-alphaAMG solver for the 2D Schwinger-model Wilson-Dirac operator.

A thin layer over the C ABI (include/ddamg.h, libddamg.so) that keeps the reference's
operator names (JFNCastellanos/DDalphaAMG-SM): D_phi / D_dagger_phi, Level.D_operator,
P_vc / Pdagg_v, SAP, setUpPhase, v_cycle / k_cycle, FGMRES with a multigrid preconditioner.
Fields are numpy complex128 arrays laid out [site][dof] with site = x*Nt + t (x slow),
mu = 0 along t, mu = 1 along x.  Every call runs on the GPU; a missing library raises.
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import CYCLE_K, CYCLE_V, PREC_DOUBLE, PREC_MIXED, DDAMGError, Params, SolveInfo, check

__all__ = ["Solver", "Params", "SolveInfo", "DDAMGError", "default_params", "read_parameters", "read_binary",
           "write_binary", "from_halo", "to_halo", "gauge_metropolis", "gaussian_field", "PREC_DOUBLE", "PREC_MIXED", "CYCLE_V", "CYCLE_K"]


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def default_params(Nx=0, Nt=0, levels=2, m0=0.0, rows=(), **kw):
    """Reference defaults (src/variables.cpp:100-134) plus geometry; keyword overrides any field."""
    p = Params()
    check(_lib.load().ddamg_params_default(ctypes.byref(p)))
    p.Nx, p.Nt, p.levels, p.m0 = Nx, Nt, levels, m0
    for i, r in enumerate(rows):
        for k in range(6):
            p.rows[i][k] = int(r[k])
    for k, v in kw.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def read_parameters(path, levels, params=None):
    """readParameters (include/params.h:18-111)."""
    p = params if params is not None else default_params()
    check(_lib.load().ddamg_parse_params_file(path.encode(), levels, ctypes.byref(p)))
    return p


def read_binary(path, Nx, Nt):
    """read_binary (src/io.cpp:4-55): returns [site][mu] complex128."""
    out = np.zeros(2 * Nx * Nt, dtype=np.complex128)
    check(_lib.load().ddamg_read_binary(path.encode(), Nx, Nt, _dp(out)))
    return out


def write_binary(path, Nx, Nt, field):
    f = _c(field)
    check(_lib.load().ddamg_write_binary(path.encode(), Nx, Nt, _dp(f)))


def from_halo(halo, Nx, Nt, dof):
    """The reference's halo spinor layout (x, t in 1..N of an (Nx+2) x (Nt+2) grid) -> compact [site][dof]."""
    halo = _c(halo)
    out = np.empty(Nx * Nt * dof, dtype=np.complex128)
    check(_lib.load().ddamg_from_halo(_dp(halo), Nx, Nt, dof, _dp(out)))
    return out


def to_halo(compact, Nx, Nt, dof):
    """compact [site][dof] -> the reference's halo spinor layout (halo sites zero)."""
    compact = _c(compact)
    out = np.empty((Nx + 2) * (Nt + 2) * dof, dtype=np.complex128)
    check(_lib.load().ddamg_to_halo(_dp(compact), Nx, Nt, dof, _dp(out)))
    return out


def gauge_metropolis(Nx, Nt, beta, sweeps, seed, delta=1.0, device=0):
    """U(1) Metropolis on the GPU; returns (theta [site][mu], acceptance of the last sweep)."""
    th = np.zeros(2 * Nx * Nt)
    acc = ctypes.c_double(0)
    check(_lib.load().ddamg_gauge_metropolis(Nx, Nt, beta, sweeps, seed, delta, _dp(th), ctypes.byref(acc), device))
    return th, acc.value


def gaussian_field(n, seed):
    out = np.zeros(n, dtype=np.complex128)
    check(_lib.load().ddamg_gaussian_field(n, seed, _dp(out)))
    return out


# iteration counters of the metadata file (src/variables.cpp:9-17), in ddamg_counter order
COUNTER_NAMES = ("CG", "BiCG", "GMRES", "SAP", "FGMRES_SAP", "vCycle", "kCycle")


def set_stencil_kernel(kind):
    """D_W kernel choice, process-wide: 0 default, 1 register kernels, 2 staged tiles (bulk copies into
    shared memory)."""
    check(_lib.load().ddamg_set_stencil_kernel(int(kind)))


def stencil_kernel():
    k = ctypes.c_int(0)
    check(_lib.load().ddamg_get_stencil_kernel(ctypes.byref(k)))
    return k.value


def write_metadata(params, counts, cycle, tol, path=None):
    """writeMetadata (src/io.cpp:72-145) from parameters and counters alone (host only, no device)."""
    c = (ctypes.c_longlong * 7)(*[int(v) for v in counts])
    check(_lib.load().ddamg_write_metadata_params(ctypes.byref(params), c, cycle, tol,
                                                  path.encode() if path else None))


class Solver:
    """One multigrid hierarchy on one GPU (AlgebraicMG + FGMRES_AMG of the reference)."""

    def __init__(self, params):
        self.L = _lib.load()
        self.params = params
        h = ctypes.c_void_p()
        check(self.L.ddamg_create(ctypes.byref(params), ctypes.byref(h)))
        self.h = h
        self.Nx, self.Nt, self.levels = params.Nx, params.Nt, params.levels
        self._sizes = [self.Nx * self.Nt * 2]
        self._ntest = []
        for l in range(self.levels - 1):
            r = params.rows[l]
            self._ntest.append(r[3])
            self._sizes.append(r[1] * r[2] * 2 * r[3])

    def close(self):
        if getattr(self, "h", None):
            self.L.ddamg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def size(self, level):
        return self._sizes[level]

    # ------------------------------------------------------------ inputs
    def load_gauge(self, U):
        U = _c(U)
        check(self.L.ddamg_load_gauge(self.h, _dp(U)))

    # ------------------------------------------------------------ operators
    def D_phi(self, phi, nrhs=1):
        phi = _c(phi)
        out = np.empty_like(phi)
        check(self.L.ddamg_apply_dirac(self.h, 0, _dp(phi), _dp(out), nrhs))
        return out

    def D_dagger_phi(self, phi, nrhs=1):
        phi = _c(phi)
        out = np.empty_like(phi)
        check(self.L.ddamg_apply_dirac(self.h, 1, _dp(phi), _dp(out), nrhs))
        return out

    def D_operator(self, level, v):
        v = _c(v)
        out = np.empty(self.size(level), dtype=np.complex128)
        check(self.L.ddamg_apply_level_op(self.h, level, _dp(v), _dp(out)))
        return out

    def Pdagg_v(self, level, v):
        v = _c(v)
        out = np.empty(self.size(level + 1), dtype=np.complex128)
        check(self.L.ddamg_restrict(self.h, level, _dp(v), _dp(out)))
        return out

    def P_vc(self, level, vc):
        vc = _c(vc)
        out = np.empty(self.size(level), dtype=np.complex128)
        check(self.L.ddamg_prolong(self.h, level, _dp(vc), _dp(out)))
        return out

    def SAP(self, level, v, x0=None, nu=2, tol=1e-10):
        """SAP_C::SAP (src/sap.cpp:81-165); returns (x, iterations)."""
        v = _c(v)
        x = np.zeros(self.size(level), dtype=np.complex128) if x0 is None else np.array(x0, dtype=np.complex128)
        it = ctypes.c_int(0)
        check(self.L.ddamg_sap(self.h, level, _dp(v), _dp(x), nu, tol, ctypes.byref(it)))
        return x, it.value

    def SAP_batched(self, level, v, nrhs, x0=None, nu=2, tol=1e-10):
        """SAP on nrhs vectors stored back to back, in the level's working precision."""
        v = _c(v)
        x = np.zeros(v.size, dtype=np.complex128) if x0 is None else np.array(x0, dtype=np.complex128)
        check(self.L.ddamg_sap_batched(self.h, level, _dp(v), _dp(x), nrhs, nu, tol))
        return x

    # ------------------------------------------------------------ setup
    def setup_random_count(self):
        n = ctypes.c_int64(0)
        check(self.L.ddamg_setup_random_count(self.h, ctypes.byref(n)))
        return n.value

    def setUpPhase(self, seed=None, vectors=None):
        """AlgebraicMG::setUpPhase (src/amg.cpp:4-62) from a seed or an explicit random stream."""
        if vectors is not None:
            v = _c(vectors)
            check(self.L.ddamg_setup_with_vectors(self.h, _dp(v), v.size))
        else:
            check(self.L.ddamg_setup(self.h, 0 if seed is None else int(seed)))

    def test_vectors(self, level):
        out = np.empty(self._ntest[level] * self.size(level), dtype=np.complex128)
        check(self.L.ddamg_get_test_vectors(self.h, level, _dp(out)))
        return out

    def set_test_vectors(self, level, tv):
        tv = _c(tv)
        check(self.L.ddamg_set_test_vectors(self.h, level, _dp(tv)))

    def orthonormalize(self, level):
        check(self.L.ddamg_orthonormalize(self.h, level))

    def makeCoarseLinks(self, level):
        check(self.L.ddamg_build_coarse_links(self.h, level))

    def coarse_links(self, level, which):
        """G1 (which=1), G2 (2), G3 (3) of level >= 1 in the reference layout (include/level.h:349-365)."""
        C = self._ntest[level - 1]
        n = (self.size(level) // (2 * C)) * 4 * C * C * (1 if which == 1 else 2)
        out = np.empty(n, dtype=np.complex128)
        check(self.L.ddamg_get_coarse_links(self.h, level, which, _dp(out)))
        return out

    # ------------------------------------------------------------ solvers
    def coarse_gmres(self, b):
        b = _c(b)
        x = np.empty_like(b)
        it = ctypes.c_int(0)
        check(self.L.ddamg_coarse_solve(self.h, _dp(b), _dp(x), ctypes.byref(it)))
        return x, it.value

    def v_cycle(self, eta):
        eta = _c(eta)
        psi = np.empty_like(eta)
        check(self.L.ddamg_vcycle(self.h, _dp(eta), _dp(psi)))
        return psi

    def k_cycle(self, eta):
        eta = _c(eta)
        psi = np.empty_like(eta)
        check(self.L.ddamg_kcycle(self.h, _dp(eta), _dp(psi)))
        return psi

    def applyMultilevel(self, rhs, x0=None, max_cycles=100, tol=1e-10, allow_not_converged=False):
        """AlgebraicMG::applyMultilevel (src/amg.cpp:177-243): cycles of the handle's kind on the iterate
        until ||rhs - D x|| < tol ||rhs||; returns (x, cycles run, relative residual)."""
        rhs = _c(rhs)
        x = np.zeros_like(rhs) if x0 is None else np.array(x0, dtype=np.complex128)
        n = ctypes.c_int(0)
        rel = ctypes.c_double(0)
        check(self.L.ddamg_apply_multilevel(self.h, _dp(rhs), _dp(x), max_cycles, tol, ctypes.byref(n),
                                            ctypes.byref(rel)),
              allow=(_lib.NOT_CONVERGED,) if allow_not_converged else ())
        return x, n.value, rel.value

    def fgmres_sap(self, b, blocks_x=4, blocks_t=4, m=20, restarts=50, tol=1e-10, allow_not_converged=False):
        """FGMRES_SAP (include/sap.h:236-333): FGMRES(m) on D_W preconditioned by one fine-level SAP
        iteration over blocks_x x blocks_t Schwarz blocks (counts); returns (x, SolveInfo)."""
        b = _c(b)
        x = np.empty_like(b)
        info = SolveInfo()
        check(self.L.ddamg_fgmres_sap(self.h, _dp(b), _dp(x), blocks_x, blocks_t, m, restarts, tol, ctypes.byref(info)),
              allow=(_lib.NOT_CONVERGED,) if allow_not_converged else ())
        return x, info

    def SAP_fine(self, v, blocks_x, blocks_t, x0=None, nu=2, tol=1e-10):
        """SAP_C::SAP of SAP_fine_level over blocks_x x blocks_t blocks (Methods::SAP); returns (x, iterations)."""
        v = _c(v)
        x = np.zeros_like(v) if x0 is None else np.array(x0, dtype=np.complex128)
        it = ctypes.c_int(0)
        check(self.L.ddamg_sap_fine(self.h, _dp(v), _dp(x), blocks_x, blocks_t, nu, tol, ctypes.byref(it)))
        return x, it.value

    def counters(self):
        """Iterations of the last run of each method (-1: not run), as a dict in the metadata file's order."""
        c = (ctypes.c_longlong * 7)()
        check(self.L.ddamg_get_counters(self.h, c))
        return dict(zip(COUNTER_NAMES, list(c)))

    def writeMetadata(self, cycle, tol, path=None):
        """writeMetadata (src/io.cpp:72-145): the run metadata file; path None gives the reference's name."""
        check(self.L.ddamg_write_metadata(self.h, path.encode() if path else None, cycle, tol))

    def set_coarse_barrier_polls(self, polls):
        """Polls after which a grid barrier of the coarsest-level GMRES gives up (DEVICE_TIMEOUT)."""
        check(self.L.ddamg_set_coarse_barrier_polls(self.h, int(polls)))

    def solve(self, b, nrhs=1, allow_not_converged=False):
        """FGMRES_AMG_{v,k}_cycle::fgmres from x0 = 0; returns (x, [SolveInfo])."""
        b = _c(b)
        x = np.empty_like(b)
        info = (SolveInfo * nrhs)()
        check(self.L.ddamg_solve(self.h, _dp(b), _dp(x), nrhs, info),
              allow=(_lib.NOT_CONVERGED,) if allow_not_converged else ())
        return x, list(info)

    def solve_device(self, b_ptr, x_ptr, nrhs=1):
        info = (SolveInfo * nrhs)()
        check(self.L.ddamg_solve_device(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr), nrhs, info))
        return list(info)

    def gmres_plain(self, b, m=50, restarts=200, tol=1e-10):
        b = _c(b)
        x = np.empty_like(b)
        info = SolveInfo()
        check(self.L.ddamg_gmres_plain(self.h, _dp(b), _dp(x), m, restarts, tol, ctypes.byref(info)),
              allow=(_lib.NOT_CONVERGED,))
        return x, info

    def bi_cgstab(self, b, x0=None, max_iter=10000, tol=1e-10):
        """bi_cgstab (src/conjugate_gradient.cpp:87-176) on D_W; returns (x, SolveInfo).  Like the
        reference, info.iterations is k+1 at convergence and max_iter otherwise."""
        b = _c(b)
        x = np.empty_like(b)
        info = SolveInfo()
        x0c = _c(x0) if x0 is not None else None  # kept alive across the call
        check(self.L.ddamg_bicgstab(self.h, _dp(b), _dp(x0c) if x0c is not None else None, _dp(x), max_iter, tol,
                                    ctypes.byref(info)),
              allow=(_lib.NOT_CONVERGED,))
        return x, info

    def conjugate_gradient(self, phi, max_iter=10000, tol=1e-10):
        """conjugate_gradient (src/conjugate_gradient.cpp:4-83): CG on D^dagger D x = phi from x0 = phi;
        returns (x, SolveInfo), info.iterations = k+1 at convergence."""
        phi = _c(phi)
        x = np.empty_like(phi)
        info = SolveInfo()
        check(self.L.ddamg_cg_normal(self.h, _dp(phi), _dp(x), max_iter, tol, ctypes.byref(info)),
              allow=(_lib.NOT_CONVERGED,))
        return x, info

    def CG(self, b, max_iter=10000, tol=1e-10):
        """Methods::CG (src/methods.cpp:42-58): D^dagger b, then conjugate_gradient; x solves D x = b."""
        return self.conjugate_gradient(self.D_dagger_phi(b), max_iter=max_iter, tol=tol)

    def hmc_trajectory(self, theta, beta, md_steps=20, tau=1.0, seed=0, cg_tol=1e-10):
        """One HMC trajectory of the two-flavour Schwinger model from theta ([site][mu], updated in place);
        returns HmcInfo (accepted, dH, plaquette, cg_iterations, seconds).  The handle's gauge field becomes
        the returned one; run setUpPhase again before solving."""
        th = np.ascontiguousarray(theta, dtype=np.float64)
        info = _lib.HmcInfo()
        check(self.L.ddamg_hmc_trajectory(self.h, th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), beta, md_steps,
                                          tau, seed, cg_tol, ctypes.byref(info)))
        if th is not theta:
            theta[...] = th
        return info

    def hmc_force(self, theta, phi, beta, cg_tol=1e-12):
        """dS/dtheta of beta sum_P (1 - cos theta_P) + phi^dagger (D^dagger D)^-1 phi at theta ([site][mu])."""
        th = np.ascontiguousarray(theta, dtype=np.float64)
        phi = _c(phi)
        out = np.empty(2 * self.Nx * self.Nt)
        check(self.L.ddamg_hmc_force(self.h, th.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dp(phi), beta, cg_tol,
                                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def gradient(self, eta, b):
        """dL/dtheta_mu(x) for L = Re(eta^dagger D^-1 b); returns ([site][mu] float64, infos)."""
        eta, b = _c(eta), _c(b)
        out = np.empty(2 * self.Nx * self.Nt)
        info = (SolveInfo * 2)()
        check(self.L.ddamg_gradient(self.h, _dp(eta), _dp(b), _dp(out), info))
        return out, list(info)

    def link_derivative(self, psi, lam):
        psi, lam = _c(psi), _c(lam)
        out = np.empty(2 * self.Nx * self.Nt)
        check(self.L.ddamg_link_derivative(self.h, _dp(psi), _dp(lam), _dp(out)))
        return out

    def stream(self):
        s = ctypes.c_void_p()
        check(self.L.ddamg_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def profile(self, enable):
        check(self.L.ddamg_profile(self.h, int(bool(enable))))

    def profile_query(self, kind, level):
        """(total ms, launches) of kind 0 SAP sweep / 1 coarsest GMRES / 2 level operator /
        3 orthonormalisation / 4 coarse-link construction at a level."""
        ms = ctypes.c_double(0)
        n = ctypes.c_longlong(0)
        check(self.L.ddamg_profile_query(self.h, kind, level, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def autotune_report(self):
        """The tensor-core autotuner's measurements and choices, one line per (level, batch width)."""
        buf = ctypes.create_string_buffer(1 << 14)
        check(self.L.ddamg_autotune_report(self.h, buf, len(buf)))
        return buf.value.decode()

    @staticmethod
    def launch_count():
        c = ctypes.c_longlong(0)
        check(_lib.load().ddamg_launch_count(None, ctypes.byref(c)))
        return c.value
