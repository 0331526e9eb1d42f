"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
baseline.  Only tests/, ``__graft_entry__.smoke()`` and the CPU legs of
``bench.py`` import this module; the product package never does.

The oracle restates the Fortran reference's finite-temperature sweep
(src/dqmc_ft_core, src/dqmc_config_u, src/dqmc_config_h0, lib/s_matrix.f90,
lib/m_spring.f90, src/dqmc_measure/equaltime_measure.f90).  Parity against
reference *output* is unpinned: the reference needs Fortran + MPI + MKL, none
of which exist here, and it ships no golden vectors.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")

SQUARE, HONEYCOMB, CHAIN, CUBIC, R_CUBIC = 1, 2, 3, 4, 5
FAST, DELAY, SUBMATRIX, SUBMATRIX_G, SUBMATRIX_G_EXACT = 0, 1, 2, 3, 4
CHECKERBOARD, FFT, DENSE = 0, 1, 2
HS_EXACT, HS_GENERAL4 = 0, 1
LEFT_FORWARD, LEFT_BACKWARD, RIGHT_FORWARD, RIGHT_BACKWARD, LEFT_FORWARD_HC = range(5)


class OrcParams(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32), ("l1", C.c_int32), ("l2", C.c_int32),
        ("beta", C.c_double), ("dtau", C.c_double), ("rt", C.c_double), ("t2", C.c_double),
        ("t3", C.c_double), ("nu", C.c_double), ("mu", C.c_double), ("rhub", C.c_double),
        ("rv", C.c_double), ("alpha", C.c_double), ("theta", C.c_double),
        ("xmag", C.c_double), ("flux_x", C.c_double), ("flux_y", C.c_double),
        ("dimer", C.c_double), ("rndness", C.c_double),
        ("nflr", C.c_int32), ("lproju", C.c_int32), ("lstabilize", C.c_int32),
        ("nwrap", C.c_int32), ("nsweep", C.c_int32), ("nbin", C.c_int32), ("nublock", C.c_int32),
        ("update", C.c_int32), ("kinetic", C.c_int32), ("hs", C.c_int32),
        ("proj", C.c_int32), ("lprojv", C.c_int32), ("obs_mid_len", C.c_int32),
        ("ltau", C.c_int32), ("dyntau", C.c_double),
        ("l3", C.c_int32), ("rtd", C.c_double),
        ("rhub_plq", C.c_double), ("lprojplqu", C.c_int32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i32, dbl = C.c_void_p, C.c_int32, C.c_double
        L.orc_model_new.restype = vp
        L.orc_model_new.argtypes = [C.POINTER(OrcParams)]
        L.orc_model_free.argtypes = [vp]
        L.orc_chain_new.restype = vp
        L.orc_chain_new.argtypes = [vp, i32, C.c_int]
        L.orc_chain_free.argtypes = [vp]
        L.orc_sfmt_stream.restype = dbl
        L.orc_sfmt_u32.restype = C.c_uint32
        L.orc_test_seed.restype = i32
        L.orc_test_seed.argtypes = [i32]
        L.orc_chain_uniform.restype = dbl
        L.orc_chain_uniform.argtypes = [vp]
        for name in ("orc_sweep_start_0b", "orc_obser_init"):
            getattr(L, name).argtypes = [vp]
        L.orc_sweep_b0.argtypes = [vp, C.c_int, C.c_int]
        L.orc_sweep_0b.argtypes = [vp, C.c_int, C.c_int]
        L.orc_sweep_dyn.argtypes = [vp]
        L.orc_dyn_bins.argtypes = [vp, vp]
        L.orc_dyn_mats.argtypes = [vp, vp, vp, vp]
        L.orc_green_tau.argtypes = [C.c_int] + [vp] * 13
        L.orc_sweep_b0_slices.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.orc_bins_size.argtypes = [vp]
        L.orc_bins_size.restype = C.c_int
        L.orc_update.argtypes = [vp, C.c_int, vp]
        L.orc_measure.argtypes = [vp, C.c_int]
        L.orc_h0_prop.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int]
        L.orc_u_prop.argtypes = [vp, vp, C.c_int, C.c_int, vp, C.c_int]
        L.orc_bmat_left_forward.argtypes = [vp, C.c_int, C.c_int, vp]
        L.orc_bmat_left_forward_hc.argtypes = [vp, C.c_int, C.c_int, vp]
        L.orc_stablize_0b.argtypes = [vp, C.c_int]
        L.orc_stablize_b0.argtypes = [vp, C.c_int]
        L.orc_stack_get.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.orc_stack_set.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.orc_chain_set_phase.argtypes = [vp, dbl, dbl]
        L.orc_green_equaltime.argtypes = [C.c_int] + [vp] * 10
        L.orc_zgeqr2.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp]
        L.orc_zgeqp2.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp, vp]
        L.orc_zung2r.argtypes = [C.c_int, C.c_int, C.c_int, vp, C.c_int, vp]
        L.orc_zgetf2.argtypes = [C.c_int, C.c_int, vp, C.c_int, vp]
        L.orc_zmcpt.argtypes = [C.c_int, C.c_int, vp, vp]
        L.orc_inv_logdet_lu.argtypes = [C.c_int, vp, vp]
        for name in ("orc_proj_sweep_start_0b",):
            getattr(L, name).argtypes = [vp]
        L.orc_proj_sweep_b0.argtypes = [vp, C.c_int, C.c_int]
        L.orc_proj_sweep_0b.argtypes = [vp, C.c_int, C.c_int]
        L.orc_proj_get_trial.argtypes = [vp, vp, vp]
        L.orc_proj_set_trial.argtypes = [vp, vp]
        L.orc_proj_get.argtypes = [vp, vp, vp, vp]
        L.orc_proj_set.argtypes = [vp, vp, vp, vp]
        L.orc_proj_green.argtypes = [vp]
        L.orc_vconf_get.argtypes = [vp, vp]
        L.orc_vconf_set.argtypes = [vp, vp]
        L.orc_proj_update.argtypes = [vp, C.c_int, C.c_int]
        L.orc_proj_update_flavour.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.orc_proj_sweep_b0_slices.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.orc_vconf_prop.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_int, vp, C.c_int]
        L.orc_chain_trace.argtypes = [vp, C.c_int]
        L.orc_chain_trace_count.argtypes = [vp]
        L.orc_chain_trace_count.restype = C.c_int
        L.orc_chain_trace_get.argtypes = [vp, C.c_int, vp, vp]
        L.orc_qr_pqmc_d.argtypes = [C.c_int, C.c_int, vp, vp]
        L.orc_qr_pqmc_d.restype = dbl
        L.orc_eig_he_d.argtypes = [C.c_int, vp, vp, vp]
        for name in ("orc_model_dims", "orc_model_tables", "orc_model_hs", "orc_model_kinetic",
                     "orc_model_h0mat", "orc_chain_set_conf", "orc_chain_get_conf",
                     "orc_chain_set_green", "orc_chain_get_green", "orc_chain_get_diag",
                     "orc_get_bins", "orc_set_lapack"):
            getattr(L, name).restype = None
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    assert a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def use_scipy_lapack(enable: bool = True) -> None:
    """Route the oracle's zgemm/zgeqrf/zgeqp3/zungqr/zgetrf/ztrtri through
    scipy's bundled BLAS/LAPACK (used by the timed CPU baseline)."""
    L = lib()
    if not enable:
        L.orc_set_lapack(None, None, None, None, None, None)
        L.orc_set_zheev.argtypes = [C.c_void_p]
        L.orc_set_zheev(None)
        return
    from scipy.linalg import cython_blas, cython_lapack

    def fp(mod, name):
        cap = mod.__pyx_capi__[name]
        C.pythonapi.PyCapsule_GetName.restype = C.c_char_p
        C.pythonapi.PyCapsule_GetName.argtypes = [C.py_object]
        C.pythonapi.PyCapsule_GetPointer.restype = C.c_void_p
        C.pythonapi.PyCapsule_GetPointer.argtypes = [C.py_object, C.c_char_p]
        return C.c_void_p(C.pythonapi.PyCapsule_GetPointer(cap, C.pythonapi.PyCapsule_GetName(cap)))

    L.orc_set_lapack.argtypes = [C.c_void_p] * 6
    L.orc_set_lapack(fp(cython_blas, "zgemm"), fp(cython_lapack, "zgeqrf"), fp(cython_lapack, "zgeqp3"),
                     fp(cython_lapack, "zungqr"), fp(cython_lapack, "zgetrf"), fp(cython_lapack, "ztrtri"))
    L.orc_set_zheev.argtypes = [C.c_void_p]
    L.orc_set_zheev(fp(cython_lapack, "zheev"))


def make_params(**kw) -> OrcParams:
    """Defaults of src/model_para.f90:166-206 overridden by keyword args."""
    d = dict(lattice=SQUARE, l1=2, l2=2, beta=20.0, dtau=0.05, rt=1.0, t2=0.0, t3=0.0, nu=0.0,
             mu=0.0, rhub=0.0, rv=0.0, alpha=0.2, theta=0.0, xmag=0.0, flux_x=0.0, flux_y=0.0,
             dimer=0.0, rndness=0.0, nflr=2, lproju=0, lstabilize=1, nwrap=10, nsweep=20, nbin=10,
             nublock=0, update=DELAY, kinetic=CHECKERBOARD, hs=HS_GENERAL4, proj=0, lprojv=0,
             obs_mid_len=1, ltau=0, dyntau=0.0, l3=1, rtd=1.0, rhub_plq=0.0, lprojplqu=0)
    d.update(kw)
    return OrcParams(**d)


class Model:
    def __init__(self, **kw):
        self.params = make_params(**kw)
        self.ptr = lib().orc_model_new(C.byref(self.params))
        if not self.ptr:
            raise ValueError("oracle: unsupported parameters")
        dims = np.zeros(10, np.int32)
        lib().orc_model_dims(C.c_void_p(self.ptr), _ptr(dims))
        (self.ndim, self.lq, self.ltrot, self.nst, self.nublock, self.lcomp,
         self.nn_nf, self.nn_lf, self.nsub, self.z_plq) = (int(x) for x in dims)
        self.ne = self.ndim // 2 + int(self.params.nu * self.ndim / 8.0)   # model_para.f90:376
        self.proj = bool(self.params.proj)
        # src/model_para.f90:455-459
        self.ntdm = max(0, int(round(self.params.dyntau / self.params.dtau))) if self.params.ltau else 0

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_model_free(C.c_void_p(self.ptr))
            self.ptr = None

    def tables(self):
        N, lq = self.ndim, self.lq
        nsn = {SQUARE: 4, HONEYCOMB: 6, CHAIN: 2, CUBIC: 12, R_CUBIC: 12}[self.params.lattice]
        nnlist = np.zeros((N, self.nn_nf), np.int32)
        nnlf = np.zeros(self.nn_lf, np.int32)
        lst = np.zeros((N, 2), np.int32)
        imj = np.zeros((lq, lq), np.int32)
        plq = np.zeros((lq, self.z_plq), np.int32)
        sn = np.zeros((N, nsn), np.int32)
        lib().orc_model_tables(C.c_void_p(self.ptr), _ptr(nnlist), _ptr(nnlf), _ptr(lst), _ptr(imj),
                               _ptr(plq), _ptr(sn))
        return dict(nnlist=nnlist, nnlf_list=nnlf, list=lst, imj=imj, plq_cord=plq, snlist=sn)

    def hs(self):
        lc = self.lcomp
        out = dict(bmat=np.zeros(lc, complex), bmat_inv=np.zeros(lc, complex),
                   delta=np.zeros((lc, lc - 1), complex), phase=np.zeros(lc, complex),
                   phase_ratio=np.zeros((lc, lc - 1), complex), gaml=np.zeros(lc), etal=np.zeros(lc))
        alpha = C.c_double()
        lib().orc_model_hs(C.c_void_p(self.ptr), _ptr(out["bmat"]), _ptr(out["bmat_inv"]), _ptr(out["delta"]),
                           _ptr(out["phase"]), _ptr(out["phase_ratio"]), _ptr(out["gaml"]), _ptr(out["etal"]),
                           C.byref(alpha))
        out["alpha"] = alpha.value
        return out

    def kinetic(self):
        nb = self.nn_nf * self.nn_lf
        urt = np.zeros((nb, 2, 2), complex)
        urtm1 = np.zeros((nb, 2, 2), complex)
        e = np.zeros(self.lq, complex)
        ei = np.zeros(self.lq, complex)
        lib().orc_model_kinetic(C.c_void_p(self.ptr), _ptr(urt), _ptr(urtm1), _ptr(e), _ptr(ei))
        return dict(urt=urt, urtm1=urtm1, exph0k=e, exph0kinv=ei)

    def h0mat(self):
        h = np.zeros((self.ndim, self.ndim), complex, order="F")
        lib().orc_model_h0mat(C.c_void_p(self.ptr), _ptr(h))
        return h

    def h0_prop(self, op: int, nf: int, g: np.ndarray) -> None:
        assert g.dtype == complex and g.flags["F_CONTIGUOUS"]
        n2 = g.shape[1] if op in (LEFT_FORWARD, LEFT_BACKWARD, LEFT_FORWARD_HC) else g.shape[0]
        lib().orc_h0_prop(C.c_void_p(self.ptr), op, nf, _ptr(g), n2)

    def u_prop(self, conf: np.ndarray, op: int, nt: int, g: np.ndarray) -> None:
        conf = np.ascontiguousarray(conf, np.int32)
        n2 = g.shape[1] if op in (LEFT_FORWARD, LEFT_BACKWARD, LEFT_FORWARD_HC) else g.shape[0]
        lib().orc_u_prop(C.c_void_p(self.ptr), _ptr(conf), op, nt, _ptr(g), n2)


class Chain:
    def __init__(self, model: Model, seed: int, draw_conf: bool = True):
        self.model = model
        self.ptr = lib().orc_chain_new(C.c_void_p(model.ptr), int(seed), int(draw_conf))

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().orc_chain_free(C.c_void_p(self.ptr))
            self.ptr = None

    @property
    def _p(self):
        return C.c_void_p(self.ptr)

    def conf(self) -> np.ndarray:
        c = np.zeros((self.model.ltrot, self.model.ndim), np.int32)
        lib().orc_chain_get_conf(self._p, _ptr(c))
        return c

    def set_conf(self, conf: np.ndarray) -> None:
        c = np.ascontiguousarray(conf, np.int32)
        lib().orc_chain_set_conf(self._p, _ptr(c))

    def green(self) -> np.ndarray:
        N = self.model.ndim
        g = np.zeros((N, N), complex, order="F")
        lib().orc_chain_get_green(self._p, _ptr(g))
        return g

    def set_green(self, g: np.ndarray) -> None:
        g = np.asfortranarray(g, complex)
        lib().orc_chain_set_green(self._p, _ptr(g))

    def set_phase(self, z: complex) -> None:
        lib().orc_chain_set_phase(self._p, z.real, z.imag)

    def diag(self) -> dict:
        d = np.zeros(15)
        lib().orc_chain_get_diag(self._p, _ptr(d))
        return dict(phase=complex(d[0], d[1]), logweight=complex(d[2], d[3]), max_wrap_error=d[4],
                    max_phasediff=d[5], avglog10error=d[6], logcount=d[7], accepted=d[8], proposed=d[9],
                    accepted_v=d[10], proposed_v=d[11], near_ties=int(d[12]), accepted_plq=d[13],
                    proposed_plq=d[14])

    def conf_plq(self) -> np.ndarray:
        """The plaquette field conf_plqu as [ltrot][lq]."""
        out = np.zeros((self.model.ltrot, self.model.lq), np.int32)
        lib().orc_chain_get_conf_plq(self._p, _ptr(out))
        return out

    def set_conf_plq(self, conf: np.ndarray) -> None:
        a = np.ascontiguousarray(conf, np.int32)
        lib().orc_chain_set_conf_plq(self._p, _ptr(a))

    def trace(self, capacity: int) -> None:
        """Record (fresh G, wrap error) at the next `capacity` wrap checks."""
        lib().orc_chain_trace(self._p, int(capacity))

    def trace_get(self):
        """[(G, wrap error)] recorded since trace()."""
        L = lib()
        n = L.orc_chain_trace_count(self._p)
        N = self.model.ndim
        out = []
        for i in range(n):
            g = np.zeros((N, N), complex, order="F")
            e = C.c_double()
            L.orc_chain_trace_get(self._p, i, _ptr(g), C.byref(e))
            out.append((g, e.value))
        return out

    def max_dyn_error(self) -> float:
        """xmax_dyn of the projective unequal-time pass."""
        f = lib().orc_chain_max_dyn_error
        f.restype = C.c_double
        return float(f(self._p))

    # ---- projective path ----
    def vconf(self) -> np.ndarray:
        m = self.model
        v = np.zeros((m.ltrot, m.nn_nf, m.ndim), np.int32)
        lib().orc_vconf_get(self._p, _ptr(v))
        return v

    def set_vconf(self, v: np.ndarray) -> None:
        v = np.ascontiguousarray(v, np.int32)
        lib().orc_vconf_set(self._p, _ptr(v))

    def trial(self):
        N = self.model.ndim
        p = np.zeros((N, N), complex, order="F")
        w = np.zeros(N)
        lib().orc_proj_get_trial(self._p, _ptr(p), _ptr(w))
        return p, w

    def set_trial(self, p: np.ndarray) -> None:
        p = np.asfortranarray(p, complex)
        lib().orc_proj_set_trial(self._p, _ptr(p))

    def proj_state(self):
        N, ne = self.model.ndim, self.model.ne
        ur = np.zeros((N, ne), complex, order="F")
        ul = np.zeros((ne, N), complex, order="F")
        li = np.zeros((ne, ne), complex, order="F")
        lib().orc_proj_get(self._p, _ptr(ur), _ptr(ul), _ptr(li))
        return ur, ul, li

    def set_proj_state(self, ur=None, ul=None, ulrinv=None) -> None:
        args = []
        keep = []
        for a in (ur, ul, ulrinv):
            if a is None:
                args.append(None)
            else:
                a = np.asfortranarray(a, complex)
                keep.append(a)
                args.append(_ptr(a))
        lib().orc_proj_set(self._p, *args)

    def proj_green(self) -> np.ndarray:
        lib().orc_proj_green(self._p)
        return self.green()

    def proj_update(self, nt: int, nf: int, flavour=None) -> None:
        if flavour is None:
            lib().orc_proj_update(self._p, nt, nf)
        else:
            lib().orc_proj_update_flavour(self._p, nt, nf, int(flavour))

    def proj_sweep_b0_slices(self, nslices: int, lupdate=True, lmeasure=True) -> None:
        lib().orc_proj_sweep_b0_slices(self._p, int(lupdate), int(lmeasure), int(nslices))

    def proj_sweep_start(self) -> None:
        lib().orc_proj_sweep_start_0b(self._p)

    def proj_sweep_b0(self, lupdate=True, lmeasure=True) -> None:
        lib().orc_proj_sweep_b0(self._p, int(lupdate), int(lmeasure))

    def proj_sweep_0b(self, lupdate=True, lmeasure=True) -> None:
        lib().orc_proj_sweep_0b(self._p, int(lupdate), int(lmeasure))

    def uniform(self) -> float:
        return lib().orc_chain_uniform(self._p)

    def sweep_start(self) -> None:
        lib().orc_sweep_start_0b(self._p)

    def sweep_b0(self, lupdate=True, lmeasure=True) -> None:
        lib().orc_sweep_b0(self._p, int(lupdate), int(lmeasure))

    def sweep_b0_slices(self, nslices: int, lupdate=True, lmeasure=True) -> None:
        lib().orc_sweep_b0_slices(self._p, int(lupdate), int(lmeasure), int(nslices))

    def sweep_0b(self, lupdate=True, lmeasure=True) -> None:
        lib().orc_sweep_0b(self._p, int(lupdate), int(lmeasure))

    def obser_init(self) -> None:
        lib().orc_obser_init(self._p)

    # ---- unequal-time measurement (ltau) ----
    def sweep_dyn(self) -> None:
        """push_stage, 0b sweep without updates measuring znn_tau, pop_stage."""
        if lib().orc_sweep_dyn(self._p) != 0:
            raise RuntimeError("sweep_dyn needs ltau = 1")

    def dyn_bins(self) -> np.ndarray:
        """znn_tau_bin as [ntdm+1, 2 (no_j), 2 (no_i), lq] complex."""
        m = self.model
        out = np.zeros(m.lq * 4 * (m.ntdm + 1), complex)
        if lib().orc_dyn_bins(self._p, _ptr(out)) != 0:
            raise RuntimeError("dyn_bins needs ltau = 1")
        return out.reshape(m.ntdm + 1, 2, 2, m.lq)

    def dyn_mats(self):
        """(G(0,0), G(tau,0), G(0,tau)) after the last unequal-time pass."""
        N = self.model.ndim
        g00, gt0, g0t = (np.zeros((N, N), complex, order="F") for _ in range(3))
        lib().orc_dyn_mats(self._p, _ptr(g00), _ptr(gt0), _ptr(g0t))
        return g00, gt0, g0t

    def update(self, nt: int) -> np.ndarray:
        acc = np.zeros(self.model.ndim, np.int32)
        lib().orc_update(self._p, nt, _ptr(acc))
        return acc

    def measure(self, nt: int = 1) -> None:
        lib().orc_measure(self._p, nt)

    def bins(self) -> dict:
        n = lib().orc_bins_size(C.c_void_p(self.model.ptr))
        out = np.zeros(n)
        lib().orc_get_bins(self._p, _ptr(out))
        return unpack_bins(out, self.model.lq)

    def stack(self, n: int):
        N = self.model.ndim
        u = np.zeros((N, N), complex, order="F")
        v = np.zeros((N, N), complex, order="F")
        d = np.zeros(N)
        ld = np.zeros(2)
        lib().orc_stack_get(self._p, n, _ptr(u), _ptr(d), _ptr(v), _ptr(ld))
        return u, d, v, complex(ld[0], ld[1])

    def bmat_left_forward(self, nt1: int, nt2: int, g: np.ndarray) -> None:
        lib().orc_bmat_left_forward(self._p, nt1, nt2, _ptr(g))

    def bmat_left_forward_hc(self, nt1: int, nt2: int, g: np.ndarray) -> None:
        lib().orc_bmat_left_forward_hc(self._p, nt1, nt2, _ptr(g))


def vconf_prop(model: Model, vconf: np.ndarray, op: int, nt: int, nf: int, nflag: int, g: np.ndarray) -> None:
    vconf = np.ascontiguousarray(vconf, np.int32)
    assert g.dtype == complex and g.flags["F_CONTIGUOUS"]
    n2 = g.shape[1] if op in (LEFT_FORWARD, LEFT_BACKWARD, LEFT_FORWARD_HC) else g.shape[0]
    lib().orc_vconf_prop(C.c_void_p(model.ptr), _ptr(vconf), op, nt, nf, nflag, _ptr(g), n2)


def qr_pqmc(a: np.ndarray):
    """s_zgeQR_pqmc: (Q, log|det R|) with det R > 0."""
    a = np.asfortranarray(a, complex)
    q = np.zeros_like(a, order="F")
    lw = lib().orc_qr_pqmc_d(a.shape[0], a.shape[1], _ptr(a), _ptr(q))
    return q, lw


def eig_he(h: np.ndarray):
    h = np.asfortranarray(h, complex)
    n = h.shape[0]
    w = np.zeros(n)
    v = np.zeros((n, n), complex, order="F")
    lib().orc_eig_he_d(n, _ptr(h), _ptr(w), _ptr(v))
    return w, v


def unpack_bins(flat: np.ndarray, lq: int) -> dict:
    z = flat[:-1].view(complex)
    k = 0
    out = {}
    out["energy"] = z[k:k + 10].copy(); k += 10
    for name in ("cpcm", "spsm", "nn", "pair_onsite"):
        out[name] = z[k:k + 4 * lq].reshape(2, 2, lq).copy(); k += 4 * lq   # [no_j][no_i][imj]
    for name in ("jj", "bb", "pair_nn", "pair_sn"):
        out[name] = z[k:k + lq].copy(); k += lq
    out["zn"] = z[k:k + 2].copy(); k += 2
    out["zj"] = z[k]; out["zb"] = z[k + 1]
    out["nobs"] = int(round(flat[-1]))
    return out
