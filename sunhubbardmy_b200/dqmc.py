"""ctypes host mirror of the reference's sweep driver over libdqmc_gpu.so.

Names follow the reference: ``dqmc.in`` namelists (src/model_para.f90),
``sweep_start`` (dqmc_ft_sweep_start_0b, or dqmc_proj_sweep_start_0b when
``proj=1``), ``sweep_b0`` / ``sweep_0b`` (dqmc_ft_sweep_b0/0b or
dqmc_proj_sweep_b0/0b), ``obser_init``, ``update`` / ``proj_update``,
``h0_prop`` / ``u_prop`` (the h0conf / uconf type-bound procedures).
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

SQUARE, HONEYCOMB, CHAIN, CUBIC, R_CUBIC = 1, 2, 3, 4, 5
FAST, DELAY, SUBMATRIX = 0, 1, 2
CHECKERBOARD, FFT, DENSE = 0, 1, 2
EXACT, GENERAL4 = 0, 1

_HERE = os.path.dirname(os.path.abspath(__file__))


def lib_path() -> str:
    return os.path.join(_HERE, "_lib", "libdqmc_gpu.so")


# return codes of include/dqmc_gpu.h
EINVAL, ECUDA, ENOMEM, ESTATE, ENUMERIC, EWRAP = -1, -2, -3, -4, -5, -6
FAIL_SINGULAR, FAIL_NONFINITE, FAIL_WRAP = 1, 2, 4


class DqmcError(RuntimeError):
    """A failed library call; ``code`` is its DQMC_E* return value."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


class DqmcParams(C.Structure):
    """Mirror of ``dqmc_params`` in include/dqmc_gpu.h."""
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
        ("ndim", C.c_int32), ("lq", C.c_int32), ("ltrot", C.c_int32), ("nst", C.c_int32),
        ("ne", C.c_int32), ("lcomp", C.c_int32),
        ("ltau", C.c_int32), ("ntdm", C.c_int32), ("dyntau", C.c_double),
        ("l3", C.c_int32), ("rtd", C.c_double),
        ("rhub_plq", C.c_double), ("lprojplqu", C.c_int32),
    ]

    @classmethod
    def make(cls, **kw) -> "DqmcParams":
        """Defaults of src/model_para.f90:166-206, overridden by keywords."""
        d = dict(lattice=SQUARE, l1=2, l2=2, beta=20.0, dtau=0.05, rt=1.0, t2=0.0, t3=0.0, nu=0.0,
                 mu=0.0, rhub=0.0, rv=0.0, alpha=0.2, theta=0.0, xmag=0.0, flux_x=0.0, flux_y=0.0,
                 dimer=0.0, rndness=0.0, nflr=2, lproju=0, lstabilize=1, nwrap=10, nsweep=20,
                 nbin=10, nublock=0, update=DELAY, kinetic=CHECKERBOARD, hs=GENERAL4, proj=0,
                 lprojv=0, obs_mid_len=1, ltau=0, dyntau=0.0, l3=1, rtd=1.0, rhub_plq=0.0, lprojplqu=0)
        d.update(kw)
        p = cls(**d)
        rc = load_library().dqmc_params_derive(C.byref(p))
        if rc != 0:
            raise DqmcError(f"dqmc_params_derive: {_last_error()}")
        return p

    def tables(self) -> dict:
        """Lattice / kinetic tables built by the library (1-based, host only)."""
        N, lq = self.ndim, self.lq
        hc = self.lattice == HONEYCOMB
        nnf, z, nsn = {HONEYCOMB: (3, 6, 6), CHAIN: (2, 1, 2), CUBIC: (6, 8, 12),
                       R_CUBIC: (4, 8, 12)}.get(self.lattice, (4, 4, 4))
        nlf = {HONEYCOMB: lq, R_CUBIC: 3 * lq}.get(self.lattice, lq // 2)
        t = dict(nnlist=np.zeros((N, nnf), np.int32), nnlf_list=np.zeros(nlf, np.int32),
                 list=np.zeros((N, 2), np.int32), imj=np.zeros((lq, lq), np.int32),
                 plq_cord=np.zeros((lq, z), np.int32), snlist=np.zeros((N, nsn), np.int32),
                 urt=np.zeros((nnf * nlf, 2, 2), complex), exph0k=np.zeros(lq, complex))
        rc = load_library().dqmc_model_tables(C.byref(self), *[_ptr(t[k]) for k in
                                              ("nnlist", "nnlf_list", "list", "imj", "plq_cord", "snlist", "urt", "exph0k")])
        if rc != 0:
            raise DqmcError(f"dqmc_model_tables: {_last_error()}")
        return t

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class DqmcDiag(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "phase_re", "phase_im", "logweight_re", "logweight_im", "max_wrap_error", "max_phasediff",
        "avglog10error_sum", "logcount", "avgexpphasediff_sum", "accepted", "proposed", "nobs",
        "accepted_v", "proposed_v", "blk_proposed", "blk_stage1", "blk_accepted", "blk_sum_logratio",
        "blk_err_learned", "blk_err_zero", "max_dyn_error", "dyn_log10_sum", "dyn_count", "info",
        "restabilized", "near_ties", "accepted_plq", "proposed_plq")]


_lib = None

# Every entry point declared in include/dqmc_gpu.h with (restype, argtypes).
_vp, _i, _d = C.c_void_p, C.c_int, C.c_double
SIGNATURES = {
    "dqmc_params_derive": (_i, [_vp]),
    "dqmc_model_tables": (_i, [_vp] * 9),
    "dqmc_gpu_create": (_i, [_vp, _i, _i, _vp, _i, C.POINTER(_vp)]),
    "dqmc_gpu_destroy": (_i, [_vp]),
    "dqmc_gpu_last_error": (C.c_char_p, []),
    "dqmc_gpu_set_conf": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_conf": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_set_conf_all": (_i, [_vp, _vp]),
    "dqmc_gpu_get_conf_all": (_i, [_vp, _vp]),
    "dqmc_gpu_get_green": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_set_green": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_stack": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp]),
    "dqmc_gpu_set_stack": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp]),
    "dqmc_gpu_set_checks": (_i, [_vp, _d, _i]),
    "dqmc_gpu_trace_wraps": (_i, [_vp, _i, _i]),
    "dqmc_gpu_trace_count": (_i, [_vp, _i]),
    "dqmc_gpu_trace_get": (_i, [_vp, _i, _i, _vp, _vp]),
    "dqmc_gpu_sweep_start": (_i, [_vp]),
    "dqmc_gpu_sweep_b0": (_i, [_vp, _i, _i]),
    "dqmc_gpu_sweep_0b": (_i, [_vp, _i, _i]),
    "dqmc_gpu_sweeps": (_i, [_vp, _i, _i]),
    "dqmc_gpu_obser_init": (_i, [_vp]),
    "dqmc_gpu_nbins": (_i, [_vp, _i]),
    "dqmc_gpu_get_bins": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_diag": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_energy_all": (_i, [_vp, _vp]),
    "dqmc_gpu_reset_diag": (_i, [_vp]),
    "dqmc_gpu_h0_prop": (_i, [_vp, _i, _i]),
    "dqmc_gpu_u_prop": (_i, [_vp, _i, _i]),
    "dqmc_gpu_update": (_i, [_vp, _i]),
    "dqmc_gpu_measure": (_i, [_vp]),
    "dqmc_gpu_set_phase": (_i, [_vp, _i, _d, _d]),
    "dqmc_gpu_draw_u32": (_i, [_vp, _i, _i, _vp]),
    "dqmc_gpu_get_rng": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_set_rng": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_set_work": (_i, [_vp, _i, _i, _vp]),
    "dqmc_gpu_get_work": (_i, [_vp, _i, _i, _vp]),
    "dqmc_gpu_test_zgemm": (_i, [_vp, _i, _i, _i, _i, _i, _i, _i, _i, _d]),
    "dqmc_gpu_test_qr": (_i, [_vp, _i, _i, _vp]),
    "dqmc_gpu_last_sweeps_ms": (_d, [_vp]),
    "dqmc_gpu_time_op": (_i, [_vp, _i, _i, _vp]),
    "dqmc_gpu_sweep_kernels": (_i, [_vp]),
    "dqmc_gpu_sweep_profile": (_i, [_vp, _i, _i, _vp, _vp]),
    "dqmc_gpu_sweep_dyn": (_i, [_vp]),
    "dqmc_gpu_sweeps_multi": (_i, [_vp, _i, _i, _i, _vp]),
    "dqmc_gpu_sweep_start_multi": (_i, [_vp, _i]),
    "dqmc_gpu_get_dyn_bins": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_dyn_mats": (_i, [_vp, _i, _vp, _vp, _vp]),
    "dqmc_gpu_qr_logdet_noalloc": (_i, [_i, _vp, _vp, _vp, _vp]),
    "dqmc_gpu_noalloc_error": (C.c_char_p, []),
    "dqmc_gpu_set_vconf": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_vconf": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_set_conf_plq": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_conf_plq": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_trial": (_i, [_vp, _i, _vp, _vp]),
    "dqmc_gpu_set_trial": (_i, [_vp, _i, _vp]),
    "dqmc_gpu_get_proj": (_i, [_vp, _i, _vp, _vp, _vp]),
    "dqmc_gpu_set_proj": (_i, [_vp, _i, _vp, _vp, _vp]),
    "dqmc_gpu_proj_update": (_i, [_vp, _i, _i]),
    "dqmc_gpu_proj_green": (_i, [_vp]),
    "dqmc_trial_state": (_i, [_vp, C.c_int32, _i, _vp, _vp]),
    "dqmc_nn_create": (_i, [_i, _i, _i, C.c_uint64, C.POINTER(_vp)]),
    "dqmc_nn_destroy": (_i, [_vp]),
    "dqmc_nn_nparams": (_i, []),
    "dqmc_nn_set_params": (_i, [_vp, _vp]),
    "dqmc_nn_get_params": (_i, [_vp, _vp]),
    "dqmc_nn_forward": (_i, [_vp, _vp, _i, _vp]),
    "dqmc_nn_gradient": (_i, [_vp, _vp, _i, _vp, _vp, _vp]),
    "dqmc_nn_train_step": (_i, [_vp, _vp, _vp, _i, _d, _vp]),
    "dqmc_nn_train_recorded": (_i, [_vp, _vp, _vp, _vp, _i, _d, _vp]),
    "dqmc_nn_train_recorded_pairs": (_i, [_vp, _vp, _vp, _vp, _vp, _i, _d, _vp]),
    "dqmc_gpu_record": (_i, [_vp, _i]),
    "dqmc_gpu_record_count": (_i, [_vp]),
    "dqmc_gpu_record_get": (_i, [_vp, _i, _vp, _vp]),
    "dqmc_gpu_record_values": (_i, [_vp, _vp]),
    "dqmc_gpu_sweep_learned": (_i, [_vp, _vp, _i, _i, _i, C.c_uint64]),
}


def load_library() -> C.CDLL:
    """Load the CUDA library; raises if it has not been built (no fallback)."""
    global _lib
    if _lib is None:
        path = lib_path()
        if not os.path.exists(path):
            raise DqmcError(f"{path} is missing: build it with __graft_entry__.build() "
                            "(make -C sunhubbardmy_b200/csrc); there is no CPU fallback")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _last_error() -> str:
    s = load_library().dqmc_gpu_last_error()
    return s.decode() if s else ""


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise DqmcError(f"{what} failed ({rc}): {_last_error()}", rc)


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


def test_seed(irank: int) -> int:
    """abs((irank*1981+2008)*951049) in 32-bit integers (src/dqmc_util.f90:72)."""
    v = ((irank * 1981 + 2008) * 951049) & 0xFFFFFFFF
    if v >= 1 << 31:
        v -= 1 << 32
    return abs(v)


def qr_logdet_noalloc(n: int, a_dev: int, q_dev: int, logdetq_dev: int, stream: int = 0) -> None:
    """Allocation-free QR of a caller-owned device matrix (see
    dqmc_gpu_qr_logdet_noalloc in include/dqmc_gpu.h): for callers that cannot
    allocate device memory; all arguments are raw device addresses."""
    L = load_library()
    rc = L.dqmc_gpu_qr_logdet_noalloc(int(n), C.c_void_p(a_dev), C.c_void_p(q_dev),
                                      C.c_void_p(logdetq_dev), C.c_void_p(stream))
    if rc != 0:
        raise DqmcError(f"qr_logdet_noalloc failed ({rc}): {L.dqmc_gpu_noalloc_error().decode()}")


def sweeps_concurrent(handles, n: int, lmeasure: bool = True) -> float:
    """n whole sweeps of several Dqmc handles at once, each on its own stream
    (dqmc_gpu_sweeps_multi); returns the device ms per sweep of all of them."""
    arr = (C.c_void_p * len(handles))(*[g.h for g in handles])
    ms = C.c_double()
    _check(load_library().dqmc_gpu_sweeps_multi(arr, len(handles), n, int(lmeasure), C.byref(ms)), "sweeps_multi")
    return ms.value


def sweep_start_concurrent(handles) -> None:
    """dqmc_ft_sweep_start_0b of several Dqmc handles at once, each on its own
    stream (dqmc_gpu_sweep_start_multi)."""
    arr = (C.c_void_p * len(handles))(*[g.h for g in handles])
    _check(load_library().dqmc_gpu_sweep_start_multi(arr, len(handles)), "sweep_start_multi")


def trial_state(params: DqmcParams, seed: int, draw_conf: bool = True):
    """Host-only: the trial state (eigenvectors, eigenvalues) dqmc_gpu_create
    computes for a walker with this seed (no GPU needed)."""
    N = params.ndim
    p = np.zeros((N, N), complex, order="F")
    w = np.zeros(N)
    _check(load_library().dqmc_trial_state(C.byref(params), int(seed), int(draw_conf), _ptr(p), _ptr(w)),
           "dqmc_trial_state")
    return p, w


# ----------------------------------------------------------------------------
# dqmc.in namelist reader (src/model_para.f90:155-218)
# ----------------------------------------------------------------------------
_NL_RE = re.compile(r"&(\w+)(.*?)/", re.S)


def _parse_value(v: str):
    v = v.strip().rstrip(",").strip()
    lv = v.lower()
    if lv in (".true.", "t", ".t.", "true"):
        return True
    if lv in (".false.", "f", ".f.", "false"):
        return False
    lv = lv.replace("d", "e")
    try:
        if re.fullmatch(r"[+-]?\d+", lv):
            return int(lv)
        return float(lv)
    except ValueError:
        return v.strip("'\"")


def read_dqmc_in(path_or_text: str) -> dict:
    """Parse the &model_para and &ctrl_para namelists of a dqmc.in file."""
    text = path_or_text
    if os.path.exists(path_or_text):
        with open(path_or_text) as f:
            text = f.read()
    text = re.sub(r"!.*", "", text)
    out = {}
    for grp, body in _NL_RE.findall(text):
        for key, val in re.findall(r"(\w+)\s*=\s*([^=]+?)(?=,?\s*\w+\s*=|$)", body.strip(), re.S):
            out[key.lower()] = _parse_value(val)
    if "la" in out:
        out["l1"] = out.pop("la")
    if "lb" in out:
        out["l2"] = out.pop("lb")
    if "lc" in out:            # the cubic lattice's third length (-DCUBIC namelist)
        out["l3"] = out.pop("lc")
    for k in ("lprojv", "lproju", "lprojplqu", "lstabilize", "ltau"):
        if k in out:
            out[k] = int(bool(out[k]))
    keep = {f for f, _ in DqmcParams._fields_}
    return {k: v for k, v in out.items() if k in keep}


# ----------------------------------------------------------------------------
# driver
# ----------------------------------------------------------------------------
class Dqmc:
    """n_chains independent DQMC chains advanced together on the GPU."""

    def __init__(self, params, n_chains: int = 1, seeds=None, draw_conf: bool = True):
        if isinstance(params, DqmcParams):
            params = [params]
        self.params = list(params)
        arr = (DqmcParams * len(self.params))(*self.params)
        if seeds is None:
            seeds = [test_seed(c) for c in range(n_chains)]
        self.seeds = np.ascontiguousarray(seeds, np.int32)
        assert len(self.seeds) == n_chains
        self.n_chains = n_chains
        h = C.c_void_p()
        L = load_library()
        _check(L.dqmc_gpu_create(C.cast(arr, C.c_void_p), len(self.params), n_chains, _ptr(self.seeds),
                                 int(draw_conf), C.byref(h)), "dqmc_gpu_create")
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            load_library().dqmc_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def chain_params(self, c: int) -> DqmcParams:
        return self.params[c % len(self.params)]

    def ndim(self, c: int = 0) -> int:
        return self.chain_params(c).ndim

    @property
    def ltrot(self) -> int:
        return self.params[0].ltrot

    # state
    def conf(self, c: int = 0) -> np.ndarray:
        out = np.zeros((self.ltrot, self.ndim(c)), np.int32)
        _check(load_library().dqmc_gpu_get_conf(self.h, c, _ptr(out)), "get_conf")
        return out

    def set_conf(self, conf: np.ndarray, c: int = 0) -> None:
        a = np.ascontiguousarray(conf, np.int32)
        _check(load_library().dqmc_gpu_set_conf(self.h, c, _ptr(a)), "set_conf")

    def conf_all(self, out: np.ndarray | None = None) -> np.ndarray:
        n = sum(self.ltrot * self.ndim(c) for c in range(self.n_chains))
        if out is None:
            out = np.zeros(n, np.int32)
        _check(load_library().dqmc_gpu_get_conf_all(self.h, _ptr(out)), "get_conf_all")
        return out

    def set_conf_all(self, conf: np.ndarray) -> None:
        _check(load_library().dqmc_gpu_set_conf_all(self.h, _ptr(conf)), "set_conf_all")

    def green(self, c: int = 0) -> np.ndarray:
        N = self.ndim(c)
        g = np.zeros((N, N), complex, order="F")
        _check(load_library().dqmc_gpu_get_green(self.h, c, _ptr(g)), "get_green")
        return g

    def set_green(self, g: np.ndarray, c: int = 0) -> None:
        a = np.asfortranarray(g, complex)
        _check(load_library().dqmc_gpu_set_green(self.h, c, _ptr(a)), "set_green")

    def stack(self, n: int, c: int = 0):
        """(Ust(n), Dst(n), Vst(n), logdetQst(n)) of one chain's UDV stack."""
        N = self.ndim(c)
        u = np.zeros((N, N), complex, order="F")
        v = np.zeros((N, N), complex, order="F")
        d = np.zeros(N)
        ld = np.zeros(1, complex)
        _check(load_library().dqmc_gpu_get_stack(self.h, c, int(n), _ptr(u), _ptr(d), _ptr(v), _ptr(ld)),
               "get_stack")
        return u, d, v, complex(ld[0])

    def set_stack(self, n: int, u=None, d=None, v=None, logdetq=None, c: int = 0) -> None:
        """Overwrite parts of stack entry n (None keeps a part)."""
        keep = []

        def arg(x, dtype, fortran=False):
            if x is None:
                return None
            a = np.asfortranarray(x, dtype) if fortran else np.ascontiguousarray(x, dtype)
            keep.append(a)
            return _ptr(a)
        ld = None if logdetq is None else np.array([logdetq], complex)
        _check(load_library().dqmc_gpu_set_stack(self.h, c, int(n), arg(u, complex, True), arg(d, float),
                                                 arg(v, complex, True), arg(ld, complex)), "set_stack")

    def rng_state(self, c: int = 0) -> np.ndarray:
        """SFMT state of chain c: 625 int32 words, pt32(0:623) then idx."""
        out = np.zeros(625, np.int32)
        _check(load_library().dqmc_gpu_get_rng(self.h, c, _ptr(out)), "get_rng")
        return out

    def set_rng_state(self, state: np.ndarray, c: int = 0) -> None:
        a = np.ascontiguousarray(state, np.int32)
        assert a.size == 625
        _check(load_library().dqmc_gpu_set_rng(self.h, c, _ptr(a)), "set_rng")

    def trace_wraps(self, capacity: int, c: int = 0) -> None:
        """Record (fresh G, wrap error) at the next `capacity` wrap checks of chain c."""
        _check(load_library().dqmc_gpu_trace_wraps(self.h, c, int(capacity)), "trace_wraps")

    def trace_get(self, c: int = 0):
        """[(G, wrap error)] recorded since trace_wraps."""
        L = load_library()
        n = L.dqmc_gpu_trace_count(self.h, c)
        _check(min(n, 0), "trace_count")
        N = self.ndim(c)
        out = []
        for i in range(n):
            g = np.zeros((N, N), complex, order="F")
            e = C.c_double()
            _check(L.dqmc_gpu_trace_get(self.h, c, i, _ptr(g), C.byref(e)), "trace_get")
            out.append((g, e.value))
        return out

    def set_checks(self, wrap_tol: float = 0.0, restabilize: bool = False) -> None:
        """Numerical checks of the sweep calls (dqmc_gpu_set_checks): a wrap
        error above wrap_tol (> 0) raises DqmcError with code EWRAP; with
        restabilize the stack and G are rebuilt from the HS field instead."""
        _check(load_library().dqmc_gpu_set_checks(self.h, float(wrap_tol), int(restabilize)), "set_checks")

    def set_phase(self, z: complex, c: int = 0) -> None:
        _check(load_library().dqmc_gpu_set_phase(self.h, c, z.real, z.imag), "set_phase")

    def diag(self, c: int = 0) -> dict:
        d = DqmcDiag()
        _check(load_library().dqmc_gpu_get_diag(self.h, c, C.byref(d)), "get_diag")
        return dict(phase=complex(d.phase_re, d.phase_im), logweight=complex(d.logweight_re, d.logweight_im),
                    max_wrap_error=d.max_wrap_error, max_phasediff=d.max_phasediff,
                    avglog10error=d.avglog10error_sum, logcount=d.logcount,
                    avgexpphasediff=d.avgexpphasediff_sum, accepted=d.accepted, proposed=d.proposed,
                    nobs=d.nobs, accepted_v=d.accepted_v, proposed_v=d.proposed_v,
                    blk_proposed=d.blk_proposed, blk_stage1=d.blk_stage1, blk_accepted=d.blk_accepted,
                    blk_sum_logratio=d.blk_sum_logratio, blk_err_learned=d.blk_err_learned,
                    blk_err_zero=d.blk_err_zero, max_dyn_error=d.max_dyn_error,
                    dyn_log10_sum=d.dyn_log10_sum, dyn_count=d.dyn_count, info=int(d.info),
                    restabilized=int(d.restabilized), near_ties=int(d.near_ties),
                    accepted_plq=d.accepted_plq, proposed_plq=d.proposed_plq)

    def energy_all(self) -> np.ndarray:
        """energy_bin(1:10) of every chain, shape (n_chains, 10) complex."""
        out = np.zeros((self.n_chains, 10), complex)
        _check(load_library().dqmc_gpu_get_energy_all(self.h, _ptr(out)), "get_energy_all")
        return out

    def reset_diag(self) -> None:
        _check(load_library().dqmc_gpu_reset_diag(self.h), "reset_diag")

    # sweep
    def sweep_start(self) -> None:
        _check(load_library().dqmc_gpu_sweep_start(self.h), "sweep_start")

    def sweep_b0(self, lupdate: bool = True, lmeasure: bool = True) -> None:
        _check(load_library().dqmc_gpu_sweep_b0(self.h, int(lupdate), int(lmeasure)), "sweep_b0")

    def sweep_0b(self, lupdate: bool = True, lmeasure: bool = True) -> None:
        _check(load_library().dqmc_gpu_sweep_0b(self.h, int(lupdate), int(lmeasure)), "sweep_0b")

    def sweeps(self, n: int, lmeasure: bool = True) -> float:
        """n x (b0 + 0b) through a captured CUDA graph; returns device ms per sweep."""
        L = load_library()
        _check(L.dqmc_gpu_sweeps(self.h, int(n), int(lmeasure)), "sweeps")
        return L.dqmc_gpu_last_sweeps_ms(self.h)

    def obser_init(self) -> None:
        _check(load_library().dqmc_gpu_obser_init(self.h), "obser_init")

    def bins_raw(self, c: int = 0) -> np.ndarray:
        L = load_library()
        n = L.dqmc_gpu_nbins(self.h, c)
        out = np.zeros(n, complex)
        _check(L.dqmc_gpu_get_bins(self.h, c, _ptr(out)), "get_bins")
        return out

    def bins(self, c: int = 0) -> dict:
        from .io import unpack_bins
        d = self.diag(c)
        return unpack_bins(self.bins_raw(c), self.chain_params(c).lq, int(round(d["nobs"])))

    # operator-level procedures
    def h0_prop(self, op: int, nf: int = 1) -> None:
        _check(load_library().dqmc_gpu_h0_prop(self.h, op, nf), "h0_prop")

    def u_prop(self, op: int, nt: int) -> None:
        _check(load_library().dqmc_gpu_u_prop(self.h, op, nt), "u_prop")

    def update(self, nt: int) -> None:
        _check(load_library().dqmc_gpu_update(self.h, nt), "update")

    def measure(self) -> None:
        _check(load_library().dqmc_gpu_measure(self.h), "measure")

    def draw_u32(self, count: int, c: int = 0) -> np.ndarray:
        out = np.zeros(count, np.uint32)
        _check(load_library().dqmc_gpu_draw_u32(self.h, c, count, _ptr(out)), "draw_u32")
        return out

    def sweep_kernels(self) -> int:
        """Kernel launches in one captured sweep (b0 + 0b)."""
        return load_library().dqmc_gpu_sweep_kernels(self.h)

    def time_op(self, op: int, reps: int = 3) -> float:
        """Device ms of one launch of sweep kernel `op` over all chains."""
        ms = C.c_double()
        _check(load_library().dqmc_gpu_time_op(self.h, op, reps, C.byref(ms)), "time_op")
        return ms.value

    # unequal-time measurement (params.ltau = 1)
    def sweep_dyn(self) -> None:
        """push_stage, 0b sweep without updates measuring znn_tau, pop_stage
        (the ltau pass of dqmc_sweep)."""
        _check(load_library().dqmc_gpu_sweep_dyn(self.h), "sweep_dyn")

    def dyn_bins(self, c: int = 0) -> np.ndarray:
        """znn_tau_bin of chain c as [ntdm+1, 2 (no_j), 2 (no_i), lq] complex."""
        p = self.chain_params(c)
        out = np.zeros(p.lq * 4 * (p.ntdm + 1), complex)
        _check(load_library().dqmc_gpu_get_dyn_bins(self.h, c, _ptr(out)), "get_dyn_bins")
        return out.reshape(p.ntdm + 1, 2, 2, p.lq)

    def dyn_mats(self, c: int = 0):
        """(G(0,0), G(beta,0), G(0,beta)) after the last unequal-time pass."""
        N = self.ndim(c)
        mats = [np.zeros((N, N), complex, order="F") for _ in range(3)]
        _check(load_library().dqmc_gpu_get_dyn_mats(self.h, c, *[_ptr(x) for x in mats]), "get_dyn_mats")
        return tuple(mats)

    PROFILE_KINDS = ("update", "stab", "green", "prop_left", "measure", "prop_right", "bprod", "other")

    def sweep_profile(self, n: int = 1, lmeasure: bool = True) -> dict:
        """Device time per kind over n sweeps run launch by launch (events
        after every launch group): {kind: (total ms, launch groups)}."""
        ms = (C.c_double * 8)()
        gr = (C.c_int * 8)()
        _check(load_library().dqmc_gpu_sweep_profile(self.h, n, int(lmeasure), ms, gr), "sweep_profile")
        return {k: (ms[i], gr[i]) for i, k in enumerate(self.PROFILE_KINDS)}

    # diagnostics on the tensor-core kernels
    def set_work(self, which: int, m: np.ndarray, c: int = 0) -> None:
        a = np.asfortranarray(m, complex)
        _check(load_library().dqmc_gpu_set_work(self.h, c, which, _ptr(a)), "set_work")

    def work(self, which: int, c: int = 0) -> np.ndarray:
        N = self.ndim(c)
        g = np.zeros((N, N), complex, order="F")
        _check(load_library().dqmc_gpu_get_work(self.h, c, which, _ptr(g)), "get_work")
        return g

    def test_zgemm(self, m, n, k, opa, opb, a, b, c, beta=0.0) -> None:
        _check(load_library().dqmc_gpu_test_zgemm(self.h, m, n, k, opa, opb, a, b, c, float(beta)), "test_zgemm")

    # training pairs and learned sweeps (finite temperature, square lattice)
    def record(self, capacity: int) -> None:
        """Record (field, nflr Re log W) of every chain at every stabilisation
        into a ring of `capacity` pairs (0 stops recording)."""
        _check(load_library().dqmc_gpu_record(self.h, int(capacity)), "record")

    def record_count(self) -> int:
        return load_library().dqmc_gpu_record_count(self.h)

    def record_get(self, i: int):
        p = self.chain_params(0)
        f = np.zeros((p.ltrot, p.l1, p.l2), np.int8)
        v = C.c_double()
        _check(load_library().dqmc_gpu_record_get(self.h, int(i), _ptr(f), C.byref(v)), "record_get")
        return f, v.value

    def record_values(self, capacity: int) -> np.ndarray:
        out = np.zeros(capacity)
        _check(load_library().dqmc_gpu_record_values(self.h, _ptr(out)), "record_values")
        return out

    def sweeps_learned(self, nn, n: int, lmeasure: bool = True, seed: int = 0, lupdate: bool = True) -> float:
        """n sweeps with global block proposals from the effective action nn;
        returns device ms per sweep."""
        L = load_library()
        _check(L.dqmc_gpu_sweep_learned(self.h, nn.h, int(n), int(lupdate), int(lmeasure), C.c_uint64(seed)),
               "sweep_learned")
        return L.dqmc_gpu_last_sweeps_ms(self.h)

    # projective path (params.proj = 1)
    def vconf(self, c: int = 0) -> np.ndarray:
        """t-V bond field vconf%conf as [ltrot][nn_nf][ndim] (bond index fastest)."""
        nnf = {HONEYCOMB: 3, CHAIN: 2, CUBIC: 6, R_CUBIC: 4}.get(self.chain_params(c).lattice, 4)
        out = np.zeros((self.ltrot, nnf, self.ndim(c)), np.int32)
        _check(load_library().dqmc_gpu_get_vconf(self.h, c, _ptr(out)), "get_vconf")
        return out

    def set_vconf(self, v: np.ndarray, c: int = 0) -> None:
        a = np.ascontiguousarray(v, np.int32)
        _check(load_library().dqmc_gpu_set_vconf(self.h, c, _ptr(a)), "set_vconf")

    def conf_plq(self, c: int = 0) -> np.ndarray:
        """Plaquette field hconf%conf_plqu as [ltrot][lq] (plaquette fastest)."""
        out = np.zeros((self.ltrot, self.chain_params(c).lq), np.int32)
        _check(load_library().dqmc_gpu_get_conf_plq(self.h, c, _ptr(out)), "get_conf_plq")
        return out

    def set_conf_plq(self, v: np.ndarray, c: int = 0) -> None:
        a = np.ascontiguousarray(v, np.int32)
        _check(load_library().dqmc_gpu_set_conf_plq(self.h, c, _ptr(a)), "set_conf_plq")

    def trial(self, c: int = 0):
        """(proj, w): trial eigenvectors (ndim x ndim) and eigenvalues of walker c."""
        N = self.ndim(c)
        p = np.zeros((N, N), complex, order="F")
        w = np.zeros(N)
        _check(load_library().dqmc_gpu_get_trial(self.h, c, _ptr(p), _ptr(w)), "get_trial")
        return p, w

    def set_trial(self, proj: np.ndarray, c: int = 0) -> None:
        a = np.asfortranarray(proj, complex)
        _check(load_library().dqmc_gpu_set_trial(self.h, c, _ptr(a)), "set_trial")

    def proj_state(self, c: int = 0):
        """(UR, UL, ULRINV) of walker c in the reference's layouts."""
        N, ne = self.ndim(c), self.chain_params(c).ne
        ur = np.zeros((N, ne), complex, order="F")
        ul = np.zeros((ne, N), complex, order="F")
        li = np.zeros((ne, ne), complex, order="F")
        _check(load_library().dqmc_gpu_get_proj(self.h, c, _ptr(ur), _ptr(ul), _ptr(li)), "get_proj")
        return ur, ul, li

    def set_proj_state(self, ur=None, ul=None, ulrinv=None, c: int = 0) -> None:
        keep = [None if a is None else np.asfortranarray(a, complex) for a in (ur, ul, ulrinv)]
        ptrs = [None if a is None else _ptr(a) for a in keep]
        _check(load_library().dqmc_gpu_set_proj(self.h, c, *ptrs), "set_proj")

    def proj_update(self, nt: int, nf: int) -> None:
        _check(load_library().dqmc_gpu_proj_update(self.h, nt, nf), "proj_update")

    def proj_green(self) -> None:
        _check(load_library().dqmc_gpu_proj_green(self.h), "proj_green")

    def test_qr(self, a: int, q: int) -> np.ndarray:
        ld = np.zeros(2 * self.n_chains)
        _check(load_library().dqmc_gpu_test_qr(self.h, a, q, _ptr(ld)), "test_qr")
        return ld.view(complex)
