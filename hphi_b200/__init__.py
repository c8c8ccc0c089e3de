"""hphi_b200: B200 engine for HPhi's matrix-free H*v and the Lanczos / TPQ loops.

The compute path is the CUDA shared library ``libhphi_b200.so`` built from
``hphi_b200/csrc`` (see ``build.py``); this module is a thin ctypes binding over its
C-ABI (``include/hphi_b200.h``).  Names follow the reference's operator set:

  ========================  ==================================================
  this module               reference (HPhi 3.5.2)
  ========================  ==================================================
  ``Hamiltonian(path)``     ReadDefFileNInt / ReadDefFileIdxPara, check, setmem_large
                            (src/readdef.c:463,1006; src/check.c:51; src/xsetmem.c:153)
  ``H.sz()``                sz (src/sz.c:62) -> list_1, list_2_1, list_2_2
  ``H.diagonalcalc()``      diagonalcalc (src/diagonalcalc.c:84) -> list_Diagonal
  ``H.mltply(v0, v1)``      mltply (src/mltply.c:56): v0 += H v1, returns prdct
  ``H.calc_by_lanczos()``   CalcByLanczos (src/CalcByLanczos.c:55)
  ``H.calc_by_tpq()``       CalcByTPQ (src/CalcByTPQ.c:52)
  ========================  ==================================================

Host vectors use HPhi's layout (complex128, length dim+1, element 0 unused).  There
is no CPU fallback: if the library or a CUDA device is missing the calls raise.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

__all__ = ["Hamiltonian", "Batch", "Server", "HPhiError", "inspect_terms", "inspect_green", "standard_mode",
           "load_library",
           "library_path", "REAL64", "COMPLEX128", "INFO_FIELDS", "EXPORTED_SYMBOLS"]

REAL64 = 0
COMPLEX128 = 1
_HERE = os.path.dirname(os.path.abspath(__file__))
INFO_FIELDS = ["dim", "nsite", "calc_model", "calc_type", "size_list_2_1", "size_list_2_2", "is_gc",
               "vec_type", "n_offdiag", "n_diag", "lanczos_max", "num_ave", "native_order", "exct", "kernel",
               "n_green_one", "n_green_two"]
EXPORTED_SYMBOLS = ["hphi_version", "hphi_last_error", "hphi_open_expert", "hphi_close", "hphi_info",
                    "hphi_sz", "hphi_diagonalcalc", "hphi_mltply", "hphi_mltply_device", "hphi_lanczos",
                    "hphi_lanczos_eigenvector", "hphi_tpq", "hphi_tem", "hphi_run", "hphi_inspect_terms",
                    "hphi_lanczos_tridiagonal", "hphi_mltply_device_async", "hphi_stream",
                    "hphi_synchronize", "hphi_to_native", "hphi_from_native", "hphi_mltply_device_noalloc",
                    "hphi_lanczos_steps", "hphi_batch_create", "hphi_batch_lanczos", "hphi_batch_tuning",
                    "hphi_batch_free", "hphi_server_create", "hphi_server_submit", "hphi_server_step",
                    "hphi_server_poll", "hphi_server_clock", "hphi_server_free", "hphi_lobpcg",
                    "hphi_reference_start", "hphi_expec_green", "hphi_expec_cisajs", "hphi_expec_cisajscktaltdc",
                    "hphi_inspect_green", "hphi_expec_green_device", "hphi_spectrum",
                    "hphi_stdface"]
FP64 = 0
FP32 = 1
BATCH_GRAPH = 1
BATCH_REFINE = 2
BATCH_RESULT_FIELDS = 5
SERVE_RESULT_FIELDS = 8


class HPhiError(RuntimeError):
    """A C-ABI call returned an error status."""


def library_path() -> str:
    return os.environ.get("HPHI_B200_LIB", os.path.join(_HERE, "libhphi_b200.so"))


_lib: Optional[ctypes.CDLL] = None


def load_library() -> ctypes.CDLL:
    """Loads libhphi_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not os.path.exists(path):
        raise HPhiError(f"{path} not found: build it with `python -m hphi_b200.build` "
                        "(there is no CPU fallback)")
    lib = ctypes.CDLL(path)
    P, I, D, VP = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p
    pd = ctypes.POINTER(ctypes.c_double)
    pu64 = ctypes.POINTER(ctypes.c_uint64)
    pi64 = ctypes.POINTER(ctypes.c_int64)
    lib.hphi_version.restype = ctypes.c_char_p
    lib.hphi_last_error.restype = ctypes.c_char_p
    lib.hphi_open_expert.argtypes = [ctypes.c_char_p, I, ctypes.POINTER(P)]
    lib.hphi_close.argtypes = [P]
    lib.hphi_close.restype = None
    lib.hphi_info.argtypes = [P, pi64, I]
    lib.hphi_sz.argtypes = [P, pu64, pu64, pu64]
    lib.hphi_diagonalcalc.argtypes = [P, pd]
    lib.hphi_mltply.argtypes = [P, pd, pd, pd]
    lib.hphi_mltply_device.argtypes = [P, I, VP, VP, D, D, pd]
    lib.hphi_lanczos.argtypes = [P, pd, ctypes.c_char_p, pd, I]
    lib.hphi_lanczos_eigenvector.argtypes = [P, pd]
    lib.hphi_tpq.argtypes = [P, pd, ctypes.c_char_p, pd, I]
    lib.hphi_tem.argtypes = [P, pd, ctypes.c_char_p, pd, I]
    lib.hphi_run.argtypes = [P, ctypes.c_char_p]
    lib.hphi_spectrum.argtypes = [P, pd, ctypes.c_char_p, pd, I]
    lib.hphi_mltply_device_async.argtypes = [P, I, VP, VP, VP, VP]
    lib.hphi_mltply_device_noalloc.argtypes = [P, I, VP, VP, D, D, pd]
    lib.hphi_to_native.argtypes = [P, I, VP, VP]
    lib.hphi_from_native.argtypes = [P, I, VP, VP]
    lib.hphi_stream.argtypes = [P]
    lib.hphi_stream.restype = ctypes.c_void_p
    lib.hphi_synchronize.argtypes = [P]
    lib.hphi_lanczos_tridiagonal.argtypes = [P, pd, pd, I, ctypes.POINTER(I)]
    lib.hphi_inspect_terms.argtypes = [ctypes.c_char_p, pu64, pd, I, pu64, pd, I, pi64]
    lib.hphi_lanczos_steps.argtypes = [P, I, ctypes.c_uint64, pd, I]
    lib.hphi_lobpcg.argtypes = [P, pd, ctypes.c_char_p, pd, I]
    lib.hphi_batch_create.argtypes = [ctypes.POINTER(P), I, I, ctypes.POINTER(P)]
    lib.hphi_batch_lanczos.argtypes = [P, I, ctypes.c_uint64, I, D, pd, pd]
    lib.hphi_batch_tuning.argtypes = [P, I, ctypes.POINTER(I)]
    lib.hphi_batch_free.argtypes = [P]
    lib.hphi_batch_free.restype = None
    lib.hphi_server_create.argtypes = [I, I, ctypes.c_int64, I, I, ctypes.POINTER(P)]
    lib.hphi_server_submit.argtypes = [P, ctypes.c_char_p, ctypes.c_uint64, D, pi64]
    lib.hphi_server_step.argtypes = [P, pi64]
    lib.hphi_server_poll.argtypes = [P, pi64, pd]
    lib.hphi_server_clock.argtypes = []
    lib.hphi_server_clock.restype = D
    lib.hphi_server_free.argtypes = [P]
    lib.hphi_server_free.restype = None
    lib.hphi_reference_start.argtypes = [ctypes.c_int64, I, I, I, I, I, I, pd]
    pint = ctypes.POINTER(I)
    lib.hphi_expec_green.argtypes = [P, I, I, pint, pd, pd]
    lib.hphi_expec_cisajs.argtypes = [P, pd, pd, ctypes.c_char_p]
    lib.hphi_expec_cisajscktaltdc.argtypes = [P, pd, pd, ctypes.c_char_p]
    lib.hphi_inspect_green.argtypes = [ctypes.c_char_p, I, pint, I]
    lib.hphi_expec_green_device.argtypes = [P, I, I, pint, I, VP, pd]
    for name in EXPORTED_SYMBOLS:
        if name not in ("hphi_version", "hphi_last_error", "hphi_close", "hphi_stream", "hphi_batch_free",
                        "hphi_server_clock", "hphi_server_free"):
            getattr(lib, name).restype = I
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != 0:
        raise HPhiError(load_library().hphi_last_error().decode())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _as_hphi_vector(v: np.ndarray, dim: int) -> np.ndarray:
    v = np.ascontiguousarray(v, dtype=np.complex128)
    if v.shape != (dim + 1,):
        raise ValueError(f"expected an HPhi vector of length dim+1 = {dim + 1}, got {v.shape}")
    return v


REF_LANCZOS, REF_TPQ, REF_LOBPCG = 0, 1, 2


def reference_start(dim: int, kind: int = REF_LANCZOS, initial_iv: int = -1, sample: int = 0, vec_type: int = 1,
                    threads: int = 1, count: int = 1) -> np.ndarray:
    """The reference's random start vector(s) drawn with `threads` OpenMP threads (dSFMT-19937
    per thread, static-schedule rows): an array (count, dim + 1) of complex128 in HPhi's layout
    (element 0 unused); Lanczos / LOBPCG vectors are normalised, TPQ ones are not."""
    v = np.zeros((max(count, 1), dim + 1), dtype=np.complex128)
    _check(load_library().hphi_reference_start(int(dim), int(kind), int(initial_iv), int(sample), int(vec_type),
                                               int(threads), int(count), _dptr(v.view(np.float64))))
    return v


def standard_mode(stan_in: str, out_dir: str) -> str:
    """Standard mode (`HPhi -sdry stan.in`): writes the expert-mode files of the keyword file
    `stan_in` into `out_dir`; returns the path of the namelist.def written there.  Host only."""
    lib = load_library()
    lib.hphi_stdface.argtypes = [ctypes.c_char_p, ctypes.c_char_p]
    os.makedirs(out_dir, exist_ok=True)
    _check(lib.hphi_stdface(stan_in.encode(), out_dir.encode()))
    return os.path.join(out_dir, "namelist.def")


def inspect_terms(namelist_def: str):
    """Compiled terms of an expert-mode input, read on the host (no device needed).

    Returns (masks[n_off, 4] = (cm, cv, flip, sign_mask), coefs[n_off] complex,
    dmasks[n_diag, 2] = (cm, cv), dcoefs[n_diag])."""
    lib = load_library()
    counts = (ctypes.c_int64 * 2)()
    path = os.fsencode(namelist_def)
    _check(lib.hphi_inspect_terms(path, None, None, 0, None, None, 0, counts))
    no, nd = int(counts[0]), int(counts[1])
    masks = np.zeros((max(no, 1), 4), dtype=np.uint64)
    coefs = np.zeros((max(no, 1), 2))
    dmasks = np.zeros((max(nd, 1), 2), dtype=np.uint64)
    dcoefs = np.zeros(max(nd, 1))
    pu = ctypes.POINTER(ctypes.c_uint64)
    _check(lib.hphi_inspect_terms(path, masks.ctypes.data_as(pu), _dptr(coefs), no, dmasks.ctypes.data_as(pu),
                                  _dptr(dcoefs), nd, counts))
    return masks[:no], coefs[:no, 0] + 1j * coefs[:no, 1], dmasks[:nd], dcoefs[:nd]


def inspect_green(namelist_def: str, body: int) -> np.ndarray:
    """OneBodyG (body 1: rows of 4 ints) or TwoBodyG (body 2: rows of 8 ints) rows of an
    expert-mode input as the reader keeps them, read on the host (no device needed)."""
    lib = load_library()
    path = os.fsencode(namelist_def)
    w = 4 * (1 if body == 1 else 2 if body == 2 else body)
    cap = 1 << 16
    while True:  # one read (and one set of reader warnings) unless the rows exceed the buffer
        rows = np.zeros((cap, w), dtype=np.int32)
        n = lib.hphi_inspect_green(path, int(body), rows.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), cap)
        if n < 0:
            raise HPhiError(lib.hphi_last_error().decode())
        if n <= cap:
            return rows[:n]
        cap = n


class Hamiltonian:
    """An expert-mode HPhi input resident on one CUDA device."""

    def __init__(self, namelist_def: str, device: int = 0):
        lib = load_library()
        h = ctypes.c_void_p()
        _check(lib.hphi_open_expert(os.fsencode(namelist_def), int(device), ctypes.byref(h)))
        self._h = h
        self.device = device
        info = (ctypes.c_int64 * len(INFO_FIELDS))()
        _check(lib.hphi_info(h, info, len(INFO_FIELDS)))
        self.info = {k: int(info[i]) for i, k in enumerate(INFO_FIELDS)}
        self.dim = self.info["dim"]

    # -------------------------------------------------------------- lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            load_library().hphi_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    # ------------------------------------------------------------ reference ops
    def sz(self):
        """list_1 (length dim+1), list_2_1, list_2_2 as uint64 arrays (HPhi layout)."""
        l1 = np.zeros(self.dim + 1, dtype=np.uint64)
        l21 = np.zeros(self.info["size_list_2_1"], dtype=np.uint64)
        l22 = np.zeros(self.info["size_list_2_2"], dtype=np.uint64)
        pu = ctypes.POINTER(ctypes.c_uint64)
        _check(load_library().hphi_sz(self._h, l1.ctypes.data_as(pu), l21.ctypes.data_as(pu),
                                      l22.ctypes.data_as(pu)))
        return l1, l21, l22

    def diagonalcalc(self) -> np.ndarray:
        d = np.zeros(self.dim + 1, dtype=np.float64)
        _check(load_library().hphi_diagonalcalc(self._h, _dptr(d)))
        return d

    def mltply(self, v0: np.ndarray, v1: np.ndarray) -> complex:
        """v0 += H v1 in place (HPhi layout, complex128); returns prdct = <v1|H|v1>."""
        if not (isinstance(v0, np.ndarray) and v0.dtype == np.complex128 and v0.flags.c_contiguous):
            raise TypeError("v0 must be a contiguous complex128 array (it is updated in place)")
        _as_hphi_vector(v0, self.dim)
        v1 = _as_hphi_vector(v1, self.dim)
        pr = np.zeros(2)
        _check(load_library().hphi_mltply(self._h, _dptr(v0.view(np.float64)), _dptr(v1.view(np.float64)),
                                          _dptr(pr)))
        return complex(pr[0], pr[1])

    def expec_green(self, vec: np.ndarray, rows, body: int) -> np.ndarray:
        """<vec| O |vec> for Green's function rows (body 1: (i, s1, j, s2) -> c+_{i s1} c_{j s2};
        body 2: (i, s1, j, s2, k, s3, l, s4) -> c+ c c+ c; spin models: site transitions),
        with the reference's rules per model; vec in HPhi's layout.  Complex array per row."""
        vec = _as_hphi_vector(vec, self.dim)
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1, 4 * (1 if body == 1 else 2 if body == 2
                                                                                     else body)))
        out = np.zeros(2 * max(len(r), 1))
        _check(load_library().hphi_expec_green(self._h, int(body), len(r),
                                               r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                               _dptr(vec.view(np.float64)), _dptr(out)))
        return out[0:2 * len(r):2] + 1j * out[1:2 * len(r):2]

    def expec_green_device(self, vec_ptr: int, vec_type: int, rows, body: int) -> np.ndarray:
        """expec_green on a device vector in HPhi's row order (REAL64 or COMPLEX128)."""
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1, 4 * (1 if body == 1 else 2 if body == 2
                                                                                     else body)))
        out = np.zeros(2 * max(len(r), 1))
        _check(load_library().hphi_expec_green_device(self._h, int(body), len(r),
                                                      r.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                      int(vec_type), ctypes.c_void_p(vec_ptr), _dptr(out)))
        return out[0:2 * len(r):2] + 1j * out[1:2 * len(r):2]

    def expec_cisajs(self, vec: np.ndarray, path: Optional[str] = None) -> np.ndarray:
        """expec_cisajs for the input's OneBodyG rows; writes the reference's file when path is given."""
        return self._expec_model_green(1, vec, path)

    def expec_cisajscktaltdc(self, vec: np.ndarray, path: Optional[str] = None) -> np.ndarray:
        """expec_cisajscktaltdc for the input's TwoBodyG rows; writes the reference's file when path is given."""
        return self._expec_model_green(2, vec, path)

    def _expec_model_green(self, body: int, vec: np.ndarray, path: Optional[str]) -> np.ndarray:
        vec = _as_hphi_vector(vec, self.dim)
        n = self.info["n_green_one" if body == 1 else "n_green_two"]
        out = np.zeros(2 * max(n, 1))
        fn = load_library().hphi_expec_cisajs if body == 1 else load_library().hphi_expec_cisajscktaltdc
        _check(fn(self._h, _dptr(vec.view(np.float64)), _dptr(out), os.fsencode(path) if path else None))
        return out[0:2 * n:2] + 1j * out[1:2 * n:2]

    def mltply_device(self, v0_ptr: int, v1_ptr: int, vec_type: int, acc: float = 1.0,
                      scale: float = 1.0) -> complex:
        """Device form: v0 = acc*v0 + scale*H v1 on 0-based device arrays (raw pointers)."""
        pr = np.zeros(2)
        _check(load_library().hphi_mltply_device(self._h, int(vec_type), ctypes.c_void_p(v0_ptr),
                                                 ctypes.c_void_p(v1_ptr), float(acc), float(scale), _dptr(pr)))
        return complex(pr[0], pr[1])

    def mltply_device_async(self, v0_ptr: int, v1_ptr: int, vec_type: int, coef_ptr: int, prdct_ptr: int) -> None:
        """Enqueue v0 = coef[0]*v0 + coef[1]*H v1 on the handle's stream (all device pointers)."""
        _check(load_library().hphi_mltply_device_async(self._h, int(vec_type), ctypes.c_void_p(v0_ptr),
                                                       ctypes.c_void_p(v1_ptr), ctypes.c_void_p(coef_ptr),
                                                       ctypes.c_void_p(prdct_ptr)))

    def mltply_device_noalloc(self, v0_ptr: int, v1_ptr: int, vec_type: int, acc: float = 1.0,
                              scale: float = 1.0) -> complex:
        """v0 = acc*v0 + scale*H v1 on native-order device vectors without allocating device
        memory: the call's scratch is a fixed static device array shared by all calls on the
        device, so calls must not overlap on the GPU.  Waits for the stream; returns prdct."""
        pr = np.zeros(2)
        _check(load_library().hphi_mltply_device_noalloc(self._h, int(vec_type), ctypes.c_void_p(v0_ptr),
                                                         ctypes.c_void_p(v1_ptr), float(acc), float(scale),
                                                         _dptr(pr)))
        return complex(pr[0], pr[1])

    def to_native(self, in_ptr: int, out_ptr: int, vec_type: int) -> None:
        """HPhi order -> the engine's native order (0-based device vectors, in != out)."""
        _check(load_library().hphi_to_native(self._h, int(vec_type), ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr)))

    def from_native(self, in_ptr: int, out_ptr: int, vec_type: int) -> None:
        """Native order -> HPhi order (0-based device vectors, in != out)."""
        _check(load_library().hphi_from_native(self._h, int(vec_type), ctypes.c_void_p(in_ptr),
                                               ctypes.c_void_p(out_ptr)))

    def mltply_raw(self, v0_ptr: int, v1_ptr: int) -> complex:
        """mltply on raw host pointers (HPhi layout, complex128, dim+1 elements each)."""
        pr = np.zeros(2)
        pd = ctypes.POINTER(ctypes.c_double)
        _check(load_library().hphi_mltply(self._h, ctypes.cast(v0_ptr, pd), ctypes.cast(v1_ptr, pd), _dptr(pr)))
        return complex(pr[0], pr[1])

    @property
    def stream(self) -> int:
        """cudaStream_t of the handle (as an integer), for external events / streams."""
        return int(load_library().hphi_stream(self._h) or 0)

    def synchronize(self) -> None:
        _check(load_library().hphi_synchronize(self._h))

    def calc_by_lanczos(self, v_init: Optional[np.ndarray] = None, output_dir: Optional[str] = None) -> dict:
        res = np.zeros(17)
        vi = None if v_init is None else _as_hphi_vector(v_init, self.dim)
        _check(load_library().hphi_lanczos(self._h, None if vi is None else _dptr(vi.view(np.float64)),
                                           None if output_dir is None else os.fsencode(output_dir),
                                           _dptr(res), len(res)))
        keys = ["converged", "steps", "e_target", "e1", "e2", "e3", "e4", "energy", "var", "doublon", "sz",
                "check_diff", "check_var", "cg_rounds", "cg_iterations", "cg_diff", "cg_var"]
        out = {k: float(res[i]) for i, k in enumerate(keys)}
        out["converged"] = bool(res[0])
        out["steps"] = int(res[1])
        out["cg_rounds"] = int(res[13])
        out["cg_iterations"] = int(res[14])
        return out

    def lanczos_tridiagonal(self):
        """(alpha, beta) of the last calc_by_lanczos run (reference's alpha[1..itr], beta[1..itr])."""
        steps = ctypes.c_int()
        _check(load_library().hphi_lanczos_tridiagonal(self._h, None, None, 0, ctypes.byref(steps)))
        n = steps.value
        a, b = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        _check(load_library().hphi_lanczos_tridiagonal(self._h, _dptr(a), _dptr(b), n, ctypes.byref(steps)))
        return a[:n], b[:n]

    def lanczos_eigenvector(self) -> np.ndarray:
        v = np.zeros(self.dim + 1, dtype=np.complex128)
        _check(load_library().hphi_lanczos_eigenvector(self._h, _dptr(v.view(np.float64))))
        return v

    def calc_by_tpq(self, v_init: Optional[Sequence[np.ndarray]] = None, output_dir: Optional[str] = None,
                    nresult: Optional[int] = None) -> np.ndarray:
        n = nresult or self.info["lanczos_max"]
        res = np.zeros(n)
        buf = None
        if v_init is not None:
            buf = np.ascontiguousarray(np.stack([_as_hphi_vector(v, self.dim) for v in v_init]))
            if buf.shape[0] < self.info["num_ave"]:
                raise ValueError("need one start vector per TPQ sample (NumAve)")
        _check(load_library().hphi_tpq(self._h, None if buf is None else _dptr(buf.view(np.float64)),
                                       None if output_dir is None else os.fsencode(output_dir), _dptr(res), n))
        return res

    def calc_by_tem(self, v_init: Optional[np.ndarray] = None, output_dir: Optional[str] = None,
                    nresult: Optional[int] = None) -> np.ndarray:
        """Real-time evolution (CalcByTEM, CalcType 4) from v_init (HPhi layout, dim+1
        complex128) or, when None, from <SpectrumVec>_rank_0.dat in output_dir.  Writes SS.dat,
        Norm.dat, Flct.dat and the step files; returns the energy of each step."""
        n = nresult or self.info["lanczos_max"]
        res = np.zeros(n)
        buf = None if v_init is None else np.ascontiguousarray(_as_hphi_vector(v_init, self.dim))
        _check(load_library().hphi_tem(self._h, None if buf is None else _dptr(buf.view(np.float64)),
                                       None if output_dir is None else os.fsencode(output_dir), _dptr(res), n))
        return res

    def calc_spectrum(self, vec: Optional[np.ndarray] = None, output_dir: Optional[str] = None,
                      n_omega: int = 0) -> np.ndarray:
        """Dynamical Green's function (CalcSpectrum with CalcSpec 1, Lanczos): the excitation
        operators of the input act on vec (HPhi layout, dim+1 complex128) or, when None, on
        <SpectrumVec>_rank_0.dat in output_dir; writes <head>_DynamicalGreen.dat and
        <head>_TMComponents.dat.  Returns (n_omega, 2) complex: omega (OmegaOrg included), G."""
        res = np.zeros(4 * max(n_omega, 0))
        buf = None if vec is None else np.ascontiguousarray(_as_hphi_vector(vec, self.dim))
        _check(load_library().hphi_spectrum(self._h, None if buf is None else _dptr(buf.view(np.float64)),
                                            None if output_dir is None else os.fsencode(output_dir),
                                            _dptr(res) if n_omega > 0 else None, int(n_omega)))
        r = res.reshape(-1, 4)
        return np.stack([r[:, 0] + 1j * r[:, 1], r[:, 2] + 1j * r[:, 3]], axis=1)

    def calc_by_lobpcg(self, v_init: Optional[Sequence[np.ndarray]] = None,
                       output_dir: Optional[str] = None) -> dict:
        """Block LOBPCG for the exct lowest states (CalcByLOBPCG).  v_init: exct start vectors
        in HPhi layout (dim+1 complex128 each).  Returns converged, steps, residual and per-state
        energy, var (<Hx|Hx>), doublon, sz arrays; raises if not converged."""
        k = max(1, self.info["exct"])
        buf = None
        if v_init is not None:
            buf = np.ascontiguousarray(np.stack([_as_hphi_vector(v, self.dim) for v in v_init]))
        n = 3 + 4 * k
        res = np.zeros(n)
        rc = load_library().hphi_lobpcg(self._h, None if buf is None else _dptr(buf.view(np.float64)),
                                        None if output_dir is None else os.fsencode(output_dir), _dptr(res), n)
        out = {"converged": bool(res[0]), "steps": int(res[1]), "residual": float(res[2])}
        per = res[3:].reshape(k, 4)
        for j, key in enumerate(["energy", "var", "doublon", "sz"]):
            out[key] = per[:k, j].copy()
        if rc != 0:
            raise HPhiError(load_library().hphi_last_error().decode())
        return out

    def run(self, output_dir: str = "output") -> None:
        _check(load_library().hphi_run(self._h, os.fsencode(output_dir)))

    def lanczos_steps(self, steps: int, seed: int = 1, nev: int = 4) -> np.ndarray:
        """Fixed-length Lanczos (exactly `steps` steps, convergence test off) from the hashed
        start vector of `seed`; returns the nev lowest tridiagonal eigenvalues."""
        e = np.zeros(max(nev, 1))
        _check(load_library().hphi_lanczos_steps(self._h, int(steps), ctypes.c_uint64(seed), _dptr(e), nev))
        return e[:nev]


class Batch:
    """Many open Hamiltonians advanced together by the batched Lanczos engine.

    precision FP64 or FP32 (vector storage; sums, dots and scalars stay FP64).  The
    Hamiltonians must stay open while the batch lives."""

    def __init__(self, hamiltonians: Sequence[Hamiltonian], precision: int = FP64):
        lib = load_library()
        self._members = list(hamiltonians)
        arr = (ctypes.c_void_p * len(self._members))(*[h.handle.value for h in self._members])
        b = ctypes.c_void_p()
        _check(lib.hphi_batch_create(arr, len(self._members), int(precision), ctypes.byref(b)))
        self._b = b
        self.precision = precision

    def __len__(self):
        return len(self._members)

    def lanczos(self, steps: int, seed: int = 1, graph: bool = True, refine: bool = False,
                replay_tol: float = 1e-9) -> dict:
        """`steps` Lanczos steps for every instance (instance i starts from the hashed vector
        of seed + 1000003*i).  With refine, the ground state is rebuilt (replay truncated where
        the rest of the Ritz vector is below replay_tol) and refined in FP64.  Returns arrays
        e_lanczos, e_refined, residual, steps, replay_steps and the phase timings in ms."""
        n = len(self._members)
        res = np.zeros(n * BATCH_RESULT_FIELDS)
        tim = np.zeros(4)
        flags = (BATCH_GRAPH if graph else 0) | (BATCH_REFINE if refine else 0)
        _check(load_library().hphi_batch_lanczos(self._b, int(steps), ctypes.c_uint64(seed), flags,
                                                 float(replay_tol), _dptr(res), _dptr(tim)))
        r = res.reshape(n, BATCH_RESULT_FIELDS)
        return {"e_lanczos": r[:, 0].copy(), "e_refined": r[:, 1].copy(), "residual": r[:, 2].copy(),
                "steps": r[:, 3].astype(int), "replay_steps": r[:, 4].astype(int),
                "forward_ms": float(tim[0]), "replay_ms": float(tim[1]), "refine_ms": float(tim[2]),
                "tuned_hv_ms": float(tim[3])}

    def tuning(self, retune: bool = False) -> dict:
        shape = (ctypes.c_int * 3)()
        _check(load_library().hphi_batch_tuning(self._b, 1 if retune else 0, shape))
        return {"threads": shape[0], "rows_per_thread": shape[1], "ctas_per_sm": shape[2]}

    def close(self) -> None:
        if getattr(self, "_b", None) is not None and self._b.value:
            load_library().hphi_batch_free(self._b)
            self._b = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching Lanczos request server on one device (see hphi_server_create)."""

    FIELDS = ["status", "energy", "e_lanczos", "residual", "steps", "dim", "wait_s", "latency_s"]

    def __init__(self, device: int = 0, precision: int = FP64, hbm_budget: int = 0, max_active: int = 64,
                 steps_per_iteration: int = 16):
        lib = load_library()
        s = ctypes.c_void_p()
        _check(lib.hphi_server_create(int(device), int(precision), int(hbm_budget), int(max_active),
                                      int(steps_per_iteration), ctypes.byref(s)))
        self._s = s

    @staticmethod
    def clock() -> float:
        return float(load_library().hphi_server_clock())

    def submit(self, namelist_def: str, seed: int = 1, arrival: float = -1.0) -> int:
        rid = ctypes.c_int64()
        _check(load_library().hphi_server_submit(self._s, os.fsencode(namelist_def), ctypes.c_uint64(seed),
                                                 float(arrival), ctypes.byref(rid)))
        return rid.value

    def step(self) -> dict:
        c = (ctypes.c_int64 * 3)()
        _check(load_library().hphi_server_step(self._s, c))
        return {"active": c[0], "queued": c[1], "finished": c[2]}

    def poll(self) -> list:
        """All finished requests as (request_id, dict) pairs."""
        out = []
        lib = load_library()
        while True:
            rid = ctypes.c_int64()
            res = np.zeros(SERVE_RESULT_FIELDS)
            rc = lib.hphi_server_poll(self._s, ctypes.byref(rid), _dptr(res))
            if rc < 0:
                raise HPhiError(lib.hphi_last_error().decode())
            if rc == 0:
                return out
            d = {k: float(res[i]) for i, k in enumerate(self.FIELDS)}
            d["status"] = int(res[0])
            d["steps"] = int(res[4])
            d["dim"] = int(res[5])
            if d["status"] < 0:
                d["error"] = lib.hphi_last_error().decode()
            out.append((rid.value, d))

    def close(self) -> None:
        if getattr(self, "_s", None) is not None and self._s.value:
            load_library().hphi_server_free(self._s)
            self._s = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
