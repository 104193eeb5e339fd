"""Python mirror of magnum.af's script API (python/magnumaf.pyx) over the
B200 C ABI (include/maf_b200.h).

Class and method names, argument meaning and defaults follow the reference's
Cython module: ``Mesh``, ``State``, ``DemagField``, ``ExchangeField``,
``DmiField``, ``BulkDMIExchangeField``, ``UniaxialAnisotropyField``,
``CubicAnisotropyField``, ``ExternalField``, ``LLGIntegrator`` and
``Constants``.  ArrayFire arrays are replaced by NumPy arrays of the same
shape: a vector field is ``(nx, ny, nz, 3)``, a scalar field ``(nx, ny, nz)``
(or ``(nx, ny, nz, 1)``).  Arrays returned by the library are Fortran-ordered,
i.e. exactly the reference's column-major memory.

The compute path is the CUDA library ``libmafb200.so`` only; importing this
module fails loudly when the library is missing, and every compute call
raises ``MafError`` when no GPU is available.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.normpath(os.path.join(_HERE, "..", "..", "lib", "libmafb200.so"))

if not os.path.exists(_LIB_PATH):
    raise ImportError(
        "libmafb200.so not found at %s; build it with `python magnum.af_b200/build.py` "
        "(there is no CPU fallback)" % _LIB_PATH)

lib = C.CDLL(_LIB_PATH)

_P = C.c_void_p
_D = C.c_double
_I = C.c_int
_DP = C.POINTER(C.c_double)
_FP = C.POINTER(C.c_float)

# exported symbols and their signatures (include/maf_b200.h)
_SIGS = {
    "maf_last_error": (C.c_char_p, []),
    "maf_version": (_I, [C.POINTER(_I), C.POINTER(_I)]),
    "maf_device_count": (_I, [C.POINTER(_I)]),
    "maf_state_create": (_I, [C.POINTER(_P), _I, _I, _I, _D, _D, _D, _D, _DP, _DP, _I]),
    "maf_state_destroy": (_I, [_P]),
    "maf_state_get_m": (_I, [_P, _DP]),
    "maf_state_set_m": (_I, [_P, _DP]),
    "maf_state_load_m": (_I, [_P, _DP]),
    "maf_state_get_t": (_I, [_P, _DP]),
    "maf_state_set_t": (_I, [_P, _D]),
    "maf_state_get_steps": (_I, [_P, C.POINTER(C.c_ulonglong)]),
    "maf_state_mean_m": (_I, [_P, _DP]),
    "maf_state_get_Ms_field": (_I, [_P, _DP, C.POINTER(_I)]),
    "maf_state_get_Ms": (_I, [_P, _DP]),
    "maf_state_set_stream": (_I, [_P, _P]),
    "maf_state_device_m": (_I, [_P, C.POINTER(_P)]),
    "maf_state_precision": (_I, [_P, C.POINTER(_I)]),
    "maf_term_demag_create": (_I, [C.POINTER(_P), _I, _I, _I, _D, _D, _D]),
    "maf_term_demag_create_from_tensor": (_I, [C.POINTER(_P), _I, _I, _I, _D, _D, _D, _DP]),
    "maf_term_exchange_create": (_I, [C.POINTER(_P), _D]),
    "maf_term_dmi_create": (_I, [C.POINTER(_P), _D, _D, _D, _D]),
    "maf_term_dmi_field_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP, _D, _D, _D]),
    "maf_term_bulkdmi_exchange_create": (_I, [C.POINTER(_P), _D, _D]),
    "maf_term_uniaxial_create": (_I, [C.POINTER(_P), _D, _D, _D, _D]),
    "maf_term_uniaxial_field_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP, _D, _DP, _D, _D, _D]),
    "maf_term_cubic_create": (_I, [C.POINTER(_P), _D, _D, _D, _DP, _DP]),
    "maf_term_external_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP]),
    "maf_term_external_uniform_create": (_I, [C.POINTER(_P), _D, _D, _D]),
    "maf_term_stt_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP, _D, _D, _D, _D]),
    "maf_term_sparse_exchange_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP, _D]),
    "maf_term_demag_pbc_create": (_I, [C.POINTER(_P)]),
    "maf_term_exchange_pbc_create": (_I, [C.POINTER(_P), _I, _I, _I, _DP, _D]),
    "maf_term_destroy": (_I, [_P]),
    "maf_term_H": (_I, [_P, _P, _DP]),
    "maf_term_H_f32": (_I, [_P, _P, _FP]),
    "maf_term_E": (_I, [_P, _P, _DP]),
    "maf_term_demag_tensor": (_I, [_P, _DP]),
    "maf_term_demag_real_tensor": (_I, [_P, _DP, _I]),
    "maf_llg_create": (_I, [C.POINTER(_P), _D, _DP, _I, _I, _I, C.POINTER(_P), _I, C.c_char_p, _D, _D, _D, _D, _I]),
    "maf_llg_destroy": (_I, [_P]),
    "maf_llg_add_term": (_I, [_P, _P]),
    "maf_llg_set_alpha": (_I, [_P, _D]),
    "maf_llg_step": (_I, [_P, _P]),
    "maf_llg_steps": (_I, [_P, _P, _I]),
    "maf_llg_E": (_I, [_P, _P, _DP]),
    "maf_llg_heff": (_I, [_P, _P, _DP]),
    "maf_llg_heff_f32": (_I, [_P, _P, _FP]),
    "maf_llg_heff_device": (_I, [_P, _P, _P, _P]),
    "maf_llg_heff_pipeline": (_I, [_P, _P, C.POINTER(_P), C.POINTER(_P), _I]),
    "maf_llg_heff_pipeline_m32": (_I, [_P, _P, C.POINTER(_P), C.POINTER(_P), _I]),
    "maf_llg_autotune": (_I, [_P, _P, _I, C.POINTER(_I), _DP]),
    "maf_llg_autotune_ex": (_I, [_P, _P, _I, C.POINTER(_I), _DP, C.POINTER(_I)]),
    "maf_term_demag_get_tune_ex": (_I, [_P, C.POINTER(_I)]),
    "maf_term_demag_set_tune_ex": (_I, [_P, C.POINTER(_I)]),
    "maf_term_demag_get_tune": (_I, [_P, C.POINTER(_I)]),
    "maf_term_demag_set_tune": (_I, [_P, C.POINTER(_I)]),
    "maf_llg_heff_device_profile": (_I, [_P, _P, _P, _P, _DP, _I, C.POINTER(_I)]),
    "maf_llg_pass_name": (_I, [_P, _P, _I, C.c_char_p, _I]),
    "maf_llg_attempt_profile": (_I, [_P, _P, C.c_double, _DP, _I, C.POINTER(_I)]),
    "maf_llg_profile_name": (_I, [_P, _I, C.c_char_p, _I]),
    "maf_llg_dmdt": (_I, [_P, _P, _DP]),
    "maf_llg_integrate_dense": (_I, [_P, _P, _D, _D, _DP, _I, C.POINTER(_I)]),
    "maf_llg_rk_attempt": (_I, [_P, _P, C.c_char_p, _D, _DP, _DP]),
    "maf_llg_relax": (_I, [_P, _P, _D, _I]),
    "maf_stochastic_llg_create": (_I, [C.POINTER(_P), _D, _D, _D, C.POINTER(_P), _I, C.c_char_p, C.c_ulonglong,
                                       C.c_uint]),
    "maf_stochastic_llg_destroy": (_I, [_P]),
    "maf_stochastic_llg_step": (_I, [_P, _P]),
    "maf_stochastic_llg_steps": (_I, [_P, _P, _I]),
    "maf_stochastic_llg_E": (_I, [_P, _P, _DP]),
    "maf_stochastic_llg_noise": (_I, [_P, _P, C.c_ulonglong, _DP]),
    "maf_stochastic_llg_calls": (_I, [_P, C.POINTER(C.c_ulonglong)]),
    "maf_lbfgs_create": (_I, [C.POINTER(_P), C.POINTER(_P), _I, _D, _I]),
    "maf_lbfgs_destroy": (_I, [_P]),
    "maf_lbfgs_add_term": (_I, [_P, _P]),
    "maf_lbfgs_minimize": (_I, [_P, _P, _DP]),
    "maf_lbfgs_stats": (_I, [_P, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong), _DP]),
    "maf_llg_get_h": (_I, [_P, _DP]),
    "maf_llg_counters": (_I, [_P, C.POINTER(C.c_ulonglong)]),
    "maf_llg_get_controller_state": (_I, [_P, _DP]),
    "maf_llg_set_controller_state": (_I, [_P, _DP]),
    "maf_state_set_steps": (_I, [_P, C.c_ulonglong]),
    "maf_mean_m_noalloc": (_I, [_P, C.c_longlong, _DP, _P]),
    "maf_cnn_create": (_I, [C.POINTER(_P), _I, _I, _I, C.c_ulonglong]),
    "maf_cnn_set_dilation": (_I, [_P, C.POINTER(_I), _I]),
    "maf_cnn_destroy": (_I, [_P]),
    "maf_cnn_n_params": (_I, [_P, C.POINTER(C.c_longlong)]),
    "maf_cnn_get_params": (_I, [_P, _FP]),
    "maf_cnn_set_params": (_I, [_P, _FP]),
    "maf_cnn_forward": (_I, [_P, _P, _I, _I, _I, _P]),
    "maf_cnn_loss_grad": (_I, [_P, _P, _P, _I, _I, _I, _FP, _FP]),
    "maf_cnn_train_step": (_I, [_P, _P, _P, _I, _I, _I, C.c_float, _FP]),
    "maf_stoch_batch_create": (_I, [C.POINTER(_P), C.POINTER(_P), C.POINTER(_P), _I]),
    "maf_stoch_batch_destroy": (_I, [_P]),
    "maf_stoch_batch_steps": (_I, [_P, _I]),
    "maf_stoch_batch_set_fused": (_I, [_P, _I]),
    "maf_bf16_gemm": (_I, [_P, _I, _P, _I, _P, _I, _I, _I, _I, _P]),
    # layer kernels of the warm-start U-net (magnumaf.unet)
    "maf_nn_input": (_I, [_P, _I, _I, _I, _I, _I, _P, _P, _P]),
    "maf_nn_im2col": (_I, [_P, _I, _I, _I, _I, _P, _I, _P]),
    "maf_nn_gemm": (_I, [_P, _I, _P, _I, _P, _I, _I, _I, _I, _P]),
    "maf_nn_gemm_splitk": (_I, [_P, _I, _P, _I, _P, _I, _I, _I, _I, _P, _P]),
    "maf_nn_bias_act": (_I, [_P, _I, _P, C.c_longlong, _I, _I, _P, _P, _I, _P]),
    "maf_nn_pool": (_I, [_P, _I, _I, _I, _I, _P, _P, _I, _P]),
    "maf_nn_pool_bwd": (_I, [_P, _I, _I, _I, _I, _P, _I, _P]),
    "maf_nn_up_cat": (_I, [_P, _I, _P, _I, _I, _I, _I, _P, _I, _P]),
    "maf_nn_up_cat_bwd": (_I, [_P, _I, _I, _I, _I, _I, _I, _P, _P, _P]),
    "maf_nn_relu_bwd": (_I, [_P, _P, C.c_longlong, _I, _I, _P, _P, _I, _P]),
    "maf_nn_transpose": (_I, [_P, C.c_longlong, _I, _P, _P]),
    "maf_nn_col2im": (_I, [_P, _I, _I, _I, _I, _I, _P, _I, _P]),
    "maf_nn_colsum": (_I, [_P, C.c_longlong, _I, _P, _P]),
    "maf_nn_wcast": (_I, [_P, _I, _I, _I, _I, _P, _P, _P]),
    "maf_nn_wgrad": (_I, [_P, _I, _I, _I, _P, _P]),
    "maf_nn_head": (_I, [_P, _P, _I, _P, C.c_longlong, _P, _P, _P, _P, _P]),
    "maf_nn_adam": (_I, [_P, _P, _P, _P, C.c_longlong, C.c_float, _I, _P]),
    "maf_stoch_batch_is_fused": (_I, [_P, C.POINTER(_I)]),
    "maf_term_demag_set_generic": (_I, [_P, _I]),
    "maf_string_create": (_I, [C.POINTER(_P), _P, C.POINTER(_P), _I, _I, _D, _P]),
    "maf_string_destroy": (_I, [_P]),
    "maf_string_step": (_I, [_P]),
    "maf_string_set_batched": (_I, [_P, _I]),
    "maf_string_calc_E": (_I, [_P, _DP]),
    "maf_string_run": (_I, [_P, C.c_char_p, _D, _D, _I, _I, _I, _DP, C.POINTER(_I)]),
    "maf_string_n_images": (_I, [_P, C.POINTER(_I)]),
    "maf_string_get_x": (_I, [_P, _DP, _DP]),
    "maf_string_image": (_I, [_P, _I, C.POINTER(_P)]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

MAF_FP64 = 0
MAF_FP32_FIELD = 1
_PRECISION = {"fp64": MAF_FP64, "f64": MAF_FP64, MAF_FP64: MAF_FP64,
              "fp32_field": MAF_FP32_FIELD, "fp32": MAF_FP32_FIELD, MAF_FP32_FIELD: MAF_FP32_FIELD}
ERROR_NAMES = {1: "BADARG", 2: "CUDA", 3: "OOM", 4: "NAN", 5: "TIMEOUT", 6: "UNSUPPORTED", 7: "NODEVICE"}


class MafError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("[%s] %s" % (ERROR_NAMES.get(code, code), msg))
        self.code = code


def _ck(rc):
    if rc != 0:
        raise MafError(rc, lib.maf_last_error().decode())


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_DP)


def _vec_soa(a, mesh=None) -> np.ndarray:
    """(nx,ny,nz,3) -> bytes of [3][nz][ny][nx] (Fortran order of the 4-D array)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim != 4 or a.shape[3] != 3:
        raise ValueError("expected a vector field of shape (nx, ny, nz, 3), got %s" % (a.shape,))
    if mesh is not None and a.shape[:3] != (mesh.nx, mesh.ny, mesh.nz):
        raise ValueError("field shape %s does not match the mesh" % (a.shape,))
    return np.asfortranarray(a)


def _scalar_soa(a) -> np.ndarray:
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 4:
        a = a[..., 0]
    if a.ndim != 3:
        raise ValueError("expected a scalar field of shape (nx, ny, nz[, 1])")
    return np.asfortranarray(a)


class Constants:
    """magnumaf/include/magnumaf/constants.hpp:9-22"""
    mu0 = 4e-7 * math.pi
    gamma = 1.760859644e11 * mu0
    mu_b = 9.274009994e-24
    e = -1.6021766208e-19
    kb = 1.38064852e-23
    hbar = 1.0545718e-34


class Mesh:
    def __init__(self, nx, ny, nz, dx, dy, dz):
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.dx, self.dy, self.dz = float(dx), float(dy), float(dz)

    @property
    def n(self):
        return self.nx * self.ny * self.nz


def device_count() -> int:
    n = C.c_int(0)
    _ck(lib.maf_device_count(C.byref(n)))
    return n.value


class State:
    """State(mesh, Ms, m): Ms is a float or an (nx,ny,nz[,1]) array; m is (nx,ny,nz,3).
    ``precision`` selects the FP64 form (default) or the FP32-field form."""

    def __init__(self, mesh: Mesh, Ms, m, verbose=True, mute_warning=False, precision="fp64"):
        self.mesh = mesh
        self._h = _P()
        mf = _vec_soa(m, mesh)
        prec = _PRECISION[precision]
        if np.ndim(Ms) == 0:
            _ck(lib.maf_state_create(C.byref(self._h), mesh.nx, mesh.ny, mesh.nz, mesh.dx, mesh.dy, mesh.dz,
                                     float(Ms), None, _dptr(mf), prec))
        else:
            msf = _scalar_soa(Ms)
            _ck(lib.maf_state_create(C.byref(self._h), mesh.nx, mesh.ny, mesh.nz, mesh.dx, mesh.dy, mesh.dz,
                                     float("nan"), _dptr(msf), _dptr(mf), prec))

    def __del__(self):
        if getattr(self, "_h", None) and getattr(self, "_owned", True) and lib is not None:
            lib.maf_state_destroy(self._h)
        self._h = None

    @classmethod
    def _borrowed(cls, handle, mesh, owner):
        """A view of a state handle that another object owns (e.g. a string image)."""
        obj = cls.__new__(cls)
        obj.mesh = mesh
        obj._h = handle
        obj._owned = False
        obj._owner = owner  # keeps the owner alive while the view exists
        return obj

    @property
    def precision(self) -> str:
        v = C.c_int()
        _ck(lib.maf_state_precision(self._h, C.byref(v)))
        return "fp32_field" if v.value == MAF_FP32_FIELD else "fp64"

    def __str__(self):
        mx, my, mz = self.mean_m()
        return str(self.t) + " " + str(mx) + " " + str(my) + " " + str(mz)

    @property
    def m(self) -> np.ndarray:
        out = np.empty((self.mesh.nx, self.mesh.ny, self.mesh.nz, 3), order="F")
        _ck(lib.maf_state_get_m(self._h, _dptr(out)))
        return out

    @m.setter
    def m(self, m_in):
        mf = _vec_soa(m_in, self.mesh)
        _ck(lib.maf_state_set_m(self._h, _dptr(mf)))

    def load_m(self, m_in):
        """Set m exactly as given, without normalising (checkpoints, files)."""
        mf = _vec_soa(m_in, self.mesh)
        _ck(lib.maf_state_load_m(self._h, _dptr(mf)))

    @property
    def t(self) -> float:
        v = C.c_double()
        _ck(lib.maf_state_get_t(self._h, C.byref(v)))
        return v.value

    @t.setter
    def t(self, value):
        _ck(lib.maf_state_set_t(self._h, float(value)))

    @property
    def steps(self) -> int:
        v = C.c_ulonglong()
        _ck(lib.maf_state_get_steps(self._h, C.byref(v)))
        return v.value

    @steps.setter
    def steps(self, value: int):
        _ck(lib.maf_state_set_steps(self._h, int(value)))

    def write_vti(self, outputname):
        """State::write_vti: m as a cell-centred VTK image (magnumaf.io.write_vti)."""
        from . import io
        return io.write_vti(self.m, self.mesh.dx, self.mesh.dy, self.mesh.dz, outputname)

    def read_vti(self, inputname):
        """State::_vti_reader: m from a .vti file of the same mesh, as stored."""
        from . import io
        a, _ = io.read_vti(inputname)
        if a.shape[:3] != (self.mesh.nx, self.mesh.ny, self.mesh.nz) or a.shape[3] != 3:
            raise ValueError("read_vti: the file holds a %s field" % (a.shape,))
        self.load_m(a)

    @property
    def Ms(self) -> float:
        v = C.c_double()
        _ck(lib.maf_state_get_Ms(self._h, C.byref(v)))
        return v.value

    @property
    def Ms_field(self) -> Optional[np.ndarray]:
        has = C.c_int()
        _ck(lib.maf_state_get_Ms_field(self._h, None, C.byref(has)))
        if not has.value:
            return None
        out = np.empty((self.mesh.nx, self.mesh.ny, self.mesh.nz), order="F")
        _ck(lib.maf_state_get_Ms_field(self._h, _dptr(out), C.byref(has)))
        return out

    @property
    def precision(self) -> int:
        v = C.c_int()
        _ck(lib.maf_state_precision(self._h, C.byref(v)))
        return v.value

    def mean_m(self, i=None):
        out = np.empty(3)
        _ck(lib.maf_state_mean_m(self._h, _dptr(out)))
        if i is None:
            return float(out[0]), float(out[1]), float(out[2])
        return float(out[i])

    def mean_mx(self):
        return self.mean_m(0)

    def mean_my(self):
        return self.mean_m(1)

    def mean_mz(self):
        return self.mean_m(2)

    def normalize(self):
        self.m = self.m

    def set_stream(self, stream_handle: int):
        _ck(lib.maf_state_set_stream(self._h, C.c_void_p(stream_handle)))

    def device_m(self) -> int:
        p = _P()
        _ck(lib.maf_state_device_m(self._h, C.byref(p)))
        return p.value


class FieldTerm:
    _h = None

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_term_destroy(self._h)
            self._h = None

    def H_in_Apm(self, state: State) -> np.ndarray:
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), order="F")
        _ck(lib.maf_term_H(self._h, state._h, _dptr(out)))
        return out

    def H_in_Apm_f32(self, state: State) -> np.ndarray:
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), dtype=np.float32, order="F")
        _ck(lib.maf_term_H_f32(self._h, state._h, out.ctypes.data_as(_FP)))
        return out

    def H_in_T(self, state: State) -> np.ndarray:
        return self.H_in_Apm(state) * Constants.mu0

    def Energy_in_J(self, state: State) -> float:
        v = C.c_double()
        _ck(lib.maf_term_E(self._h, state._h, C.byref(v)))
        return v.value

    def Energy_in_eV(self, state: State) -> float:
        return self.Energy_in_J(state) / 1.6021766208e-19


_TENSOR_CACHE_MAX = 4 << 30     # bytes kept in the tensor cache before it is shrunk
_TENSOR_CACHE_SHRINK = 2 << 30  # size it is shrunk to (oldest files first)


def tensor_cache_dir() -> str:
    return os.environ.get("MAGNUMAF_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "magnumaf_b200"))


def _tensor_cache_file(mesh: Mesh) -> str:
    return os.path.join(tensor_cache_dir(), "Nred_v1_%d_%d_%d_%r_%r_%r.npy" % (
        mesh.nx, mesh.ny, mesh.nz, float(mesh.dx), float(mesh.dy), float(mesh.dz)))


def _shrink_tensor_cache(verbose=False):
    d = tensor_cache_dir()
    files = [os.path.join(d, f) for f in os.listdir(d) if f.startswith("Nred_") and f.endswith(".npy")]
    files = [f for f in files if os.path.isfile(f)]
    if sum(os.path.getsize(f) for f in files) <= _TENSOR_CACHE_MAX:
        return
    files.sort(key=os.path.getmtime, reverse=True)  # newest first, remove from the back
    while files and sum(os.path.getsize(f) for f in files) > _TENSOR_CACHE_SHRINK:
        old = files.pop()
        if verbose:
            print("removing cached demag tensor", old)
        os.remove(old)


class DemagField(FieldTerm):
    """DemagField(mesh, verbose=False, caching=False, nthreads=4): the tensor is
    assembled on the GPU.  With ``caching`` the reduced spectral tensor is kept on
    disk (``tensor_cache_dir()``, key: mesh sizes and spacings; the cache is shrunk
    oldest-first beyond 4 GiB) and read back on the next construction for the same
    mesh (the reference's get_Nfft caching, demag_field.cpp:185-199).  ``nthreads``
    is accepted for signature compatibility."""

    def __init__(self, mesh: Mesh, verbose=False, caching=False, nthreads=4):
        self.mesh = mesh
        self._h = _P()
        if caching:
            path = _tensor_cache_file(mesh)
            shape = self._tensor_shape()
            if os.path.exists(path):
                try:
                    N = np.load(path)
                    if N.shape != shape or N.dtype != np.float64:
                        raise ValueError("cached tensor has the wrong shape")
                    _ck(lib.maf_term_demag_create_from_tensor(C.byref(self._h), mesh.nx, mesh.ny, mesh.nz, mesh.dx,
                                                              mesh.dy, mesh.dz, _dptr(np.ascontiguousarray(N))))
                    if verbose:
                        print("read demag tensor from", path)
                    return
                except (OSError, ValueError) as e:
                    if verbose:
                        print("ignoring cached demag tensor (%s), computing it" % e)
                    self._h = _P()
        _ck(lib.maf_term_demag_create(C.byref(self._h), mesh.nx, mesh.ny, mesh.nz, mesh.dx, mesh.dy, mesh.dz))
        if caching:
            os.makedirs(tensor_cache_dir(), exist_ok=True)
            tmp = path + ".%d.tmp" % os.getpid()
            with open(tmp, "wb") as f:
                np.save(f, self.spectral_tensor())
            os.replace(tmp, path)
            if verbose:
                print("saved demag tensor to", path)
            _shrink_tensor_cache(verbose)

    def _tensor_shape(self):
        m = self.mesh
        return (4 if m.nz == 1 else 6, 1 if m.nz == 1 else m.nz + 1, m.ny + 1, m.nx + 1)

    def spectral_tensor(self) -> np.ndarray:
        """Reduced real spectral tensor [ncomp][kz][ky][kx] (C order)."""
        m = self.mesh
        ncomp = 4 if m.nz == 1 else 6
        kz = 1 if m.nz == 1 else m.nz + 1
        out = np.empty((ncomp, kz, m.ny + 1, m.nx + 1))
        _ck(lib.maf_term_demag_tensor(self._h, _dptr(out)))
        return out

    @property
    def tune(self):
        """Kernel variants of this mesh's passes: (cols_wide, convz_reg, xinv_run), see LLGIntegrator.autotune."""
        ch = (_I * 3)()
        _ck(lib.maf_term_demag_get_tune(self._h, ch))
        return tuple(ch)

    @tune.setter
    def tune(self, choices):
        ch = (_I * 3)(*[int(c) for c in choices])
        _ck(lib.maf_term_demag_set_tune(self._h, ch))

    @property
    def generic(self) -> bool:
        return bool(getattr(self, "_generic", False))

    @generic.setter
    def generic(self, on):
        """Run every pass with the run-time-plan kernels (those of the batched passes)."""
        _ck(lib.maf_term_demag_set_generic(self._h, int(bool(on))))
        self._generic = bool(on)

    @property
    def tune_ex(self):
        """All kernel choices: (cols_wide, convz_reg, xinv_run, cols_pipe, cols_plan); cols_plan 0: both
        y passes radix 16 16 R, 1: both 16 R 16, 2: the inverse only, 3: the forward only."""
        ch = (_I * 5)()
        _ck(lib.maf_term_demag_get_tune_ex(self._h, ch))
        return tuple(ch)

    @tune_ex.setter
    def tune_ex(self, choices):
        ch = (_I * 5)(*[int(c) for c in choices])
        _ck(lib.maf_term_demag_set_tune_ex(self._h, ch))

    def get_N(self, symmetric=False) -> np.ndarray:
        """Real-space Newell tensor [Px, Py, Pz, 6] (the reference's setup_N layout);
        symmetric=True returns the parity-exact tensor the spectral pipeline uses."""
        m = self.mesh
        Px, Py, Pz = 2 * m.nx, 2 * m.ny, (1 if m.nz == 1 else 2 * m.nz)
        out = np.empty((6, Pz, Py, Px))
        _ck(lib.maf_term_demag_real_tensor(self._h, _dptr(out), int(bool(symmetric))))
        return out.transpose(3, 2, 1, 0)


class DemagFieldPBC(FieldTerm):
    """DemagFieldPBC() (python/magnumaf.pyx:1123-1140, demag_field_pbc.cpp):
    periodic demag through the scalar potential; the mesh is the evaluated
    state's (nx must be even)."""

    def __init__(self):
        self._h = _P()
        _ck(lib.maf_term_demag_pbc_create(C.byref(self._h)))


def _sparse_exchange(term, A, mesh, create, who):
    if mesh is None:
        raise MafError(1, who + ": a mesh is required")
    term._h = _P()
    if np.ndim(A) == 0:
        term.A = float(A)
        _ck(create(C.byref(term._h), mesh.nx, mesh.ny, mesh.nz, None, term.A))
    else:
        a = _scalar_soa(A)
        if a.shape != (mesh.nx, mesh.ny, mesh.nz):
            raise MafError(1, "%s: A field of shape %s on a %dx%dx%d mesh"
                           % (who, a.shape, mesh.nx, mesh.ny, mesh.nz))
        term.A = None
        _ck(create(C.byref(term._h), mesh.nx, mesh.ny, mesh.nz, _dptr(a), 0.0))


class ExchangeField(FieldTerm):
    """ExchangeField(A) is the zero-padded Laplacian (exchange_field.cpp); with a
    mesh, ExchangeField(A, mesh) and ExchangeField(A_field, mesh) are the sparse
    matrix form of SparseExchangeField (python/magnumaf.pyx:1172-1195)."""

    def __init__(self, A, mesh: Mesh = None, verbose=False):
        if mesh is not None:
            _sparse_exchange(self, A, mesh, lib.maf_term_sparse_exchange_create, "ExchangeField")
            return
        if np.ndim(A) != 0:
            raise MafError(1, "When passing A as an array, you must provide a mesh, "
                                           "i.e. ExchangeField(A, mesh).")
        self.A = float(A)
        self._h = _P()
        _ck(lib.maf_term_exchange_create(C.byref(self._h), self.A))


class SparseExchangeField(FieldTerm):
    """SparseExchangeField(A, mesh) with a scalar or cell-wise A
    (sparse_exchange_field.cpp:8-18,25-330)."""

    def __init__(self, A, mesh: Mesh, verbose=False):
        _sparse_exchange(self, A, mesh, lib.maf_term_sparse_exchange_create, "SparseExchangeField")


class ExchangeFieldPBC(FieldTerm):
    """ExchangeFieldPBC(A, mesh): exchange with periodic boundaries in x, y and z
    (exchange_field_pbc.cpp:9-225)."""

    def __init__(self, A, mesh: Mesh, verbose=False):
        _sparse_exchange(self, A, mesh, lib.maf_term_exchange_pbc_create, "ExchangeFieldPBC")


class DmiField(FieldTerm):
    def __init__(self, D, D_axis=(0.0, 0.0, 1.0)):
        self._h = _P()
        ax = [float(v) for v in D_axis]
        if np.ndim(D) == 0:
            self.D = float(D)
            _ck(lib.maf_term_dmi_create(C.byref(self._h), self.D, *ax))
        else:
            d = _scalar_soa(D)
            nx, ny, nz = d.shape
            _ck(lib.maf_term_dmi_field_create(C.byref(self._h), nx, ny, nz, _dptr(d), *ax))


class BulkDMIExchangeField(FieldTerm):
    def __init__(self, D, A):
        self._h = _P()
        _ck(lib.maf_term_bulkdmi_exchange_create(C.byref(self._h), float(D), float(A)))


class UniaxialAnisotropyField(FieldTerm):
    def __init__(self, Ku1, Ku1_axis=(0.0, 0.0, 1.0)):
        self._h = _P()
        scalar_axis = np.ndim(Ku1_axis) == 1
        if np.ndim(Ku1) == 0 and scalar_axis:
            self.Ku1 = float(Ku1)
            ax = np.asarray(Ku1_axis, dtype=np.float64)
            self.Ku1_axis = list(ax / math.sqrt(float(np.sum(ax * ax))))
            _ck(lib.maf_term_uniaxial_create(C.byref(self._h), self.Ku1, *[float(v) for v in Ku1_axis]))
            return
        kf = None if np.ndim(Ku1) == 0 else _scalar_soa(Ku1)
        af = None if scalar_axis else _vec_soa(Ku1_axis)
        shape = (kf if kf is not None else af).shape[:3]
        ax = [0.0, 0.0, 1.0] if not scalar_axis else [float(v) for v in Ku1_axis]
        self.Ku1 = Ku1
        _ck(lib.maf_term_uniaxial_field_create(C.byref(self._h), shape[0], shape[1], shape[2],
                                               None if kf is None else _dptr(kf),
                                               float(Ku1) if kf is None else 0.0,
                                               None if af is None else _dptr(af), *ax))


class CubicAnisotropyField(FieldTerm):
    def __init__(self, Kc1, Kc2=0.0, Kc3=0.0, c1=(1.0, 0.0, 0.0), c2=(0.0, 1.0, 0.0)):
        self._h = _P()
        a = np.asarray(c1, dtype=np.float64)
        b = np.asarray(c2, dtype=np.float64)
        _ck(lib.maf_term_cubic_create(C.byref(self._h), float(Kc1), float(Kc2), float(Kc3), _dptr(a), _dptr(b)))


class SpinTransferTorqueField(FieldTerm):
    """SpinTransferTorqueField(pol, eta_damp, eta_field, j_e, fl_thickness) (python/magnumaf.pyx:1690-1730):
    pol is a (nx, ny, nz, 3) polarisation field (normalised on construction)."""

    def __init__(self, pol, eta_damp: float, eta_field: float, j_e: float, fl_thickness: float):
        pf = _vec_soa(pol)
        nx, ny, nz = pf.shape[:3]
        self.eta_damping, self.eta_field, self.j_e, self.fl_thickness = (float(eta_damp), float(eta_field),
                                                                          float(j_e), float(fl_thickness))
        self._h = _P()
        _ck(lib.maf_term_stt_create(C.byref(self._h), nx, ny, nz, _dptr(pf), self.eta_damping, self.eta_field,
                                    self.j_e, self.fl_thickness))


class ExternalField(FieldTerm):
    def __init__(self, array_in):
        self._h = _P()
        h = _vec_soa(array_in)
        self.shape = h.shape
        nx, ny, nz, _ = h.shape
        _ck(lib.maf_term_external_create(C.byref(self._h), nx, ny, nz, _dptr(h)))

    @staticmethod
    def uniform(hx, hy, hz):
        t = ExternalField.__new__(ExternalField)
        t._h = _P()
        _ck(lib.maf_term_external_uniform_create(C.byref(t._h), float(hx), float(hy), float(hz)))
        return t

    def set_homogeneous_field(self, x, y, z):
        nx, ny, nz, _ = self.shape
        h = np.empty((nx, ny, nz, 3), order="F")
        h[..., 0], h[..., 1], h[..., 2] = x, y, z
        old = self._h
        self._h = _P()
        _ck(lib.maf_term_external_create(C.byref(self._h), nx, ny, nz, _dptr(h)))
        lib.maf_term_destroy(old)


class LLGIntegrator:
    """LLGIntegrator(alpha, terms, mode="RKF45", hmin=1e-15, hmax=3.5e-10,
    atol=1e-6, rtol=1e-6, dissipation_term_only=False)"""

    def __init__(self, alpha, terms: Sequence[FieldTerm], mode="RKF45", hmin=1e-15, hmax=3.5e-10, atol=1e-6,
                 rtol=1e-6, dissipation_term_only=False):
        self._h = _P()
        self._terms = list(terms)  # keep the Python objects alive
        arr = (_P * max(1, len(self._terms)))(*[t._h for t in self._terms])
        if np.ndim(alpha) == 0:
            self._alpha = float(alpha)
            _ck(lib.maf_llg_create(C.byref(self._h), self._alpha, None, 0, 0, 0, arr, len(self._terms),
                                   mode.encode(), hmin, hmax, atol, rtol, int(bool(dissipation_term_only))))
        else:
            af = _scalar_soa(alpha)
            self._alpha = af
            nx, ny, nz = af.shape
            _ck(lib.maf_llg_create(C.byref(self._h), 0.0, _dptr(af), nx, ny, nz, arr, len(self._terms),
                                   mode.encode(), hmin, hmax, atol, rtol, int(bool(dissipation_term_only))))

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_llg_destroy(self._h)
            self._h = None

    def step(self, state: State):
        _ck(lib.maf_llg_step(self._h, state._h))

    def steps(self, state: State, n: int):
        _ck(lib.maf_llg_steps(self._h, state._h, int(n)))

    def Eeff_in_J(self, state: State) -> float:
        v = C.c_double()
        _ck(lib.maf_llg_E(self._h, state._h, C.byref(v)))
        return v.value

    E = Eeff_in_J

    def H_in_Apm(self, state: State) -> np.ndarray:
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), order="F")
        _ck(lib.maf_llg_heff(self._h, state._h, _dptr(out)))
        return out

    def H_in_Apm_f32(self, state: State) -> np.ndarray:
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), dtype=np.float32, order="F")
        _ck(lib.maf_llg_heff_f32(self._h, state._h, out.ctypes.data_as(_FP)))
        return out

    def dmdt(self, state: State) -> np.ndarray:
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), order="F")
        _ck(lib.maf_llg_dmdt(self._h, state._h, _dptr(out)))
        return out

    def rk_attempt(self, state: State, scheme: str, dt: float):
        """One attempt of `scheme` with step dt, no controller: returns (m + sumbk, err)."""
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), order="F")
        err = C.c_double()
        _ck(lib.maf_llg_rk_attempt(self._h, state._h, scheme.encode(), float(dt), _dptr(out), C.byref(err)))
        return out, err.value

    def add_terms(self, *args):
        for t in args:
            _ck(lib.maf_llg_add_term(self._h, t._h))
            self._terms.append(t)

    def relax(self, state: State, precision=1e-10, ncalcE=100, nprint=1000, verbose=True):
        _ck(lib.maf_llg_relax(self._h, state._h, float(precision), int(ncalcE)))

    def integrate_dense(self, state: State, time_in_s, write_every_dt_in_s, filename=None, verbose=False,
                        append=False) -> np.ndarray:
        """Returns the rows (t, <mx>, <my>, <mz>) and, like the reference, writes
        them to `filename` when one is given."""
        max_rows = int(math.ceil(time_in_s / write_every_dt_in_s)) + 4
        rows = np.zeros((max_rows, 4))
        n = C.c_int()
        _ck(lib.maf_llg_integrate_dense(self._h, state._h, float(time_in_s), float(write_every_dt_in_s),
                                        _dptr(rows), max_rows, C.byref(n)))
        rows = rows[: n.value]
        if filename:
            with open(filename, "a" if append else "w") as f:
                for r in rows:
                    f.write("%r\t%r\t%r\t%r\n" % tuple(r))
        return rows

    @property
    def alpha(self):
        return self._alpha

    @alpha.setter
    def alpha(self, value):
        self._alpha = float(value)
        _ck(lib.maf_llg_set_alpha(self._h, self._alpha))

    @property
    def h(self) -> float:
        v = C.c_double()
        _ck(lib.maf_llg_get_h(self._h, C.byref(v)))
        return v.value

    def counters(self):
        out = (C.c_ulonglong * 4)()
        _ck(lib.maf_llg_counters(self._h, out))
        return {"accepted": out[0], "rejected": out[1], "hmin": out[2], "hmax": out[3]}

    def controller_state(self):
        """[h, errold, reject, hnext, accepted, rejected, hmin, hmax, accumulated_steps] (for checkpoints)."""
        out = np.zeros(9)
        _ck(lib.maf_llg_get_controller_state(self._h, _dptr(out)))
        return out.tolist()

    def set_controller_state(self, values):
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.size != 9:
            raise ValueError("9 values expected")
        _ck(lib.maf_llg_set_controller_state(self._h, _dptr(v)))

    def heff_device(self, state: State, m_dev_ptr: int, H_dev_ptr: int):
        """Field of a device-resident m into a device-resident H (no sync)."""
        _ck(lib.maf_llg_heff_device(self._h, state._h, C.c_void_p(m_dev_ptr), C.c_void_p(H_dev_ptr)))

    def autotune_ex(self, state: State, reps: int = 3) -> dict:
        """The full autotuner search (maf_llg_autotune_ex): four timed configurations,
        the y passes' tile, pipelining and radix sequence chosen jointly; cached per
        mesh, precision and term kinds within the process."""
        ch = (_I * 5)()
        ms = np.zeros(20)
        cached = _I()
        _ck(lib.maf_llg_autotune_ex(self._h, state._h, int(reps), ch, _dptr(ms), C.byref(cached)))
        names = ("cols_wide", "convz_reg", "xinv_run", "cols_pipe", "cols_plan")
        out = {k: ch[i] for i, k in enumerate(names)}
        out["cached"] = bool(cached.value)
        out["pass_ms"] = [ms[5 * c:5 * c + 5].tolist() for c in range(4)]
        return out

    def autotune(self, state: State, reps: int = 3) -> dict:
        """Pick the faster kernel variant per demag pass on this state's mesh
        (see maf_llg_autotune); returns the choices and both configurations'
        per-pass times in ms."""
        ch = (_I * 3)()
        ms = np.zeros(10)
        _ck(lib.maf_llg_autotune(self._h, state._h, int(reps), ch, _dptr(ms)))
        return {"cols_wide": ch[0], "convz_reg": ch[1], "xinv_run": ch[2], "pass_ms_default": ms[:5].tolist(),
                "pass_ms_alternative": ms[5:].tolist()}

    def heff_pipeline(self, state: State, m_host_ptrs, H_host_ptrs, m_float32: bool = False):
        """Fields of several host magnetisations in a row, host copies overlapped
        with the evaluations (pass pinned buffers): m_host_ptrs[i] -> H_host_ptrs[i]
        (addresses of double [3][N] inputs -- float [3][N] with m_float32 -- and of
        float/double [3][N] outputs)."""
        n = len(m_host_ptrs)
        if len(H_host_ptrs) != n:
            raise ValueError("as many outputs as inputs")
        mp = (_P * max(n, 1))(*[C.c_void_p(p) for p in m_host_ptrs])
        hp = (_P * max(n, 1))(*[C.c_void_p(p) for p in H_host_ptrs])
        fn = lib.maf_llg_heff_pipeline_m32 if m_float32 else lib.maf_llg_heff_pipeline
        _ck(fn(self._h, state._h, mp, hp, n))

    def heff_device_profile(self, state: State, m_dev_ptr: int, H_dev_ptr: int):
        """One field evaluation with per-pass CUDA-event timing: [(name, ms), ...]."""
        ms = np.zeros(16)
        n = C.c_int()
        _ck(lib.maf_llg_heff_device_profile(self._h, state._h, C.c_void_p(m_dev_ptr), C.c_void_p(H_dev_ptr),
                                            _dptr(ms), 16, C.byref(n)))
        out = []
        buf = C.create_string_buffer(64)
        for i in range(n.value):
            _ck(lib.maf_llg_pass_name(self._h, state._h, i, buf, 64))
            out.append((buf.value.decode(), float(ms[i])))
        return out


    def attempt_profile(self, state: State, dt: float):
        """One Runge-Kutta attempt of this integrator's scheme with step dt (the state
        is not changed), with CUDA events between its kernels: [(name, ms), ...]."""
        cap = 256
        ms = np.zeros(cap)
        n = C.c_int()
        _ck(lib.maf_llg_attempt_profile(self._h, state._h, float(dt), _dptr(ms), cap, C.byref(n)))
        out = []
        buf = C.create_string_buffer(64)
        for i in range(n.value):
            _ck(lib.maf_llg_profile_name(self._h, i, buf, 64))
            out.append((buf.value.decode(), float(ms[i])))
        return out


class LBFGS_Minimizer:
    """LBFGS_Minimizer(terms=[], tol=1e-6, maxiter=230, verbose=0) (python/magnumaf.pyx:1786-1835)."""

    def __init__(self, terms: Sequence[FieldTerm] = (), tol=1e-6, maxiter=230, verbose=0):
        self._h = _P()
        self._terms = list(terms)
        arr = (_P * max(1, len(self._terms)))(*[t._h for t in self._terms])
        _ck(lib.maf_lbfgs_create(C.byref(self._h), arr, len(self._terms), float(tol), int(maxiter)))

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_lbfgs_destroy(self._h)
            self._h = None

    def add_terms(self, *args):
        for t in args:
            _ck(lib.maf_lbfgs_add_term(self._h, t._h))
            self._terms.append(t)

    def minimize(self, state: State) -> float:
        v = C.c_double()
        _ck(lib.maf_lbfgs_minimize(self._h, state._h, C.byref(v)))
        return v.value

    def stats(self):
        it, fe = C.c_ulonglong(), C.c_ulonglong()
        g = C.c_double()
        _ck(lib.maf_lbfgs_stats(self._h, C.byref(it), C.byref(fe), C.byref(g)))
        return {"iterations": it.value, "fevals": fe.value, "grad_max": g.value}


class ConvNet:
    """The learned warm-start network (maf_cnn_*): 3x3 convolutions with ReLU,
    output normalize(m + conv_L(...)), trained with the library's own kernels.
    Array arguments are device pointers (e.g. torch CUDA tensors' data_ptr()),
    NCHW float32: x [B][cin][H][W] with m in channels 0..2, y and targets [B][3][H][W]."""

    def __init__(self, cin: int, width: int = 16, depth: int = 4, seed: int = 0, dilation=None):
        self.cin, self.width, self.depth = int(cin), int(width), int(depth)
        self._h = _P()
        _ck(lib.maf_cnn_create(C.byref(self._h), self.cin, self.width, self.depth, int(seed)))
        self.dilation = [1] * self.depth
        if dilation is not None:
            d = [int(v) for v in dilation]
            _ck(lib.maf_cnn_set_dilation(self._h, (_I * len(d))(*d), len(d)))
            self.dilation = d

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_cnn_destroy(self._h)
            self._h = None

    @property
    def n_params(self) -> int:
        n = C.c_longlong()
        _ck(lib.maf_cnn_n_params(self._h, C.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        out = np.empty(self.n_params, dtype=np.float32)
        _ck(lib.maf_cnn_get_params(self._h, out.ctypes.data_as(_FP)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError("expected %d parameters" % self.n_params)
        _ck(lib.maf_cnn_set_params(self._h, p.ctypes.data_as(_FP)))

    def forward(self, x_ptr: int, B: int, H: int, W: int, y_ptr: int):
        _ck(lib.maf_cnn_forward(self._h, C.c_void_p(x_ptr), B, H, W, C.c_void_p(y_ptr)))

    def loss_grad(self, x_ptr: int, t_ptr: int, B: int, H: int, W: int, want_grad: bool = True):
        loss = C.c_float()
        g = np.empty(self.n_params, dtype=np.float32) if want_grad else None
        _ck(lib.maf_cnn_loss_grad(self._h, C.c_void_p(x_ptr), C.c_void_p(t_ptr), B, H, W, C.byref(loss),
                                  g.ctypes.data_as(_FP) if want_grad else None))
        return loss.value, g

    def train_step(self, x_ptr: int, t_ptr: int, B: int, H: int, W: int, lr: float) -> float:
        loss = C.c_float()
        _ck(lib.maf_cnn_train_step(self._h, C.c_void_p(x_ptr), C.c_void_p(t_ptr), B, H, W, float(lr),
                                   C.byref(loss)))
        return loss.value


class StochasticBatch:
    """Members (Stochastic_LLG, State) advanced together: after one eager step,
    pairs of steps of every member replay one captured CUDA graph with each member
    on its own stream.  Bit-identical to stepping the members one by one.

    fused=True: every pass of a step is one launch for all members (a device
    work table of (member, tile) pairs over the run-time-plan kernels) when every
    member is a 2-D mesh with one DemagField and scalar parameters; bit-identical
    to the members stepped one by one with DemagField.generic = True."""

    def __init__(self, members, fused=False):
        self._members = list(members)
        its = (_P * len(self._members))(*[it._h for it, _ in self._members])
        sts = (_P * len(self._members))(*[st._h for _, st in self._members])
        self._h = _P()
        _ck(lib.maf_stoch_batch_create(C.byref(self._h), its, sts, len(self._members)))
        if fused:
            _ck(lib.maf_stoch_batch_set_fused(self._h, 1))

    @property
    def fused_active(self) -> bool:
        """Whether the captured graph runs the batched passes."""
        v = _I()
        _ck(lib.maf_stoch_batch_is_fused(self._h, C.byref(v)))
        return bool(v.value)

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_stoch_batch_destroy(self._h)
            self._h = None

    def steps(self, n: int):
        _ck(lib.maf_stoch_batch_steps(self._h, int(n)))


class StringMethod:
    """StringMethod(state, inputimages, n_interp, dt, llg) (python/magnumaf.pyx:1034-1068).

    ``inputimages`` are States or m arrays (nx, ny, nz, 3); arrays become states
    with the template state's Ms (or Ms_field).  ``run`` returns the lowest
    energy barrier max(E) - E[0] in J and writes the reference's .dat files
    under ``filepath``.  The images stay on the device; ``images`` gives views."""

    def __init__(self, state: State, inputimages, n_interp, dt, llg: LLGIntegrator):
        if not inputimages or len(inputimages) == 1:
            raise RuntimeError("StringMethod: invalid inputimages provided, please add at least two "
                               "states/magnetizations for interpolation of initial path.")
        self._h = _P()
        self._llg = llg
        self.mesh = state.mesh
        ms_field = state.Ms_field
        ms = ms_field if ms_field is not None else state.Ms
        self._inputs = [a if isinstance(a, State) else State(state.mesh, ms, a, precision=state.precision)
                        for a in inputimages]
        arr = (_P * len(self._inputs))(*[a._h for a in self._inputs])
        _ck(lib.maf_string_create(C.byref(self._h), state._h, arr, len(self._inputs), int(n_interp), float(dt),
                                  llg._h))
        self.n_interp = int(n_interp)

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_string_destroy(self._h)
            self._h = None

    def run(self, filepath, string_abort_rel_diff=1e-12, string_abort_abs_diff=1e-27, string_steps=10000,
            every_string_to_vti=50, verbose=True):
        dE = C.c_double()
        it = C.c_int()
        _ck(lib.maf_string_run(self._h, str(filepath).encode(), float(string_abort_rel_diff),
                               float(string_abort_abs_diff), int(string_steps), int(every_string_to_vti),
                               int(bool(verbose)), C.byref(dE), C.byref(it)))
        self.iterations = it.value
        return dE.value

    def step(self):
        _ck(lib.maf_string_step(self._h))

    def set_batched(self, substeps: int):
        """Advance all images together in one CUDA graph: each image integrates its
        dt with `substeps` fixed RK4 steps (its own demag buffers and stream).
        Not the reference's integration (one adaptive integrator stepping the images
        one after the other); substeps=0 returns to it."""
        _ck(lib.maf_string_set_batched(self._h, int(substeps)))

    def calc_E(self) -> np.ndarray:
        out = np.empty(self.n_interp)
        _ck(lib.maf_string_calc_E(self._h, _dptr(out)))
        return out

    def x(self):
        x = np.empty(self.n_interp)
        xi = np.empty(self.n_interp)
        _ck(lib.maf_string_get_x(self._h, _dptr(x), _dptr(xi)))
        return x, xi

    @property
    def images(self):
        out = []
        for i in range(self.n_interp):
            h = _P()
            _ck(lib.maf_string_image(self._h, i, C.byref(h)))
            out.append(State._borrowed(h, self.mesh, self))
        return out


class Stochastic_LLG:
    """Stochastic_LLG(alpha, T, dt, state, terms=[], smode="Heun") (python/magnumaf.pyx:881-910):
    fixed-step Heun / SemiHeun / detRK4 at temperature T [K] with time step dt [s].
    ``seed`` and ``member`` select the counter-based random stream (the reference
    seeds from the wall clock)."""

    def __init__(self, alpha, T, dt, state: State, terms: Sequence[FieldTerm] = (), smode="Heun", seed=0,
                 member=0):
        self._h = _P()
        self._terms = list(terms)
        arr = (_P * max(1, len(self._terms)))(*[t._h for t in self._terms])
        self.alpha, self.T, self.dt = float(alpha), float(T), float(dt)
        _ck(lib.maf_stochastic_llg_create(C.byref(self._h), self.alpha, self.T, self.dt, arr, len(self._terms),
                                          str(smode).encode(), int(seed), int(member)))

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:
            lib.maf_stochastic_llg_destroy(self._h)
            self._h = None

    def step(self, state: State):
        _ck(lib.maf_stochastic_llg_step(self._h, state._h))

    def steps(self, state: State, n: int):
        _ck(lib.maf_stochastic_llg_steps(self._h, state._h, int(n)))

    def Eeff_in_J(self, state: State) -> float:
        v = C.c_double()
        _ck(lib.maf_stochastic_llg_E(self._h, state._h, C.byref(v)))
        return v.value

    def thermal_field(self, state: State, index: int) -> np.ndarray:
        """The thermal field h_th of noise index `index`, (nx, ny, nz, 3)."""
        out = np.empty((state.mesh.nx, state.mesh.ny, state.mesh.nz, 3), order="F")
        _ck(lib.maf_stochastic_llg_noise(self._h, state._h, int(index), _dptr(out)))
        return out

    @property
    def calls(self) -> int:
        v = C.c_ulonglong()
        _ck(lib.maf_stochastic_llg_calls(self._h, C.byref(v)))
        return v.value
