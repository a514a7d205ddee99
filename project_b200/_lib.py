"""ctypes binding of libuppe_b200.so (the C ABI declared in include/uppe_b200.h).

There is no CPU fallback: if the library is missing or no CUDA device is
visible, loading raises.
"""
import ctypes
import os

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, 'libuppe_b200.so')
_lib = None

UPPE_C64, UPPE_C128 = 0, 1
STATUS_NONFINITE, STATUS_MIN_STEP, STATUS_MAX_ATTEMPTS, STATUS_RETRIED = 1, 2, 4, 64
# line limits of uppe1d_propagate_noalloc (its static device array)
UPPE_NOALLOC_MAX_NT_C64, UPPE_NOALLOC_MAX_NT_C128 = 16384, 8192
# timing slots of uppe3d_tuning: eleven y-pass candidates, then two t-pass ones
UPPE3D_TUNE_SLOTS = 13

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_LL = ctypes.c_longlong


class Desc3D(ctypes.Structure):
    _fields_ = [('Nx', _I), ('Ny', _I), ('Nt', _I), ('precision', _I), ('dt', _D),
                ('aw', _P), ('ksq', _P), ('kref', _P), ('valid', _P), ('shock', _P),
                ('filt', _P), ('kperp2', _P), ('damp', _P), ('lut_n', _I),
                ('lut_log10I', _P), ('lut_W', _P), ('gamma_kerr', _D), ('gamma_hoke', _D),
                ('Ui', _D), ('sigma_drude', _D), ('omega0_tau_c', _D), ('rate_rec', _D),
                ('rho_nt', _D), ('ava_coef', _D), ('plasma_on', _I), ('omega_abs', _P)]


class Result3D(ctypes.Structure):
    _fields_ = [('z', _D), ('h', _D), ('err', _D), ('attempts', _LL), ('accepted', _LL),
                ('fail_count', _I), ('status', _I), ('A_scale', _D)]


class State3D(ctypes.Structure):
    """uppe3d_state: the adaptive loop's state between two attempts."""
    _fields_ = [('z', _D), ('h', _D), ('L', _D), ('tol', _D), ('max_step', _D), ('min_step', _D),
                ('err', _D), ('A_scale', _D), ('peak_ion', _D), ('attempts', _LL), ('accepted', _LL),
                ('max_attempts', _LL), ('fail_count', _I), ('status', _I), ('done', _I)]


class InstDesc1D(ctypes.Structure):
    _fields_ = [('Nt', _I), ('dt', _D), ('L', _D), ('tol', _D), ('max_step', _D),
                ('min_step', _D), ('max_attempts', _LL), ('raman', _I), ('plasma', _I),
                ('f_R', _D), ('A_eff', _D), ('Ui', _D), ('sigma_drude', _D),
                ('omega0_tau_c', _D), ('rate_rec', _D), ('rho_nt', _D), ('ava_coef', _D),
                ('hist_cap', _I), ('omega0', _D), ('cost', _D)]


class Desc1D(ctypes.Structure):
    _fields_ = [('n_inst', _I), ('precision', _I), ('inst', ctypes.POINTER(InstDesc1D)),
                ('D', _P), ('G', _P), ('H', _P), ('lut_n', _I), ('lut_log10I', _P), ('lut_W', _P)]


class Result1D(ctypes.Structure):
    _fields_ = [('z', _D), ('h', _D), ('err', _D), ('attempts', _LL), ('accepted', _LL),
                ('status', _I), ('hist_count', _I), ('energy', _D), ('photons', _D), ('peak_ion', _D)]


STATUS_HIST_FULL = 8


class DescRF(ctypes.Structure):
    _fields_ = [('Nx', _I), ('Ny', _I), ('Nt', _I), ('precision', _I), ('dt', _D),
                ('kk', _P), ('kref', _P), ('w', _P), ('filt', _P), ('kperp2', _P), ('damp', _P),
                ('lut_n', _I), ('lut_log10I', _P), ('lut_W', _P), ('I_coef', _D), ('aval_coef', _D),
                ('chi3e', _D), ('chi5e', _D), ('rate_rec', _D), ('rho_nt', _D), ('Ui', _D),
                ('e_charge', _D), ('m_e', _D), ('tau_c', _D), ('raman_H', _P), ('raman_fR', _D)]


class Op1D(ctypes.Structure):
    _fields_ = [('inst', _I), ('record', _I), ('amp', _D), ('gdd', _D), ('tod', _D)]

# name -> (restype, argtypes)
SIGNATURES = {
    'uppe_last_error': (ctypes.c_char_p, []),
    'uppe3d_plan_create': (_I, [ctypes.POINTER(Desc3D), ctypes.POINTER(_P)]),
    'uppe3d_plan_destroy': (_I, [_P]),
    'uppe3d_field_bytes': (_LL, [_P]),
    'uppe3d_set_field': (_I, [_P, _P, _P]),
    'uppe3d_attempt': (_I, [_P, _D, ctypes.POINTER(_D), _P]),
    'uppe3d_commit': (_I, [_P, _I, _P]),
    'uppe3d_propagate': (_I, [_P, _D, _D, _D, _D, _LL, ctypes.POINTER(Result3D), _P]),
    'uppe3d_begin': (_I, [_P, _D, _D, _D, _D, _LL, _P]),
    'uppe3d_run_steps': (_I, [_P, _I, _P]),
    'uppe3d_get_result': (_I, [_P, ctypes.POINTER(Result3D), _P]),
    'uppe3d_save_state': (_I, [_P, _P, ctypes.POINTER(State3D), _P]),
    'uppe3d_load_state': (_I, [_P, _P, ctypes.POINTER(State3D), _P]),
    'uppe3d_resume': (_I, [_P, ctypes.POINTER(Result3D), _P]),
    'uppe3d_get_spectrum': (_I, [_P, _P, _P]),
    'uppe3d_get_field': (_I, [_P, _P, _P]),
    'uppe3d_launches_per_step': (_I, [_P]),
    'uppe3d_diagnostics': (_I, [_P, _D, _D, ctypes.POINTER(_D), _P]),
    'uppe3d_set_step_log': (_I, [_P, _P, _LL, _P]),
    'uppe3d_adjoint_work_bytes': (_LL, [_P, _I, _I]),
    'uppe3d_adjoint': (_I, [_P, _P, _I, _I, _P, _P, _P, _P, _P]),
    'uppe1d_plan_create': (_I, [ctypes.POINTER(Desc1D), ctypes.POINTER(_P)]),
    'uppe1d_plan_destroy': (_I, [_P]),
    'uppe1d_field_elems': (_LL, [_P]),
    'uppe1d_hist_elems': (_LL, [_P]),
    'uppe1d_hist_slots': (_LL, [_P]),
    'uppe1d_propagate': (_I, [_P, _P, _P, _P, ctypes.POINTER(Result1D), _P]),
    'uppe1d_propagate_logged': (_I, [_P, _P, _P, _I, ctypes.POINTER(Result1D), _P]),
    'uppe1d_propagate_schedule': (_I, [_P, _P, _P, _I, ctypes.POINTER(Result1D), _P]),
    'uppe3d_mirror': (_I, [_P, _P, _D, _D, _D, _D, _P]),
    'uppe_rf_plan_create': (_I, [ctypes.POINTER(DescRF), ctypes.POINTER(_P)]),
    'uppe_rf_plan_destroy': (_I, [_P]),
    'uppe_rf_set_field': (_I, [_P, _P, ctypes.POINTER(_D), _P]),
    'uppe_rf_attempt': (_I, [_P, _D, ctypes.POINTER(_D), _P]),
    'uppe_rf_commit': (_I, [_P, _I, _P]),
    'uppe_rf_get_field': (_I, [_P, _P, _P]),
    'uppe_rf_get_spectrum': (_I, [_P, _P, _P]),
    'uppe_rf_spec_bins': (_I, [_P]),
    'uppe_spectrum_field': (_I, [_P, _P, _I, _I, _D, _D, _D, _D, _P, _P]),
    'uppe3d_beam_diag_elems': (_LL, [_P]),
    'uppe3d_beam_diagnostics': (_I, [_P, _P, _P, _P]),
    'uppe1d_run_programs': (_I, [_P, _I, ctypes.POINTER(_LL), ctypes.POINTER(Op1D), _P, _P,
                                 ctypes.POINTER(Result1D), _P]),
    'uppe1d_adjoint_work_elems': (_LL, [_I, _I, _I]),
    'uppe1d_adjoint': (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    'uppe1d_propagate_noalloc': (_I, [ctypes.POINTER(InstDesc1D), _I, _P, _P, _P, _I, _P, _P, _P,
                                      ctypes.POINTER(Result1D), _P]),
    'uppe1d_last_activity': (_I, [_P, ctypes.POINTER(_D), ctypes.POINTER(_D), _P]),
    'uppe1d_uses_clusters': (_I, [_P]),
    'uppe_fft_c128': (_I, [_P, _P, _P, _I, _I, _D, _I, _I, _P]),
    'uppe_spectral_phase': (_I, [_P, _I, _D, _D, _D, _P]),
    'uppe_exact_ft': (_I, [_P, _I, _P, _P, _I, _P, _P]),
    'uppe3d_transform_t': (_I, [_P, _P, _P, _I, _D, _P]),
    'uppe3d_tuning': (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_float)]),
    'uppe3d_set_tuning': (_I, [_P, _I, _I, _I, _I, _I]),
    'uppe_pattern_probe': (_I, [_I, _I, _P, _P, _I, _P]),
    'uppe3d_profile_attempt': (_I, [_P, _I, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(_I),
                                    ctypes.POINTER(_D), ctypes.POINTER(_I), _P]),
}


def load(require_gpu=True):
    """Load the library (raises if it is missing, or if no GPU when required)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'{LIB_PATH} is missing: build it with `python -m project_b200.build` '
                           '(there is no CPU fallback)')
    if require_gpu and not torch.cuda.is_available():
        raise RuntimeError('project_b200 needs a CUDA GPU (sm_100a); there is no CPU fallback')
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, what):
    if rc != 0:
        msg = load(require_gpu=False).uppe_last_error()
        raise RuntimeError(f'{what} failed (rc={rc}): {msg.decode() if msg else ""}')


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
