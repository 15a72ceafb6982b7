"""ctypes binding of libinqb200.so (the C ABI declared in include/inqb.h).

The library is built in-tree (``python -m inq_b200.build``).  There is no CPU
fallback: if the shared library is missing or no sm_100 device is present the
calls raise.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libinqb200.so")

INQB_OK = 0
REAL_SPACE, FOURIER_SPACE = 0, 1
F64, F32 = 0, 1

_lock = threading.Lock()
_lib = None


class InqbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"inqb error {code}: {msg}")
        self.code = code


P = C.c_void_p
I = C.c_int
D = C.c_double
LL = C.c_longlong
DP = C.POINTER(C.c_double)

# name: (restype, argtypes)
SIGNATURES = {
    "inqb_ctx_create": (I, [I, C.POINTER(P)]),
    "inqb_ctx_destroy": (I, [P]),
    "inqb_last_error": (C.c_char_p, [P]),
    "inqb_ctx_synchronize": (I, [P]),
    "inqb_ctx_stream": (I, [P, C.POINTER(P)]),
    "inqb_ctx_launch_count": (I, [P, C.POINTER(LL)]),
    "inqb_ctx_set_option": (I, [P, C.c_char_p, LL]),
    "inqb_device_alloc_count": (I, [C.POINTER(LL)]),
    "inqb_ctx_mem_info": (I, [P, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "inqb_basis_create": (I, [P, DP, I, I, I, C.POINTER(P)]),
    "inqb_basis_destroy": (I, [P]),
    "inqb_basis_volume_element": (I, [P, DP]),
    "inqb_orbitals_create": (I, [P, P, I, I, DP, I, I, I, C.POINTER(P)]),
    "inqb_orbitals_wrap": (I, [P, P, P, I, I, DP, I, I, I, C.POINTER(P)]),
    "inqb_orbitals_destroy": (I, [P]),
    "inqb_orbitals_upload": (I, [P, P]),
    "inqb_orbitals_download": (I, [P, P]),
    "inqb_orbitals_device_ptr": (I, [P, C.POINTER(P)]),
    "inqb_orbitals_copy": (I, [P, P]),
    "inqb_orbitals_fill": (I, [P, D, D]),
    "inqb_orbitals_set_space": (I, [P, I]),
    "inqb_orbitals_info": (I, [P, C.POINTER(I), C.POINTER(I), C.POINTER(I), C.POINTER(LL)]),
    "inqb_orbitals_randomize_gsphere": (I, [P, C.c_uint64, D]),
    "inqb_orbitals_convert": (I, [P, P]),
    "inqb_to_fourier": (I, [P, P]),
    "inqb_to_real": (I, [P, P, I]),
    "inqb_laplacian": (I, [P, P, D, DP]),
    "inqb_hamiltonian_create": (I, [P, P, I, C.POINTER(P)]),
    "inqb_hamiltonian_destroy": (I, [P]),
    "inqb_hamiltonian_set_option": (I, [P, C.c_char_p, LL]),
    "inqb_potential_set": (I, [P, DP]),
    "inqb_vector_potential_set": (I, [P, DP]),
    "inqb_hamiltonian_set_interaction": (I, [P, DP, I, I]),
    "inqb_update_hamiltonian": (I, [P, DP, DP]),
    "inqb_projectors_set": (I, [P, I, I, I, P, P, P, P, P, P]),
    "inqb_projectors_build_gaussian": (I, [P, I, DP, D, D, DP]),
    "inqb_projectors_build_gaussian_device": (I, [P, I, DP, D, D, DP]),
    "inqb_projectors_move": (I, [P, DP]),
    "inqb_projectors_build_radial": (I, [P, I, DP, P, I, DP, I, D, I, DP, P, P, DP]),
    "inqb_projectors_info": (I, [P, C.POINTER(I), C.POINTER(I), C.POINTER(LL)]),
    "inqb_spherical_grid": (I, [DP, I, I, I, DP, D, LL, P, P, P, C.POINTER(LL)]),
    "inqb_projectors_get": (I, [P, P, P, P, P]),
    "inqb_apply": (I, [P, P, P]),
    "inqb_apply_host": (I, [P, I, DP, I, I, P, P, I]),
    "inqb_apply_host_many": (I, [P, I, I, DP, I, I, P, P, I]),
    "inqb_steepest_descent": (I, [P, P]),
    "inqb_orbitals_save": (I, [P, C.c_char_p]),
    "inqb_orbitals_load": (I, [P, C.c_char_p]),
    "inqb_field_save": (I, [C.c_char_p, DP, LL, I]),
    "inqb_field_load": (I, [C.c_char_p, DP, LL, I]),
    "inqb_array_save": (I, [C.c_char_p, DP, LL]),
    "inqb_array_load": (I, [C.c_char_p, DP, LL]),
    "inqb_non_local": (I, [P, P, P]),
    "inqb_non_local_energy": (I, [P, P, DP, DP]),
    "inqb_kinetic_expectation_value": (I, [P, P, DP]),
    "inqb_overlap": (I, [P, P, DP]),
    "inqb_overlap_diagonal": (I, [P, P, DP]),
    "inqb_overlap_diagonal_noalloc": (I, [P, P, P]),
    "inqb_orthogonalize": (I, [P]),
    "inqb_shift": (I, [D, D, P, P]),
    "inqb_rotate": (I, [P, DP]),
    "inqb_rotate_to": (I, [P, P, DP, DP, DP]),
    "inqb_ctx_check_wait_timeout": (I, [P, LL]),
    "inqb_cholesky_inverse": (I, [I, DP, DP]),
    "inqb_hermitian_eigen": (I, [I, DP, DP, DP]),
    "inqb_eigenvalues": (I, [P, P, DP, DP]),
    "inqb_subspace_diagonalization": (I, [P, P, DP]),
    "inqb_exponential_in_place": (I, [P, D, D, P, I]),
    "inqb_exponential_2_for_1": (I, [P, D, D, D, D, P, P, I]),
    "inqb_density": (I, [C.POINTER(P), I, C.POINTER(DP), DP]),
    "inqb_kick": (I, [P, DP]),
    "inqb_dipole": (I, [P, DP, DP]),
    "inqb_batch_apply": (I, [P, I, C.POINTER(P), C.POINTER(P), C.POINTER(P), I]),
    "inqb_graph_capture_begin": (I, [P]),
    "inqb_graph_capture_end": (I, [P, C.POINTER(P)]),
    "inqb_graph_launch": (I, [P, P]),
    "inqb_graph_destroy": (I, [P]),
    "inqb_etrs_step": (I, [P, C.POINTER(P), I, C.POINTER(DP), D, I, D, DP, DP, C.POINTER(I)]),
}


def load(path: str | None = None):
    """Load (once) and return the CDLL with argtypes set: ``path``, else the INQB_LIBRARY environment
    variable, else the in-tree build.  Raises if the library is absent."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = path or os.environ.get("INQB_LIBRARY") or LIB_PATH
        if not os.path.exists(p):
            raise InqbError(-1, f"{p} is missing: build it with `python -m inq_b200.build`")
        lib = C.CDLL(p)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(code, ctx_handle=None):
    if code != INQB_OK:
        lib = load()
        msg = lib.inqb_last_error(ctx_handle)
        raise InqbError(code, msg.decode() if msg else "")


def dptr(arr):
    """ctypes double* of a contiguous float64 numpy array."""
    import numpy as np
    assert arr.dtype == np.float64 and arr.flags.c_contiguous
    return arr.ctypes.data_as(DP)
