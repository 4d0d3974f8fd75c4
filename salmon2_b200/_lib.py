"""ctypes loader for ``libsalmon_b200.so`` (the sm_100a CUDA library).

The library is built in-tree (``make -C salmon2_b200/csrc``).  There is no CPU
fallback: if the shared object is missing or cannot be loaded, every entry
point raises :class:`SB200Error`.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsalmon_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "salmon_b200.h")

SB200_OK = 0
ERROR_NAMES = {1: "INVALID_ARG", 2: "BAD_SHAPE", 3: "UNSUPPORTED", 4: "OOM", 5: "CUDA", 6: "TIMEOUT", 7: "STATE"}
PREC_FP64, PREC_MIXED = 0, 1
TRANS_TR, TRANS_LO = 0, 1
PRECOND_NONE, PRECOND_LOWPASS, PRECOND_LEARNED = 0, 1, 2
LEARNED_CHANNELS, LEARNED_NPARAM = 16, 8241
KIND_NAMES = ["prep", "project", "hpsi", "observables", "moments", "finalize", "potential", "k7"]


class SB200Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"salmon_b200 error {code} ({ERROR_NAMES.get(code, '?')}): {msg}")
        self.code = code


_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_vp = C.c_void_p

# name -> (restype, argtypes); mirrors include/salmon_b200.h
SIGNATURES = {
    "sb200_ctx_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    "sb200_ctx_destroy": (C.c_int, [_vp]),
    "sb200_ctx_set_stream": (C.c_int, [_vp, _vp]),
    "sb200_ctx_sync": (C.c_int, [_vp]),
    "sb200_last_error": (C.c_char_p, []),
    "sb200_version": (C.c_char_p, []),
    "sb200_set_timing": (C.c_int, [_vp, C.c_int]),
    "sb200_kernel_times": (C.c_int, [_vp, _dp, C.POINTER(C.c_long), C.c_int]),
    "sb200_set_grid": (C.c_int, [_vp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _dp, C.c_double, C.c_double, _dp, _dp]),
    "sb200_set_orbitals": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]),
    "sb200_set_vlocal": (C.c_int, [_vp, _dp]),
    "sb200_set_pp": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, _ip, _ip, _dp, _dp, _ip, _dp]),
    "sb200_set_vec_Ac": (C.c_int, [_vp, _dp]),
    "sb200_set_precision": (C.c_int, [_vp, C.c_int]),
    "sb200_orbital_block_bytes": (C.c_size_t, [_vp]),
    "sb200_orbitals_from_ref": (C.c_int, [_vp, _vp, _vp]),
    "sb200_orbitals_to_ref": (C.c_int, [_vp, _vp, _vp]),
    "sb200_hpsi": (C.c_int, [_vp, _vp, _vp]),
    "sb200_hpsi_tt": (C.c_int, [_vp, _vp, _vp, _vp]),
    "sb200_calc_eigen_energy": (C.c_int, [_vp, _vp, _vp, _vp, _dp, _dp, _dp]),
    "sb200_taylor": (C.c_int, [_vp, _vp, _vp, _vp, _dp, C.c_int]),
    "sb200_calc_density": (C.c_int, [_vp, _vp, _vp]),
    "sb200_calc_current": (C.c_int, [_vp, _vp, _dp, _dp]),
    "sb200_calc_dip": (C.c_int, [_vp, _vp, _dp]),
    "sb200_exc_cor_pz": (C.c_int, [_vp, _vp, _vp, _dp]),
    "sb200_hartree_periodic": (C.c_int, [_vp, _dp, _vp, _vp]),
    "sb200_update_vlocal": (C.c_int, [_vp, _vp, _vp, _vp]),
    "sb200_hartree_isolated_ft": (C.c_int, [_vp, _dp, _vp, _vp]),
    "sb200_check_grid_barrier": (C.c_int, [_vp, C.c_int]),
    "sb200_hartree_isolated_cg": (C.c_int, [_vp, _vp, _vp, C.c_int, C.c_int, _dp, C.c_int, _ip, C.c_double,
                                            C.c_int, _ip]),
    "sb200_set_lattice": (C.c_int, [_vp, _dp, _dp]),
    "sb200_set_micro_ac": (C.c_int, [_vp, _vp, _vp]),
    "sb200_set_symmetrized_stencil": (C.c_int, [_vp, C.c_int]),
    "sb200_set_absorbing_boundary": (C.c_int, [_vp, C.c_int, C.c_double, C.c_double, C.c_double]),
    "sb200_set_length_gauge": (C.c_int, [_vp, C.c_int]),
    "sb200_set_propagator": (C.c_int, [_vp, C.c_int]),
    "sb200_set_predictor_corrector": (C.c_int, [_vp, C.c_int]),
    "sb200_set_gram_schmidt_interval": (C.c_int, [_vp, C.c_int]),
    "sb200_calc_microscopic_current": (C.c_int, [_vp, _vp, _vp]),
    "sb200_init_ps_ky": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), _ip, _ip, C.c_int, _ip, _ip, _dp, C.c_double,
                                   C.c_int, _ip, _dp, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _dp, _dp]),
    "sb200_rt_set_start": (C.c_int, [_vp, C.c_int, _dp, _dp]),
    "sb200_rt_get_state": (C.c_int, [_vp, _ip, _dp, _dp]),
    "sb200_write_restart": (C.c_int, [_vp, C.c_char_p, C.c_int, C.c_int, _vp, C.c_int, C.c_int, C.c_int]),
    "sb200_read_restart": (C.c_int, [_vp, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _vp, _ip,
                                     _dp]),
    "sb200_set_psmask": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double]),
    "sb200_init_ps": (C.c_int, [C.c_int, C.POINTER(C.c_char_p), _ip, _ip, C.c_int, _ip, _ip, _dp, C.c_double,
                                C.c_int, _ip, _dp, _ip, _ip, _ip, _ip, _dp, _dp, _ip, _dp, _dp]),
    "sb200_set_hartree_cg": (C.c_int, [_vp, _vp, C.c_int, C.c_int, _dp, C.c_int, _ip, C.c_double, C.c_int]),
    "sb200_set_self_consistent": (C.c_int, [_vp, C.c_int, _vp, _dp]),
    "sb200_nccl_unique_id": (C.c_int, [_vp]),
    "sb200_set_density_comm": (C.c_int, [_vp, C.c_int, C.c_int, _vp]),
    "sb200_rt_propagate": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_double, _dp, C.c_int, _dp, C.c_int, _dp,
                                     _dp, _dp, C.POINTER(C.c_void_p)]),
    "sb200_gs_from_ref": (C.c_int, [_vp, _vp, _vp]),
    "sb200_gs_to_ref": (C.c_int, [_vp, _vp, _vp]),
    "sb200_hpsi_real": (C.c_int, [_vp, _vp, _vp]),
    "sb200_gscg": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_double, _dp]),
    "sb200_gram_schmidt_real": (C.c_int, [_vp, _vp]),
    "sb200_gram_schmidt_complex": (C.c_int, [_vp, _vp]),
    "sb200_subspace_diag_real": (C.c_int, [_vp, _vp, _dp]),
    "sb200_learned_init": (C.c_int, [_vp, _vp, C.c_int, C.c_int]),
    "sb200_learned_get_params": (C.c_int, [_vp, _vp, C.c_int]),
    "sb200_learned_forward": (C.c_int, [_vp, _vp, _vp, C.c_int]),
    "sb200_learned_loss_grad": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, _dp, _vp]),
    "sb200_learned_train_step": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_float, _dp]),
    "sb200_batch_create": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_void_p)]),
    "sb200_batch_destroy": (C.c_int, [_vp]),
    "sb200_batch_set_tiles": (C.c_int, [_vp, _ip, _ip]),
    "sb200_batch_get_tiles": (C.c_int, [_vp, _ip, _ip]),
    "sb200_batch_autotune": (C.c_int, [_vp, _vp, _vp, C.c_int, _ip, _ip]),
    "sb200_batch_propagate": (C.c_int, [_vp, _vp, _vp, _vp, C.c_int, C.c_double, _dp, C.c_int, _vp, _vp]),
    "sb200_impulse_kick": (C.c_int, [_vp, _vp, C.c_double, _dp]),
    "sb200_hpsi_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _ip,
                                     C.c_double, _dp, _dp, _vp, _vp, C.c_int, C.c_int, C.c_int, _vp, _vp, _vp,
                                     _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}


def build(force: bool = False) -> str:
    """Compile the CUDA library for sm_100a with nvcc (no GPU needed)."""
    cmd = ["make", "-s", "-C", os.path.join(HERE, "csrc")]
    if force:
        subprocess.run(cmd + ["clean"], check=True)
    subprocess.run(cmd + ["-j4"], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise SB200Error(5, f"{LIB_PATH} is missing: build it with `make -C salmon2_b200/csrc`")
        try:
            L = C.CDLL(LIB_PATH)
        except OSError as e:  # no CUDA driver / runtime
            raise SB200Error(5, f"cannot load {LIB_PATH}: {e}") from e
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != SB200_OK:
        raise SB200Error(rc, lib().sb200_last_error().decode())
    return rc
