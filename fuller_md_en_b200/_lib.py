"""ctypes binding of libfullermd_cuda.so (declared in include/fullermd.h).

The library is built in-tree by ``python -m fuller_md_en_b200.build``.  There
is no fallback: if the shared object is missing or no CUDA device is
usable, every call raises.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_longlong, c_void_p
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfullermd_cuda.so"

_dp = POINTER(c_double)
_ip = POINTER(c_int)

FMD_OK, FMD_ERR_ARG, FMD_ERR_CUDA, FMD_ERR_CAPACITY, FMD_ERR_NONFINITE, FMD_ERR_STATE = range(6)
FMD_PREC_FP64, FMD_PREC_FP32_PAIR = 0, 1
FMD_PHYS_MM_BONDED, FMD_PHYS_REBO, FMD_PHYS_QUAT = 1, 2, 4
FMD_REBO2_BOND_ORDER, FMD_REBO2_LJ_SWITCH = 1, 2
FMD_FF_AIREBO, FMD_FF_MM = 0, 1
FMD_SYS_RIGID, FMD_SYS_AIREBO, FMD_SYS_MM = 0, 1, 2


class NPT(ctypes.Structure):
    """fmd_npt: NPTState of the reference (LJ:425, AI:511, MM:804)."""
    _fields_ = [("xi", c_double), ("Q", c_double), ("Vg", c_double * 9), ("W", c_double),
                ("Pe", c_double), ("Tt", c_double), ("Nf", c_int)]


class Rebo2Knots(ctypes.Structure):
    """fmd_rebo2_knots: spline knots of the REBO-II extension -- P_CC(N, 0)
    at N = 0..4 {P, dP/dN}; pi^rc_CC and T_CC at N_ij, N_ji = 0..4,
    N_conj = 0..9 {f, f_x, f_y, f_z, f_xy, f_xz, f_yz, f_xyz}."""
    _fields_ = [("pcc", c_double * 10), ("pirc", c_double * 2000), ("tcc", c_double * 2000)]


class MMTopology(ctypes.Structure):
    """fmd_mm_topology: FlatTopology of the reference (MM:226-237)."""
    _fields_ = [("nb", c_int), ("b_i0", _ip), ("b_i1", _ip), ("b_kb", _dp), ("b_r0", _dp),
                ("nang", c_int), ("ang_i0", _ip), ("ang_i1", _ip), ("ang_i2", _ip), ("ang_kth", _dp),
                ("ang_th0", _dp),
                ("ndih", c_int), ("dih_i0", _ip), ("dih_i1", _ip), ("dih_i2", _ip), ("dih_i3", _ip),
                ("dih_vn", _dp), ("dih_mult", _ip), ("dih_gamma", _dp),
                ("nimp", c_int), ("imp_i0", _ip), ("imp_i1", _ip), ("imp_i2", _ip), ("imp_i3", _ip),
                ("imp_ki", _dp), ("imp_gamma", _dp)]


class RunParams(ctypes.Structure):
    _fields_ = [("dt", c_double), ("T", c_double), ("Pe", c_double), ("T_cold", c_double),
                ("coldstart", c_int), ("warmup", c_int), ("nsteps", c_int), ("nlup", c_int),
                ("gavg_from", c_int), ("gavg_to", c_int), ("nc", c_int), ("nmol", c_int),
                ("precision", c_int), ("use_graphs", c_int)]


class Obs(ctypes.Structure):
    _fields_ = [("step", c_int), ("T", c_double), ("P", c_double), ("a", c_double), ("KE", c_double),
                ("E", c_double * 8)]


class SgTrainArgs(ctypes.Structure):
    _fields_ = [("steps", c_int), ("batch", c_int), ("n_train", c_int), ("seed", c_int), ("lr", c_double),
                ("lr_final", c_double), ("wE", c_double), ("wF", c_double), ("wW", c_double), ("clip", c_double)]


class SgStatus(ctypes.Structure):
    """fmd_sg_status: judge record of the learned REBO term of a system."""
    _fields_ = [("attached", c_int), ("active", c_int), ("judged", c_int), ("takeover_step", c_int),
                ("rmse_last", c_double), ("rmse_max", c_double)]


class BatchTuning(ctypes.Structure):
    """fmd_batch_tuning: launch shapes the batch autotuner chose."""
    _fields_ = [("lj_threads", c_int), ("lj_unroll", c_int), ("lj_atoms_per_block", c_int), ("lj_staged", c_int),
                ("bonded_threads", c_int), ("bonded_terms_per_block", c_int), ("lj_ms", c_double),
                ("bonded_ms", c_double), ("blocks_lj", c_int), ("blocks_bonded", c_int), ("blocks_atom", c_int)]


class Avg(ctypes.Structure):
    _fields_ = [("n", c_int), ("sT", c_double), ("sP", c_double), ("sa", c_double), ("sE", c_double * 8)]


# name -> (restype, argtypes)
_SIGS = {
    "fmd_version": (c_int, []),
    "fmd_ctx_create": (c_int, [POINTER(c_void_p), c_int]),
    "fmd_ctx_destroy": (c_int, [c_void_p]),
    "fmd_ctx_set_stream": (c_int, [c_void_p, c_void_p]),
    "fmd_ctx_get_stream": (c_void_p, [c_void_p]),
    "fmd_ctx_synchronize": (c_int, [c_void_p]),
    "fmd_ctx_set_precision": (c_int, [c_void_p, c_int]),
    "fmd_ctx_last_error": (c_char_p, [c_void_p]),
    "fmd_status_string": (c_char_p, [c_int]),
    "fmd_device_info": (c_int, [c_int, c_char_p, c_int, POINTER(c_double)]),
    "fmd_mat_inv9": (c_int, [c_void_p, _dp, _dp]),
    "fmd_apply_pbc": (c_int, [c_void_p, _dp, _dp, _dp, c_int]),
    "fmd_nlist_rigid": (c_int, [c_void_p, _dp, _dp, _dp, c_int, c_double, c_int, _ip, _ip, _ip]),
    "fmd_nlist_lj_half": (c_int, [c_void_p, _dp, _dp, _dp, c_int, _ip, c_double, c_int, _ip, _ip, _ip]),
    "fmd_nlist_rebo": (c_int, [c_void_p, _dp, _dp, _dp, c_int, _ip, c_double, c_int, _ip, _ip, _ip]),
    "fmd_lj_rigid_forces": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, _ip, _ip, c_int, c_int, c_int,
                                    c_double, c_int, _dp, _dp, _dp, _dp]),
    "fmd_rebo_forces": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, c_int, _dp, _dp, _dp]),
    "fmd_lj_half_forces": (c_int, [c_void_p, c_int, _dp, _dp, _dp, _ip, _ip, c_int, c_int, _dp, _dp, _dp]),
    "fmd_rebo2_coeffs": (c_int, [POINTER(Rebo2Knots), _dp]),
    "fmd_rebo2_forces": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, c_int, POINTER(Rebo2Knots), _dp, _dp,
                                 _dp]),
    "fmd_lj_switch_forces": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, _ip, _ip, c_int, c_int,
                                     POINTER(Rebo2Knots), _dp, _dp, _dp]),
    "fmd_rebo_forces_noalloc": (c_int, [c_void_p, _dp, _dp, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                        c_void_p, c_void_p]),
    "fmd_airebo_forces": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, _ip, _ip, c_int, _dp, _dp, _dp]),
    "fmd_mm_forces": (c_int, [c_void_p, POINTER(MMTopology), _dp, _dp, _dp, _ip, _ip, _dp, _ip, c_int,
                              c_int, _dp, _dp, _dp]),
    "fmd_rigid_step": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, c_double,
                               c_double, c_int, c_int, c_double, c_double, POINTER(NPT), _ip, _ip, c_int,
                               c_int, _dp]),
    "fmd_airebo_step": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, _dp, c_int, c_double,
                                POINTER(NPT), _ip, _ip, _ip, _ip, _dp]),
    "fmd_mm_step": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, _dp, c_int, c_double, POINTER(NPT),
                            POINTER(MMTopology), _ip, _ip, _dp, _ip, c_int, _dp]),
    "fmd_system_create_rigid": (c_int, [c_void_p, POINTER(RunParams), c_int, c_int, _dp, c_double,
                                        c_double, c_double, c_int, _dp, _dp, _dp, _dp, _dp, POINTER(NPT),
                                        POINTER(c_void_p)]),
    "fmd_system_create_airebo": (c_int, [c_void_p, POINTER(RunParams), c_int, _dp, _dp, _dp, _ip, _dp,
                                         POINTER(NPT), POINTER(c_void_p)]),
    "fmd_system_create_mm": (c_int, [c_void_p, POINTER(RunParams), c_int, _dp, _dp, _ip,
                                     POINTER(MMTopology), _dp, _dp, POINTER(NPT), POINTER(c_void_p)]),
    "fmd_system_create_mm_replicated": (c_int, [c_void_p, POINTER(RunParams), c_int, c_int, _dp, _dp,
                                                POINTER(MMTopology), _dp, POINTER(NPT), POINTER(c_void_p)]),
    "fmd_system_init": (c_int, [c_void_p]),
    "fmd_system_run": (c_int, [c_void_p, c_int, c_int, POINTER(Obs)]),
    "fmd_system_enqueue": (c_int, [c_void_p, c_int, c_int]),
    "fmd_system_enqueue_obs": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "fmd_system_wait_obs": (c_int, [c_void_p, c_int]),
    "fmd_system_averages": (c_int, [c_void_p, POINTER(Avg)]),
    "fmd_system_download": (c_int, [c_void_p, _dp, _dp, _dp, _dp, _dp, POINTER(NPT)]),
    "fmd_system_lists": (c_int, [c_void_p, _ip, _ip, _ip, _ip]),
    "fmd_system_virial": (c_int, [c_void_p, _dp, _dp]),
    "fmd_system_destroy": (c_int, [c_void_p]),
    "fmd_system_kernel_ms": (c_int, [c_void_p, c_int, c_int, POINTER(c_double)]),
    "fmd_system_step_kernels": (c_int, [c_void_p, c_int, c_int, POINTER(c_int)]),
    "fmd_system_site_pairs": (c_int, [c_void_p, POINTER(c_longlong)]),
    "fmd_system_lj_shape": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "fmd_system_set_lj_shape": (c_int, [c_void_p, c_int, c_int, c_int]),
    "fmd_system_lj_shape_pruned": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int), POINTER(c_int)]),
    "fmd_system_set_lj_prune": (c_int, [c_void_p, c_double]),
    "fmd_system_forces": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "fmd_system_lj_rows": (c_int, [c_void_p, c_void_p, c_void_p]),
    "fmd_system_lj_full_rows": (c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_int)]),
    "fmd_system_set_physics": (c_int, [c_void_p, c_int]),
    "fmd_system_set_rebo2": (c_int, [c_void_p, POINTER(Rebo2Knots), c_int]),
    "fmd_system_lj_prune": (c_int, [c_void_p, POINTER(c_double), POINTER(c_longlong), POINTER(c_longlong)]),
    "fmd_sg_nparams": (c_int, []),
    "fmd_sg_create": (c_int, [c_void_p, _dp, POINTER(c_void_p)]),
    "fmd_sg_set_params": (c_int, [c_void_p, _dp]),
    "fmd_sg_get_params": (c_int, [c_void_p, _dp]),
    "fmd_sg_destroy": (c_int, [c_void_p]),
    "fmd_sg_rebo_forces": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, c_int, _dp, _dp, _dp]),
    "fmd_sg_last_rows": (c_int, [c_void_p, c_int, _ip, _ip, _ip, POINTER(c_float), POINTER(c_float),
                                 POINTER(c_float)]),
    "fmd_sg_data_create": (c_int, [c_void_p, POINTER(c_void_p)]),
    "fmd_sg_data_destroy": (c_int, [c_void_p]),
    "fmd_sg_data_count": (c_int, [c_void_p]),
    "fmd_sg_data_add": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, c_int]),
    "fmd_sg_data_add_system": (c_int, [c_void_p, c_void_p]),
    "fmd_sg_data_get": (c_int, [c_void_p, c_int, _ip, _dp, _dp, _dp]),
    "fmd_sg_loss_grad": (c_int, [c_void_p, _dp, _dp, _dp, _ip, _ip, c_int, c_int, _dp, c_double, _dp, c_double,
                                 c_double, c_double, _dp, _dp]),
    "fmd_sg_train": (c_int, [c_void_p, c_void_p, POINTER(SgTrainArgs), _dp]),
    "fmd_sg_eval": (c_int, [c_void_p, c_void_p, c_int, c_int, _dp]),
    "fmd_sg_feature_stats": (c_int, [c_void_p, c_void_p, c_int, c_int, _dp, _dp]),
    "fmd_system_use_surrogate": (c_int, [c_void_p, c_void_p, c_int, c_double]),
    "fmd_batch_create": (c_int, [c_void_p, c_int, POINTER(c_void_p), c_int, POINTER(c_void_p)]),
    "fmd_batch_run": (c_int, [c_void_p, c_int, c_int]),
    "fmd_batch_enqueue": (c_int, [c_void_p, c_int, c_int]),
    "fmd_batch_observables": (c_int, [c_void_p, POINTER(Obs)]),
    "fmd_batch_get_tuning": (c_int, [c_void_p, POINTER(BatchTuning)]),
    "fmd_batch_step_kernels": (c_int, [c_void_p, c_int, c_int, POINTER(c_int)]),
    "fmd_batch_step_kernels_conditional": (c_int, [c_void_p, c_int, c_int, POINTER(c_int)]),
    "fmd_batch_destroy": (c_int, [c_void_p]),
    "fmd_system_surrogate_status": (c_int, [c_void_p, POINTER(SgStatus)]),
}

_lib = None


class FmdError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def exported_symbols() -> list[str]:
    return sorted(_SIGS)


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Loads the library and declares every C-ABI signature.  Raises if the
    shared object has not been built; there is no CPU fallback."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FmdError(FMD_ERR_CUDA, f"{p} is not built; run `python -m fuller_md_en_b200.build`")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
