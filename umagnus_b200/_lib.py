"""ctypes binding of the in-tree CUDA library libumagnus_b200.so.

The product path has no fallback: if the library is missing or no sm_100
GPU is present, every call raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libumagnus_b200.so")

c_int, c_float, c_double, c_void_p, c_size_t = ctypes.c_int, ctypes.c_float, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
c_ll = ctypes.c_longlong
P = c_void_p  # every device pointer


class UmagError(RuntimeError):
    pass


class SimParams(ctypes.Structure):
    _fields_ = [
        ("N", c_int * 3), ("cell", c_double * 3), ("pbc", c_int * 3),
        ("regions", P), ("vol", P),
        ("Ms", P), ("Ms_mul", c_float),
        ("alpha", P), ("alpha_mul", c_float),
        ("Ku1", P), ("Ku1_mul", c_float),
        ("Ku2", P), ("Ku2_mul", c_float),
        ("anisU", P * 3), ("anisU_mul", c_float * 3),
        ("aLUT", P), ("dLUT", P), ("bextLUT", P * 3),
        ("enable_demag", c_int), ("openbc", c_int), ("precess", c_int), ("asymptotic_radius", c_int),
        ("demag_kernel", c_int), ("demag_accuracy", c_double), ("frozen_lut", P),
        ("Kc1", P), ("Kc1_mul", c_float), ("Kc2", P), ("Kc2_mul", c_float), ("Kc3", P), ("Kc3_mul", c_float),
        ("anisC1", P * 3), ("anisC1_mul", c_float * 3), ("anisC2", P * 3), ("anisC2_mul", c_float * 3),
        ("dbulkLUT", P), ("temp", P), ("temp_mul", c_float), ("therm_seed", ctypes.c_ulonglong),
        ("nodemag_lut", P),
    ]


class SolverParams(ctypes.Structure):
    _fields_ = [("solver", c_int), ("dt", c_double), ("min_dt", c_double), ("max_dt", c_double),
                ("fix_dt", c_double), ("max_err", c_double), ("rel_err", c_double), ("min_slope", c_double),
                ("headroom", c_double), ("gamma_ll", c_double)]


class Tuning(ctypes.Structure):
    _fields_ = [("torque_block", c_int * 2), ("stage_threads", c_int), ("stage_waves", c_int), ("err_waves", c_int),
                ("torque_tma", c_int)]


class SolverState(ctypes.Structure):
    _fields_ = [("time", c_double), ("dt", c_double), ("last_err", c_double), ("peak_err", c_double),
                ("last_torque", c_double), ("nsteps", c_ll), ("nundone", c_ll), ("nevals", c_ll),
                ("status", c_int)]


class EnsInstance(ctypes.Structure):
    _fields_ = [("N", c_int * 3), ("cell", c_double * 3), ("Ms", c_float), ("Aex", c_float), ("alpha", c_float),
                ("Dind", c_float), ("Ku1", c_float), ("Ku2", c_float), ("anisU", c_float * 3), ("B_ext", c_float * 3)]


class AdjParams(ctypes.Structure):
    _fields_ = [("N", c_int * 3), ("cell", c_double * 3), ("alpha", c_float), ("anisU", c_float * 3),
                ("enable_demag", c_int), ("demag_kernel", c_int), ("demag_accuracy", c_double),
                ("dt", c_double), ("gamma_ll", c_double), ("nsteps", c_int), ("K", c_int), ("probe", c_int * 4),
                ("avg_from", c_int), ("w_probe", c_double), ("w_target", c_double), ("target", c_double * 3),
                ("no_graph", c_int), ("solver", c_int), ("Dind", c_float), ("pbc", c_int * 3),
                ("vol", c_void_p), ("regions", c_void_p), ("nregions", c_int)]


# name -> argtypes (restype int unless listed in _RESTYPE)
_SIGS = {
    "umag_init": [c_int], "umag_release": [], "umag_last_error": [], "umag_set_stream": [P], "umag_sync": [],
    "umag_version": [],
    "umag_malloc": [ctypes.POINTER(c_void_p), c_size_t], "umag_free": [P],
    "umag_memcpy_htod": [P, P, c_size_t], "umag_memcpy_dtoh": [P, P, c_size_t], "umag_memcpy_dtod": [P, P, c_size_t],
    "umag_memset_f32": [P, c_float, c_size_t],
    "umag_add_exchange": [P, P, P, P, P, P, P, c_float, P, P, c_int, c_int, c_int, c_double, c_double, c_double, c_int],
    "umag_add_dmi": [P, P, P, P, P, P, P, c_float, P, P, P, c_int, c_int, c_int, c_double, c_double, c_double, c_int,
                     c_int],
    "umag_add_uniaxial_anisotropy2": [P, P, P, P, P, P, P, c_float, P, c_float, P, c_float, P, c_float, P, c_float, P,
                                      c_float, c_int],
    "umag_add_dmi_bulk": [P, P, P, P, P, P, P, c_float, P, P, P, c_int, c_int, c_int, c_double, c_double, c_double,
                          c_int, c_int],
    "umag_add_cubic_anisotropy2": [P, P, P, P, P, P, P, c_float, P, c_float, P, c_float, P, c_float, P, P, P, P,
                                   c_int],
    "umag_region_addv": [P, P, P, P, P, P, P, c_int], "umag_region_decode": [P, P, P, c_int],
    "umag_zero_mask": [P, P, P, P, P, c_int],
    "umag_thermal_noise": [P, P, P, c_int, ctypes.c_ulonglong, c_ll],
    "umag_set_temperature": [P, P, c_float, P, c_float, P, c_float, P, c_float, c_int],
    "umag_lltorque": [P, P, P, P, P, P, P, P, P, P, c_float, c_int],
    "umag_llnoprecess": [P, P, P, P, P, P, P, P, P, c_int],
    "umag_madd": [c_int, P, c_int, P, P, c_int],
    "umag_normalize": [P, P, P, P, c_int], "umag_vecnorm": [P, P, P, P, c_int], "umag_div": [P, P, P, c_int],
    "umag_add_dot_product": [P, c_float, P, P, P, P, P, P, c_int],
    "umag_max_vec_norm": [P, P, P, c_int, ctypes.POINTER(c_double)],
    "umag_max_vec_diff": [P, P, P, P, P, P, c_int, ctypes.POINTER(c_double)],
    "umag_max_abs": [P, c_int, ctypes.POINTER(c_double)],
    "umag_sum": [P, c_int, ctypes.POINTER(c_double)], "umag_dot": [P, P, c_int, ctypes.POINTER(c_double)],
    "umag_demag_new_newell": [c_int, c_int, c_int, ctypes.POINTER(c_int), c_double, c_double, c_double, c_int, c_int,
                              ctypes.POINTER(c_void_p)],
    "umag_demag_new_from_kernel": [c_int, c_int, c_int, P, ctypes.POINTER(c_void_p)],
    "umag_demag_exec": [P, P, P, P, P, P, P, P, P, c_float],
    "umag_demag_new_brute": [c_int, c_int, c_int, P, c_double, c_double, c_double, c_double, P],
    "umag_demag_exec_pass": [P, c_int, P, P, P, P, P, P, P, P, c_float],
    "umag_demag_get_spectrum": [P, P], "umag_demag_get_kernel": [P, P],
    "umag_demag_padded_size": [P, ctypes.POINTER(c_int)], "umag_demag_free": [P],
    "umag_demag_exec_noalloc": [c_int, c_int, c_int, P, P, P, P, P, P, P, P, P, c_float, P],
    "umag_debug_plant_fault": [P, ctypes.c_uint],
    "umag_solver_defaults": [ctypes.POINTER(SolverParams)],
    "umag_sim_new": [ctypes.POINTER(SimParams), ctypes.POINTER(SolverParams), ctypes.POINTER(c_void_p)],
    "umag_sim_free": [P], "umag_sim_set_m": [P, P, P, P], "umag_sim_restore_m": [P, P, P, P], "umag_sim_get_m": [P, P, P, P],
    "umag_sim_m_ptrs": [P, P], "umag_sim_torque": [P, P, P, P, P, P, P], "umag_sim_steps": [P, c_int],
    "umag_sim_run": [P, c_double, c_int, c_ll], "umag_sim_get_state": [P, ctypes.POINTER(SolverState)],
    "umag_sim_set_time": [P, c_double, c_double], "umag_sim_average_m": [P, ctypes.POINTER(c_double)],
    "umag_sim_use_graph": [P, c_int, c_int], "umag_sim_launches_per_step": [P, ctypes.POINTER(c_int)],
    "umag_sim_torque_evals": [P, c_int],
    "umag_sim_energies": [P, ctypes.POINTER(c_double)], "umag_sim_energy_density": [P, P], "umag_sim_relax": [P, c_double],
    "umag_sim_set_solver": [P, ctypes.POINTER(SolverParams)], "umag_sim_set_param": [P, c_int, P, c_float],
    "umag_sim_get_tuning": [P, ctypes.POINTER(Tuning)], "umag_sim_set_tuning": [P, ctypes.POINTER(Tuning)],
    "umag_field_read_info": [ctypes.c_char_p, P], "umag_field_read": [ctypes.c_char_p, P, c_size_t, P],
    "umag_ovf_write": [ctypes.c_char_p, P, P, ctypes.c_char_p, c_int], "umag_dump_write": [ctypes.c_char_p, P, P],
    "umag_format_float": [c_double, c_int, ctypes.c_char_p, c_int],
    "umag_ens_new": [c_int, P, P, c_int, ctypes.POINTER(c_void_p)], "umag_ens_free": [P],
    "umag_ens_new_general": [c_int, P, P, P, c_int, ctypes.POINTER(c_void_p)],
    "umag_ens_class_general": [P, c_int, ctypes.POINTER(c_int)],
    "umag_ens_set_m": [P, c_int, P], "umag_ens_get_m": [P, c_int, P], "umag_ens_get_state": [P, c_int, P],
    "umag_ens_run": [P, c_double, c_int, c_ll], "umag_ens_count": [P, ctypes.POINTER(c_int), ctypes.POINTER(c_int)],
    "umag_ens_class_info": [P, c_int, ctypes.POINTER(c_int), ctypes.POINTER(c_int)],
    "umag_ens_get_tuning": [P, c_int, ctypes.POINTER(Tuning)], "umag_ens_set_tuning": [P, c_int, ctypes.POINTER(Tuning)],
    "umag_adj_new": [ctypes.POINTER(AdjParams), ctypes.POINTER(c_void_p)], "umag_adj_free": [P],
    "umag_adj_forward": [P, P, P, c_float, c_float, ctypes.POINTER(c_float), ctypes.POINTER(c_double)],
    "umag_adj_final_m": [P, P],
    "umag_adj_backward": [P, P, P, ctypes.POINTER(c_double), ctypes.POINTER(c_double), ctypes.POINTER(c_double)],
    "umag_adj_forward_regions": [P, P, P, ctypes.POINTER(c_float), ctypes.POINTER(c_float), ctypes.POINTER(c_float),
                                 ctypes.POINTER(c_double)],
    "umag_adj_backward_regions": [P, P, P, ctypes.POINTER(c_double), ctypes.POINTER(c_double),
                                  ctypes.POINTER(c_double)],
}
_RESTYPE = {"umag_last_error": ctypes.c_char_p, "umag_version": ctypes.c_char_p, "umag_solver_defaults": None}

_lib = None


def exported_names():
    return list(_SIGS)


def load():
    """Load the library (no device work).  Raises if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise UmagError(f"{LIB_PATH} is missing: run `python -m umagnus_b200.build` (no CPU fallback exists)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _RESTYPE.get(name, c_int)
        _lib = L
    return _lib


def check(status):
    if status != 0:
        raise UmagError(f"umagnus_b200 error {status}: {load().umag_last_error().decode()}")
    return status


_initialised = None


def init(device=0):
    """opencl.Init(gpu) (opencl/init.go:48)."""
    global _initialised
    L = load()
    if _initialised is None:
        check(L.umag_init(device))
        _initialised = device
    elif _initialised != device:
        raise UmagError(f"already initialised on device {_initialised}")
    return L
