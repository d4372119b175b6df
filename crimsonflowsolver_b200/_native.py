"""ctypes binding of libcrimson_b200.so (the C ABI in include/crimson_b200.h).

The library is built in-tree by ``crimsonflowsolver_b200.build()`` (nvcc,
sm_100a).  Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcrimson_b200.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "crimson_b200.h")

c_int_p = ctypes.POINTER(ctypes.c_int)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_void_p = ctypes.c_void_p

OK = 0
ERRORS = {1: "ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "OOM", 5: "PATTERN", 6: "SINGULAR", 7: "NONFINITE", 8: "STATE"}


class Params(ctypes.Structure):
    _fields_ = [("rho", ctypes.c_double), ("mu", ctypes.c_double), ("alfi", ctypes.c_double),
                ("almi", ctypes.c_double), ("gami", ctypes.c_double), ("Delt", ctypes.c_double),
                ("Dtgl", ctypes.c_double), ("dtsfct", ctypes.c_double), ("taucfct", ctypes.c_double),
                ("flmpl", ctypes.c_double), ("flmpr", ctypes.c_double), ("stabflux_coeff", ctypes.c_double),
                ("idiff", ctypes.c_int), ("iconvflow", ctypes.c_int), ("itau", ctypes.c_int),
                ("ibksiz", ctypes.c_int), ("ndofBC", ctypes.c_int), ("nthreads", ctypes.c_int)]


class SubLs(ctypes.Structure):
    _fields_ = [("absTol", ctypes.c_double), ("relTol", ctypes.c_double), ("iNorm", ctypes.c_double),
                ("fNorm", ctypes.c_double), ("dB", ctypes.c_double), ("callD", ctypes.c_double),
                ("suc", ctypes.c_int), ("mItr", ctypes.c_int), ("sD", ctypes.c_int), ("itr", ctypes.c_int),
                ("cM", ctypes.c_int), ("cN", ctypes.c_int), ("cD", ctypes.c_int), ("reserve", ctypes.c_int)]


class LsStats(ctypes.Structure):
    _fields_ = [("GM", SubLs), ("CG", SubLs), ("RI", SubLs), ("LS_type", ctypes.c_int), ("Resm", ctypes.c_int),
                ("Resc", ctypes.c_int)]


class StepArgs(ctypes.Structure):
    _fields_ = [("nitr", ctypes.c_int), ("inflow_scale", ctypes.c_double), ("rescontrol", ctypes.c_int),
                ("res_criteria", ctypes.c_double), ("min_iters", ctypes.c_int)]


class StepStats(ctypes.Structure):
    _fields_ = [("nsolves", ctypes.c_int), ("ri_itr", ctypes.c_int * 16), ("gm_itr", ctypes.c_int * 16),
                ("cg_itr", ctypes.c_int * 16), ("ri_inorm", ctypes.c_double * 16),
                ("ri_fnorm", ctypes.c_double * 16), ("q_out", ctypes.c_double * 8), ("p_out", ctypes.c_double * 8),
                ("refine_steps", ctypes.c_int * 16), ("refine_rel", ctypes.c_double * 16),
                ("res_norm", ctypes.c_double * 16)]


# name -> (restype, argtypes)
SIGNATURES = {
    "crimson_ctx_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.POINTER(Params), ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, c_int_p, c_dbl_p]),
    "crimson_ctx_destroy": (ctypes.c_int, [c_void_p]),
    "crimson_set_params": (ctypes.c_int, [c_void_p, ctypes.POINTER(Params)]),
    "crimson_set_bc": (ctypes.c_int, [c_void_p, c_int_p, c_dbl_p]),
    "crimson_set_boundary": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p, c_int_p, c_dbl_p]),
    "crimson_set_outlets": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p, c_int_p, c_dbl_p]),
    "crimson_genadj": (ctypes.c_int, [c_void_p, c_int_p, c_int_p, ctypes.c_longlong,
                                      ctypes.POINTER(ctypes.c_longlong)]),
    "crimson_elmgmr": (ctypes.c_int, [c_void_p, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p,
                                      ctypes.c_int]),
    "crimson_elmgmr_device": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_dbl_p, c_dbl_p, c_void_p, c_void_p,
                                             c_void_p, ctypes.c_int]),
    "crimson_elmgmr_sclr": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_double, c_dbl_p, c_dbl_p, c_dbl_p,
                                           c_dbl_p, c_dbl_p, c_dbl_p, ctypes.c_int]),
    "crimson_elmgmr_sclr_device": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_double, c_void_p, c_void_p,
                                                  c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int]),
    "crimson_memls_ls_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.c_int, ctypes.c_int,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                               c_dbl_p, c_dbl_p, c_int_p]),
    "crimson_memls_ls_free": (ctypes.c_int, [c_void_p]),
    "crimson_memls_ls_set_precision": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "crimson_memls_refine_info": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int), c_dbl_p]),
    "crimson_memls_ls_set_schur": (ctypes.c_int, [c_void_p, ctypes.c_int]),
    "crimson_memls_schur_info": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                                c_dbl_p]),
    "crimson_memls_ls_set_log": (ctypes.c_int, [c_void_p, ctypes.c_char_p]),
    "crimson_memls_lhs_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.c_int, ctypes.c_int,
                                                ctypes.c_longlong, c_int_p, c_int_p, c_int_p, ctypes.c_int]),
    "crimson_memls_lhs_create_from_ctx": (ctypes.c_int, [ctypes.POINTER(c_void_p), c_void_p, ctypes.c_int]),
    "crimson_memls_lhs_free": (ctypes.c_int, [c_void_p]),
    "crimson_memls_bc_create": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                               c_int_p, c_dbl_p]),
    "crimson_memls_solve": (ctypes.c_int, [c_void_p, c_void_p, ctypes.c_int, c_dbl_p, c_dbl_p, c_int_p, c_dbl_p,
                                           ctypes.POINTER(LsStats)]),
    "crimson_solflow_device": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int_p,
                                              c_dbl_p, c_void_p, ctypes.POINTER(LsStats)]),
    "crimson_solflow_device_transposed": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                                         c_int_p, c_dbl_p, c_void_p, ctypes.POINTER(LsStats)]),
    "crimson_elmgmr_vjp": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_dbl_p, c_dbl_p, c_void_p, c_void_p,
                                          c_void_p, c_void_p, c_dbl_p, c_dbl_p, c_dbl_p]),
    "crimson_rcr_state": (ctypes.c_int, [c_void_p, ctypes.c_int, c_dbl_p, c_dbl_p, ctypes.c_int]),
    "crimson_spmv4_prepare": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p]),
    "crimson_elmgmr_device_f32": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_dbl_p, c_dbl_p, c_void_p,
                                                 c_void_p]),
    "crimson_solflow_device_f32": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int_p,
                                                  c_dbl_p, c_void_p, ctypes.POINTER(LsStats)]),
    "crimson_spmv4_apply": (ctypes.c_int, [c_void_p, c_void_p, c_void_p]),
    "crimson_set_inflow": (ctypes.c_int, [c_void_p, ctypes.c_int, c_int_p, c_dbl_p]),
    "crimson_set_rcr": (ctypes.c_int, [c_void_p, ctypes.c_int, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p]),
    "crimson_state_set": (ctypes.c_int, [c_void_p, c_dbl_p, c_dbl_p]),
    "crimson_state_get": (ctypes.c_int, [c_void_p, c_dbl_p, c_dbl_p]),
    "crimson_step": (ctypes.c_int, [c_void_p, c_void_p, c_void_p, ctypes.POINTER(StepArgs),
                                    ctypes.POINTER(StepStats)]),
    "crimson_ctx_stream": (c_void_p, [c_void_p]),
    "crimson_pvsq_noalloc": (ctypes.c_int, [ctypes.c_int, c_int_p, c_void_p, c_void_p, c_void_p, c_dbl_p, c_dbl_p,
                                            c_void_p, c_dbl_p, c_void_p]),
    "crimson_launch_count": (ctypes.c_ulonglong, []),
    "crimson_memls_kernel_time": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, c_dbl_p]),
    "crimson_memls_cg_layout": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                               ctypes.POINTER(ctypes.c_longlong)]),
    "crimson_netlist_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.c_int, c_int_p, c_int_p, c_int_p,
                                              c_dbl_p, c_dbl_p, c_dbl_p, ctypes.c_int, c_dbl_p, ctypes.c_int, c_int_p,
                                              c_dbl_p, ctypes.c_int, c_int_p, c_int_p, c_dbl_p, ctypes.c_int]),
    "crimson_netlist_create_member": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.c_int, c_int_p, c_int_p,
                                                     c_int_p, c_dbl_p, c_dbl_p, c_dbl_p, ctypes.c_int, c_dbl_p,
                                                     ctypes.c_int, c_int_p, c_dbl_p, ctypes.c_int, c_int_p, c_int_p,
                                                     c_dbl_p, ctypes.c_int, ctypes.c_int, c_int_p]),
    "crimson_netlist_loop_create": (ctypes.c_int, [ctypes.POINTER(c_void_p), ctypes.c_int, ctypes.POINTER(c_void_p),
                                                   c_void_p, ctypes.c_int, c_int_p, c_int_p, c_int_p]),
    "crimson_netlist_loop_free": (None, [c_void_p]),
    "crimson_netlist_loop_implicit_coefficients": (ctypes.c_int, [c_void_p, ctypes.c_double, c_dbl_p, c_dbl_p]),
    "crimson_netlist_loop_update": (ctypes.c_int, [c_void_p, ctypes.c_double, c_dbl_p, c_dbl_p]),
    "crimson_netlist_loop_finalize_step": (ctypes.c_int, [c_void_p]),
    "crimson_netlist_free": (None, [c_void_p]),
    "crimson_netlist_flow_permitted": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "crimson_netlist_implicit_coefficients": (ctypes.c_int, [c_void_p, ctypes.c_double, c_dbl_p, c_dbl_p]),
    "crimson_netlist_update": (ctypes.c_int, [c_void_p, ctypes.c_double, ctypes.c_double]),
    "crimson_netlist_update_pressure": (ctypes.c_int, [c_void_p, ctypes.c_double, ctypes.c_double]),
    "crimson_netlist_get_parameter": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "crimson_netlist_set_parameter": (ctypes.c_int, [c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
    "crimson_netlist_finalize_step": (ctypes.c_int, [c_void_p]),
    "crimson_netlist_get": (ctypes.c_int, [c_void_p, c_dbl_p, c_dbl_p, c_int_p, c_dbl_p]),
    "crimson_netlist_state_size": (ctypes.c_int, [c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "crimson_netlist_state": (ctypes.c_int, [c_void_p, c_dbl_p, ctypes.c_int]),
    "crimson_set_outlet_netlist": (ctypes.c_int, [c_void_p, ctypes.c_int, c_void_p]),
    "crimson_set_outlet_netlist_loop": (ctypes.c_int, [c_void_p, c_void_p, c_int_p]),
    "crimson_outlet_state": (ctypes.c_int, [c_void_p, ctypes.c_int, c_dbl_p, c_dbl_p]),
    "crimson_version": (ctypes.c_char_p, []),
    "crimson_last_error": (ctypes.c_char_p, []),
}

_lib = None


def build(verbose: bool = False) -> str:
    """Compile libcrimson_b200.so for sm_100a with nvcc (make in csrc/)."""
    out = subprocess.run(["make", "-C", os.path.join(_HERE, "csrc")], capture_output=not verbose, text=True)
    if out.returncode != 0:
        raise RuntimeError("building libcrimson_b200.so failed:\n" + (out.stdout or "") + (out.stderr or ""))
    return LIB_PATH


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run crimsonflowsolver_b200.build() (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str) -> None:
    if rc != OK:
        msg = lib().crimson_last_error()
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)} ({msg.decode() if msg else ''})")


def ip(a):
    return a.ctypes.data_as(c_int_p) if a is not None else None


def dp(a):
    return a.ctypes.data_as(c_dbl_p) if a is not None else None
