"""ctypes binding of liblpm_b200.so (the C ABI declared in include/lpm_b200.h).

The library is loaded from the package directory (built in-tree by build.py).  There is no fallback: if the library
is missing, or no CUDA device is present when a GPU entry point is called, an error is raised.
"""
import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblpm_b200.so")

LPM_F64, LPM_F32 = 0, 1
LAYOUT_REF, LAYOUT_SOA = 0, 1
ENGINE_AUTO, ENGINE_LAUNCHED, ENGINE_PERSISTENT = 0, 1, 2
STATUS_OK, STATUS_NOT_CONVERGED, STATUS_BREAKDOWN = 0, 1, 2

_c_i32, _c_i64, _c_p, _c_sz, _c_d = ctypes.c_int32, ctypes.c_int64, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_double
_P = ctypes.POINTER


class Lattice(ctypes.Structure):
    _fields_ = [("dim", _c_i32), ("nx", _c_i32), ("ny", _c_i32), ("nz", _c_i32), ("n", _c_i64), ("nbr", _c_p)]


class Batch(ctypes.Structure):
    _fields_ = [("nsys", _c_i32), ("rhs_per_set", _c_i32), ("nmask", _c_i32), ("reserved", _c_i32)]


class CgOpts(ctypes.Structure):
    _fields_ = [("tol", _c_d), ("maxit", _c_i32), ("check", _c_i32), ("poll", _c_i32), ("precheck", _c_i32),
                ("prof", _P(_c_d)), ("tol_sys", _c_p), ("engine", _c_i32), ("reserved", _c_i32)]


class IrOpts(ctypes.Structure):
    _fields_ = [("tol", _c_d), ("inner_tol", _c_d), ("maxit", _c_i32), ("max_outer", _c_i32), ("check", _c_i32),
                ("poll", _c_i32), ("prof", _P(_c_d)), ("x_is_zero", _c_i32), ("engine", _c_i32)]


class AmgOpts(ctypes.Structure):
    _fields_ = [("agg", _c_i32), ("coarse_max", _c_i32), ("max_levels", _c_i32), ("nu", _c_i32), ("nu_c", _c_i32),
                ("gamma", _c_i32), ("w_from", _c_i32), ("power_its", _c_i32), ("omega", _c_d),
                ("rho0_per_box", _c_i32), ("reserved", _c_i32)]


_SIGS = {
    "lpm_abi_version": ([], ctypes.c_int),
    "lpm_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "lpm_graph_stats": ([_P(_c_i64), _P(_c_i64), _P(_c_i64)], None),
    "lpm_set_wait_limit_ns": ([ctypes.c_uint64], ctypes.c_uint64),
    "lpm_set_tma_wait_polls": ([ctypes.c_uint32], ctypes.c_uint32),
    "lpm_pack_coef_f32": ([_c_p, _c_p, _c_i64, _c_i32, _c_i32, _c_p], ctypes.c_int),
    "lpm_pack_coef_f64": ([_c_p, _c_p, _c_i64, _c_i32, _c_i32, _c_p], ctypes.c_int),
    "lpm_kmv_scratch_bytes": ([_P(Lattice), _c_i32, _c_i32], _c_i64),
    "lpm_kmv_sc_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_sz, _c_p], ctypes.c_int),
    "lpm_kmv_sc_f32": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_sz, _c_p], ctypes.c_int),
    "lpm_kmv_sq_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_sz, _c_p], ctypes.c_int),
    "lpm_kmv_sq_f32": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_sz, _c_p], ctypes.c_int),
    "lpm_block_jacobi_f64": ([_P(Lattice), _c_p, _c_p, _c_i32, _c_i32, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_block_jacobi_f32": ([_P(Lattice), _c_p, _c_p, _c_i32, _c_i32, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_cg_workspace_bytes": ([_P(Lattice), _P(Batch), _c_i32, _c_i32], _c_i64),
    "lpm_cg_persistent_fits": ([_P(Lattice), _P(Batch), ctypes.c_int32], ctypes.c_int),
    "lpm_cg_batched_f64": ([_P(Lattice), _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(CgOpts),
                            _c_p, _c_sz, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_cg_batched_f32": ([_P(Lattice), _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(CgOpts),
                            _c_p, _c_sz, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_csr_workspace_bytes": ([_c_i64], _c_i64),
    "lpm_csr_pcg_f64": ([_c_i64, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p, _P(CgOpts), _c_p, _c_sz, _c_p, _c_p, _c_p,
                         _c_p], ctypes.c_int),
    "lpm_ir_workspace_bytes": ([_P(Lattice), _P(Batch), _c_i32], _c_i64),
    "lpm_ir_batched": ([_P(Lattice), _c_p, _c_p, _c_i32, _c_p, _c_p, _c_p, _P(Batch), _c_p, _c_p, _c_p, _P(IrOpts),
                        _c_p, _c_sz, _c_p, _c_p, _c_p, _P(_c_i32), _c_p], ctypes.c_int),
    "lpm_grad_scratch_bytes": ([_P(Lattice), _c_i32], _c_i64),
    "lpm_bond_grad_sc": ([_P(Lattice), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_i32, _c_p, _c_sz,
                          _c_p], ctypes.c_int),
    "lpm_bond_grad_sq": ([_P(Lattice), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_i32, _c_p, _c_sz,
                          _c_p], ctypes.c_int),
    "lpm_stress_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_d, _c_p, _c_p, _c_sz, _c_p],
                       ctypes.c_int),
    "lpm_energy_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p], ctypes.c_int),
    "lpm_bond_scatter_f64": ([_c_i32, _c_i64, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_bond_gather_sym_f64": ([_c_i32, _c_i64, _c_i64, _c_p, _c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_group_eigmin_sc": ([_P(Lattice), _c_i32, _c_p, _c_p, _c_p, _c_i32, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_solid_nbr": ([_c_i32, _c_i32, _c_i32, _c_i32, _c_i32, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_build_nbr": ([_c_i32, _c_i32, _c_i32, _c_i32, _c_i64, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_energy_vjp_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_p, _c_i32, _c_p,
                            _c_sz, _c_p], ctypes.c_int),
    "lpm_stress_vjp_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_d, _c_p, _c_p, _c_p,
                            _c_i32, _c_p, _c_sz, _c_p], ctypes.c_int),
    "lpm_kmv_vjp_f64": ([_P(Lattice), _c_p, _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p, _c_p, _c_i32, _c_p,
                         _c_sz, _c_p], ctypes.c_int),
    "lpm_autotune_kmv": ([_P(Lattice), _P(Batch), _c_p, _c_p, _c_p, _c_sz, _P(_c_i32), _P(_c_i32), _c_p],
                         ctypes.c_int),
    "lpm_tune_kmv_set": ([_P(Lattice), _P(Batch), _c_i32, _c_i32], ctypes.c_int),
    "lpm_kmv_f64_static": ([_P(Lattice), _c_p, _c_p, _c_p, _c_i32, _P(Batch), _c_p, _c_p], ctypes.c_int),
    "lpm_amg_default_opts": ([_P(AmgOpts)], None),
    "lpm_amg_create": ([_P(Lattice), _P(Batch), _c_p, _c_i32, _c_p, _P(AmgOpts), _P(_c_p)], ctypes.c_int),
    "lpm_amg_destroy": ([_c_p], None),
    "lpm_amg_setup": ([_c_p, _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_amg_get_rho0": ([_c_p, _c_p], ctypes.c_int),
    "lpm_amg_set_rho0": ([_c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_amg_apply": ([_c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_amg_pcg_f32": ([_c_p, _c_p, _c_p, _P(CgOpts), _c_p, _c_p, _c_p, _c_p], ctypes.c_int),
    "lpm_ir_amg": ([_P(Lattice), _c_p, _c_p, _c_i32, _c_p, _P(Batch), _c_p, _c_p, _c_p, _P(IrOpts), _c_p, _c_sz,
                    _c_p, _c_p, _c_p, _P(_c_i32), _c_p], ctypes.c_int),
    "lpm_amg_info": ([_c_p, _c_i32, _P(_c_i32), _c_p, _P(_c_i64)], ctypes.c_int),
    "lpm_amg_get_level": ([_c_p, _c_i32, _c_i32, _c_i32, _c_p, _c_p, _c_p], ctypes.c_int),
}

_lib = None


class LPMError(RuntimeError):
    pass


def load():
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LPMError("%s is missing: build it with `python %s/build.py` (nvcc, sm_100a)" % (LIB_PATH, HERE))
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib


def graph_stats():
    """(captures, graphs held, cache flushes) of the library's CUDA-graph cache, process-wide."""
    c, e, f = _c_i64(0), _c_i64(0), _c_i64(0)
    load().lpm_graph_stats(ctypes.byref(c), ctypes.byref(e), ctypes.byref(f))
    return int(c.value), int(e.value), int(f.value)


def exported_symbols():
    return sorted(_SIGS)


def check(rc, what):
    if rc != 0:
        msg = load().lpm_status_string(int(rc)).decode()
        raise LPMError("%s failed: %s (code %d)" % (what, msg, rc))


def require_cuda(t):
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise LPMError("the LPM GPU path needs CUDA tensors (got %s); there is no CPU fallback" %
                       (getattr(t, "device", type(t)),))


def stream_ptr(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t):
    return ctypes.c_void_p(0 if t is None else t.data_ptr())
