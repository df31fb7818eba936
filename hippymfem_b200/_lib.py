"""ctypes binding of ``libhippymfem_b200.so`` (the C ABI of ``include/hippymfem_b200.h``).

The library is the only compute path: if it is missing this module raises at import,
and every call checks that its tensors live on a CUDA device.  There is no CPU
fallback.
"""

import ctypes
import os

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libhippymfem_b200.so")

HM_OK, HM_ERR_ARG, HM_ERR_CUDA, HM_ERR_NONFINITE = 0, 1, 2, 3
HM_ERR_NOMEM, HM_ERR_NOCONV, HM_ERR_RANGE, HM_ERR_UNSUPPORTED = 4, 5, 6, 7
HM_STATUS_NONFINITE, HM_STATUS_RANGE = 1, 2
HM_FP64, HM_FP32 = 0, 1


class NotConvergedError(RuntimeError):
    """An iterative solve stopped at its iteration limit before its tolerance."""


_EXC = {HM_ERR_ARG: ValueError, HM_ERR_CUDA: RuntimeError, HM_ERR_NONFINITE: RuntimeError,
        HM_ERR_NOMEM: MemoryError, HM_ERR_NOCONV: NotConvergedError,
        HM_ERR_RANGE: IndexError, HM_ERR_UNSUPPORTED: NotImplementedError}

if not os.path.exists(LIBPATH):
    raise ImportError("libhippymfem_b200.so is not built (%s); run "
                      "`python hippymfem_b200/build.py`" % LIBPATH)

lib = ctypes.CDLL(LIBPATH)

_p = ctypes.c_void_p
_i32, _i64, _d = ctypes.c_int, ctypes.c_int64, ctypes.c_double

# name: (restype, argtypes) -- one entry per declaration of include/hippymfem_b200.h
SIGNATURES = {
    "hm_error_string": (ctypes.c_char_p, [_i32]),
    "hm_version": (_i32, []),
    "hm_pattern_build": (_i32, [_p, _p, _i64, _i32, _i32, _i64, _i64, _i32, _i32, _p, _p, _i64,
                                _p, _p]),
    "hm_lattice_create": (_i32, [_i32, _i32, _i32, _d, _d, _d, _p]),
    "hm_lattice_destroy": (_i32, [_p]),
    "hm_lattice_sizes": (_i32, [_p, _i32, _p, _p, _p, _p]),
    "hm_lattice_pattern": (_i32, [_p, _p, _p, _p, _p]),
    "hm_lattice_transpose_map": (_i32, [_p, _p, _p, _p]),
    "hm_lattice_quadrature": (_i32, [_p, _p, _p, _p, _i32, _p, _p, _p]),
    "hm_lattice_assemble": (_i32, [_p, _p, _i32, _p, _p, _d, _p, _p, _p, _p, _p, _p, _p, _i32,
                                   _p]),
    "hm_lattice_residual_noalloc": (_i32, [_p, _p, _p, _p, _d, _p, _p, _p, _p, _i32, _p, _p]),
    "hm_lattice_jacobian_bytes": (_i64, [_p, _i32]),
    "hm_lattice_jacobian_prepare": (_i32, [_p, _p, _i32, _p, _i32, _p]),
    "hm_lattice_apply_A": (_i32, [_p, _p, _i32, _p, _p, _p, _p]),
    "hm_lattice_diag_A": (_i32, [_p, _p, _i32, _p, _p, _p]),
    "hm_csr_spmv": (_i32, [_i64, _p, _p, _p, _p, _p, _d, _d, _p]),
    "hm_csr_spmv_t": (_i32, [_i64, _p, _p, _p, _p, _p, _p, _d, _d, _p]),
    "hm_lattice_observation_workspace_bytes": (_i64, [_i64]),
    "hm_lattice_observation": (_i32, [_p, _p, _i64, _p, _p, _p, _p, _p]),
    "hm_csr_transpose_workspace_bytes": (_i64, [_i64]),
    "hm_csr_transpose": (_i32, [_i64, _i64, _i64, _p, _p, _p, _p, _p, _p, _p, _p]),
    "hm_csr_diag": (_i32, [_i64, _p, _p, _p, _p]),
    "hm_pcg_workspace_bytes": (_i64, [_i64]),
    "hm_pcg": (_i32, [_i64, _p, _p, _p, _p, _p, _i32, _p, _p, _p, _p, _d, _i32, _i32, _p, _p,
                      _p, _p]),
    "hm_pcg_mixed_workspace_bytes": (_i64, [_i64]),
    "hm_pcg_mixed": (_i32, [_p, _p, _p, _p, _p, _p, _p, _d, _d, _i32, _i32, _i32, _p, _p, _p, _p,
                            _p]),
    "hm_device_status": (_i32, [_p, _i32]),
    "hm_pcg_plan_create": (_i32, [_p, _p, _p, _p, _p, _p, _p, _p, _i32, _p]),
    "hm_pcg_plan_solve": (_i32, [_p, _d, _d, _i32, _i32, _p, _p, _p, _p]),
    "hm_pcg_plan_destroy": (_i32, [_p]),
    "hm_lattice_quadrature_dir": (_i32, [_p, _p, _p, _p, _p, _i32, _p, _p, _p]),
    "hm_mg_workspace_bytes": (_i64, [_p]),
    "hm_mg_create": (_i32, [_p, _p, _i32, _i32, _p]),
    "hm_mg_setup": (_i32, [_p, _p, _p, _p, _p]),
    "hm_mg_apply": (_i32, [_p, _p, _p, _p]),
    "hm_mg_levels": (_i32, [_p]),
    "hm_mg_set_tail_nodes": (_i32, [_p, _i64]),
    "hm_mg_set_fused": (_i32, [_p, _i32]),
    "hm_mg_single_workspace_bytes": (_i64, [_p]),
    "hm_mg_set_single": (_i32, [_p, _p, _p]),
    "hm_mg_destroy": (_i32, [_p]),
    "hm_pcg_mg": (_i32, [_p, _p, _p, _d, _i32, _i32, _p, _p, _p, _p]),
    "hm_pcg_plan_set_mg": (_i32, [_p, _p]),
    "hm_lattice_dof_permutation": (_i32, [_p, _p, _p, _p]),
    "hm_lattice_caller_map": (_i32, [_p, _p, _p, _p, _p, _p, _p]),
    "hm_gather_f64": (_i32, [_i64, _p, _p, _p, _p]),
    "hm_lattice_element_blocks": (_i32, [_p, _p, _i32, _i64, _i64, _p, _p, _p, _p, _p, _p]),
    "hm_hessian_workspace_bytes": (_i64, [_i64, _i64]),
    "hm_hessian_create": (_i32, [_p, _p, _p, _p, _p, _p, _p, _i64, _p, _p, _p, _p, _p, _p, _d,
                                 _p, _p, _p, _p]),
    "hm_hessian_apply": (_i32, [_p, _p, _p, _d, _i32, _p, _p]),
    "hm_hessian_destroy": (_i32, [_p]),
    "hm_lattice_consistent_workspace_bytes": (_i64, [_p]),
    "hm_lattice_assemble_consistent": (_i32, [_p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "hm_pcg_group_create": (_i32, [_p, _i32, _p]),
    "hm_pcg_group_solve": (_i32, [_p, _d, _i32, _p, _p, _p]),
    "hm_pcg_group_destroy": (_i32, [_p]),
    "hm_lattice_add_boundary_mass": (_i32, [_p, _d, _p, _p]),
    "hm_lattice_vectors_workspace_bytes": (_i64, [_p, _i32]),
    "hm_lattice_vectors": (_i32, [_p, _p, _p, _p, _p, _d, _p, _p, _p, _p, _i32, _p, _p, _p]),
    "hm_lattice_vectors_at": (_i32, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _d, _p, _p, _p, _p,
                                     _p, _p, _p]),
    "hm_dot_workspace_bytes": (_i64, [_i64]),
    "hm_dot": (_i32, [_i64, _p, _p, _p, _p, _p]),
}

for _name, (_res, _args) in SIGNATURES.items():
    try:
        _f = getattr(lib, _name)
    except AttributeError as exc:
        raise ImportError("libhippymfem_b200.so lacks %s: it is older than its sources; run "
                          "`python hippymfem_b200/build.py`" % _name) from exc
    _f.restype = _res
    _f.argtypes = _args


def check(rc, what=""):
    """Raise the reference's exception type for a non-zero status."""
    if rc != HM_OK:
        msg = lib.hm_error_string(rc).decode()
        raise _EXC.get(rc, RuntimeError)("%s: %s" % (what, msg) if what else msg)


def ptr(t):
    """Device pointer of a CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("hippymfem_b200 works on CUDA tensors only (got a %s tensor)"
                         % t.device)
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return ctypes.c_void_p(t.data_ptr())


def hptr(a):
    """Host pointer of a contiguous numpy array."""
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
