"""The allocation-free residual entry point against the allocating one.  GPU.

Some callers of this library cannot allocate device memory at the moment they need a
residual or a gradient: their process's GPU memory is already held by another runtime's
pool (JAX/XLA claims most of the device at start-up by default, MFEM/hypre may sit on an
Umpire pool), or they run a loop that must not pay for an allocation.
``hm_lattice_residual_noalloc`` serves them: its one scratch buffer is a fixed device
array inside the library, so it works for lattices of at most 8192 elements.

The test calls it through the C ABI twice in a row, with different inputs each time, so
that anything the first call left in the shared scratch would show in the second, and
compares every result with ``hm_lattice_quadrature`` + ``hm_lattice_assemble``, the
entry points that take a workspace from the caller.  The file is named to be collected
last: if it fails, a run that stops at the first failure has run everything else.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12      # relative, as the other FP64 parity tests


def _allocating(mesh, U, M, P, marker, f):
    from hippymfem_b200 import _lib
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    dev = U.device
    quad = torch.empty(mesh.quad_bytes() // 8, dtype=torch.float64, device=dev)
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    out = [torch.empty(mesh.ndof, dtype=torch.float64, device=dev) for _ in range(3)]
    check(lib.hm_lattice_quadrature(mesh.handle, ptr(U), ptr(M), ptr(P), _lib.HM_FP64,
                                    ptr(quad), ptr(status), stream_ptr()))
    check(lib.hm_lattice_assemble(mesh.handle, ptr(quad), _lib.HM_FP64, None, ptr(marker),
                                  float(f), None, None, None, None, ptr(out[0]), ptr(out[1]),
                                  ptr(out[2]), 1, stream_ptr()))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    return [o.cpu().numpy() for o in out]


def _noalloc_call(mesh, U, M, P, f, marker, out, status):
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    check(lib.hm_lattice_residual_noalloc(mesh.handle, ptr(U), ptr(M), ptr(P), f,
                                          ptr(marker), ptr(out[0]), ptr(out[1]),
                                          ptr(out[2]), 1, ptr(status), stream_ptr()),
          "hm_lattice_residual_noalloc")


@pytest.mark.parametrize("n,L", [((6, 5, 7), (1.0, 0.8, 1.2)),
                                 ((16, 16, 32), (1.0, 1.0, 2.0))])   # exactly 8192 elements
def test_noalloc_residual_matches_the_allocating_path_twice(cuda, n, L):
    from hippymfem_b200 import BoxMesh, DirichletBC, Q2Space

    mesh = BoxMesh(n, L=L)
    assert mesh.ne <= 8192
    marker = DirichletBC(Q2Space(mesh)).marker
    nd = mesh.ndof
    for seed, f in ((1, 1.0), (2, -0.5)):
        rng = np.random.default_rng(seed)
        U, M, P = (torch.as_tensor(rng.standard_normal(nd) * s, device=cuda)
                   for s in (1.0, 0.3, 1.0))
        out = [torch.full((nd,), float("nan"), dtype=torch.float64, device=cuda)
               for _ in range(3)]
        status = torch.zeros(1, dtype=torch.int32, device=cuda)
        _noalloc_call(mesh, U, M, P, f, marker, out, status)
        torch.cuda.synchronize()
        assert int(status.item()) == 0
        ref = _allocating(mesh, U, M, P, marker, f)
        for got, want in zip(out, ref):
            got = got.cpu().numpy()
            assert np.isfinite(got).all()
            assert np.abs(got - want).max() <= TOL * np.abs(want).max()


def test_noalloc_call_takes_no_device_memory(cuda):
    """Once the library's code and its fixed array are resident (a first call), a call
    changes neither the device's free memory nor torch's allocations."""
    from hippymfem_b200 import BoxMesh

    mesh = BoxMesh((10, 9, 8))
    nd = mesh.ndof
    rng = np.random.default_rng(3)
    U, M, P = (torch.as_tensor(rng.standard_normal(nd), device=cuda) for _ in range(3))
    M = 0.2 * M
    out = [torch.empty(nd, dtype=torch.float64, device=cuda) for _ in range(3)]
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    _noalloc_call(mesh, U, M, P, 1.0, None, out, status)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(3):
        _noalloc_call(mesh, U, M, P, 1.0, None, out, status)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
    assert int(status.item()) == 0


def test_noalloc_rejects_a_lattice_beyond_its_scratch(cuda):
    from hippymfem_b200 import BoxMesh
    from hippymfem_b200._lib import check, lib, ptr, stream_ptr

    mesh = BoxMesh((21, 20, 20))                       # 8400 elements > 8192
    z = torch.zeros(mesh.ndof, dtype=torch.float64, device=cuda)
    out = torch.empty_like(z)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    with pytest.raises(MemoryError):
        check(lib.hm_lattice_residual_noalloc(mesh.handle, ptr(z), ptr(z), ptr(z), 1.0, None,
                                              None, ptr(out), None, 0, ptr(status),
                                              stream_ptr()), "hm_lattice_residual_noalloc")
