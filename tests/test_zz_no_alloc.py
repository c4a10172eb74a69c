"""The allocation-free CG entry point gives the same solve as gf_pcg_solve.

Callers that cannot allocate device memory at solve time (a host framework
that owns the device pool, or a serving loop that must not allocate after
start-up) use gf_pcg_solve_static, whose scratch is a fixed device array
inside the library.  This file is collected last so that a failing run that
stops at the first failure has already run every other test.
"""

from __future__ import annotations

import ctypes

import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _system(n: int, nz: int):
    from gridfoam_b200.fv import fvm
    from tests.golden.cases import pipe_case
    from tests.golden.device_harness import device_case

    _, _, grid, algo = device_case(case_def=pipe_case(n, nz))
    gamma = torch.linspace(0.2, 0.5, grid.num_cells, dtype=torch.float64, device="cuda")
    A = -fvm.laplacian(gamma, algo.p)
    gen = torch.Generator(device="cpu").manual_seed(5)
    rhs = torch.randn((1, grid.num_cells), generator=gen, dtype=torch.float64).cuda()
    return grid, A, rhs


def _descriptor(grid, A, rhs, x, stats, variant, mixed, work=None):
    from gridfoam_b200 import _lib

    k = _lib.GfKrylov()
    k.n = grid.num_cells
    k.width = grid.ell_width
    k.ncomp = 1
    k.max_iter = 5000
    k.max_restart = 5
    k.norm_inf = 0
    k.jacobi = 1
    k.atol = 1e-10
    k.rtol = 0.0
    k.nbr = _lib.ptr(grid.dev["ell_nbr"])
    k.diag = _lib.ptr(A.diag_store)
    k.val = _lib.ptr(A.val)
    k.rhs = _lib.ptr(rhs)
    k.x = _lib.ptr(x)
    k.stats = _lib.ptr(stats)
    if work is not None:
        k.work = _lib.ptr(work)
        k.work_len = work.numel()
    k.variant = variant
    k.mixed = mixed
    k.max_outer = 20 if mixed else 1
    k.inner_eta = 1e-4
    return k


# (CG launch shape, FP32 inner iterations): the register kernel, and the
# single-reduction halo kernels of the FP64 and the FP32-inner solve, whose
# halo flags live in the scratch and must be reset by every call.
SHAPES = [(0, 0), (10, 0), (10, 1)]


@pytest.mark.parametrize("variant,mixed", SHAPES, ids=["v0-fp64", "v10-fp64", "v10-fp32inner"])
def test_static_scratch_matches_workspace_solve(variant, mixed):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    from gridfoam_b200 import _lib

    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    # Two systems of different sizes (both >= 16,384 cells, where the
    # FP32-inner halo kernel applies), solved with a sized workspace first.
    systems = [_system(24, 48), _system(20, 44)]
    refs = []
    for grid, A, rhs in systems:
        n = grid.num_cells
        kind = 2 + 100 * grid.ell_width if mixed else 0
        assert lib.gf_krylov_workspace_size(n, 1, kind) <= lib.gf_pcg_static_scratch_doubles()
        work = torch.empty(lib.gf_krylov_workspace_size(n, 1, kind), dtype=torch.float64, device="cuda")
        x_ref = torch.zeros_like(rhs)
        st_ref = torch.zeros((1, 5), dtype=torch.float64, device="cuda")
        _lib.call("gf_pcg_solve", ctypes.byref(_descriptor(grid, A, rhs, x_ref, st_ref, variant, mixed, work)),
                  stream)
        torch.cuda.synchronize()
        assert int(st_ref[0, 3]) == 1
        refs.append((x_ref, st_ref))

    # Calls in a row on the one shared array, alternating sizes.
    for i in (0, 1, 0, 1):
        grid, A, rhs = systems[i]
        x_ref, st_ref = refs[i]
        x = torch.zeros_like(rhs)
        st = torch.zeros((1, 5), dtype=torch.float64, device="cuda")
        _lib.call("gf_pcg_solve_static", ctypes.byref(_descriptor(grid, A, rhs, x, st, variant, mixed)), stream)
        torch.cuda.synchronize()
        assert int(st[0, 2]) == int(st_ref[0, 2]) and int(st[0, 3]) == 1
        torch.testing.assert_close(x, x_ref, rtol=1e-12, atol=1e-14)
        torch.testing.assert_close(st, st_ref, rtol=1e-12, atol=0.0)


def test_static_scratch_rejects_oversized_systems():
    """The size check runs on the host before anything is launched."""
    from gridfoam_b200 import _lib

    lib = _lib.load()
    k = _lib.GfKrylov()
    k.n = 10_000_000
    k.width = 6
    k.ncomp = 1
    status = lib.gf_pcg_solve_static(ctypes.byref(k), None)
    assert status == _lib.GF_ERR_INVALID
    assert b"static scratch" in lib.gf_last_error()
