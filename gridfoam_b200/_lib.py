"""ctypes binding of the gridfoam_b200 C ABI (``include/gridfoam_b200.h``).

The shared library is built in-tree by ``gridfoam_b200.csrc.build``.  There
is no CPU fallback: every operator of this package launches the library's
kernels, and loading fails loudly when the library is missing.
"""

from __future__ import annotations

import collections
import ctypes
import pathlib

import torch

LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libgridfoam_b200.so"

P = ctypes.c_void_p
I32 = ctypes.c_int32
I64 = ctypes.c_int64
F64 = ctypes.c_double

GF_OK = 0
GF_MAX_ITER = 1
GF_BREAKDOWN = 2
GF_NONFINITE = 3
GF_ERR_INVALID = 100
GF_ERR_CUDA = 101
GF_ERR_TIMEOUT = 102

BC_NONE, BC_DIRICHLET, BC_NEUMANN, BC_SLIP, BC_INLET_OUTLET, BC_FIXED_FLUX_P = range(6)

DIV_CODES = {
    "none": 0,
    "upwind": 1,
    "linear": 2,
    "vanleer": 3,
    "minmod": 4,
    "superbee": 5,
    "monotonized_central": 6,
    "limitedlinear": 7,
    "koren": 8,
}


class GfMesh(ctypes.Structure):
    _fields_ = [
        ("n_cells", I64),
        ("n_faces", I64),
        ("n_domain", I64),
        ("n_imm", I64),
        ("n_bnd", I64),
        ("ell_width", I32),
        ("reserved", I32),
        ("owner", P),
        ("neighbour", P),
        ("weight", P),
        ("mag_sf", P),
        ("delta", P),
        ("sf", P),
        ("imm_index", P),
        ("volume", P),
        ("center", P),
        ("lsq_ata_inv", P),
        ("ell_code", P),
        ("ell_nbr", P),
        ("bnd_cell", P),
        ("bnd_sf", P),
        ("bnd_mag_sf", P),
        ("bnd_d", P),
        ("bnd_mag_d", P),
        ("bnd_near", P),
        ("face_pos_owner", P),
        ("face_pos_neigh", P),
        ("n_hang", I64),
        ("hang_face", P),
        ("face_hang", P),
        ("hang_offset", P),
        ("hang_move_o", P),
        ("hang_move_n", P),
        ("face_axis", P),
        ("ell_len", P),
    ]


class GfBc(ctypes.Structure):
    _fields_ = [("ncomp", I32), ("reserved", I32), ("kind", P), ("value", P)]


class GfBcState(ctypes.Structure):
    _fields_ = [("frac", P), ("refv", P), ("refg", P), ("psib", P)]


class GfBcAux(ctypes.Structure):
    _fields_ = [
        ("phi_bnd", P),
        ("ffp_phi_pred", P),
        ("ffp_u_kind", P),
        ("ffp_u_psib", P),
        ("ffp_coeff", P),
    ]


class GfAssembly(ctypes.Structure):
    _fields_ = [
        ("ncomp", I32),
        ("div_scheme", I32),
        ("lap_harmonic", I32),
        ("use_ddt", I32),
        ("div_sign", F64),
        ("lap_sign", F64),
        ("ddt_a", F64),
        ("ddt_b", F64),
        ("ddt_c", F64),
        ("dt", F64),
        ("gamma_scalar", F64),
        ("phi", P),
        ("psi", P),
        ("grad_psi", P),
        ("psi_old", P),
        ("psi_older", P),
        ("gamma", P),
        ("bc_kind", P),
        ("frac", P),
        ("refv", P),
        ("refg", P),
        ("diag", P),
        ("val", P),
        ("source", P),
        ("lap_corrected", I32),
        ("reserved", I32),
        ("grad_lsq", P),
        ("ffc", P),
    ]


class GfKrylov(ctypes.Structure):
    _fields_ = [
        ("n", I64),
        ("width", I32),
        ("ncomp", I32),
        ("max_iter", I32),
        ("max_restart", I32),
        ("norm_inf", I32),
        ("jacobi", I32),
        ("atol", F64),
        ("rtol", F64),
        ("nbr", P),
        ("diag", P),
        ("val", P),
        ("rhs", P),
        ("x", P),
        ("work", P),
        ("work_len", I64),
        ("stats", P),
        ("mixed", I32),
        ("max_outer", I32),
        ("inner_eta", F64),
        ("stride_y", I64),
        ("stride_z", I64),
        ("symmetric", I32),
        ("block_cap", I32),
        ("variant", I32),
        ("single_reduction", I32),
        ("inner_margin", F64),
        ("spin_limit", I64),
        ("row_len", P),
    ]


class GfDdtCorr(ctypes.Structure):
    _fields_ = [
        ("rau", P),
        ("u_old", P),
        ("u_older", P),
        ("phi_old", P),
        ("phi_older", P),
        ("b", F64),
        ("c", F64),
        ("dt", F64),
    ]


_SIGNATURES = {
    "gf_last_error": ([], ctypes.c_char_p),
    "gf_version": ([], ctypes.c_int),
    "gf_krylov_workspace_size": ([I64, I32, I32], I64),
    "gf_bc_state": ([P, P, P, P, P, P], ctypes.c_int),
    "gf_lsq_grad": ([P, I32, P, P, P, P, P], ctypes.c_int),
    "gf_assemble": ([P, P, P], ctypes.c_int),
    "gf_momentum_finalize": ([P, I32, F64, P, P, P, P, P, P], ctypes.c_int),
    "gf_pressure_finalize": ([P, P, P, P, P, I64, F64, P], ctypes.c_int),
    "gf_fixed_values": ([P, I32, P, P, P, I64, P, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_spmv": ([P, I32, P, P, P, P, P], ctypes.c_int),
    "gf_pcg_solve": ([P, P], ctypes.c_int),
    "gf_pcg_solve_static": ([P, P], ctypes.c_int),
    "gf_pcg_static_scratch_doubles": ([], I64),
    "gf_bicgstab_solve": ([P, P], ctypes.c_int),
    "gf_pcg_solve_batched": ([P, I32, P, P], ctypes.c_int),
    "gf_bicgstab_solve_batched": ([P, I32, P, P], ctypes.c_int),
    "gf_batch_max_blocks": ([I32], ctypes.c_int),
    "gf_rau_hbya": ([P, I32, P, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_simplec_rAtU": ([P, P, P, P, P], ctypes.c_int),
    "gf_face_flux": ([P, I32, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_fvc_div": ([P, I32, P, P, P], ctypes.c_int),
    "gf_reconstruct": ([P, P, P, P], ctypes.c_int),
    "gf_interpolate": ([P, I32, P, P, P, P, P, P], ctypes.c_int),
    "gf_gauss_grad": ([P, I32, P, P, P], ctypes.c_int),
    "gf_sn_grad": ([P, I32, P, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_correct_phi": ([P, P, P, P, P, P, P, P, F64, I32, P, P, P, P], ctypes.c_int),
    "gf_close_fixed_flux": ([P, I64, P, P, P, P, P], ctypes.c_int),
    "gf_correct_velocity": ([P, P, P, P, P, P], ctypes.c_int),
    "gf_set_cell_values": ([I64, I32, I64, P, P, I64, P, P], ctypes.c_int),
    "gf_gather_bnd": ([I64, I32, I64, P, P, P, P], ctypes.c_int),
    "gf_adjust_phi": ([P, P, P, P], ctypes.c_int),
    "gf_relax_field": ([I64, F64, P, P, P], ctypes.c_int),
    "gf_axpby": ([I64, F64, P, F64, P, P, P], ctypes.c_int),
    "gf_ell_to_ldu": ([P, P, P, P, P], ctypes.c_int),
    "gf_ldu_to_ell": ([P, P, P, P, P], ctypes.c_int),
    "gf_field_residual": ([P, I32, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_matrix_flux": ([P, I32, P, P, P, P, P], ctypes.c_int),
    "gf_adjoint_ldu_grads": ([P, I32, P, P, P, P, P, P], ctypes.c_int),
    "gf_laplacian_adjoint": ([P, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_div_adjoint": ([P, P, P, P, P, P, P, P], ctypes.c_int),
    "gf_force_integral": ([P, I64, P, P, P, P, P, P, P, P, P, F64, F64, F64, F64, F64, P, P, P], ctypes.c_int),
    "gf_continuity_scratch_doubles": ([], I64),
    "gf_continuity_sums": ([I64, P, P, P, P, P], ctypes.c_int),
    "gf_octree_face_keys": ([P, I64, I64, I64, P, I64, I32, P, P], ctypes.c_int),
}

EXPORTED = tuple(_SIGNATURES)

_LIB: ctypes.CDLL | None = None


def load() -> ctypes.CDLL:
    """Load the library and declare every entry point (raises when absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"gridfoam_b200 CUDA library not found at {LIB_PATH}; build it with "
            "`python -m gridfoam_b200.csrc.build` (there is no CPU fallback)"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _LIB = lib
    return lib


def ptr(t: torch.Tensor | None):
    """Device pointer of a tensor (None stays NULL)."""
    if t is None:
        return None
    return ctypes.c_void_p(t.data_ptr())


def stream_ptr() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class GfError(RuntimeError):
    """A gridfoam_b200 library call failed."""


# Kernels launched per entry point (for launch accounting).
_LAUNCHES_PER_CALL = {"gf_fixed_values": 3, "gf_close_fixed_flux": 2, "gf_field_residual": 2, "gf_continuity_sums": 2,
                      "gf_pcg_solve_batched": 2, "gf_bicgstab_solve_batched": 2}
LAUNCHES: collections.Counter = collections.Counter()
# Launches known only after the device ran (the split CG's graph loop runs
# two kernels an iteration): callables giving their counts, kept while
# TRACK_DEFERRED is set (see ``launch_total``).
TRACK_DEFERRED = False
DEFERRED_LAUNCHES: list = []


def clear_launches() -> None:
    LAUNCHES.clear()
    DEFERRED_LAUNCHES.clear()


def launch_total() -> int:
    """Kernels launched since ``clear_launches`` (read after a synchronize)."""
    return sum(LAUNCHES.values()) + sum(int(f()) for f in DEFERRED_LAUNCHES)


def call(name: str, *args) -> int:
    """Call ``name`` and raise :class:`GfError` on a non-zero status."""
    lib = load()
    status = getattr(lib, name)(*args)
    LAUNCHES[name] += _LAUNCHES_PER_CALL.get(name, 1)
    if status != GF_OK:
        msg = lib.gf_last_error().decode(errors="replace")
        raise GfError(f"{name} failed with status {status}: {msg}")
    return status
