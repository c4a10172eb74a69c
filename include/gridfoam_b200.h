/*
 * gridfoam_b200 C ABI: sm_100a kernels for gridfoam's per-iteration hot path.
 *
 * The reference (ricosjp/gridfoam v0.3.0) is pure Python/PyTorch and has no
 * FFI; its drop-in boundary is its Python operator/solver API.  The entry
 * points below are what that API's operations bind to in this library.
 * Each declaration names the reference function it replaces (paths relative
 * to the reference's src/gridfoam).
 *
 * Conventions
 *  - All pointers are device pointers unless noted; sizes are element counts.
 *  - The caller owns every buffer, including workspaces; nothing allocates.
 *  - Multi-component cell arrays are component-major ("SoA"):
 *    value(c, k) = a[k * n_cells + c].  Face arrays use the extended face
 *    layout [internal faces F | boundary faces Nb]; boundary faces are
 *    ordered [domain Fb | immersed upper Fi | immersed lower Fi], i.e. the
 *    reference's packed FaceField order after the single-sided block.
 *  - Matrices are stored by rows in ELL form: diag[C] plus one coefficient
 *    per (slot, cell), val[k * C + c], the coefficient of cell nbr[k*C+c]
 *    in row c.  Slots that hold boundary faces carry a zero coefficient.
 *  - Every function enqueues work on `stream` (a cudaStream_t) and returns
 *    a status code without synchronising.  No exception crosses the ABI;
 *    gf_last_error() returns the calling thread's last error message.
 */
#ifndef GRIDFOAM_B200_H
#define GRIDFOAM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
    GF_OK = 0,
    GF_MAX_ITER = 1,      /* Krylov stopped at max_iter (not an error) */
    GF_BREAKDOWN = 2,     /* BiCGStab exhausted its restart budget */
    GF_NONFINITE = 3,     /* non-finite residual encountered */
    GF_ERR_INVALID = 100, /* invalid argument; see gf_last_error() */
    GF_ERR_CUDA = 101,    /* CUDA runtime error at launch */
    GF_ERR_TIMEOUT = 102  /* a bounded device-side wait expired */
};

/* Boundary-condition kinds, one per boundary face (boundaries/**). */
enum {
    GF_BC_NONE = 0,          /* no condition (uncovered or empty patch) */
    GF_BC_DIRICHLET = 1,     /* boundaries/basic/dirichlet.py:35-73 */
    GF_BC_NEUMANN = 2,       /* boundaries/basic/neumann.py:35-73 */
    GF_BC_SLIP = 3,          /* boundaries/basic/slip.py:40-101 */
    GF_BC_INLET_OUTLET = 4,  /* boundaries/derived/inlet_outlet.py:44-123 */
    GF_BC_FIXED_FLUX_P = 5   /* boundaries/derived/fixed_flux_pressure.py:127-252 */
};

/* Convection schemes (fv/schemes/div.py:447-456). */
enum {
    GF_DIV_NONE = 0,
    GF_DIV_UPWIND = 1,
    GF_DIV_LINEAR = 2,
    GF_DIV_VANLEER = 3,
    GF_DIV_MINMOD = 4,
    GF_DIV_SUPERBEE = 5,
    GF_DIV_MC = 6,
    GF_DIV_LIMITEDLINEAR = 7,
    GF_DIV_KOREN = 8
};

/* Mesh on the device (core/grid/axis_projected.py:97-211 plus the cached
 * fv/kernels/face_geometry.py:107-262 quantities and the ELL adjacency). */
typedef struct gf_mesh {
    int64_t n_cells;   /* C */
    int64_t n_faces;   /* F internal faces, immersed ones included */
    int64_t n_domain;  /* Fb domain-boundary faces */
    int64_t n_imm;     /* Fi immersed faces */
    int64_t n_bnd;     /* Nb = Fb + 2 Fi */
    int32_t ell_width; /* W slots per cell */
    int32_t reserved;
    /* internal faces [F] */
    const int32_t* owner;
    const int32_t* neighbour;
    const double* weight;   /* w: psi_f = w psi_O + (1-w) psi_N */
    const double* mag_sf;   /* |Sf| */
    const double* delta;    /* 1 / |d . n| */
    const double* sf;       /* Sf, [3][F] */
    const int32_t* imm_index; /* immersed ordinal or -1 */
    /* cells [C] */
    const double* volume;
    const double* center;     /* [3][C] */
    const double* lsq_ata_inv;/* [9][C], row-major 3x3 per cell */
    /* ELL adjacency [W][C]: slot code s = (face << 1) | side, face < F an
     * internal face (side 0: cell is owner), face >= F the domain face
     * face - F; -1 marks an empty slot.  nbr is the coupled cell (the cell
     * itself for boundary or empty slots).  A row's used slots come first
     * (no used slot after an empty one): the octree kernels (6 < W <= 12)
     * stop a row at its first empty slot from slot 6 on. */
    const int32_t* ell_code;
    const int32_t* ell_nbr;
    /* boundary faces [Nb] */
    const int32_t* bnd_cell;
    const double* bnd_sf;     /* outward Sf, [3][Nb] */
    const double* bnd_mag_sf;
    const double* bnd_d;      /* cell centre to boundary point, [3][Nb] */
    const double* bnd_mag_d;
    const uint8_t* bnd_near;  /* near-boundary flag (immersed faces only) */
    /* face -> ELL position of the owner / neighbour row [F] */
    const int32_t* face_pos_owner;
    const int32_t* face_pos_neigh;
    /* Hanging (coarse-fine) faces, fv/kernels/face_geometry.py:141-162: the
     * H internal faces whose centre is off the owner-neighbour segment. */
    int64_t n_hang;              /* H (0: no hanging faces, arrays unread) */
    const int32_t* hang_face;    /* [H] internal face index, ascending */
    const int32_t* face_hang;    /* [F] hanging ordinal or -1 */
    const double* hang_offset;   /* [3][H] face centre - linear-weight point */
    const double* hang_move_o;   /* [3][H] face centre - owner centre, normal part 0 */
    const double* hang_move_n;   /* [3][H] face centre - neighbour centre, normal part 0 */
    /* Axis (0, 1, 2) of every internal face [F], or NULL.  Faces of the
     * axis-projected grid are axis-aligned: sf[k][f] = 0 for k != axis, so
     * kernels given this array read and gather one component per face. */
    const int8_t* face_axis;
    /* One past the last internal-face slot of each row [C], or NULL: slots
     * from ell_len[c] on hold boundary faces or nothing (zero matrix
     * coefficients), so row products may stop there. */
    const uint8_t* ell_len;
} gf_mesh_t;

/* Per-face boundary-condition table of one field (value-fraction form). */
typedef struct gf_bc {
    int32_t ncomp;
    int32_t reserved;
    const int8_t* kind;    /* [Nb] GF_BC_* */
    const double* value;   /* [ncomp][Nb] Dirichlet value / Neumann gradient /
                              inletOutlet reverse-inflow value */
} gf_bc_t;

/* Evaluated boundary state (fv/boundary_ops.py:311-326). */
typedef struct gf_bc_state {
    double* frac;  /* [Nb] */
    double* refv;  /* [ncomp][Nb] */
    double* refg;  /* [ncomp][Nb] */
    double* psib;  /* [ncomp][Nb] */
} gf_bc_state_t;

/* Inputs some conditions read besides the field itself. */
typedef struct gf_bc_aux {
    const double* phi_bnd;      /* inletOutlet: flux on boundary faces [Nb] */
    const double* ffp_phi_pred; /* fixedFluxPressure: phiHbyA on boundary faces [Nb] */
    const int8_t* ffp_u_kind;   /* fixedFluxPressure: velocity BC kinds [Nb] */
    const double* ffp_u_psib;   /* fixedFluxPressure: velocity face values [3][Nb] */
    const double* ffp_coeff;    /* fixedFluxPressure: rAtU cell values [C] */
} gf_bc_aux_t;

/* One generic matrix assembly: ddt + div_sign * div(phi, psi)
 * + lap_sign * laplacian(gamma, psi) (fv/fvm/{ddt,div,laplacian}.py). */
typedef struct gf_assembly {
    int32_t ncomp;
    int32_t div_scheme;     /* GF_DIV_*; GF_DIV_NONE disables convection */
    int32_t lap_harmonic;   /* 1: Gauss harmonic gamma interpolation */
    int32_t use_ddt;
    double div_sign;
    double lap_sign;        /* 0 disables the Laplacian */
    double ddt_a, ddt_b, ddt_c, dt;
    double gamma_scalar;    /* used when gamma == NULL */
    const double* phi;      /* convective flux, extended face layout */
    const double* psi;      /* [ncomp][C] current field */
    const double* grad_psi; /* [ncomp*3][C] cell gradient (TVD only) */
    const double* psi_old;  /* [ncomp][C] */
    const double* psi_older;/* [ncomp][C] or NULL */
    const double* gamma;    /* [C] or NULL */
    const int8_t* bc_kind;  /* [Nb] */
    const double* frac;     /* boundary state of psi */
    const double* refv;
    const double* refg;
    double* diag;           /* out [C] */
    double* val;            /* out [W][C] */
    double* source;         /* out [ncomp][C] */
    /* Hanging faces (meshes with n_hang > 0): */
    int32_t lap_corrected;  /* 1: corrected Laplacian (explicit skewness
                               source on hanging faces, laplacian.py:162-176) */
    int32_t reserved;
    const double* grad_lsq; /* [ncomp*3][C] least-squares gradient of psi
                               for the hanging corrections of the linear
                               convection value and the Laplacian */
    double* ffc;            /* out [ncomp][F] or NULL: the Laplacian's face
                               flux correction (FvMatrix.face_flux_correction),
                               0 off hanging faces */
} gf_assembly_t;

/* Persistent Krylov solve of A x = b for ncomp right-hand sides sharing A
 * (solvers/krylov.py:34-82). */
typedef struct gf_krylov {
    int64_t n;            /* cells */
    int32_t width;        /* ELL width */
    int32_t ncomp;        /* 1..3 */
    int32_t max_iter;
    int32_t max_restart;
    int32_t norm_inf;     /* 1: L-inf stopping norm, 0: L2 */
    int32_t jacobi;       /* 1: Jacobi preconditioner, 0: identity */
    double atol, rtol;
    const int32_t* nbr;   /* [W][n] */
    const double* diag;   /* [n] */
    const double* val;    /* [W][n] */
    const double* rhs;    /* [ncomp][n] */
    double* x;            /* [ncomp][n], initial guess in, solution out */
    double* work;         /* workspace, gf_krylov_workspace_size() doubles */
    int64_t work_len;
    double* stats;        /* out [ncomp][5]: initial residual, final residual,
                             iterations, converged (0/1), status (GF_*) */
    int32_t mixed;        /* 1: FP32 inner iterations inside FP64 iterative
                             refinement (CG: one system; BiCGStab: every
                             component); 0: FP64 throughout */
    int32_t max_outer;    /* refinement cycles allowed when mixed (>= 1) */
    double inner_eta;     /* inner FP32 cycle stops at eta * |r_true| */
    int64_t stride_y;     /* > 0: the ELL is a uniform lexicographic box with
                             slots -x,+x,-y,+y,-z,+z, so neighbours are
                             c -+ 1, c -+ stride_y, c -+ stride_z (nbr unread) */
    int64_t stride_z;
    int32_t symmetric;    /* 1 (box only): A is symmetric, only + slots read */
    int32_t block_cap;    /* > 0: at most this many persistent blocks (tuning) */
    int32_t variant;      /* CG launch shape (0..31, see gf_krylov.cu and
                             solvers/autotune.py); 19..31: the split CG, two
                             plain kernels an iteration, run as a CUDA graph
                             while-loop on the stream (every permitted
                             iteration enqueued inside a stream capture, or
                             with the environment variable GF_SPLIT_GRAPH=0) */
    int32_t single_reduction; /* 1 (FP64 CG, one system): Chronopoulos-Gear
                             CG, one grid reduction per iteration; needs the
                             kind-0 workspace (7 vectors) */
    double inner_margin;  /* mixed: an FP32 cycle also ends once its residual
                             is below margin * threshold, in (0, 1]; 0: 0.5 */
    int64_t spin_limit;   /* > 0: polls after which every bounded device wait
                             (grid barrier, halo flag, copy stage) gives up and
                             the solve ends with GF_ERR_TIMEOUT; 0: the
                             default, about a second of polling */
    const uint8_t* row_len; /* [n] or NULL: row c's entries are in slots
                             0 .. row_len[c]-1 (gf_mesh_t ell_len); the
                             kernels skip the rest of the row */
} gf_krylov_t;

const char* gf_last_error(void);
int gf_version(void);

/* Number of doubles a workspace for gf_pcg_solve / gf_bicgstab_solve needs
 * (kind 0: CG, 1: BiCGStab, 2 + 100 width: mixed-precision CG, 3 + 100 width:
 * mixed-precision BiCGStab; width = ELL width). */
int64_t gf_krylov_workspace_size(int64_t n, int32_t ncomp, int32_t kind);

/* fv/boundary_ops.py:311-326 and the evaluate() methods of boundaries/**:
 * fraction, reference value/gradient and face value on every boundary face. */
int gf_bc_state(const gf_mesh_t* m, const gf_bc_t* bc, const double* psi,
                const gf_bc_aux_t* aux, gf_bc_state_t* out, void* stream);

/* fv/kernels/least_squares.py:29-101 (full-cell least-squares gradient);
 * grad is [ncomp*3][C] with value(c, k, j) = grad[(k*3 + j) * C + c]. */
int gf_lsq_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi,
                const int8_t* bc_kind, const double* psib, double* grad,
                void* stream);

/* fv/fvm/ddt.py:7-40, fv/fvm/div.py:15-73, fv/fvm/laplacian.py:101-201
 * (orthogonal part; meshes without hanging faces). */
int gf_assemble(const gf_mesh_t* m, const gf_assembly_t* a, void* stream);

/* algorithms/simple.py:306-311 (relaxation) and :316-318 (predictor source
 * b - V grad p).  relax <= 0 skips relaxation; grad may be NULL. */
int gf_momentum_finalize(const gf_mesh_t* m, int32_t ncomp, double relax,
                         const double* psi, const double* grad, double* diag,
                         double* source, double* pred_source, void* stream);

/* algorithms/utils/pressure_correction.py:121-131: source -= div(phi) V and
 * reference_value.py:33-51 (ref_cell < 0 skips). div_out receives div(phi). */
int gf_pressure_finalize(const gf_mesh_t* m, const double* phi, double* diag,
                         double* source, double* div_out, int64_t ref_cell,
                         double ref_value, void* stream);

/* core/fvmatrix.py:325-394 with_fixed_values: symmetric elimination of the
 * n_fixed prescribed cells.  fixed_mask [C] flags the cells and
 * `prescribed` [ncomp][C] holds their values (zero elsewhere); `cells` is
 * unused and may be NULL.  scratch holds >= 257 doubles. */
int gf_fixed_values(const gf_mesh_t* m, int32_t ncomp, const double* diag,
                    const double* val, const double* source, int64_t n_fixed,
                    const int32_t* cells, const double* prescribed,
                    const uint8_t* fixed_mask, double* out_diag,
                    double* out_val, double* out_source, double* scratch,
                    void* stream);

/* core/fvmatrix.py:292-323 multiply: y = A x for ncomp vectors. */
int gf_spmv(const gf_mesh_t* m, int32_t ncomp, const double* diag,
            const double* val, const double* x, double* y, void* stream);

/* solvers/cg.py:237-336: Jacobi-preconditioned CG, one persistent
 * cooperative launch for the whole solve, ncomp systems at once. */
int gf_pcg_solve(const gf_krylov_t* k, void* stream);

/* No counterpart in the reference.  Allocation-free variant of
 * gf_pcg_solve for callers that cannot allocate device memory at solve
 * time (a host framework that owns the device pool through its own caching
 * allocator, or a serving loop that must not allocate after start-up).
 * k->work and k->work_len are ignored: the scratch is a file-scope device
 * array of gf_pcg_static_scratch_doubles() doubles (14.3 MiB) that every GPU
 * loading this library holds until exit.  It fits one FP64 system of up to
 * 262,144 cells, or one FP32-inner (mixed) system of up to 229,376 cells at
 * ELL width 6 (fewer for wider rows: 166,830 at width 12).  A system fits
 * when gf_krylov_workspace_size(n, 1, kind) <= gf_pcg_static_scratch_doubles()
 * with kind 0 (FP64) or 2 + 100 * width (mixed).  Larger systems are
 * rejected with GF_ERR_INVALID.  The first
 * call on a device looks up the array's device address
 * (cudaGetSymbolAddress); make that first call before any stream capture.
 * All calls share the one array, so calls that overlap on the GPU (other
 * streams, other host threads) race; serialise them.  Results are those of
 * gf_pcg_solve. */
int gf_pcg_solve_static(const gf_krylov_t* k, void* stream);
int64_t gf_pcg_static_scratch_doubles(void);

/* solvers/bicgstab.py:76-272: right-preconditioned BiCGStab with breakdown
 * restarts, one persistent cooperative launch, ncomp systems at once. */
int gf_bicgstab_solve(const gf_krylov_t* k, void* stream);

/* Batched solves for the solve server (no counterpart in the reference,
 * which solves one case at a time, solvers/krylov.py:34-82): the systems of
 * up to 16 independent cases in ONE cooperative launch (CG: FP64 or, with
 * mixed = 1, FP32 inner iterations in FP64 refinement; BiCGStab: FP64).  System i
 * runs on blocks[i] persistent blocks of its own with its own workspace and
 * statistics, exactly as gf_pcg_solve / gf_bicgstab_solve run it on a grid
 * of blocks[i] blocks (register kernel, 256 threads a block for CG, 512 for
 * BiCGStab), so its result does not depend on the other systems in the
 * batch.  The block counts must fit on the device at once
 * (gf_batch_max_blocks); CG systems have ncomp 1, BiCGStab systems share
 * one ncomp.  Two launches: a reset of the control blocks, then the solves. */
int gf_pcg_solve_batched(const gf_krylov_t* systems, int32_t count,
                         const int32_t* blocks, void* stream);
int gf_bicgstab_solve_batched(const gf_krylov_t* systems, int32_t count,
                              const int32_t* blocks, void* stream);
/* Co-resident blocks of the batched CG (bicgstab 0) or BiCGStab (1) kernel
 * on the current device, or -1. */
int gf_batch_max_blocks(int32_t bicgstab);

/* core/fvmatrix.py:242-290 and algorithms/simple.py:336-337:
 * rAU = 1 / (diag / V), HbyA = rAU * H(psi); h1 (may be NULL) receives
 * H1() (fvmatrix.py:250-264). */
int gf_rau_hbya(const gf_mesh_t* m, int32_t ncomp, const double* diag,
                const double* val, const double* source, const double* psi,
                double* rau, double* hbya, double* h1, void* stream);

/* algorithms/utils/pressure_correction.py:163-194 (bounded SIMPLEC rAtU). */
int gf_simplec_rAtU(const gf_mesh_t* m, const double* rau, const double* h1,
                    double* ratu, void* stream);

/* fv/flux.py:32-129: face flux of a velocity-like cell field on every face.
 * mode 0 (correct_flux with internal update): boundary faces take the
 * velocity BC face value.  mode 1 (compute_phi_hbya): boundary faces take
 * vel_P.Sf, U_b.Sf on non-assignable velocity patches, 0 on uncovered domain
 * faces.  ddt (optional, PISO/PIMPLE): adds interpolate(rAU) * ddtCorr
 * (fv/fvc/ddt_corr.py:13-78) on single-sided faces.  grad_vel ([9][C]
 * least-squares gradient of vel, or NULL) adds the hanging-face offset
 * correction of the interpolated velocity before the dot with Sf. */
typedef struct gf_ddtcorr {
    const double* rau;        /* [C] */
    const double* u_old;      /* [3][C] */
    const double* u_older;    /* [3][C] or NULL */
    const double* phi_old;    /* [F] */
    const double* phi_older;  /* [F] or NULL */
    double b, c, dt;
} gf_ddtcorr_t;

int gf_face_flux(const gf_mesh_t* m, int32_t mode, const double* vel,
                 const int8_t* u_kind, const double* u_psib,
                 const gf_ddtcorr_t* ddt, const double* grad_vel, double* phi,
                 void* stream);

/* fv/fvc/reconstruct.py:28-117: cell velocity U [3][C] from the face flux
 * phi (extended layout [F | Nb]): (sum |Sf| n n^T)^-1 sum n phi over every
 * face of the cell. */
int gf_reconstruct(const gf_mesh_t* m, const double* phi, double* U, void* stream);

/* fv/fvc/div.py:15-64: div(phi) = face sum / V for ncomp face fields. */
int gf_fvc_div(const gf_mesh_t* m, int32_t ncomp, const double* phi,
               double* out, void* stream);

/* fv/schemes/interpolate.py:20-63 + fv/boundary_ops.py:545-593: linear face
 * values and boundary face values (BC value or zero-gradient fill).  grad
 * ([ncomp*3][C] least-squares gradient, or NULL) adds the hanging-face
 * offset correction (fv/kernels/face_interpolation.py:45-96). */
int gf_interpolate(const gf_mesh_t* m, int32_t ncomp, const double* psi,
                   const int8_t* bc_kind, const double* psib,
                   const double* grad, double* out, void* stream);

/* fv/kernels/gauss_gradient.py:15-73 and fv/schemes/grad.py:21-43 (the
 * 'linear' gradient scheme): Green-Gauss gradient of ncomp face fields
 * psi_f ([ncomp][F + Nb], as gf_interpolate writes them); grad is
 * [ncomp*3][C] with value(c, k, j) = grad[(k*3 + j) * C + c]. */
int gf_gauss_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi_f,
                  double* grad, void* stream);

/* fv/fvc/sn_grad.py:16-55 (internal part + boundary normal gradient,
 * boundary_ops.py:405-437).  grad ([ncomp*3][C] least-squares gradient, or
 * NULL for the uncorrected scheme) adds the hanging-face correction
 * (fv/kernels/face_interpolation.py:99-145). */
int gf_sn_grad(const gf_mesh_t* m, int32_t ncomp, const double* psi,
               const int8_t* bc_kind, const double* frac, const double* refv,
               const double* refg, const double* grad, double* out,
               void* stream);

/* algorithms/utils/pressure_correction.py:270-305 correct_phi without the
 * fixed-cell closure: phi = phiHbyA - flux(p) on single faces (flux(p)
 * includes ffc, the pressure Laplacian's hanging-face flux correction, when
 * not NULL), boundary faces phiHbyA_b + sign coeff_P |Sf| snGrad_b(p).
 * simplec = 1: the SIMPLEC flux update (pressure_correction.py:257-264),
 * phiHbyA += interpolate(coeff) snGrad(p) |Sf| with sign +1, coeff =
 * rAtU - rAU, and snGrad corrected on hanging faces by grad_p (the
 * least-squares gradient of p, or NULL). */
int gf_correct_phi(const gf_mesh_t* m, const double* phi_pred,
                   const double* coeff, const double* p, const int8_t* p_kind,
                   const double* frac, const double* refv, const double* refg,
                   double sign, int32_t simplec, const double* grad_p,
                   const double* ffc, double* phi, void* stream);

/* pressure_correction.py:308-335 fixed-cell flux closure. face_list holds
 * the n_faces boundary faces flagged fixed; area_frac their area share;
 * scratch holds >= n_faces doubles. */
int gf_close_fixed_flux(const gf_mesh_t* m, int64_t n_faces,
                        const int32_t* face_list, const double* area_frac,
                        double* phi, double* scratch, void* stream);

/* pressure_correction.py:338-363: out = base - coeff * grad (ncomp=3). */
int gf_correct_velocity(const gf_mesh_t* m, const double* base,
                        const double* coeff, const double* grad, double* out,
                        void* stream);

/* fv/boundary_ops.py:538-542: out[cells[i], k] = values[k][i]. */
int gf_set_cell_values(int64_t n_cells, int32_t ncomp, int64_t n_set,
                       const int32_t* cells, const double* values,
                       int64_t values_stride, double* out, void* stream);

/* Gather prescribed values: values[k][i] = refv[k][faces[i]]. */
int gf_gather_bnd(int64_t n_bnd, int32_t ncomp, int64_t n, const int32_t* faces,
                  const double* refv, double* values, void* stream);

/* fv/adjust_phi.py:44-127: class[b] = 0 skip, 1 fixed-value, 2 adjustable,
 * per domain face.  Runs on the device without a host round trip. */
int gf_adjust_phi(const gf_mesh_t* m, const int8_t* face_class, double* phi,
                  void* stream);

/* algorithms/simple.py:386: p = p_old + alpha (p - p_old). */
int gf_relax_field(int64_t n, double alpha, const double* old, double* cur,
                   void* stream);

/* out = a x + b y elementwise (matrix algebra of core/fvmatrix.py:181-211). */
int gf_axpby(int64_t n, double a, const double* x, double b, const double* y,
             double* out, void* stream);

/* LDU <-> ELL conversions for the FvMatrix.upper/lower API. */
int gf_ell_to_ldu(const gf_mesh_t* m, const double* val, double* upper,
                  double* lower, void* stream);
int gf_ldu_to_ell(const gf_mesh_t* m, const double* upper, const double* lower,
                  double* val, void* stream);

/* algorithms/utils/residual.py:12-36: |A psi - b|_2 / (|b|_2 + eps), summed
 * over components; written to out[0]. scratch holds >= 512 doubles. */
int gf_field_residual(const gf_mesh_t* m, int32_t ncomp, const double* diag,
                      const double* val, const double* source,
                      const double* psi, double* scratch, double* out,
                      void* stream);

/* fvmatrix.py:424-468 flux on all internal faces (0 on immersed ones):
 * out[f] = upper psi_N - lower psi_O (+ ffc[f] when ffc is not NULL). */
int gf_matrix_flux(const gf_mesh_t* m, int32_t ncomp, const double* val,
                   const double* psi, const double* ffc, double* out,
                   void* stream);

/* ---- Adjoint (reverse-mode) kernels ---------------------------------- */

/* solvers/adjoint/ldu_grads.py:11-53: for x = A^-1 b and lambda = A^-T xbar
 * (both [ncomp][C]): grad_diag[c] = -sum_k lambda_kc x_kc,
 * grad_upper[f] = -sum_k lambda_kO x_kN, grad_lower[f] = -sum_k lambda_kN
 * x_kO over all F internal faces; the source gradient is lambda itself. */
int gf_adjoint_ldu_grads(const gf_mesh_t* m, int32_t ncomp, const double* lambda,
                         const double* x, double* grad_diag, double* grad_upper,
                         double* grad_lower, void* stream);

/* Reverse of fvm.laplacian(gamma, psi) (fv/fvm/laplacian.py:101-201, the
 * assembly described by `a` with lap_sign 1, linear gamma interpolation):
 * given the cotangents of diag [C], upper/lower [F] and source [ncomp][C],
 * writes the gradient with respect to the per-cell diffusivity, g_gamma [C].
 * Includes the hanging-face skewness source when a->lap_corrected. */
int gf_laplacian_adjoint(const gf_mesh_t* m, const gf_assembly_t* a,
                         const double* g_diag, const double* g_upper,
                         const double* g_lower, const double* g_source,
                         double* g_gamma, void* stream);

/* Reverse of fvm.div(phi, psi) (fv/fvm/div.py:15-73 with the scheme in `a`):
 * the transpose of the face-flux -> coefficient map.  Writes g_phi over the
 * extended face layout [F internal | Nb boundary]. */
int gf_div_adjoint(const gf_mesh_t* m, const gf_assembly_t* a,
                   const double* g_diag, const double* g_upper,
                   const double* g_lower, const double* g_source,
                   double* g_phi, void* stream);

/* ---- Post-processing -------------------------------------------------- */

/* post/forces/sampling.py:69-168 + integration.py:76-187: force on an
 * immersed patch from its n axis-projected boundary samples (faces: boundary
 * face indices, upper and lower sides).  anchor_normal [3][n_imm] is the
 * body-outward surface normal per anchor (immersed face); a sample is kept
 * when its outward direction points into the body.  Writes per-sample rows
 * samples[12][n] (pressure force xyz, viscous force xyz, force xyz, moment
 * about (cx, cy, cz) xyz; zero for dropped samples) and total[6] (force,
 * moment), summed in a fixed order.  nu_eff [C] or NULL for nu_scalar. */
int gf_force_integral(const gf_mesh_t* m, int64_t n, const int32_t* faces,
                      const double* anchor_normal, const int8_t* p_kind,
                      const gf_bc_state_t* p_state, const double* p,
                      const int8_t* u_kind, const gf_bc_state_t* u_state,
                      const double* U, const double* nu_eff, double nu_scalar,
                      double rho, double cx, double cy, double cz,
                      double* samples, double* total, void* stream);

/* post/diagnostics/continuity.py:11-49 (the sums of compute_continuity_error,
 * without its host round trip): from div = fvc.div(phi) [n] and the cell
 * volumes [n], out[0] = sum |div| V, out[1] = sum div V, out[2] = sum V, each
 * summed in a fixed order (the same bits on every launch).  scratch holds
 * gf_continuity_scratch_doubles() doubles.  The caller forms
 * local = dt out[0] / out[2] and global = dt out[1] / out[2]. */
int64_t gf_continuity_scratch_doubles(void);
int gf_continuity_sums(int64_t n, const double* div, const double* vol,
                       double* scratch, double* out, void* stream);

/* No counterpart in the reference, which takes its mesh from the external
 * fluxel package (core/grid/factory.py:32-65; hanging-face contract
 * core/grid/axis_projected.py:715-767).  Internal faces of a 2:1-balanced
 * octree along `axis` (0..2): ids [fx][fy][fz] (C order) is the leaf covering
 * each finest-level cell, corner [3][n_cells] the leaves' finest-level lower
 * corners.  keys gets one entry per face position of the [fx - (axis == 0)]
 * [fy - (axis == 1)][fz - (axis == 2)] lower cells: owner * n_cells +
 * neighbour at the one position that emits each leaf pair (the corner of
 * their shared rectangle with the smallest tangential coordinates), -1
 * elsewhere, -2 where an id lies outside [0, n_cells).  Sorting the
 * non-negative keys gives the faces in (owner, neighbour) order. */
int gf_octree_face_keys(const int64_t* ids, int64_t fx, int64_t fy, int64_t fz,
                        const int64_t* corner, int64_t n_cells, int32_t axis,
                        int64_t* keys, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRIDFOAM_B200_H */
