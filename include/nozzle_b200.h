/*
 * nozzle_b200.h -- C ABI of the B200 nodal-DG backend for the 2D Euler nozzle.
 *
 * Every entry point takes plain pointers and sizes.  Device arrays are owned
 * by the caller (the Python backend allocates them as torch tensors); the
 * library never allocates, frees or retains device memory except inside a
 * solver object, which only records the caller's pointers.  Every function
 * returns 0 on success and a negative code on failure, with a message from
 * nzb_last_error().  Numerical failure (NaN, overflow) is not an error: it
 * propagates into the returned residual, as in the reference solver.
 *
 * Device layouts ("SoA"): a state is (4, NP, E) doubles -- component s, node i,
 * element e at [(s * NP + i) * E + e] -- so a warp reading one (s, i) plane
 * reads 32 consecutive elements.  The reference's (E, NP, 4) layout is
 * converted by nzb_pack_state / nzb_unpack_state.
 *
 * Reference interfaces replaced (reference repository paths):
 *   nzb_residual (op RESIDUAL)   Backend.residual          src/backends/base.py:118-120,
 *                                 assembly.residual         src/spatial/assembly.py:153-157
 *   nzb_residual (op RATE)       NumbaBackend._rate_into    src/backends/numba_backend.py:213-234,
 *                                 _numba_kernels.element_rate src/backends/_numba_kernels.py:586-664
 *   nzb_inverse_mass             Backend.inverse_mass      src/backends/base.py:122-124
 *   nzb_limit                    Backend.limit / positivity_limit
 *                                 src/backends/numba_backend.py:247-281,
 *                                 src/backends/_numba_kernels.py:927-1093
 *   nzb_stage                    stage / combine_ssp / local_dt / rms_weighted fused
 *                                 src/backends/_numba_kernels.py:789-850
 *   nzb_norm                     Backend.norm              src/backends/numba_backend.py:178-181
 *   nzb_solver_*                 NumbaBackend.run          src/backends/numba_backend.py:283-337
 *   nzb_vjp, nzb_adjoint_*       jax.vjp of assembly.residual and the RK4 march of
 *                                 DifferentiableCase.adjoint_solve src/sensitivity.py:289-383
 *   nzb_vjp_coords               jax.vjp of the residual w.r.t. the design variables
 *                                 through the node coordinates     src/sensitivity.py:453-458
 *   nzb_observables              boundary_trace, axial_momentum_flux, mass_flux, entropy_error
 *                                 and the exit averages of performance()
 *                                                                  src/post/postprocess.py:56-255
 *   nzb_geometry                 the coordinate-dependent part of build_operators
 *                                                                  src/spatial/operators.py:240-303
 *   nzb_gen_geometry             the same for any order and geometry order, in the
 *                                 reference's per-element layout   src/spatial/operators.py:209-342
 *   nzb_initial_state,           initial_state(..., "quasi1d")     src/timestepping/initialize.py:41-102
 *   nzb_gen_initial_state
 *   nzb_gen_observables          the integrals of performance() on the generic path
 */
#ifndef NOZZLE_B200_H
#define NOZZLE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Element kinds and the flux / boundary codes used in the arrays below. */
enum { NZB_TRI = 0, NZB_QUAD = 1 };
enum { NZB_ROE = 0, NZB_HLLC = 1, NZB_AUSMUP = 2 };
enum { NZB_INFLOW = 1, NZB_OUTFLOW = 2, NZB_WALL = 3, NZB_AXIS = 4 };
enum { NZB_OP_RESIDUAL = 0, NZB_OP_RATE = 1 };

/* Mesh and operators of one mesh, all device pointers, all owned by the caller.
 *
 * affine = 1: straight-sided triangles; geo holds (5, E) = xi_x, xi_y, eta_x,
 *             eta_y, det and the volume / mass operators come from the
 *             reference-element tables uploaded by nzb_upload_tables.
 * affine = 0: any straight-sided element (bilinear quadrilaterals): geo holds
 *             (2*NV, E) = the NV vertex x then y coordinates, from which the
 *             kernels rebuild the Jacobian at every volume point; minv holds
 *             (NP*NP, E) the inverse mass matrices.
 * face_nbr  (NF, E): element across face f, or -1 on a boundary.
 * face_code (NF, E): side (bit 0: 0 owner, 1 neighbour) | neighbour's local
 *             face << 1 | boundary tag << 4.
 * face_edge (NF, E): global edge id.
 * edge_geo  (n_edge, 4): nx, ny (owner's outward unit normal), |dX/dsigma|,
 *             edge length.  Edges are straight: one normal per edge.
 * Batches of independent instances share one mesh descriptor: their elements
 * are concatenated (connectivity offset accordingly) and
 * elem_inst   (E)      instance of each element (null: a single instance),
 * inst_status (n_inst) nonzero = retired: its elements are left untouched,
 * inst_p_back (n_inst) back pressure of each instance (null: phys.p_back).
 * The Superbee slope limiter (physics limiter 2) needs each instance's
 * domain-wide maximum of the cell averages: stages and nzb_limit then run
 * three passes after the element kernel -- cell averages, their maximum per
 * instance (lim_scale holds 4 per instance: n_inst of them with elem_inst, one
 * without), the slope limiter with the positivity limiter -- and count an
 * element as scaled when either limiter changed it.  elem_share is each
 * element's area over its own instance's domain area.
 * edge_pass = 1 splits every residual / stage into two launches: one thread
 * per edge evaluates each edge's fluxes once (the reference's edge_pass), then
 * the element kernel lifts them; edge_pass = 0 evaluates the fluxes inside the
 * element kernel, from both sides.  Both evaluate the same formulas and agree
 * to round-off (the compiler may contract multiply-adds differently); which is
 * faster depends on the element kind, order and mesh size.
 * split = 4 (orders >= 1) runs the element kernel with four threads per
 * element -- faces and volume points split over a block's four warps, the
 * projection by component, the limiter's probe points split -- and ignores
 * edge_pass; split = 0 or 1 runs one thread per element.  It agrees with the
 * one-thread kernels to round-off (a few sums associate differently).
 * vjp_split = 4 (orders >= 1) runs the adjoint state kernel the same way:
 * faces and volume points split over four warps, each warp gathering one
 * component of every node in the one-thread kernel's order; it agrees with
 * the one-thread kernel to round-off.
 */
typedef struct {
  int32_t kind;
  int32_t order;
  int32_t affine;
  int32_t edge_pass; /* 1: face fluxes in a separate edge pass (needs edge_conn, edge_flux, edge_speed) */
  int64_t n_elem;
  int64_t n_edge;
  const double* geo;
  const double* minv;
  const double* area;
  const int32_t* face_nbr;
  const int32_t* face_code;
  const int32_t* face_edge;
  const double* edge_geo;
  const int32_t* elem_inst;
  const int32_t* inst_status;
  const double* inst_p_back;
  const int32_t* edge_conn; /* (3, n_edge): owner element, neighbour (-1: boundary),
                               owner face | neighbour face << 3 | boundary tag << 6 */
  double* edge_flux;        /* (n_edge, NQF, 4) scratch of the edge pass, 16-byte aligned */
  double* edge_speed;       /* (n_edge) scratch of the edge pass */
  const double* elem_share; /* (E) A_e / A_domain, for the Superbee limiter (limiter 2) */
  double* lim_means;        /* (4, E) scratch of the Superbee limiter */
  double* lim_scale;        /* (4 * max(1, n_inst)) scratch of the Superbee limiter */
  int32_t split;            /* threads per element of the forward kernels: 0 or 1, or 4 */
  int32_t n_inst;           /* instances of a batch (elem_inst values lie in [0, n_inst)); 0 or 1: one */
  int32_t vjp_split;        /* threads per element of the adjoint state kernel (nzb_vjp, nzb_adjoint_*): 0 or 1, or 4 */
  int32_t reserved;
  /* Optional block lists (null: every block).  The forward element kernel
   * (residuals, rates, stages, nzb_limit's positivity pass) and the adjoint
   * state kernel (nzb_vjp, nzb_adjoint_*) then run only the listed blocks:
   * block b holds elements [b W, (b + 1) W), W = nzb_block_width(mesh, 0) for
   * the forward kernel and nzb_block_width(mesh, 1) for the adjoint one.  An
   * element of an unlisted block is left as an element of a retired instance
   * is: a batch lists the blocks that hold elements of instances still
   * marching, so a launch late in a march no longer spans every retired block.
   * Entries outside [0, ceil(n_elem / W)) are skipped; the edge pass, the
   * Superbee passes and every other kernel ignore the lists; block-partial norms (norm_partial) are
   * refused with a list, since unlisted blocks would leave stale partials. */
  const int32_t* fwd_blocks;
  int64_t n_fwd_blocks;
  const int32_t* vjp_blocks;
  int64_t n_vjp_blocks;
} nzb_mesh;

/* Gas, operating point and limiter constants, evaluated on the host exactly
 * as the reference evaluates them (src/config.py, src/physics/boundary.py). */
typedef struct {
  double gamma;
  double entropy_fix;
  double hllc_low_mach;
  int32_t flux;
  int32_t limiter;        /* 0 none, 1 positivity, 2 Superbee TVB then positivity (ignored at p = 0) */
  /* inflow: cos/sin of the inflow angle, a_t^2 = gamma R T_t, a_t, rho_t */
  double in_cos, in_sin, in_at2, in_at, in_rho_t;
  /* outflow: back pressure, backflow reservoir density (0 = off), p_t, band */
  double p_back, bf_rho_t, bf_p_t, bf_band;
  /* positivity limiter */
  double lim_fraction, rho_floor, p_floor, lebesgue;
  int32_t lim_steps;
  int32_t reserved;
  /* residual-norm component weights (1, 1/a_t, 1/a_t, 1/a_t^2) */
  double norm_w[4];
  double tvb_constant; /* Superbee's TVB constant (limiter 2) */
} nzb_physics;

/* Tables of one reference element: see the packer in layout.py for the order.
 * Must be called once per device and (kind, order) before any other call on
 * that kind and order.  Host pointer. */
int nzb_upload_tables(int kind, int order, const double* tables, int64_t n);
/* Number of doubles nzb_upload_tables expects for (kind, order). */
int64_t nzb_table_size(int kind, int order);

/* Reference (E, NP, 4) <-> device (4, NP, E).  perm (nullable) maps device
 * element index -> reference element index. */
int nzb_pack_state(const double* src_aos, double* dst_soa, int64_t n_elem, int np,
                   const int32_t* perm, void* stream);
int nzb_unpack_state(const double* src_soa, double* dst_aos, int64_t n_elem, int np,
                     const int32_t* perm, void* stream);

/* op RESIDUAL: out = R(U) with M dU/dt = -R.  op RATE: out = -M^-1 R(U).
 * wave (nullable) receives sum_f s_f l_f per element. */
int nzb_residual(const nzb_mesh* mesh, const nzb_physics* phys, int op, const double* U,
                 double* out, double* wave, void* stream);

/* out = M^-1 R. */
int nzb_inverse_mass(const nzb_mesh* mesh, const double* R, double* out, void* stream);

/* Positivity limiter in place.  counters (nullable, device, 2 x uint64)
 * accumulate (scaled, repaired); flags (nullable, device, E bytes) receive
 * bit 0 = scaled, bit 1 = cell mean repaired. */
int nzb_limit(const nzb_mesh* mesh, const nzb_physics* phys, double* U,
              unsigned long long* counters, uint8_t* flags, void* stream);

/* One fused explicit stage:
 *   stage 1: dt_e = dt_factor * 2 A_e / max(wave_e, 1e-10) (written to dt),
 *            out = limit(V + dt F(V)),  norm_partial[block] = sum (w F)^2
 *   stage 2: out = limit(a U0 + b (V + dt F(V)))   (dt read)
 * out may alias U0 (each element reads only its own U0) but not V.
 * norm_partial, counters, flags are nullable.  norm_partial needs
 * nzb_norm_blocks(E) doubles. */
typedef struct {
  const double* V;
  const double* U0;
  double* out;
  double* dt;
  double* norm_partial;
  double* elem_norm; /* (E, nullable): per-element sum (w F)^2 of stage 1, for batches */
  unsigned long long* counters;
  uint8_t* flags;
  double dt_factor;
  double a;
  double b;
  int32_t stage;
  int32_t reserved;
} nzb_stage_args;
int nzb_stage(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_stage_args* args, void* stream);

/* Upper bound on the partial-sum slots any kernel here writes for n_elem
 * elements (size norm_partial buffers with it). */
int64_t nzb_norm_blocks(int64_t n_elem);
/* Blocks (= partial-sum slots written by stage 1) of the element kernel. */
int64_t nzb_element_blocks(const nzb_mesh* mesh);
/* Elements per block W of the forward element kernel (which = 0) or of the
 * adjoint state kernel (which = 1) for the mesh's variant (split, vjp_split):
 * the unit of the fwd_blocks / vjp_blocks lists.  -1 for a bad argument. */
int64_t nzb_block_width(const nzb_mesh* mesh, int which);
/* out[0] = sqrt(sum partial[0..n_partial) / count) -- fixed summation order. */
int nzb_norm_finalize(const double* partial, int64_t n_partial, double count, double* out, void* stream);
/* Weighted RMS of a (4, NP, E) array: out[0] = sqrt(mean((w_s A)^2)).
 * partial needs nzb_norm_blocks(E) doubles of scratch. */
int nzb_norm(const double* A, int64_t n_elem, int np, const double* w4, double* partial, double* out,
             void* stream);

/* nzb_norm without a scratch argument, for callers that cannot allocate
 * device memory: a host application that passes this library only buffers
 * from a fixed pool it manages itself, or a loop that must never enter the
 * CUDA allocator (cudaFree, for one, synchronizes the whole device).  It has
 * no counterpart in the reference solver.
 *
 * The per-block partial sums go to a fixed array in the library's device
 * memory (512 KiB on every GPU that loads the library, held until exit), so
 * n_elem is limited to 8,388,608; a larger n_elem is rejected with an error
 * and nothing is launched.  No call allocates or frees memory.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  The
 * address is kept per device ordinal for the life of the process, which
 * assumes the device's primary context (the one the CUDA runtime and torch
 * use) throughout: after cudaDeviceReset, or from another driver-API context
 * on the same device, the kept address is not valid there.  All
 * calls share the array, which keeps the last call's partial sums -- each call
 * overwrites every slot it reads -- and calls that overlap on the GPU (other
 * streams, other host threads) race on it. */
int nzb_norm_noalloc(const double* A, int64_t n_elem, int np, const double* w4, double* out, void* stream);

/* A steady-march solver over caller-owned buffers.  Every step maps S0 -> S0
 * (scratch S1, S2); a chunk of n steps is captured once as a CUDA graph and
 * replayed.  res (device double) receives the norm of the last step's stage-1
 * rate; counters (device 2 x uint64) accumulate limiter activity. */
typedef struct nzb_solver nzb_solver;
typedef struct {
  double* S0;
  double* S1;
  double* S2;
  double* dt;
  double* norm_partial;
  double* res;
  unsigned long long* counters;
} nzb_buffers;
int nzb_solver_create(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_buffers* buf,
                      int scheme_ssprk3, double dt_factor, nzb_solver** out);
int nzb_solver_run(nzb_solver* solver, int n_steps, void* stream);
int nzb_solver_destroy(nzb_solver* solver);

/* ---- batched steady march: many independent instances, one launch per stage
 * and bucket.  Instances are grouped in buckets of one (kind, order); each
 * bucket is an nzb_mesh over the concatenated elements of its instances, with
 * elem_inst / inst_status / inst_p_back set.  The march bookkeeping of every
 * instance (src/timestepping/march.py:125-230) runs on the device after each
 * chunk: the residual of its last step's stage-1 rate, then convergence,
 * non-finite, divergence, stall window and iteration cap; a retired instance
 * stops being advanced.  A chunk of n steps is one CUDA graph. */
typedef struct {
  int64_t n_inst;
  const int64_t* inst_begin;  /* (n_inst) first element, in the global element numbering */
  const int64_t* inst_end;    /* (n_inst) one past the last element */
  const double* inst_count;   /* (n_inst) 4 * NP * E_i, the norm's divisor */
  const double* inst_tol;     /* (n_inst) tolerance * residual scale */
  double* elem_norm;          /* (sum E) per-element norm contributions (scratch) */
  int32_t* status;            /* (n_inst) 0 running, 1 converged, 2 non-finite, 3 diverged, 4 stalled, 5 max_iterations */
  int32_t* iterations;        /* (n_inst) steps taken */
  double* res0;               /* (n_inst) */
  double* res;                /* (n_inst) residual at the last check */
  double* window;             /* (n_inst * stall_window) */
  int32_t* window_count;      /* (n_inst) */
  int32_t* n_running;         /* (1) */
  double divergence_factor;
  double stall_ratio;
  int32_t stall_window;
  int32_t max_iterations;
} nzb_batch_march;
typedef struct nzb_batch nzb_batch;
/* buckets: n_buckets meshes (device pointers inside), their physics and
 * buffers (S0, S1, S2, dt used; res / norm_partial / counters ignored),
 * elem_offset[b] = the bucket's first element in the global numbering,
 * dt_factor[b]. */
int nzb_batch_create(int n_buckets, const nzb_mesh* meshes, const nzb_physics* phys, const nzb_buffers* buffers,
                     const int64_t* elem_offset, const double* dt_factor, const nzb_batch_march* march,
                     nzb_batch** out);
/* Advance every running instance by n_steps (first = 1 for the initial
 * single step that sets res0), then run the device check. */
int nzb_batch_run(nzb_batch* batch, int n_steps, int first, void* stream);
int nzb_batch_destroy(nzb_batch* batch);

/* ---- discrete adjoint ----------------------------------------------------------
 * Products with the transposed Jacobians of the UNFOLDED residual R (M dU/dt =
 * -R, src/spatial/assembly.py:153-157) and the adjoint pseudo-time march of
 * DifferentiableCase.adjoint_solve (src/sensitivity.py:289-383):
 *   dlam/dtau = -M^-1 ((dR/dU)^T lam - seed),  classical RK4, frozen local step,
 * which replace the reference's jax.vjp of assembly.residual.  The flux
 * Jacobians are exact (forward-mode dual numbers through the same flux code);
 * the limiter is not part of the linearisation, as in the reference.
 *
 * nzb_vjp modes:
 *   VJP     out = (dR/dU)^T lam
 *   DEFECT  out = (dR/dU)^T lam - seed (out nullable); norm_partial[block] and
 *           elem_norm[e] (both nullable) receive sums of its squares
 *   RATE    out = -M^-1 ((dR/dU)^T lam - seed)
 *   RK4     stage k of lam_new = lam0 + dt/6 (f0 + 2 f1 + 2 f2 + f3), with
 *           f_k = RATE at lam (this stage's input): stages 0..2 store f_k and
 *           write the next input lam0 + c dt f_k to out (c = 1/2, 1/2, 1);
 *           stage 3 overwrites lam0 with lam_new.  lam must not alias out
 *           (stages 0-2) or lam0 (stage 3). */
enum { NZB_ADJ_VJP = 0, NZB_ADJ_DEFECT = 1, NZB_ADJ_RATE = 2, NZB_ADJ_RK4 = 3 };
typedef struct {
  int32_t mode;
  int32_t stage;
  const double* U;    /* (4, NP, E) linearisation state */
  const double* lam;  /* (4, NP, E) */
  const double* seed; /* (4, NP, E) dJ/dU */
  double* out;
  double* lam0;
  const double* dt;   /* (E) frozen local step */
  double* f0;
  double* f1;
  double* f2;
  double* norm_partial; /* nzb_element_blocks(mesh) doubles */
  double* elem_norm;    /* (E) */
} nzb_adjoint_args;
int nzb_vjp(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_adjoint_args* args, void* stream);

/* (dR/dX)^T lam per element vertex and (dR/dp_back)^T lam per element, the
 * products DifferentiableCase.value_and_gradient takes through the node
 * coordinates (src/sensitivity.py:453-458, src/spatial/operators.py:207-303).
 * verts (2 NV, E): vertex x then y coordinates (NV = 3 triangles, 4 quads);
 * dgs (16 doubles in HOST memory, row f, column v): the face tangent dX/dsigma
 * of face f is sum_v dgs[4 f + v] X_v (the reference's dgeom_dsigma_face,
 * straight edges); it is copied into the kernel's parameters;
 * gvert (2 NV, E) out; gpb (E) out, nullable.  Summing gvert over the
 * elements that share a node gives d(lam . R)/d(node). */
int nzb_vjp_coords(const nzb_mesh* mesh, const nzb_physics* phys, const double* U, const double* lam,
                   const double* verts, const double* dgs, double* gvert, double* gpb, void* stream);

/* dt_e = coefficient * 2 A_e / max(wave_e, 1e-10): local_time_step
 * (src/timestepping/step.py:171-183). */
int nzb_local_dt(const nzb_mesh* mesh, const double* wave, double coefficient, double* dt, void* stream);

/* The adjoint march over many independent instances (buckets as for
 * nzb_batch_*; a single solve is one bucket with one instance, elem_inst
 * nullable).  Each bucket: U (converged state), seed, lam (in/out), scratch
 * Y1, Y2, f0, f1, f2 (all (4, NP, E)) and dt (E).  nzb_adjoint_run(n_steps =
 * 0) takes the defect of the current lam as res0 (with lam = 0: rms(seed));
 * n_steps > 0 advances every running instance n_steps RK4 steps, then
 * measures res = rms((dR/dU)^T lam - seed) and sets status: 1 converged (res
 * <= tolerance * res0, or res0 = 0), 2 non-finite, 5 iteration cap. */
typedef struct {
  const double* U;
  const double* seed;
  double* lam;
  double* Y1;
  double* Y2;
  double* f0;
  double* f1;
  double* f2;
  const double* dt;
} nzb_adjoint_buffers;
typedef struct {
  int64_t n_inst;
  const int64_t* inst_begin; /* (n_inst) first element, global numbering */
  const int64_t* inst_end;
  const double* inst_count;  /* (n_inst) 4 * NP * E_i */
  double* elem_norm;         /* (sum E) scratch */
  int32_t* status;           /* (n_inst) 0 running, 1 converged, 2 non-finite, 5 iteration cap */
  int32_t* iterations;       /* (n_inst) */
  double* res0;              /* (n_inst) */
  double* res;               /* (n_inst) */
  int32_t* n_running;        /* (1) */
  double tolerance;
  int32_t max_iterations;
  int32_t reserved;
} nzb_adjoint_march;
typedef struct nzb_adjoint nzb_adjoint;
int nzb_adjoint_create(int n_buckets, const nzb_mesh* meshes, const nzb_physics* phys,
                       const nzb_adjoint_buffers* buffers, const int64_t* elem_offset,
                       const nzb_adjoint_march* march, nzb_adjoint** out);
int nzb_adjoint_run(nzb_adjoint* adjoint, int n_steps, void* stream);
int nzb_adjoint_destroy(nzb_adjoint* adjoint);

/* The integrals behind the parity observables of performance()
 * (src/post/postprocess.py:56-75,155-192,193-255), per instance of a mesh or
 * bucket, over the half channel that is meshed.  Boundary sums run over the
 * face quadrature points with ds = w_q |dX/dsigma| and the owner-side trace;
 * the entropy sum runs over the volume points with w_q det_q. */
enum {
  NZB_OBS_MOM_OUT = 0,   /* outflow  sum (rho vx vn + p nx) ds */
  NZB_OBS_MOM_IN = 1,    /* inflow   the same */
  NZB_OBS_WALL_PX = 2,   /* wall     sum p nx ds */
  NZB_OBS_MASS_IN = 3,   /* inflow   sum rho vn ds */
  NZB_OBS_MASS_OUT = 4,  /* outflow  the same */
  NZB_OBS_EXIT_LEN = 5,  /* outflow  sum ds */
  NZB_OBS_EXIT_MACH = 6, /* outflow  sum M ds */
  NZB_OBS_EXIT_P = 7,    /* outflow  sum p ds */
  NZB_OBS_EXIT_T = 8,    /* outflow  sum p / (R rho) ds */
  NZB_OBS_ENTROPY = 9,   /* volume   sum (p rho^-gamma / s_t - 1)^2 w det */
  NZB_OBS_AREA = 10,     /* sum of the element areas */
  NZB_NOBS = 11
};
typedef struct {
  const double* U;        /* (4, NP, E) state */
  int32_t n_seg;          /* instances */
  int32_t reserved;
  const int32_t* bedges;  /* inflow, outflow and wall edges of every instance, grouped by instance */
  const int32_t* bseg;    /* (n_seg + 1) offsets into bedges */
  const int32_t* eseg;    /* (n_seg + 1) element offsets: instance i owns [eseg[i], eseg[i + 1]) */
  double r_gas;           /* gas constant (exit temperature) */
  double s_t;             /* p_t^(1 - gamma) (R T_t)^gamma (entropy reference) */
  double* out;            /* (n_seg, NZB_NOBS) */
} nzb_obs_args;
/* All arrays device memory; one deterministic launch (fixed summation order). */
int nzb_observables(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_obs_args* args, void* stream);

/* The metric terms of a mesh from its node coordinates, on the device: the
 * coordinate-dependent part of build_operators (src/spatial/operators.py:
 * 240-303) for straight-sided elements.  mesh supplies kind, order, affine,
 * n_elem and n_edge; the outputs are the arrays an nzb_mesh points to (they may
 * be the mesh's own).  dgs is as for nzb_vjp_coords (host memory, copied into
 * the kernel's parameters).  All other arrays device memory. */
typedef struct {
  const double* X;           /* (n_node, 2) node coordinates */
  const int32_t* elem_nodes; /* (E, NV) vertex node ids, NV = 3 triangles, 4 quads */
  const int32_t* edge_conn;  /* (3, n_edge) as in nzb_mesh: owner, neighbour, owner face in bits 0-2 */
  double dgs[16];            /* tangent of face f = sum_v dgs[4 f + v] X_v */
  double* geo;               /* out: affine (5, E) xi_x, xi_y, eta_x, eta_y, det; else (2 NV, E) vertex x then y */
  double* minv;              /* out, general geometry only: (NP * NP, E) inverse mass matrices */
  double* area;              /* out: (E) */
  double* edge_geo;          /* out: (n_edge, 4) unit normal, |dX/dsigma|, length */
} nzb_geometry_args;
int nzb_geometry(const nzb_mesh* mesh, const nzb_geometry_args* args, void* stream);

/* The quasi-1D initial state, L2-projected onto the basis on the device
 * (src/timestepping/initialize.py:41-102, initial_condition = "quasi1d"): at
 * every volume point the state interpolated linearly in x from the instance's
 * quasi-1D solution, with vy = vx clip(y / y_w(x), 0, 1) y_w'(x), y_w the
 * instance's wall and its slope by central differences with h = 1e-6 L; then
 * U = M^-1 sum_q phi_q w_q det_q u_q.  mesh supplies kind, order, affine,
 * n_elem, minv (general geometry) and, for a batch, elem_inst (instance 0
 * without).  wall[i * NZB_WALL_PARAMS + k], per instance: family (0 conical,
 * 1 cubic Hermite: bell / smooth / moc, 2 cubic Bezier, 3 bezier8), length,
 * throat_x, 1 - throat_x, y_throat, y_inlet, y_exit, the Hermite end slopes
 * tan(theta) (1 - throat_x) length at the throat and at the exit, the Bezier
 * control heights c1, c2, h, and the eight bezier8 offsets (fractions of
 * y_throat).  All arrays device memory. */
#define NZB_WALL_PARAMS 20
typedef struct {
  const double* verts;      /* (2 NV, E): vertex x, then vertex y, of every element */
  const double* wall;       /* (n_inst, NZB_WALL_PARAMS) */
  const double* q1d;        /* the instances' quasi-1D solutions, concatenated: per instance its n points'
                               x (increasing), then density, then axial velocity, then pressure */
  const int64_t* q1d_begin; /* (n_inst + 1): first point of each instance's solution (a solution has n >= 2) */
  double* out;              /* (4, NP, E) */
} nzb_initial_args;
int nzb_initial_state(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_initial_args* args, void* stream);

/* ---- any order, curved (Q = 2) elements: the reference's per-element operators
 *
 * The kernels above take straight-sided elements of order 0..3 with their
 * tables in constant memory.  These entry points take what the reference's
 * build_operators produces (src/spatial/operators.py:139-206), for any order
 * and geometry order, in its layout: the state is (E, NP, 4), per element
 * grad_x / grad_y (E, NP, NQV) (weak-form gradients w det (dphi/dx, dphi/dy)),
 * grad_x_m / grad_y_m and face_basis_m (E, NF, NP, NQF) with the inverse mass
 * folded in, per edge point the owner's normal (n_edge, NQF, 2) and
 * |dX/dsigma| (n_edge, NQF).  Edges are numbered as the reference numbers
 * them: interior first, then boundary (src/geometry/mesh.py:34-66).  All
 * arrays device memory; NP up to 36 (triangles to p = 7, quadrilaterals to
 * p = 5). */
typedef struct {
  int32_t np, nqv, nqf, nface;
  int64_t n_elem, n_int, n_bnd;
  const double* phi_vol;      /* (NP, NQV) */
  const double* phi_face;     /* (2, NF, NP, NQF): side 0 owner's points, side 1 reversed */
  const double* w_face;       /* (NQF) */
  const double* grad_x;       /* (E, NP, NQV) */
  const double* grad_y;
  const double* grad_x_m;     /* (E, NP, NQV) */
  const double* grad_y_m;
  const double* face_basis_m; /* (E, NF, NP, NQF) */
  const int32_t* face_edge;   /* (E, NF) global edge id */
  const int32_t* face_side;   /* (E, NF) 0 owner, 1 neighbour */
  const double* face_sign;    /* (E, NF) +1 owner, -1 neighbour */
  const int32_t* edge_elem;   /* (n_edge, 2) owner, neighbour (boundary edges: owner, owner) */
  const int32_t* edge_face;   /* (n_edge, 2) local faces */
  const int32_t* edge_tag;    /* (n_bnd) boundary tag of each boundary edge */
  const double* edge_normal;  /* (n_edge, NQF, 2) */
  const double* edge_jac;     /* (n_edge, NQF) */
  const double* edge_length;  /* (n_edge) */
  const double* elem_area;    /* (E) */
  const double* mean_weights; /* (E, NP) cell-average weights */
} nzb_gen_mesh;
/* unfolded = 1: out = the residual R (src/backends/_numba_kernels.py:667-759, apply_mass false);
 * 0: out = the rate -M^-1 R (:586-664).  wave (E, nullable) the wave-speed sums; fw (n_edge, NQF, 4)
 * and smax (n_edge) scratch of the edge pass. */
int nzb_gen_rate(const nzb_gen_mesh* mesh, const nzb_physics* phys, int unfolded, const double* U, double* out,
                 double* wave, double* fw, double* smax, void* stream);
/* The positivity limiter in place (src/backends/_numba_kernels.py:927-1093); counters (device 2 x
 * uint64, nullable) accumulate the scaled and repaired elements. */
int nzb_gen_limit(const nzb_gen_mesh* mesh, const nzb_physics* phys, double* U, unsigned long long* counters,
                  void* stream);
/* One stage's update: stage 1 sets dt = dt_factor 2 A / max(wave, 1e-10) and the per-block partial
 * sums of the weighted squares of F (partial: nzb_gen_blocks(mesh) doubles, nullable); then
 * out = a U0 + b (V + dt F), or V + dt F when a = 0 (src/backends/_numba_kernels.py:789-850). */
typedef struct {
  int32_t stage, pad;
  double dt_factor, a, b;
  const double* V;
  const double* U0;
  const double* F;
  const double* wave;
  double* dt;
  double* out;
  double* partial;
} nzb_gen_update_args;
int nzb_gen_update(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_update_args* args, void* stream);
int64_t nzb_gen_blocks(const nzb_gen_mesh* mesh);
/* The Superbee TVB slope limiter, then the positivity limiter, in place (src/spatial/limiter.py:
 * 246-429 and apply_limiter): the cell averages into means ((E, 4) scratch), their domain maxima
 * max_e |ubar_s| into scale (4 scratch), then per element the slope factor from its face-averaged
 * traces and its neighbours' averages with the threshold tvb share max|ubar_s| (share (E): A_e /
 * A_domain), and the positivity limiter.  counters (device 2 x uint64, nullable) accumulate the
 * elements either limiter changed and the repaired ones. */
int nzb_gen_superbee(const nzb_gen_mesh* mesh, const nzb_physics* phys, double* U, const double* share,
                     double* means, double* scale, unsigned long long* counters, void* stream);

/* The coordinate-dependent operators of the generic path built on the device
 * from the node coordinates, for any order and geometry order (the
 * coordinate part of build_operators, src/spatial/operators.py:209-342): per
 * element the Jacobian at every volume point, grad_x / grad_y, the mass
 * matrix and its inverse, grad_x_m / grad_y_m / face_basis_m, the area and the
 * cell-average weights; per edge (from its owner) the unit normal and
 * |dX/dsigma| at every face point and the length.  The mesh supplies the
 * sizes, phi_vol, phi_face, w_face, face_side, edge_elem and edge_face; the
 * outputs are the arrays a nzb_gen_mesh then points to.  bad (device int32,
 * zeroed here) counts volume points with a non-positive Jacobian, where the
 * reference's build raises. */
typedef struct {
  int32_t ng;                  /* geometry nodes per element (3 / 4 straight, 6 / 9 curved) */
  int32_t reserved;
  const double* X;             /* (n_nodes, 2) node coordinates */
  const int32_t* elem_nodes;   /* (E, NG) geometry nodes, reference order */
  const double* w_vol;         /* (NQV) */
  const double* dphi_dxi;      /* (NP, NQV) */
  const double* dphi_deta;     /* (NP, NQV) */
  const double* dgeom_dxi;     /* (NG, NQV) */
  const double* dgeom_deta;    /* (NG, NQV) */
  const double* dgeom_dsigma;  /* (NF, NG, NQF) */
  double* grad_x;              /* (E, NP, NQV) */
  double* grad_y;
  double* grad_x_m;
  double* grad_y_m;
  double* face_basis_m;        /* (E, NF, NP, NQF) */
  double* inv_mass;            /* (E, NP, NP) */
  double* elem_area;           /* (E) */
  double* mean_weights;        /* (E, NP) */
  double* edge_normal;         /* (n_edge, NQF, 2) */
  double* edge_jac;            /* (n_edge, NQF) */
  double* edge_length;         /* (n_edge) */
  int32_t* bad;                /* device counter */
} nzb_gen_geometry_args;
int nzb_gen_geometry(const nzb_gen_mesh* mesh, const nzb_gen_geometry_args* args, void* stream);

/* The quasi-1D initial state of one instance on the generic path, projected on
 * the device (src/timestepping/initialize.py:41-102) as nzb_initial_state does
 * for the specialised meshes: the point coordinates and Jacobians from the
 * element's geometry nodes (curved elements included), the wall of
 * NZB_WALL_PARAMS numbers, the quasi-1D solution, the element's inverse mass;
 * out is the reference-layout (E, NP, 4) state.  The mesh supplies the sizes
 * and phi_vol. */
typedef struct {
  int32_t ng;                  /* geometry nodes per element */
  int32_t reserved;
  const double* X;             /* (n_nodes, 2) */
  const int32_t* elem_nodes;   /* (E, NG) */
  const double* geom_vol;      /* (NG, NQV) geometry shape functions at the volume points */
  const double* dgeom_dxi;     /* (NG, NQV) */
  const double* dgeom_deta;    /* (NG, NQV) */
  const double* w_vol;         /* (NQV) */
  const double* inv_mass;      /* (E, NP, NP) */
  const double* wall;          /* (NZB_WALL_PARAMS) */
  const double* q1d;           /* (4, n_q1d): x (increasing), density, axial velocity, pressure */
  int64_t n_q1d;               /* >= 2 */
  double* out;                 /* (E, NP, 4) */
} nzb_gen_initial_args;
int nzb_gen_initial_state(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_initial_args* args,
                          void* stream);

/* The parity observables' NZB_NOBS sums (as nzb_observables) on the generic
 * path: the boundary integrals with the owner-side traces and the normals and
 * |dX/dsigma| at every face point, the entropy deviation with w det from the
 * geometry nodes.  The mesh supplies phi_vol, phi_face, w_face, edge_elem,
 * edge_face, edge_tag, edge_normal, edge_jac and elem_area. */
typedef struct {
  int32_t ng;                  /* geometry nodes per element */
  int32_t reserved;
  const double* X;             /* (n_nodes, 2) */
  const int32_t* elem_nodes;   /* (E, NG) */
  const double* dgeom_dxi;     /* (NG, NQV) */
  const double* dgeom_deta;    /* (NG, NQV) */
  const double* w_vol;         /* (NQV) */
  const double* U;             /* (E, NP, 4) */
  double s_t;                  /* the entropy reference p_t^(1 - gamma) (R T_t)^gamma */
  double r_gas;
  double* out;                 /* (NZB_NOBS) */
} nzb_gen_obs_args;
int nzb_gen_observables(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_obs_args* args,
                        void* stream);

const char* nzb_last_error(void);
int nzb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NOZZLE_B200_H */
