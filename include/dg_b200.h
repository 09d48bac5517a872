/*
 * dg_b200.h -- C ABI of the B200-native residual + RK-stage path for
 * IhmeGroup/DG-MPI's 3D Euler solver on periodic hexahedral meshes (and its
 * 2D form on quadrilaterals, the dg2d_* entry points at the end).
 *
 * One library, libdg_b200.so, exports everything below.  Plain C types only
 * (no CUDA or torch types), so a C++ stepper inside the reference, ctypes, or
 * any FFI can bind it.  Paths in the comments are relative to the reference
 * project root.
 *
 * Ownership: the caller owns every host buffer; buffers are read or written
 * during the call and never retained.  A context owns all device memory,
 * streams and graphs it creates.  Tables and connectivity are immutable after
 * dg_create.
 *
 * Errors: every int-returning call returns DG_OK (0) or a DG_ERR_* code and
 * never throws; dg_last_error() gives the message for the last failure on that
 * context (the reference reports errors through C++ exceptions,
 * src/common/my_exceptions.h:14-115, device printf and assert; none of those
 * cross this boundary).
 *
 * Threading: a context is used by one host thread at a time; different
 * contexts may run concurrently (each has its own stream).  All calls are
 * synchronous with respect to the host buffers they take.
 *
 * Layout contract: host-side solution arrays are row-major Uc[ne][nb][5]
 * (Kokkos LayoutRight, the CPU build's layout; src/io/writer.cpp:72), with
 * nb = (p+1)^3 equidistant-Lagrange coefficients indexed k(p+1)^2+j(p+1)+i
 * (src/numerics/basis/tools.cpp:215-247).  The device layout is private.
 */
#ifndef DG_B200_H
#define DG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define DG_B200_ABI_VERSION 1

/* ---- status codes ---- */
#define DG_OK 0
#define DG_ERR_ARG 1          /* bad argument or inconsistent mesh/tables */
#define DG_ERR_CUDA 2         /* a CUDA runtime call failed */
#define DG_ERR_NONPHYSICAL 3  /* device status word: rho<=0, p<=0 or NaN seen */
#define DG_ERR_TIMEOUT 4      /* a bounded device wait gave up */
#define DG_ERR_UNSUPPORTED 5  /* valid input this build does not handle */
#define DG_ERR_NOMEM 6        /* device or host allocation failed */

/* numerical flux, [Physics] convective_flux_fcn (src/common/enums.h:80-91) */
#define DG_FLUX_LAX_FRIEDRICHS 0
#define DG_FLUX_HLLC 1

/* arithmetic of the residual: FP64 throughout, or the mixed-precision form
 * whose traces, fluxes and volume / lift contractions run in FP32 while the
 * stored solution, the residual accumulation, the inverse mass, the geometric
 * factors and the RK stage update stay FP64 */
#define DG_PREC_FP64 0
#define DG_PREC_MIXED_FP32 1

/* initial-condition / exact-solution families ([InitialCondition] name) */
#define DG_IC_UNIFORM 0        /* "Uniform": data = conserved state[5] */
#define DG_IC_VORTEX_REF 1     /* "IsentropicVortex": the reference's 3D vortex */
#define DG_IC_SPHERE 2         /* "Sphere" */
#define DG_IC_VORTEX_XY 3      /* "IsentropicVortexXY": data = rho,u,v,p,beta,xc,yc,Lx,Ly */
#define DG_IC_TAYLOR_GREEN 4   /* "TaylorGreen": data = Mach */
#define DG_IC_VORTEX_2D 5      /* 2D "IsentropicVortex": data = rho,u,v,p,strength (dg2d_* only) */

typedef struct dg_ctx dg_ctx;

/* A hexahedral mesh in the reference's in-memory form (src/mesh/mesh.h:
 * node_coords, elem_to_node_IDs, interior_faces).  interior_faces rows are
 * (rankL, elemL, faceL, orientL, rankR, elemR, faceR, orientR)
 * (src/mesh/mesh.h:280-284); on one GPU every rank entry must equal `rank`.
 * Every face must be interior (periodic meshes).  Elements may be general
 * trilinear hexahedra: when one is not a parallelepiped, the context keeps,
 * as the reference's helpers do, per-point metric terms and face normals and
 * a dense inverse mass matrix per element (nb^2 doubles each: 32 KB at p = 3,
 * 373 KB at p = 5) and runs the general-geometry kernel variants; such meshes
 * are not accepted by dg_batch_create or dg_create_partitioned
 * (DG_ERR_UNSUPPORTED), and an element whose Jacobian is not positive at a
 * quadrature point is rejected (DG_ERR_ARG). */
typedef struct dg_mesh_desc {
    int nnode;
    const double* node_coords;         /* [nnode][3] */
    int nelem;
    const unsigned* elem_to_node_ids;  /* [nelem][8], gbasis node order, x fastest */
    int nface;
    const unsigned* interior_faces;    /* [nface][8] */
    int rank;
} dg_mesh_desc;

typedef struct dg_case_desc {
    int order;       /* [Numerics] order, p = 0..5 */
    int flux;        /* DG_FLUX_* */
    double gamma;    /* [Physics] gamma (src/physics/base/base.cpp:28) */
    double gas_constant; /* [Physics] GasConstant (base.cpp:29) */
    int precision;   /* DG_PREC_* */
    int device;      /* CUDA device ordinal */
} dg_case_desc;

/* Replaces Solver<3>::Solver + precompute_matrix_helpers +
 * allocate_face_residual_views (src/solver/base.cpp:20-111, 563-598) and the
 * stepper's allocate_helpers (src/numerics/timestepping/stepper.cpp:57-69):
 * builds the 1D basis/quadrature tables, geometry classes, the periodic face
 * gather table (from interior_faces and the face-point permutations of
 * src/solver/helpers.cpp:326-378) and allocates device state. */
int dg_create(const dg_case_desc* cd, const dg_mesh_desc* md, dg_ctx** out);

/* Releases the context (Mesh::finalize / MemoryNetwork::finalize). */
void dg_destroy(dg_ctx* ctx);

/* Message of the last failing call on ctx (or of the last failing dg_create
 * when ctx is NULL). Never NULL. */
const char* dg_last_error(const dg_ctx* ctx);

int dg_num_basis(const dg_ctx* ctx);     /* nb = (p+1)^3 */
int dg_num_elements(const dg_ctx* ctx);

/* Host -> device copy of Uc[ne][nb][5]; replaces Kokkos::deep_copy(Uc, h_Uc)
 * after init_state_from_fcn / read_in_coefficients (base.cpp:113-279). */
int dg_set_state(dg_ctx* ctx, const double* Uc);

/* Device -> host copy of the current state; replaces
 * Solver::copy_from_device_to_host (base.cpp:226-230). */
int dg_get_state(dg_ctx* ctx, double* Uc);

/* R(U) of the current state into res[ne][nb][5] (host); replaces
 * Solver<3>::get_residual (base.cpp:401-561): volume integral, face traces,
 * on-device periodic face gather (in place of construct_face_states +
 * MemoryNetwork::communicate_face_solution, memory_network.cpp:55-175),
 * numerical flux, L=-F/R=+F scatter and face lift. */
int dg_residual(dg_ctx* ctx, double* res);

/* dt * M^-1 R(U) into dU[ne][nb][5] (host); replaces get_residual followed
 * by SolverTools::mult_inv_mass_matrix (src/solver/tools.cpp:124-139). */
int dg_mass_inverse_residual(dg_ctx* ctx, double dt, double* dU);

/* Advances the device state by nsteps classic RK4 steps of size dt; replaces
 * nsteps calls of RK4<3>::take_time_step (stepper.cpp:71-142), one fused
 * kernel per stage, the four stages of a step replayed from a CUDA graph. */
int dg_rk4_steps(dg_ctx* ctx, double dt, int nsteps);

/* dg_rk4_steps with CUDA events recorded on the context's stream around the
 * graph launches; *device_ms receives the device time of the nsteps steps
 * (the reference's Utils::Timer "Time to Solution", base.cpp:386-395, on the
 * device clock). */
int dg_rk4_steps_timed(dg_ctx* ctx, double dt, int nsteps, double* device_ms);

/* ---- stage-kernel launch variants and their tuner ----
 * Each order has a few compiled variants of the fused stage kernel (elements
 * per CTA, threads per CTA, variable groups of the pointwise phase).  The
 * tuner times one RK stage of every variant of the context's precision on its
 * mesh and current state (the state is not modified; the RK accumulator, dead
 * between steps, serves as scratch, so call it between steps) and selects the
 * fastest (entries of the other precision or geometry kind report -1 ms); callers cache the result
 * per (order, precision, GPU) and restore it with dg_set_stage_variant. */
int dg_num_stage_variants(int order);
int dg_stage_variant_info(int order, int variant, int* elems_per_cta, int* threads_per_cta, int* groups,
                          int* precision);
/* Options of a variant: bit 0 -- the variable groups' pencil tasks run in one
 * phase; bit 1 -- one coefficient buffer, refilled with the next batch once
 * the face traces have read it (more resident CTAs, less prefetch overlap);
 * bit 2 -- unfused volume (z interpolation, pointwise flux and contractions as
 * separate passes over all quadrature points; the groups count is unused);
 * bit 3 -- traces and lifts split into one task per output row; bit 4 -- one
 * face-flux point per thread and iteration (fewer registers); bit 5 -- general
 * (trilinear) geometry: per-point metric terms and normals and a dense
 * inverse mass matrix per element, the variants a context on a non-affine
 * mesh runs (and the only ones it accepts); bit 6 -- every interior face's
 * flux computed once by a face kernel launched before the stage kernel (the
 * elements read their six faces' fluxes);
 * bits 8..11 -- the minimum of resident CTAs per SM the kernel was compiled
 * for (0: none; a register cap); bit 12 -- the six faces' lifted fluxes
 * added inside the inverse mass's first pass instead of a pass of their own. */
int dg_stage_variant_flags(int order, int variant, int* flags);
int dg_set_stage_variant(dg_ctx* ctx, int variant);
int dg_get_stage_variant(const dg_ctx* ctx);
/* RK4 steps of a face-kernel variant on a context without ghosts as `chunks`
 * (1..64) element chunks per stage: the chunks' face-flux launches on a
 * second stream of the context, each chunk's stage launch after its face
 * launch, so a chunk's face kernel runs beside the previous chunk's stage
 * kernel.  The arithmetic is unchanged (bit-identical states); 1 (the
 * default) is one face launch and one stage launch per stage.
 * DG_ERR_UNSUPPORTED for partitioned contexts and contexts without a face
 * list. */
int dg_set_stage_chunks(dg_ctx* ctx, int chunks);
int dg_get_stage_chunks(const dg_ctx* ctx);
int dg_tune_stage(dg_ctx* ctx, int reps, int* best_variant, double* ms_per_variant);

/* Forward Euler, replaces FE<3>::take_time_step (stepper.cpp:23-55). */
int dg_fe_steps(dg_ctx* ctx, double dt, int nsteps);

/* L2 projection of an initial condition onto the basis, on the host side of
 * the library (C++/OpenMP); replaces Solver::init_state_from_fcn
 * (base.cpp:113-223) + SolverTools::L2_projection (tools.cpp:66-122).
 * Writes the device state and, if Uc != NULL, a host copy. */
int dg_project_ic(dg_ctx* ctx, int ic_type, const double* data, int ndata, double t, double* Uc);

/* Volume-normalised L2 error of the device state against an exact solution
 * (FP64 device reduction); replaces get_error(solver, 2, true)
 * (src/post/main.cpp:30-201).  err[5], one per conserved variable. */
int dg_l2_error(dg_ctx* ctx, int ic_type, const double* data, int ndata, double t, double* err);

/* Volume-averaged kinetic energy (1/V) * integral of |rho u|^2 / (2 rho). */
int dg_kinetic_energy(dg_ctx* ctx, double* ke);

/* Allocation-free kinetic energy.  No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc -- applications whose device memory
 * is owned by a framework allocator or a fixed arena that forbids allocations
 * behind its back: the call allocates nothing.  The caller passes device
 * pointers to a state d_state [nelem][5][nb] (the device layout of
 * dg_device_state) and to per-element Jacobian determinants d_djac [nelem];
 * the result, (1/V) * integral of |rho u|^2 / (2 rho) over the mesh with
 * V = sum of 8 * djac, is written to the device double d_ke.  Work is queued
 * on `stream` (a cudaStream_t, NULL for the default stream) and the call does
 * not wait for it.  d_state must be complete on `stream` when the call is
 * made: a state written by a context's calls is written on dg_stream(ctx),
 * which does not wait for other streams, so record an event on dg_stream(ctx)
 * and make `stream` wait on it (or synchronise) first.
 *
 * Affine meshes only: one det J per element is applied at every quadrature
 * point, which is exact for parallelepiped elements (every mesh of
 * dg_mesh_periodic_box).  On a trilinear (non-affine) mesh the Jacobian varies
 * inside an element and the result differs from dg_kinetic_energy, which
 * evaluates it per point.  For an affine mesh, d_djac[e] is the constant
 * Jacobian determinant of element e (for a uniform box with element size
 * h, (hx/2)(hy/2)(hz/2)).  d_state, d_djac and d_ke must be memory of the
 * current device (checked; DG_ERR_ARG otherwise).
 *
 * Scratch lives in a static device array of 32768 doubles (256 KB) that every
 * GPU loading this library holds until the process exits; it holds two
 * partial sums for each of at most 16384 blocks of 64 elements, which bounds
 * nelem to 1,048,576 (a 96^3 mesh fits), and larger meshes are rejected with
 * DG_ERR_ARG.  All calls on a device share that array: two calls whose
 * work overlaps on the GPU (for example on two streams) race and corrupt each
 * other's result, so serialise them.  Each call overwrites every scratch entry
 * it reads, so nothing is carried over from an earlier call.  The first call on a device
 * does a one-time set-up (loads the basis tables and looks up the array's
 * device address with that device current); make that first call before any
 * stream capture.  That set-up is cached per device for the life of the
 * process: a cudaDeviceReset between calls invalidates it (the tables and
 * the array's address belong to the reset context), so do not reset a device
 * that this call has used. */
int dg_kinetic_energy_noalloc(int order, int nelem, const double* d_state, const double* d_djac,
                              double* d_ke, void* stream);

/* Total mesh volume (sum of element volumes, MeshTools::get_total_volume). */
int dg_total_volume(const dg_ctx* ctx, double* vol);

/* Device status word accumulated since the last call (bit 0: non-positive
 * density, bit 1: non-positive pressure, bit 2: NaN, bit 3: HLLC found no
 * valid wave ordering -- the reference's assert branch,
 * src/physics/euler/functions.cpp:389-398); cleared by the call. */
int dg_status(dg_ctx* ctx, unsigned* flags);

/* Waits for all work of ctx. */
int dg_sync(dg_ctx* ctx);

/* Failure-detection probe of the bounded device waits: one CTA on `device`
 * waits, through the same bounded mbarrier wait the tensor-core kernel's
 * waits use, on a barrier that nothing completes (arrive = 0) or that one of
 * its threads completes first (arrive = 1).  The first gives up after about
 * limit_cycles SM cycles (0 .. 4e9) and returns DG_ERR_TIMEOUT, the second
 * returns DG_OK; *waited_cycles (may be NULL) receives the cycles the wait
 * took.  The kernel returns normally either way and leaves nothing in flight,
 * so the device stays usable.  Error text: dg_last_error(NULL). */
int dg_probe_bounded_wait(int device, long long limit_cycles, int arrive, long long* waited_cycles);

/* Raw device pointers for callers that keep data resident (benchmarks,
 * multi-GPU exchange).  Layout of the device state: [ne][5][nb]. */
void* dg_device_state(dg_ctx* ctx);

/* ---- domain decomposition over several GPUs ----
 *
 * Replaces the partitioned mesh of src/mesh/mesh.cpp:399-470 and the ghost
 * trace exchange MemoryNetwork::communicate_face_solution
 * (src/memory/memory_network.cpp:55-175).  A rank's mesh lists its owned
 * elements first -- the first `ninterior` of them share no face with another
 * rank -- followed by ghost elements: copies of the neighbouring ranks'
 * elements across the partition faces (node coordinates included, so the
 * face normals are computed exactly as on the owner).  Face rows carry the
 * owners' ranks in columns 0 and 4 like the reference's partitioned
 * interior_faces; elements are local ids of this mesh.
 *
 * The exchange moves, per face between an owned element and a ghost, one
 * boundary slice of 5 (p+1)^2 coefficients each way (the coefficients of the
 * element on that face; the receiver interpolates them as the on-device
 * gather does).  Slices are grouped per peer rank and ordered by the face's
 * left side (rank, owner-local element id, face), so slot i of one rank's
 * send range for a peer is slot i of the peer's receive range.  Transport is
 * the caller's (NCCL, CUDA-aware MPI, a peer copy): per RK stage s the caller
 * packs the stage's input buffer, exchanges, unpacks, and launches the stage
 * (the interior part may run while the exchange is in flight). */
typedef struct dg_part_desc {
    int nowned;              /* owned elements: local ids [0, nowned) */
    int ninterior;           /* owned elements [0, ninterior) have no ghost neighbour */
    const int* ghost_rank;   /* [nelem - nowned] owner rank of each ghost */
    const int* ghost_elem;   /* [nelem - nowned] the ghost's local id on its owner */
} dg_part_desc;

/* buffers of the RK4 stepper: stage s (1..4) reads DG_BUF_U0, DG_BUF_STAGE_A,
 * DG_BUF_STAGE_B, DG_BUF_STAGE_A and writes STAGE_A, STAGE_B, STAGE_A, U0 */
#define DG_BUF_U0 0
#define DG_BUF_STAGE_A 1
#define DG_BUF_STAGE_B 2

/* dg_create for one rank of a partitioned mesh (md->rank is this rank). */
int dg_create_partitioned(const dg_case_desc* c, const dg_mesh_desc* m, const dg_part_desc* part, dg_ctx** out);

/* Slab decomposition of the periodic box of dg_mesh_periodic_box along `axis`
 * (layer * nparts / n[axis]) into the mesh of rank `part` in the form above.
 * Sizes first: call with NULL arrays to get nnode / nelem / nface / nowned /
 * ninterior.  global_elem[nelem] receives each local element's id in the
 * unpartitioned box. */
int dg_partition_periodic_box(const int n[3], const double x0[3], const double len[3], unsigned rotate_seed,
                              int nparts, int part, int axis,
                              int* nnode, double* node_coords, int* nelem, unsigned* elem_to_node_ids,
                              int* nface, unsigned* interior_faces,
                              int* nowned, int* ninterior, int* ghost_rank, int* ghost_elem, int* global_elem);

/* Host-side halo plan of a partitioned mesh (no GPU needed): per peer its
 * rank and its [offset, offset + count) range of slices; per slice the owned
 * (element, face) sent and the ghost (element, face) received.  Sizes first:
 * with NULL arrays, *npeers and *nslices only. */
int dg_halo_plan(const dg_mesh_desc* m, const dg_part_desc* part, int* npeers, int* peer_rank, int* peer_offset,
                 int* peer_count, int* nslices, int* send_elem, int* send_face, int* recv_elem, int* recv_face);

/* The context's halo: number of peers, a peer's rank and slice range, and
 * the doubles per slice (5 (p+1)^2). */
int dg_halo_num_peers(const dg_ctx* ctx);
int dg_halo_peer(const dg_ctx* ctx, int i, int* rank, int* offset, int* count);
int dg_halo_slice_doubles(const dg_ctx* ctx);

/* Gathers the outgoing slices of buffer `buf` (DG_BUF_*) into the device
 * array d_send [nslices][5][(p+1)^2] / scatters d_recv into the ghost
 * elements of `buf`.  Queued on `stream` (NULL: the context's stream). */
int dg_halo_pack(dg_ctx* ctx, int buf, double* d_send, void* stream);
int dg_halo_unpack(dg_ctx* ctx, int buf, const double* d_recv, void* stream);

/* RK4 stage s (1..4) with time step dt on the context's stream, over the
 * owned elements (range 0), the interior ones (range 1) or the others
 * (range 2); not synchronised.  Four stages on all owned elements make one
 * dg_rk4_steps step. */
int dg_rk4_stage(dg_ctx* ctx, int stage, double dt, int range);

/* The context's CUDA stream (a cudaStream_t), for ordering a transport. */
void* dg_stream(dg_ctx* ctx);

/* ---- batched ensembles ----
 *
 * Many independent cases (each its own periodic mesh, order and time step)
 * advanced together by the `dg_batch_*` entry points (the reference runs one
 * case per process, so there is no reference function they replace; each
 * case's arithmetic is exactly that of a dg_ctx on the same case).  Cases of the same (order, flux, gamma, gas
 * constant) share one group: their meshes are concatenated, each element
 * scaling its update by its own case's dt.  dg_batch_rk4_steps replays a CUDA
 * graph of one RK4 step: by default each group's launches, one group after
 * another; in single-launch mode (every group of order 1..5 on affine
 * elements) each RK stage is ONE persistent launch over all groups, after one
 * face-flux launch over all groups, whose blocks start on per-group ranges
 * weighted by the groups' work and then claim element batches of any group
 * from per-group counters until all are done (128 threads per block, each
 * order's configuration one of its compiled variants).  dg_batch_tune keeps
 * whichever form is faster on the batch.  All cases must name the same device
 * and precision.  Results per case are bit-identical to a dg_ctx of that case
 * running the same stage variant (dg_batch_group_info). */
typedef struct dg_batch dg_batch;

int dg_batch_create(int ncases, const dg_case_desc* cases, const dg_mesh_desc* meshes, dg_batch** out);
void dg_batch_destroy(dg_batch* b);
/* Message of the last failed call on b (or of the last failed dg_batch_create
 * of this thread when b is NULL). */
const char* dg_batch_last_error(const dg_batch* b);
int dg_batch_num_groups(const dg_batch* b);
/* order, number of cases, elements and current stage variant of group g */
int dg_batch_group_info(const dg_batch* b, int g, int* order, int* ncases, int* nelem, int* variant);
/* order, elements, group and time step of case c */
int dg_batch_case_info(const dg_batch* b, int c, int* order, int* nelem, int* group, double* dt);
/* host state of case c, layout [nelem][nb][5] as for dg_set_state */
int dg_batch_set_state(dg_batch* b, int c, const double* Uc);
int dg_batch_get_state(dg_batch* b, int c, double* Uc);
/* dg_project_ic for case c (Uc may be NULL) */
int dg_batch_project_ic(dg_batch* b, int c, int ic_type, const double* data, int ndata, double t, double* Uc);
/* dg_cfl_time_step for case c on a host state of that case */
int dg_batch_cfl_time_step(dg_batch* b, int c, const double* Uc, double cfl, double* dt);
/* time step of case c (default 0: the case does not move) */
int dg_batch_set_time_step(dg_batch* b, int c, double dt);
/* nsteps RK4 steps of every case, each with its own dt */
int dg_batch_rk4_steps(dg_batch* b, int nsteps);
/* the same, device time of the graph launches in milliseconds */
int dg_batch_rk4_steps_timed(dg_batch* b, int nsteps, double* device_ms);
/* picks the fastest stage variant of every group (dg_tune_stage per group),
 * then times `reps` RK4 steps in per-group mode and in single-launch mode (when
 * every group can run it) and keeps the faster mode; the state is unchanged */
int dg_batch_tune(dg_batch* b, int reps);
/* single = 1: one launch per RK stage for all groups (DG_ERR_UNSUPPORTED when
 * a group has order 0 or non-affine elements); 0: one launch per group and
 * stage (each group back to its own variant).  No counterpart in the
 * reference (one case per process). */
int dg_batch_set_launch_mode(dg_batch* b, int single);
/* 1 in single-launch mode, 0 in per-group mode */
int dg_batch_get_launch_mode(const dg_batch* b);
/* dg_l2_error for case c */
int dg_batch_l2_error(dg_batch* b, int c, int ic_type, const double* data, int ndata, double t, double* err);
/* status flags of all groups since the last call (bits as dg_status) */
int dg_batch_status(dg_batch* b, unsigned* flags);

/* ---- host-side mesh helper (replaces reading an HDF5 mesh file,
 * src/mesh/mesh.cpp:79-204, for periodic boxes) ---- */

/* Uniform periodic box [x0,x0+L0]x[x1,x1+L1]x[x2,x2+L2] with n0*n1*n2 hex
 * elements, element id i + n0*(j + n1*k).  Nodes are not shared across the
 * periodic boundary (every element is a proper parallelepiped); periodicity
 * lives in interior_faces.  If rotate_seed != 0, every element's local node
 * numbering is replaced by one of the 24 proper rotations of the cube
 * (seeded), which exercises non-trivial face orientations.  Sizes first:
 * call with NULL arrays to get nnode/nelem/nface. */
int dg_mesh_periodic_box(const int n[3], const double x0[3], const double len[3],
                         unsigned rotate_seed,
                         int* nnode, double* node_coords,
                         int* nelem, unsigned* elem_to_node_ids,
                         int* nface, unsigned* interior_faces);

/* ---- mesh and solution files in the reference's HDF5 schemas (host only,
 * no GPU; a self-contained reader/writer of the HDF5 subset these files use:
 * version 0 superblock, symbol-table groups, version 1 object headers,
 * contiguous or compact integer / IEEE float datasets; other HDF5 files are
 * refused with DG_ERR_ARG and a message, never guessed) ---- */

/* Replaces Mesh::read_mesh (src/mesh/mesh.cpp:79-204): reads Dimension,
 * QOrder, nElem, nNode, nIFace, nNodePerElem, NodeCoords, Elem2Nodes and
 * IFaceData.  node_coords is [nnode][dim], elem_to_node_ids
 * [nelem][nnode_per_elem] (the file's gbasis node order), interior_faces
 * [nface][8] in the dg_mesh_desc row form with both rank entries 0.  Sizes
 * first: with all three arrays NULL only the counts are returned.  Any
 * dimension and element type is read; dg_create takes dim 3, qorder 1,
 * nnode_per_elem 8 meshes whose faces are all interior (periodic). */
int dg_mesh_read_h5(const char* path, int* dim, int* qorder, int* nnode_per_elem, int* nnode, double* node_coords,
                    int* nelem, unsigned* elem_to_node_ids, int* nface, unsigned* interior_faces);

/* Writes a hexahedral mesh in that format (Dimension 3, QOrder 1,
 * nNodePerElem 8, nNodePerFace 4, nBFaceGroup 0, 64-bit integers as the
 * reference's mesh files store them); dg_mesh_read_h5 reads it back exactly. */
int dg_mesh_write_h5(const char* path, const dg_mesh_desc* md);

/* Replaces Writer::write (src/io/writer.cpp:10-64) for one rank: the
 * attributes Number of Ranks / Dimensions / Elements / Nodes / Nodes Per
 * Element / Basis Functions / State Variables, Solver Final Time and Stored
 * Layout (1: row-major), the dataset Number of Elements per Partition, and the
 * parallel datasets Node Coordinates, Local to Global Node ID, Element Global
 * Node IDs, Local to Global Element IDs and Solution Coefficients (each with
 * its _offsets and _dims, src/io/HDF5Wrapper.h:775-880).  Uc is [nelem][nb][5]
 * with nb = (order+1)^3. */
int dg_solution_write_h5(const char* path, const dg_mesh_desc* md, int order, const double* Uc, double time);

/* Replaces Solver::read_in_coefficients (src/solver/base.cpp:234-279) and
 * Reader's serialisation (src/io/reader.h:28-80): reads Solution Coefficients
 * of every rank block, in either stored layout, into Uc[nelem][nb][ns] in
 * global element order (Local to Global Element IDs).  Sizes first: with Uc
 * NULL only nelem, nb, ns and the file's Solver Final Time are returned. */
int dg_solution_read_h5(const char* path, int* nelem, int* nb, int* ns, double* time, double* Uc);

/* Host-side time step from a CFL number on a given state (the reference has
 * none; [Stepper] timestep is used as is): dt = cfl * h_min /
 * ((2p+1) * max over element nodes of (|u| + c)). */
int dg_cfl_time_step(dg_ctx* ctx, const double* Uc, double cfl, double* dt);

/* ---- host-side tables (no GPU needed) ---- */

/* n-point Gauss-Legendre rule, ascending nodes; replaces the tables of
 * Nodes::get_gauss_legendre_segment_nodes (src/numerics/nodes.cpp:97-) and
 * SegmentQuadrature::get_segment_weights_gl (quadrature/segment.cpp:7-). */
int dg_gauss_legendre(int n, double* x, double* w);

/* Face-point order of orientation `orient` (0..7) on an npts = n1*n1 face
 * grid; replaces get_face_pts_order_wrt_orient0_hexahedron
 * (src/numerics/basis/shape.cpp:326-428). */
int dg_face_orientation_order(int orient, int npts, int* order);

/* 1D tables of order p: B[m][n] and D[m][n] (values / derivatives of the
 * equidistant Lagrange basis at the m = p+2 Gauss-Legendre points) and the
 * inverse 1D mass matrix Minv[n][n] (n = p+1); the 3D operators of
 * src/solver/helpers.cpp:5-100 are their tensor products. */
int dg_basis_tables(int p, double* B, double* D, double* Minv);

/* ======================================================================
 * 2D quadrilaterals (Solver<2> with LagrangeQuad, src/solver/base.cpp
 * instantiated for dim 2): a separate context type, FP64.
 *
 * The same residual and RK stage as the 3D path on periodic meshes of
 * parallelograms, with the reference's 2D rules: (p+2)^2 Gauss points per
 * element (quadrature/quadrilateral.cpp:36-41), p+1 Gauss points per edge
 * (segment quadrature of order 2p+1, segment.cpp:424-426, helpers.cpp:225),
 * edge points ordered by the two orientations of
 * get_face_pts_order_wrt_orient0_quadrilateral (shape.cpp:43-66), normals
 * (dy/ds, -dx/ds) of the left element's edge (shape.cpp:154-210).
 * Host state layout Uc[ne][nb][4] (rho, rho u, rho v, rho E), nb = (p+1)^2,
 * basis index j(p+1)+i.
 * ====================================================================== */

/* A quadrilateral mesh: node_coords [nnode][2], elem_to_node_ids [nelem][4]
 * (gbasis node order, x fastest), interior_faces [nface][8] rows (rankL,
 * elemL, faceL, orientL, rankR, elemR, faceR, orientR) with local faces
 * 0..3 (get_local_nodes_on_face_quadrilateral, shape.cpp:125-152) and
 * orientations 0 / 1; every element a parallelogram (to 1e-9 of its size:
 * the Jacobian is taken at the element's centre).  Element edges that
 * are no interior face (the boundary edges of a non-periodic mesh) add
 * nothing to the residual, as in the reference, whose residual loops over the
 * interior faces only (src/solver/base.cpp:470-561). */
typedef struct dg_mesh2d_desc {
    int nnode;
    const double* node_coords;
    int nelem;
    const unsigned* elem_to_node_ids;
    int nface;
    const unsigned* interior_faces;
    int rank;
} dg_mesh2d_desc;

typedef struct dg_ctx2d dg_ctx2d;

/* Solver<2>::Solver + precompute_matrix_helpers: tables, connectivity,
 * geometry, device buffers.  cd->precision must be DG_PREC_FP64;
 * DG_ERR_UNSUPPORTED for non-parallelogram elements.  Errors of a failed
 * create: dg_last_error(NULL). */
int dg2d_create(const dg_case_desc* cd, const dg_mesh2d_desc* md, dg_ctx2d** out);
void dg2d_destroy(dg_ctx2d* ctx);
const char* dg2d_last_error(const dg_ctx2d* ctx);
int dg2d_num_basis(const dg_ctx2d* ctx);
int dg2d_set_state(dg_ctx2d* ctx, const double* Uc);
int dg2d_get_state(dg_ctx2d* ctx, double* Uc);
/* R(U) of the current state (Solver<2>::get_residual, base.cpp:401-561) */
int dg2d_residual(dg_ctx2d* ctx, double* res);
/* RK4 / FE steps on the device state (stepper.cpp:23-142) */
int dg2d_rk4_steps(dg_ctx2d* ctx, double dt, int nsteps);
int dg2d_rk4_steps_timed(dg_ctx2d* ctx, double dt, int nsteps, double* device_ms);
int dg2d_fe_steps(dg_ctx2d* ctx, double dt, int nsteps);
/* L2 projection of an initial condition (init_state_from_fcn,
 * base.cpp:113-223) into Uc (may be NULL) and the device state; ic_type
 * DG_IC_UNIFORM (data = 4 conserved values), DG_IC_VORTEX_2D, or
 * DG_IC_VORTEX_XY (evaluated at (x, y, 0)) */
int dg2d_project_ic(dg_ctx2d* ctx, int ic_type, const double* data, int ndata, double t, double* Uc);
/* volume-normalised L2 error of the device state against the same
 * families at time t (get_error, src/post/main.cpp:30-201); err[4] */
int dg2d_l2_error(dg_ctx2d* ctx, int ic_type, const double* data, int ndata, double t, double* err);
/* the device status word (the 3D bits); DG_ERR_NONPHYSICAL when set */
int dg2d_status(dg_ctx2d* ctx, unsigned* flags);

/* Periodic box [x0,x0+L0]x[x1,x1+L1] of n0*n1 quadrilaterals, element id
 * i + n0 j; faces (right, top) of each element in element order; with
 * rotate_seed != 0 every element's local numbering is rotated by a seeded
 * multiple of 90 degrees.  Sizes first (NULL arrays). */
int dg_mesh2d_periodic_box(const int n[2], const double x0[2], const double len[2], unsigned rotate_seed,
                           int* nnode, double* node_coords, int* nelem, unsigned* elem_to_node_ids, int* nface,
                           unsigned* interior_faces);

/* Writer::write for a 2D state (Uc[ne][nb][4]; Number of Dimensions 2,
 * Number of Nodes Per Element 4, Number of State Variables 4) */
int dg2d_solution_write_h5(const char* path, const dg_mesh2d_desc* md, int order, const double* Uc, double time);

#ifdef __cplusplus
}
#endif
#endif
