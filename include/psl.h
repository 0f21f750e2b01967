/*
 * psl.h -- C ABI of the B200-native PeriodicShiftLBM lattice update.
 *
 * Drop-in for the reference's per-step update path: each entry point replaces one of the
 * reference's free functions (cited beside it).  The reference binds these at compile
 * time (header-only C++/TNL); here they are plain C symbols over an opaque grid handle,
 * so C++, Python (ctypes) or any FFI can drive them.
 *
 * Conventions
 *   - Every function returns an int status: PSL_OK (0) or a PSL_ERR_* code; the message of
 *     the last error on the calling thread is psl_last_error().  No exception crosses the
 *     ABI.
 *   - A grid owns its device memory (populations, markers, scratch); the caller owns every
 *     host buffer it passes.
 *   - All device work of a grid is issued on the grid's CUDA stream (default: the legacy
 *     default stream; see psl_grid_set_stream) and is stream-ordered; functions that return
 *     host data synchronise that stream.
 *   - Grids that exchange data (coarse/fine) must share one stream.
 *   - There is no CPU fallback: without a usable CUDA device, psl_grid_create fails.
 */
#ifndef PSL_H
#define PSL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PSL_OK 0
#define PSL_ERR_INVALID 1  /* bad argument or inconsistent grid */
#define PSL_ERR_CUDA 2     /* CUDA runtime error */
#define PSL_ERR_NOMEM 3    /* device allocation failed */
#define PSL_ERR_STATE 4    /* device health flag set (non-finite density) or barrier timeout */

typedef struct psl_grid psl_grid;

/* Population storage in HBM.  Arithmetic is FP32 in the three production forms. */
#define PSL_STORAGE_F32 0       /* f_q as float (216 B moved per cell update) */
#define PSL_STORAGE_F16_SHIFTED 1  /* f_q - w_q as IEEE half (108 B per cell update) */
#define PSL_STORAGE_BF16_SHIFTED 2 /* f_q - w_q as bfloat16 (108 B per cell update) */
#define PSL_STORAGE_F64 3       /* f_q as double with FP64 arithmetic: the FP64 oracle runs
                                   that the reduced-precision forms are measured against */

/* Per-grid metadata; mirrors InfoStruct (include/types.h:73-75). */
typedef struct psl_info {
  int grid_id;                 /* refinement level, 0 = coarsest (InfoStruct::gridID) */
  float res;                   /* cell size in physical units (mm) */
  int cell_count_x, cell_count_y, cell_count_z;
  float ox, oy, oz;            /* physical position of cell (0,0,0) */
  float nu;                    /* lattice kinematic viscosity */
  float dt_phys;               /* physical time step (s) */
  int i_subgrid_start, j_subgrid_start, k_subgrid_start; /* finer block on this grid, */
  int i_subgrid_end, j_subgrid_end, k_subgrid_end;       /* half-open; all 0 = none   */
} psl_info;

/* The flow-past-sphere case hooks (flowAroundSphere/flowAroundSphereMainSingle.cu:41-92). */
typedef struct psl_sphere_case {
  float sphere_x, sphere_y, sphere_z, sphere_r; /* physical units */
  float u_in;        /* inlet / given velocity (lattice units) */
  float rho_given;   /* given density at the outlet */
  int wall_mode;     /* 0: free-slip y/z walls; 1: velocity-given y/z walls (reference driver) */
  float smagorinsky; /* Smagorinsky constant; 0 disables LES */
  uint32_t seed;     /* start-state noise seed */
  float noise_amp;   /* start-state velocity noise amplitude (uniform +-amp) */
} psl_sphere_case;

/* Marker byte (psl_set_markers): kind in bits 0-2, outer-normal index in bits 3-7,
 * normal index = (nx+1)*9 + (ny+1)*3 + (nz+1).  For PSL_CELL_SKIP the upper bits are 1 for
 * a ghost cell (fine-grid boundary layer), 0 for a refined-interior cell and 2 for a
 * refined-interior cell that the case marks bounce-back (reported solid by the exports). */
#define PSL_CELL_SKIP 0
#define PSL_CELL_FLUID 1
#define PSL_CELL_SOLID 2
#define PSL_CELL_GIVEN_U 3
#define PSL_CELL_GIVEN_RHO 4
#define PSL_CELL_GIVEN_NONE 5
#define PSL_CELL_GIVEN_BOTH 6
#define PSL_CELL_MIRROR 7

/* ---- grid lifetime (replaces GridStruct construction, fArray.setSizes(27, N) and
 *      shifter = IntArrayType(27, 0): flowAroundSphereMainSingle.cu:171-182) ---- */
int psl_grid_create(const psl_info* info, int storage, psl_grid** out);
/* The population rows are mapped twice back to back in virtual memory when the row size is a
 * multiple of the driver's mapping granularity (2 MiB: 1,048,576 cells in FP16/BF16,
 * 524,288 in FP32) and 55 N < 2^32, so the update addresses cell + shift without the
 * periodic wrap; other grids, and grids made with PSL_GRID_ONE_MAPPING, use one plain
 * allocation.  Results are the same bits either way. */
#define PSL_GRID_ONE_MAPPING 1u
int psl_grid_create_ex(const psl_info* info, int storage, unsigned int flags, psl_grid** out);
/* rows_mapped_twice: 1 when the rows are mapped twice; row_stride: elements from one
 * population row to the next (2N when mapped twice). */
int psl_grid_get_layout(const psl_grid* grid, int* rows_mapped_twice, long long* row_stride);
int psl_grid_destroy(psl_grid* grid);
int psl_grid_set_stream(psl_grid* grid, void* cuda_stream);
int psl_grid_get_info(const psl_grid* grid, psl_info* info, long long* cell_count, int* storage);

/* ---- hook equivalents (evaluated once into per-cell markers; see psl_hooks.cuh) ---- */
/* getMarkers / getGivenRhoUxUyUz / getSmagorinskyConstant of the sphere case. */
int psl_apply_sphere_case(psl_grid* grid, const psl_sphere_case* sc);
/* Caller-computed markers, one byte per cell in cell order (i fastest). */
int psl_set_markers(psl_grid* grid, const uint8_t* host_markers);
int psl_get_markers(psl_grid* grid, uint8_t* host_markers);
/* getGivenRhoUxUyUz with one value for every boundary cell. */
int psl_set_given(psl_grid* grid, float rho, float ux, float uy, float uz);
/* getGivenRhoUxUyUz per cell: host (rho, ux, uy, uz) x N, or NULL to return to uniform. */
int psl_set_given_field(psl_grid* grid, const float* host_rho_u);
/* getSmagorinskyConstant (uniform per grid); 0 disables LES. */
int psl_set_smagorinsky(psl_grid* grid, float cs);
/* getSmagorinskyConstant(i, j, k, Info) per cell (include/applyLocalCellUpdate.h:68, e.g.
 * NACA0012/NACA0012Main.cu:74): host constants x N in cell order (i fastest), each finite
 * and >= 0 (0: no LES at that cell), evaluated once from the case's hook and kept on the
 * device (4 bytes per cell, read by every update); NULL returns to the uniform constant.
 * Used by the plain, customised and scalar-transport updates; the learned closure, when
 * attached, replaces the Smagorinsky rate altogether.  Not for grids in a batch. */
int psl_set_smagorinsky_field(psl_grid* grid, const float* host_cs);
/* The customised update of the reference's rotating-machinery cases
 * (M35Full/applyLocalCellUpdateCustomized.h, M40Impeller/applyLocalCellUpdateCustomized.h)
 * on PS grids.  Selected when a body force is set or the markers hold either of:
 *   PSL_CELL_SOLID with normal bits 1 (marker 0x0A): moving wall -- applyMovingBounceback
 *     (boundaryConditions/applyMovingBounceback.h:8-60) with the cell's given velocity;
 *   PSL_CELL_FLUID with normal bits 1 (marker 0x09): forced-velocity cell -- force
 *     rho (u_given - u), the cases' getForcing hook (M35Full/m35Main.cu:101-119).
 * Every collided cell adds the uniform body force (lattice units) and collides with the
 * forcing collision (M40Impeller/applyCollisionCustomized.h:6-16).  Not combined with the
 * learned closure. */
int psl_set_body_force(psl_grid* grid, float gx, float gy, float gz);

/* Scalar transport (scalarTransportFunctions.h:10-176, Zhang, Fan & Chen 2011): 27 FP32
 * scalar populations T_q stored and streamed like the flow populations; in
 * psl_apply_local_cell_update they bounce back and mirror with f, take the prescribed
 * concentration where one is given, and collide after the flow collision with relaxation
 * time tauT (applyScalarTransportCollision).  Single grids (the coarse/fine transfer does
 * not carry T); not combined with forcing, moving walls or the learned closure.  T starts
 * at 0. */
int psl_enable_scalar_transport(psl_grid* grid, float tauT);
/* Per-cell prescribed concentration, N host floats, NaN where none (getGivenT with the
 * givenT marker); NULL removes it. */
int psl_set_scalar_given_field(psl_grid* grid, const float* givenT);
/* Scalar populations in logical order [27][N] (host). */
int psl_get_scalar_populations(psl_grid* grid, float* host);
int psl_set_scalar_populations(psl_grid* grid, const float* host);
/* Concentration of every cell, sum_q f_q T_q / rho (FP64), N host doubles. */
int psl_get_scalar(psl_grid* grid, double* host);

/* ---- the per-step update ---- */
/* fillEquilibriumFromFunction (fillEquilibrium.h:1-22) with the sphere case's start hook. */
int psl_fill_equilibrium_sphere(psl_grid* grid, const psl_sphere_case* sc);
/* fillEquilibriumFromFunction with a uniform (rho, u). */
int psl_fill_equilibrium_uniform(psl_grid* grid, float rho, float ux, float uy, float uz);
/* fillEquilibriumFromFunction with a field hook: rho_u is a host array of four
 * logical-order planes [4][N] (rho, ux, uy, uz). */
int psl_fill_equilibrium_field(psl_grid* grid, const float* rho_u);
/* applyStreaming (applyStreaming.h:11-31): updates the 27 periodic shifts; no kernel. */
int psl_apply_streaming(psl_grid* grid);
/* applyLocalCellUpdate (applyLocalCellUpdate.h:1-74): the fused gather / boundary /
 * cumulant+LES collision / scatter kernel. */
int psl_apply_local_cell_update(psl_grid* grid);
/* applyBCPeriodicX / applyBCPeriodicY (boundaryConditions/periodicXY.h:11,57). */
int psl_apply_bc_periodic_x(psl_grid* grid);
int psl_apply_bc_periodic_y(psl_grid* grid);
/* applyCoarseFineGridCommunication (gridRefinementFunctions.h:433-526): one kernel, launched
 * twice in stream order on the coarse grid's stream (restriction onto the coarse ring, then
 * prolongation into the fine shell). */
int psl_apply_coarse_fine_grid_communication(psl_grid* coarse, psl_grid* fine);
/* fillCoarseGridFromFine (gridRefinementFunctions.h:528-535): every coarse cell of
 * [iS+1, iE-1) x [jS+1, jE-1) x [kS+1, kE-1) (inside the refinement block) becomes the
 * rescaled average of its 8 fine children, as the reference does before exporting the coarse
 * level.  Stream-ordered on the coarse grid's stream. */
int psl_fill_coarse_grid_from_fine(psl_grid* coarse, psl_grid* fine);
/* updateGrid recursion of the case driver (flowAroundSphereMainSingle.cu:158-167):
 * streaming + update on grids[level], two steps of level+1, coarse/fine transfer.
 * Kernels go to each grid's stream in call order.  When all levels share one stream and the
 * top grid's refinement block lies at least three cells inside it in z, the top grid's cells
 * away from the block are updated on a lowest-priority stream of the library's own beside the
 * fine updates and the transfer, which run on a highest-priority stream of its own; the
 * grid's stream waits for both before the call returns,
 * so later work on it sees the whole step, and the result is the serial order's bit for bit
 * (not under stream capture, scalar transport or the customised update: serial order there).
 * The periodic shifts are kernel
 * parameters taken when the update is launched, so a step recorded by stream capture replays
 * with that step's shifts: for replaying steps from a CUDA graph use psl_batch_*, whose
 * kernels derive the shifts from a step counter on the device. */
int psl_update_grid(psl_grid** grids, int levels, int level);

/* ---- reductions (FP64) ---- */
/* getSphereDrag (flowAroundSphereMainSingle.cu:99-156): momentum exchange summed over
 * the solid cells of the sphere's bounding box, lattice units of `grid`; force[0] is the
 * drag (x), force[1..2] the y and z components. */
int psl_sphere_force(psl_grid* grid, const psl_sphere_case* sc, double* force3);
/* The same without waiting: enqueued on the grid's stream, `force3` (device memory or pinned
 * host memory, 3 doubles) holds the force once the stream has passed this point
 * (psl_synchronize, or an event recorded after the call).  A step loop that keeps the drag
 * of every step in a pinned host array reads it back every step and synchronises once. */
int psl_sphere_force_async(psl_grid* grid, const psl_sphere_case* sc, double* force3);

/* Torque (r x F, r = cell centre - point3, physical units of the grid) and force of the
 * momentum exchange summed over the solid cells of the box [lo3, hi3), FP64.  Counterpart
 * of getTorque (M35Full/m35Main.cu:176-260, which sums -F_x y + F_y x of forced-velocity
 * cells through its case's forcing hook) for bounce-back bodies; force3 may be NULL. */
int psl_torque(psl_grid* grid, const int* lo3, const int* hi3, const float* point3, double* torque3, double* force3);
/* getTorque (M35Full/m35Main.cu:176-260) on a PS grid: over the forced-velocity cells
 * (marker 0x09) with k >= k_min (the reference's case skips k < 5), the forcing
 * g = rho (u_given - u) of the cell's stored populations -- the library's forced cells are
 * driven toward their given velocity, where the reference's case computes its target in
 * getForcing -- converted to physical force (convertToPhysicalForce: rho_nominal_phys
 * (res/1000)^4 / dt_phys^2), summed as -g_x y + g_y x with (x, y) = (i res + ox, j res + oy),
 * divided by 1000 (N mm -> N m).  FP64 sums (the reference sums in FP32).  force3 (may be
 * NULL): the summed physical forcing. */
int psl_forcing_torque(psl_grid* grid, int k_min, float rho_nominal_phys, double* torque, double* force3);

/* getFlowReportGeneral (flowReportFunctions.h:2-251) over a grid hierarchy (grids[0]
 * coarsest): section plane `plane` at finest-grid index `cut_index`, cropped to the physical
 * bounds {xmin, ymin, zmin, xmax, ymax, zmax}; mean velocity and density over the non-solid
 * pixels and their area (FlowReportStruct, include/types.h:123), summed in FP64. */
#define PSL_PLANE_XY 0
#define PSL_PLANE_ZY 1
#define PSL_PLANE_ZX 2
typedef struct psl_flow_report {
  double ux, uy, uz;
  double rho;
  double area; /* pixel count x (target cell size)^2, physical units (mm^2 in the reference) */
} psl_flow_report;
int psl_get_flow_report(psl_grid* const* grids, int levels, int plane, int cut_index, const float* bounds6,
                        psl_flow_report* report);

/* exportSectionCutPlotGeneral (plotter/exportSectionCutPlot.h:1-88) without the file: the
 * section `plane` at layer `cut` of one grid, V x H pixels (XY: H = Nx, V = Ny; ZY: H = Nz,
 * V = Ny; ZX: H = Nz, V = Nx), each five floats (p, u_horizontal, u_vertical, u_normal,
 * solid) in physical units: p = (rho - 1) rho_nominal_phys soundspeed_phys^2 and
 * u (res / 1000) / dt_phys, rho and u summed in FP32 in getRhoUxUyUz's order
 * (cellFunctions.h:135-155).  Writes V and H; with out == NULL only those.  out holds
 * `capacity` floats on the host (at least 5 V H).  The reference's plotter file is this
 * record behind the header {plot number, V, H, 5} (int32). */
int psl_export_section_cut(psl_grid* grid, int plane, int cut, float rho_nominal_phys, float soundspeed_phys,
                           float* out, long long capacity, int* vertical, int* horizontal);

/* Momentum-exchange force over the solid cells of the box [box_lo3, box_hi3), FP64, on
 * caller-owned buffers, allocating no device memory.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc when they need the force: step loops running
 * inside CUDA stream capture, applications whose device memory belongs to another
 * allocator's pool or a fixed budget, and loops that must not block on an allocation.
 *   populations  device pointer to 27 FP32 rows of row_stride elements (row q holds
 *                population q at the periodic-shift address (cell + shifts27[q]) mod N)
 *   shifts27     host array, each in [0, cell_count); cell_count = nx*ny*nz
 *   markers      device marker bytes (cells of kind PSL_CELL_SOLID are summed)
 *   force3       device pointer; receives (Fx, Fy, Fz) in lattice units
 * Work is queued on cuda_stream (NULL = legacy default stream); nothing is synchronised.
 * Partial sums live in a fixed 24.6 KB array inside the library, held by every GPU that
 * loads it until exit; the box may hold at most 4,194,304 cells (else PSL_ERR_INVALID).
 * Calls outside stream capture look that array up (cudaGetSymbolAddress, current device);
 * calls inside capture reuse the last address found outside it, so make one call outside
 * capture first (after a device reset too).  All calls share the array, so calls whose
 * kernels overlap on the GPU (different streams) race; order them on one stream. */
int psl_momentum_exchange_force_noalloc(const float* populations, long long row_stride, const int* shifts27,
                                        long long cell_count, const uint8_t* markers, int nx, int ny, int nz,
                                        const int* box_lo3, const int* box_hi3, double* force3, void* cuda_stream);

/* ---- learned subgrid closure ----
 * A per-cell MLP (10 features -> 32 -> 32 -> 1, ReLU, softplus output) that replaces the
 * Smagorinsky rate of getOmegaLES (cellFunctions.h:157-198): omega = 1/(3 (nu + nu_t) + 1/2).
 * No reference counterpart.  Features of a cell, from its post-streaming populations after
 * the boundary condition: Pi = (C - rho/3 I)/rho with C the second-order central moments,
 * x = (Pi_xx, Pi_yy, Pi_zz, Pi_xy, Pi_xz, Pi_yz, tr Pi, |Pi|, det Pi / |Pi|^2, width); the
 * network sees (x - in_shift) * in_scale.  Weights are rounded to FP16 on the device and
 * evaluated on the tensor cores with FP32 accumulation. */
typedef struct psl_sgs_mlp {
  float w1[32][10];  /* layer 1: h1 = relu(w1 x' + b1) */
  float b1[32];
  float w2[32][32];  /* layer 2: h2 = relu(w2 h1 + b2) */
  float b2[32];
  float w3[32];      /* output: nu_t = out_scale * softplus(w3 . h2 + b3) */
  float b3;
  float in_shift[10];
  float in_scale[10];
  float out_scale;
} psl_sgs_mlp;
/* Use the closure in psl_apply_local_cell_update of `grid` (NULL: back to Smagorinsky).
 * `filter_width` is the width feature of this grid (its cell size over the coarsest
 * grid's).  Cells fall back to Smagorinsky if the closure's tensor-core step times out
 * (health bit 2). */
int psl_set_sgs_mlp(psl_grid* grid, const psl_sgs_mlp* mlp, float filter_width);
/* Run the closure on every `interval`-th psl_apply_local_cell_update of `grid` only (1, the
 * default: every update).  That update keeps each collided cell's nu_t as FP16 (2 bytes per
 * cell on the device); the updates in between relax with the kept nu_t and skip the
 * network.  16-bit storage (FP16 / BF16) only.  The first update after this call, after
 * psl_set_sgs_mlp, and after populations, markers or shifts are set from outside the update
 * (fill, set, case, fillCoarseGridFromFine) always runs the closure.  No reference
 * counterpart. */
int psl_set_sgs_mlp_interval(psl_grid* grid, int interval);
/* The closure alone on host features (count x 10 raw features) -> nu_t (count floats),
 * through the same tensor-core device code (parity tests). */
int psl_sgs_mlp_infer(const psl_sgs_mlp* mlp, const float* features, int count, float* nu_t);

/* ---- training of the closure (CUDA kernels; samples stay on the device) ----
 * Samples are raw 10-feature rows with an eddy-viscosity target.  The loss is the mean of
 * (softplus(z) - target/out_scale)^2 over a batch; the normalisation (in_shift, in_scale,
 * out_scale) is part of the parameters and is not trained. */
typedef struct psl_sgs_trainer psl_sgs_trainer;
int psl_sgs_trainer_create(long long capacity, psl_sgs_trainer** out);
int psl_sgs_trainer_destroy(psl_sgs_trainer* trainer);
int psl_sgs_trainer_clear(psl_sgs_trainer* trainer);
int psl_sgs_trainer_count(const psl_sgs_trainer* trainer, long long* count);
/* Append n host samples (features n x 10, targets n). */
int psl_sgs_trainer_add_samples(psl_sgs_trainer* trainer, const float* features, const float* targets, long long n);
/* Append samples box-filtered 2x from a fine periodic box: `fine` is (2M+1) x (2M+1) x 2M
 * cells (x/y duplicated faces of applyBCPeriodicX/Y, z periodic through the shift); coarse
 * cell id (row-major, x fastest) is taken when id % stride == phase % stride.  Features are
 * those of the 2:1-averaged, fine-to-coarse rescaled populations; the target is
 * max(0, -tau^d : S / (2 S : S)) with tau the subfilter stress of the 8 children and S the
 * strain rate of the filtered velocity (coarse lattice units). */
int psl_sgs_trainer_add_filtered(psl_sgs_trainer* trainer, psl_grid* fine, int M, int stride, unsigned int phase);
int psl_sgs_trainer_get_samples(psl_sgs_trainer* trainer, long long first, long long n, float* features,
                                float* targets);
int psl_sgs_trainer_set_params(psl_sgs_trainer* trainer, const psl_sgs_mlp* mlp); /* also resets Adam */
int psl_sgs_trainer_get_params(psl_sgs_trainer* trainer, psl_sgs_mlp* mlp);
/* Mean loss over samples [first, first + count) and its gradient (w1..b3 fields of *grad;
 * the normalisation fields are zero), with the current parameters. */
int psl_sgs_trainer_gradient(psl_sgs_trainer* trainer, long long first, long long count, psl_sgs_mlp* grad,
                             double* loss);
/* `steps` Adam steps (beta 0.9 / 0.999) on random batches of `batch` samples; *last_loss
 * is the mean loss of the last batch (before its update). */
int psl_sgs_trainer_train(psl_sgs_trainer* trainer, int steps, int batch, float lr, unsigned int seed,
                          double* last_loss);

/* ---- batched form ----
 * Many independent single-level grids (e.g. sphere cases of different sizes and Reynolds
 * numbers) advanced together: each step is ONE persistent kernel over the tiles of all
 * member grids plus a one-thread kernel that advances a device step counter; the grids'
 * periodic shifts are derived from that counter on the device, so the step is captured
 * once in a CUDA graph and replayed.  No reference counterpart: the reference advances
 * one grid hierarchy per process.  Members must share device and storage, have no
 * refinement block and stay alive while the batch exists (psl_grid_destroy refuses a
 * member grid).  A member grid's own calls (psl_sphere_force, psl_get_populations, ...)
 * stay valid between batch runs: psl_batch_run brings the grid's shifts up to date and
 * orders the grid's stream after the batch's work.  The batch reads each grid's viscosity,
 * Smagorinsky constant and given values when it is created (or retuned); a member grid
 * streamed on its own fails the next psl_batch_run. */
typedef struct psl_batch psl_batch;
typedef struct psl_batch_tuning {
  int threads;       /* threads per CTA: a multiple of 32, at most 256 */
  int tile_cells;    /* consecutive cells per warp tile: a multiple of 32 */
  int blocks_per_sm; /* resident CTAs per SM in the persistent grid; 0: a grid of as many
                        CTAs as the tiles need (each warp's tile loop then runs once) */
  float ms_per_step; /* time per step measured by psl_batch_autotune (0 if not tuned) */
} psl_batch_tuning;
int psl_batch_create(psl_grid* const* grids, int count, psl_batch** out);
int psl_batch_destroy(psl_batch* batch);
/* Advance every member grid by `steps` steps (graph replays on the batch's stream; not
 * synchronised). */
int psl_batch_run(psl_batch* batch, int steps);
int psl_batch_synchronize(psl_batch* batch);
/* The batch's own CUDA stream (created non-blocking), for timing with events. */
int psl_batch_get_stream(const psl_batch* batch, void** stream);
int psl_batch_get_tuning(const psl_batch* batch, psl_batch_tuning* tuning);
int psl_batch_set_tuning(psl_batch* batch, const psl_batch_tuning* tuning);
/* Project-written autotuner: times every candidate launch shape (threads 64/128/256 x
 * warp tiles of 32-1024 cells x {max, max/2, 0} CTAs per SM) over `trial_steps` steps on the
 * batch itself, adopts the fastest and reports it in *chosen.  The populations and the
 * step counter are saved first and restored afterwards, so tuning does not advance the
 * simulation. */
int psl_batch_autotune(psl_batch* batch, int trial_steps, psl_batch_tuning* chosen);

/* ---- data movement ---- */
/* Populations in logical order: host[q * N + cell] = f_q of `cell` (FP32 for every storage). */
int psl_get_populations(psl_grid* grid, float* host);
/* Macroscopic fields in logical order, summed in FP64 from the stored populations
 * (getRhoUxUyUz, cellFunctions.h:135-155): host[0*N + cell] = rho, host[1*N + cell] = ux,
 * host[2*N + cell] = uy, host[3*N + cell] = uz.  No reference counterpart as one call: the
 * reference's exporters evaluate getRhoUxUyUz per cell on the host. */
int psl_get_macroscopic(psl_grid* grid, double* host);
int psl_set_populations(psl_grid* grid, const float* host);
int psl_get_shifts(const psl_grid* grid, int* shifts27);
int psl_set_shifts(psl_grid* grid, const int* shifts27);
int psl_synchronize(psl_grid* grid);
/* Health word of the update kernels (bit 0: non-finite density seen; bit 2: a wait of the
 * learned closure timed out; bit 1 is not used); read and clear. */
int psl_check_health(psl_grid* grid, unsigned int* flags);

/* ---- single-cell entry points (unit parity of the device functions) ----
 * op: 0 collision (args: nu, cs), 1 rescale (a0: coarse_to_fine), 2 MBBC (args: rho,u),
 * 3 restoreRho, 4 restoreUxUyUz, 5 restoreRhoUxUyUz, 6 mirror, 7 forced collision
 * (args: nu, cs, gx, gy).  f: count x 27 host floats (in/out), args: count x 4 host floats;
 * a0: normal index for the boundary ops. */
int psl_debug_cells(int op, int a0, float* host_f, const float* host_args, int count);

const char* psl_last_error(void);
const char* psl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PSL_H */
