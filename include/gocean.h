/*
 * gocean.h -- C ABI of the B200-native CDKLM16 time step.
 *
 * Every entry point returns GO_OK (0) on success and a negative status
 * otherwise; go_last_error() gives the message of the last failure on the
 * calling thread.  No exception crosses this boundary.  Device pointers are
 * caller-owned (the library never frees them); pitches are in BYTES, as in
 * the reference's PyCUDA calls.  Entry points that take a stream are
 * asynchronous on that stream unless their comment says otherwise.  A
 * go_domain handle is not thread-safe: use one handle per host thread.
 *
 * Reference interfaces replaced (paths inside metno/gpu-ocean):
 *   gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:429   cdklm_swe_2D
 *   gpu_ocean/SWESimulators/gpu_kernels/max_dt.cu:42,147         per_block_max_dt, max_dt_reduction
 *   gpu_ocean/SWESimulators/gpu_kernels/boundary_kernels.cu:35,76  periodicBoundary_NS/EW
 *   gpu_ocean/SWESimulators/gpu_kernels/boundary_kernels.cu:121-246 *_boundary_intersections_*
 *   gpu_ocean/SWESimulators/gpu_kernels/initBm_kernel.cu:38      initBm
 *   gpu_ocean/SWESimulators/CDKLM16.py:179-228   #defines baked into the JIT module
 *   gpu_ocean/SWESimulators/CDKLM16.py:494-598   step() RK2 launch sequence
 */
#ifndef GOCEAN_H
#define GOCEAN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GO_OK 0
#define GO_ERR_INVALID (-1)     /* bad argument (shape, pointer, pitch, code) */
#define GO_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define GO_ERR_UNSUPPORTED (-3) /* valid in the reference, not built here */
#define GO_ERR_NOMEM (-4)

/* Boundary codes, gpu_ocean/SWESimulators/Common.py:824-857. */
#define GO_BC_WALL 1
#define GO_BC_PERIODIC 2
#define GO_BC_FLOW_RELAXATION 3   /* open: relaxation towards an exterior solution over a sponge */
#define GO_BC_LINEAR_SPONGE 4     /* open: linear between the outer and inner sponge edges */

/* Bottom friction law.  QUADRATIC is what the reference kernel compiles
 * (CDKLM16_kernel.cu:884-900 without use_linear_friction); LINEAR is the
 * #ifdef branch at CDKLM16_kernel.cu:885. */
#define GO_FRICTION_QUADRATIC 0
#define GO_FRICTION_LINEAR 1

/* Device status word bits (go_domain_status). */
#define GO_STATUS_NONFINITE 0x1u /* a written cell held NaN or Inf */
#define GO_STATUS_ADJ_SCOPE 0x2u /* reserved: raised by earlier adjoint builds that
                                   covered no land or shallow cells */
#define GO_STATUS_TIMEOUT 0x4u   /* a bounded wait in a step kernel gave up
                                   (a TMA tile that never arrived) */
#define GO_STATUS_BOUNDS 0x8u    /* the checked-index build (lib/libgocean_debug.so,
                                   built with -DGO_DEBUG_BOUNDS) met a global or
                                   shared index outside its array and skipped it */

typedef struct go_domain go_domain;

/* Scheme constants of one domain: what the reference bakes into its JIT
 * module as #defines (CDKLM16.py:179-191) plus the boundary codes it packs
 * per launch (CDKLM16.py:620-624). */
typedef struct go_domain_desc {
    int nx, ny;            /* interior cells; arrays are (ny+4) x (nx+4) */
    float dx, dy;          /* DX, DY */
    float g;               /* GRAV */
    float r;               /* FRIC */
    float theta;           /* THETA (minmod), default 1.3 */
    float desing_eps;      /* KPSIMULATOR_DESING_EPS, default 0.1 */
    float flux_slope_eps;  /* KPSIMULATOR_FLUX_SLOPE_EPS, default 0.1 */
    float depth_cutoff;    /* KPSIMULATOR_DEPTH_CUTOFF, default 1e-5 */
    int rk_order;          /* 2 (Heun); 1 = forward Euler */
    int bc_north, bc_east, bc_south, bc_west; /* GO_BC_* */
    int friction_law;      /* GO_FRICTION_* */
    float north_x, north_y;/* (sin a, cos a) of a constant grid angle a */
} go_domain_desc;

/* Create / destroy a domain handle.  Allocates a small device table
 * (Coriolis per row) and a status word. */
int go_domain_create(const go_domain_desc* desc, go_domain** out);
int go_domain_destroy(go_domain* d);

/* Coriolis parameter per ghost-inclusive row j = 0..ny+3, as the reference
 * samples its f texture at cell centres (CDKLM16_kernel.cu:49-58;
 * texture built at CDKLM16.py:310-351).  n == 1 sets an f-plane.
 * Synchronous host->device copy. */
int go_domain_set_coriolis(go_domain* d, const float* f_rows_host, int n);

/* Uniform wind stress (kinematic, N/m^2 / rho_w): current and next values
 * of the reference's 1x1 wind textures (common.cu:601-650).  The kernel
 * forms wind_t*next + (1-wind_t)*current as the reference does. */
int go_domain_set_wind_uniform(go_domain* d, float x_cur, float x_next,
                               float y_cur, float y_next);

/* Per-cell wind stress: four device arrays of ny x nx interior cells
 * (caller-owned, pitch in bytes), the reference's wind textures sampled at
 * each cell.  Pass NULL to return to uniform wind. */
int go_domain_set_wind_field(go_domain* d, const float* x_cur, const float* x_next,
                             const float* y_cur, const float* y_next, int pitch);

/* ---------------------------------------------------------------------
 * Drifters (gpu_ocean/SWESimulators/GPUDrifterCollection.py) and flow
 * observation at drifter cells.  positions: (num_drifters + 1) rows of
 * (x, y) floats in metres from the south-west interior corner (the last row
 * is the observation's position), device, pitch in bytes.
 * --------------------------------------------------------------------- */

/* A wind field (host, h rows x w columns) as a bilinear, clamped,
 * normalised texture for wind drift (GPUDrifterCollection.py:120-176); the
 * handle is passed to go_drift_passive.  go_wind_texture_destroy frees it. */
int go_wind_texture_create(const float* field, int w, int h, uint64_t* texture);
int go_wind_texture_destroy(uint64_t texture);

/* One Euler step of every drifter and the observation position with the
 * flow velocity bilinear between the four nearest cell centres, plus
 * wind_drift_factor x the wind (textures: X current, X next, Y current,
 * Y next; may be NULL when the factor is 0), then the periodic wrap
 * (passiveDrifterKernel, gpu_ocean/SWESimulators/gpu_kernels/
 * driftKernels.cu:108-207; called from GPUDrifterCollection.py:209-232).
 * Cells outside the arrays are clamped (the reference reads there). */
int go_drift_passive(void* stream, int nx, int ny, float dx, float dy, float dt, int x_zero_cell,
                     int y_zero_cell, const float* eta, int eta_pitch, const float* hu, int hu_pitch,
                     const float* hv, int hv_pitch, const float* Hm, int Hm_pitch, int periodic_north_south,
                     int periodic_east_west, int num_drifters, float* positions, int positions_pitch,
                     float sensitivity, float wind_t, float wind_drift_factor, const uint64_t* wind_textures);

/* Periodic wrap of every position (enforceBoundaryConditions,
 * driftKernels.cu:211-250). */
int go_drift_enforce_bc(void* stream, float domain_size_x, float domain_size_y, int periodic_north_south,
                        int periodic_east_west, int num_drifters, float* positions, int positions_pitch);

/* (hu, hv) of the cell under each drifter into observation (device,
 * num_drifters rows of 2 floats, pitch in bytes) (observeUnderlyingFlow,
 * gpu_ocean/SWESimulators/gpu_kernels/observationKernels.cu:29-81). */
int go_observe_flow(void* stream, int nx, int ny, float dx, float dy, int x_zero_cell, int y_zero_cell,
                    const float* hu, int hu_pitch, const float* hv, int hv_pitch, int num_drifters,
                    const float* positions, int positions_pitch, float* observation, int observation_pitch);

/* ---------------------------------------------------------------------
 * Open boundaries (codes 3 and 4; gpu_ocean/SWESimulators/gpu_kernels/
 * boundary_kernels.cu:264-539, Common.py:1073-1309).  go_boundary_condition
 * and go_cdklm_step (after each RK stage) then run the reference's ghost
 * sequence: north-south periodic copy or open kinds, then east-west.
 * --------------------------------------------------------------------- */

/* Sponge widths in ghost-inclusive cells from the outer edge (the
 * reference's spongeCells). */
int go_domain_set_sponge(go_domain* d, int north, int east, int south, int west);

/* A float4 (h, hu, hv, unused) texture of w x h texels (host, row-major)
 * for the flow relaxation's exterior solution, bilinear, clamped,
 * normalised (Common.py:1098-1103).  Free with go_wind_texture_destroy. */
int go_bc_texture_create(const float* texels, int w, int h, uint64_t* texture);

/* Exterior solution of the flow relaxation: textures {NS current, NS next,
 * EW current, EW next} (NS: row 0 south, row 1 north; EW: column 0 west,
 * column 1 east) and the time weight bc_t in [0, 1] used by the following
 * launches (BoundaryConditionsArakawaA.update_bc_values,
 * Common.py:1073-1216).  The caller keeps the textures alive. */
int go_domain_set_open_bc(go_domain* d, const uint64_t* textures, float bc_t);

/*
 * Stochastic model error (OceanStateNoise): SOAR-correlated perturbations of
 * eta on a coarse grid, geostrophically balanced hu and hv.  Replaces the
 * kernels of gpu_ocean/SWESimulators/gpu_kernels/ocean_noise.cu and
 * reductions.cu as gpu_ocean/SWESimulators/OceanStateNoise.py:343-571
 * launches them.  All arrays are device memory, row-major, pitches in bytes;
 * every call is asynchronous on its stream.
 */

/* LCG random numbers (ocean_noise.cu:81-200, OceanStateNoise.py:343-372):
 * each of the seed_nx x seed_ny 64-bit seeds advances twice and writes a
 * pair of N(0,1) numbers (normal != 0, Box-Muller) or U[0,1) numbers into
 * columns 2i, 2i+1 of its row of the random_nx-wide buffer. */
int go_noise_lcg(void* stream, int normal, int seed_nx, int seed_ny, int random_nx, uint64_t* seed,
                 int seed_pitch, float* random, int random_pitch);

/* XORWOW generators (the reference's default, pycuda's
 * XORWOWRandomNumberGenerator, OceanStateNoise.py:160-168): bytes of one
 * generator state, seeding of n generators (subsequence g for generator g),
 * and a fill of an nx x ny field with N(0,1) (normal != 0) or U(0,1]. */
size_t go_noise_xorwow_state_bytes(void);
int go_noise_xorwow_init(void* stream, uint64_t seed, int n_generators, void* states);
int go_noise_xorwow_fill(void* stream, int normal, int n_generators, void* states, int nx, int ny, float* out,
                         int out_pitch);

/* SOAR covariance with cut-off 2 applied to the random field, written (or
 * added, additive != 0) times perturbation_scale to all (coarse_nx + 4) x
 * (coarse_ny + 4) cells of the coarse buffer (ocean_noise.cu:249-372).  The
 * random field is coarse_nx (+8 unless periodic east-west) by coarse_ny
 * (+8 unless periodic north-south). */
int go_noise_soar(void* stream, int coarse_nx, int coarse_ny, float coarse_dx, float coarse_dy, float soar_q0,
                  float soar_L, float perturbation_scale, int periodic_north_south, int periodic_east_west,
                  const float* random, int random_pitch, float* coarse, int coarse_pitch, int additive);

/* Adds the coarse perturbation (coarse grid = model grid) to eta and the
 * geostrophically balanced d_hu, d_hv to hu, hv in the interior cells;
 * cells with a land corner in Hi become 0 (ocean_noise.cu:379-508).  The
 * angle and Coriolis textures are handles of go_wind_texture_create (the
 * reference's angle_tex and coriolis_f_tex: bilinear, clamped, normalised
 * over the ghost-inclusive grid); the Coriolis texture is read where f == 0.
 * y0_reference_cell is accepted and unused, as in the reference.  The cells
 * perturbed are the interior cells the reference's 16 x 16-block launch
 * reaches from the ghost offset (all of them for ghost offset 2). */
int go_noise_geostrophic(void* stream, int nx, int ny, float dx, float dy, int ghost_x, int ghost_y, float g,
                         float f, float beta, float y0_reference_cell, const float* coarse, int coarse_pitch,
                         float* eta, int eta_pitch, float* hu, int hu_pitch, float* hv, int hv_pitch,
                         const float* Hi, int Hi_pitch, float land_value, uint64_t angle_texture,
                         uint64_t coriolis_texture);

/* As go_noise_geostrophic with a coarser perturbation grid: d_eta is the
 * bicubic interpolation of the coarse buffer, shifted by (offset_i,
 * offset_j) model cells; land cells are left unchanged
 * (ocean_noise.cu:522-772, common.cu:696-819). */
int go_noise_bicubic(void* stream, int nx, int ny, int ghost_x, int ghost_y, float dx, float dy, int coarse_nx,
                     int coarse_ny, int coarse_ghost_x, int coarse_ghost_y, float coarse_dx, float coarse_dy,
                     int offset_i, int offset_j, float g, float f, float beta, float y0_reference_cell,
                     const float* coarse, int coarse_pitch, float* eta, int eta_pitch, float* hu, int hu_pitch,
                     float* hv, int hv_pitch, const float* Hi, int Hi_pitch, float land_value,
                     uint64_t angle_texture, uint64_t coriolis_texture);

/* The model error of an ensemble, batched across members: every member's
 * draws, SOAR field and balanced perturbation (coarse grid = model grid, one
 * field, not additive) in one launch per kernel, each member bit for bit
 * what go_noise_lcg (or go_noise_xorwow_fill), go_noise_soar and
 * go_noise_geostrophic give it alone.  Replaces the per-member perturbSim of
 * the reference's ensembles (OceanNoiseEnsemble.py:506-531 through
 * CDKLM16.py:580-582).  The members share the grid, the boundary kinds, the
 * generator kind and soar_L; each has its own buffers and parameters. */
typedef struct go_noise_member {
    uint64_t* seed;           /* LCG seeds, seed_ny x seed_nx (NULL with XORWOW) */
    void* xorwow_states;      /* XORWOW states (NULL with LCG) */
    float* random;            /* random field */
    float* coarse;            /* coarse buffer, (ny+4) x (nx+4) */
    float* eta;
    float* hu;
    float* hv;
    const float* Hi;          /* (ny+5) x (nx+5) */
    uint64_t angle_texture;   /* go_wind_texture_create handles */
    uint64_t coriolis_texture;
    int seed_pitch, random_pitch, coarse_pitch, eta_pitch, hu_pitch, hv_pitch, Hi_pitch; /* bytes */
    int n_generators;         /* XORWOW generators */
    float soar_q0, g, f, beta, land_value, reserved;
} go_noise_member;

typedef struct go_noise_batch go_noise_batch;

/* Checks the members (host array of n) against the shared geometry and
 * copies their descriptors to the device (synchronous). */
int go_noise_batch_create(const go_noise_member* members, int n, int nx, int ny, float dx, float dy,
                          int ghost_x, int ghost_y, float soar_L, int periodic_north_south,
                          int periodic_east_west, int use_lcg, go_noise_batch** out);
int go_noise_batch_destroy(go_noise_batch* b);

/* One perturbation of every member: new normal draws (update_random_field
 * != 0), SOAR with amplitude (float)((double)soar_q0 x q0_scale) and
 * perturbation_scale, then the balance. */
int go_noise_batch_perturb(go_noise_batch* b, void* stream, double q0_scale, float perturbation_scale,
                           int update_random_field);

/* result[0] = sum a^2 over an nx x ny field; with b also result[1] = sum
 * b^2 and result[2] = sum a b (reductions.cu squareSum, squareSumDouble).
 * Accumulates in double, deterministic order.  scratch: device bytes of
 * go_noise_reduce_scratch_bytes(), zeroed once before first use (the call
 * leaves it ready for the next). */
size_t go_noise_reduce_scratch_bytes(void);
int go_noise_square_sums(void* stream, int nx, int ny, const float* a, int a_pitch, const float* b, int b_pitch,
                         float* result, void* scratch, size_t scratch_bytes);

/* nu <- nu made perpendicular to xi and rescaled to its former norm, from
 * the three sums of go_noise_square_sums (ocean_noise.cu:206-241). */
int go_noise_make_perpendicular(void* stream, int nx, int ny, const float* xi, int xi_pitch, float* nu,
                                int nu_pitch, const float* reduction);

/* North vector (sin a, cos a) of a constant grid angle a, computed on the
 * device with sinf/cosf as the reference's kernel forms it from its angle
 * texture (gpu_ocean/SWESimulators/gpu_kernels/CDKLM16_kernel.cu:68-77), for
 * go_domain_desc.north_x / north_y.  Synchronous (a set-up call). */
int go_north_vector(float angle, float* north_x, float* north_y);

/* Samples a wind stress array (host, h rows x w columns, row-major) at the
 * interior cells of an nx x ny grid into out (device, ny rows, pitch in
 * bytes) the way the reference's kernel reads its wind textures
 * (gpu_ocean/SWESimulators/gpu_kernels/common.cu:616-650,
 * gpu_ocean/SWESimulators/Simulator.py:171-213): one bilinear, clamped,
 * normalised texture lookup per cell at ((i + 2.5) / nx, (j + 2.5) / ny),
 * so the values equal the reference's.  Synchronises the stream (a set-up
 * call, once per wind interval).  Hand the result to
 * go_domain_set_wind_field. */
int go_sample_wind(void* stream, const float* field, int w, int h, int nx, int ny, float* out,
                   int out_pitch);

/* Launch shape of the step kernel: shape 0 = 192 threads x 2 blocks/SM,
 * 1 = 192 x 3, 2 = 128 x 4, 3 = 256 x 2, 4 = 128 x 5; 5 = 128 x 5, 6 = 96 x 6
 * and 7 = 192 x 3 with each thread reading its column's inputs two rows
 * ahead through shared memory (cp.async).  Default: when the grid needs more
 * than one wave of blocks, shape 5, or 6 where 96-wide blocks compute at
 * least 4% fewer columns; else 4.  Each block marches down a strip of
 * rows_per_block rows (0 = automatic: the height in {2, 4, 8, 16, 24} that
 * minimises whole waves of blocks times the strip length plus its 4
 * recomputed halo rows).  Chosen by the autotuner; every shape computes
 * identical results. */
int go_domain_set_launch(go_domain* d, int shape, int rows_per_block);
/* Shape 8: the column-pair kernel.  Blocks of 64 threads, each thread two
 * adjacent columns in packed FP32x2 arithmetic (sm_100 FADD2/FFMA2), inputs
 * of the boundary-free blocks staged through shared memory by TMA tile
 * loads; the boundary frame runs as a second kernel on a high-priority
 * stream beside them.  Arrays whose base or pitch is not a multiple of 16
 * bytes take the boundary path everywhere. */
#define GO_SHAPE_PAIR 8

/* How quotients are evaluated.  EXACT keeps every '/' of the reference
 * kernel (div.full.f32 under its --prec-div=false).  RCP (the default)
 * multiplies by reciprocals (rcp.approx.ftz) of shared denominators; on
 * B200 the two give bit-identical results over the tested ranges, and both
 * reproduce the reference kernel bit for bit on the parity workloads. */
#define GO_ARITH_EXACT 0
#define GO_ARITH_RCP 1
int go_domain_set_arith(go_domain* d, int mode);

/* Self-check of the two quotient modes: writes a[i] / b[i] as the stage
 * kernel evaluates it under GO_ARITH_EXACT to q_div and under GO_ARITH_RCP
 * to q_rcp, for n device floats each (compiled with the stage kernel's
 * flags).  No counterpart in the reference; tests use it to pin the
 * equivalence of the two modes over the scheme's denominators. */
int go_check_quotients(void* stream, const float* a, const float* b, int n, float* q_div, float* q_rcp);

/* Whether the bathymetry may hold land (corners equal to the land value,
 * Common.py:1333-1337).  1 (the default) keeps every land test of the
 * reference kernel; 0 asserts there is none and skips them. */
int go_domain_set_land(go_domain* d, int may_have_land);

/* Bathymetry set-up (Common.py:1319-1389): fixes the ghost corners of Hi
 * in place (periodic wrap or wall mirror, boundary_kernels.cu:121-246) and
 * writes Bm = mean of the wet corners, land_value where all four are land
 * (initBm_kernel.cu:38-107).  Hi is (ny+5) x (nx+5), Bm (ny+4) x (nx+4). */
int go_init_bathymetry(go_domain* d, void* stream, float* Hi, int Hi_pitch,
                       float* Bm, int Bm_pitch, float land_value);

/* Periodic ghost-cell refresh, north-south then east-west
 * (Common.py:1219-1239 -> boundary_kernels.cu:35-110).  Walls: no-op. */
int go_boundary_condition(go_domain* d, void* stream, float* eta, float* hu,
                          float* hv, int pitch);

/* One Runge-Kutta sub-step: the drop-in for one cdklm_swe_2D launch
 * (CDKLM16_kernel.cu:429-1006) followed by the periodic ghost refresh of
 * its output that CDKLM16.step() issues after it (CDKLM16.py:539-540,
 * 585-586).  Argument meaning follows the kernel: *0 is the input state,
 * *1 the output; rk_step 1 reads Q^n from the output buffer at each cell
 * and writes Q^{n+1} over it.  The three input arrays must share one
 * pitch, as must the three outputs.  Hm is accepted for ABI parity and not
 * read: the cell bathymetry is derived from Hi in the kernel.  The packed
 * boundary code (north<<24 | south<<16 | east<<8 | west) must match the
 * domain's. */
int go_cdklm_swe_2D(go_domain* d, void* stream, float dt, int rk_step,
                    const float* eta0, int eta0_pitch, const float* hu0, int hu0_pitch,
                    const float* hv0, int hv0_pitch,
                    float* eta1, int eta1_pitch, float* hu1, int hu1_pitch,
                    float* hv1, int hv1_pitch,
                    const float* Hi, int Hi_pitch, const float* Hm, int Hm_pitch,
                    float land_value, float wind_stress_t, int boundary_conditions);

/* n_steps Heun RK2 steps of size dt (CDKLM16.py:533-544 + 585-586):
 * stage 0 h0 -> h1, stage 1 h1 -> h0 (in place).  The state ends in h0;
 * h1 holds the last Q*. */
int go_cdklm_step(go_domain* d, void* stream, int n_steps, float dt, float wind_stress_t,
                  float* eta0, float* hu0, float* hv0, int pitch0,
                  float* eta1, float* hu1, float* hv1, int pitch1,
                  const float* Hi, int Hi_pitch, float land_value);

/* Exact CFL limit min over wet interior cells of 0.25*dx/|u +- c| and
 * 0.25*dy/|v +- c| (max_dt.cu:42-194 without its block-reduction gap).
 * Writes one float to dt_dev (device).  Not scaled by the Courant number
 * (CDKLM16.updateDt multiplies on the host, CDKLM16.py:739). */
int go_max_dt(go_domain* d, void* stream, const float* eta, const float* hu,
              const float* hv, int pitch, const float* Bm, int Bm_pitch,
              float land_value, float* dt_dev);

/* ---------------------------------------------------------------------
 * Batched stepping.  No counterpart entry point in the reference: it
 * replaces the member-by-member loops of its ensembles
 * (OceanNoiseEnsemble.py:506-531, OceanModelEnsemble.py:105-117,
 * EnsembleFromFiles.py:302-324), which call CDKLM16.step once per member.
 * One launch per RK stage covers every member through a packed list of
 * (member, column block, row block) tiles; members may have different
 * sizes, bathymetry and time steps but must share the kernel variant
 * (friction law, grid angle, uniform vs per-cell wind).
 * --------------------------------------------------------------------- */
typedef struct go_batch go_batch;

/* Batch over n existing domain handles (not owned; keep them alive). */
int go_batch_create(go_domain* const* members, int n, go_batch** out);
int go_batch_destroy(go_batch* b);

/* State buffers, bathymetry and time step of member m (as go_cdklm_step). */
int go_batch_set_member(go_batch* b, int m, float dt, float* eta0, float* hu0, float* hv0, int pitch0,
                        float* eta1, float* hu1, float* hv1, int pitch1, const float* Hi, int Hi_pitch,
                        float land_value, float wind_stress_t);

/* Launch shape (as go_domain_set_launch) and persistent grid size: blocks
 * = 0 launches one block per tile, blocks > 0 that many blocks walking the
 * tile list.  Default: 32-row strips, one block per tile, and the shape
 * chosen as for a single grid from the column work of all members. */
int go_batch_set_launch(go_batch* b, int shape, int rows_per_block, int blocks);
int go_batch_set_arith(go_batch* b, int mode);

/* New per-member time steps (n floats, host).  A captured graph reads them
 * at its next launch; no re-capture is needed. */
int go_batch_set_dt(go_batch* b, void* stream, const float* dt_host);

/* Number of tiles of the packed list (commits pending member changes). */
int go_batch_tiles(go_batch* b, int* ntiles);

/* n_steps RK2 steps of every member: 2 launches per step. */
int go_batch_step(go_batch* b, void* stream, int n_steps);

/* Capture n_steps batched steps on stream (non-default) into a CUDA graph,
 * and replay it; steps_done (optional) receives n_steps. */
int go_batch_graph_capture(go_batch* b, void* stream, int n_steps);
int go_batch_graph_launch(go_batch* b, void* stream, int* steps_done);

/* ---------------------------------------------------------------------
 * Adjoint (reverse mode) of the RK2 step.  No counterpart in the
 * reference, which has no adjoint.  Built for north-up grids (other grid
 * angles are rejected with GO_ERR_UNSUPPORTED); land, dry and
 * desingularised cells are differentiated through the branch the forward
 * takes (land and dry cells are constants of the stage, desingularised
 * cells use u = hu / D(h), D the desingularisation denominator).  The
 * Hi passed must be the one the forward read, and a domain with land needs
 * go_domain_set_land(d, 1) for go_traj_step as for the forward.
 * A state is three device arrays of (ny+4) x (nx+4) floats sharing a pitch
 * in bytes; adjoint states hold their values at the interior cells.
 * --------------------------------------------------------------------- */
typedef struct go_state {
    float* eta;
    float* hu;
    float* hv;
    int pitch;             /* bytes */
} go_state;

/* Launch form of the adjoint stage: GO_ADJ_TILE (one block per tile of 32
 * columns and rows_per_strip = 8, 12 or 16 rows, 0 = automatic: 8 below
 * ~350 k cells, else 16; the forward is recomputed with a 3-cell halo),
 * GO_ADJ_MARCH64 / GO_ADJ_MARCH128 (one thread per column, blocks of 64 or
 * 128 columns marching up strips of rows_per_strip rows, 0 = automatic),
 * GO_ADJ_AUTO (the default: the tile form below ~1 M cells, else marching,
 * 64 up to 1024 columns).  The forms agree to FP32 rounding. */
#define GO_ADJ_AUTO 0
#define GO_ADJ_TILE 1
#define GO_ADJ_MARCH64 2
#define GO_ADJ_MARCH128 3
int go_domain_set_adjoint_launch(go_domain* d, int kind, int rows_per_strip);

/* One forward step that keeps its stages: q_star = stage 0 of q_n,
 * q_next = stage 1 (reading Q^n from q_n instead of its output buffer).
 * Bit-identical to go_cdklm_step; q_n is left unchanged. */
int go_traj_step(go_domain* d, void* stream, float dt, float wind_stress_t,
                 const go_state* q_n, const go_state* q_star, const go_state* q_next,
                 const float* Hi, int Hi_pitch, float land_value);

/* Adjoint of one RK stage (the reverse of go_cdklm_swe_2D) given its input
 * q_in, its stored output q_out and lam_out, the adjoint of the output.
 * Writes lam_in, the adjoint of the input (ghost-cell adjoint moved to the
 * interior cells the ghosts mirror or wrap).  rk_step 1 also writes lam_qn,
 * the adjoint of Q^n; for rk_step 0 a non-NULL lam_qn is added to lam_in.
 * lam_wx/lam_wy (optional, ny x nx, pitch in bytes) accumulate the adjoint
 * of the per-cell wind stress. */
int go_adjoint_stage(go_domain* d, void* stream, int rk_step, float dt,
                     const go_state* q_in, const go_state* q_out, const go_state* lam_out,
                     const go_state* lam_in, const go_state* lam_qn,
                     float* lam_wx, float* lam_wy, int wind_pitch,
                     const float* Hi, int Hi_pitch);

/* Adjoint of one RK2 step: lam_n = (dQ^{n+1}/dQ^n)^T lam_next from the
 * step's q_n, q_star, q_next (as go_traj_step stores them).  lam_n may be
 * lam_next (in place); the two scratch states must be distinct from both. */
int go_adjoint_step(go_domain* d, void* stream, float dt,
                    const go_state* q_n, const go_state* q_star, const go_state* q_next,
                    const go_state* lam_next, const go_state* lam_n,
                    const go_state* scratch_star, const go_state* scratch_qn,
                    float* lam_wx, float* lam_wy, int wind_pitch,
                    const float* Hi, int Hi_pitch);

/* Batched adjoint step: every member's lam <- (dQ^{n+1}/dQ^n)^T lam in four
 * launches (stage-1 adjoint of all members over a packed tile list, ghost
 * fold, stage-0 adjoint, fold).  Members keep fixed buffers, so a captured
 * CUDA graph can replay the step; they must share the friction law.
 * set_member's buffers mean what go_adjoint_step's mean (lam in place). */
typedef struct go_adjoint_batch go_adjoint_batch;
int go_adjoint_batch_create(go_domain* const* members, int n, go_adjoint_batch** out);
int go_adjoint_batch_destroy(go_adjoint_batch* b);
/* Marching blocks of 64 or 128 columns and strips of rows (0 = 32). */
int go_adjoint_batch_set_launch(go_adjoint_batch* b, int block_columns, int rows_per_strip);
int go_adjoint_batch_set_member(go_adjoint_batch* b, int m, float dt,
                                const go_state* q_n, const go_state* q_star, const go_state* q_next,
                                const go_state* lam, const go_state* scratch_star,
                                const go_state* scratch_qn, float* lam_wx, float* lam_wy,
                                int wind_pitch, const float* Hi, int Hi_pitch);
int go_adjoint_batch_step(go_adjoint_batch* b, void* stream);

/* Observation misfit J += sum w_eta (eta - eta_obs)^2 + w_vel ((hu - hu_obs)^2
 * + (hv - hv_obs)^2) over n_obs interior cells of an nx x ny grid (device
 * int pairs (i, j), 0-based interior indices, pairs outside the interior
 * are skipped; device float triples of observed values), accumulated in
 * FP64 into J_dev. */
int go_obs_misfit(void* stream, const go_state* q, int nx, int ny, int n_obs,
                  const int* obs_ij, const float* obs_values, float w_eta, float w_vel,
                  double* J_dev);

/* Adds dJ/dQ of that misfit to lam at the observed cells. */
int go_obs_adjoint(void* stream, const go_state* q, const go_state* lam, int nx, int ny,
                   int n_obs, const int* obs_ij, const float* obs_values, float w_eta,
                   float w_vel);

/* ---------------------------------------------------------------------
 * Allocation-free step.  No counterpart in the reference (its CDKLM16
 * allocates through pycuda).  The go_cdklm_step of a domain described by
 * desc, with a uniform wind (wind_x, wind_y) and no domain handle, for
 * callers that cannot call cudaMalloc: the Coriolis table (n_rows = 1 or
 * ny+4 floats, host) and the status word live in a static __device__
 * array of 65,808 bytes per device, so ny + 4 <= 16388 (larger ny is
 * rejected with GO_ERR_INVALID).  The status word is cleared at the start
 * of each call; status_out (optional, host) receives it after a stream
 * synchronize.  The first call on each device (and the first after a
 * cudaDeviceReset, which gives the device a new context) looks up the
 * array's address and may load the module: make it outside stream capture.
 * Calls on one device share the array, so overlapping calls race: order
 * them on one stream or one host thread.  With n_rows = ny+4 the table is
 * copied from f_rows_host by cudaMemcpyAsync on the stream: when that host
 * memory is page-locked the copy runs after the call returns, so keep the
 * table unchanged until the stream has passed the call.  The input's
 * periodic ghost cells must be current (the step kernels refresh them for
 * their outputs; CDKLM16.step refreshes them once at t = 0, this call does
 * not).
 * --------------------------------------------------------------------- */
int go_cdklm_step_static(const go_domain_desc* desc, void* stream, const float* f_rows_host,
                         int n_rows, float wind_x, float wind_y, int n_steps, float dt,
                         float* eta0, float* hu0, float* hv0, int pitch0,
                         float* eta1, float* hu1, float* hv1, int pitch1,
                         const float* Hi, int Hi_pitch, float land_value, uint32_t* status_out);

/* ---------------------------------------------------------------------
 * Model error: eta += std_dev * (Gaussian random field with correlation
 * exp(-r^2 / (2 L^2)), L = corr_cells, unit variance), periodic in x (and
 * in y when north/south are periodic).  Normals come from Philox4x32-10
 * (Salmon et al., SC'11) keyed by (key0, key1) with counter (index / 4,
 * event, 0, 0) and Box-Muller; a separable Gaussian filter correlates them.
 * The same (keys, event) give the same field in the single and the batched
 * form.  No counterpart in the reference (its OceanStateNoise draws model
 * error by another method).
 * --------------------------------------------------------------------- */

/* Scratch floats go_grf_perturb needs for an nx x ny grid (0 if invalid). */
size_t go_grf_scratch_floats(int nx, int ny, float corr_cells);

/* Adds the field for (key0, key1, event) to the interior of eta (device,
 * (ny+4) x (nx+4), pitch in bytes) and rewrites its periodic ghost images. */
int go_grf_perturb(go_domain* d, void* stream, float* eta, int pitch, uint32_t key0,
                   uint32_t key1, uint32_t event, float std_dev, float corr_cells,
                   float* scratch, size_t scratch_floats);

/* go_max_dt for every member of the batch in one launch, on the members'
 * current state (h0): writes n floats to dt_dev (device), member order.
 * The cell-mean bathymetry is recomputed from the corners as
 * go_init_bathymetry computes it, so each value equals go_max_dt's.
 * Replaces the per-member CFL reductions of the reference's ensembles
 * (gpu_ocean/SWESimulators/OceanModelEnsemble.py:112-125, one updateDt
 * per particle). */
int go_batch_max_dt(go_batch* b, void* stream, float* dt_dev);

/* Scratch floats go_batch_grf_perturb needs for all members. */
size_t go_batch_grf_scratch_floats(go_batch* b, float corr_cells);

/* go_grf_perturb for every member m of the batch, keys (key0, m), on the
 * members' current state (h0), in two launches. */
int go_batch_grf_perturb(go_batch* b, void* stream, uint32_t key0, uint32_t event,
                         float std_dev, float corr_cells, float* scratch,
                         size_t scratch_floats);

/* The ensemble event loop on the device, in one launch of a CUDA graph with
 * two nested WHILE nodes: for events e = first_event .. first_event +
 * n_events - 1, every member advances `interval` model seconds at the
 * common dt by the reference's step(t_end) rule (whole steps while one
 * fits, then one step of float32(t_end - t_now); CDKLM16.py:494-598), gets
 * go_batch_grf_perturb's model error (key0, e, std_dev, corr_cells), and
 * the common dt becomes float32(courant x the least go_batch_max_dt limit)
 * -- what the reference's ensembles do member by member from the host
 * (OceanNoiseEnsemble.py:506-531), with no host round trip per event.
 * dt is the members' common dt on entry; t_members (n doubles, member
 * order) their model times, advanced in place by the float64 sum of the
 * steps each took; *steps_out the steps per member, *dt_out the common dt
 * on return (also the members' batch dt).  Every member sees the same
 * steps and states, bit for bit, as the host loop of go_batch_step,
 * go_batch_grf_perturb, go_batch_max_dt and go_batch_set_dt.  The graph is
 * captured on the first call and reused while key0, std_dev, corr_cells,
 * scratch and the batch's members and launch stay the same; scratch must
 * stay allocated while it is in use.  Wind stays at the members' bound
 * wind_stress_t.  Synchronous. */
int go_batch_run_events(go_batch* b, void* stream, uint32_t first_event, int n_events,
                        double interval, float dt, double courant, uint32_t key0,
                        float std_dev, float corr_cells, float* scratch,
                        size_t scratch_floats, double* t_members, long long* steps_out,
                        float* dt_out);

/* Device status word (GO_STATUS_* bits) accumulated by the step kernels;
 * synchronous read, optionally clearing it. */
int go_domain_status(go_domain* d, uint32_t* status, int clear);

/* Kernel launches the domain's last RK stage issued (1 for launch shapes
 * 0..7; for the column-pair shape the boundary frame, the interior region
 * and, at periodic east/west sides, the ghost-column copy; 0 before the
 * first step). */
int go_domain_stage_launches(go_domain* d, int* launches);

/* Test hooks of the failure-detection tests (0 in normal runs).
 * GO_DEBUG_SKIP_TMA: the column-pair kernel issues none of its TMA tile
 * loads, so its bounded waits on the tiles' mbarriers run out; the stage
 * then sets GO_STATUS_TIMEOUT, leaves the region's cells unwritten and
 * returns, and the context stays usable.  Applies to stages prepared
 * after the call (a batch takes it from its members at go_batch_set_member). */
#define GO_DEBUG_SKIP_TMA 0x1u
int go_domain_set_debug(go_domain* d, unsigned flags);

/* Status words of every member of a batch (n values to status_host, member
 * order): each member's step kernels write only its own word, so a member
 * whose state went non-finite is flagged alone and the others step on
 * unchanged.  Synchronous; clear != 0 resets the words.  Replaces the
 * reference's dead-member bookkeeping (BaseOceanStateEnsemble.py:108-110,
 * EnsembleFromFiles.py:315), which looks for NaN in downloaded states. */
int go_batch_status(go_batch* b, uint32_t* status_host, int clear);

/* Message of the last failed call on this host thread ("" if none). */
const char* go_last_error(void);

/* Library version string. */
const char* go_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GOCEAN_H */
