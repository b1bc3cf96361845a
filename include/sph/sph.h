/*
 * sph.h — C-ABI of the B200-native adaptive SPH step (sca2012_b200).
 *
 * This is the drop-in boundary for the reference's per-step particle pipeline.
 * In the reference the host class SPHSystem calls C++-linkage launch wrappers
 * that take raw device pointers (SPH-3D-2/sph_system.cuh:1-91,
 * SPH-2D/sph_system.cuh:1-72) and mirrors every constant into a __constant__
 * SysParam block re-uploaded each step (SPH-3D-2/sph_param.h:8-87,
 * SPH-2D/sph_param.h:6-70, set_parameters at SPH-3D-2/sph_system.cu:34-37).
 * Here the same responsibilities sit behind an opaque handle:
 *
 *   sph_config            <- SysParam + the SPHSystem constructor constants
 *                            (SPH-3D-2/sph_system.cpp:6-229, SPH-2D/sph_system.cpp:5-146)
 *   sph_config_preset     <- the three reference constructors (2D, 3D-2, 3D-4)
 *                            plus the synthetic SI-unit workloads
 *   sph_create/destroy    <- SPHSystem::SPHSystem / ~SPHSystem (alloc_array calls)
 *   sph_add_particles     <- SPHSystem::add_particle + the H2D copy_array
 *                            (SPH-3D-2/sph_system.cpp:285-300, :263)
 *   sph_step              <- SPHSystem::animation() / animate()
 *                            (SPH-3D-2/sph_system.cpp:302-404, SPH-2D/sph_system.cpp:190-264)
 *   sph_get_state         <- the D2H copy_array of m_host_mem at the end of a step
 *                            (SPH-3D-2/sph_system.cpp:401)
 *   sph_get_debug         <- reads of m_dev_hash / m_dev_index / m_cell_start /
 *                            m_cell_end / m_trans_vel (the step's intermediates)
 *   sph_density_grid,     <- integrate_dens + integrate_normal + SPHSystem::marching_cube
 *   sph_extract_surface      (SPH-3D-2/sph_system.cu:2185-2351, sph_system.cpp:406-542)
 *
 * Conventions: every call returns an int status (SPH_OK == 0).  All pointers
 * in signatures are HOST pointers unless the name says _dev.  A handle owns
 * its device memory and its CUDA stream; it is not thread-safe, separate
 * handles are independent.  Particle vectors are passed with `dim` floats per
 * particle (2 or 3).  The particle count lives on the device; sph_step does
 * not synchronise with the host.
 */
#ifndef SCA2012_B200_SPH_H
#define SCA2012_B200_SPH_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SPH_OK             0
#define SPH_ERR_INVALID    1  /* bad argument / config */
#define SPH_ERR_CAPACITY   2  /* particle capacity exceeded (add or split) */
#define SPH_ERR_CUDA       3  /* CUDA runtime error */
#define SPH_ERR_NO_DEVICE  4  /* no CUDA device / kernels not loadable */
#define SPH_ERR_NONFINITE  5  /* non-finite position detected by the step */
#define SPH_ERR_RANGE      6  /* size beyond a fixed maximum of the entry point */
#define SPH_ERR_TIMEOUT    7  /* a grid-wide barrier of the persistent step gave up waiting */

/* ---- presets (sph_config_preset) ---- */
#define SPH_PRESET_REF_2D    0  /* SPH-2D/sph_system.cpp:5-146            */
#define SPH_PRESET_REF_3D2   1  /* SPH-3D-2/sph_system.cpp:6-229          */
#define SPH_PRESET_REF_3D4   2  /* SPH-3D-4/sph_system.cpp:6-229          */
#define SPH_PRESET_DAM_2D    3  /* 2D dam break, 4096 particles, SI units */
#define SPH_PRESET_DAM_3D2   4  /* 3D two-way adaptive, 131072 particles  */
#define SPH_PRESET_DAM_3D4   5  /* 3D four-way adaptive, 1114112 particles */
#define SPH_PRESET_ROLLOUT_3D 6 /* 32^3 block, two-way, differentiable    */

/* integrator variants */
#define SPH_INTEGRATE_REF3D  0  /* v+=a*dt/rho; v+=g*dt/rho; x+=v*dt; walls; ev=(ev+v)/2 (SPH-3D-2/sph_system.cu:237-321) */
#define SPH_INTEGRATE_REF2D  1  /* a=(a+g*dt)/rho; v+=a*dt; ev=(ev+v)/2; x+=v*dt; walls (SPH-2D/sph_system.cu:219-251) */
#define SPH_INTEGRATE_PHYS   2  /* v+=(F/m+g)*dt; x+=v*dt; walls; ev=(ev+v)/2 */

/* split criteria */
#define SPH_SPLIT_WAVELET    0  /* energy*co_energy + surface*co_surface > split_criteria (SPH-3D-2/sph_system.cu:1564) */
#define SPH_SPLIT_DEFICIT    1  /* neighbour count < split_min_neighbors or rho < split_density_ratio*rho0 */

/* merge criteria */
#define SPH_MERGE_WAVELET    0  /* level 2 and energy*co_energy + surface*co_surface < merge_criteria (SPH-3D-2/sph_system.cu:1694) */
#define SPH_MERGE_WAVELET_CELL 1 /* 2D: criterion read from the particle whose index equals the cell index (SPH-2D/sph_system.cu:1207) */
#define SPH_MERGE_INTERIOR   2  /* level 2 and interior (not split-flagged) for merge_interior_steps steps, paired per cell */
#define SPH_MERGE_SIBLING    3  /* a split group (parent + children, sph_state_view.sibling) merges back when every
                                   member is level 2 and interior for merge_interior_steps steps */

typedef struct sph_sphere {
    float pos[3];
    float radius;
    float damping;
} sph_sphere;

/*
 * Every physical constant of one solver instance.  Per-level arrays use
 * index 0 for level 1 ("large") and index 1 for level 2 ("small"), the two
 * particle levels of the reference.  Kernel coefficients are stored exactly
 * as the reference stores them (float, computed on the host).
 */
typedef struct sph_config {
    uint32_t dim;            /* 2 or 3 */
    uint32_t max_particle;   /* capacity of the handle */
    float world[3];          /* x, y, z extent (2D: x, y; z unused) */
    float cell_size;         /* uniform hash cell edge (= level-1 kernel length) */
    uint32_t ncell[3];       /* cells per axis (2D: ncell[2] == 1) */

    float mass[2], kernel[2], kernel2[2], kernel6[2], radius[2];
    float poly6[2], spiky[2], visco[2], grad_poly6[2], lapc_poly6[2], poly6_radius[2];

    float gravity[3];
    float wall_damping;      /* velocity factor at a wall (reference: -0.6) */
    float rest_density;
    float gas_constant;
    float time_step;
    float viscosity;
    float surface_threshold; /* |grad c| above which surface tension acts */
    float surface_coef;      /* 0.1 (3D-2), 0.02 (3D-4), 0.04 (2D) */
    float co_surface, co_energy;
    float split_criteria, merge_criteria;
    float density_skip_r2;   /* density loop skips pairs closer than this (3D 1e-4, 2D 1e-12) */
    float lapc_three_quarters; /* factor in (r2 - f*(h2-r2)); reference integer 3/4 == 0 */

    uint32_t split_ways;     /* 2 or 4 */
    uint32_t use_split, use_merge;
    uint32_t integrator;     /* SPH_INTEGRATE_* */
    uint32_t kernel_h6_twice;/* 1: spiky/visco terms divided by h^6 a second time (reference) */
    uint32_t energy_large_kernel; /* 1: wavelet energy uses the level-1 kernel for all levels (3D) */
    uint32_t energy_mass_weight;  /* 1: energy *= mass (3D-4) */
    uint32_t energy_skip_close;   /* 1: energy loop skips r2 < 1e-4 (3D); 0: keeps it (2D) */
    uint32_t split_rule;     /* SPH_SPLIT_* */
    uint32_t merge_rule;     /* SPH_MERGE_* */
    uint32_t split_min_neighbors;   /* SPH_SPLIT_DEFICIT */
    float split_density_ratio;      /* SPH_SPLIT_DEFICIT */
    uint32_t merge_interior_steps;  /* SPH_MERGE_INTERIOR, SPH_MERGE_SIBLING */
    uint32_t split_copies_fields;   /* 1: child copies dens/press/surface (2D) */

    /* obstacles and interactive forces (reference integrator / force kernel) */
    uint32_t use_cylinder;
    sph_sphere sphere[3];
    uint32_t push_left, push_right; /* 3D push forces (SPH-3D-4/sph_system.cu:229-242) */
    uint32_t push_y_div;            /* y threshold = height / push_y_div (3D-2 5, 3D-4 10) */
    uint32_t extern_force_on;       /* 2D mouse force (SPH-2D/sph_system.cu:781-789) */
    float extern_click[2], extern_force[2], extern_len, extern_coe;

    /* density grid / marching cubes (SPH-3D-2/sph_system.cpp:86-92) */
    uint32_t dens_mul;
    float den_size;
    uint32_t ndens[3];
    float iso_value;
    uint32_t mc_interpolate; /* 0: edge midpoints (reference); 1: linear interpolation */
    uint32_t splat_with_kernel; /* 0: grid splat radius = particle radius (reference); 1: kernel length */
    uint32_t grid_every;     /* density grid + surface inside every k-th step (0: never); the
                                reference's display mode 2 is 1 (SPH-3D-2/sph_system.cpp:336-362) */
    uint32_t max_triangles;  /* device mesh capacity (0: 3 per grid node) */
    uint32_t compensated_positions; /* 1: positions carry an FP32 low part and x += v dt is a
                                       compensated (Fast2Sum) update; 0: plain FP32 (reference) */
    float close_r2;          /* the force loop (and the energy loop with energy_skip_close) skips
                                pairs with r^2 below this: reference 1e-4, a constant of its unit
                                system (SPH-3D-2/sph_system.cu:801-804, SPH-2D/sph_system.cu:584) */
    uint32_t walk_only;      /* 1: the force and energy passes walk the cell stencil themselves
                                instead of reading the neighbour lists the density pass records
                                (same pairs, same order, same results; a comparison switch) */
} sph_config;

/* Host view of a particle state (SoA).  Vectors hold `dim` floats per
 * particle.  Any pointer may be NULL on read to skip that field. */
typedef struct sph_state_view {
    uint32_t n;
    float *pos, *vel, *ev, *acc;
    float *dens, *press, *energy, *surface;
    uint32_t *level;
    uint32_t *interior;      /* SPH_MERGE_INTERIOR / SPH_MERGE_SIBLING counter */
    uint32_t *scene;         /* scene index of each particle (batched scenes; 0 otherwise) */
    uint32_t *sibling;       /* next member of the particle's split group, 0xffffffff for none (NULL: none) */
} sph_state_view;

/* One scene of a batch: its walled box inside the handle's world and the
 * constants that differ between scenes.  Boxes must be at least
 * SPH_SCENE_GAP_CELLS cells apart so no particle pair across scenes is ever
 * within a kernel length. */
#define SPH_SCENE_GAP_CELLS 2
typedef struct sph_scene {
    float lo[3], hi[3];      /* walls: particles stay in [lo + r, hi - r] */
    float viscosity;
    float gas_constant;
} sph_scene;

/* Intermediates of the last step (host arrays sized by the caller).
 * n_sorted = particle count the step started with; total_cell = cells. */
typedef struct sph_debug_view {
    uint32_t n_sorted, total_cell;
    uint32_t *hash;          /* [n_sorted] cell key of each sorted slot      */
    uint32_t *index;         /* [n_sorted] particle index of each sorted slot */
    uint32_t *cell_start;    /* [total_cell] first sorted slot, 0xffffffff if empty */
    uint32_t *cell_end;      /* [total_cell] one past last slot, 0 if empty  */
    float *trans_vel;        /* [n_sorted*dim] wavelet-transformed velocity, by particle index */
    uint32_t *nbr_count;     /* [n_sorted] neighbours within own kernel, by particle index */
    uint32_t *split_flag;    /* [n_sorted] 1 if the particle split, by particle index */
    uint32_t *removed;       /* [n_sorted] 1 if merged away, by particle index */
} sph_debug_view;

/* Triangle soup of the iso-surface (host arrays, 3 floats per corner). */
typedef struct sph_mesh_view {
    uint32_t max_triangles;
    uint32_t num_triangles;  /* out: triangles produced (may exceed max) */
    float *v0, *v1, *v2;
    float *n0, *n1, *n2;
} sph_mesh_view;

typedef struct sph_handle sph_handle;

/* sizeof(sph_config), for foreign-function bindings to check their layout. */
size_t sph_config_size(void);

/* Fills *cfg with a preset.  Reference presets reproduce the reference
 * constructors' constants bit for bit. */
int sph_config_preset(int preset, sph_config *cfg);

int sph_create(const sph_config *cfg, sph_handle **out);
int sph_destroy(sph_handle *h);

/* Replaces runtime-adjustable constants (time step, toggles, forces...).
 * The cell grid, dimension and capacity must match the handle's. */
int sph_set_config(sph_handle *h, const sph_config *cfg);
int sph_get_config(const sph_handle *h, sph_config *cfg);

/* Appends n particles (pos/vel: n*dim floats, level: 1 or 2). */
int sph_add_particles(sph_handle *h, uint32_t n, const float *pos, const float *vel,
                      const uint32_t *level);

/* Replaces the whole state; NULL optional fields are zero-filled. */
int sph_set_state(sph_handle *h, const sph_state_view *st);

/* Advances nsteps steps on the handle's stream (asynchronous). */
int sph_step(sph_handle *h, int nsteps);

/* Batched scenes: many independent scenes advance in the same launches.
 * Each particle carries a scene index (sph_state_view.scene); scene s
 * integrates inside scenes[s].lo/hi with its own viscosity and stiffness,
 * all other constants are the handle's.  Every scene's particles evolve
 * exactly as they would alone in a handle with the same world.  nscenes = 0
 * returns to the single-scene box [0, world]. */
int sph_set_scenes(sph_handle *h, uint32_t nscenes, const sph_scene *scenes);

/* on != 0: sph_step replays each step as a CUDA graph (one per buffer
 * parity, recaptured when the config or the launch grid changes); steps that
 * build the density grid and surface run uncaptured.  Same results, fewer
 * launch overheads for small particle counts. */
int sph_set_graph(sph_handle *h, int on);

/* on != 0: sph_step runs each step inside ONE cooperative launch (the stages
 * separated by grid-wide barriers instead of launch boundaries), for scenes
 * small enough that launches and the drain between them, not the work, set
 * the step time.  Consecutive steps that cannot split (use_split = 0) share
 * a launch, up to 256 of them, up to the next surface step.  Results are bit
 * for bit those of the ordinary launches; steps that build the density grid
 * and surface, and profiled steps, use the ordinary launches.  Takes
 * precedence over sph_set_graph.  No counterpart in the reference, which
 * launches every stage separately (SPH-3D-2/sph_system.cpp:302-404).
 * spin_limit: how many times a block polls a barrier before it gives up
 * (SPH_PERSISTENT_SPIN_DEFAULT: about a second; 0: at the first poll).  A
 * block that gives up ends the launch with SPH_ERR_TIMEOUT (reported by
 * sph_sync); that step writes no state, later steps do nothing until the
 * state is restored with sph_set_state, and the handle stays usable. */
#define SPH_PERSISTENT_SPIN_DEFAULT (1u << 22)
int sph_set_persistent(sph_handle *h, int on, uint32_t spin_limit);

/* Synchronises and returns the device-side status (capacity / non-finite). */
int sph_sync(sph_handle *h);

int sph_get_num_particles(sph_handle *h, uint32_t *n);
int sph_get_state(sph_handle *h, sph_state_view *st);
int sph_get_debug(sph_handle *h, sph_debug_view *dbg);

/* Particle records in the reference's own layout (the Particle class,
 * SPH-3D-2/sph_system.h:8-24: 72 bytes in 3D; SPH-2D/sph_system.h:7-22:
 * 56 bytes in 2D).  sph_read_particles is the per-step readback of
 * SPHSystem::animation() (copy_array(m_host_mem, m_dev_mem, ...),
 * SPH-3D-2/sph_system.cpp:401); sph_write_particles is the upload after
 * add_box_particle (:263).  The layout conversion runs on the device; the
 * host transfer is one contiguous copy (fastest from page-locked memory).
 * sph_read_particles writes *n_out records (fails if capacity_bytes is too
 * small). */
uint32_t sph_particle_record_size(const sph_handle *h);
int sph_read_particles(sph_handle *h, void *host_dst, uint64_t capacity_bytes, uint32_t *n_out);
int sph_write_particles(sph_handle *h, const void *host_src, uint32_t n);

/* Per-stage timing: when on, each sph_step records a CUDA event after every
 * stage; sph_stage_times returns the last step's stage durations (ms) and
 * names, up to max entries, and the number of stages. */
int sph_set_profiling(sph_handle *h, int on);
int sph_stage_times(sph_handle *h, float *ms, const char **names, int max, int *count);

/* The handle's CUDA stream (a cudaStream_t), for callers timing or
 * ordering work against the step. */
void *sph_get_stream(sph_handle *h);

/* Runs the handle's work on `stream` (a cudaStream_t; NULL = the handle's own
 * stream) from now on, after the work already queued has finished.  The caller
 * keeps ownership of its stream and must not destroy it while the handle uses
 * it. */
int sph_set_stream(sph_handle *h, void *stream);

/* on != 0: the step also keeps per-particle debug intermediates
 * (wavelet-transformed velocity) for sph_get_debug. */
int sph_set_debug(sph_handle *h, int on);

/* Number of kernel launches the last sph_step issued. */
int sph_last_launch_count(const sph_handle *h, uint32_t *launches);

/* Particle counts of the last step (the per-step line the reference's
 * SPH-3D-4 app prints as its L/S counts, SPH-3D-4/sph_main.cpp:819, and the
 * split/merge activity behind it).  Synchronises with the handle's stream.
 * n_split: particles that split (0 when the capacity guard suppressed the
 * step's splits, split_suppressed = 1); n_removed: particles merged away;
 * n_end = n_start + n_split * (ways - 1) - n_removed; n_level2: level-2
 * particles after the step; error: the step's SPH_ERR_* bits (1 << code). */
typedef struct {
    uint32_t n_start, n_split, n_removed, n_end, n_level2, split_suppressed, error;
} sph_step_stats;
int sph_last_step_stats(sph_handle *h, sph_step_stats *out);

/* Density grid of the current state (splat + normals on the device), copied
 * to host arrays of ndens[0]*ndens[1]*ndens[2] floats / 3*that floats. */
int sph_density_grid(sph_handle *h, float *dens, float *normal);

/* Triangles of the surface extracted on the device by the last step that
 * built the density grid (grid_every), appended in the reference's cell
 * order (x outer, y, z inner; SPH-3D-2/sph_system.cpp:517-542).  Returns
 * SPH_ERR_CAPACITY if the surface had more triangles than the capacities
 * (max_triangles of the config or of the mesh view): the mesh then holds the
 * first triangles and num_triangles the full count. */
int sph_extract_surface(sph_handle *h, sph_mesh_view *mesh);

/* Marching cubes on the device over a caller-supplied grid (host arrays in
 * sph_density_grid's layout), with sph_extract_surface's output. */
int sph_surface_from_grid(sph_handle *h, const float *dens, const float *normal, sph_mesh_view *mesh);

/* Headless POV-Ray scene files, replacing the reference app's make_mesh /
 * make_particle (SPH-3D-2/sph_main.cpp:114-220): one smooth_triangle per mesh
 * triangle, or one sphere per particle (red r 0.3 for level 1, yellow r 0.24
 * for level 2); positions are p * scale + offset per axis (NULL: 1 and 0). */
int sph_write_pov_mesh(const sph_mesh_view *mesh, const float *scale, const float *offset, const char *path);
int sph_write_pov_particles(const float *pos, const uint32_t *level, uint32_t n, uint32_t dim, const float *scale,
                            const float *offset, const char *path);

/* Asynchronous readback: converts the current state to reference Particle
 * records on a side stream, writing them and the record count straight into
 * page-locked host memory that is mapped for the device (cudaHostAlloc with
 * cudaHostAllocMapped, or cudaHostRegister with cudaHostRegisterMapped;
 * both pointers 4-byte aligned, else SPH_ERR_INVALID).
 * Returns at once; the next sph_step overlaps the copy (it works on the other
 * state buffer) and a later step that would overwrite the buffer being read
 * waits for it.  sph_readback_wait blocks until the records and *count_dst
 * are in host memory.  At most capacity_bytes are written (the count is still
 * the full one). */
int sph_read_particles_async(sph_handle *h, void *mapped_dst, uint64_t capacity_bytes, uint32_t *mapped_count_dst);
int sph_readback_wait(sph_handle *h);

/*
 * Cell sort that allocates nothing.  No counterpart in the reference (its
 * cell sort is calc_hash + thrust::sort_by_key + find_start_end, which
 * allocate; see sph_step).  For callers that cannot call cudaMalloc — a host
 * program whose device memory belongs to another allocator, or a loop that
 * cannot afford cudaMalloc's implicit device synchronisation.  Sorts n
 * particles (pos_dev: n*dim floats on the device) by cell key exactly like
 * sph_step does and writes, all on the device, key_dev[n] and index_dev[n]
 * (cell key and particle index of each sorted slot) and cell_start_dev /
 * cell_end_dev (one entry per cell; 0xffffffff / 0 for an empty cell).
 * Scratch lives in one fixed static device array: at most
 * SPH_NOALLOC_MAX_PARTICLES particles and SPH_NOALLOC_MAX_CELLS cells, larger
 * inputs return SPH_ERR_RANGE.  The first call on a device looks up the
 * array's device address; make it before any stream capture begins.  The
 * address is kept for the life of the process: after cudaDeviceReset on a
 * device it is stale, so do not call this entry point on that device again
 * in the same process.  Calls
 * share the array, so calls that overlap on the GPU race.  Asynchronous on
 * `stream` (a cudaStream_t, NULL = default stream).
 */
#define SPH_NOALLOC_MAX_PARTICLES (1u << 18)
#define SPH_NOALLOC_MAX_CELLS (1u << 16)
int sph_sort_cells_noalloc(const sph_config *cfg, uint32_t n, const float *pos_dev, uint32_t *key_dev,
                           uint32_t *index_dev, uint32_t *cell_start_dev, uint32_t *cell_end_dev, void *stream);

/*
 * Differentiable rollout.  No counterpart in the reference (it has no
 * gradients); the forward is sph_step itself.  Supported for the SI physics:
 * SPH_INTEGRATE_PHYS, surface_coef 0, no obstacles or interactive forces.
 *
 * sph_rollout_forward advances nsteps from the current state and keeps the
 * state at steps 0, k, 2k, ... (k = checkpoint_every) and the final state on
 * the device.  sph_splat_loss splats the current state onto a node grid,
 * G_g = sum_i m_i W_poly6(|x_g - x_i|, h_i), and returns
 * loss = mean_g (G_g - target_g)^2 (target: host array, x fastest).
 * sph_rollout_backward returns the gradient of the last loss with respect to
 * the initial velocities and positions (host arrays, n0 x dim, in the order
 * of the state the forward started from; NULL skips) and to the viscosity and
 * gas constant (d_params[2s], d_params[2s+1] for scene s; one scene without
 * batched scenes; nparams = the array's length).  It replays each checkpoint
 * interval with its topology recorded -- cell lists, wall contacts, split
 * flags, merge groups -- and runs the adjoint kernels back through it, so the
 * gradient is that of the forward with its topology held fixed.  The handle
 * is left holding the final state.  Any state change in between (step,
 * set_state, ...) invalidates the rollout.
 */
typedef struct sph_loss_grid {
    uint32_t n[3];           /* nodes per axis (n[2] = 1 in 2D) */
    float origin[3];         /* position of node (0, 0, 0) */
    float spacing;
} sph_loss_grid;

int sph_rollout_forward(sph_handle *h, uint32_t nsteps, uint32_t checkpoint_every);
int sph_splat_loss(sph_handle *h, const sph_loss_grid *grid, const float *target, float *grid_out, double *loss);
int sph_rollout_backward(sph_handle *h, float *d_vel0, float *d_pos0, double *d_params, uint32_t nparams);

/* Topology of forward step `step` of the last rollout in particle indices of
 * that step, for an independent (e.g. FP64 host) replay.  Counts are always
 * set; each non-NULL array is filled (dens_nbr / force_nbr only when
 * dens_cap / force_cap hold the pair counts). */
typedef struct sph_topology_view {
    uint32_t n, n_next, n_split, n_removed, split_on;   /* out */
    uint32_t n_dens_pairs, n_force_pairs;               /* out */
    uint32_t dens_cap, force_cap;                       /* in */
    uint32_t *level;                 /* n: 1 or 2 */
    uint32_t *dens_off, *dens_nbr;   /* n + 1 / pairs: CSR of j != i with r^2 < h_i^2 */
    uint32_t *force_off, *force_nbr; /* n + 1 / pairs: force pairs; bit 30 = h_i - r > 0, bit 31 = h_j - r > 0 */
    uint32_t *wall;                  /* n: bit 2d = clamped at the high wall of axis d, 2d+1 = low wall */
    uint32_t *split;                 /* n: split this step */
    uint32_t *dst;                   /* n: index of the particle's own record next step, 0xffffffff if merged away */
    uint32_t *child;                 /* n: index of its first child record (split particles) */
    uint32_t *merge_leader;          /* n: particle index of its merge group's leader, 0xffffffff if none */
    float *pos, *vel, *ev;           /* n x dim: the state the step started from */
} sph_topology_view;

int sph_rollout_topology(sph_handle *h, uint32_t step, sph_topology_view *v);

/* Conserved quantities of the current state, summed in FP64 on the device
 * (deterministic order): out[0] total mass, out[1..3] momentum, out[4]
 * kinetic energy, out[5] gravitational potential energy -m g.x, out[6] their
 * sum.  Synchronous. */
int sph_conserved(sph_handle *h, double out[7]);

/*
 * Launch shapes.  Each tuned stage of the step launches `block` threads per
 * block and at most blocks_per_sm x (SM count) blocks, its threads looping
 * grid-stride over the particles (so blocks_per_sm sets how many particles a
 * thread covers).  Results do not depend on the shapes.  sph_autotune times
 * the candidates on the handle's current state (the state is restored after
 * every trial and at the end), `reps` steps per candidate, stage by stage, and
 * keeps the fastest; block in {128, 256, 512} (force and energy: 128, 256;
 * force with and without a register cap), blocks_per_sm in {2, 4, 8, 16, 32, 64}.
 * Defaults: 256 threads and 8 per SM for hash, scatter, reorder and merge;
 * 128 threads and 64 per SM for density, force, energy and write; no cap.
 */
#define SPH_TUNE_HASH     0
#define SPH_TUNE_SCATTER  1
#define SPH_TUNE_REORDER  2
#define SPH_TUNE_DENSITY  3
#define SPH_TUNE_FORCE    4
#define SPH_TUNE_ENERGY   5
#define SPH_TUNE_MERGE    6
#define SPH_TUNE_WRITE    7
#define SPH_TUNE_STAGES   8
typedef struct sph_tuning {
    uint32_t block[SPH_TUNE_STAGES];
    uint32_t blocks_per_sm[SPH_TUNE_STAGES];   /* 1..64 */
    uint32_t reg_cap[SPH_TUNE_STAGES];         /* force and energy: 1 = register-capped build (8 blocks
                                                  of 128 or 4 of 256 resident per SM, 64 registers);
                                                  0 elsewhere */
    float step_ms_before, step_ms_after;       /* sph_autotune: mean step time before / after */
} sph_tuning;

int sph_set_tuning(sph_handle *h, const sph_tuning *t);
int sph_get_tuning(const sph_handle *h, sph_tuning *t);
int sph_autotune(sph_handle *h, uint32_t reps, sph_tuning *out);

/* Human-readable text of the last error on this handle (static storage). */
const char *sph_last_error(const sph_handle *h);

#ifdef __cplusplus
}
#endif
#endif
