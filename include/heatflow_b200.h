/*
 * heatflow_b200.h -- C ABI of libheatflow_b200.so, the sm_100a implementation of Heatflow-MPM's Eulerian air substep.
 *
 * Every entry point takes plain pointers, sizes and a cudaStream_t (passed as void*), returns an hf_status, never
 * synchronises the stream on its own (the set-up calls that upload tables say so), and never allocates device memory:
 * all device buffers -- fields, the scene table, the work table and the workspace -- belong to the caller.
 *
 * The reference (pietis/Heatflow-MPM) has no native layer: every stage is a Warp kernel launched from Python.  Each
 * entry point below names the reference function or kernels it replaces (file:line within that repository).
 *
 * Data layout (identical to the reference's Warp arrays, C order, k fastest):
 *   cell fields (n,n,n) float32; u (n+1,n,n), v (n,n+1,n), w (n,n,n+1) float32; particle positions/velocities (P,3).
 *   cell flags (n,n,n) uint8: bit0 = fixed (Dirichlet) cell, bit1 = heater source cell.
 * The temperature T and the face velocities u,v,w are double-buffered: buffer [parity] is current, where parity is
 * the scene's device-side hf_scene_state.parity, flipped by the last stage of every substep (so a captured CUDA graph
 * of a substep can be replayed without re-recording).
 */
#ifndef HEATFLOW_B200_H
#define HEATFLOW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HF_ABI_VERSION 1

typedef enum hf_status {
    HF_OK = 0,
    HF_ERR_ARG = 1,        /* invalid argument (null pointer, size out of range, misaligned buffer) */
    HF_ERR_CUDA = 2,       /* a CUDA runtime call failed; hf_last_error() has the text */
    HF_ERR_WORKSPACE = 3,  /* workspace smaller than hf_workspace_bytes() */
    HF_ERR_DEVICE = 4      /* no sm_100 device, or a cooperative launch cannot fit the grid */
} hf_status;

/* per-scene solver status word, in hf_scene_state.status (bit set) */
#define HF_SCENE_OK 0
#define HF_SCENE_HEAT_MAXITER 1      /* heat CG stopped at maxiter above its tolerance */
#define HF_SCENE_PRESSURE_MAXITER 2  /* pressure CG stopped at maxiter above its tolerance */
#define HF_SCENE_NONFINITE 4         /* a CG residual became NaN/inf */
#define HF_SCENE_BARRIER_TIMEOUT 8   /* a grid barrier of a persistent kernel gave up (bounded wait) */
#define HF_SCENE_CORRECTED 16        /* a CG solve was restarted by the outer defect correction (HF_FLAG_DEFECT_CORRECTION) */

/* hf_scene.flags */
#define HF_FLAG_BUOYANCY 1u          /* GridConfig.buoyancy (grid.py:18) */
#define HF_FLAG_SOURCE 2u            /* heater source active: rate > 0 (solver.py:76) */
#define HF_FLAG_PARTICLES 4u         /* particle coupling on: obstacle fields rebuilt every substep (solver.py:65-72) */
#define HF_FLAG_ACTIVE 8u            /* scene takes part in batched calls (serving slots) */
#define HF_FLAG_DEFECT_CORRECTION 16u /* after each CG solve converges, form the true residual b - A x in fp64; above the
                                         tolerance, restart CG from x with it (at most twice).  Not in the reference:
                                         off by default; the solves run in the streaming CG kernel */

/* Mutable device-side state of one scene (caller allocates sizeof(hf_scene_state) bytes of device memory, zeroed). */
typedef struct hf_scene_state {
    int32_t parity;        /* index of the current T / u,v,w buffer */
    int32_t status;        /* HF_SCENE_* bits of the last substep */
    int64_t substeps;      /* substeps completed */
    int32_t heat_iters;    /* heat CG iterations performed in the last substep (HeatField.cg_iters, heat.py:210) */
    int32_t pressure_iters;/* pressure CG iterations performed in the last substep (AirGrid.cg_iters, grid.py:249) */
    double heat_rr, heat_atol;       /* final r.r and absolute tolerance of the heat solve */
    double pressure_rr, pressure_atol;
    double pressure_bb, heat_bb;     /* b.b of the last solves (||r||/||b|| = sqrt(rr/bb)) */
    double rhs_mean;                 /* mean removed from the pressure rhs (grid.py:238-241) */
    int64_t total_heat_iters, total_pressure_iters;
    /* Particle footprint (cells, inclusive, lo i,j,k then hi i,j,k) of the current and the previous substep: the
     * obstacle fields are rebuilt only inside their union.  An empty box has lo > hi; initialise both to empty
     * (lo = INT32_MAX, hi = INT32_MIN) before the first substep. */
    int32_t box[6];
    int32_t box_prev[6];
    /* fp64 norm^2 of the true residual b - A x at the end of the last heat / pressure solve (scenes with
       HF_FLAG_DEFECT_CORRECTION; -1 otherwise) */
    double heat_true_rr, pressure_true_rr;
} hf_scene_state;

/* One scene: sizes, physical parameters and device pointers of its fields.  The same struct is the element of the
 * device-side scene table (hf_plan.scenes_dev); it holds no host pointers. */
typedef struct hf_scene {
    int32_t n;                 /* cells per edge (AirGrid.n, grid.py:183) */
    int32_t n_particles;       /* material particles (0: air-only) */
    uint32_t flags;            /* HF_FLAG_* */
    int32_t cg_max_iter;       /* GridConfig.cg_max_iter (400) */
    int32_t heat_maxiter;      /* HeatField.diffuse maxiter (200) */
    int32_t reserved_i[3];
    /* Physical parameters as the reference's Python floats (double).  Kernels round them to binary32 exactly where
     * Warp does at launch; derived scalars (rho/dt, dt/rho) are formed in double first, as the Python code does. */
    double h, rho, t_amb, alpha_f_min, g;          /* GridConfig (grid.py:13-22); g = 9.81 (grid.py:219) */
    double cg_tol, heat_tol;                       /* relative CG tolerances (grid.py:21; heat.py:198) */
    double kappa_air, kappa_mat;                   /* thermal diffusivities (solver.py:15; mpm.py:17) */
    double rate, t_cap;                            /* heater source rate [K/s] and cap (heater.py:51-52) */
    double vol, k_particle;                        /* particle volume spacing^3 and K_PARTICLE (solver.py:16) */
    double t_sol, t_liq, y_solid, mu_s, mu_l, t_max; /* melt law (heat.py:161-174) */
    /* double-buffered state */
    float *T[2];
    float *u[2], *v[2], *w[2];
    /* temperature stage */
    float *Tw, *kap, *hrhs, *hdiag, *tfix, *alpha, *tsum;
    uint8_t *cell_flags;
    /* air grid */
    float *p, *rhs, *pdiag, *alpha_s;
    float *ax, *ay, *az, *qx, *qy, *qz, *kx, *ky, *kz, *mx, *my, *mz;
    /* static obstacle fields (heater body), added every substep (grid.py:206-213); NULL = none */
    float *st_alpha, *st_kx, *st_ky, *st_kz, *st_mx, *st_my, *st_mz;
    /* CG vectors (n^3 each): residual, preconditioned residual, search direction (2 buffers), A*p */
    float *cg_r, *cg_z, *cg_p[2], *cg_Ap;
    /* particles (P,3) / (P): positions and velocities in, temperature/melt/yield/viscosity in-out */
    float *pos, *pvel, *ptemp, *pmelt, *pyield, *pvisc;
    /* harmonic face diffusivities 2 k_a k_b / (k_a + k_b + 1e-12) of the three face lattices (heat.py:50-52) */
    float *hkx, *hky, *hkz;
    /* alpha_f of the low y and z face of every cell in cell layout (n,n,n) (copies of ay, az for tiled loads) */
    float *ayc, *azc;
    /* the heat diffusivity of the low z face of every cell in cell layout (n,n,n) (a copy of hkz for tiled loads) */
    float *hkzc;
    /* 12 fixed-point accumulators of (n+1)^3 int64 each (coupled scenes only), zero on entry, left zero */
    long long *acc;
    hf_scene_state *state;
} hf_scene;

/* hf_plan.options */
#define HF_PLAN_STREAMING_CG 1u      /* never use the register-resident CG variant (single-scene plans use it when
                                        the scene's tiles fit one block per SM) */
#define HF_PLAN_NO_TMA 2u            /* resident pressure CG without the TMA-staged stencil */
#define HF_PLAN_STREAMING_HEAT 4u    /* the heat CG of a single-scene plan in the streaming kernel (pressure unchanged) */
#define HF_PLAN_SINGLE_REDUCTION_CG 8u /* single-scene plans with n % 4 == 0: the pressure solve with one grid barrier
                                          per CG iteration instead of two -- the classic vector recurrences, beta from
                                          the expansion of the next r.z in the iteration's partials (D'Azevedo,
                                          Eijkhout & Romine 1993), the classic stopping test; results within ~1e-6
                                          relative of the classic method, so it is off by default.  Uses the scene's
                                          hdiag as scratch during the pressure solve. */
#define HF_PLAN_MAPS_READY 0x8000u   /* set by hf_plan_upload: the workspace holds the scenes' TMA descriptors (the
                                        streaming pressure CG stages its stencil boxes with TMA when every active scene
                                        has n % 4 == 0) */
#define HF_PLAN_LANES_SHIFT 8        /* options bits 8..11: lanes of the streaming CG launch (independent scene groups
                                        solved side by side, each lane with its own barrier; 0 = one lane) */
#define HF_PLAN_RES_TILES_SHIFT 12   /* options bits 12..13: tiles per 256-thread group of the resident CG variant (1..3;
                                        0 = the fewest that fit; more tiles per group = fewer threads, more registers) */

/* A batch of scenes ready to launch: tables in device memory plus the host copy used to size launches. */
typedef struct hf_plan {
    int32_t num_scenes;
    int32_t num_chunks;        /* 1024-cell work items over all scenes */
    int32_t num_tiles;         /* 4 x 8 x 32-cell tiles over all scenes (work items of the CG solves) */
    int32_t group_cells;       /* most cells of one CG group of the streaming solve (0 = a default that keeps a group's
                                  CG vectors in L2) */
    void *tiles_dev;           /* device: int32 quadruples (scene, i0, j0, k0) [num_tiles] */
    const hf_scene *scenes_host;   /* host copy, valid while the plan is used */
    void *scenes_dev;          /* device: hf_scene[num_scenes] */
    void *work_dev;            /* device: int32 pairs (scene, first cell) [num_chunks] */
    void *workspace;           /* device: >= hf_workspace_bytes(num_scenes, num_chunks, num_tiles) bytes */
    size_t workspace_bytes;
    int32_t persistent_blocks; /* grid of the persistent CG kernels (0 = choose: SMs x occupancy) */
    int32_t options;           /* HF_PLAN_* bits */
} hf_plan;

/* ---------------------------------------------------------------------------------------------------- set-up */
int hf_abi_version(void);
const char *hf_last_error(void);
int hf_cells_per_chunk(void);
/* workspace bytes for a plan of num_scenes scenes, num_chunks chunks and num_tiles tiles */
size_t hf_workspace_bytes(int num_scenes, int num_chunks, int num_tiles);
/* number of 1024-cell chunks / 4x8x32 tiles of a scene of n cells per edge */
int hf_chunks_for(int n);
int hf_tiles_for(int n);
/* Writes the scene table, the chunk and tile work tables and the scenes' TMA descriptors (into the workspace) to the
 * device, fills plan.num_chunks/num_tiles and sets HF_PLAN_MAPS_READY.  Blocking: the stream is synchronised before
 * return (set-up call, not for the per-substep path).  Call it again whenever a scene's buffers change. */
int hf_plan_upload(hf_plan *plan, void *stream);

/* --------------------------------------------------------------------------------- per-substep stages (batched) */
/* solver.py:65-72 + grid.py:202-213 + grid.py:46-67 + heat.py:44-47: obstacle fields of every scene -- particle
 * scatter (k_scatter_particles solver.py:19-38, k_scatter_heat heat.py:12-18) into fixed-point accumulators, plus the
 * static heater fields, face fractions alpha_f with zeroed wall fluxes, and the conductivity kappa.  Scenes without
 * HF_FLAG_PARTICLES are skipped unless `all_scenes` is set (used once at set-up to fill their static fields); per
 * substep, a coupled scene is rebuilt only inside the footprint boxes of its particles (this and the previous substep). */
int hf_obstacle_fields(const hf_plan *plan, int all_scenes, void *stream);
/* solver.py:74-79 + heat.py:108-118: k_blend, k_apply_fixed, k_source (rate > 0), k_advect, k_heat_rhs */
int hf_temperature_stage(const hf_plan *plan, double dt, void *stream);
/* heat.py:198-210: k_heat_diag + warp.optim.linear.cg(k_heat_matvec, M = diag, tol, maxiter, check_every=10),
 * solved in place in T[parity^1] by one persistent cooperative kernel with device-side convergence */
int hf_heat_solve(const hf_plan *plan, double dt, void *stream);
/* heat.py:161-174 k_particle_update (FLIP increment, melt fraction, yield stress, viscosity) */
int hf_particle_update(const hf_plan *plan, void *stream);
/* grid.py:219-233: k_advect_face x3 (into u,v,w[parity^1]), k_buoyancy, k_relax x3 */
int hf_face_stage(const hf_plan *plan, double dt, void *stream);
/* grid.py:235-251 + 140-153: k_divergence_rhs, device-side mean removal (replaces the host read-back of
 * grid.py:239), k_jacobi, warp.optim.linear.cg(k_laplacian, check_every=20) warm-started from p, k_project x3; then
 * flips every scene's parity (end of substep) */
int hf_pressure_solve(const hf_plan *plan, double dt, void *stream);
/* the two launches of hf_pressure_solve, separately (grid.py:237 k_divergence_rhs + per-chunk sums for the mean;
 * grid.py:238-251 mean removal, k_jacobi, CG, k_project and the end of the substep) */
int hf_divergence_stage(const hf_plan *plan, double dt, void *stream);
int hf_pressure_cg(const hf_plan *plan, double dt, void *stream);
/* the whole air substep in order (solver.py:63-88 minus the MPM step) */
int hf_substep(const hf_plan *plan, double dt, void *stream);

/* ------------------------------------------------------------------------------------------ getters (one scene) */
/* grid.py:156-162 k_cell_velocity: out (n^3,3) float32 from u,v,w[parity] of scene `s` (host copy of the table) */
int hf_cell_velocity(const hf_plan *plan, int s, float *out, void *stream);
/* grid.py:257-263: max|div(alpha_f u + q)| * h and max |u|,|v|,|w|; result written to out_dev[0] (float, device) */
int hf_divergence_max(const hf_plan *plan, int s, float *out_dev, void *stream);
int hf_speed_max(const hf_plan *plan, int s, float *out_dev, void *stream);
/* solver.py:105-110 frame_dict as written by scripts/run_scene.py:31-40: grid_T (n^3), the cell-centred air velocity
   (n^3 x 3, grid.py:156-162) and the particles' temperature and melt fraction (n_particles each) of scene `s`, converted
   to binary16 (round to nearest even, as numpy's astype(float16)) into device buffers; any output may be NULL */
int hf_pack_frame(const hf_plan *plan, int s, void *grid_T, void *air_u, void *temp, void *melt, void *stream);
/* solver.py:95-96 grid_T and the face velocities without a host read-back of the parity: the current buffer of
   scene `s`'s T (which = 0: n^3 floats) or u, v, w (which = 1, 2, 3: (n+1) n^2 floats) copied into device memory `out`,
   so that a caller can download it asynchronously while the next substeps run */
int hf_current_field(const hf_plan *plan, int s, int which, float *out, void *stream);

/* ------------------------------------------------------------- single-kernel entry points (parity, unit tests) */
/* grid.py:94-115 k_laplacian: out = alpha * L(p) / h^2 + beta * y (n^3 arrays, one scene) */
int hf_k_laplacian(int n, double h, double alpha, double beta, const float *p, const float *ax, const float *ay,
                   const float *az, const float *y, float *out, void *stream);
/* heat.py:94-105 k_heat_matvec */
int hf_k_heat_matvec(int n, double h, double dt, double alpha, double beta, const float *x, const float *kap,
                     const uint8_t *cell_flags, const float *y, float *out, void *stream);
/* The division by the cell size that every sampling stage performs (fields.py:14-15 divides each coordinate of a
   sample point by h): out[i] = x[i] / y, correctly rounded, by the kernels' constant-divisor method (a precomputed
   reciprocal pair and one correction; see hf_device.cuh).  For checking that method against IEEE division. */
int hf_k_divide_by(int count, const float *x, float y, float *out, void *stream);

/* Failure detection (no counterpart in the reference, whose solves cannot time out).  Every spin-wait of the persistent
   CG kernels -- grid and lane barriers, TMA copies -- gives up after limit_ns (default 2 s), sets
   HF_SCENE_BARRIER_TIMEOUT in the scenes of the launch, and every block returns, leaving the context usable.
   absent_block >= 0 keeps that block of each CG launch from arriving at its first grid barrier, so that a test can
   make the wait run out on purpose (-1: normal operation).  Applies to later launches on the current device;
   synchronous.  Restore (2000000000, -1) after a test. */
int hf_set_wait_limit(unsigned long long limit_ns, int absent_block);

/* ------------------------------------------------------------------------------------ scene set-up on the device */
/* Geometry of one scene's heater and optional static sphere.  The host fills it from the heater's parameters: the
 * frame of heater.py:24-31 (Heater.frame) and the thresholds of heater.py:42-49, each evaluated by the expression
 * heater.py writes (e.g. shell_out = R + 0.006 + h / 2), so that the device compares against the same binary64 values. */
typedef struct hf_heater_geometry {
    int32_t kind;            /* 0: no heater (off), 1: the trough heater of heater.py:33-49, 2: a box heater block */
    int32_t fan;             /* 1 when the fan runs (fan > 0): fan outlet cells and fan faces */
    double centre[3], facing[3], axis[3], up[3];   /* trough frame (heater.py:24-31) */
    double half_length;      /* L2 = length / 2 */
    double shell_in;         /* R - h / 2 */
    double shell_out;        /* R + 0.006 + h / 2 */
    double cap_half;         /* h / 2 */
    double cap_radius;       /* R + 0.006 */
    double rod_half;         /* L2 - 0.015 */
    double rod_radius;       /* 0.007 + h / 2 */
    double rod_front;        /* 0.03: rods at q = -0.03 */
    double rod_dz;           /* 0.03: rods at r = -0.03 and r = +0.03 */
    double fan_half;         /* L2 - 0.02 */
    double fan_high;         /* R - 0.01 */
    double fan_depth;        /* 0.015 */
    double trough_half;      /* L2 - 0.015 */
    double trough_radius;    /* R - 0.004 */
    int32_t box_lo[3], box_hi[3];   /* box heater: rods in i in [lo0, hi0), j in [lo1, hi1), k in [0, hi2) */
    int32_t box_trough;      /* box heater: the trough-air layer k (the fan layer is k + 1) */
    int32_t sphere;          /* 1: a static solid sphere */
    double t_rod, t_amb;     /* Dirichlet values of rods and walls */
    float m_face[3];         /* momentum weight of a fan face per axis: float32(K_FAN * fan * facing[axis]) */
    float k_solid, k_fan;    /* K_SOLID and K_FAN as float32 (heater.py:7) */
    float sphere_t;          /* the sphere's cells are fixed at this temperature */
    int32_t sphere_lo, sphere_hi, sphere_top;   /* sphere cells lie in i, j in [lo, hi), k in [0, top) */
    int32_t pad_;
    double sphere_c, sphere_zc, sphere_rr;      /* centre (c, c, zc) and squared radius */
} hf_heater_geometry;

/* heater.py:33-65 Heater.masks and solver.py:48-56 on the device, for one scene of edge n and cell size h:
 *   cell_class (n^3 bytes): the heater's cell type (0 air, 1 shell, 2 rod, 3 fan, 4 trough air), + 8 on sphere cells;
 *   cell_flags (n^3 bytes): bit0 fixed (rods, side walls and ceiling, sphere), bit1 source (fan and trough air);
 *   tfix (n^3 floats): rods t_rod, walls t_amb, sphere sphere_t (sphere before rods before walls), 0 elsewhere;
 *   alpha (n^3 floats): static solid fraction, 1 on shell, rod and sphere cells;
 *   kx, ky, kz / mx, my, mz (face lattices): static relaxation and momentum weights (heater.py:53-63; sphere faces
 *   K_SOLID toward rest).
 * counts (device, 2 ints, cleared by the call): [0] source cells (the host forms heater.py:52's rate from it),
 * [1] cells whose class depends on a comparison closer than 1e-12 m to its threshold (0 means the classes do not
 * depend on the host CPU's floating-point evaluation order). */
int hf_scene_statics(const hf_heater_geometry *geometry, int n, double h, uint8_t *cell_class, uint8_t *cell_flags,
                     float *tfix, float *alpha, float *kx, float *ky, float *kz, float *mx, float *my, float *mz,
                     int32_t *counts, void *stream);
/* shapes.py:13-17 _inside (Warp's mesh_query_point_sign_winding_number): generalized winding number of each of
 * num_points points (x, y, z float32) against a triangle soup (num_tri x 9 floats: v0, v1, v2); flag[i] = 1 when it
 * exceeds threshold (0.5: inside); winding (optional) receives the numbers themselves.  Exact sum over all triangles. */
int hf_winding_inside(const float *tri, int num_tri, const float *points, int num_points, float threshold,
                      int32_t *flag, float *winding, void *stream);

/* ------------------------------------------------------------------------------------ without device allocation */
/* No counterpart in the reference: an entry point for callers that cannot allocate device memory (code running where
 * no allocator may be called -- inside an allocator callback, under a memory budget owned by someone else, or in a
 * host that plans all device memory up front).  It performs hf_pressure_solve for ONE scene of edge n <= 64
 * (hf_noalloc_max_edge()): divergence of the face velocities, mean removal, Jacobi-PCG warm-started from p, and the
 * projection of u, v, w in place.  The caller passes the inputs and outputs only (reference layouts; qx/qy/qz may all
 * be NULL for zero solid flux); the scene record, work tables, CG workspace and CG vectors live in a fixed file-scope
 * device array of hf_noalloc_scratch_bytes() bytes (9 MiB) that every GPU loading the library holds until exit.
 * No cudaMalloc/cudaFree or allocating library call is made.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress), so make it before any stream capture; the address is cached per device together with the
 * context it belongs to and looked up again after cudaDeviceReset or under another context.  All calls on a device share the array: calls whose
 * GPU work overlaps race; each call clears what must start at zero.  state_out (device, optional) receives the solve
 * statistics.  Returns HF_ERR_ARG for n > 64. */
size_t hf_noalloc_scratch_bytes(void);
int hf_noalloc_max_edge(void);
int hf_pressure_solve_noalloc(int n, double h, double rho, double dt, double cg_tol, int cg_max_iter, float *u, float *v,
                              float *w, const float *ax, const float *ay, const float *az, const float *qx,
                              const float *qy, const float *qz, float *p, hf_scene_state *state_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HEATFLOW_B200_H */
