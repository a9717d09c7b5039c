/*
 * giftbte.h — C ABI of the B200-native steady synthetic phonon-BTE solver.
 *
 * This is the drop-in boundary for GiftBTE's StaticBTESynthetic path
 * (Order=2, IterativeScheme=Synthetic, MatrixSolver=LU). Plain C types only:
 * pointers and sizes, no C++ or torch types. Every call returns a status code
 * (GBTE_OK = 0) and never throws or exits; the message of the last failure on
 * a handle is available from gbte_last_error(). A handle owns one CUDA stream
 * and its device memory; it is not thread-safe, distinct handles are
 * independent.
 *
 * Reference interfaces replaced (paths inside the GiftBTE project):
 *   gbte_create          StaticBTESynthetic::StaticBTESynthetic(BTEMesh*,
 *                        BTEBoundaryCondition*, BTEBand*, BTEAngle*, int, int)
 *                        includes/StaticBTESynthetic/StaticBTESynthetic.h:177,
 *                        with the mesh topology of BTEMesh::setMeshParams /
 *                        setMeshParams1 (src/BTEMesh/BTEMesh.cpp:600-1023)
 *                        and the quadrature of BTEAngle (src/BTEAngle/
 *                        BTEAngle.cpp:11-190)
 *   gbte_create_from_deck  the input stage of main() (src/BTEMain.cpp:87-362):
 *                        CONTROL / GEOMETRY / PHONON keyword files, BC table,
 *                        COMSOL or MSH mesh, DATABASE band table
 *   gbte_set_initial     the writes into solver.temperature[],
 *                        heatFlux*Global[] and boundaryThermal[] before solve
 *                        (src/Solution/Solution.cpp:266-285)
 *   gbte_fourier_initial the Fourier pre-solve that seeds those arrays
 *                        (src/StaticFourier/StaticFourier.cpp:934-976,
 *                        src/Solution/Solution.cpp:236-255)
 *   gbte_solve           StaticBTESynthetic::solve(Use_Backup, Num_Max_Iter,
 *                        Use_Limiter, error_temp_limit, error_flux_limit)
 *                        includes/StaticBTESynthetic/StaticBTESynthetic.h:221
 *   gbte_get_fields      the reads of totalEnergy[], temperature[],
 *                        heatFlux{X,Y,Z}Global[], temperatureband[] after
 *                        solve (src/Solution/Solution.cpp:408-413)
 *   gbte_write_outputs   StaticBTESynthetic::_print_out and
 *                        SolutionAll::_print_out (StaticBTESynthetic.cpp:
 *                        2613-2653, Solution.cpp:128-233)
 *   gbte_destroy         StaticBTESynthetic::~StaticBTESynthetic
 *                        (StaticBTESynthetic.cpp:52-223)
 */
#ifndef GIFTBTE_B200_H
#define GIFTBTE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GBTE_ABI_VERSION 1

/* status codes */
#define GBTE_OK 0
#define GBTE_ERR_ARG -1          /* invalid argument or inconsistent sizes */
#define GBTE_ERR_IO -2           /* a deck file is missing or malformed */
#define GBTE_ERR_CUDA -3         /* a CUDA call failed */
#define GBTE_ERR_DIVERGED -4     /* NaN/Inf or 10 consecutive margin increases */
#define GBTE_ERR_TIMEOUT -5      /* a bounded device-side wait gave up */
#define GBTE_ERR_NOMEM -6        /* device allocation failed */
#define GBTE_ERR_MESH -7         /* mesh topology error (open face, no periodic partner) */
#define GBTE_ERR_UNSUPPORTED -8  /* input outside the implemented scope */
#define GBTE_ERR_EXCHANGE -9     /* the exchange function of a direction shard returned non-zero */
#define GBTE_ERR_NOT_CONVERGED 1 /* max_iter reached before the margins (not an error) */

/* precision of the band intensities */
#define GBTE_FP64 0        /* plain FP64 drop-in form */
#define GBTE_FP32_MIXED 1  /* FP32 intensities and sweeps, FP64 moments, macro solve and margins */

typedef struct gbte_handle gbte_handle;

/* Unstructured mesh, coordinates already scaled to metres (node * ScaleX..).
 * 2D: triangles (3 vertices) or quads (4 vertices, COMSOL order
 * v0 v1 v2 v3 with edges v0-v1, v1-v3, v3-v2, v2-v0); boundary elements are
 * edges (2 vertices). 3D: tetrahedra; boundary elements are triangles. */
typedef struct {
    int dimension;            /* 2 or 3 */
    int num_nodes;
    int num_cells;
    int num_boundary_elements;
    const double *node_xyz;   /* [num_nodes * 3] */
    const int *cell_ptr;      /* [num_cells + 1], CSR into cell_verts */
    const int *cell_verts;
    const int *cell_region;   /* [num_cells], 0-based geometry region */
    const int *belem_ptr;     /* [num_boundary_elements + 1] */
    const int *belem_verts;
    const int *belem_tag;     /* [num_boundary_elements], tag as in the BC file */
    double scale_x, scale_y, scale_z;  /* ScaleX/Y/Z (the LSQ stencil is scaled by 1/ScaleX) */
} gbte_mesh_view;

/* Band table (DATABASE columns), material-major [m * num_bands + b]. */
typedef struct {
    int num_materials;
    int num_bands;
    const double *group_velocity;
    const double *relaxation_time;
    const double *heat_capacity;
    const double *lattice_ratio;
    const double *heat_ratio;
    int num_regions;
    const int *region_material;  /* [num_regions], 0-based material of each region */
    int material_dimension;      /* 2 or 3: kappa_bulk = sum C v^2 tau / dim */
} gbte_band_table;

/* Boundary conditions: type 1 isothermal (value = wall T), 2 diffuse,
 * 3 specular, 5 interface between two materials (transmissivity table
 * below), < 0 periodic (partner tag = -type, value = temperature jump),
 * 6 partially specular (value = specularity p in [0, 1]; no counterpart in
 * the reference): an incoming intensity is p times the outgoing value of the
 * outgoing direction nearest its mirror image plus (1 - p) times the diffuse
 * value; the synthetic (macro) correction treats the wall as diffuse; p = 0
 * and p = 1 are exactly types 2 and 3. */
typedef struct {
    int num;
    const int *tag;
    const int *type;
    const double *value;
    /* type 5 (interface wall between two materials,
     * StaticBTESynthetic.cpp:2152-2190): the transmissivity of every band
     * from each material's side, [num][num_materials * num_bands], rows of
     * other types ignored (the interface file's "matter" blocks,
     * BTEBoundaryCondition.cpp:22-35). NULL when no row has type 5. */
    const double *transmissivity;
} gbte_bc_table;

typedef struct {
    int method;   /* 1 = CADOM (uniform midpoint), 2 = Gauss-Legendre, 0 = the explicit list below */
    int n_theta;
    int n_phi;
    /* method 0: the directions and weights as a caller already holds them
     * (BTEAngle::direction / weight / SolidAngle, includes/BTEAngle/
     * BTEAngle.h:12-14); the solver uses s_d = direction_d and the mode
     * weight weight_d / solid_angle as the reference does
     * (StaticBTESynthetic.cpp:603-610) */
    int num_directions;
    const double *direction_xyz;  /* [num_directions * 3] */
    const double *weight;         /* [num_directions] */
    double solid_angle;           /* 2 pi (2D material) or 4 pi (3D material) */
} gbte_angle_spec;

typedef struct {
    int precision;            /* GBTE_FP64 or GBTE_FP32_MIXED */
    int use_limiter;          /* Order=2limit: the gradient limiter of _get_gradient_larger
                                 (StaticBTESynthetic.cpp:1372-1422); GBTE_FP64 only */
    int max_iter;
    double err_temp;          /* ResidualTemp */
    double err_flux;          /* ResidualFlux */
    const double *cell_heat;  /* [num_cells] W/m^3, may be NULL (no source) */
    void *stream;             /* cudaStream_t to run on; NULL = the handle creates one */
    int device;               /* CUDA device ordinal */
    int verbose;              /* 1: print the per-iteration margins like the reference */
    double macro_rtol;        /* relative residual of the macro CG solve; 0 = default 1e-13 */
    int profile;              /* 1: time every kernel launch with CUDA events (gbte_stats.kernel_ms) */
    int sweep_bands;          /* bands per CTA of the upwind sweep (1..32); 0 = automatic */
    int sweep_far_slots;      /* on-chip slots per direction for upwind reads older than the sweep's
                                 ring: 0 = automatic (2048), < 0 = none (such reads go to memory) */
    int direction_batch;      /* most directions whose gradient/residual/correction buffers are held at
                                 once; 0 = automatic (all that fit in device memory) */
    const double *cell_scatter; /* [num_cells] scattering-rate multiplier s_c > 0 (no counterpart in the
                                 reference): the transport uses tau_b / s_c in cell c; the synthetic
                                 correction keeps the band table's tau; NULL = 1 everywhere */
    int cell_order;           /* 0 = automatic: cells are renumbered inside the library along a Morton
                                 curve of their centres (per geometry of a batch) for memory locality;
                                 1 = keep the caller's order. Every cell array of this ABI is in the
                                 caller's order either way; results agree to rounding. */
    int order;                /* spatial order of the transport: 0 or 2 = second order (CONTROL Order=2,
                                 StaticBTESynthetic::solve), 1 = first order (Order=1, solve_firstorder:
                                 upwind cell values, no gradient reconstruction) */
    int scheme;               /* 0 = Synthetic (IterativeScheme=Synthetic: the macro correction), 1 =
                                 Sequential (IterativeScheme=Sequential, solve_DOM /
                                 solve_DOM_firstorder: plain source iteration, T from the moments) */
    int macro_exact;          /* 1: every macro CG solve reaches macro_rtol from its start, as the
                                 reference's LU solve is exact, so the outer iterates follow the
                                 reference's step by step; 0 (default): a solve warm-started from the
                                 previous outer iteration stops after a 3e-3 residual reduction (same
                                 fixed point, fewer CG iterations) */
    int sweep_vector;         /* bands each thread of the upwind sweep updates (1, 2, or 4 in FP32;
                                 the band count must be a multiple); 0 = automatic. Results do not
                                 depend on it. */
    int sweep_kernel;         /* 1 = the block sweep (a CTA per direction and chunk of bands, one
                                 barrier per level), 2 = the warp-independent sweep (a warp per
                                 direction and sweep_vector bands, no block barrier), 3 = the
                                 wide-level sweep (corrections read back from device memory, no
                                 shared-memory ring: for levels of thousands of cells, e.g. 3D
                                 tetrahedra; plans without far slots only), 0 = the fastest on the
                                 first outer iteration. Results do not depend on it. */
    int gradient_dirs;        /* launch shape of the LSQ gradient: 1, 2 or 4 = a thread per cell and
                                 4 bands covering that many directions (one load of a stencil entry
                                 serves them all); 5, 6 = a warp per cell, lanes over band groups
                                 and directions, 1 or 2 directions per lane (band count <= 128);
                                 7, 8 = shared-memory tiles: a CTA per block of consecutive cells
                                 (3D: 32 or 64, 2D: 64 or 128) stages the block's stencil once and,
                                 direction by direction, the rows of the block's stencil union;
                                 9, 10 = the tiles of 7, 8 with eight lanes per cell (FP32-mixed
                                 form, band count a multiple of 32, 40 or 48; others run 2);
                                 0 = the fastest on the first outer iteration. Results do not
                                 depend on it. */
    int residual_form;        /* launch shape of the second-order residual: 1 = a thread per cell
                                 and 4 bands, 5, 6 = a warp per cell as for gradient_dirs, 7, 8 =
                                 shared-memory tiles of the blocks of gradient_dirs 7, 8 (the
                                 block's cells and face neighbours); 0 = the fastest on the first
                                 outer iteration. Results do not depend on it. */
    int adjoint_history;      /* gbte_vjp: Anderson acceleration of the transposed iteration with
                                 this many difference pairs (1..8); 0 = 6; -1 = the plain iteration
                                 lam += A^-T r. The fixed point, and the stopping rule, are the same. */
} gbte_options;

#define GBTE_NUM_KERNELS 16

typedef struct {
    int iterations;
    double err_temp;          /* last temperature margin */
    double err_flux;          /* last heat-flux margin */
    double solve_ms;          /* device time of the outer loop (CUDA events) */
    double setup_ms;          /* host+device setup inside gbte_create */
    double transport_ms;      /* gradient + residual + sweep + boundary + moments */
    double macro_ms;          /* synthetic correction (CG solves) */
    long long macro_cg_iterations;
    long long updates;        /* band*direction*cell updates performed */
    int num_directions;
    int num_bands;
    int num_cells;
    int max_levels;           /* deepest sweep over all directions */
    int lagged_faces;         /* upwind faces lagged to break cycles (3D) */
    int inner_iterations;     /* macro Picard steps in the last outer iteration */
    long long kernel_launches;            /* kernels launched by this solve */
    double kernel_ms[GBTE_NUM_KERNELS];   /* per-kernel device time when options.profile = 1 */
    long long kernel_count[GBTE_NUM_KERNELS];
    int sweep_bands;          /* bands-per-CTA cap of the sweep in use (options.sweep_bands, or
                                 the autotuner's pick on the handle's first outer iteration) */
    int direction_batch;      /* directions per batch of the transport stage */
    int sweep_stage_levels;   /* levels the sweep stages ahead in shared memory (autotuned, 2..4) */
    int sweep_vector;         /* bands per sweep thread in use (options.sweep_vector or autotuned) */
    int sweep_threads;        /* threads per sweep CTA in use */
    int sweep_kernel;         /* sweep kernel in use: 1 block, 2 warp-independent, 3 wide-level */
    int gradient_dirs;        /* gradient launch shape in use (0: the 1-band form ran) */
    int residual_form;        /* residual launch shape in use (0: the 1-band form ran) */
} gbte_stats;

/* Name of kernel slot i of gbte_stats.kernel_ms (NULL past the last one). */
const char *gbte_kernel_name(int i);

/* Host-only summary of a deck or mesh (no CUDA needed): what gbte_create
 * would build. Replaces the reference's stdout trace of the input stage. */
typedef struct {
    int dimension;
    int num_nodes;
    int num_cells;
    int num_faces;             /* global face list (Element_Faces) */
    int num_boundaries;        /* boundary elements matched to the BC table */
    int num_boundary_sides;    /* 2 * num_boundaries */
    int num_bands;
    int num_directions;
    int num_materials;
    int max_levels;            /* deepest upwind sweep over all directions */
    int lagged_faces;          /* upwind faces lagged to break cycles */
    double kappa_bulk;         /* material 0 */
    double capacity_bulk;      /* material 0 */
    double total_volume;
    double max_iter_or_zero;   /* MaxNumIter from CONTROL (decks only) */
    double err_temp, err_flux; /* ResidualTemp / ResidualFlux from CONTROL (decks only) */
    int max_level_width;       /* widest sweep level (cells) */
    int sweep_ring;            /* on-chip correction ring of the sweep (positions) */
    int far_slots;             /* on-chip slots for upwind reads older than the ring */
    long long far_refs;        /* upwind reads older than the ring, all directions */
    long long index_entries_checked; /* entries range-checked (0 unless GBTE_DEBUG is set or built in) */
    int transient;             /* CONTROL State=Transient (decks only) */
    double time_step;          /* TimeStep and TotalTime from CONTROL (decks only; -1 if absent) */
    double total_time;
} gbte_deck_info;

int gbte_inspect_deck(const char *dir, gbte_deck_info *info);
int gbte_inspect_mesh(const gbte_mesh_view *mesh, const gbte_band_table *bands, const gbte_bc_table *bcs,
                      const gbte_angle_spec *angles, gbte_deck_info *info);

/* Default options (FP64, max_iter 10000, margins 1e-6/1e-4 as the reference). */
void gbte_default_options(gbte_options *opt);

/* sizeof(gbte_options) as this library was built: a caller compiled against
 * another version of this header can check it before passing options (no
 * counterpart in the reference). */
size_t gbte_options_size(void);

int gbte_create(const gbte_mesh_view *mesh, const gbte_band_table *bands, const gbte_bc_table *bcs,
                const gbte_angle_spec *angles, const gbte_options *opt, gbte_handle **out);

/* Batched solve of `num` independent geometries (no counterpart in the
 * reference, which solves one geometry per run): one handle over their
 * disjoint union, so every kernel launch of the outer iteration serves all
 * geometries at once (each sweep CTA walks one geometry's levels of one
 * direction). All geometries share the band table, the angular quadrature,
 * ScaleX and the options; meshes[k] and bcs[k] describe geometry k with its
 * own boundary tags. The fields of the handle (gbte_set_initial,
 * gbte_get_fields, options.cell_heat) are the geometries' cell arrays
 * concatenated in order; gbte_batch_geometries gives the offsets. The outer
 * iteration stops when every geometry's own margins are below the limits,
 * and the macro Picard loop when every geometry's own change is. */
int gbte_batch_create(int num, const gbte_mesh_view *meshes, const gbte_band_table *bands,
                      const gbte_bc_table *bcs, const gbte_angle_spec *angles, const gbte_options *opt,
                      gbte_handle **out);

/* Number of geometries of a handle (1 for gbte_create) and, when
 * cell_offsets is not NULL, their cell ranges [num + 1]. */
int gbte_batch_geometries(gbte_handle *h, int *num, int *cell_offsets);

/* Reads <dir>/input/{CONTROL,GEOMETRY,PHONON} and the files they name
 * (relative paths resolved against <dir>, like the reference's CWD).
 * Options from CONTROL (Order, margins, MaxNumIter) override *opt. */
int gbte_create_from_deck(const char *dir, const gbte_options *opt, gbte_handle **out);

/* Initial lattice temperature [num_cells] (required before the first solve
 * unless gbte_fourier_initial is used), optional initial heat flux
 * [num_cells*3] (the previous-iterate flux of the first margin), optional
 * boundary temperatures overriding the BC values per boundary element
 * [num_boundary_elements] (NULL keeps the BC values). */
int gbte_set_initial(gbte_handle *h, const double *T0, const double *q0, const double *boundary_thermal);

/* Fourier pre-solve with kappa_bulk on the device; sets T0 and q0. */
int gbte_fourier_initial(gbte_handle *h);

/* Allocation-free variant of gbte_fourier_initial (no counterpart in the
 * reference): the same Fourier pre-solve, with all of its scratch vectors
 * taken from one static device array inside this library instead of memory
 * allocated on the device. It is for callers that must not allocate device
 * memory once their run has started, typically because they hand out all
 * device memory from their own pool reserved at start-up, or run under a
 * fixed device-memory limit, where an allocation mid-run can fail, stall or
 * fragment that pool. Such a caller creates the handle during start-up and
 * re-seeds it here later. The call allocates nothing on the device or in
 * pinned memory. Limits: at most 131072 cells and 131072 node slots (nodes x
 * materials); larger meshes get GBTE_ERR_ARG. The static array (about 7.9 MB)
 * is held by every GPU that loads the library until the process exits. The
 * first call on each device looks up the array's device address and keeps
 * it for the life of that device's primary context (a caller that tears the
 * context down with cudaDeviceReset must not call this entry point again in
 * the same process); make that first call before any stream capture. All
 * calls share the one array, so calls that overlap on the GPU (other threads
 * or streams) race; the CG reduction slots are cleared on every solve,
 * everything else is written before it is read. Results go to the handle as
 * with gbte_fourier_initial: the same temperature and flux; for an
 * FP32-mixed handle the gradient of the stored base temperature is formed
 * on the device here (on the host there), so it can differ in the last bits.
 * Handles of a batched solve (gbte_batch_create) get GBTE_ERR_UNSUPPORTED. */
int gbte_fourier_initial_noalloc(gbte_handle *h);

/* Runs the outer source iteration until both margins are below the limits
 * (GBTE_OK), max_iter is reached (GBTE_ERR_NOT_CONVERGED) or it diverges.
 * stats may be NULL. */
int gbte_solve(gbte_handle *h, gbte_stats *stats);

/* gbte_solve with the per-call limits of the reference's
 * solve(Use_Backup, Num_Max_Iter, Use_Limiter, error_temp_limit,
 * error_flux_limit): runs at most max_iter further outer iterations from the
 * current state and stops when both margins are at or below the limits
 * (limits of 0 run exactly max_iter iterations). */
int gbte_solve_with(gbte_handle *h, int max_iter, double err_temp, double err_flux, gbte_stats *stats);

/* Result fields (any pointer may be NULL):
 * T_energy [Nc]  totalEnergy      -> Temperature.dat
 * T_lattice[Nc]  macro temperature -> TempLattice.dat
 * q        [Nc*3] heat flux        -> HeatFlux.dat
 * T_band   [Nb*Nc] band temperatures -> Tempband.dat */
int gbte_get_fields(gbte_handle *h, double *T_energy, double *T_lattice, double *q, double *T_band);

/* Writes Temperature.dat, TempLattice.dat, HeatFlux.dat, Tempband.dat and
 * Result.vtk into <dir> in the reference's formats (17 significant digits). */
int gbte_write_outputs(gbte_handle *h, const char *dir);

/* Sizes of the problem held by a handle (any pointer may be NULL). */
int gbte_get_sizes(gbte_handle *h, int *num_cells, int *num_bands, int *num_directions, int *num_boundary_sides);

/* Cell centres [Nc*3] and volumes [Nc] as the solver sees them. */
int gbte_get_geometry(gbte_handle *h, double *centers, double *volumes);

/* Adjoint of the converged solve (no counterpart in the reference, which
 * has no derivatives). For the objective
 *   J = sum_c T_bar[c] T[c] + sum_c q_bar[c] . q[c]
 * of the fields gbte_get_fields returns (T the macro lattice temperature, q
 * the heat flux; either cotangent may be NULL = 0), it writes:
 *   grad_tau[Nb]        dJ/d alpha_b for a multiplier alpha_b on band b's
 *                       relaxation time (transport and synthetic correction
 *                       alike), at alpha = 1
 *   grad_scatter[Nc]    dJ/d s_c for the cell scattering multipliers
 *                       (options.cell_scatter), at their current values
 *   grad_specularity[n] dJ/dp per row of the boundary table given at
 *                       creation (partially specular rows, type 6; 0 for the
 *                       other rows)
 * Any output may be NULL. It differentiates the fixed point the last
 * gbte_solve reached, implicitly: the adjoint state solves the transposed
 * equations by the transposed source iteration (sweeps in the opposite
 * directions, the transposed synthetic correction, Anderson-accelerated by
 * default: options.adjoint_history), until the residual of the adjoint
 * equations, ||(dF/de)^T lam + dJ/de||, is <= tol ||dJ/de||, or max_iter
 * iterations ran. Call it after a solve that
 * converged to tight margins; the gradient is that of the state the solve
 * left. FP64 handles only (GBTE_ERR_UNSUPPORTED otherwise), not batched
 * handles. It keeps one more band-state array (Nd*Nc*Nb doubles) and
 * reuses the transport scratch; a later gbte_solve continues unchanged. */
typedef struct {
    int iterations;     /* transposed source iterations */
    int picard_steps;   /* Picard steps of the synthetic correction, transposed */
    double change;      /* last relative change of the gradient */
    double vjp_ms;      /* device time of the adjoint solve and the assembly */
    double residual;    /* ||(dF/de)^T lam + dJ/de|| / ||dJ/de|| at the returned gradient */
} gbte_vjp_stats;

int gbte_vjp(gbte_handle *h, const double *T_bar, const double *q_bar, int max_iter, double tol, double *grad_tau,
             double *grad_scatter, double *grad_specularity, gbte_vjp_stats *st);

/* The explicit transient solver (Transient::solve, src/TransientBTE/
 * TransientSolver.cpp:11-302, which the reference runs for CONTROL
 * State=Transient from src/Solution/Solution.cpp:500-520). It starts from the
 * thermal grating T = cos(2 pi x / ScaleX) (transient.cpp:586-604), whatever
 * gbte_set_initial gave, and the reference's starting wall values, then takes
 * explicit steps e <- e (1 - dt / tau) - dt Re (second-order upwind fluxes,
 * the equilibrium C T_old / tau, the incoming walls) for the integers
 * n < total_time / time_step, stopping early when both margins (sum |T -
 * T_old| / Nc / max |T|, and the same for |q|) reach err_temp and err_flux.
 * After each step the lattice temperature of cell probe_cell (the caller's
 * numbering) is written to probe_history[step] for the first history_len
 * steps (the reference's TTG.dat records cell 0); may be NULL.
 * gbte_get_fields then gives the final lattice temperature and heat flux.
 * FP64 handles of one geometry, second order (GBTE_ERR_UNSUPPORTED
 * otherwise). The TDTR heat pulses (IsTDTR) are not built: the reference
 * stops there ("contact us", src/BTEMain.cpp:154-165). */
typedef struct {
    long long steps;   /* explicit steps taken */
    long long updates; /* band * direction * cell updates */
    double err_temp;   /* margins of the last step */
    double err_flux;
    double solve_ms;   /* device time */
} gbte_transient_stats;

int gbte_transient_solve(gbte_handle *h, double time_step, double total_time, double err_temp, double err_flux,
                         int probe_cell, double *probe_history, long long history_len, gbte_transient_stats *st);

/* Direction sharding of one solve over several handles (one per GPU and
 * process, or several in one process): the reference's decomposition of the
 * directions over MPI ranks (StaticBTESynthetic.cpp:247-300), with its
 * per-iteration MPI_Allreduce of the moments (StaticBTESyntheticSolver.cpp:
 * 130-136) and MPI_Allgather of the boundary intensities
 * (StaticBTESynthetic.cpp:2220-2226). Here one sum over a contiguous block
 * replaces both: every handle zeroes the boundary values of the directions
 * it does not hold, so the sum of those is their union.
 *
 * After the call, the handle's transport stage covers directions
 * [dir_begin, dir_begin + dir_count) only. Every outer iteration then calls
 *   exchange(user, buf, count, stream)
 * twice: once on the moments and boundary values of the iteration, once on
 * the margins. buf is device memory of `count` doubles; the function must
 * replace it, in place, by its element-wise sum over all handles of the
 * shard set (an NCCL all-reduce of ncclDouble/ncclSum on `stream`, a
 * cudaStream_t, does exactly that), ordered after the work enqueued on
 * `stream` and before the work enqueued after it returns. It returns 0, or
 * a non-zero code that makes gbte_solve return GBTE_ERR_EXCHANGE. Every
 * handle of a set must be created from the same inputs and options, its
 * blocks must cover every direction exactly once, and all of them must call
 * gbte_set_initial (or gbte_fourier_initial) and gbte_solve alike: the
 * margins of the handle holding direction 0 decide for all of them, so
 * they stop at the same iteration. Fields are the whole solve's on every
 * handle. dir_count = 0 or exchange = NULL returns to all directions. Not
 * for gbte_vjp (GBTE_ERR_UNSUPPORTED). No counterpart in the reference
 * beyond its MPI decomposition. */
typedef int (*gbte_exchange_fn)(void *user, double *buf, size_t count, void *stream);

int gbte_set_direction_shard(gbte_handle *h, int dir_begin, int dir_count, gbte_exchange_fn exchange, void *user);

/* Turns per-launch kernel timing (options.profile) on or off for the next
 * solves of a handle. While it is on, the transport stage is launched kernel
 * by kernel instead of as the CUDA graph. No counterpart in the reference. */
int gbte_set_profile(gbte_handle *h, int on);

const char *gbte_last_error(const gbte_handle *h);
const char *gbte_status_string(int status);
int gbte_destroy(gbte_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* GIFTBTE_B200_H */
