// Device-side solver of the steady synthetic phonon BTE (internal header).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "gbte_internal.h"

namespace gbte {

// Pointers into device memory describing the flattened mesh.
struct DMesh {
    int dim, nc, nn, nbs, nbd, nslot, ncf, nf;
    double inv_Lx;
    const int *cf_ptr, *cf_nbr, *cf_bside, *cf_bound, *cf_v, *cf_face;
    const double *cf_area, *cf_nx, *cf_ny, *cf_nz, *cf_fx, *cf_fy, *cf_fz;
    const double *vol, *cx, *cy, *cz, *heat;
    const double *tsc;  // 1 / s_c: per-cell scale of the relaxation time (scattering multiplier s_c)
    int nmat;           // materials: node values are kept per (node, material) slot
    const int *matter;  // [nc] cell material, nullptr with one material
    // Wall faces read their node values at the raw node index of the slot
    // array; where that slot's material is not the wall cell's, the value is
    // formed again with the cell material's coefficients ("cross" values):
    // cf_x[3k + t] is the cross value of vertex t of cell-face k, or -1;
    // cross value x interpolates the entries xs_ptr[x] .. xs_ptr[x + 1] of
    // xs_src (y >= 0: cell y_cell[y] under material y_mat[y]; -1 - s: wall
    // side s under material x_mat[x]) with weights xs_w.
    int ncross_x, ncross_y;
    const int *cf_x, *x_mat, *xs_ptr, *xs_src, *y_cell, *y_mat;
    const double *xs_w;
    const int *nbr_ptr, *nbr_idx;
    const double *lsq_w;
    const float *lsq_wf;
    const float4 *lsq_pk;  // per stencil entry {w_x, w_y, w_z, neighbour index bits} in FP32
    const float4 *lsq_ws;  // per cell {sum w_x, sum w_y, sum w_z, 0} of the FP32 weights
    const float4 *cf_r4, *cf_rn4;  // per cell-face FP32 offsets to the face centre from the cell / its neighbour
    const double *face_w;
    const int *f_cf0;
    const int *b_type, *b_connect;
    const double *b_T;
    const int *bs_cell, *bs_cf;
    const double *bs_trans;  // [2*nbd][nb] interface transmissivity per side, or nullptr
    const int *nv_ptr, *nv_src;
    const double *nv_w;
    const int *nt_ptr, *nt_src;
    const double *nt_w;
    const double *node_x, *node_y, *node_z;
};

// Band/direction constants. Band arrays are material-major [m * nb + b];
// mat[c] is cell c's material (nullptr with one material, whose offset is 0).
struct DPhys {
    int nb, nd, nmat;
    const double *vmag, *tau, *C, *lat, *hr;  // [nmat * nb]
    double kappa, capb;                       // material 0's (the one material of most decks)
    const double *kap, *capm;                 // [nmat] kappa_bulk and C_bulk per material
    const int *mat;                           // [nc] or nullptr
    const double *sx, *sy, *sz, *w;           // [nd]
};
// band-array offset of cell c's material
__host__ __device__ __forceinline__ int mat_off(const DPhys &p, int c) { return p.mat ? p.mat[c] * p.nb : 0; }

struct SolverConfig {
    int precision = 0;
    int use_limiter = 0;
    int max_iter = 10000;
    double err_temp = 1e-6, err_flux = 1e-4;
    double macro_rtol = 1e-13;
    int verbose = 0;
    int profile = 0;
    int sweep_bands = 0;      // bands per sweep CTA, 0 = automatic
    int sweep_vector = 0;     // bands per sweep thread (1, 2, 4), 0 = automatic
    int sweep_kernel = 0;     // 1: block sweep kernel, 2: warp-independent kernel, 3: wide-level kernel, 0 = automatic
    int sweep_far_slots = 0;  // far-slot cap of the sweep plan: 0 = automatic, < 0 = none
    int gradient_dirs = 0;    // gradient launch shape (1, 2, 4: directions per thread; 5, 6: warp per cell;
                              // 7, 8: shared-memory tiles), 0 = automatic
    int residual_form = 0;    // residual launch shape (1: thread per cell; 5, 6: warp per cell; 7, 8: tiles),
                              // 0 = automatic
    int adjoint_anderson = 6; // history of the adjoint's Anderson acceleration (0: plain iteration)
    int direction_batch = 0;  // most directions per transport batch, 0 = automatic
    std::vector<double> cell_scatter;  // scattering-rate multiplier s_c per cell (empty: 1)
    int order = 2;            // 2: second-order upwind faces (solve); 1: first order (solve_firstorder)
    bool sequential = false;  // Sequential scheme (solve_DOM): no macro correction, T = T_lat
    bool macro_exact = false; // macro CG solves to macro_rtol even from a warm start
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
};

enum KernelId {
    K_GRADIENT = 0, K_RESIDUAL, K_SWEEP, K_BOUND_OUT, K_MOMENTS, K_SIDE_MOMENTS, K_NODE_INTERP, K_REMACRO,
    K_GATHER, K_MACRO_BC, K_TINTERP, K_MACRO_RHS, K_PCG, K_REDUCE, K_COPY, K_INIT, K_NUM
};
const char *kernel_name(int k);

struct VjpStats {
    int iterations = 0, picard_steps = 0;
    double change = 0, ms = 0, residual = 0;
};

struct TransientStats {
    long long steps = 0, updates = 0;
    double err_temp = 0, err_flux = 0, ms = 0;
};

struct SolveStats {
    int iterations = 0, inner_iterations = 0;
    double err_temp = 0, err_flux = 0, solve_ms = 0, transport_ms = 0, macro_ms = 0;
    long long cg_iterations = 0, updates = 0, launches = 0;
    double kernel_ms[K_NUM] = {0};
    long long kernel_count[K_NUM] = {0};
};

// Launch plan of the cluster-resident CG for one CSR system: cluster size
// (0 = the system does not fit, use the grid-wide kernel), the per-CTA
// layout bounds (off-diagonals per row K, rows, halo entries, sends),
// whether the two-level preconditioner is on, the dynamic shared memory and
// the partitioned system in device memory.
struct CgPlan {
    int C = 0, K = 0, nrmax = 0, hmax = 0, smax = 0, coarse = 0;
    size_t smem = 0;
    int *part_ptr = nullptr, *perm = nullptr, *ell_col = nullptr, *nsend = nullptr, *snd_src = nullptr,
        *snd_dst = nullptr, *agg_ptr = nullptr;
    double *ell_val = nullptr, *diag = nullptr, *ainv = nullptr;
};

// Sum of `count` doubles of device memory over the handles of a direction
// shard set, in place, after the work already enqueued on `stream`; the
// solver enqueues its next work on `stream` once the call returns. 0 = ok.
typedef int (*ExchangeFn)(void *user, double *buf, size_t count, void *stream);

class Solver {
public:
    ~Solver();
    Error init(const FlatMesh &m, const Bands &b, const Angles &a, const std::vector<double> &cell_heat,
               const SolverConfig &cfg);
    Error set_initial(const double *T0, const double *q0, const double *boundary_thermal_per_bside);
    Error fourier_initial();
    Error fourier_initial_noalloc();
    int fourier_iterations = 0;
    Error solve(SolveStats &st);
    Error get_fields(double *T_energy, double *T_lattice, double *q, double *T_band);
    // Vector-Jacobian product of the converged fixed point: given cotangents
    // of the lattice temperature (Tbar, nc) and heat flux (qbar, 3 nc), the
    // derivatives of <Tbar, T> + <qbar, q> with respect to a multiplier on
    // each band's relaxation time (g_tau, nb), each cell's scattering
    // multiplier (g_cell, nc) and each boundary's specularity (g_bnd, nbd;
    // partially specular walls only)
    Error vjp(const double *Tbar, const double *qbar, int max_iter, double tol, double *g_tau, double *g_cell,
              double *g_bnd, VjpStats &st);
    // Explicit transient run from the grating start (FP64 form): steps of dt
    // up to total, stopping early when both margins reach their limits; the
    // temperature of cell `probe` after each step goes to hist[0 .. cap);
    // wall_cell[ib]: this handle's index of the cell numbered ib in the
    // caller's order (empty: the same order), for the start's specular walls
    Error transient(double dt, double total, double err_t, double err_q, int probe, double *hist, long long cap,
                    const std::vector<int> &wall_cell, TransientStats &st);
    // Direction shard: this handle's transport covers directions
    // [begin, begin + count) only, and every outer iteration sums the moments
    // and boundary values over the shard set through `fn` (count = 0 or
    // fn = NULL: all directions, no exchange)
    Error set_shard(int begin, int count, ExchangeFn fn, void *user);
    int shard_begin() const { return dlo_; }
    int shard_end() const { return dhi_ < 0 ? ang.nd : dhi_; }

    FlatMesh mesh;
    Bands bands;
    Angles ang;
    Schedule sched;
    SolverConfig cfg;
    bool initialised = false;
    std::string last_error;
    int tuned_sweep_bands_ = 0;  // bands-per-CTA cap the sweep autotuner picked (0 = not yet)
    int tuned_sweep_look_ = 4;   // levels the sweep stages in shared memory (the autotuner's pick)
    int tuned_sweep_vb_ = 1;     // bands per sweep thread (the autotuner's pick)
    int tuned_sweep_threads_ = 256;  // most threads per sweep CTA (the autotuner's pick)
    int tuned_sweep_warp_ = 0;   // 1: the warp-independent sweep kernel won (the autotuner's pick)
    int tuned_sweep_wpc_ = 1;    // warps per CTA of that kernel
    int tuned_sweep_wide_ = 0;   // 1: the wide-level sweep kernel won (the autotuner's pick)
    int tuned_grad_dirs_ = 0;    // directions per gradient thread (1, 2 or 4; 0 = not yet tuned)
    int last_grad_dirs_ = 0;     // the same, of the last solve's gradient launches (0: 1-band form)
    // tiles of the shared-memory gradient (gradient_dirs 7, 8), built by the
    // first solve for two block sizes
    struct TileDev {
        int B = 0, nblk = 0, umax = 0, qmax = 0;
        int *ptr = nullptr, *cells = nullptr;
        unsigned short *loc = nullptr;
    };
    std::vector<TileDev> tiles_;
    struct FaceTileDev {
        int B = 0, nblk = 0, umax = 0;
        int *ptr = nullptr, *cells = nullptr;
        unsigned short *floc = nullptr;
    };
    std::vector<FaceTileDev> ftiles_;  // tiles of the shared-memory residual (residual_form 7, 8)
    bool tiles_built_ = false;
    Error grad_tiles();
    int tuned_res_form_ = 0;     // residual launch shape (1 thread per cell, 5/6 warp per cell; 0 = not yet tuned)
    int last_res_form_ = 0;      // the same, of the last solve's residual launches (0: 1-band form)
    // launch shape of the last solve's sweep (last_sweep_warp_: 0 block, 1 warp, 2 wide-level kernel)
    int last_sweep_vb_ = 0, last_sweep_threads_ = 0, last_sweep_warp_ = 0;
    int ndb_ = 1;                // directions per batch of the gradient/residual/correction buffers

private:
    template <typename S, int DIM> Error solve_t(SolveStats &st);
    template <int DIM>
    Error transient_t(double dt, double total, double err_t, double err_q, int probe, double *hist, long long cap,
                      const std::vector<int> &wall_cell, TransientStats &st);
    Error alloc_all();
    Error cg_solve(const CgPlan &pl, const int *ptr, const int *idx, const double *val, const double *dinv, double *x,
                   const double *b, double rtol, double eta, long long &iters, double *scal, double *r, double *z,
                   double *p, double *Ap, const double *t1, double *sq);
    Error cg_plan(const std::vector<int> &ptr, const std::vector<int> &idx, const std::vector<double> &val,
                  CgPlan &pl);
    CgPlan kplan_, kfplan_;  // macro and Fourier systems
    void *dalloc(size_t bytes);
    std::vector<void *> allocs_;
    DMesh dm_{};
    DPhys dp_{};
    // state
    // storage-type arrays: deviations [nd][nc][nb]; gradients (x DIM),
    // residuals (level order) and sweep corrections (cell order) for one
    // batch of ndb_ directions [ndb_][nc][nb]
    void *eps_ = nullptr, *grad_ = nullptr, *res_ = nullptr, *corr_ = nullptr;
    double *Tbase_ = nullptr, *gTb_ = nullptr;
    double *Bflux_ = nullptr;  // [nd][nc] base-field face flux sums of the residual
    double *eb_ = nullptr, *eb_snap_ = nullptr;
    double *T_ = nullptr, *Told_ = nullptr, *Tlat_ = nullptr, *E_ = nullptr, *q_ = nullptr, *qold_ = nullptr,
           *Tband_ = nullptr, *remacro_ = nullptr, *Th_ = nullptr, *Q_ = nullptr, *Ths_ = nullptr, *Qs_ = nullptr,
           *ThV_ = nullptr, *QV_ = nullptr, *bTm_ = nullptr, *bTovr_ = nullptr, *TV_ = nullptr, *rhs_ = nullptr,
           *T1_ = nullptr, *red_ = nullptr;
    // cross values of wall faces (multi-material): per (cell, material) pair
    // moments ThC/QC (in the exchanged block) and their node values ThX/QX
    double *ThC_ = nullptr, *QC_ = nullptr, *ThX_ = nullptr, *QX_ = nullptr;
    // diffuse weights / specular map
    double *dif_w_ = nullptr;
    double *dsum_ = nullptr;  // [wall side][band] diffuse re-emission sums
    int *spec_src_ = nullptr;
    int *tr_nf_ = nullptr;  // transient start: mirror direction per (wall side, direction)
    bool need_snapshot_ = false;
    // schedule on device
    int *lvl_cells_ = nullptr, *lvl_ptr_ = nullptr, *dir_lvl_off_ = nullptr;
    int ring_ = 0;           // on-chip ring of the sweep (positions, power of two)
    int far_slots_ = 0;      // on-chip far slots of the sweep (0: far reads go to memory)
    // level-ordered sweep records per direction: sum of outgoing A/V (s.n)
    // and up to 4 incoming (neighbour position, A/V (s.n)) pairs
    void *rec_ = nullptr;  // SweepRec<storage type>[nd][nc] in level order
    int *pos_of_ = nullptr;
    double *wtab_ = nullptr;
    double *kb_ = nullptr;
    // warm starts of the macro solves: solution of each Picard step of the
    // previous outer iteration
    std::vector<double *> warm_;
    std::vector<char> warm_ok_;
    double last_margin_ = 1.0;
    unsigned char *lag_ = nullptr;
    // Fourier pre-solve system (StaticFourier._get_coefficient_macro), negated, CSR
    int *KF_ptr_ = nullptr, *KF_idx_ = nullptr;
    double *KF_val_ = nullptr, *KF_dinv_ = nullptr, *bTF_ = nullptr;
    int *bF_dir_ = nullptr;
    bool fourier_singular_ = true;
    // macro matrix (negated, SPD), CSR
    int *K_ptr_ = nullptr, *K_idx_ = nullptr;
    double *K_val_ = nullptr, *K_dinv_ = nullptr;
    double *cg_r_ = nullptr, *cg_z_ = nullptr, *cg_p_ = nullptr, *cg_Ap_ = nullptr, *cg_scal_ = nullptr;
    double *h_pinned_ = nullptr;
    // independent geometries of a batched solve (1 otherwise): cell ranges on
    // the device, and pinned per-geometry reduction results
    int ncomp_ = 1;
    int *comp_ptr_d_ = nullptr;
    int *comp_done_d_ = nullptr;  // per geometry: its Picard loop is done
    Error picard_components(double limit, std::vector<char> &done, double &internal);
    double *h_comp_ = nullptr;
    bool have_initial_ = false;
    bool started_ = false;
    int coop_blocks_ = 0;
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    // per-launch profiling (options.profile)
    std::vector<cudaEvent_t> pev_;
    std::vector<int> pid_;
    int pused_ = 0;
    void prof_begin(int id);
    void prof_end();
    void prof_collect(SolveStats &st);
    long long launches_ = 0;
    int last_inner_ = 0;  // Picard steps of the last outer iteration's macro correction
    // the transport stage of one outer iteration as a CUDA graph (built on
    // the first iteration that is not the autotuner's; off when the stream
    // cannot be captured)
    cudaGraphExec_t tgraph_ = nullptr;
    long long tgraph_launches_ = 0;
    // a direction-sharded solve: the stage after the exchange as a second graph
    cudaGraphExec_t tgraph2_ = nullptr;
    long long tgraph2_launches_ = 0;
    // direction shard [dlo_, dhi_) (dhi_ < 0: all directions) and its exchange
    int dlo_ = 0, dhi_ = -1;
    ExchangeFn xfn_ = nullptr;
    void *xuser_ = nullptr;
    // Tlat, E, q, Tband, Th, Q and the boundary values in one block, the
    // buffer of the exchange (xch_n_ doubles)
    double *xch_ = nullptr;
    size_t xch_n_ = 0;
    bool graph_ok_ = true;
    // adjoint state and scratch (allocated by the first vjp)
    double *adj_lam_ = nullptr, *adj_ebar_ = nullptr, *adj_ebb_ = nullptr, *adj_dbar_ = nullptr;
    double *adj_cell_ = nullptr;  // per-cell / per-side / per-node cotangents, one block
    int *adj_int_ = nullptr;      // transposed stencil, boundary cells, periodic readers, opposite directions
    double *adj_wt_ = nullptr;    // transposed stencil weights and stencil weight sums
    size_t adj_nT_ = 0, adj_nbcell_ = 0, adj_nper_ = 0, adj_nsinv_ = 0;
    std::vector<int> spec_h_;  // specular source per (wall side, direction), host copy
    double *adj_warm_ = nullptr;  // reverse Picard solutions of the previous adjoint iteration
    int adj_warm_n_ = 0;
    double *adj_aa_ = nullptr;    // Anderson history of the adjoint iteration (adj_aa_n_ pairs)
    int adj_aa_n_ = 0;
    Error adj_setup();
};

}  // namespace gbte
