// Host-side data structures of the B200 solver (not part of the C ABI).
#pragma once
#include <cstdint>
#include <memory>
#include <new>
#include <type_traits>
#include <string>
#include <utility>
#include <vector>

namespace gbte {

// An allocator whose resize leaves new elements default-initialised (no
// zeroing for scalars), so that a large host array is first written, and
// its pages first touched, by the threads that fill it.
template <typename T>
struct DefaultInitAlloc : std::allocator<T> {
    template <typename U>
    struct rebind {
        using other = DefaultInitAlloc<U>;
    };
    DefaultInitAlloc() = default;
    template <typename U>
    DefaultInitAlloc(const DefaultInitAlloc<U> &) noexcept {}
    template <typename U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void *>(p)) U;
    }
    template <typename U, typename... A>
    void construct(U *p, A &&...a) {
        ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
    }
};
template <typename T>
using HostArray = std::vector<T, DefaultInitAlloc<T>>;

struct Error {
    int code;
    std::string msg;
};

// Raw mesh as read from a deck (coordinates in metres).
struct RawMesh {
    int dim = 2;
    std::vector<double> xyz;               // [nn*3]
    std::vector<int> cptr, cverts, creg;   // cells
    std::vector<int> bptr, bverts, btag;   // boundary elements
    double Lx = 1, Ly = 1, Lz = 1;
    // independent geometries of a batched solve: cells comp_ptr[k] ..
    // comp_ptr[k+1] (no face or node shared between them); empty = one
    std::vector<int> comp_ptr;
    int nn() const { return (int)(xyz.size() / 3); }
    int nc() const { return (int)cptr.size() - 1; }
    int nbe() const { return (int)bptr.size() - 1; }
};

struct Bands {
    int nmat = 1, nb = 0, material_dim = 3;
    std::vector<double> v, tau, C, lat, hr;  // [m*nb + b]
    std::vector<int> region_material;
    std::vector<double> kappa, capb;         // per material (BTEBand.cpp:791-803)
};

struct BCs {
    std::vector<int> tag, type;
    std::vector<double> value;
    std::vector<double> trans;  // [rows][nmat * nb] transmissivity of type-5 rows (empty: none)
};

struct Angles {
    int nd = 0;
    double solid = 0;
    std::vector<double> sx, sy, sz, w;  // direction cosines, weight / SolidAngle
};

// Flattened mesh in structure-of-arrays / CSR form. Cell faces keep the
// reference's per-cell face order (BTEMesh.cpp:722-772); boundaries keep the
// reference's boundary order and (boundary, side) numbering, so a boundary
// side is s = 2*ib + icell exactly like ebound[...][ib*2+icell].
struct FlatMesh {
    int dim = 2, nc = 0, nn = 0, nmat = 1;
    double Lx = 1;
    // cells
    std::vector<int> matter;
    std::vector<double> vol, cx, cy, cz;
    std::vector<int> cf_ptr;  // [nc+1]
    // cell faces (k = cf_ptr[c] + j)
    std::vector<double> cf_area, cf_nx, cf_ny, cf_nz, cf_fx, cf_fy, cf_fz;
    std::vector<int> cf_nbr, cf_bside, cf_bound, cf_face;
    std::vector<int> cf_v;  // [ncf*3] face vertices (third = -1 in 2D)
    // global faces (Element_Faces order, BTEMesh.cpp:987-1021)
    std::vector<int> f_cell0, f_cf0, f_cell1, f_cf1, f_bound;
    // vertex-neighbour least-squares stencil (StaticBTESynthetic.cpp:453-465,
    // 967-1025); weights already include the 1/ScaleX factors
    std::vector<int> nbr_ptr, nbr_idx;
    std::vector<double> lsq_w;  // [entry*3]
    // 3D face tangential LSQ (FaceMatrix, StaticBTESynthetic.cpp:1617-1649), [f*9]
    std::vector<double> face_w;
    // boundaries (after BC matching, BTEMesh.cpp:845-866)
    std::vector<int> b_type, b_connect, b_tag;
    std::vector<double> b_T;
    std::vector<int> bs_cell, bs_cf;  // [2*nbd], -1 if absent
    std::vector<double> bs_trans;     // [2*nbd][nb] transmissivity seen from each side (type 5), else empty
    // node slots (node*nmat + matter): inverse-distance interpolation.
    // e-interpolation with boundary override (StaticBTESynthetic.cpp:1541-1616):
    // src >= 0 is a cell, src < 0 is boundary side (-1 - src)
    std::vector<int> nv_ptr, nv_src;
    std::vector<double> nv_w;
    // temperature interpolation over cells only (:2276-2305)
    std::vector<int> nt_ptr, nt_src;
    std::vector<double> nt_w;
    std::vector<double> node_x, node_y, node_z;
    // raw cell vertex lists (for output)
    std::vector<int> cptr, cverts;
    // independent geometries (batched solve): cells comp_ptr[k] .. comp_ptr[k+1]
    std::vector<int> comp_ptr;
    int ncomp() const { return (int)comp_ptr.size() - 1; }

    int ncf() const { return (int)cf_area.size(); }
    int nbd() const { return (int)b_type.size(); }
    int nbs() const { return 2 * nbd(); }
    int nf() const { return (int)f_cell0.size(); }
};

// Per-direction upwind schedule: cells in level order. With several
// independent geometries (components), each component's cells keep their
// own position range (its cell range) and their own levels, so that one
// sweep CTA can walk one component of one direction.
struct Schedule {
    int ncomp = 1;
    std::vector<int> lvl_cells;   // [nd*nc]
    std::vector<int> lvl_ptr;     // concatenated level offsets (positions within the direction)
    std::vector<int> dir_lvl_off; // [nd*ncomp+1] offsets into lvl_ptr: levels of (d, comp) are
                                  // lvl_ptr[dir_lvl_off[d*ncomp+comp] .. dir_lvl_off[d*ncomp+comp+1]-1]
    std::vector<uint8_t> lag;     // [nd*nc] bit j set: face j of the cell is lagged (empty if none)
    int max_levels = 0;
    int lagged_faces = 0;
};

// Read a deck directory (reference file formats).
struct Deck {
    RawMesh mesh;
    Bands bands;
    BCs bcs;
    int angle_method = 2, n_theta = 4, n_phi = 4;
    std::string order = "2", method = "Sequential", matrix = "LU";
    int max_iter = 10000;
    double err_temp = 1e-6, err_flux = 1e-4, tref = 300, uniform_heat = 0;
    bool transient = false;                      // CONTROL State=Transient
    double time_step = -1, total_time = -1;      // CONTROL TimeStep, TotalTime
    std::vector<double> cell_heat;
};
Error read_deck(const std::string &dir, Deck &deck);

// Level-order records of the upwind sweep of every direction, position P =
// d*nc + (index in the direction's level order). The sweep keeps the
// corrections of the last `ring` positions (a power of two, at least the
// widest level) on chip; an upwind reference further back is a far
// reference. With far slots enabled (far_cap > 0), the cell read that way
// also stores its correction into an on-chip far slot, allocated per
// direction over the interval from its own level to its last far reader's
// level; np then holds -(1 + slot) for that neighbour. Without far slots,
// np always holds the neighbour's position and far references are read
// from global memory.
struct SweepPlan {
    int ring = 0, max_width = 0, far_slots = 0;
    long long far_refs = 0;  // upwind references outside the ring (all directions)
    bool far_enabled = false;
    // (nd*nc records: built one direction per thread, each thread filling its
    // direction's ranges, so the arrays skip the zeroing of resize)
    HostArray<int> np;      // [nd*nc*4] position (>= 0) or -(1 + far slot); 0 past nin
    HostArray<double> a;    // [nd*nc*4] A_f/V (s.n_f) of the upwind faces (< 0); 0 past nin
    HostArray<double> sig;  // [nd*nc] sum of the outgoing A_f/V (s.n_f)
    HostArray<int> nin;     // [nd*nc] upwind neighbours (<= 4)
    HostArray<int> cell;    // [nd*nc] the cell at this position
    HostArray<int> far_w;   // [nd*nc] far slot this cell stores into, -1 none
};

// Cell order for locality: cells sorted by the Morton code of their centre
// (within each component, so components keep their ranges). perm[k] = the
// original index of the cell placed at k. Only the order of cells changes:
// faces, neighbours and stencils are the same sets, so results agree to
// rounding.
void locality_order(const RawMesh &raw, std::vector<int> &perm);
void reorder_cells(RawMesh &raw, const std::vector<int> &perm);
// In place, for each of the ncols arrays of nc = perm.size() rows of w
// values: row k moves to row perm[k] (internal cell order -> the caller's).
// perm must be a permutation of 0 .. nc - 1. Columns, or ranges of rows when
// there are few columns, run on the host's threads.
void scatter_rows(const std::vector<int> &perm, double *const *cols, int ncols, int w);

// Disjoint union of independent geometries for one batched solve: nodes,
// cells and boundary elements concatenated, the boundary tags of geometry k
// (and the tags its periodic types name) shifted by k * (largest tag + 1),
// comp_ptr set to the geometries' cell ranges. All share ScaleX.
Error make_union(const std::vector<RawMesh> &meshes, const std::vector<BCs> &bcs, RawMesh &out, BCs &out_bcs);

Error make_angles(int method, int ntheta, int nphi, int material_dim, Angles &out);
// an explicit direction set: unit vectors [n * 3], weights summing to the solid angle
Error explicit_angles(int n, const double *xyz, const double *weight, double solid, Angles &out);
Error build_flat_mesh(const RawMesh &raw, const BCs &bcs, const Bands &bands, FlatMesh &out);
void build_schedule(const FlatMesh &m, const Angles &a, Schedule &out, int nthreads);
// min_ring: the smallest ring (rounded up to a power of two and to the
// widest level); far_cap: most far slots allowed, 0 disables them. The
// solver uses kSweepMinRing and kSweepFarCap.
constexpr int kSweepMinRing = 512;
constexpr int kSweepFarCap = 2048;
Error build_sweep_plan(const FlatMesh &m, const Angles &a, const Schedule &s, int min_ring, int far_cap,
                       SweepPlan &out);

// Tiles of the shared-memory LSQ gradient: cells split into blocks of B
// consecutive cells (the solver's Morton order); block k's union is its own
// B cells (local index = position in the block) followed by every other
// stencil neighbour of its cells in ascending order. loc[q] is the local
// index of stencil entry q in its cell's block union.
struct GradTiles {
    int B = 0, nblk = 0, umax = 0, qmax = 0;
    std::vector<int> ptr;            // [nblk + 1] offsets into cells
    std::vector<int> cells;          // union cells of every block
    std::vector<unsigned short> loc; // [stencil entries]
};
Error build_grad_tiles(const FlatMesh &m, int B, GradTiles &out);

// Tiles of the shared-memory residual: the same blocks, each union its own
// cells then its cells' interior face neighbours outside it (ascending);
// floc[k] is the union index of face slot k's neighbour (0xFFFF on walls).
struct FaceTiles {
    int B = 0, nblk = 0, umax = 0;
    std::vector<int> ptr, cells;
    std::vector<unsigned short> floc;  // [cell-face slots]
};
Error build_face_tiles(const FlatMesh &m, int B, FaceTiles &out);

// Index checks, the stand-in for a device memory checker: every CSR offset
// and index array of the flattened mesh, the level schedule and the sweep
// records is checked against the range it indexes (offsets monotone and
// spanning their entries, every level order a permutation, every upwind
// reference an earlier position or a far slot). Enabled by building with
// -DGBTE_DEBUG or by a non-zero GBTE_DEBUG environment variable; gbte_create
// and gbte_inspect_* then run it and fail with GBTE_ERR_MESH on the first
// entry out of range. `checked` counts the entries looked at.
bool index_checks_enabled();
Error check_indices(const FlatMesh &m, int nb, const Schedule &s, int nd, const SweepPlan &sp, long long &checked);
// the same for the shared-memory tiles (either may be null)
Error check_tiles(const FlatMesh &m, const GradTiles *g, const FaceTiles *f, long long &checked);

}  // namespace gbte
