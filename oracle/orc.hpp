// ORACLE — test infrastructure only.
//
// CPU, FP64 restatement of the IBLGF-AMR lattice-Green's-function FMM path
// (reference project ComputationalFlowPhysics/IBLGF-AMR). It is the checker
// for the CUDA product in iblgf-amr_b200/: only tests/, __graft_entry__.smoke()
// and bench.py's cpu_baseline leg load it. Nothing in the product links it.
//
// Parity pins (see tests/test_oracle_*.py):
//   * LGF table: against values produced by the reference's own generator
//     include/iblgf/lgf/lgf_table_gen/lgf_integrator.py (scipy quad), committed
//     as tests/golden/lgf_table_sample.json, and Watson's constant G(0).
//   * block convolution: tests/conv_test/convFFTTest.cpp (direct sum, 1e-8) and
//     tests/conv_test/convSingleBlockTest.cpp (impulse vs LGF, 1e-8).
//   * FMM: tests/conv_test/ffmTest.cpp (impulse vs LGF, 1e-8).
//   * Poisson: tests/poisson/poisson_Test.cpp configs config_1_lv_0/1
//     (manufactured vortex-ring solution, EXP_LInf).
// The reference itself cannot be built here (MPI, Boost, FFTW, xtensor, HDF5
// absent; src/lgf/lgf_gl_lookup.cpp missing from the mount), so parity is
// "restatement pinned by the reference's KATs and its table generator".
#pragma once
#include <array>
#include <complex>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

namespace orc
{
using u64 = std::uint64_t;
using cplx = std::complex<double>;

// ---------------------------------------------------------------- LGF table
// include/iblgf/lgf/lgf_gl_lookup.hpp:33-52 (get), :74-119 (asym),
// lgf_table_gen/python_lgf.py:9-21 (N_max 100, n1>=n2>=n3 ordering).
constexpr int kLgfNmax = 100;
int lgf_table_size();
const std::vector<double>& lgf_table();      // positive integrals, generated once
double lgf_asym(int n1, int n2, int n3);      // lgf_gl_lookup.hpp:74-119
double lgf_get(int x, int y, int z);          // returns -table or asym
// e^{-6 alpha} I_n1(2a) I_n2(2a) I_n3(2a): lgf_ge.hpp:158-167
void bessel_ie_all(double x, int nmax, double* out);  // e^{-x} I_n(x), n=0..nmax

// ---------------------------------------------------------------- FFT
// Complex mixed-radix FFT of any length (own code; replaces FFTW).
struct Fft1d
{
    int n = 0;
    std::vector<int> factors;
    std::vector<cplx> tw_fwd, tw_bwd;
    explicit Fft1d(int n_ = 1);
    void run(cplx* x, int stride, bool forward, cplx* work) const;
};

// ---------------------------------------------------------------- Keys
// include/iblgf/domain/octree/key.hpp and bitmasks.hpp (Dim 3: max_level 19,
// 5 level bits, 2 flag bits).
constexpr int kMaxLevel = 19;
u64 key_make(int x, int y, int z, int level);
int key_level(u64 k);
std::array<int, 3> key_coord(u64 k);
u64 key_parent(u64 k);
u64 key_child(u64 k, int i);
int key_child_number(u64 k, int level);
bool key_is_end(u64 k);
u64 key_neighbor(u64 k, int dx, int dy, int dz);
std::vector<u64> key_neighbor_keys(u64 k);    // 27, z slowest, self at 13
std::vector<u64> key_infl_keys(u64 k);        // key.hpp:226-250

// ---------------------------------------------------------------- Tree
struct Octant
{
    u64 key = 0;
    int level = 0;
    Octant* parent = nullptr;
    std::array<std::unique_ptr<Octant>, 8> child{};
    bool has_data = false;
    int bbase[3] = {0, 0, 0};  // block base (level cell units, no buffer)
    int data_level = 0;        // refinement level given at allocation
    bool leaf = false, correction = false, physical = false, aim_deletion = false;
    bool old_correction = false;  // base-level correction flag before the last adaptation
    bool ib = false, ext_ib = false;  // immersed-boundary blocks (server.hpp:544-576)
    std::array<Octant*, 27> neighbor{};
    std::array<Octant*, 189> influence{};
    int n_infl = 0;
    std::array<std::array<bool, 2>, 50> mask{};
    int idx = -1;              // position in the canonical octant order
};

using RefinePred = int (*)(void* user, const int* base, const int* extent,
                           int refinement_level, int diff_level);

struct Domain
{
    int e = 0;                 // block_extent
    int Nb = 0;                // e + 2
    int bd_base[3], bd_extent[3];
    int base_shift[3];         // bounding_box.base() / e
    int base_level = 0, depth = 0;
    double dx_base = 1.0;
    std::unique_ptr<Octant> root;
    std::vector<Octant*> octs; // canonical order: (level, key), has_data only
    std::vector<std::map<u64, Octant*>> level_maps;
    int key_bd_extent[3];

    Octant* find(u64 k) const;
    Octant* insert(u64 k);
    Octant* refine_child(Octant* o, int i);
    void alloc(Octant* o, int data_level);
    void construct_level_maps();
    void construct_leaf_flags_from_search();
    void construct_lists();
    void finalize();           // canonical order + idx
    int refinement_level(const Octant* o) const { return o->level - base_level; }
    std::vector<u64> unfound_neighbors(Octant* o, bool correction_as_neighbors);
    bool try_2to1(u64 k, std::map<u64, bool>& checklist);
    void refine(Octant* o, bool ratio_2to1);
    void init_refine(int nRef, int level_up_max, RefinePred pred, void* user);
    void mark_correction();
    // adaptation (server side of Domain::adapt): attempts (key, level change);
    // returns the parents of new leaves above the base level, (level, key)
    // order. Octants keep their idx of the previous canonical order until
    // finalize(); new ones have idx -1.
    std::vector<Octant*> adapt(const std::vector<std::pair<u64, int>>& attempts, bool& base_mesh_update);
    bool leaf_search(const Octant* o, bool require_data) const;
    void delete_oct(Octant* o);
};

std::unique_ptr<Domain> domain_create(const int* bd_base, const int* bd_extent,
    int block_extent, double dx_base, int n_blocks, const int* block_base,
    const int* block_ext);

// ---------------------------------------------------------------- Fields
// A field: one Nb^3 array (x fastest, buffers included) per octant in
// canonical order.
using Field = std::vector<double>;

// ---------------------------------------------------------------- FMM
enum MaskType { STREAM = 0, AMR2AMR = 1, IB2xIB = 2, xIB2IB = 3, IB2AMR = 4 };
int fmm_mask_idx_gen(int type, int refinement_level = 0, int non_leaf_as_source = 0);
void fmm_lgf_mask_build(Domain& d, bool subtract_non_leaf);
void fmm_stream_mask_build(Domain& d);
// IB2xIB, xIB2IB and IB2AMR masks from the octants' ib / ext_ib flags
// (fmm.hpp:70-190); IB2AMR also marks the parents of IB blocks as IB
void fmm_ib_mask_build(Domain& d);

struct Solver
{
    Domain* d;
    int Nb, P;
    int intrp_order = 5;
    Fft1d fft;
    // fmm_nli.hpp Nli matrices (Nb x Nb, two halves)
    std::vector<double> nli_sub[2];
    // cell_center_nli matrices: intrp [4] (rel pos 0/1 x child 0/1), coarsify [4]
    std::vector<double> cc_intrp[4], cc_antrp[4];
    // LGF spectra cache: (level_diff, base offset) -> half spectrum
    std::map<std::array<int, 4>, std::vector<cplx>> spectra;
    // LGF_GE spectra cache: (alpha, base offset) -> half spectrum
    std::map<std::tuple<double, int, int, int>, std::vector<cplx>> spectra_ge;
    double ge_alpha = -1.0;
    std::vector<double> ge_f;  // e^{-2 alpha} I_n(2 alpha)
    Field fmm_s, fmm_t;
    explicit Solver(Domain* d, int intrp_order = 5);

    const std::vector<cplx>& lgf_spectrum(int level_diff, int bx, int by, int bz);
    void fwd_half(const double* block, std::vector<cplx>& out);  // Nb^3 -> half
    void fmm_apply(const Field& src, Field& tgt, int level, bool non_leaf_as_source,
                   double add_with_scale, int fmm_type);
    void apply_lgf(const Field& src, Field& tgt, int fmm_type, bool use_correction,
                   bool subtract_non_leaf);
    // integrating factor (LGF_GE, neighbour only): lgf_ge.hpp, fmm.hpp:754-770
    double lgf_ge_get(int x, int y, int z, double alpha);
    const std::vector<cplx>& lgf_ge_spectrum(double alpha, int bx, int by, int bz);
    void fmm_apply_ge(const Field& src, Field& tgt, int level, bool non_leaf_as_source,
                      double add_with_scale, double alpha, int fmm_type = AMR2AMR);
    void apply_if(const Field& src, Field& tgt, double alpha_base, bool subtract_non_leaf,
                  const int* rp = nullptr, int fmm_type = AMR2AMR);
    // cell_center_nli transfers; rp = relative position per axis (0: node
    // coincides with the child's, 1: half a cell off), cell {1,1,1} when null
    void cc_intrp_level(Field& from, Field& to, int level, bool correction_only, const int* rp = nullptr);
    // nli_intrp_node of one child: f[child c of p] = interpolation of f[p]
    void cc_intrp_child(Field& f, Octant* p, int c, const int* rp);
    void coarsify_all(Field& f, const int* rp = nullptr);
    void copy_level_interior(const Field& src, Field& dst, int l) const;
};

// ---------------------------------------------------------------- IF-HERK
// Mesh objects of a field's components (domain::MeshObject) and their
// relative positions for the cell-centred transfers.
enum MeshType { MESH_CELL = 0, MESH_FACE = 1, MESH_EDGE = 2 };
void mesh_relpos(int mesh, int comp, int rp[3]);

struct VField
{
    int mesh = MESH_CELL;
    std::vector<Field> c;  // 1 (cell) or 3 (face, edge) component fields
};

// Ifherk::time_step without immersed boundary (ifherk.hpp:1078-1200)
struct Ifherk
{
    Domain* d;
    Solver* s;
    double dt, Re;
    double T = 0.0, T_last_vel_refresh = 0.0;
    bool force_refresh = false;  // base_mesh_update of the last adaptation
    double a[6] = {1.0 / 3, -1.0, 2.0, 0.0, 0.75, 0.25};
    // immersed boundary (optional): force of the previous step per stage
    // (IB::force_prev, the CG warm start), CG settings, frame velocity
    struct IbSystem* ib = nullptr;
    std::vector<std::array<double, 3>> force_prev[4];
    double cg_threshold = 1e-3;
    int cg_max_iter = 40, stage_idx = 0;
    double frame_vel[3] = {0.0, 0.0, 0.0};
    double c[4] = {0.0, 1.0 / 3, 1.0, 1.0};
    double alpha[3] = {0.0, 0.0, 0.0};
    VField u, p, q_i, g_i, d_i, r_i, u_i, w_1, w_2, cell_aux, face_aux, edge_aux, stream_f;
    bool write_prev_force = true;

    Ifherk(Domain* d, Solver* s, double dt, double Re);
    double coeff_a(int i, int j) const;
    void time_step();

    void clean(VField& f, bool non_leaf_only);
    void up(VField& f);
    void down_to_correction(VField& f);
    void up_and_down(VField& f);
    void smooth2zero(VField& f, Octant* o, int ngb);
    void clean_leaf_correction_boundary(VField& f, int l, bool leaf_only_boundary);
    void op_level(int op, const std::vector<const Field*>& in, const std::vector<Field*>& out, int l,
                  double scale);
    void exchange(VField& f, int l);
    void copy(const VField& from, VField& to, double scale);
    void add(const VField& from, VField& to, double scale);
    void nonlinear(VField& src, VField& tgt, double scale);
    void divergence(VField& src, VField& tgt);
    void gradient(VField& src, VField& tgt);
    void apply_if(const VField& src, VField& tgt, double alpha_base);
    void lin_sys(double alpha_k);
    void pad_velocity();
    void adapt_corr_time_step();
};

// ---------------------------------------------------------------- IB
// Immersed boundary on the finest level (ib.hpp, client.hpp:1262-1320,
// server.hpp:544-576) and its force solve (linsys.hpp:113-531).
double yang3(double x);  // ib.hpp:690-705
struct IbSystem
{
    Domain* d;
    Solver* s;
    int ib_level = 0;            // refinement level of the IB (the finest)
    double Re = 1.0;
    double ddf_radius = 4.5, safety_dis = 0.0;
    std::vector<std::array<double, 3>> X;                       // point coordinates
    std::vector<std::vector<Octant*>> infl;                     // leaf blocks per point
    std::vector<std::vector<std::vector<std::array<int, 3>>>> pts;  // interior nodes (local index) per block
    VField face_aux, face_aux2, cell_aux2;
    int iterations = 0;

    IbSystem(Domain* d, Solver* s, const std::vector<std::array<double, 3>>& X, double Re);
    bool overlap(int i, const Octant* o, int radius_level) const;   // ib_block_overlap
    void projection(const VField& u, std::vector<std::array<double, 3>>& f) const;
    void smearing(const std::vector<std::array<double, 3>>& f, VField& u, bool cleaning = true) const;
    void clean_ib_region_boundary(VField& f, int l, int width) const;
    void clean_face_boundary(VField& f, int l, bool leaf_only_boundary, int width) const;
    void apply_schur(VField& src, VField& tgt);
    void et_h_s_e(const std::vector<std::array<double, 3>>& fin, std::vector<std::array<double, 3>>& fout,
                  double alpha);
    // ib_solve (linsys.hpp:113-129) + CG_solve (:170-230); f: initial guess in, force out
    void solve(const VField& u, double alpha, std::vector<std::array<double, 3>>& f, double threshold,
               int max_iter);
    // LinSysSolver::pressure_correction (linsys.hpp:131-145): p -= L^-1 div E f
    void pressure_correction(const std::vector<std::array<double, 3>>& f, VField& p);
};
std::vector<std::array<double, 3>> sphere_points(double dx_base, int ib_level, double ibph);

void nli_matrix(int Nb, int pts_cap, double* mat /* Nb x 2Nb, (p,c) at p*2Nb+c */);
void buffer_exchange(Domain& d, Field& f, int level);
void apply_op(Domain& d, int op, const std::vector<const Field*>& in, const std::vector<Field*>& out,
              int level, double scale, bool skip_correction = false);
void cc_matrix(int Nb, int pts_cap, int relpos, double* mat);

}  // namespace orc
