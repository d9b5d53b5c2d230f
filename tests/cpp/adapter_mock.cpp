// Drives include/iblgf_b200/adapter.hpp through a minimal stand-in for the
// reference's Domain / Octant / DataField / Setup types (only the members the
// adapter uses), the way reference setups (tests/poisson/vortexrings.hpp,
// ifherk.hpp) call PoissonSolver, Fmm, the LGF kernel objects and Operator.
//
//   adapter_mock <in.bin> <out.bin> [mode alpha level]
// in.bin: int e, bd_base[3], bd_extent[3]; double dx; int n; uint64 keys[n];
//         int flags[n]; double source[n][Nb^3]  (octants in any order)
// modes (out.bin in the input's octant order):
//   poisson  PoissonSolver::solve<source, phi>()                 -> phi
//   if       PoissonSolver::apply_lgf_IF<source, phi>(alpha)      -> phi
//   fmm_gl   Fmm::apply<source, phi>(LGF_GL, level, nlas 1, 0.5)  -> phi
//   fmm_ge   Fmm::apply<source, phi>(LGF_GE alpha, level, 0, 1)   -> phi
//   ops      Operator::levelGradient<source, face>(l) for every level, then
//            the per-block Operator::curl<face, edge>(it->data(), dx) on
//            every octant                                         -> face[3], edge[3]
//   kernels  LGF_GL::get and LGF_GE(alpha)::get at 64 fixed offsets -> 2 x 64 values,
//            then Helmholtz(c = alpha)::get at 16 fixed 2-D offsets, the same
//            after change_level(1), and a default-constructed Helmholtz's
//            get(3, 1)                                          -> 2 x 16 + 1 values
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "iblgf_b200/adapter.hpp"

struct Key
{
    uint64_t v;
    uint64_t id() const { return v; }
};
struct Block
{
    std::vector<double> v;
    double* data() { return v.data(); }
    std::size_t size() const { return v.size(); }
};
struct DataBlock  // the octant's data block (it->data())
{
    int dummy = 0;
};
constexpr int kTags = 4;
struct Octant
{
    Key k;
    int flags = 0;
    int level = 0;
    DataBlock db;
    std::array<std::vector<Block>, kTags> f;  // [tag][component]
    bool has_data() const { return true; }
    Key key() const { return k; }
    bool is_leaf() const { return flags & 1; }
    bool is_correction() const { return flags & 2; }
    DataBlock& data() { return db; }
    Block& data_r(int tag, std::size_t comp) { return f[tag][comp]; }
};
struct Box
{
    std::array<int, 3> b, e;
    const std::array<int, 3>& base() const { return b; }
    const std::array<int, 3>& extent() const { return e; }
};
struct Domain
{
    using octant_t = Octant;
    struct It
    {
        std::vector<std::unique_ptr<Octant>>::iterator i;
        Octant* operator->() { return i->get(); }
        Octant* ptr() { return i->get(); }
        It& operator++()
        {
            ++i;
            return *this;
        }
        bool operator!=(const It& o) const { return i != o.i; }
    };
    std::vector<std::unique_ptr<Octant>> octs;
    std::array<int, 3> ext;
    Box box;
    double dx;
    It begin() { return {octs.begin()}; }
    It end() { return {octs.end()}; }
    const std::array<int, 3>& block_extent() const { return ext; }
    const Box& bounding_box() const { return box; }
    double dx_base() const { return dx; }
};
struct Simulation
{
    using domain_type = Domain;
    std::unique_ptr<Domain> domain_;
};
struct Setup
{
    using simulation_t = Simulation;
    using domain_t = Domain;
};
template<int T, std::size_t N>
struct field
{
    static int tag() { return T; }
    static std::size_t nFields() { return N; }
};
using source_f = field<0, 1>;
using phi_f = field<1, 1>;
using face_f = field<2, 3>;
using edge_f = field<3, 3>;

int main(int argc, char** argv)
{
    if (argc != 3 && argc != 6) return 2;
    const std::string mode = argc == 6 ? argv[3] : "poisson";
    const double alpha = argc == 6 ? std::atof(argv[4]) : 0.0;
    const int level = argc == 6 ? std::atoi(argv[5]) : 0;
    FILE* fi = std::fopen(argv[1], "rb");
    if (!fi) return 2;
    int e, bb[3], be[3], n;
    double dx;
    bool ok = std::fread(&e, 4, 1, fi) == 1 && std::fread(bb, 4, 3, fi) == 3 && std::fread(be, 4, 3, fi) == 3 &&
              std::fread(&dx, 8, 1, fi) == 1 && std::fread(&n, 4, 1, fi) == 1;
    if (!ok) return 2;
    const std::size_t B = (std::size_t)(e + 2) * (e + 2) * (e + 2);
    std::vector<uint64_t> keys(n);
    std::vector<int> flags(n);
    ok = std::fread(keys.data(), 8, n, fi) == (size_t)n && std::fread(flags.data(), 4, n, fi) == (size_t)n;
    Simulation sim;
    sim.domain_ = std::make_unique<Domain>();
    Domain& d = *sim.domain_;
    d.ext = {e, e, e};
    d.box = {{bb[0], bb[1], bb[2]}, {be[0], be[1], be[2]}};
    d.dx = dx;
    for (int i = 0; i < n && ok; ++i)
    {
        auto o = std::make_unique<Octant>();
        o->k = {keys[i]};
        o->flags = flags[i];
        o->level = (int)((keys[i] >> 2) & 31);
        const std::size_t comps[kTags] = {1, 1, 3, 3};
        for (int t = 0; t < kTags; ++t) o->f[t].assign(comps[t], Block{std::vector<double>(B, 0.0)});
        ok = std::fread(o->f[0][0].v.data(), 8, B, fi) == B;
        d.octs.push_back(std::move(o));
    }
    std::fclose(fi);
    if (!ok) return 2;
    // the adapter must not depend on the domain's iteration order
    std::vector<Octant*> in_order;
    for (auto& o : d.octs) in_order.push_back(o.get());
    std::mt19937 rng(5);
    std::shuffle(d.octs.begin(), d.octs.end(), rng);

    std::vector<double> out;
    auto put = [&](int tag, std::size_t ncomp) {
        for (std::size_t k = 0; k < ncomp; ++k)
            for (Octant* o : in_order) out.insert(out.end(), o->f[tag][k].v.begin(), o->f[tag][k].v.end());
    };
    try
    {
        if (mode == "poisson")
        {
            iblgf::b200::PoissonSolver<Setup> psolver(&sim);
            psolver.solve<source_f, phi_f>();
            put(1, 1);
        }
        else if (mode == "if")
        {
            iblgf::b200::PoissonSolver<Setup> psolver(&sim);
            psolver.apply_lgf_IF<source_f, phi_f>(alpha);
            put(1, 1);
        }
        else if (mode == "fmm_gl" || mode == "fmm_ge")
        {
            iblgf::b200::Fmm<Setup> fmm(&d);
            if (mode == "fmm_gl")
            {
                iblgf::b200::LGF_GL k;
                fmm.apply<source_f, phi_f>(&d, &k, level, true, 0.5);
            }
            else
            {
                iblgf::b200::LGF_GE k;
                k.alpha_base_level() = alpha;
                fmm.apply<source_f, phi_f>(&d, &k, level, false, 1.0);
            }
            put(1, 1);
        }
        else if (mode == "ops")
        {
            using Op = iblgf::b200::Operator<Domain>;
            Op::bound_domain() = &d;
            int bl = 0, depth = 0, no = 0;
            iblgf_ctx* c = iblgf::b200::device_domain(&d).ctx();
            iblgf::b200::check(c, iblgf_domain_info(c, &bl, &depth, &no));
            for (int l = bl; l < depth; ++l) Op::levelGradient<source_f, face_f>(&d, l);
            for (auto& o : d.octs)
                Op::curl<face_f, edge_f>(o->data(), dx / std::pow(2.0, o->level - bl));
            put(2, 3);
            put(3, 3);
        }
        else if (mode == "kernels")
        {
            iblgf::b200::LGF_GL gl;
            iblgf::b200::LGF_GE ge;
            ge.alpha_base_level() = alpha;
            ge.change_level(0);
            std::vector<std::array<int, 3>> pts;
            for (int i = 0; i < 64; ++i) pts.push_back({i % 7 - 3, (i / 7) % 5 - 2, i / 35 * 37 - 5});
            for (auto& p : pts) out.push_back(gl.get(p));
            for (auto& p : pts) out.push_back(ge.get(p));
            iblgf::b200::Helmholtz h(alpha);
            std::vector<std::array<int, 2>> p2;
            for (int i = 0; i < 16; ++i) p2.push_back({i % 5 - 2, i / 5 * 3 - 4});
            for (auto& p : p2) out.push_back(h.get(p));
            h.change_level(1);
            for (auto& p : p2) out.push_back(h.get(p[0], p[1]));
            iblgf::b200::Helmholtz h0;
            out.push_back(h0.get(3, 1));
        }
        else
            return 2;
    }
    catch (const std::exception& ex)
    {
        std::fprintf(stderr, "adapter_mock: %s\n", ex.what());
        return 1;
    }
    FILE* fo = std::fopen(argv[2], "wb");
    std::fwrite(out.data(), 8, out.size(), fo);
    std::fclose(fo);
    return 0;
}
