// Drives include/iblgf_b200/adapter.hpp through a minimal stand-in for the
// reference's Domain / Octant / DataField / Setup types (only the members the
// adapter uses), the way a reference setup (tests/poisson/vortexrings.hpp)
// would call PoissonSolver<Setup>::solve<source, phi>().
//
//   adapter_mock <in.bin> <out.bin>
// in.bin: int e, bd_base[3], bd_extent[3]; double dx; int n; uint64 keys[n];
//         int flags[n]; double source[n][Nb^3]  (octants in any order)
// out.bin: double target[n][Nb^3] in the same order.
#include <algorithm>
#include <array>
#include <cstdio>
#include <memory>
#include <random>
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
struct Octant
{
    Key k;
    int flags = 0;
    std::array<Block, 2> f;
    bool has_data() const { return true; }
    Key key() const { return k; }
    bool is_leaf() const { return flags & 1; }
    bool is_correction() const { return flags & 2; }
    Block& data_r(int tag, std::size_t) { return f[tag]; }
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
struct source_f
{
    static int tag() { return 0; }
    static std::size_t nFields() { return 1; }
};
struct phi_f
{
    static int tag() { return 1; }
    static std::size_t nFields() { return 1; }
};

int main(int argc, char** argv)
{
    if (argc != 3) return 2;
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
        o->f[0].v.resize(B);
        o->f[1].v.assign(B, 0.0);
        ok = std::fread(o->f[0].v.data(), 8, B, fi) == B;
        d.octs.push_back(std::move(o));
    }
    std::fclose(fi);
    if (!ok) return 2;
    // the adapter must not depend on the domain's iteration order
    std::vector<Octant*> in_order;
    for (auto& o : d.octs) in_order.push_back(o.get());
    std::mt19937 rng(5);
    std::shuffle(d.octs.begin(), d.octs.end(), rng);

    iblgf::b200::PoissonSolver<Setup> psolver(&sim);
    psolver.solve<source_f, phi_f>();

    FILE* fo = std::fopen(argv[2], "wb");
    for (Octant* o : in_order) std::fwrite(o->f[1].v.data(), 8, B, fo);
    std::fclose(fo);
    return 0;
}
