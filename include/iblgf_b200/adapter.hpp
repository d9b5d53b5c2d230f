// C++ adapter: the reference's solver templates on top of the iblgf_b200
// C ABI, so a reference setup switches its typedefs and keeps its calls.
//
//   reference                                          this adapter
//   ------------------------------------------------   --------------------------------------
//   fmm::Fmm<Setup>::apply<Src,Tgt>(domain, kernel,    iblgf::b200::Fmm<Setup>::apply<Src,Tgt>(...)
//     level, non_leaf_as_source, scale, fmm_type)        (include/iblgf/fmm/fmm.hpp:729-870), kernel
//                                                        LGF_GL or LGF_GE (dispatched on its type)
//   solver::PoissonSolver<Setup>::apply_lgf<S,T>()     iblgf::b200::PoissonSolver<Setup>::apply_lgf<S,T>()
//     / solve<S,T>() / apply_lgf_IF<S,T>(alpha, type)    (solver/poisson/poisson.hpp:131, 428-494, 1362)
//     / use_correction() / subtract_non_leaf()
//   lgf::LGF_GL<3>, lgf::LGF_GE<3>: get(coord),        iblgf::b200::LGF_GL, LGF_GE (lgf_gl.hpp:73-105,
//     get_key(block, level_diff), change_level,          lgf_ge.hpp:33-190, lgf.hpp:204-209)
//     neighbor_only(), alpha_base_level()
//   domain::Operator::laplace / gradient / divergence  iblgf::b200::Operator (operators.hpp:1386-1513,
//     / curl / curl_transpose / nonlinear (per block),    2416-2531; level wrappers :521-650)
//     levelDivergence / levelGradient / domain*
//
// Requirements on the domain (all members the reference Domain already has):
//   domain->begin()/end()  depth-first octant iteration; it->has_data(),
//   it->key().id(), it->is_leaf(), it->is_correction(), it->data() (the
//   octant's data block, the argument of the per-block operators) and
//   it->data_r(tag, i) giving a DataField whose .data() / .size() is the
//   Nb^3 block (x fastest); domain->block_extent()[0],
//   domain->bounding_box().base()/.extent(), domain->dx_base(). Field types
//   provide tag() and nFields() as the reference's REGISTER_FIELDS types do.
//
// The octree is imported once per domain (iblgf_domain_import) on first use
// and shared by every adapter object of that domain; call
// device_domain(domain).reset() after the reference adapts its mesh. Fields
// are staged through host memory in the canonical octant order of the
// library; the per-block operators move only the block they act on.
#pragma once
#include <cmath>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "../iblgf_b200.h"

namespace iblgf
{
namespace b200
{
inline void check(iblgf_ctx* c, int rc)
{
    if (rc != IBLGF_OK) throw std::runtime_error(std::string("iblgf_b200: ") + iblgf_last_error(c));
}

// Device state of one domain on one GPU: the imported octree, the octant
// order, scratch fields and the octant of every data block.
template<class Domain>
class DeviceDomain
{
  public:
    using octant_t = typename Domain::octant_t;

    explicit DeviceDomain(Domain* d, int precision = IBLGF_FP64, int device = 0)
    : domain_(d)
    , precision_(precision)
    , device_(device)
    {
    }
    ~DeviceDomain() { reset(); }
    DeviceDomain(const DeviceDomain&) = delete;
    DeviceDomain& operator=(const DeviceDomain&) = delete;

    void reset()
    {
        if (ctx_) iblgf_destroy(ctx_);
        ctx_ = nullptr;
        order_.clear();
        index_of_.clear();
        scratch_.clear();
    }

    iblgf_ctx* ctx()
    {
        if (!ctx_) init();
        return ctx_;
    }
    int base_level()
    {
        ctx();
        return base_level_;
    }

    // host -> device for a reference field component into scratch field `which`
    template<class Field>
    int upload(std::size_t comp, int which)
    {
        ctx();
        const std::size_t B = block_elems();
        staging_.assign(order_.size() * B, 0.0);
        for (std::size_t i = 0; i < order_.size(); ++i)
        {
            auto& f = order_[i]->data_r(Field::tag(), comp);
            if (f.size() != B) throw std::runtime_error("iblgf_b200: block size mismatch");
            std::copy(f.data(), f.data() + B, staging_.begin() + i * B);
        }
        int id = scratch_field(which);
        check(ctx_, iblgf_field_upload(ctx_, id, staging_.data(), staging_.size()));
        return id;
    }

    template<class Field>
    void download(int id, std::size_t comp)
    {
        const std::size_t B = block_elems();
        staging_.assign(order_.size() * B, 0.0);
        check(ctx_, iblgf_field_download(ctx_, id, staging_.data(), staging_.size()));
        for (std::size_t i = 0; i < order_.size(); ++i)
        {
            auto& f = order_[i]->data_r(Field::tag(), comp);
            std::copy(staging_.begin() + i * B, staging_.begin() + (i + 1) * B, f.data());
        }
    }

    // one octant's block of a field component, host <-> scratch field `which`
    template<class Field>
    int upload_octant(int idx, std::size_t comp, int which)
    {
        auto& f = order_.at(idx)->data_r(Field::tag(), comp);
        if (f.size() != block_elems()) throw std::runtime_error("iblgf_b200: block size mismatch");
        const int id = scratch_field(which);
        check(ctx_, iblgf_field_upload_octants(ctx_, id, &idx, 1, f.data()));
        return id;
    }
    template<class Field>
    void download_octant(int id, int idx, std::size_t comp)
    {
        auto& f = order_.at(idx)->data_r(Field::tag(), comp);
        check(ctx_, iblgf_field_download_octants(ctx_, id, &idx, 1, f.data()));
    }

    // canonical index of the octant whose data block this is (-1 if none)
    int octant_of_block(const void* block)
    {
        ctx();
        auto it = index_of_.find(block);
        return it == index_of_.end() ? -1 : it->second;
    }

    int scratch_field(int which)
    {
        ctx();
        while ((int)scratch_.size() <= which)
        {
            int id = -1;
            check(ctx_, iblgf_field_create(ctx_, &id));
            scratch_.push_back(id);
        }
        return scratch_[which];
    }

    std::size_t block_elems() const
    {
        const std::size_t nb = (std::size_t)domain_->block_extent()[0] + 2;
        return nb * nb * nb;
    }

    bool subtract_non_leaf_ = false;

  private:
    void init()
    {
        iblgf_config cfg{};
        cfg.block_extent = domain_->block_extent()[0];
        const auto bb = domain_->bounding_box();
        for (int d = 0; d < 3; ++d)
        {
            cfg.bd_base[d] = bb.base()[d];
            cfg.bd_extent[d] = bb.extent()[d];
        }
        cfg.dx_base = domain_->dx_base();
        cfg.precision = precision_;
        cfg.device = device_;
        cfg.intrp_order = 5;
        if (iblgf_create(&cfg, &ctx_) != IBLGF_OK)
            throw std::runtime_error(std::string("iblgf_b200: ") + iblgf_last_error(nullptr));
        std::vector<uint64_t> keys;
        std::vector<int> flags;
        std::unordered_map<uint64_t, octant_t*> by_key;
        for (auto it = domain_->begin(); it != domain_->end(); ++it)
        {
            if (!it->has_data()) continue;
            const uint64_t k = it->key().id();
            keys.push_back(k);
            flags.push_back((it->is_leaf() ? 1 : 0) | (it->is_correction() ? 2 : 0));
            by_key[k] = it.ptr();
        }
        check(ctx_, iblgf_domain_import(ctx_, (int)keys.size(), keys.data(), flags.data()));
        check(ctx_, iblgf_domain_finalize(ctx_, subtract_non_leaf_ ? 1 : 0));
        int depth = 0, n = 0;
        check(ctx_, iblgf_domain_info(ctx_, &base_level_, &depth, &n));
        std::vector<uint64_t> canon(n);
        check(ctx_, iblgf_domain_octants(ctx_, canon.data(), nullptr, nullptr, nullptr));
        order_.resize(n);
        for (int i = 0; i < n; ++i)
        {
            order_[i] = by_key.at(canon[i]);
            index_of_[static_cast<const void*>(&order_[i]->data())] = i;
        }
        scratch_.clear();
    }

    Domain* domain_;
    int precision_, device_;
    int base_level_ = 0;
    iblgf_ctx* ctx_ = nullptr;
    std::vector<octant_t*> order_;
    std::unordered_map<const void*, int> index_of_;
    std::vector<int> scratch_;
    std::vector<double> staging_;
};

// The device domain of a domain: one per domain object for the process,
// created on first use (FP64 on device 0 unless an adapter object created
// it first with other settings) and shared by PoissonSolver, Fmm and
// Operator calls on that domain.
template<class Domain>
DeviceDomain<Domain>& device_domain(Domain* d, int precision = IBLGF_FP64, int device = 0)
{
    static std::map<const Domain*, std::unique_ptr<DeviceDomain<Domain>>> registry;
    auto& slot = registry[d];
    if (!slot) slot = std::make_unique<DeviceDomain<Domain>>(d, precision, device);
    return *slot;
}

// ----------------------------------------------------------------- kernels
namespace detail
{
// context that evaluates kernel values for kernel objects outside a domain
inline iblgf_ctx* kernel_ctx()
{
    static std::unique_ptr<iblgf_ctx, int (*)(iblgf_ctx*)> c(nullptr, iblgf_destroy);
    if (!c)
    {
        iblgf_config cfg{};
        cfg.block_extent = 16;
        cfg.bd_extent[0] = cfg.bd_extent[1] = cfg.bd_extent[2] = 16;
        cfg.dx_base = 1.0;
        cfg.precision = IBLGF_FP64;
        cfg.intrp_order = 5;
        iblgf_ctx* x = nullptr;
        if (iblgf_create(&cfg, &x) != IBLGF_OK)
            throw std::runtime_error(std::string("iblgf_b200: ") + iblgf_last_error(nullptr));
        c.reset(x);
    }
    return c.get();
}
template<class K, class = void>
struct has_alpha_base : std::false_type
{
};
template<class K>
struct has_alpha_base<K, std::void_t<decltype(std::declval<K&>().alpha_base_level())>> : std::true_type
{
};
template<class K, class = void>
struct has_laplace_flag : std::false_type
{
};
template<class K>
struct has_laplace_flag<K, std::void_t<decltype(std::declval<K&>().LaplaceLGF())>> : std::true_type
{
};
}  // namespace detail

// LGF_GL<3> (lgf_gl.hpp:73-105): the 7-point-Laplacian LGF; get() evaluates
// on the device (table lookup or asymptotic expansion, lgf_gl_lookup.hpp)
class LGF_GL
{
  public:
    bool neighbor_only() const noexcept { return false; }
    bool LaplaceLGF() const noexcept { return true; }
    void change_level(int) noexcept {}
    template<class Coord>
    double get(const Coord& c) const
    {
        const int xyz[3] = {(int)c[0], (int)c[1], (int)c[2]};
        double v = 0.0;
        check(detail::kernel_ctx(), iblgf_lgf_get(detail::kernel_ctx(), xyz, 1, &v));
        return v;
    }
    // spectrum cache key of a block (lgf_gl.hpp:73-79): its base
    template<class BlockDescriptor>
    std::tuple<int, int, int> get_key(const BlockDescriptor& b, int /*level_diff*/) const
    {
        const auto base = b.base();
        return std::tuple<int, int, int>(base[0], base[1], base[2]);
    }
};

// LGF_GE<3> (lgf_ge.hpp:33-190): the integrating-factor kernel
// E(n; alpha) = prod_i e^{-2 alpha} I_{n_i}(2 alpha), neighbour-only;
// change_level(ld) sets alpha = alpha_base_level * 4^ld (lgf_ge.hpp:81-84)
class LGF_GE
{
  public:
    bool neighbor_only() const noexcept { return true; }
    double& alpha_base_level() noexcept { return alpha_base_; }
    double alpha() const noexcept { return alpha_; }
    void change_level(int level_diff) noexcept { alpha_ = alpha_base_ * std::pow(4.0, level_diff); }
    void flip_alpha() noexcept { alpha_ = -alpha_; }
    template<class Coord>
    double get(const Coord& c) const
    {
        const int xyz[3] = {(int)c[0], (int)c[1], (int)c[2]};
        double v = 0.0;
        check(detail::kernel_ctx(), iblgf_lgf_ge_get(detail::kernel_ctx(), alpha_, xyz, 1, &v));
        return v;
    }
    template<class BlockDescriptor>
    std::tuple<double, int, int, int> get_key(const BlockDescriptor& b, int /*level_diff*/) const
    {
        const auto base = b.base();
        return std::tuple<double, int, int, int>(alpha_, base[0], base[1], base[2]);
    }

  private:
    double alpha_base_ = 0.0, alpha_ = 0.0;
};

// lgf::Helmholtz<2> (lgf/helmholtz.hpp:37-193): the 2-D screened kernel of
// one z mode of the Fourier-in-z solvers. c is the coarse level's value;
// change_level(ld) sets c_level = c / 2^ld and origin = origin_val(c_level)
// (:127-158); get() returns the trapezoidal integral of helmholtz_lookup.hpp
// minus the origin the object holds (:161-176), evaluated on the device. As in
// the reference, the default constructor holds c = 0.1 with origin 0 until a
// change_c / change_level sets it. c must be > 0 (mode 0 uses the Laplace
// kernel, whose origin series diverges).
class Helmholtz
{
  public:
    Helmholtz() : c_(0.1), c_level_(0.1), origin_(0.0) {}
    explicit Helmholtz(double C) : c_(C), c_level_(C) { origin_ = origin_val(C); }
    bool neighbor_only() const noexcept { return false; }
    bool LaplaceLGF() const noexcept { return false; }
    bool HelmholtzLGF() const noexcept { return true; }
    double return_c() const noexcept { return c_level_; }
    double origin() const noexcept { return origin_; }
    void change_c(double C)
    {
        c_ = c_level_ = C;
        origin_ = origin_val(C);
    }
    void change_level(int level_diff)
    {
        c_level_ = c_ * std::pow(0.5, level_diff);
        origin_ = origin_val(c_level_);
    }
    template<class Coord>
    double get(const Coord& c) const
    {
        return get((int)c[0], (int)c[1]);
    }
    double get(int N, int M) const
    {
        const int nm[2] = {N, M};
        double v = 0.0;  // the device value is the integral minus origin_val(c_level)
        check(detail::kernel_ctx(), iblgf_helm2d_get(detail::kernel_ctx(), c_level_, 1, nm, &v));
        return v + origin_val(c_level_) - origin_;
    }
    template<class BlockDescriptor>
    std::tuple<bool, double, int, int> get_key(const BlockDescriptor& b, int /*level_diff*/) const
    {
        const auto base = b.base();
        return std::tuple<bool, double, int, int>(true, c_level_, base[0], base[1]);
    }

  private:
    static double origin_val(double C)
    {
        double o = 0.0;
        if (iblgf_helm2d_origin(C, &o) != IBLGF_OK) throw std::runtime_error("iblgf_b200: Helmholtz needs c > 0");
        return o;
    }
    double c_, c_level_, origin_;
};

// ----------------------------------------------------------------- solvers
// PoissonSolver<Setup> (solver/poisson/poisson.hpp:46): apply_lgf / solve /
// apply_lgf_IF for every component of the source field.
template<class Setup>
class PoissonSolver
{
  public:
    using simulation_type = typename Setup::simulation_t;
    using domain_type = typename simulation_type::domain_type;

    explicit PoissonSolver(simulation_type* sim, int precision = IBLGF_FP64, int device = 0)
    : dev_(b200::device_domain(sim->domain_.get(), precision, device))
    {
    }

    template<class Source, class Target>
    void apply_lgf(int fmm_type = IBLGF_AMR2AMR)
    {
        iblgf_ctx* c = dev_.ctx();
        check(c, iblgf_poisson_options(c, use_correction_ ? 1 : 0, subtract_non_leaf_ ? 1 : 0));
        for (std::size_t comp = 0; comp < Source::nFields(); ++comp)
        {
            const int src = dev_.template upload<Source>(comp, 0);
            const int tgt = dev_.template upload<Target>(comp, 1);
            check(c, iblgf_poisson_apply_lgf(c, src, tgt, fmm_type));
            dev_.template download<Target>(tgt, comp);
        }
    }

    template<class Source, class Target>
    void solve()
    {
        apply_lgf<Source, Target>();
    }

    // apply_lgf_IF (poisson.hpp:428-494): e^{alpha L} with the LGF_GE kernel,
    // alpha = alpha_base * 4^(level - base level)
    template<class Source, class Target>
    void apply_lgf_IF(double alpha_base, int fmm_type = IBLGF_AMR2AMR)
    {
        iblgf_ctx* c = dev_.ctx();
        check(c, iblgf_poisson_options(c, use_correction_ ? 1 : 0, subtract_non_leaf_ ? 1 : 0));
        for (std::size_t comp = 0; comp < Source::nFields(); ++comp)
        {
            const int src = dev_.template upload<Source>(comp, 0);
            const int tgt = dev_.template upload<Target>(comp, 1);
            check(c, iblgf_poisson_apply_if(c, src, tgt, alpha_base, fmm_type));
            dev_.template download<Target>(tgt, comp);
        }
    }

    bool& use_correction() noexcept { return use_correction_; }
    bool& subtract_non_leaf() noexcept { return subtract_non_leaf_; }
    DeviceDomain<domain_type>& device_domain() noexcept { return dev_; }

  private:
    DeviceDomain<domain_type>& dev_;
    bool use_correction_ = true;
    bool subtract_non_leaf_ = false;
};

// Fmm<Setup> (fmm/fmm.hpp:698): apply<Source,Target>(domain, kernel, level,
// non_leaf_as_source, add_with_scale, fmm_type). The kernel selects the
// sweep: a neighbour-only kernel with alpha_base_level() (LGF_GE, the
// adapter's or the reference's) runs the integrating-factor branch at
// alpha_base * 4^(level - base level), as the kernel's change_level sets it
// before the reference's apply_if calls apply; a kernel whose LaplaceLGF()
// is true (LGF_GL, the adapter's or the reference's) runs the full sweep.
// Kernel types with neither member do not compile; a kernel that has them
// but is neither (the reference's Helmholtz kernels) is rejected at run time.
template<class Setup>
class Fmm
{
  public:
    using domain_t = typename Setup::domain_t;

    explicit Fmm(domain_t* d, int /*Nb*/ = 0, int precision = IBLGF_FP64, int device = 0)
    : dev_(b200::device_domain(d, precision, device))
    {
    }

    template<class Source, class Target, class Kernel>
    void apply(domain_t*, Kernel* kernel, int level, bool non_leaf_as_source, double add_with_scale = 1.0,
               int fmm_type = IBLGF_AMR2AMR)
    {
        iblgf_ctx* c = dev_.ctx();
        int which = IBLGF_KERNEL_GL;
        double alpha = 0.0;
        static_assert(detail::has_alpha_base<Kernel>::value || detail::has_laplace_flag<Kernel>::value,
                      "Fmm::apply takes LGF_GL or LGF_GE kernels");
        if constexpr (detail::has_alpha_base<Kernel>::value)
        {
            if (!kernel->neighbor_only()) throw std::runtime_error("iblgf_b200: unsupported kernel (not LGF_GE)");
            which = IBLGF_KERNEL_GE;
            alpha = kernel->alpha_base_level() * std::pow(4.0, level - dev_.base_level());
        }
        else
        {
            if (!kernel->LaplaceLGF() || kernel->neighbor_only())
                throw std::runtime_error("iblgf_b200: unsupported kernel (not LGF_GL)");
        }
        const int src = dev_.template upload<Source>(0, 0);
        const int tgt = dev_.template upload<Target>(0, 1);
        check(c, iblgf_fmm_apply_kernel(c, src, tgt, level, non_leaf_as_source ? 1 : 0, add_with_scale, fmm_type,
                                        which, alpha));
        dev_.template download<Target>(tgt, 0);
    }

  private:
    DeviceDomain<domain_t>& dev_;
};

// --------------------------------------------------------------- operators
// domain::Operator's block operators and level wrappers. The per-block forms
// keep the reference's signatures (block = it->data(), dx_level); each moves
// the block's input components to the device, applies the operator to that
// octant and brings the outputs back, so they are a drop-in but pay a host
// round trip per block: the level wrappers run a whole level per launch.
// op codes of iblgf_op_apply: 0 laplace, 1 gradient, 2 divergence, 3 curl,
// 4 curl_transpose, 5 nonlinear.
template<class Domain>
class Operator
{
  public:
    template<class Src, class Dst, class Block>
    static void laplace(Block& block, double /*dx_level*/)
    {
        block_op<Src, Src, Dst>(block, 0, 1.0);
    }
    template<class Src, class Dst, class Block>
    static void gradient(Block& block, double /*dx_level*/)
    {
        block_op<Src, Src, Dst>(block, 1, 1.0);
    }
    template<class Src, class Dst, class Block>
    static void divergence(Block& block, double /*dx_level*/)
    {
        block_op<Src, Src, Dst>(block, 2, 1.0);
    }
    template<class Src, class Dst, class Block>
    static void curl(Block& block, double /*dx_level*/)
    {
        block_op<Src, Src, Dst>(block, 3, 1.0);
    }
    template<class Src, class Dst, class Block>
    static void curl_transpose(Block& block, double /*dx_level*/, double scale = 1.0)
    {
        block_op<Src, Src, Dst>(block, 4, scale);
    }
    // nonlinear<Face, Edge, Dst>(block): face velocity and edge vorticity in
    template<class Face, class Edge, class Dst, class Block>
    static void nonlinear(Block& block)
    {
        block_op<Face, Edge, Dst>(block, 5, 1.0);
    }

    // level wrappers (operators.hpp:521-650)
    template<class Src, class Dst>
    static void levelDivergence(Domain* d, int l)
    {
        level_op<Src, Dst>(d, 2, l, true, false, 1.0);
    }
    template<class Src, class Dst>
    static void levelGradient(Domain* d, int l)
    {
        level_op<Src, Dst>(d, 1, l, false, true, 1.0);
    }
    template<class Src, class Dst>
    static void domainDivergence(Domain* d)
    {
        DeviceDomain<Domain>& dev = device_domain(d);
        int bl = 0, depth = 0, n = 0;
        check(dev.ctx(), iblgf_domain_info(dev.ctx(), &bl, &depth, &n));
        for (int l = bl; l < depth; ++l) levelDivergence<Src, Dst>(d, l);
    }
    template<class Src, class Dst>
    static void domainGradient(Domain* d, double scale = 1.0)
    {
        DeviceDomain<Domain>& dev = device_domain(d);
        int bl = 0, depth = 0, n = 0;
        check(dev.ctx(), iblgf_domain_info(dev.ctx(), &bl, &depth, &n));
        for (int l = bl; l < depth; ++l) level_op<Src, Dst>(d, 1, l, false, true, scale);
    }

    // the domain whose blocks the per-block operators act on
    static Domain*& bound_domain()
    {
        static Domain* d = nullptr;
        return d;
    }

  private:
    template<class A, class B, class Dst, class Block>
    static void block_op(Block& block, int op, double scale)
    {
        Domain* d = bound_domain();
        if (!d) throw std::runtime_error("iblgf_b200: Operator<Domain>::bound_domain() is not set");
        DeviceDomain<Domain>& dev = device_domain(d);
        const int idx = dev.octant_of_block(&block);
        if (idx < 0) throw std::runtime_error("iblgf_b200: block is not a data block of the bound domain");
        iblgf_ctx* c = dev.ctx();
        int in[6], out[3];
        int n_in = 0, w = 0;
        for (std::size_t k = 0; k < A::nFields(); ++k) in[n_in++] = dev.template upload_octant<A>(idx, k, w++);
        if (!std::is_same<A, B>::value)
            for (std::size_t k = 0; k < B::nFields(); ++k) in[n_in++] = dev.template upload_octant<B>(idx, k, w++);
        for (std::size_t k = 0; k < Dst::nFields(); ++k) out[k] = dev.template upload_octant<Dst>(idx, k, w++);
        check(c, iblgf_op_apply_octants(c, op, in, n_in, out, (int)Dst::nFields(), &idx, 1, scale));
        for (std::size_t k = 0; k < Dst::nFields(); ++k) dev.template download_octant<Dst>(out[k], idx, k);
    }

    template<class Src, class Dst>
    static void level_op(Domain* d, int op, int l, bool exchange_src, bool exchange_dst, double scale)
    {
        DeviceDomain<Domain>& dev = device_domain(d);
        iblgf_ctx* c = dev.ctx();
        int in[3], out[3];
        int w = 0;
        for (std::size_t k = 0; k < Src::nFields(); ++k)
        {
            in[k] = dev.template upload<Src>(k, w++);
            if (exchange_src) check(c, iblgf_buffer_exchange(c, in[k], l));
        }
        for (std::size_t k = 0; k < Dst::nFields(); ++k) out[k] = dev.template upload<Dst>(k, w++);
        check(c, iblgf_op_apply(c, op, in, (int)Src::nFields(), out, (int)Dst::nFields(), l, scale));
        for (std::size_t k = 0; k < Dst::nFields(); ++k)
        {
            if (exchange_dst) check(c, iblgf_buffer_exchange(c, out[k], l));
            dev.template download<Dst>(out[k], k);
        }
    }
};

}  // namespace b200
}  // namespace iblgf
