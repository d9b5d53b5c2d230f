// C++ adapter: the reference's solver templates on top of the iblgf_b200
// C ABI, so a reference setup switches its typedefs and keeps its calls.
//
//   reference                                        this adapter
//   ----------------------------------------------   ------------------------------------
//   fmm::Fmm<Setup>::apply<Src,Tgt>(domain, kernel,  iblgf::b200::Fmm<Setup>::apply<Src,Tgt>(...)
//     level, non_leaf_as_source, scale, fmm_type)      (include/iblgf/fmm/fmm.hpp:729-870)
//   solver::PoissonSolver<Setup>::apply_lgf<S,T>()   iblgf::b200::PoissonSolver<Setup>::apply_lgf<S,T>()
//     / solve<S,T>() / use_correction()                (solver/poisson/poisson.hpp:131, 1362, 1494)
//
// Requirements on the domain (all members the reference Domain already has):
//   domain->begin()/end()  depth-first octant iteration; it->has_data(),
//   it->key().id(), it->is_leaf(), it->is_correction(), it->data_r(tag, i)
//   giving a DataField whose .data() / .size() is the Nb^3 block (x fastest);
//   domain->block_extent()[0], domain->bounding_box().base()/.extent(),
//   domain->dx_base(). Field types provide tag() and nFields() as the
//   reference's REGISTER_FIELDS types do.
//
// The octree is imported once (iblgf_domain_import) on first use; call
// reset() after the reference adapts its mesh. Fields are staged through host
// memory in the canonical octant order of the library.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
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

// Shared state of one domain on one GPU.
template<class Domain>
class DeviceDomain
{
  public:
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
    }

    iblgf_ctx* ctx()
    {
        if (!ctx_) init();
        return ctx_;
    }

    // host -> device for a reference field component
    // which: 0 for sources, 1 for targets (two device scratch fields)
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

    int scratch_field(int which)
    {
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
        std::unordered_map<uint64_t, typename Domain::octant_t*> by_key;
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
        int bl = 0, depth = 0, n = 0;
        check(ctx_, iblgf_domain_info(ctx_, &bl, &depth, &n));
        std::vector<uint64_t> canon(n);
        check(ctx_, iblgf_domain_octants(ctx_, canon.data(), nullptr, nullptr, nullptr));
        order_.resize(n);
        for (int i = 0; i < n; ++i) order_[i] = by_key.at(canon[i]);
        scratch_.clear();
    }

  public:
    bool subtract_non_leaf_ = false;

  private:
    Domain* domain_;
    int precision_, device_;
    iblgf_ctx* ctx_ = nullptr;
    std::vector<typename Domain::octant_t*> order_;
    std::vector<int> scratch_;
    std::vector<double> staging_;
};

// PoissonSolver<Setup> (solver/poisson/poisson.hpp:46): apply_lgf / solve for
// the LGF_GL kernel, every component of the source field.
template<class Setup>
class PoissonSolver
{
  public:
    using simulation_type = typename Setup::simulation_t;
    using domain_type = typename simulation_type::domain_type;

    explicit PoissonSolver(simulation_type* sim, int precision = IBLGF_FP64, int device = 0)
    : dev_(sim->domain_.get(), precision, device)
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

    bool& use_correction() noexcept { return use_correction_; }
    bool& subtract_non_leaf() noexcept { return subtract_non_leaf_; }
    DeviceDomain<domain_type>& device_domain() noexcept { return dev_; }

  private:
    DeviceDomain<domain_type> dev_;
    bool use_correction_ = true;
    bool subtract_non_leaf_ = false;
};

// Fmm<Setup> (fmm/fmm.hpp:698): apply<Source,Target>(domain, kernel, level,
// non_leaf_as_source, add_with_scale, fmm_type) with the LGF_GL kernel.
template<class Setup>
class Fmm
{
  public:
    using domain_t = typename Setup::domain_t;

    explicit Fmm(domain_t* d, int /*Nb*/ = 0, int precision = IBLGF_FP64, int device = 0)
    : dev_(d, precision, device)
    {
    }

    template<class Source, class Target, class Kernel>
    void apply(domain_t*, Kernel*, int level, bool non_leaf_as_source, double add_with_scale = 1.0,
               int fmm_type = IBLGF_AMR2AMR)
    {
        iblgf_ctx* c = dev_.ctx();
        const int src = dev_.template upload<Source>(0, 0);
        const int tgt = dev_.template upload<Target>(0, 1);
        check(c, iblgf_fmm_apply(c, src, tgt, level, non_leaf_as_source ? 1 : 0, add_with_scale, fmm_type));
        dev_.template download<Target>(tgt, 0);
    }

  private:
    DeviceDomain<domain_t> dev_;
};

}  // namespace b200
}  // namespace iblgf
