// extern "C" boundary of the library (include/iblgf_b200.h). Every entry
// point catches exceptions and turns them into a status code plus a message
// in iblgf_last_error(); nothing throws across the boundary.
#include <cstring>
#include <exception>
#include <new>

#include "ctx.hpp"

struct iblgf_ctx
{
    iblgf_b200::Ctx c;
};

namespace
{
thread_local std::string g_create_err;

template<class F>
int guard(iblgf_ctx* x, F&& f)
{
    if (!x) return IBLGF_EINVAL;
    try
    {
        f(x->c);
        return IBLGF_OK;
    }
    catch (const iblgf_b200::Error& e)
    {
        x->c.err = e.what();
        return e.code;
    }
    catch (const std::bad_alloc&)
    {
        x->c.err = "host allocation failed";
        return IBLGF_ENOMEM;
    }
    catch (const std::exception& e)
    {
        x->c.err = e.what();
        return IBLGF_EINTERNAL;
    }
}

void need_field(iblgf_b200::Ctx& c, int f)
{
    if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
    if (f < 0 || f >= (int)c.fields.size()) throw iblgf_b200::Error(IBLGF_EINVAL, "bad field id");
}
}  // namespace

namespace iblgf_b200
{
void launch_lgf_eval(Ctx& c, const int* d_coords, size_t n, double* d_out);
void poisson_release(Ctx& c);
double measure_fma_peak(Ctx& c, int precision);
double measure_tc_rate(Ctx& c, int n);
double helm2d_origin(double c);
void helm2d_table(Ctx& c, double cz, int nx, int ny, double* dev_out);
void helm2d_check_table(double cz, int nx, int ny);
void helm2d_points(Ctx& c, double cz, int count, const int* host_nm, double* host_out);
void helm2d_apply(Ctx& c, double cz, int nx, int ny, const double* dev_f, double* dev_u, double scale);
void helm2d_op(Ctx& c, int op, int nb, int n_blocks, int n_modes, double dx, double lz, double scale,
               const unsigned char* host_mode_mask, const double* dev_src, double* dev_dst);
void helm2d_nonlinear(Ctx& c, int nb, int n_blocks, int n_planes, const unsigned char* host_plane_mask,
                      const double* dev_face, const double* dev_edge, double* dev_dst);
void helm2d_real_op(Ctx& c, int op, int nb, int n_blocks, int np, double dx, double dx_fine, double cz, double scale,
                    const double* a, int a_comp, const double* b, int b_comp, double* d, int d_comp, double* e);
void wait_selftest(Ctx& c, long long polls);
long long first_nonfinite(Ctx& c, const double* p, size_t n);
}  // namespace iblgf_b200

extern "C" {

int iblgf_create(const iblgf_config* cfg, iblgf_ctx** out)
{
    if (!cfg || !out) return IBLGF_EINVAL;
    *out = nullptr;
    auto* x = new (std::nothrow) iblgf_ctx;
    if (!x) return IBLGF_ENOMEM;
    x->c.cfg = *cfg;
    const int rc = guard(x, [](iblgf_b200::Ctx& c) { iblgf_b200::ctx_init(c); });
    if (rc != IBLGF_OK)
    {
        g_create_err = x->c.err;
        if (x->c.own_stream && x->c.stream) cudaStreamDestroy(x->c.stream);
        delete x;
        return rc;
    }
    *out = x;
    return IBLGF_OK;
}

int iblgf_destroy(iblgf_ctx* x)
{
    if (!x) return IBLGF_EINVAL;
    cudaStreamSynchronize(x->c.stream);
    iblgf_b200::poisson_release(x->c);
    iblgf_b200::ns_release(x->c);
    iblgf_b200::batch_release(x->c);
    iblgf_b200::ib_release(x->c);
    iblgf_b200::copy_stream_release(x->c);
    x->c.fields.clear();  // stream-ordered frees on the context stream
    x->c.leaf_stage.release();
    x->c.exchange_buf.release();  // stream-ordered: before the stream goes
    cudaStreamSynchronize(x->c.stream);
    if (x->c.own_stream) cudaStreamDestroy(x->c.stream);
    delete x;
    return IBLGF_OK;
}

const char* iblgf_last_error(iblgf_ctx* x) { return x ? x->c.err.c_str() : g_create_err.c_str(); }

int iblgf_synchronize(iblgf_ctx* x)
{
    return guard(x, [](iblgf_b200::Ctx& c) {
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        if (c.copy_stream) IBLGF_CUDA(cudaStreamSynchronize(c.copy_stream));
        iblgf_b200::check_status(c);
    });
}

int iblgf_domain_add_blocks(iblgf_ctx* x, int n, const int* base, const int* extent)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain already finalized");
        iblgf_b200::add_blocks(c, n, base, extent);
    });
}

int iblgf_domain_import(iblgf_ctx* x, int n, const uint64_t* keys, const int* flags)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain already finalized");
        if (n <= 0 || !keys || !flags) throw iblgf_b200::Error(IBLGF_EINVAL, "bad import arguments");
        c.tree.import_octants(n, keys, flags);
        c.has_blocks = true;
    });
}

int iblgf_domain_restart(iblgf_ctx* x, int n, const uint64_t* keys, const unsigned char* leaf)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain already finalized");
        if (n <= 0 || !keys || !leaf) throw iblgf_b200::Error(IBLGF_EINVAL, "bad restart arguments");
        c.tree.restart(n, keys, leaf);
        c.has_blocks = true;
    });
}

int iblgf_domain_init_refine(iblgf_ctx* x, int n_ref, int global_refinement, iblgf_refine_fn pred, void* user)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain already finalized");
        if (n_ref < 0 || global_refinement < 0) throw iblgf_b200::Error(IBLGF_EINVAL, "negative refinement");
        c.tree.init_refine(n_ref, global_refinement, pred, user);
    });
}

int iblgf_domain_finalize(iblgf_ctx* x, int subtract_non_leaf)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain already finalized");
        c.subtract_non_leaf = subtract_non_leaf != 0;
        iblgf_b200::domain_finalize(c);
    });
}

int iblgf_domain_info(iblgf_ctx* x, int* base_level, int* depth, int* n_octants)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
        if (base_level) *base_level = c.tree.base_level;
        if (depth) *depth = c.tree.depth;
        if (n_octants) *n_octants = c.n_oct;
    });
}

int iblgf_domain_octants(iblgf_ctx* x, uint64_t* keys, int* levels, int* flags, int* bbase)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
        for (int i = 0; i < c.n_oct; ++i)
        {
            if (keys) keys[i] = c.keys[i];
            if (levels) levels[i] = c.levels[i];
            if (flags) flags[i] = c.flags[i];
            if (bbase)
                for (int d = 0; d < 3; ++d) bbase[3 * i + d] = c.bbase[3 * i + d];
        }
    });
}

int iblgf_domain_lists(iblgf_ctx* x, int* nbr, int* infl, int* n_infl)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
        if (nbr) std::memcpy(nbr, c.nbr.data(), c.nbr.size() * sizeof(int));
        if (infl) std::memcpy(infl, c.infl.data(), c.infl.size() * sizeof(int));
        if (n_infl) std::memcpy(n_infl, c.n_infl.data(), c.n_infl.size() * sizeof(int));
    });
}

int iblgf_domain_masks(iblgf_ctx* x, int mask_idx, unsigned char* st)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::need_single(c);
        if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
        if (mask_idx < 0 || mask_idx >= (int)c.masks.size()) throw iblgf_b200::Error(IBLGF_EINVAL, "bad mask index");
        std::memcpy(st, c.masks[mask_idx].data(), c.masks[mask_idx].size());
    });
}

int iblgf_field_create(iblgf_ctx* x, int* field)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "domain not finalized");
        if (!field) throw iblgf_b200::Error(IBLGF_EINVAL, "null field pointer");
        *field = iblgf_b200::field_create(c);
    });
}

int iblgf_field_zero(iblgf_ctx* x, int f)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        IBLGF_CUDA(cudaMemsetAsync(c.field(f), 0, c.field_elems() * sizeof(double), c.stream));
    });
}

int iblgf_field_upload(iblgf_ctx* x, int f, const double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        if (count != c.field_elems() || !host) throw iblgf_b200::Error(IBLGF_EINVAL, "field size mismatch");
        IBLGF_CUDA(cudaMemcpyAsync(c.field(f), host, count * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    });
}

int iblgf_field_download(iblgf_ctx* x, int f, double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        if (count != c.field_elems() || !host) throw iblgf_b200::Error(IBLGF_EINVAL, "field size mismatch");
        IBLGF_CUDA(cudaMemcpyAsync(host, c.field(f), count * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        iblgf_b200::check_status(c);  // synchronises the stream
    });
}

int iblgf_field_upload_leaves(iblgf_ctx* x, int f, const double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        iblgf_b200::field_upload_leaves(c, f, host, count);
    });
}

int iblgf_field_download_leaves(iblgf_ctx* x, int f, double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        iblgf_b200::field_download_leaves(c, f, host, count);
    });
}

int iblgf_field_upload_leaves_async(iblgf_ctx* x, int f, const double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        iblgf_b200::field_upload_leaves_async(c, f, host, count);
    });
}

int iblgf_field_download_leaves_async(iblgf_ctx* x, int f, double* host, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        iblgf_b200::field_download_leaves_async(c, f, host, count);
    });
}

int iblgf_field_device_ptr(iblgf_ctx* x, int f, double** dptr)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        *dptr = c.field(f);
    });
}

int iblgf_fmm_apply(iblgf_ctx* x, int source, int target, int level, int nlas, double scale, int fmm_type)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, source);
        need_field(c, target);
        iblgf_b200::fmm_apply(c, source, target, level, nlas != 0, scale, fmm_type);
    });
}

int iblgf_poisson_apply_lgf(iblgf_ctx* x, int source, int target, int fmm_type)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, source);
        need_field(c, target);
        iblgf_b200::poisson_apply_lgf(c, source, target, fmm_type);
    });
}

int iblgf_poisson_apply_if(iblgf_ctx* x, int source, int target, double alpha_base, int fmm_type)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, source);
        need_field(c, target);
        iblgf_b200::apply_if(c, source, target, alpha_base, fmm_type);
    });
}

int iblgf_poisson_options(iblgf_ctx* x, int use_correction, int subtract_non_leaf)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        c.use_correction = use_correction != 0;
        if (c.finalized && (subtract_non_leaf != 0) != c.subtract_non_leaf)
            throw iblgf_b200::Error(IBLGF_EINVAL, "subtract_non_leaf is fixed at finalize (masks depend on it)");
        c.subtract_non_leaf = subtract_non_leaf != 0;
    });
}

int iblgf_op_apply(iblgf_ctx* x, int op, const int* in, int n_in, const int* out, int n_out, int level, double scale)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!in || !out) throw iblgf_b200::Error(IBLGF_EINVAL, "null field list");
        for (int i = 0; i < n_in; ++i) need_field(c, in[i]);
        for (int i = 0; i < n_out; ++i) need_field(c, out[i]);
        iblgf_b200::apply_op(c, op, in, n_in, out, n_out, level, scale);
    });
}

int iblgf_buffer_exchange(iblgf_ctx* x, int field, int level)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, field);
        iblgf_b200::buffer_exchange(c, field, level);
    });
}

int iblgf_lgf_table(iblgf_ctx* x, double* host_out, size_t count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (count != c.d_lgf_table.n || !host_out) throw iblgf_b200::Error(IBLGF_EINVAL, "table size is 176851");
        IBLGF_CUDA(cudaMemcpyAsync(host_out, c.d_lgf_table.p, count * sizeof(double), cudaMemcpyDeviceToHost,
                                   c.stream));
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int iblgf_lgf_get(iblgf_ctx* x, const int* coords, size_t n, double* host_out)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!n) return;
        if (!coords || !host_out) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        iblgf_b200::DevBuf<int> dc;
        iblgf_b200::DevBuf<double> dout;
        dc.alloc(3 * n);
        dout.alloc(n);
        IBLGF_CUDA(cudaMemcpyAsync(dc.p, coords, 3 * n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        iblgf_b200::launch_lgf_eval(c, dc.p, n, dout.p);
        IBLGF_CUDA(cudaMemcpyAsync(host_out, dout.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int iblgf_lgf_ge_get(iblgf_ctx* x, double alpha, const int* coords, size_t n, double* host_out)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!n) return;
        if (!coords || !host_out) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        const int ge = iblgf_b200::ge_table(c, alpha);
        iblgf_b200::DevBuf<int> dc;
        iblgf_b200::DevBuf<double> dout;
        dc.alloc(3 * n);
        dout.alloc(n);
        IBLGF_CUDA(cudaMemcpyAsync(dc.p, coords, 3 * n * sizeof(int), cudaMemcpyHostToDevice, c.stream));
        iblgf_b200::launch_lgf_ge_eval(c, ge, dc.p, n, dout.p);
        IBLGF_CUDA(cudaMemcpyAsync(host_out, dout.p, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int iblgf_fmm_apply_kernel(iblgf_ctx* x, int source, int target, int level, int nlas, double scale, int fmm_type,
                           int kernel, double alpha)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, source);
        need_field(c, target);
        if (kernel == IBLGF_KERNEL_GL)
            iblgf_b200::fmm_apply(c, source, target, level, nlas != 0, scale, fmm_type);
        else if (kernel == IBLGF_KERNEL_GE)
        {
            if (fmm_type != IBLGF_AMR2AMR && fmm_type != IBLGF_IB2xIB)
                throw iblgf_b200::Error(IBLGF_EINVAL, "the LGF_GE kernel sweeps with AMR2AMR or IB2xIB masks");
            const int ge = iblgf_b200::ge_table(c, alpha);
            iblgf_b200::fmm_apply(c, source, target, level, nlas != 0, scale, fmm_type, ge);
        }
        else
            throw iblgf_b200::Error(IBLGF_EINVAL, "kernel must be IBLGF_KERNEL_GL or IBLGF_KERNEL_GE");
    });
}

int iblgf_op_apply_octants(iblgf_ctx* x, int op, const int* in, int n_in, const int* out, int n_out,
                           const int* octants, int n, double scale)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!in || !out || (n > 0 && !octants)) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        for (int i = 0; i < n_in; ++i) need_field(c, in[i]);
        for (int i = 0; i < n_out; ++i) need_field(c, out[i]);
        iblgf_b200::apply_op_octants(c, op, in, n_in, out, n_out, octants, n, scale);
    });
}

int iblgf_field_upload_octants(iblgf_ctx* x, int field, const int* octants, int n, const double* host)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, field);
        if (n > 0 && (!octants || !host)) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        const size_t B = c.block_elems();
        for (int i = 0; i < n; ++i)
        {
            if (octants[i] < 0 || octants[i] >= c.n_oct) throw iblgf_b200::Error(IBLGF_EINVAL, "octant out of range");
            IBLGF_CUDA(cudaMemcpyAsync(c.field(field) + (size_t)octants[i] * B, host + (size_t)i * B,
                                       B * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        }
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int iblgf_field_download_octants(iblgf_ctx* x, int field, const int* octants, int n, double* host)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, field);
        if (n > 0 && (!octants || !host)) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        const size_t B = c.block_elems();
        for (int i = 0; i < n; ++i)
        {
            if (octants[i] < 0 || octants[i] >= c.n_oct) throw iblgf_b200::Error(IBLGF_EINVAL, "octant out of range");
            IBLGF_CUDA(cudaMemcpyAsync(host + (size_t)i * B, c.field(field) + (size_t)octants[i] * B,
                                       B * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        }
        iblgf_b200::check_status(c);  // synchronises the stream
    });
}

int iblgf_conv_block(iblgf_ctx* x, const double* src, const double* kernel, double* out, double scale)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!src || !kernel || !out) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        iblgf_b200::launch_conv_block(c, src, kernel, out, scale);
    });
}

int iblgf_ns_step(iblgf_ctx* x, const int* u_fields, int p_field, double dt, double Re, double* T, int n_steps)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!u_fields || !T) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        if (n_steps < 0) throw iblgf_b200::Error(IBLGF_EINVAL, "negative step count");
        iblgf_b200::ns_step(c, u_fields, p_field, dt, Re, T, n_steps);
    });
}

int iblgf_batch_add_problem(iblgf_ctx* x, const int* bd_base, const int* bd_extent, int n_boxes, const int* base,
                            const int* extent, int n_ref, iblgf_refine_fn pred, void* user, int* problem)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        const int id = iblgf_b200::batch_add_problem(c, bd_base, bd_extent, n_boxes, base, extent, n_ref, pred, user);
        if (problem) *problem = id;
    });
}

int iblgf_batch_finalize(iblgf_ctx* x, int subtract_non_leaf)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        c.subtract_non_leaf = subtract_non_leaf != 0;
        iblgf_b200::batch_finalize(c);
    });
}

int iblgf_batch_problem_info(iblgf_ctx* x, int problem, int* info)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!c.batch || !c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "batch not finalized");
        if (problem < 0 || problem >= (int)c.sub.size() || !info)
            throw iblgf_b200::Error(IBLGF_EINVAL, "bad problem index");
        const iblgf_b200::Ctx& s = *c.sub[problem];
        info[0] = c.sub_off[problem];
        info[1] = s.n_oct;
        info[2] = s.tree.base_level;
        info[3] = s.tree.depth;
    });
}

int iblgf_batch_problem_octants(iblgf_ctx* x, int problem, uint64_t* keys, int* levels, int* flags, int* bbase)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!c.batch || !c.finalized) throw iblgf_b200::Error(IBLGF_EINVAL, "batch not finalized");
        if (problem < 0 || problem >= (int)c.sub.size()) throw iblgf_b200::Error(IBLGF_EINVAL, "bad problem index");
        const iblgf_b200::Ctx& s = *c.sub[problem];
        for (int i = 0; i < s.n_oct; ++i)
        {
            if (keys) keys[i] = s.keys[i];
            if (levels) levels[i] = s.levels[i];
            if (flags) flags[i] = s.flags[i];
            if (bbase)
                for (int d = 0; d < 3; ++d) bbase[3 * i + d] = s.bbase[3 * i + d];
        }
    });
}

int iblgf_batch_apply_lgf(iblgf_ctx* x, int src, int tgt)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::batch_apply_lgf(c, src, tgt); });
}

int iblgf_ns_options(iblgf_ctx* x, const double* frame_vel, double cg_threshold, int cg_max_iter)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ns_options(c, frame_vel, cg_threshold, cg_max_iter); });
}

int iblgf_adapt(iblgf_ctx* x, int n_attempts, const uint64_t* keys, const int* level_change, int n_interp,
                const int* interp_fields, const int* interp_mesh, int* base_mesh_update)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::domain_adapt(c, n_attempts, reinterpret_cast<const iblgf_b200::u64*>(keys), level_change,
                                 n_interp, interp_fields, interp_mesh, base_mesh_update);
    });
}

int iblgf_ns_fields(iblgf_ctx* x, int* ids)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ns_fields(c, ids); });
}

int iblgf_ns_clean(iblgf_ctx* x, int field, int non_leaf_only, int width)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ns_clean(c, field, non_leaf_only != 0, width); });
}

int iblgf_ns_clean_leaf_correction_boundary(iblgf_ctx* x, const int* fields, int n, int level, int leaf_only_boundary)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::ns_clean_leaf_correction_boundary(c, fields, n, level, leaf_only_boundary != 0);
    });
}

int iblgf_block_norms(iblgf_ctx* x, const int* fields, int n_comp, double* max_out, double* rms_out)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::block_norms(c, fields, n_comp, max_out, rms_out); });
}

int iblgf_ib_force(iblgf_ctx* x, int stage, double* out, int* iters)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ib_force(c, stage, out, iters); });
}

int iblgf_ib_stage_status(iblgf_ctx* x, int stage, int* iters, int* converged)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        int nc = 0;
        iblgf_b200::ib_force(c, stage, nullptr, iters, &nc);
        if (converged) *converged = nc ? 0 : 1;
    });
}

int iblgf_ib_warmstart(iblgf_ctx* x, int mode, int train_steps, int epochs, double lr, unsigned seed)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ib_warmstart(c, mode, train_steps, epochs, lr, seed); });
}

int iblgf_ib_warmstart_info(iblgf_ctx* x, double* info)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!info) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        iblgf_b200::ib_warmstart_info(c, info);
    });
}

int iblgf_ws_check(iblgf_ctx* x, int n_samples, int n_points, const float* params, const float* inputs,
                   const float* targets, float* outputs, float* grads, float* loss)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (n_samples <= 0 || n_points <= 0 || !params || !inputs || !targets || !outputs || !grads || !loss)
            throw iblgf_b200::Error(IBLGF_EINVAL, "bad arguments");
        iblgf_b200::ws_check(c, n_samples, n_points, params, inputs, targets, outputs, grads, loss);
    });
}

int iblgf_ib_set_points(iblgf_ctx* x, int n, const double* coords, double Re)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::ib_set_points(c, n, coords, Re); });
}

int iblgf_ib_flags(iblgf_ctx* x, int* flags)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!flags) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        iblgf_b200::ib_flags(c, flags);
    });
}

int iblgf_ib_solve(iblgf_ctx* x, const int* u_fields, double alpha, double threshold, int max_iter, double* force,
                   int* iters)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!u_fields || !force) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        if (max_iter < 0) throw iblgf_b200::Error(IBLGF_EINVAL, "negative iteration limit");
        if (!iblgf_b200::ib_solve(c, u_fields, alpha, threshold, max_iter, force, iters))
            throw iblgf_b200::Error(IBLGF_ENOTCONVERGED, "IB force CG reached max_iter without converging "
                                                         "(force and iteration count written)");
    });
}

int iblgf_domain_partition(iblgf_ctx* x, int n_ranks, int* owner)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!owner) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        const std::vector<int> w = iblgf_b200::domain_partition(c, n_ranks);
        std::copy(w.begin(), w.end(), owner);
    });
}

int iblgf_domain_set_owner(iblgf_ctx* x, const int* owner, int rank, iblgf_exchange_fn exchange, void* user)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { iblgf_b200::domain_set_owner(c, owner, rank, exchange, user); });
}

int iblgf_mac_variant(iblgf_ctx* x, int variant)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (variant < -1 || variant > 3)
            throw iblgf_b200::Error(IBLGF_EINVAL, "MAC variant must be -1, 0, 1, 2 or 3");
        c.mac_variant_forced = variant;
    });
}

int iblgf_ge_direct(iblgf_ctx* x, int enable)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        c.ge_direct_enabled = enable != 0;
    });
}

int iblgf_mac_tuning(iblgf_ctx* x, double* out, int max_rows, int* n_rows)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!n_rows || (max_rows > 0 && !out)) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        const int n = (int)c.mac_tuning.size();
        *n_rows = n;
        for (int i = 0; i < n && i < max_rows; ++i)
            for (int j = 0; j < 8; ++j) out[8 * i + j] = c.mac_tuning[i][j];
    });
}

int iblgf_conv_block_noalloc(iblgf_ctx* x, const double* src, const double* kernel, double* out, double scale)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!src || !kernel || !out) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        iblgf_b200::launch_conv_block_noalloc(c, src, kernel, out, scale);
    });
}

int iblgf_kernel_launches(iblgf_ctx* x, long long* count)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { *count = c.launches; });
}

int iblgf_profile(iblgf_ctx* x, int enable)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        for (auto& ev : c.prof_events)
            for (auto e : ev) cudaEventDestroy(e);
        c.prof_events.clear();
        for (long long& v : c.stats) v = 0;
        c.profile = enable != 0;
    });
}

int iblgf_profile_read(iblgf_ctx* x, double* out4)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        IBLGF_CUDA(cudaStreamSynchronize(c.stream));
        for (int i = 0; i < 4; ++i) out4[i] = 0.0;
        for (auto& ev : c.prof_events)
        {
            float ms[4];
            for (int i = 0; i < 4; ++i) IBLGF_CUDA(cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]));
            // [0] forward transforms, [1] MAC, [2] inverse + interpolation + add,
            // [3] zero / copy / anterpolation
            out4[0] += ms[1];
            out4[1] += ms[2];
            out4[2] += ms[3];
            out4[3] += ms[0];
        }
    });
}

int iblgf_stats(iblgf_ctx* x, long long* out8)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        for (int i = 0; i < 8; ++i) out8[i] = c.stats[i];
    });
}

int iblgf_stats_n(iblgf_ctx* x, long long* out, int n)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!out || n < 1 || n > iblgf_b200::kNumStats) throw iblgf_b200::Error(IBLGF_EINVAL, "bad stats count");
        for (int i = 0; i < n; ++i) out[i] = c.stats[i];
    });
}

int iblgf_fma_peak(iblgf_ctx* x, int precision, double* tflops)
{
    return guard(x, [&](iblgf_b200::Ctx& c) { *tflops = iblgf_b200::measure_fma_peak(c, precision); });
}

int iblgf_helm2d_origin(double c, double* out)
{
    if (!out || !(c > 0.0)) return IBLGF_EINVAL;
    *out = iblgf_b200::helm2d_origin(c);
    return IBLGF_OK;
}

int iblgf_helm2d_lgf(iblgf_ctx* x, double c, int nx, int ny, double* host_out)
{
    return guard(x, [&](iblgf_b200::Ctx& cx) {
        if (!host_out) throw iblgf_b200::Error(IBLGF_EINVAL, "bad table arguments");
        iblgf_b200::helm2d_check_table(c, nx, ny);
        iblgf_b200::DevBuf<double> d;
        d.alloc((size_t)nx * ny);
        iblgf_b200::helm2d_table(cx, c, nx, ny, d.p);
        IBLGF_CUDA(cudaMemcpyAsync(host_out, d.p, (size_t)nx * ny * sizeof(double), cudaMemcpyDeviceToHost, cx.stream));
        IBLGF_CUDA(cudaStreamSynchronize(cx.stream));
    });
}

int iblgf_helm2d_get(iblgf_ctx* x, double c, int n, const int* host_nm, double* host_out)
{
    return guard(x, [&](iblgf_b200::Ctx& cx) { iblgf_b200::helm2d_points(cx, c, n, host_nm, host_out); });
}

int iblgf_helm2d_apply(iblgf_ctx* x, double c, int nx, int ny, const double* host_f, double* host_u, double scale)
{
    return guard(x, [&](iblgf_b200::Ctx& cx) {
        if (!host_f || !host_u || nx < 1 || ny < 1 || nx > 6144 || ny > 65535)
            throw iblgf_b200::Error(IBLGF_EINVAL, "bad arguments (1 <= nx <= 6144, 1 <= ny <= 65535)");
        const size_t n = (size_t)nx * ny;
        iblgf_b200::DevBuf<double> f, u;
        f.alloc(n);
        u.alloc(n);
        IBLGF_CUDA(cudaMemcpyAsync(f.p, host_f, n * sizeof(double), cudaMemcpyHostToDevice, cx.stream));
        IBLGF_CUDA(cudaMemcpyAsync(u.p, host_u, n * sizeof(double), cudaMemcpyHostToDevice, cx.stream));
        iblgf_b200::helm2d_apply(cx, c, nx, ny, f.p, u.p, scale);
        IBLGF_CUDA(cudaMemcpyAsync(host_u, u.p, n * sizeof(double), cudaMemcpyDeviceToHost, cx.stream));
        IBLGF_CUDA(cudaStreamSynchronize(cx.stream));
    });
}

int iblgf_helm2d_op(iblgf_ctx* x, int op, int nb, int n_blocks, int n_modes, double dx_level, double lz,
                    double scale, const double* dev_src, double* dev_dst)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (n_blocks && (!dev_src || !dev_dst)) throw iblgf_b200::Error(IBLGF_EINVAL, "null field");
        iblgf_b200::helm2d_op(c, op, nb, n_blocks, n_modes, dx_level, lz, scale, nullptr, dev_src, dev_dst);
    });
}

int iblgf_helm2d_op_modes(iblgf_ctx* x, int op, int nb, int n_blocks, int n_modes, const unsigned char* mode_mask,
                          double dx_level, double lz, double scale, const double* dev_src, double* dev_dst)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (n_blocks && (!dev_src || !dev_dst)) throw iblgf_b200::Error(IBLGF_EINVAL, "null field");
        iblgf_b200::helm2d_op(c, op, nb, n_blocks, n_modes, dx_level, lz, scale, mode_mask, dev_src, dev_dst);
    });
}

int iblgf_helm2d_real_op(iblgf_ctx* x, int op, int nb, int n_blocks, int n_planes, double dx_level, double dx_fine,
                         double c, double scale, const double* dev_a, int a_comp, const double* dev_b, int b_comp,
                         double* dev_d, int d_comp, double* dev_e)
{
    return guard(x, [&](iblgf_b200::Ctx& cx) {
        iblgf_b200::helm2d_real_op(cx, op, nb, n_blocks, n_planes, dx_level, dx_fine, c, scale, dev_a, a_comp, dev_b,
                                   b_comp, dev_d, d_comp, dev_e);
    });
}

int iblgf_helm2d_nonlinear(iblgf_ctx* x, int nb, int n_blocks, int n_planes, const unsigned char* plane_mask,
                           const double* dev_face, const double* dev_edge, double* dev_dst)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (n_blocks && (!dev_face || !dev_edge || !dev_dst)) throw iblgf_b200::Error(IBLGF_EINVAL, "null field");
        iblgf_b200::helm2d_nonlinear(c, nb, n_blocks, n_planes, plane_mask, dev_face, dev_edge, dev_dst);
    });
}

int iblgf_wait_selftest(iblgf_ctx* x, long long polls)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        iblgf_b200::wait_selftest(c, polls);
        iblgf_b200::check_status(c);  // synchronises; IBLGF_ETIMEOUT when the wait ran out
    });
}

int iblgf_field_first_nonfinite(iblgf_ctx* x, int f, long long* index)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        need_field(c, f);
        if (!index) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        *index = iblgf_b200::first_nonfinite(c, c.field(f), c.field_elems());
    });
}

int iblgf_debug_fail_alloc(long long after)
{
    if (after < -1) return IBLGF_EINVAL;
    iblgf_b200::alloc_fail_countdown().store(after);
    return IBLGF_OK;
}

int iblgf_tc_mma_rate(iblgf_ctx* x, int n, double* clocks)
{
    return guard(x, [&](iblgf_b200::Ctx& c) {
        if (!clocks) throw iblgf_b200::Error(IBLGF_EINVAL, "null argument");
        *clocks = iblgf_b200::measure_tc_rate(c, n);
        iblgf_b200::check_status(c);
    });
}

}  // extern "C"
