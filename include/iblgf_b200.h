/* iblgf_b200 — B200-native (sm_100a) lattice-Green's-function FMM Poisson
 * path of IBLGF-AMR behind a plain C ABI.
 *
 * Every entry point returns 0 on success and a non-zero IBLGF_E* code on
 * failure; iblgf_last_error() then holds a message. No C++ exception crosses
 * this boundary. One context per host thread; all device work of a context is
 * ordered on the context's CUDA stream.
 *
 * Field layout: a field holds one Nb^3 block per octant (Nb = block_extent+2,
 * one buffer cell on each side), x fastest, octants in the canonical order
 * returned by iblgf_domain_octants (tree level ascending, then Morton key) —
 * the reference's DataField column-major cube (linalg_xtensor.hpp cube_wrap)
 * laid out block after block.
 */
#ifndef IBLGF_B200_H
#define IBLGF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct iblgf_ctx iblgf_ctx;

enum
{
    IBLGF_OK = 0,
    IBLGF_EINVAL = 1,   /* bad argument or call order */
    IBLGF_ECUDA = 2,    /* CUDA runtime error */
    IBLGF_ENOMEM = 3,   /* device allocation failed */
    IBLGF_ETIMEOUT = 4, /* a bounded device wait gave up */
    IBLGF_EINTERNAL = 5,
    IBLGF_ENOTCONVERGED = 6 /* an iterative solve stopped at its iteration limit; outputs written */
};

enum { IBLGF_FP64 = 0, IBLGF_FP32 = 1 };

/* octant_t::MASK_TYPE (include/iblgf/domain/octree/octant.hpp:69-78) */
/* mask types (octant.hpp MASK_TYPE): STREAM, AMR2AMR, and the immersed-
 * boundary ones IB2xIB (IB blocks -> IB and extended-IB blocks), xIB2IB
 * (IB and extended-IB -> IB), IB2AMR (IB -> all blocks of a level) */
enum { IBLGF_STREAM = 0, IBLGF_AMR2AMR = 1, IBLGF_IB2xIB = 2, IBLGF_xIB2IB = 3, IBLGF_IB2AMR = 4 };

typedef struct
{
    int block_extent;   /* cells per block edge (reference "block_extent") */
    int bd_base[3];     /* bounding box ("bd_base") */
    int bd_extent[3];   /* bounding box ("bd_extent") */
    double dx_base;     /* base-level spacing ("dx_base" or Lx / bd_extent) */
    int precision;      /* IBLGF_FP64 (plain) or IBLGF_FP32 (FFT/MAC in FP32) */
    int device;         /* CUDA device ordinal */
    int intrp_order;    /* cell-centred interpolation order (reference default 5) */
    void* stream;       /* cudaStream_t to order work on, or NULL for a private one */
} iblgf_config;

/* Refinement predicate (Domain::register_refinement_condition): block base
 * and extent in level cells, refinement level, and diff_level = nRef - level.
 * Return non-zero to refine. */
typedef int (*iblgf_refine_fn)(void* user, const int* base, const int* extent,
                               int refinement_level, int diff_level);

/* ---- context --------------------------------------------------------- */
int iblgf_create(const iblgf_config* cfg, iblgf_ctx** out);
int iblgf_destroy(iblgf_ctx* ctx);
const char* iblgf_last_error(iblgf_ctx* ctx);
int iblgf_synchronize(iblgf_ctx* ctx);

/* ---- domain: Domain::initialize / construct_basemesh_blocks
 *      (include/iblgf/domain/domain.hpp:107-212, 405-488),
 *      Domain::init_refine (:878-939), mark_correction (:617-736),
 *      Tree::construct_lists (tree.hpp:571-603) ------------------------- */
int iblgf_domain_add_blocks(iblgf_ctx* ctx, int n, const int* base, const int* extent);
int iblgf_domain_init_refine(iblgf_ctx* ctx, int n_ref, int global_refinement,
                             iblgf_refine_fn pred, void* user);
/* Imports an octree built elsewhere (the reference's Domain after
 * init_refine / mark_correction) instead of add_blocks + init_refine: the
 * keys of every octant that holds data (Octant::has_data) and their flags
 * (bit 0 leaf, bit 1 correction). Block bases follow
 * Tree::octant_to_level_coordinate (domain.hpp:196-201). Call once, before
 * iblgf_domain_finalize. */
int iblgf_domain_import(iblgf_ctx* ctx, int n, const uint64_t* keys, const int* flags);
/* Rebuilds the octree of a restart (Domain::Domain from restart files,
 * domain.hpp:235-290, then restart_list_construct :839-849): `keys` and
 * `leaf` (one byte each) as Tree::write stores them (tree.hpp:832-855:
 * every octant with data except the root); ancestors receive data and
 * mark_correction recomputes the correction flags. Replaces add_blocks +
 * init_refine; call once, before iblgf_domain_finalize. */
int iblgf_domain_restart(iblgf_ctx* ctx, int n, const uint64_t* keys, const unsigned char* leaf);
/* Builds the neighbour / influence lists on the device, the FMM masks
 * (FmmMaskBuilder::fmm_lgf_mask_build, fmm_vortex_streamfun_mask) and
 * allocates the working fields. subtract_non_leaf as in the reference. */
int iblgf_domain_finalize(iblgf_ctx* ctx, int subtract_non_leaf);
int iblgf_domain_info(iblgf_ctx* ctx, int* base_level, int* depth, int* n_octants);
/* flags: bit 0 leaf, bit 1 correction; bbase: block base in level cells */
int iblgf_domain_octants(iblgf_ctx* ctx, uint64_t* keys, int* levels, int* flags, int* bbase);
/* nbr: 27 per octant (z slowest, self at 13), infl: 189 per octant, -1 = none */
int iblgf_domain_lists(iblgf_ctx* ctx, int* nbr, int* infl, int* n_infl);
int iblgf_domain_masks(iblgf_ctx* ctx, int mask_idx, unsigned char* source_target);

/* ---- fields ----------------------------------------------------------- */
int iblgf_field_create(iblgf_ctx* ctx, int* field);
int iblgf_field_zero(iblgf_ctx* ctx, int field);
int iblgf_field_upload(iblgf_ctx* ctx, int field, const double* host, size_t count);
int iblgf_field_download(iblgf_ctx* ctx, int field, double* host, size_t count);
/* Leaf-interior transfers (DataField::update_device / update_host,
 * datafield.hpp:211-226, for the values a solve reads and writes): `host`
 * holds, for every leaf octant (flag bit 0) in canonical order, its
 * block_extent^3 interior values, x fastest; count = n_leaves *
 * block_extent^3. The upload zeroes the field (buffers, non-leaf blocks)
 * and scatters the interiors; the download gathers them and returns after
 * the copy. */
int iblgf_field_upload_leaves(iblgf_ctx* ctx, int field, const double* host, size_t count);
int iblgf_field_download_leaves(iblgf_ctx* ctx, int field, double* host, size_t count);
/* As iblgf_field_download_leaves, but returns at once: the gather is ordered
 * on the context stream, the copy to `host` runs on a second stream of the
 * context (overlapping the context stream's next work, e.g. the next upload
 * and solve; `host` should be pinned). iblgf_synchronize waits for it. */
int iblgf_field_download_leaves_async(iblgf_ctx* ctx, int field, double* host, size_t count);
/* As iblgf_field_upload_leaves, but returns at once: the copy from `host`
 * (pinned) runs on the context's second stream, the zeroing and scatter are
 * ordered on the context stream after it. Issued right after a solve, the
 * next input's copy runs under that solve. `host` must stay unchanged until
 * the next synchronising call; a later asynchronous upload waits for this
 * one's scatter. */
int iblgf_field_upload_leaves_async(iblgf_ctx* ctx, int field, const double* host, size_t count);
int iblgf_field_device_ptr(iblgf_ctx* ctx, int field, double** dptr);
/* Whole Nb^3 blocks of the listed octants (canonical indices) from / to
 * host memory, n blocks back to back: the reference's per-octant
 * DataField::update_device / update_host (datafield.hpp:211-226). */
int iblgf_field_upload_octants(iblgf_ctx* ctx, int field, const int* octants, int n, const double* host);
int iblgf_field_download_octants(iblgf_ctx* ctx, int field, const int* octants, int n, double* host);

/* ---- solver ----------------------------------------------------------- */
/* Fmm<Setup>::apply<Source,Target>(domain, LGF_GL, level, non_leaf_as_source,
 * add_with_scale, fmm_type)  — include/iblgf/fmm/fmm.hpp:729-870 */
/* kernel objects of Fmm::apply: LGF_GL (lgf_gl.hpp:73-105) and LGF_GE
 * (lgf_ge.hpp:33-190, neighbour-only, lgf.hpp:209) */
enum { IBLGF_KERNEL_GL = 0, IBLGF_KERNEL_GE = 1 };
/* ---- sharded sweeps (several processes / GPUs on one octree) -----------
 * iblgf_domain_partition: the reference server's load-balanced split
 * (Server::compute_distribution, decomposition/server.hpp:245-330): per
 * level from the finest, the leaf and correction octants in Morton order are
 * cut into n_ranks contiguous runs of equal load (load = the octant's
 * neighbour + influence count over the AMR2AMR sweeps it is a target of,
 * the load FmmMaskBuilder::fmm_dry accumulates, fmm.hpp:597-626); every
 * other octant goes to the rank of its least-loaded child. owner receives
 * n_octants ranks.
 * iblgf_domain_set_owner: from now on every FMM sweep of this context
 * computes only the targets with owner == rank (and the coarser targets
 * whose values are interpolated into them); before the sweep's result is
 * added into its target field, exchange(user, buf, count, stream) is called
 * with the sweep's level targets gathered into a device buffer (count
 * doubles, ordered on `stream`, a cudaStream_t), and must replace buf by its
 * sum over all ranks (an all-reduce; a non-owned block is zero in every rank
 * but its owner's), returning 0 on success. Sources are transformed on every
 * rank. owner = NULL returns to unsharded sweeps. Plans are rebuilt. */
typedef int (*iblgf_exchange_fn)(void* user, double* device_buffer, size_t count, void* stream);
int iblgf_domain_partition(iblgf_ctx* ctx, int n_ranks, int* owner);
int iblgf_domain_set_owner(iblgf_ctx* ctx, const int* owner, int rank, iblgf_exchange_fn exchange, void* user);

/* Fmm::apply<Source,Target>(domain, kernel, level, non_leaf_as_source,
 * add_with_scale, fmm_type) with the kernel named explicitly: IBLGF_KERNEL_GL
 * (as iblgf_fmm_apply) or IBLGF_KERNEL_GE at the given alpha (the kernel's
 * alpha after change_level; the neighbour-only branch, fmm.hpp:754-770,
 * scale 1 instead of dx^2, fmm.hpp:1024-1026). */
int iblgf_fmm_apply_kernel(iblgf_ctx* ctx, int source, int target, int level, int non_leaf_as_source,
                           double add_with_scale, int fmm_type, int kernel, double alpha);
int iblgf_fmm_apply(iblgf_ctx* ctx, int source, int target, int level,
                    int non_leaf_as_source, double add_with_scale, int fmm_type);
/* PoissonSolver::apply_lgf<Source,Target>(fmm_type) for one scalar field —
 * include/iblgf/solver/poisson/poisson.hpp:131-135, 587-894 */
int iblgf_poisson_apply_lgf(iblgf_ctx* ctx, int source, int target, int fmm_type);
/* PoissonSolver::apply_lgf_IF<Source,Target>(alpha_base, fmm_type) for one
 * scalar field — the integrating factor e^{alpha L} with the LGF_GE kernel
 * (include/iblgf/lgf/lgf_ge.hpp:33-190), neighbour-only FMM branch
 * (fmm.hpp:754-770), alpha = alpha_base * 4^(level - base_level)
 * (poisson.hpp:428-494). */
int iblgf_poisson_apply_if(iblgf_ctx* ctx, int source, int target, double alpha_base, int fmm_type);
/* PoissonSolver::use_correction() / subtract_non_leaf() (poisson.hpp:1494-1498) */
int iblgf_poisson_options(iblgf_ctx* ctx, int use_correction, int subtract_non_leaf);

/* ---- mimetic block operators (include/iblgf/operators/operators.hpp) ----
 * Applied to the interior of every block of tree level `level` (all levels if
 * level < 0) with dx_level = dx_base / 2^(level - base_level); the one-cell
 * buffers are read, so exchange them first as the reference's level wrappers
 * do. Vector fields are 3 component field ids (face: normal components x,y,z;
 * edge: x,y,z). op: 0 laplace (:1386, cell->cell, 1 in / 1 out),
 * 1 gradient (:1421, cell->face, 1/3), 2 divergence (:1448, face->cell, 3/1),
 * 3 curl (:1479, face->edge, 3/3), 4 curl_transpose (:2416, edge->face, 3/3,
 * times scale), 5 nonlinear (:2455, face u + edge omega -> face, 6/3).
 * Outputs must not alias inputs. */
/* The same operators on the listed octants only (canonical indices), each
 * with its own dx_level: Operator::laplace<Src,Dst>(it->data(), dx_level) and
 * the others called per block (operators.hpp:1386-1513, 2416-2531). */
int iblgf_op_apply_octants(iblgf_ctx* ctx, int op, const int* in, int n_in, const int* out, int n_out,
                           const int* octants, int n, double scale);
int iblgf_op_apply(iblgf_ctx* ctx, int op, const int* in, int n_in, const int* out, int n_out,
                   int level, double scale);
/* client::buffer_exchange<Field>(level) (domain/decomposition/client.hpp:1120):
 * every buffer cell of the level's blocks takes the overlapping interior
 * value of its same-level neighbour. */
int iblgf_buffer_exchange(iblgf_ctx* ctx, int field, int level);

/* ---- LGF kernel (include/iblgf/lgf/lgf_gl_lookup.hpp:33-52) ------------ */
/* Copies the 176851-entry N_max = 100 table (positive integrals; get() = -value)
 * that the context generated on the device. */
int iblgf_lgf_table(iblgf_ctx* ctx, double* host_out, size_t count);
/* G(n) for n host coordinate triples (x,y,z), evaluated on the device. */
int iblgf_lgf_get(iblgf_ctx* ctx, const int* coords, size_t n, double* host_out);
/* LGF_GE::get (lgf_ge.hpp:95-110): E(n; alpha) = f|n1| f|n2| f|n3| with
 * f_k = e^{-2 alpha} I_k(2 alpha), for n host coordinate triples, evaluated on
 * the device from the context's table of this alpha. */
int iblgf_lgf_ge_get(iblgf_ctx* ctx, double alpha, const int* coords, size_t n, double* host_out);

/* ---- IF-HERK time step (Ifherk::time_step, ifherk.hpp:1078-1200, with the
 * time_march loop's T += dt) -------------------------------------------------
 * Advances the face velocity (three component fields u_fields[0..2], x/y/z
 * normal components) by n_steps steps of size dt at Reynolds number Re and
 * writes the pressure of the last step into p_field; *T is the simulation time
 * (in/out). The immersed boundary and the frame velocity come from
 * iblgf_ib_set_points / iblgf_ns_options. A step whose time is far enough past
 * the last velocity refresh ((T - T_last) 3.3 / (Re dx_base^2) > 7, T_last = 0
 * initially, per context) first rebuilds u from its vorticity through the
 * base-level stream function and runs the alpha = 0 correction step
 * (pad_velocity + adapt_corr_time_step, ifherk.hpp:1093-1111, 1206-1303,
 * 1522-1573). Not covered: adaptation, body force, moving bodies (boundary
 * velocity 0). */
int iblgf_ns_step(iblgf_ctx* ctx, const int* u_fields, int p_field, double dt, double Re, double* T,
                  int n_steps);
/* Constant frame velocity (frame_vel[3], subtracted from the convecting
 * velocity as add_field_expression(frame_vel, -1) in Ifherk::nonlinear,
 * ifherk.hpp:1667-1668; NULL = 0) and the IB CG settings (cg_threshold,
 * cg_max_itr; defaults 1e-3, 40). With IB points set (iblgf_ib_set_points)
 * each stage of iblgf_ns_step runs lin_sys_with_ib_solve with the IB
 * (ifherk.hpp:1451-1517), warm-started from that stage's previous force. */
int iblgf_ns_options(iblgf_ctx* ctx, const double* frame_vel, double cg_threshold, int cg_max_iter);
/* ---- Mesh adaptation (Ifherk::adapt, ifherk.hpp:1018-1076, with the server
 * side of Domain::adapt, decomposition.hpp:182-470) ------------------------
 * attempts: n_attempts (key, level change) pairs for octants with data, the
 * output of an adapt condition (for example the one of tests/ns_amr_lgf,
 * ns_amr_lgf.hpp:402-489, built on iblgf_block_norms): +1 refine (if the 2:1
 * balance allows it, or the octant is an IB block), -1 delete; correction
 * blocks that no physical block needs are deleted, base blocks within two
 * blocks of a kept base block are added (*base_mesh_update = 1 then, and the
 * next iblgf_ns_step refreshes the velocity). Every field keeps its values on
 * the octants that stay and is zero on new ones; the n_interp listed fields
 * (interp_fields: 3 ids per entry, the first used for mesh 0 = cell, all
 * three for 1 = face / 2 = edge) are interpolated from each parent of a new
 * leaf above the base level into all its children (nli_intrp_node,
 * cell_center_nli_intrp.hpp:310-420). Octant indices change: query keys,
 * levels and flags again (iblgf_domain_info, iblgf_domain_octants). IB points stay attached. */
int iblgf_adapt(iblgf_ctx* ctx, int n_attempts, const uint64_t* keys, const int* level_change, int n_interp,
                const int* interp_fields, const int* interp_mesh, int* base_mesh_update);
/* The IF-HERK step's scratch fields that the adapt condition reads: ids[0]
 * cell_aux, ids[1..3] edge_aux (vorticity components), ids[4] the Poisson
 * solver's correction_tmp. Their values are those of the last step. */
int iblgf_ns_fields(iblgf_ctx* ctx, int* ids);
/* Ifherk::clean (ifherk.hpp:1309-1352): zero the field, or with
 * non_leaf_only every non-leaf block and the outer `width` planes of leaves. */
int iblgf_ns_clean(iblgf_ctx* ctx, int field, int non_leaf_only, int width);
/* Ifherk::clean_leaf_correction_boundary (ifherk.hpp:1355-1411) of a field of
 * n = 1..3 components at `level`: with leaf_only_boundary, correction (and, for
 * the step after an adaptation, former base-level correction) blocks are
 * zeroed; at the base level every block next to a missing (or correction)
 * neighbour is tapered towards it (smooth2zero, once per component). */
int iblgf_ns_clean_leaf_correction_boundary(iblgf_ctx* ctx, const int* fields, int n, int level,
                                            int leaf_only_boundary);
/* Operator::maxnorm and blockRootMeanSquare (operators.hpp:1149-1211) of the
 * vector (n_comp = 1..3 component fields) over each octant's interior nodes:
 * max_out[o] = max |v|, rms_out[o] = sqrt(mean |v|^2), n_octants each. */
int iblgf_block_norms(iblgf_ctx* ctx, const int* fields, int n_comp, double* max_out, double* rms_out);

/* IB force (IB::force_prev, n x 3) and CG iteration count of the last
 * step's stage 1, 2 or 3; either output may be NULL */
int iblgf_ib_force(iblgf_ctx* ctx, int stage, double* out, int* iters);
/* CG iteration count of the last solve of stage 1, 2 or 3 and whether it
 * converged (0: it stopped at cg_max_iter, where the reference's CG_solve,
 * linsys.hpp:202-229, stops silently); no counterpart in the reference.
 * Synchronises the context stream. Either output may be NULL. */
int iblgf_ib_stage_status(iblgf_ctx* ctx, int stage, int* iters, int* converged);

/* ---- immersed boundary (ib.hpp, linsys.hpp) ------------------------------
 * iblgf_ib_set_points: the IB points (n x 3 coordinates, the reference's
 * IB::coordinates_) on the finest mesh level, with IB::init's delta radius
 * 4.5 and safety distance 5 / (Re dx_ib) + 1; marks IB / extended-IB blocks
 * (ServerBase::update_ib_flag, server.hpp:544-576), builds the IB2xIB /
 * xIB2IB / IB2AMR masks (fmm.hpp:70-190) and the influence lists and yang3
 * delta weights (client.hpp:1262-1320). iblgf_ib_flags: per octant bit0
 * is_ib, bit1 is_extended_ib. iblgf_ib_solve: LinSysSolver::ib_solve +
 * CG_solve (linsys.hpp:113-230) for the face velocity u_fields[0..2] (a body
 * at rest in the frame); force (n x 3) is the initial guess in and the IB
 * force out, iters the CG iteration count. The CG runs on the device (FP64
 * iterates and dot products); a solve that stops at max_iter without
 * converging writes force and iters and returns IBLGF_ENOTCONVERGED. */
int iblgf_ib_set_points(iblgf_ctx* ctx, int n, const double* coords, double Re);
int iblgf_ib_flags(iblgf_ctx* ctx, int* flags);
int iblgf_ib_solve(iblgf_ctx* ctx, const int* u_fields, double alpha, double threshold, int max_iter,
                   double* force, int* iters);

/* ---- learned warm start of the IB force CG (no reference counterpart: the
 * reference warm-starts from IB::force_prev, ifherk.hpp:1476) -------------
 * mode 0: previous step's force of the stage (the reference). mode 2: its
 * linear extrapolation 2 f_prev - f_prev2 once the stage has two forces.
 * mode 1 (learned): until trained, mode 0; from the second step on, the next
 * train_steps steps record per stage (change of the CG right-hand side since
 * the previous step, previous force, its last change; target: the converged
 * force minus the previous force); a 1-D convolutional network over the IB
 * points in Morton order of their coordinates (9 -> 64 -> 64 -> 3 channels,
 * kernel 5, 24 451 FP32 parameters, seeded initialisation; inputs and target
 * scaled per stage) is then trained on them (full-batch Adam, `epochs`
 * steps, learning rate lr, on the device) and from then on predicts the
 * initial guess previous force + correction; CG runs to the unchanged
 * tolerance. Modes 0 and 2 stay on the device (time steps can be captured
 * as CUDA graphs); mode 1 assembles the network's inputs on the host.
 * iblgf_ib_warmstart_info: [mode, trained, samples, first loss, last loss,
 * parameters]. iblgf_ws_check: one forward + backward pass of the network
 * for given parameters (layout W1 b1 W2 b2 W3 b3), inputs [S][9][N] and
 * targets [S][3][N]; outputs [S][3][N], gradients and the mean squared loss. */
int iblgf_ib_warmstart(iblgf_ctx* ctx, int mode, int train_steps, int epochs, double lr, unsigned seed);
int iblgf_ib_warmstart_info(iblgf_ctx* ctx, double* info);
int iblgf_ws_check(iblgf_ctx* ctx, int n_samples, int n_points, const float* params, const float* inputs,
                   const float* targets, float* outputs, float* grads, float* loss);

/* ---- batches of independent problems -----------------------------------
 * Many unbounded Poisson problems of uneven size solved together: each is
 * PoissonSolver::apply_lgf (poisson.hpp:587-894) on its own octree
 * (Domain::construct_basemesh_blocks / init_refine, domain.hpp:405-488,
 * 878-939), while every stage of a sweep (anterpolation per level, forward
 * transforms, spectral MAC, inverse transforms, interpolation) runs as one
 * launch over all problems. A context becomes a batch with its first
 * iblgf_batch_add_problem (instead of iblgf_domain_add_blocks); all problems
 * share the context's block_extent, dx_base and precision, and each has its
 * own bounding box (bd_base / bd_extent), block boxes and refinement.
 * Fields (iblgf_field_*) of a batch hold the problems' octants back to back:
 * problem p occupies octants [info[0], info[0] + info[1]) of
 * iblgf_batch_problem_info, in that problem's canonical order. */
int iblgf_batch_add_problem(iblgf_ctx* ctx, const int* bd_base, const int* bd_extent, int n_boxes,
                            const int* base, const int* extent, int n_ref, iblgf_refine_fn pred, void* user,
                            int* problem);
int iblgf_batch_finalize(iblgf_ctx* ctx, int subtract_non_leaf);
/* info[0] first octant in the batch, [1] octants, [2] base level, [3] depth */
int iblgf_batch_problem_info(iblgf_ctx* ctx, int problem, int* info);
int iblgf_batch_problem_octants(iblgf_ctx* ctx, int problem, uint64_t* keys, int* levels, int* flags,
                                int* bbase);
/* apply_lgf of every problem (AMR2AMR mask) from field src into field tgt */
int iblgf_batch_apply_lgf(iblgf_ctx* ctx, int src, int tgt);

/* ---- single-block convolution (fft::Convolution, convolution.hpp:141-328)
 * out (Nb^3, device) += scale * window [Nb-1, 2Nb-2]^3 of the linear
 * convolution of src (Nb^3, device) with kernel (P^3, device, P = 2Nb-1).
 * Nb must equal the context's block size. */
int iblgf_conv_block(iblgf_ctx* ctx, const double* src, const double* kernel, double* out,
                     double scale);
/* Same result as iblgf_conv_block, but the call allocates no device memory:
 * its temporaries live in a 2 MiB static device array (1.41 MB used at
 * Nb = 18); a block needing more is rejected with IBLGF_EINVAL. For hosts
 * that must not allocate at call time (device memory already reserved for
 * their own pool, or no device-wide synchronisation from cudaFree allowed).
 * Enqueues on the context stream and returns without synchronising. The
 * scratch is shared by all contexts on a device: calls overlapping in time on
 * different streams race. The first call on a device runs a one-time set-up;
 * make it before any stream capture. No reference counterpart: the
 * reference's fft::Convolution owns FFTW buffers allocated at construction. */
int iblgf_conv_block_noalloc(iblgf_ctx* ctx, const double* src, const double* kernel, double* out,
                             double scale);

/* ---- timing / introspection ------------------------------------------- */
/* Number of kernels this library launched on the context stream so far. */
int iblgf_kernel_launches(iblgf_ctx* ctx, long long* count);
/* Phase timing by CUDA events on the context stream (no host sync while
 * enabled). iblgf_profile(ctx, 1) resets and enables; iblgf_profile_read
 * returns the summed device milliseconds since then: [0] forward transforms,
 * [1] spectral MAC, [2] inverse transforms + interpolation + add,
 * [3] zero / copy / anterpolation. */
int iblgf_profile(iblgf_ctx* ctx, int enable);
int iblgf_profile_read(iblgf_ctx* ctx, double* out4);
/* Work counters since the last iblgf_profile call: [0] FMM sweeps,
 * [1] source blocks transformed, [2] target blocks, [3] (target, source)
 * pairs, [4] distinct LGF spectra used per sweep (summed), [5] anterpolation
 * block transfers, [6] interpolation block transfers, [7] targets handled by
 * the sibling-group MAC (the rest use the general pair-list MAC). */
int iblgf_stats(iblgf_ctx* ctx, long long* out8);

/* The first n (1 <= n <= 10) counters: [0]-[7] as iblgf_stats, then [8] the
 * (target, source) spectral products the sibling-group MAC covers: a group
 * covers all 64 (child, candidate) products of every neighbour parent that
 * has a candidate, so [8] >= [3]; and [9] the floating-point operations the
 * MAC kernels execute per spectrum frequency (the block-Toeplitz group
 * kernel forms the 64 products of a parent with 27 complex multiplies).
 * IBLGF_EINVAL for n outside [1, 10]. */
int iblgf_stats_n(iblgf_ctx* ctx, long long* out, int n);

/* Sibling-group MAC autotuning (no reference counterpart). On the first
 * sweep of each plan the library times every applicable variant of the
 * group MAC on that sweep's data (0: direct kernel, 64 frequencies x 768
 * threads in FP32 / 32 x 512 in FP64; 1: direct kernel, 32 x 512 / 32 x 256;
 * 2: block-Toeplitz kernel with TMA-staged coefficients, FP32 only; 3:
 * tensor-core kernel, tcgen05 TF32 MMAs with a 3-product split and FP32
 * accumulation in tensor memory, FP32 only) and keeps the fastest.
 * iblgf_mac_variant pins a variant for later plans and sweeps (-1:
 * autotune; a pinned variant that does not apply to a plan runs variant 0).
 * iblgf_mac_tuning returns one row of 8 doubles per tuned plan: level, mask
 * index, targets, ms of variants 0, 1, 2, 3 (-1: not applicable), chosen
 * variant; n_rows receives the number of rows. */
int iblgf_mac_variant(iblgf_ctx* ctx, int variant);
/* Integrating-factor sweeps (neighbour-only, LGF_GE; fmm.hpp:754-770) whose
 * 1-D factor e^{-2a} I_m(2a) is below 2^-56 of its centre value for every
 * m > R, R in {4, 6, 8} (the smallest that holds), run as direct separable
 * sums over the 27 neighbour blocks instead of block FFT convolutions: the
 * same sums up to terms below FP64 rounding (default on). iblgf_ge_direct(ctx, 0) selects the transform path for all
 * of them. */
int iblgf_ge_direct(iblgf_ctx* ctx, int enable);
int iblgf_mac_tuning(iblgf_ctx* ctx, double* out, int max_rows, int* n_rows);
/* Measures the device's FMA throughput (TFLOP/s, 2 flops per FMA) for
 * IBLGF_FP64 or IBLGF_FP32 with a register-resident FMA chain kernel; the
 * roofline denominator of the CUDA-core kernels. */
int iblgf_fma_peak(iblgf_ctx* ctx, int precision, double* tflops);
/* Measures SM clocks per tensor-core MMA (tcgen05.mma kind::tf32, M = 128,
 * K = 8, the given N in {16, 32, 64, 128, 256}), issued back to back by one
 * thread per SM: the issue-rate bound of the tensor-core MAC (variant 3),
 * whose products have N = 16. IBLGF_EINVAL for another N. */
int iblgf_tc_mma_rate(iblgf_ctx* ctx, int n, double* clocks);

/* Failure detection (no reference counterpart: the reference ignores most
 * CUDA return codes and stops CG silently).
 * iblgf_wait_selftest runs the library's bounded mbarrier wait on a barrier
 * nothing arrives on, for `polls` polls (1 .. 2^22), and returns what a
 * kernel whose wait ran out returns: IBLGF_ETIMEOUT, the status word read
 * and cleared; the context stays usable.
 * iblgf_field_first_nonfinite sets *index to the smallest element index
 * (octant-major, x fastest) of a NaN or infinite value in field f, or -1.
 * iblgf_debug_fail_alloc arms a process-wide fault injector: the
 * (after + 1)-th device allocation of the library from now on fails with
 * IBLGF_ENOMEM without calling the allocator (then it disarms); -1 disarms.
 * The failing call returns IBLGF_ENOMEM and its context stays destroyable. */
int iblgf_wait_selftest(iblgf_ctx* ctx, long long polls);

/* Two-dimensional Helmholtz lattice Green's function, the kernel of the
 * Fourier-in-z solvers (one per z mode; lgf::Helmholtz<2>::get,
 * include/iblgf/lgf/helmholtz.hpp:152-163, Helmholtz_Lookup
 * helmholtz_lookup.hpp:45-176): get(n, m) = G_c(n, m) - origin(c), the
 * decaying solution of the five-point equation (Delta_h - c^2) g = delta;
 * c = 0 gives mode 0's kernel, the 2-D LGF of the five-point Laplacian
 * (LGF_GL<2>::get at level difference 0, lgf_gl.hpp:93-99: the regularised
 * G0 with G0(0, 0) = 0, log r / (2 pi) + 0.2573... far away).
 * iblgf_helm2d_origin: origin_val(c) (c > 0).
 * iblgf_helm2d_lgf: host_out[m * nx + n] = get(n, m), 0 <= n < nx, 0 <= m < ny.
 * iblgf_helm2d_get: host_out[i] = get(host_nm[2i], host_nm[2i + 1]) for n
 * offsets (Helmholtz<2>::get(coordinate) and get(N, M), helmholtz.hpp:161-176,
 * with c the level's c_level).
 * iblgf_helm2d_apply: host_u += scale * sum_j get(i - j) host_f[j] over a
 * uniform nx x ny cell grid (x fastest; every pair, the exact unbounded
 * solution of (Delta_h - c^2) u = f on that support); nx <= 6144, ny <= 65535.
 * Tables hold at most 2^28 entries.
 * The 2-D quadtree FMM that applies the kernel on an adaptive mesh is not
 * part of this library. */
int iblgf_helm2d_origin(double c, double* out);
int iblgf_helm2d_lgf(iblgf_ctx* ctx, double c, int nx, int ny, double* host_out);
int iblgf_helm2d_get(iblgf_ctx* ctx, double c, int n, const int* host_nm, double* host_out);
int iblgf_helm2d_apply(iblgf_ctx* ctx, double c, int nx, int ny, const double* host_f, double* host_u, double scale);
/* Complex Helmholtz (Fourier-in-z) block operators on 2-D blocks
 * (domain::Operator::laplace_helmholtz_complex, gradient_, divergence_,
 * curl_, curl_transpose_helmholtz_complex; operators.hpp:1516-1545,
 * 1585-1614, 1763-1795, 1972-2008, 2178-2217). op: 0 laplace (cell ->
 * cell), 1 gradient (cell -> face), 2 divergence (face -> cell), 3 curl
 * (face -> edge), 4 curl_transpose (edge -> face, times scale). Device
 * arrays of n_blocks blocks, each [component][nb][nb] (x fastest): scalar
 * fields 2 n_modes components (mode i: real 2i, imaginary 2i+1), vector
 * fields three groups of those (x, y, z); the z derivative of mode i is
 * i omega_i, omega_i = 2 pi i / lz. Interior nodes are written, buffers read. */
int iblgf_helm2d_op(iblgf_ctx* ctx, int op, int nb, int n_blocks, int n_modes, double dx_level, double lz,
                    double scale, const double* dev_src, double* dev_dst);
/* The same operators restricted to a set of z modes: mode_mask[i] != 0
 * selects mode i (n_modes bytes; NULL selects all); the components of the
 * other modes are left as they were. Replaces the single-mode forms
 * (laplace_/gradient_/divergence_/curl_/curl_transpose_helmholtz_complex_oneMode,
 * operators.hpp:1548, 1620, 1801, 2017, 2224: one mode selected), the
 * refined forms (gradient_/divergence_/curl_helmholtz_complex_refined,
 * :1653, 1839, 2125: the first n_modes / 2^r modes) and the ModesBool forms
 * (divergence_helmholtz_complex(..., ModesBool), _Modes, :1889, 1931).
 * n_modes <= 2048. */
int iblgf_helm2d_op_modes(iblgf_ctx* ctx, int op, int nb, int n_blocks, int n_modes, const unsigned char* mode_mask,
                          double dx_level, double lz, double scale, const double* dev_src, double* dev_dst);
/* The convective term on the z collocation planes of the Fourier-in-z
 * solver (domain::Operator::nonlinear_helmholtz, operators.hpp:2627-2766;
 * _oneMode :2776-2831 and _refined :2840-2895 through plane_mask). dev_face
 * (velocity, faces), dev_edge (vorticity, edges), dev_dst (faces): n_blocks
 * blocks of [3 n_planes][nb][nb] (x fastest; groups x, y, z, one component
 * per z plane). plane_mask[i] != 0 selects plane i (NULL: all; the single-mode
 * form selects planes mode P .. mode P + P - 1 for P planes per mode, the
 * refined form every 2^r-th plane); interior nodes of the selected planes are
 * written. n_planes <= 2048. */
int iblgf_helm2d_nonlinear(iblgf_ctx* ctx, int nb, int n_blocks, int n_planes, const unsigned char* plane_mask,
                           const double* dev_face, const double* dev_edge, double* dev_dst);
/* Real-valued block operators of the same family on 2-D blocks. Device
 * fields of n_blocks blocks, [components][nb][nb] (x fastest), with the
 * component counts given (an operator reads or writes the leading ones);
 * interior nodes written. op:
 *  0 curl_helmholtz (operators.hpp:2305-2414): dev_a face, dev_d edge, each
 *    3 n_planes components (groups x, y, z, a component per z plane); the
 *    in-plane differences over dx_level, the z difference of plane i with
 *    plane i - 1 (plane 0 with n_planes - 1) over dx_fine;
 *  1 curl_helmholtz_real (:2059-2081): face (2) -> edge (3), edge x, y zero;
 *  2 curl_helmholtz_real with Uz (:2083-2119): face (2) and the scalar dev_b
 *    (1) -> edge (3);
 *  3 curl_transpose_helmholtz_complex_linear (:2272-2303): edge (3) -> face
 *    x, y (dev_d, 2) and face z (dev_e, 1), times scale, with the c terms;
 *  4 nonlinear_linear_helm (:2534-2572): face dev_a (2), edge dev_b (3) ->
 *    dev_d (2) and dev_e (1);
 *  5 curl_transpose, 2-D branch (:2416-2453): edge scalar (1) -> face (2),
 *    times scale.
 * dx_fine is read by op 0 only, c by op 3 only, scale by ops 3 and 5. */
int iblgf_helm2d_real_op(iblgf_ctx* ctx, int op, int nb, int n_blocks, int n_planes, double dx_level, double dx_fine,
                         double c, double scale, const double* dev_a, int a_comp, const double* dev_b, int b_comp,
                         double* dev_d, int d_comp, double* dev_e);
int iblgf_field_first_nonfinite(iblgf_ctx* ctx, int f, long long* index);
int iblgf_debug_fail_alloc(long long after);

#ifdef __cplusplus
}
#endif
#endif /* IBLGF_B200_H */
