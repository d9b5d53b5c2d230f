"""Python binding of libiblgf_b200.so (the C ABI in include/iblgf_b200.h).

Host-side mirror of the reference's solver surface for scripts and tests:
`Domain` (Domain::initialize + init_refine + distribute), `Solver.fmm_apply`
(Fmm::apply) and `Solver.apply_lgf` (PoissonSolver::apply_lgf). All compute
runs in the CUDA library; there is no CPU path. Loading fails loudly if the
library has not been built (`make -C iblgf-amr_b200`).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libiblgf_b200.so")

FP64, FP32 = 0, 1
STREAM, AMR2AMR = 0, 1

REFINE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                             ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int)
# exchange(user, device_buffer, count, stream) -> 0: sum the buffer over the ranks
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p)


class Config(ctypes.Structure):
    _fields_ = [("block_extent", ctypes.c_int), ("bd_base", ctypes.c_int * 3),
                ("bd_extent", ctypes.c_int * 3), ("dx_base", ctypes.c_double),
                ("precision", ctypes.c_int), ("device", ctypes.c_int),
                ("intrp_order", ctypes.c_int), ("stream", ctypes.c_void_p)]


EXPORTS = [
    "iblgf_create", "iblgf_destroy", "iblgf_last_error", "iblgf_synchronize",
    "iblgf_domain_add_blocks", "iblgf_domain_import", "iblgf_domain_restart", "iblgf_domain_init_refine", "iblgf_domain_finalize",
    "iblgf_domain_info", "iblgf_domain_octants", "iblgf_domain_lists", "iblgf_domain_masks",
    "iblgf_field_create", "iblgf_field_zero", "iblgf_field_upload", "iblgf_field_download",
    "iblgf_field_upload_leaves", "iblgf_field_download_leaves", "iblgf_field_download_leaves_async",
    "iblgf_field_device_ptr", "iblgf_fmm_apply", "iblgf_poisson_apply_lgf", "iblgf_poisson_apply_if",
    "iblgf_poisson_options", "iblgf_op_apply", "iblgf_buffer_exchange", "iblgf_lgf_table", "iblgf_lgf_get",
    "iblgf_ns_step", "iblgf_batch_add_problem", "iblgf_batch_finalize", "iblgf_batch_problem_info",
    "iblgf_batch_problem_octants", "iblgf_batch_apply_lgf", "iblgf_ib_set_points", "iblgf_ib_flags",
    "iblgf_ib_solve", "iblgf_ns_options", "iblgf_ib_force", "iblgf_ib_stage_status", "iblgf_ib_warmstart",
    "iblgf_ib_warmstart_info",
    "iblgf_ws_check", "iblgf_conv_block", "iblgf_conv_block_noalloc",
    "iblgf_kernel_launches", "iblgf_profile", "iblgf_profile_read", "iblgf_stats", "iblgf_stats_n", "iblgf_adapt", "iblgf_block_norms", "iblgf_ns_fields", "iblgf_ns_clean",
    "iblgf_ns_clean_leaf_correction_boundary",
    "iblgf_fma_peak", "iblgf_tc_mma_rate", "iblgf_helm2d_origin", "iblgf_helm2d_lgf", "iblgf_helm2d_get", "iblgf_helm2d_apply", "iblgf_helm2d_op", "iblgf_helm2d_op_modes", "iblgf_helm2d_nonlinear", "iblgf_helm2d_real_op", "iblgf_ge_direct", "iblgf_field_upload_leaves_async", "iblgf_wait_selftest", "iblgf_field_first_nonfinite",
    "iblgf_debug_fail_alloc", "iblgf_mac_variant", "iblgf_mac_tuning", "iblgf_domain_partition", "iblgf_domain_set_owner",
    "iblgf_fmm_apply_kernel", "iblgf_lgf_ge_get", "iblgf_op_apply_octants", "iblgf_field_upload_octants",
    "iblgf_field_download_octants",
]

_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libiblgf_b200.so is not built; run `make -C %s`" % HERE)
    L = ctypes.CDLL(LIB_PATH)
    vp, ci, cd, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_size_t
    pp = ctypes.POINTER(ctypes.c_void_p)
    L.iblgf_create.argtypes = [ctypes.POINTER(Config), pp]
    L.iblgf_destroy.argtypes = [vp]
    L.iblgf_last_error.argtypes = [vp]
    L.iblgf_last_error.restype = ctypes.c_char_p
    L.iblgf_synchronize.argtypes = [vp]
    L.iblgf_domain_add_blocks.argtypes = [vp, ci, vp, vp]
    L.iblgf_domain_init_refine.argtypes = [vp, ci, ci, REFINE_FN, vp]
    L.iblgf_domain_import.argtypes = [vp, ci, vp, vp]
    L.iblgf_domain_restart.argtypes = [vp, ci, vp, vp]
    L.iblgf_domain_finalize.argtypes = [vp, ci]
    L.iblgf_domain_info.argtypes = [vp, vp, vp, vp]
    L.iblgf_domain_octants.argtypes = [vp, vp, vp, vp, vp]
    L.iblgf_domain_lists.argtypes = [vp, vp, vp, vp]
    L.iblgf_domain_masks.argtypes = [vp, ci, vp]
    L.iblgf_field_create.argtypes = [vp, vp]
    L.iblgf_field_zero.argtypes = [vp, ci]
    L.iblgf_field_upload.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_download.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_upload_leaves.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_download_leaves.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_download_leaves_async.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_upload_leaves_async.argtypes = [vp, ci, vp, sz]
    L.iblgf_field_device_ptr.argtypes = [vp, ci, pp]
    L.iblgf_fmm_apply.argtypes = [vp, ci, ci, ci, ci, cd, ci]
    L.iblgf_poisson_apply_lgf.argtypes = [vp, ci, ci, ci]
    L.iblgf_poisson_options.argtypes = [vp, ci, ci]
    L.iblgf_poisson_apply_if.argtypes = [vp, ci, ci, cd, ci]
    L.iblgf_lgf_table.argtypes = [vp, vp, sz]
    L.iblgf_op_apply.argtypes = [vp, ci, vp, ci, vp, ci, ci, cd]
    L.iblgf_buffer_exchange.argtypes = [vp, ci, ci]
    L.iblgf_lgf_get.argtypes = [vp, vp, sz, vp]
    L.iblgf_conv_block.argtypes = [vp, vp, vp, vp, cd]
    L.iblgf_ns_step.argtypes = [vp, vp, ci, cd, cd, vp, ci]
    L.iblgf_batch_add_problem.argtypes = [vp, vp, vp, ci, vp, vp, ci, REFINE_FN, vp, vp]
    L.iblgf_batch_finalize.argtypes = [vp, ci]
    L.iblgf_batch_problem_info.argtypes = [vp, ci, vp]
    L.iblgf_batch_problem_octants.argtypes = [vp, ci, vp, vp, vp, vp]
    L.iblgf_batch_apply_lgf.argtypes = [vp, ci, ci]
    L.iblgf_ib_set_points.argtypes = [vp, ci, vp, cd]
    L.iblgf_ib_flags.argtypes = [vp, vp]
    L.iblgf_ib_solve.argtypes = [vp, vp, cd, cd, ci, vp, vp]
    L.iblgf_ns_options.argtypes = [vp, vp, cd, ci]
    L.iblgf_ib_force.argtypes = [vp, ci, vp, vp]
    L.iblgf_ib_stage_status.argtypes = [vp, ci, vp, vp]
    L.iblgf_mac_variant.argtypes = [vp, ci]
    L.iblgf_domain_partition.argtypes = [vp, ci, vp]
    L.iblgf_domain_set_owner.argtypes = [vp, vp, ci, EXCHANGE_FN, vp]
    L.iblgf_mac_tuning.argtypes = [vp, vp, ci, vp]
    L.iblgf_ib_warmstart.argtypes = [vp, ci, ci, ci, cd, ctypes.c_uint]
    L.iblgf_ib_warmstart_info.argtypes = [vp, vp]
    L.iblgf_ws_check.argtypes = [vp, ci, ci, vp, vp, vp, vp, vp, vp]
    L.iblgf_conv_block_noalloc.argtypes = [vp, vp, vp, vp, cd]
    L.iblgf_kernel_launches.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.iblgf_profile.argtypes = [vp, ci]
    L.iblgf_profile_read.argtypes = [vp, vp]
    L.iblgf_stats.argtypes = [vp, vp]
    L.iblgf_stats_n.argtypes = [vp, vp, ci]
    L.iblgf_adapt.argtypes = [vp, ci, vp, vp, ci, vp, vp, vp]
    L.iblgf_ns_fields.argtypes = [vp, vp]
    L.iblgf_ns_clean.argtypes = [vp, ci, ci, ci]
    L.iblgf_ns_clean_leaf_correction_boundary.argtypes = [vp, vp, ci, ci, ci]
    L.iblgf_block_norms.argtypes = [vp, vp, ci, vp, vp]
    L.iblgf_fma_peak.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_double)]
    L.iblgf_tc_mma_rate.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_double)]
    L.iblgf_helm2d_origin.argtypes = [cd, ctypes.POINTER(ctypes.c_double)]
    L.iblgf_helm2d_lgf.argtypes = [vp, cd, ci, ci, vp]
    L.iblgf_helm2d_get.argtypes = [vp, cd, ci, vp, vp]
    L.iblgf_helm2d_apply.argtypes = [vp, cd, ci, ci, vp, vp, cd]
    L.iblgf_helm2d_op.argtypes = [vp, ci, ci, ci, ci, cd, cd, cd, vp, vp]
    L.iblgf_helm2d_op_modes.argtypes = [vp, ci, ci, ci, ci, vp, cd, cd, cd, vp, vp]
    L.iblgf_helm2d_nonlinear.argtypes = [vp, ci, ci, ci, vp, vp, vp, vp]
    L.iblgf_helm2d_real_op.argtypes = [vp, ci, ci, ci, ci, cd, cd, cd, cd, vp, ci, vp, ci, vp, ci, vp]
    L.iblgf_ge_direct.argtypes = [vp, ci]
    L.iblgf_wait_selftest.argtypes = [vp, ctypes.c_longlong]
    L.iblgf_field_first_nonfinite.argtypes = [vp, ci, ctypes.POINTER(ctypes.c_longlong)]
    L.iblgf_debug_fail_alloc.argtypes = [ctypes.c_longlong]
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# status codes (include/iblgf_b200.h)
EINVAL, ECUDA, ENOMEM, ETIMEOUT, EINTERNAL, ENOTCONVERGED = 1, 2, 3, 4, 5, 6


def debug_fail_alloc(after):
    """Arm the library's fault injector: the (after + 1)-th device
    allocation from now fails with ENOMEM (-1 disarms)."""
    rc = lib().iblgf_debug_fail_alloc(int(after))
    if rc != 0:
        raise IblgfError("iblgf_debug_fail_alloc: bad argument", rc)


class IblgfError(RuntimeError):
    """A library call failed; `code` is its status (IBLGF_E*)."""

    def __init__(self, msg, code=None):
        super().__init__(msg)
        self.code = code


class IblgfNotConverged(IblgfError):
    """An iterative solve stopped at its iteration limit; the outputs
    (force, iterations) are attached."""


def write_tree(path, keys, levels, flags):
    """Tree::write (tree.hpp:832-855): the key of every octant with data but
    the root (level 0) in depth-first order, 8 bytes each, then their leaf
    flags, one byte each. Depth-first order with children 0..7 is ascending
    key order: the coordinate bits sit above the level bits."""
    keys = np.asarray(keys, np.uint64)
    sel = np.nonzero(np.asarray(levels) > 0)[0]
    order = sel[np.argsort(keys[sel], kind="stable")]
    with open(path, "wb") as f:
        f.write(keys[order].astype("<u8").tobytes())
        f.write(((np.asarray(flags)[order] & 1) != 0).astype(np.uint8).tobytes())


def read_tree(path):
    """Tree::read (tree.hpp:857-885): (keys, leaf flags) of a tree file."""
    b = open(path, "rb").read()
    n = len(b) // 9
    keys = np.frombuffer(b, "<u8", n).astype(np.uint64)
    leaf = np.frombuffer(b, np.uint8, n, 8 * n).copy()
    return keys, leaf


def read_restart_info(path):
    """The `key = value;` lines of Ifherk::write_info (ifherk.hpp:961-983)."""
    out = {}
    for line in open(path):
        line = line.strip().rstrip(";")
        if "=" in line:
            k, v = (x.strip() for x in line.split("=", 1))
            out[k] = float(v)
    return out


class Solver:
    """Domain + LGF-FMM Poisson solver on one GPU.

    Mirrors the reference set-up sequence: Domain(dictionary) ->
    init_refine(nLevels, global_refinement) -> distribute<FmmMaskBuilder>() ->
    PoissonSolver(simulation). `predicate(base, extent, refinement_level,
    diff_level)` plays the role of Domain::register_refinement_condition().
    """

    def __init__(self, bd_base, bd_extent, block_extent, dx_base, blocks, n_levels=0,
                 global_refinement=0, predicate=None, precision=FP64, subtract_non_leaf=False,
                 intrp_order=5, device=0, stream=None, use_correction=True, import_octants=None,
                 restart_tree=None):
        L = lib()
        cfg = Config(block_extent, (ctypes.c_int * 3)(*bd_base), (ctypes.c_int * 3)(*bd_extent),
                     float(dx_base), int(precision), int(device), int(intrp_order),
                     ctypes.c_void_p(stream) if stream else None)
        h = ctypes.c_void_p()
        rc = L.iblgf_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise IblgfError("iblgf_create failed (%d): %s" % (rc, L.iblgf_last_error(None).decode()), rc)
        self._destroy = L.iblgf_destroy  # kept so that close() works during interpreter shutdown
        self.h = h
        self._async_out = []  # host buffers of asynchronous downloads in flight
        self.Nb = block_extent + 2
        self.block_extent = block_extent
        self.precision = precision
        self.dx_base = float(dx_base)
        if restart_tree is not None:
            keys, leaf = read_tree(restart_tree) if isinstance(restart_tree, str) else restart_tree
            keys = np.ascontiguousarray(keys, dtype=np.uint64)
            leaf = np.ascontiguousarray(leaf, dtype=np.uint8)
            self._check(L.iblgf_domain_restart(self.h, len(keys), _p(keys), _p(leaf)))
            n_levels, global_refinement, predicate = 0, 0, None
            self._imported = True
        elif import_octants is not None:
            keys = np.ascontiguousarray(import_octants[0], dtype=np.uint64)
            flags = np.ascontiguousarray(import_octants[1], dtype=np.int32)
            self._check(L.iblgf_domain_import(self.h, len(keys), _p(keys), _p(flags)))
            n_levels, global_refinement, predicate = 0, 0, None
            self._imported = True
        else:
            bb = np.array([b[0] for b in blocks], np.int32).ravel()
            be = np.array([b[1] for b in blocks], np.int32).ravel()
            self._check(L.iblgf_domain_add_blocks(self.h, len(blocks), _p(bb), _p(be)))
            self._imported = False
        if predicate is not None:
            def cb(user, base, ext, rl, diff):
                return 1 if predicate((base[0], base[1], base[2]), (ext[0], ext[1], ext[2]), rl, diff) else 0
            self._cb = REFINE_FN(cb)
        else:
            self._cb = REFINE_FN(lambda *a: 0)
        if not self._imported:
            self._check(L.iblgf_domain_init_refine(self.h, int(n_levels), int(global_refinement), self._cb, None))
        self._check(L.iblgf_domain_finalize(self.h, 1 if subtract_non_leaf else 0))
        self._check(L.iblgf_poisson_options(self.h, 1 if use_correction else 0, 1 if subtract_non_leaf else 0))
        self._load_octants()

    def _load_octants(self):
        L = lib()
        bl, dp, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(L.iblgf_domain_info(self.h, ctypes.byref(bl), ctypes.byref(dp), ctypes.byref(n)))
        self.base_level, self.depth, self.n = bl.value, dp.value, n.value
        self.keys = np.zeros(self.n, np.uint64)
        self.levels = np.zeros(self.n, np.int32)
        self.flags = np.zeros(self.n, np.int32)
        self.bbase = np.zeros((self.n, 3), np.int32)
        self._check(L.iblgf_domain_octants(self.h, _p(self.keys), _p(self.levels), _p(self.flags), _p(self.bbase)))

    # ------------------------------------------------------------ adaptation
    def block_norms(self, fields):
        """(max |v|, rms |v|) per octant over the interior nodes of the vector
        whose component fields are `fields` (Operator::maxnorm /
        blockRootMeanSquare, operators.hpp:1149-1211)."""
        f = np.ascontiguousarray(fields, dtype=np.int32).ravel()
        mx = np.zeros(self.n)
        rms = np.zeros(self.n)
        self._check(lib().iblgf_block_norms(self.h, _p(f), len(f), _p(mx), _p(rms)))
        return mx, rms

    def ns_fields(self):
        """Ids of the IF-HERK scratch fields the adapt condition reads:
        (cell_aux, [edge_aux x, y, z], correction_tmp)."""
        ids = np.zeros(5, np.int32)
        self._check(lib().iblgf_ns_fields(self.h, _p(ids)))
        return int(ids[0]), [int(x) for x in ids[1:4]], int(ids[4])

    def ns_clean(self, field, non_leaf_only=False, width=1):
        """Ifherk::clean (ifherk.hpp:1309-1352)."""
        self._check(lib().iblgf_ns_clean(self.h, int(field), 1 if non_leaf_only else 0, int(width)))

    def ns_clean_leaf_correction_boundary(self, fields, level, leaf_only_boundary=False):
        """Ifherk::clean_leaf_correction_boundary (ifherk.hpp:1355-1411) of a
        1- or 3-component field."""
        f = np.ascontiguousarray(fields, dtype=np.int32).ravel()
        self._check(lib().iblgf_ns_clean_leaf_correction_boundary(self.h, _p(f), len(f), int(level),
                                                                  1 if leaf_only_boundary else 0))

    def write_chombo(self, path, fields, time=0.0, dt=1, include_correction=True, base_correction_only=True):
        """Writes fields as a Chombo-HDF5 file in the reference's layout
        (Simulation::write, simulation.hpp:99-121, through
        io::H5_io::write_h5 / write_h5_withTime, IO/chombo/h5_io.hpp:161-200;
        by default with the base-level correction blocks, as Simulation::write):
        `fields` lists (name, field id) for a scalar and (name, [3 ids]) for a
        vector, whose components are named name_0, name_1, name_2."""
        import chombo_h5
        names, ids = [], []
        for name, fid in fields:
            if np.ndim(fid) == 0:
                names.append(name)
                ids.append(int(fid))
            else:
                for k, f in enumerate(fid):
                    names.append("%s_%d" % (name, k))
                    ids.append(int(f))
        vals = np.stack([self.download(f) for f in ids], 1)
        levels = chombo_h5.chombo_levels(self.keys, self.levels, self.bbase, self.block_extent, self.base_level,
                                         vals, self.flags, include_correction, base_correction_only)
        chombo_h5.write_chombo(path, names, levels, self.dx_base, time, dt)

    def read_chombo_field(self, path, name, fields, mesh):
        """Simulation::read_h5<Field> (simulation.hpp:200-204, Chombo::read_u,
        chombo_impl.hpp:216-520): the field `name` (scalar: one id; vector:
        three ids, components name_0..name_2) read from a Chombo file into the
        leaves; mesh 0 cell, 1 face, 2 edge, 3 vertex."""
        import chombo_h5
        ids = [int(fields)] if np.ndim(fields) == 0 else [int(f) for f in fields]
        vals = np.stack([self.download(f) for f in ids], 1)
        rl = self.levels - self.base_level
        corr = self.correction
        listed = (rl >= 0) & (~corr | (rl == 0))
        chombo_h5.read_field_into_blocks(chombo_h5.read_chombo(path), name, len(ids), mesh, self.dx_base, rl,
                                         self.bbase, self.block_extent, self.leaf, listed, vals)
        for k, f in enumerate(ids):
            self.upload(f, vals[:, k])
            self.synchronize()

    def write_tree(self, path):
        """Tree::write (tree.hpp:832-855) of this octree."""
        write_tree(path, self.keys, self.levels, self.flags)

    def write_restart(self, directory, fields, T, adapt_count=0, source_max=(0.0, 0.0), restart_n_last=0,
                      T_last_vel_refresh=0.0):
        """Ifherk::write_restart (ifherk.hpp:428-444): restart_field.hdf5
        (the fields, with base-level correction blocks, Simulation::write
        with restart_file, simulation.hpp:99-106), tree_info.bin and
        restart_info (Ifherk::write_info, :961-983)."""
        os.makedirs(directory, exist_ok=True)
        self.write_chombo(os.path.join(directory, "restart_field.hdf5"), fields)
        self.write_tree(os.path.join(directory, "tree_info.bin"))
        with open(os.path.join(directory, "restart_info"), "w") as f:
            for k, v in (("T", T), ("adapt_count", adapt_count), ("cell_aux_max", source_max[0]),
                         ("u_max", source_max[1]), ("restart_n_last", restart_n_last),
                         ("T_last_vel_refresh", T_last_vel_refresh)):
                f.write("%s = %s;\n" % (k, repr(float(v)) if isinstance(v, float) else v))

    def ns_march(self, u, p, dt, Re, T, n_steps, adapt_freq=0, adapt_condition=None, source_max=(1.0, 1.0),
                 updating_source_max=True, all_time_max=False):
        """Ifherk::time_march (ifherk.hpp:176-400) without output or restart.
        Per iteration: the non-leaf cleaning of cell_aux (width 2), edge_aux
        (1) and correction_tmp (2); every adapt_freq-th iteration but the
        first, source_max updated from the block RMS of cell_aux / edge_aux
        (update_source_max, :401-426) and one adaptation (Ifherk::adapt with
        coarsify_field = false, :1018-1076): cell_aux and edge_aux tapered at
        the base level, adapt_condition(solver, max cell_aux, max
        correction_tmp, max edge_aux, source_max) -> (keys, level_change),
        iblgf_adapt with the velocity interpolated; then one time step. (The
        loop's clean<u>(true) before the balance step repeats the step's own
        first clean and is left out.) Returns (T, source_max, attempts of each
        adaptation)."""
        import iblgf_setups as S
        sm = [float(source_max[0]), float(source_max[1])]
        history = []
        for it in range(int(n_steps)):
            cell, edge, corr = self.ns_fields()
            self.ns_clean(cell, True, 2)
            for e in edge:
                self.ns_clean(e, True, 1)
            self.ns_clean(corr, True, 2)
            if adapt_freq and it % adapt_freq == 0 and it != 0 and adapt_condition is not None:
                if updating_source_max:
                    sm[0] = S.update_source_max(sm[0], self.block_norms([cell])[1], all_time_max)
                    sm[1] = S.update_source_max(sm[1], self.block_norms(edge)[1], all_time_max)
                if sm[0] >= 1e-10 and sm[1] >= 1e-10:
                    self.ns_clean_leaf_correction_boundary([cell], self.base_level, True)
                    self.ns_clean_leaf_correction_boundary(edge, self.base_level, True)
                    keys, lc = adapt_condition(self, self.block_norms([cell])[0], self.block_norms([corr])[0],
                                               self.block_norms(edge)[0], sm)
                    self.adapt(keys, lc, interpolate=[(1, list(u))])
                    history.append((np.array(keys, np.uint64), np.array(lc, np.int32)))
            T = self.ns_step(u, p, dt, Re, T, 1)
        return T, sm, history

    def adapt(self, keys, level_change, interpolate=()):
        """One adaptation (Ifherk::adapt, ifherk.hpp:1018-1076): `keys` /
        `level_change` are the adapt condition's attempts (+1 refine, -1
        delete); `interpolate` lists (mesh, [field ids]) with mesh 0 cell (one
        id), 1 face, 2 edge (three ids) whose values are interpolated into the
        children of each new leaf's parent. Returns base_mesh_update; octant
        arrays (keys, levels, flags, bbase, n) are reloaded."""
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        lc = np.ascontiguousarray(level_change, dtype=np.int32)
        if len(k) != len(lc):
            raise ValueError("keys and level_change differ in length")
        fids = np.full((max(len(interpolate), 1), 3), -1, np.int32)
        mesh = np.zeros(max(len(interpolate), 1), np.int32)
        for i, (m, ids) in enumerate(interpolate):
            mesh[i] = m
            fids[i, :len(ids)] = ids
        bmu = ctypes.c_int()
        self._check(lib().iblgf_adapt(self.h, len(k), _p(k), _p(lc), len(interpolate), _p(fids), _p(mesh),
                                      ctypes.byref(bmu)))
        self._load_octants()
        return bool(bmu.value)

    # ------------------------------------------------------------ basics
    def _check(self, rc):
        if rc != 0:
            raise IblgfError("iblgf error %d: %s" % (rc, lib().iblgf_last_error(self.h).decode()), rc)

    def close(self):
        if getattr(self, "h", None):
            self._destroy(self.h)  # waits for the context's copies
            self.h = None
        self._async_out = []

    def __del__(self):
        self.close()

    @property
    def leaf(self):
        return (self.flags & 1) != 0

    @property
    def correction(self):
        return (self.flags & 2) != 0

    def lists(self):
        nbr = np.zeros((self.n, 27), np.int32)
        infl = np.zeros((self.n, 189), np.int32)
        ni = np.zeros(self.n, np.int32)
        self._check(lib().iblgf_domain_lists(self.h, _p(nbr), _p(infl), _p(ni)))
        return nbr, infl, ni

    def masks(self, idx):
        out = np.zeros((self.n, 2), np.uint8)
        self._check(lib().iblgf_domain_masks(self.h, int(idx), _p(out)))
        return out

    def zeros(self):
        return np.zeros((self.n, self.Nb, self.Nb, self.Nb))

    # ------------------------------------------------------------ fields
    def field(self, values=None):
        f = ctypes.c_int()
        self._check(lib().iblgf_field_create(self.h, ctypes.byref(f)))
        if values is not None:
            self.upload(f.value, values)
        return f.value

    def upload(self, fid, values):
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._check(lib().iblgf_field_upload(self.h, fid, _p(a), a.size))
        self._keep = a  # the copy is asynchronous; keep the host buffer alive

    def download(self, fid, out=None):
        a = self.zeros() if out is None else out
        self._check(lib().iblgf_field_download(self.h, fid, _p(a), a.size))
        return a

    @property
    def n_leaves(self):
        return int((self.flags & 1).sum())

    def upload_leaves(self, fid, values):
        """Leaf interiors (n_leaves, e, e, e) in canonical octant order into
        field `fid`; buffers and non-leaf blocks become zero."""
        a = np.ascontiguousarray(values, dtype=np.float64)
        self._check(lib().iblgf_field_upload_leaves(self.h, fid, _p(a), a.size))
        self._keep = a

    def download_leaves(self, fid, out=None):
        e = self.block_extent
        a = np.zeros((self.n_leaves, e, e, e)) if out is None else out
        self._check(lib().iblgf_field_download_leaves(self.h, fid, _p(a), a.size))
        return a

    def _leaf_host(self, what, buf):
        """(pointer, count) of a C-contiguous float64 host array or tensor of
        shape (n_leaves, e, e, e); raises otherwise."""
        e = self.block_extent
        shape = (self.n_leaves, e, e, e)
        if hasattr(buf, "data_ptr"):  # torch tensor
            import torch
            ok = (buf.dtype == torch.float64 and buf.is_contiguous() and tuple(buf.shape) == shape
                  and buf.device.type == "cpu")
            ptr, n = buf.data_ptr(), buf.numel()
        else:
            ok = (isinstance(buf, np.ndarray) and buf.dtype == np.float64 and buf.flags.c_contiguous
                  and buf.shape == shape)
            ptr, n = (buf.ctypes.data, buf.size) if ok else (0, 0)
        if not ok:
            raise IblgfError("%s: the host buffer must be a C-contiguous float64 array of shape %s" % (what, shape))
        return ptr, n

    def download_leaves_async(self, fid, out):
        """Starts the copy of the leaf interiors into `out` and returns; the
        copy is complete after synchronize(). `out` is a C-contiguous float64
        array or tensor of shape (n_leaves, e, e, e), pinned for the copy to
        overlap; it is kept alive here until synchronize() or close()."""
        ptr, n = self._leaf_host("download_leaves_async", out)
        self._check(lib().iblgf_field_download_leaves_async(self.h, fid, ctypes.c_void_p(ptr), n))
        self._async_out.append(out)

    def upload_leaves_async(self, fid, vals):
        """Starts the copy of leaf interiors from `vals` (pinned, shape
        (n_leaves, e, e, e)) into the field and returns: the copy runs on the
        library's copy stream, the scatter is ordered on the solver stream
        after it. `vals` is kept alive until synchronize() or close() and must
        not change before then."""
        ptr, n = self._leaf_host("upload_leaves_async", vals)
        self._check(lib().iblgf_field_upload_leaves_async(self.h, fid, ctypes.c_void_p(ptr), n))
        self._async_out.append(vals)

    def zero(self, fid):
        self._check(lib().iblgf_field_zero(self.h, fid))

    def device_ptr(self, fid):
        p = ctypes.c_void_p()
        self._check(lib().iblgf_field_device_ptr(self.h, fid, ctypes.byref(p)))
        return p.value

    def synchronize(self):
        self._check(lib().iblgf_synchronize(self.h))
        self._async_out = []

    # ------------------------------------------------------------ solver
    def fmm_apply(self, src, tgt, level, non_leaf_as_source, scale=1.0, fmm_type=AMR2AMR):
        self._check(lib().iblgf_fmm_apply(self.h, src, tgt, int(level), int(non_leaf_as_source),
                                          float(scale), int(fmm_type)))

    def apply_lgf(self, src, tgt, fmm_type=AMR2AMR):
        self._check(lib().iblgf_poisson_apply_lgf(self.h, src, tgt, int(fmm_type)))

    LAPLACE, GRADIENT, DIVERGENCE, CURL, CURL_TRANSPOSE, NONLINEAR = range(6)

    def op(self, op, inputs, outputs, level=-1, scale=1.0):
        """Mimetic block operator on field ids (Operator::laplace ... nonlinear)."""
        fi = np.array(inputs, np.int32)
        fo = np.array(outputs, np.int32)
        self._check(lib().iblgf_op_apply(self.h, int(op), _p(fi), len(fi), _p(fo), len(fo), int(level),
                                         float(scale)))

    def buffer_exchange(self, fid, level):
        self._check(lib().iblgf_buffer_exchange(self.h, int(fid), int(level)))

    def apply_if(self, src, tgt, alpha_base, fmm_type=AMR2AMR):
        """PoissonSolver::apply_lgf_IF (integrating factor, LGF_GE)."""
        self._check(lib().iblgf_poisson_apply_if(self.h, src, tgt, float(alpha_base), int(fmm_type)))

    def lgf_table(self):
        out = np.zeros(176851)
        self._check(lib().iblgf_lgf_table(self.h, _p(out), out.size))
        return out

    def lgf_get(self, coords):
        c = np.ascontiguousarray(np.asarray(coords, dtype=np.int32).reshape(-1, 3))
        out = np.zeros(c.shape[0])
        self._check(lib().iblgf_lgf_get(self.h, _p(c), c.shape[0], _p(out)))
        return out

    def ns_step(self, u_fields, p_field, dt, Re, T, n_steps=1):
        """IF-HERK steps (ifherk.hpp:1078-1200); returns the new time T."""
        uf = np.ascontiguousarray(np.asarray(u_fields, dtype=np.int32))
        t = ctypes.c_double(T)
        self._check(lib().iblgf_ns_step(self.h, _p(uf), int(p_field), float(dt), float(Re), ctypes.byref(t),
                                        int(n_steps)))
        return t.value

    def ns_options(self, frame_vel=(0.0, 0.0, 0.0), cg_threshold=1e-3, cg_max_iter=40):
        fv = np.ascontiguousarray(frame_vel, dtype=np.float64)
        self._check(lib().iblgf_ns_options(self.h, _p(fv), float(cg_threshold), int(cg_max_iter)))

    def ib_force(self, stage):
        out = np.zeros((len(self._ib_X), 3))
        self._check(lib().iblgf_ib_force(self.h, int(stage), _p(out), None))
        return out

    def ib_iterations(self):
        """CG iterations of stages 1..3 of the last step."""
        out = []
        for st in (1, 2, 3):
            it = ctypes.c_int()
            self._check(lib().iblgf_ib_force(self.h, st, None, ctypes.byref(it)))
            out.append(it.value)
        return out

    def partition(self, n_ranks):
        """Owner rank per octant: the reference server's load-balanced split
        (decomposition/server.hpp:245-330)."""
        out = np.zeros(self.n, np.int32)
        self._check(lib().iblgf_domain_partition(self.h, int(n_ranks), _p(out)))
        return out

    def set_owner(self, owner, rank, exchange):
        """Shard the sweeps: this context computes the targets owned by
        `rank`; exchange(device_ptr, count, stream) must replace the count
        doubles at device_ptr (ordered on the cudaStream_t `stream`) by their
        sum over the ranks. owner None ends the sharding."""
        if owner is None:
            self._check(lib().iblgf_domain_set_owner(self.h, None, 0, EXCHANGE_FN(), None))
            self._exchange = None
            return
        own = np.ascontiguousarray(owner, dtype=np.int32)

        def cb(user, ptr, count, stream):
            try:
                exchange(ptr, count, stream)
                return 0
            except Exception as e:  # reported as a failed exchange by the library
                self._exchange_error = e
                return 1

        self._exchange = EXCHANGE_FN(cb)  # kept alive while the context uses it
        self._check(lib().iblgf_domain_set_owner(self.h, _p(own), int(rank), self._exchange, None))

    def ge_direct(self, enable):
        """Integrating-factor sweeps by direct separable sums (True, default,
        where the kernel allows) or by block FFT convolutions (False)."""
        self._check(lib().iblgf_ge_direct(self.h, 1 if enable else 0))

    def mac_variant(self, variant):
        """Pin the sibling-group MAC variant (0, 1 direct tile shapes, 2
        block-Toeplitz, 3 tensor cores; -1 autotunes per plan)."""
        self._check(lib().iblgf_mac_variant(self.h, int(variant)))

    def mac_tuning(self):
        """Autotuner records: dicts with level, mask, targets, ms per variant
        (None if not applicable) and the chosen variant."""
        n = ctypes.c_int()
        self._check(lib().iblgf_mac_tuning(self.h, None, 0, ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 8))
        self._check(lib().iblgf_mac_tuning(self.h, _p(out), n.value, ctypes.byref(n)))
        return [{"level": int(r[0]), "mask": int(r[1]), "targets": int(r[2]),
                 "ms": [None if v < 0 else float(v) for v in r[3:7]], "choice": int(r[7])} for r in out[:n.value]]

    def ib_converged(self):
        """Whether each of stages 1..3 of the last step converged before
        cg_max_iter (the reference stops there silently)."""
        out = []
        for st in (1, 2, 3):
            it, ok = ctypes.c_int(), ctypes.c_int()
            self._check(lib().iblgf_ib_stage_status(self.h, st, ctypes.byref(it), ctypes.byref(ok)))
            out.append(bool(ok.value))
        return out

    def ib_warmstart(self, mode, train_steps=0, epochs=0, lr=1e-3, seed=1):
        self._check(lib().iblgf_ib_warmstart(self.h, int(mode), int(train_steps), int(epochs), float(lr), int(seed)))

    def ib_warmstart_info(self):
        out = np.zeros(6)
        self._check(lib().iblgf_ib_warmstart_info(self.h, _p(out)))
        return {"mode": int(out[0]), "trained": bool(out[1]), "samples": int(out[2]), "loss_first": out[3],
                "loss_last": out[4], "params": int(out[5])}

    def ws_check(self, params, x, t):
        """One forward + backward pass of the warm-start network on the device."""
        S, _, N = x.shape
        p = np.ascontiguousarray(params, np.float32)
        xx = np.ascontiguousarray(x, np.float32)
        tt = np.ascontiguousarray(t, np.float32)
        y = np.zeros((S, 3, N), np.float32)
        g = np.zeros_like(p)
        loss = ctypes.c_float()
        self._check(lib().iblgf_ws_check(self.h, S, N, _p(p), _p(xx), _p(tt), _p(y), _p(g), ctypes.byref(loss)))
        return y, g, loss.value

    def ib_set_points(self, X, Re):
        """IB points (n, 3) on the finest level (ib.hpp / server.hpp / client.hpp)."""
        self._ib_X = np.ascontiguousarray(X, dtype=np.float64)
        self._check(lib().iblgf_ib_set_points(self.h, len(self._ib_X), _p(self._ib_X), float(Re)))

    def ib_flags(self):
        out = np.zeros(self.n, np.int32)
        self._check(lib().iblgf_ib_flags(self.h, _p(out)))
        return out

    def ib_solve(self, u_fields, alpha, threshold=1e-3, max_iter=40, f0=None):
        """IB force solve (linsys.hpp:113-230); returns (force (n, 3), CG iterations)."""
        uf = np.ascontiguousarray(np.asarray(u_fields, dtype=np.int32))
        f = np.zeros((len(self._ib_X), 3)) if f0 is None else np.ascontiguousarray(f0, dtype=np.float64).copy()
        it = ctypes.c_int()
        rc = lib().iblgf_ib_solve(self.h, _p(uf), float(alpha), float(threshold), int(max_iter), _p(f),
                                  ctypes.byref(it))
        if rc == ENOTCONVERGED:
            err = IblgfNotConverged("IB force CG stopped at max_iter = %d without converging" % max_iter)
            err.force, err.iterations = f, it.value
            raise err
        self._check(rc)
        return f, it.value

    def conv_block(self, src_dptr, kernel_dptr, out_dptr, scale=1.0):
        self._check(lib().iblgf_conv_block(self.h, ctypes.c_void_p(src_dptr), ctypes.c_void_p(kernel_dptr),
                                           ctypes.c_void_p(out_dptr), float(scale)))

    def launches(self):
        n = ctypes.c_longlong()
        self._check(lib().iblgf_kernel_launches(self.h, ctypes.byref(n)))
        return n.value

    def profile(self, enable=True):
        self._check(lib().iblgf_profile(self.h, 1 if enable else 0))

    def stats(self):
        """[sweeps, sources, targets, pairs, unique spectra, anterp tasks,
        interp tasks, group-MAC targets, MAC products covered, MAC flops per
        frequency]"""
        out = np.zeros(10, np.int64)
        self._check(lib().iblgf_stats_n(self.h, _p(out), 10))
        return out

    def fma_peak(self, precision):
        v = ctypes.c_double()
        self._check(lib().iblgf_fma_peak(self.h, int(precision), ctypes.byref(v)))
        return v.value

    def wait_selftest(self, polls):
        """Run the bounded device wait on a barrier nothing arrives on;
        raises IblgfError with code ETIMEOUT (the expected outcome)."""
        self._check(lib().iblgf_wait_selftest(self.h, int(polls)))

    def first_nonfinite(self, fid):
        """Smallest element index of a NaN / inf in the field, or -1."""
        v = ctypes.c_longlong()
        self._check(lib().iblgf_field_first_nonfinite(self.h, fid, ctypes.byref(v)))
        return v.value

    def helm2d_lgf(self, c, nx, ny):
        """2-D Helmholtz LGF get(n, m) (lgf::Helmholtz<2>) for 0 <= n < nx,
        0 <= m < ny, as an (ny, nx) array (at most 2^28 entries)."""
        if not (0 < int(nx) and 0 < int(ny) and int(nx) * int(ny) <= 1 << 28):
            raise IblgfError("the table holds 1 .. 2^28 entries")
        out = np.zeros((ny, nx))
        self._check(lib().iblgf_helm2d_lgf(self.h, float(c), int(nx), int(ny), _p(out)))
        return out

    def helm2d_get(self, c, offsets):
        """get(n, m) of the 2-D Helmholtz LGF (c = 0: the 2-D Laplace LGF)
        at each offset of an (k, 2) integer array."""
        nm = np.ascontiguousarray(np.asarray(offsets, dtype=np.int32).reshape(-1, 2))
        out = np.zeros(nm.shape[0])
        self._check(lib().iblgf_helm2d_get(self.h, float(c), nm.shape[0], _p(nm), _p(out)))
        return out

    def helm2d_apply(self, c, f, u=None, scale=1.0):
        """u + scale * (get * f) over the uniform grid of f (shape (ny, nx))."""
        f = np.ascontiguousarray(f, dtype=np.float64)
        u = np.zeros_like(f) if u is None else np.ascontiguousarray(u, dtype=np.float64).copy()
        self._check(lib().iblgf_helm2d_apply(self.h, float(c), f.shape[1], f.shape[0], _p(f), _p(u), float(scale)))
        return u

    HELM_OPS = {"laplace": 0, "gradient": 1, "divergence": 2, "curl": 3, "curl_transpose": 4}

    @staticmethod
    def _cuda_f64(*ts):
        import torch
        for t in ts:
            if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise IblgfError("the Helmholtz block operators take contiguous float64 CUDA tensors")

    @staticmethod
    def _unit_mask(n, units):
        """A byte per unit (mode or plane): None selects all, else the
        selected indices or a boolean sequence of length n."""
        if units is None:
            return None
        m = np.asarray(units)
        if m.dtype == bool:
            if m.shape != (n,):
                raise IblgfError("a boolean mask has one entry per unit")
            out = m.astype(np.uint8)
        else:
            out = np.zeros(n, np.uint8)
            idx = m.astype(np.int64).ravel()
            if idx.size and (idx.min() < 0 or idx.max() >= n):
                raise IblgfError("unit index out of range")
            out[idx] = 1
        return out

    def helm2d_op(self, op, src, dst, n_modes, dx_level, lz, scale=1.0, modes=None):
        """A complex Helmholtz block operator on 2-D blocks (torch CUDA
        tensors [n_blocks][ncomp][nb][nb], float64); dst updated in place.
        modes: None (all modes, the plain forms), the selected mode indices
        (a single one: the _oneMode forms; range(n_modes >> r): the _refined
        forms) or a boolean sequence (the ModesBool forms)."""
        if op not in self.HELM_OPS:
            raise IblgfError("unknown Helmholtz operator %r (one of %s)" % (op, ", ".join(self.HELM_OPS)))
        self._cuda_f64(src, dst)
        k = self.HELM_OPS[op]
        sep = 2 * int(n_modes)
        cin, cout = (sep if k in (0, 1) else 3 * sep), (sep if k in (0, 2) else 3 * sep)
        nb = src.shape[-1]
        if (src.dim() != 4 or dst.dim() != 4 or tuple(src.shape[1:]) != (cin, nb, nb)
                or tuple(dst.shape) != (src.shape[0], cout, nb, nb)):
            raise IblgfError("%s takes [n_blocks][%d][nb][nb] into [n_blocks][%d][nb][nb]" % (op, cin, cout))
        mask = self._unit_mask(int(n_modes), modes)
        if mask is None:
            self._check(lib().iblgf_helm2d_op(self.h, k, nb, src.shape[0], int(n_modes),
                                              float(dx_level), float(lz), float(scale),
                                              ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr())))
        else:
            self._check(lib().iblgf_helm2d_op_modes(self.h, k, nb, src.shape[0],
                                                    int(n_modes), _p(mask), float(dx_level), float(lz), float(scale),
                                                    ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr())))

    def helm2d_nonlinear(self, face, edge, dst, n_planes, planes=None):
        """The convective term on the z collocation planes
        (nonlinear_helmholtz): face, edge, dst are torch CUDA tensors
        [n_blocks][3 n_planes][nb][nb], float64; planes as helm2d_op's modes."""
        self._cuda_f64(face, edge, dst)
        nb = face.shape[-1]
        shape = (face.shape[0], 3 * int(n_planes), nb, nb)
        if face.dim() != 4 or any(tuple(t.shape) != shape for t in (face, edge, dst)):
            raise IblgfError("the nonlinear term takes three [n_blocks][3 n_planes][nb][nb] tensors")
        mask = self._unit_mask(int(n_planes), planes)
        self._check(lib().iblgf_helm2d_nonlinear(self.h, nb, face.shape[0], int(n_planes),
                                                 None if mask is None else _p(mask),
                                                 ctypes.c_void_p(face.data_ptr()), ctypes.c_void_p(edge.data_ptr()),
                                                 ctypes.c_void_p(dst.data_ptr())))

    HELM_REAL_OPS = {"curl_planes": 0, "curl_real": 1, "curl_real_uz": 2, "curl_transpose_linear": 3,
                     "nonlinear_linear": 4, "curl_transpose_2d": 5}

    def helm2d_real_op(self, op, a, d, b=None, e=None, n_planes=1, dx_level=1.0, dx_fine=1.0, c=0.0, scale=1.0):
        """A real-valued Fourier-in-z family block operator on 2-D blocks
        (torch CUDA float64 tensors [n_blocks][components][nb][nb]; the
        operator reads a (and b) and writes d (and e, one component)):
        curl_planes (curl_helmholtz on n_planes z planes), curl_real,
        curl_real_uz (b: Uz), curl_transpose_linear (e: face z),
        nonlinear_linear (a face, b edge; e: z), curl_transpose_2d."""
        if op not in self.HELM_REAL_OPS:
            raise IblgfError("unknown Helmholtz operator %r (one of %s)" % (op, ", ".join(self.HELM_REAL_OPS)))
        k = self.HELM_REAL_OPS[op]
        ts = [t for t in (a, b, d, e) if t is not None]
        self._cuda_f64(*ts)
        nb = a.shape[-1]
        for t in ts:
            if t.dim() != 4 or t.shape[0] != a.shape[0] or tuple(t.shape[2:]) != (nb, nb):
                raise IblgfError("the real operators take [n_blocks][components][nb][nb] tensors")
        if e is not None and e.shape[1] != 1:
            raise IblgfError("e holds one component")
        ptr = lambda t: None if t is None else ctypes.c_void_p(t.data_ptr())
        self._check(lib().iblgf_helm2d_real_op(self.h, k, nb, a.shape[0], int(n_planes), float(dx_level),
                                               float(dx_fine), float(c), float(scale), ptr(a), a.shape[1], ptr(b),
                                               0 if b is None else b.shape[1], ptr(d), d.shape[1], ptr(e)))

    def tc_mma_rate(self, n):
        """SM clocks per tensor-core MMA (TF32, M = 128, K = 8, N = n)."""
        v = ctypes.c_double()
        self._check(lib().iblgf_tc_mma_rate(self.h, int(n), ctypes.byref(v)))
        return v.value

    def profile_read(self):
        out = np.zeros(4)
        self._check(lib().iblgf_profile_read(self.h, _p(out)))
        return out


def from_case(case, **kw):
    """Build a Solver for an iblgf_setups case object."""
    return Solver(case.bd_base, case.bd_extent, case.block_extent, case.dx_base, case.blocks,
                  n_levels=getattr(case, "n_levels", 0), predicate=getattr(case, "predicate", None), **kw)


class ProblemView:
    """Octants of one problem of a batch (the attributes an iblgf_setups case
    reads when it builds fields): n, levels, flags, bbase, base_level, leaf."""

    def __init__(self, offset, n, base_level, depth, keys, levels, flags, bbase):
        self.offset, self.n, self.base_level, self.depth = offset, n, base_level, depth
        self.keys, self.levels, self.flags, self.bbase = keys, levels, flags, bbase

    @property
    def leaf(self):
        return (self.flags & 1) != 0

    @property
    def correction(self):
        return (self.flags & 2) != 0


class BatchSolver(Solver):
    """Many independent unbounded Poisson problems in one context
    (iblgf_batch_*): problems = list of dicts with bd_base, bd_extent, blocks
    and optionally n_levels / predicate. Fields hold the problems' octants back
    to back; problem(i) gives the octant range and arrays of problem i."""

    def __init__(self, block_extent, dx_base, problems, precision=FP64, device=0, stream=None,
                 subtract_non_leaf=False, use_correction=True, intrp_order=5):
        L = lib()
        cfg = Config(block_extent, (ctypes.c_int * 3)(0, 0, 0), (ctypes.c_int * 3)(0, 0, 0),
                     float(dx_base), int(precision), int(device), int(intrp_order),
                     ctypes.c_void_p(stream) if stream else None)
        h = ctypes.c_void_p()
        rc = L.iblgf_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != 0:
            raise IblgfError("iblgf_create failed (%d): %s" % (rc, L.iblgf_last_error(None).decode()), rc)
        self._destroy = L.iblgf_destroy  # kept so that close() works during interpreter shutdown
        self.h = h
        self._async_out = []  # host buffers of asynchronous downloads in flight
        self.Nb = block_extent + 2
        self.block_extent = block_extent
        self.precision = precision
        self._cbs = []
        for pr in problems:
            bb = np.array([b[0] for b in pr["blocks"]], np.int32).ravel()
            be = np.array([b[1] for b in pr["blocks"]], np.int32).ravel()
            pred = pr.get("predicate")
            if pred is not None:
                def cb(user, base, ext, rl, diff, pred=pred):
                    return 1 if pred((base[0], base[1], base[2]), (ext[0], ext[1], ext[2]), rl, diff) else 0
                fn = REFINE_FN(cb)
            else:
                fn = REFINE_FN(lambda *a: 0)
            self._cbs.append(fn)
            pid = ctypes.c_int()
            self._check(L.iblgf_batch_add_problem(self.h, _p(np.array(pr["bd_base"], np.int32)),
                                                  _p(np.array(pr["bd_extent"], np.int32)), len(pr["blocks"]),
                                                  _p(bb), _p(be), int(pr.get("n_levels", 0)), fn, None,
                                                  ctypes.byref(pid)))
        self._check(L.iblgf_batch_finalize(self.h, 1 if subtract_non_leaf else 0))
        self._check(L.iblgf_poisson_options(self.h, 1 if use_correction else 0, 1 if subtract_non_leaf else 0))
        self.views = []
        for i in range(len(problems)):
            info = np.zeros(4, np.int32)
            self._check(L.iblgf_batch_problem_info(self.h, i, _p(info)))
            n = int(info[1])
            keys, levels = np.zeros(n, np.uint64), np.zeros(n, np.int32)
            flags, bbase = np.zeros(n, np.int32), np.zeros((n, 3), np.int32)
            self._check(L.iblgf_batch_problem_octants(self.h, i, _p(keys), _p(levels), _p(flags), _p(bbase)))
            self.views.append(ProblemView(int(info[0]), n, int(info[2]), int(info[3]), keys, levels, flags, bbase))
        self.n = sum(v.n for v in self.views)
        self.flags = np.concatenate([v.flags for v in self.views])
        self.levels = np.concatenate([v.levels for v in self.views])
        self.bbase = np.concatenate([v.bbase for v in self.views])

    def problem(self, i):
        return self.views[i]

    def split(self, arr):
        """Per-problem slices of a batch field array."""
        return [arr[v.offset:v.offset + v.n] for v in self.views]

    def apply_lgf(self, src, tgt, fmm_type=AMR2AMR):
        if fmm_type != AMR2AMR:
            raise IblgfError("batches support the AMR2AMR mask")
        self._check(lib().iblgf_batch_apply_lgf(self.h, src, tgt))

