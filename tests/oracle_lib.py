"""ctypes wrapper of the CPU oracle (oracle/liboracle_iblgf.so).

Test infrastructure: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py only.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle_iblgf.so")

PRED_T = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                          ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int)

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cd = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_lgf_get.restype = cd
        L.orc_lgf_get.argtypes = [ci, ci, ci]
        L.orc_lgf_table_size.restype = ci
        L.orc_lgf_table.argtypes = [vp]
        L.orc_bessel_ie.argtypes = [cd, ci, vp]
        L.orc_nli_matrix.argtypes = [ci, ci, vp]
        L.orc_cc_matrix.argtypes = [ci, ci, ci, vp]
        L.orc_domain_create.restype = vp
        L.orc_adapt.argtypes = [vp, ci, vp, vp, ci, vp, vp]
        L.orc_adapt_field.argtypes = [vp, vp, ci, ci, vp]
        L.orc_domain_create.argtypes = [vp, vp, ci, cd, ci, vp, vp]
        L.orc_domain_destroy.argtypes = [vp]
        L.orc_domain_init_refine.argtypes = [vp, ci, ci, PRED_T, vp]
        L.orc_domain_finalize.argtypes = [vp, ci]
        L.orc_domain_info.argtypes = [vp, vp, vp, vp]
        L.orc_domain_octants.argtypes = [vp, vp, vp, vp, vp]
        L.orc_domain_lists.argtypes = [vp, vp, vp, vp]
        L.orc_domain_masks.argtypes = [vp, ci, vp]
        L.orc_solver_create.argtypes = [vp, ci]
        L.orc_fmm_apply.argtypes = [vp, vp, vp, ci, ci, cd, ci]
        L.orc_apply_lgf.argtypes = [vp, vp, vp, ci, ci]
        L.orc_apply_lgf_type.argtypes = [vp, vp, vp, ci, ci, ci]
        L.orc_block_conv.argtypes = [ci, vp, vp, vp, cd]
        L.orc_op.argtypes = [vp, ci, ci, vp, ci, vp, ci, cd]
        L.orc_buffer_exchange.argtypes = [vp, vp, ci]
        L.orc_apply_if.argtypes = [vp, vp, vp, cd, ci]
        L.orc_fmm_apply_ge.argtypes = [vp, vp, vp, ci, ci, cd, cd]
        L.orc_lgf_ge_get.argtypes = [vp, ci, ci, ci, cd]
        L.orc_lgf_ge_get.restype = cd
        L.orc_ns_step.argtypes = [vp, cd, cd, cd, vp, vp, ci]
        L.orc_ib_solve.argtypes = [vp, ci, vp, cd, vp, cd, cd, ci, vp, vp, vp]
        L.orc_ns_step_ib.argtypes = [vp, cd, cd, cd, vp, vp, ci, ci, vp, vp, cd, ci, vp]
        L.orc_sphere_points.argtypes = [cd, ci, cd, vp, ci]
        L.orc_sphere_points.restype = ci
        L.orc_yang3.argtypes = [cd]
        L.orc_yang3.restype = cd
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _check(rc):
    if rc != 0:
        raise RuntimeError("oracle: " + lib().orc_last_error().decode())


def lgf_get(x, y, z):
    return lib().orc_lgf_get(int(x), int(y), int(z))


def sphere_points(dx_base, ib_level, ibph):
    """ib.hpp:179-210: Fibonacci points on the sphere R = 0.5."""
    n = lib().orc_sphere_points(float(dx_base), int(ib_level), float(ibph), None, 0)
    X = np.zeros((n, 3))
    lib().orc_sphere_points(float(dx_base), int(ib_level), float(ibph), _p(X), n)
    return X


def block_conv(src, kernel, scale=1.0):
    """Single-block convolution (reference Convolution contract)."""
    Nb = src.shape[0]
    out = np.zeros(Nb ** 3)
    _check(lib().orc_block_conv(Nb, _p(np.ascontiguousarray(src.ravel(order="F"))),
                                _p(np.ascontiguousarray(kernel.ravel(order="F"))), _p(out), scale))
    return out.reshape((Nb,) * 3, order="F")


class Domain:
    """Oracle domain: base mesh, refinement, correction marking, masks."""

    def __init__(self, bd_base, bd_extent, block_extent, dx_base, blocks, n_levels=0,
                 global_refinement=0, predicate=None, subtract_non_leaf=False, intrp_order=5):
        L = lib()
        bb = np.array([b[0] for b in blocks], dtype=np.int32).ravel()
        be = np.array([b[1] for b in blocks], dtype=np.int32).ravel()
        self.h = L.orc_domain_create(_p(np.array(bd_base, np.int32)), _p(np.array(bd_extent, np.int32)),
                                     int(block_extent), float(dx_base), len(blocks), _p(bb), _p(be))
        if not self.h:
            raise RuntimeError("oracle: " + L.orc_last_error().decode())
        self.block_extent = block_extent
        self.Nb = block_extent + 2
        self._cb = None
        if n_levels > 0 or global_refinement > 0:
            if predicate is not None:
                def cb(user, base, ext, rl, diff):
                    return 1 if predicate((base[0], base[1], base[2]), (ext[0], ext[1], ext[2]),
                                          rl, diff) else 0
                self._cb = PRED_T(cb)
            else:
                self._cb = PRED_T(lambda *a: 0)
            _check(L.orc_domain_init_refine(self.h, n_levels, global_refinement, self._cb, None))
        else:
            # init_refine with nothing to refine still marks corrections
            self._cb = PRED_T(lambda *a: 0)
            _check(L.orc_domain_init_refine(self.h, 0, 0, self._cb, None))
        _check(L.orc_domain_finalize(self.h, 1 if subtract_non_leaf else 0))
        self._subtract_non_leaf = subtract_non_leaf
        self._load_octants()
        _check(L.orc_solver_create(self.h, intrp_order))

    def _load_octants(self):
        L = lib()
        bl, dp, n = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        L.orc_domain_info(self.h, ctypes.byref(bl), ctypes.byref(dp), ctypes.byref(n))
        self.base_level, self.depth, self.n = bl.value, dp.value, n.value
        self.keys = np.zeros(self.n, np.uint64)
        self.levels = np.zeros(self.n, np.int32)
        self.flags = np.zeros(self.n, np.int32)
        self.bbase = np.zeros((self.n, 3), np.int32)
        L.orc_domain_octants(self.h, _p(self.keys), _p(self.levels), _p(self.flags), _p(self.bbase))

    def adapt(self, keys, level_change, fields=()):
        """Domain::adapt (decomposition.hpp:182-470, one process) with the
        attempts (keys, level_change); `fields` lists (array (n, Nb, Nb, Nb),
        mesh, comp) with mesh -1 (remap only) or 0 cell / 1 face / 2 edge
        (remap, then interpolation into the children of each new leaf's
        parent). Returns (base_mesh_update, remapped fields)."""
        k = np.ascontiguousarray(keys, dtype=np.uint64)
        lc = np.ascontiguousarray(level_change, dtype=np.int32)
        bmu, n = ctypes.c_int(), ctypes.c_int()
        _check(lib().orc_adapt(self.h, len(k), _p(k), _p(lc), 1 if self._subtract_non_leaf else 0,
                               ctypes.byref(bmu), ctypes.byref(n)))
        self._load_octants()
        out = []
        for f, mesh, comp in fields:
            old = np.ascontiguousarray(f, dtype=np.float64)
            new = np.zeros((self.n, self.Nb, self.Nb, self.Nb))
            _check(lib().orc_adapt_field(self.h, _p(old), int(mesh), int(comp), _p(new)))
            out.append(new)
        return bool(bmu.value), out

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_domain_destroy(self.h)
            self.h = None

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
        lib().orc_domain_lists(self.h, _p(nbr), _p(infl), _p(ni))
        return nbr, infl, ni

    def masks(self, mask_idx):
        out = np.zeros((self.n, 2), np.uint8)
        lib().orc_domain_masks(self.h, int(mask_idx), _p(out))
        return out

    def zeros(self):
        return np.zeros((self.n, self.Nb, self.Nb, self.Nb))  # [oct][z][y][x]

    def fmm_apply(self, src, tgt, level, non_leaf_as_source, scale=1.0, fmm_type=1):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.ascontiguousarray(tgt, dtype=np.float64).copy()
        _check(lib().orc_fmm_apply(self.h, _p(src), _p(out), int(level), int(non_leaf_as_source),
                                   float(scale), int(fmm_type)))
        return out

    def op(self, op, inputs, outputs, level=-1, scale=1.0):
        """Mimetic block operator; inputs/outputs are lists of fields."""
        ins = [np.ascontiguousarray(a, dtype=np.float64) for a in inputs]
        outs = [np.ascontiguousarray(a, dtype=np.float64).copy() for a in outputs]
        pin = (ctypes.c_void_p * len(ins))(*[a.ctypes.data for a in ins])
        pout = (ctypes.c_void_p * len(outs))(*[a.ctypes.data for a in outs])
        _check(lib().orc_op(self.h, int(op), len(ins), pin, len(outs), pout, int(level), float(scale)))
        return outs

    def buffer_exchange(self, f, level):
        x = np.ascontiguousarray(f, dtype=np.float64).copy()
        _check(lib().orc_buffer_exchange(self.h, _p(x), int(level)))
        return x

    def apply_if(self, src, alpha_base, tgt=None, subtract_non_leaf=False):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = self.zeros() if tgt is None else np.ascontiguousarray(tgt, dtype=np.float64).copy()
        _check(lib().orc_apply_if(self.h, _p(src), _p(out), float(alpha_base), int(subtract_non_leaf)))
        return out

    def fmm_apply_ge(self, src, tgt, level, non_leaf_as_source, scale, alpha):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = np.ascontiguousarray(tgt, dtype=np.float64).copy()
        _check(lib().orc_fmm_apply_ge(self.h, _p(src), _p(out), int(level), int(non_leaf_as_source),
                                      float(scale), float(alpha)))
        return out

    def lgf_ge_get(self, x, y, z, alpha):
        return lib().orc_lgf_ge_get(self.h, int(x), int(y), int(z), float(alpha))

    def ns_step(self, u, dt, Re, T0=0.0, n_steps=1):
        """IF-HERK steps (ifherk.hpp:1078-1200); u: (3, n, Nb, Nb, Nb) face
        velocity. Returns (u, p) after n_steps."""
        uu = np.ascontiguousarray(u, dtype=np.float64).copy()
        p = self.zeros()
        _check(lib().orc_ns_step(self.h, float(dt), float(Re), float(T0), _p(uu), _p(p), int(n_steps)))
        return uu, p

    def ns_step_ib(self, u, dt, Re, X, frame_vel=(0.0, 0.0, 0.0), T0=0.0, n_steps=1, threshold=1e-3,
                   max_iter=40):
        """IF-HERK steps with an immersed boundary (ifherk.hpp:1451-1517);
        returns (u, p, stage forces (3, n, 3) of the last step)."""
        uu = np.ascontiguousarray(u, dtype=np.float64).copy()
        p = self.zeros()
        X = np.ascontiguousarray(X, dtype=np.float64)
        fv = np.ascontiguousarray(frame_vel, dtype=np.float64)
        forces = np.zeros((3, len(X), 3))
        _check(lib().orc_ns_step_ib(self.h, float(dt), float(Re), float(T0), _p(uu), _p(p), int(n_steps), len(X),
                                    _p(X), _p(fv), float(threshold), int(max_iter), _p(forces)))
        return uu, p, forces

    def ib_solve(self, X, Re, u, alpha, threshold=1e-3, max_iter=40, f0=None):
        """IB force solve (linsys.hpp:113-230): returns (force (n, 3), flags per
        octant (bit0 is_ib, bit1 is_extended_ib), CG iterations)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        f = np.zeros((len(X), 3)) if f0 is None else np.ascontiguousarray(f0, dtype=np.float64).copy()
        flags = np.zeros(self.n, np.int32)
        it = ctypes.c_int()
        _check(lib().orc_ib_solve(self.h, len(X), _p(X), float(Re), _p(uu), float(alpha), float(threshold),
                                  int(max_iter), _p(f), _p(flags), ctypes.byref(it)))
        return f, flags, it.value

    def apply_lgf(self, src, tgt=None, use_correction=True, subtract_non_leaf=False, fmm_type=1):
        src = np.ascontiguousarray(src, dtype=np.float64)
        out = self.zeros() if tgt is None else np.ascontiguousarray(tgt, dtype=np.float64).copy()
        _check(lib().orc_apply_lgf_type(self.h, _p(src), _p(out), int(use_correction),
                                        int(subtract_non_leaf), int(fmm_type)))
        return out
