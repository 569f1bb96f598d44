"""Python binding of libqumasun_b200.so (the C ABI in include/qumasun_b200.h).

Mirrors the reference's call surfaces for the H.psi / LOBPCG path:

  laplacian8th(out, p, coef, dx, dy, dz)        ~ Laplacian8th<T>            (GridDifference8th.h:177)
  laplacian_kpoint8th(out, src, coef, d, g)     ~ LaplacianKpoint8th_ddm      (GridDifferenceKpoint8th.h:324)
  Hamiltonian.apply(psi, hpsi, g)               ~ mHamiltonianMatrix_ddm      (qumasun_base1.matrix.h:263)
  Hamiltonian.nonlocal_apply(psi, hpsi, g)      ~ ProjectionPP_bundle         (PseudoPotNonlocal_SvF2_kpoint.h:4239)
  Hamiltonian.nonlocal_project(psi, g)          ~ mInnerNonlocalPsi_v4_bundle (PseudoPotNonlocal_SvF2_kpoint.h:4463)

Arrays are torch CUDA tensors in the reference's band-bundle layouts (real:
[nb, N]; complex SoA: [nb, 2, N] i.e. re plane then im plane per band), float64
or float32.  Calls run on torch's current CUDA stream.  There is no CPU path:
if the CUDA library is missing or fails to load, import raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqumasun_b200.so")

QSB_F64 = 0
QSB_F32 = 1

_STATUS = {0: "QSB_OK", 1: "QSB_ERR_INVALID", 2: "QSB_ERR_CUDA", 3: "QSB_ERR_NOMEM", 4: "QSB_ERR_STATE",
           5: "QSB_ERR_SOLVER", 6: "QSB_ERR_NUMERIC"}


class QsbError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{_STATUS.get(status, status)}: {msg}")
        self.status = status


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"libqumasun_b200.so not built at {LIB_PATH}; run "
                          "python qumasun-workshop-template_b200/build_lib.py")
    lib = ctypes.CDLL(LIB_PATH)
    lib.qsb_last_error.restype = ctypes.c_char_p
    lib.qsb_version.restype = ctypes.c_char_p
    return lib


lib = _load()
_c_d = ctypes.c_double
_vp = ctypes.c_void_p


def _check(st):
    if st != 0:
        raise QsbError(st, lib.qsb_last_error().decode())


def version():
    return lib.qsb_version().decode()


def device_status(clear=False):
    """Device error word (bit 0: a kernel's bounded wait ran out); synchronizes."""
    code = ctypes.c_int()
    _check(lib.qsb_device_status(ctypes.byref(code), int(bool(clear))))
    return code.value


def _torch():
    import torch
    return torch


def _dtype_code(t):
    torch = _torch()
    if t.dtype == torch.float64:
        return QSB_F64
    if t.dtype == torch.float32:
        return QSB_F32
    raise TypeError(f"unsupported dtype {t.dtype}")


def _stream_ptr(t):
    torch = _torch()
    return _vp(torch.cuda.current_stream(t.device).cuda_stream)


def _dev_ptr(t):
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return _vp(t.data_ptr())


def laplacian8th(out, p, coef, dx, dy, dz, shape):
    """out += coef * FD8 Laplacian(p); p, out: [nb, N] (or [N]) CUDA tensors."""
    nx, ny, nz = shape
    N = nx * ny * nz
    nb = p.numel() // N
    assert out.dtype == p.dtype and out.numel() == p.numel()
    _check(lib.qsb_laplacian8th(_dtype_code(p), nx, ny, nz, nb, _dev_ptr(out), _dev_ptr(p), _c_d(coef), _c_d(dx),
                                _c_d(dy), _c_d(dz), _stream_ptr(p)))
    return out


def laplacian_kpoint8th(out, src, coef, dx, dy, dz, g, shape):
    """out += coef*(Lap + 2i g.grad - g^2) src for complex SoA bands [nb, 2, N]."""
    nx, ny, nz = shape
    N = nx * ny * nz
    nb = src.numel() // (2 * N)
    assert out.dtype == src.dtype and out.numel() == src.numel()
    _check(lib.qsb_laplacian_kpoint8th(_dtype_code(src), nx, ny, nz, nb, _dev_ptr(out), _dev_ptr(src), _c_d(coef),
                                       _c_d(dx), _c_d(dy), _c_d(dz), _c_d(g[0]), _c_d(g[1]), _c_d(g[2]),
                                       _stream_ptr(src)))
    return out


def apply_batch(hams, psis, hpsis):
    """H psi of several independent systems (qsb_ham_apply_batch): hams a list of
    Hamiltonian, psis / hpsis lists of [nb_i, N_i] real CUDA tensors of one dtype."""
    n = len(hams)
    dt = _dtype_code(psis[0])
    nb = np.array([p.numel() // h.N for h, p in zip(hams, psis)], np.int32)
    harr = (ctypes.c_void_p * n)(*[h._h.value for h in hams])
    parr = (ctypes.c_void_p * n)(*[_dev_ptr(p).value for p in psis])
    oarr = (ctypes.c_void_p * n)(*[_dev_ptr(p).value for p in hpsis])
    _check(lib.qsb_ham_apply_batch(dt, n, harr, nb.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), parr, oarr,
                                   _stream_ptr(psis[0])))
    return hpsis


def set_autotune(enable):
    """qsb_set_autotune: time the stencil kernels (and batched vs per-system) on first use of a shape."""
    _check(lib.qsb_set_autotune(int(bool(enable))))


def autotune_report():
    """The autotuner's decision log (qsb_autotune_report)."""
    need = ctypes.c_int()
    _check(lib.qsb_autotune_report(None, 0, ctypes.byref(need)))
    buf = ctypes.create_string_buffer(max(1, need.value))
    _check(lib.qsb_autotune_report(buf, len(buf), None))
    return buf.value.decode()


def fermi_occupations(eig, n_el, kbt, weights=None):
    """(occupations in [0, 2], mu) of the levels eig with k weights (qsb_fermi_occupations; host)."""
    e, e_p = _f64(np.asarray(eig, np.float64).ravel())
    occ, occ_p = _f64(np.zeros(len(e)))
    w, w_p = _f64(np.asarray(weights, np.float64).ravel()) if weights is not None else (None, None)
    mu = ctypes.c_double()
    _check(lib.qsb_fermi_occupations(len(e), e_p, w_p, _c_d(n_el), _c_d(kbt), occ_p, ctypes.byref(mu)))
    return occ, mu.value


def orthonormalize(X, N, dV, is_complex=False):
    """dV-weighted orthonormalisation of a band bundle in place (qsb_orthonormalize,
    the role of GramSchmidt_ddm); X: [nb, N] real or [nb, 2, N] complex SoA, fp64 CUDA."""
    if X.dtype != _torch().float64:
        raise TypeError("orthonormalize needs float64 bands")
    nb = X.numel() // ((2 if is_complex else 1) * N)
    _check(lib.qsb_orthonormalize(ctypes.c_int64(N), nb, int(is_complex), _dev_ptr(X), _c_d(dV), _stream_ptr(X)))
    return X


def _i32(a):
    a = np.ascontiguousarray(a, np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _f64(a):
    a = np.ascontiguousarray(a, np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Hamiltonian:
    """Kohn-Sham H = -1/2 FD8 Laplacian + V + V_NL on one periodic grid (device resident)."""

    def __init__(self, nx, ny, nz, dx, dy, dz):
        self.shape = (nx, ny, nz)
        self.spacing = (dx, dy, dz)
        self.N = nx * ny * nz
        h = ctypes.c_void_p()
        _check(lib.qsb_ham_create(ctypes.byref(h), nx, ny, nz, _c_d(dx), _c_d(dy), _c_d(dz)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsb_ham_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_potential(self, V):
        """V: numpy array (host) or CUDA tensor of N float64 values."""
        if hasattr(V, "is_cuda") and V.is_cuda:
            _check(lib.qsb_ham_set_potential(self._h, _dev_ptr(V), 1))
        else:
            v, vp = _f64(V)
            _check(lib.qsb_ham_set_potential(self._h, vp, 0))

    def set_projectors(self, npts, widths, coords, beta, energy):
        """Point-list projector tables (host numpy), as in include/qumasun_b200.h."""
        n, np_ = _i32(npts)
        w, wp = _i32(widths)
        c, cp = _i32(coords)
        b, bp = _f64(beta)
        e, ep = _f64(energy)
        _check(lib.qsb_ham_set_projectors(self._h, len(n), np_, wp, cp, bp, ep))

    def set_gth_projectors(self, pos, species, nl, r_l, h_l, rcut_factor=6.0):
        p, pp = _f64(np.asarray(pos, np.float64).ravel())
        s, sp = _i32(species)
        n, nlp = _i32(nl)
        r, rp = _f64(np.asarray(r_l, np.float64).ravel())
        hh, hp = _f64(np.asarray(h_l, np.float64).ravel())
        _check(lib.qsb_ham_set_gth_projectors(self._h, len(s), pp, sp, len(n), nlp, rp, hp, _c_d(rcut_factor)))

    def projector_info(self):
        tp = ctypes.c_int64()
        tw = ctypes.c_int()
        _check(lib.qsb_ham_projector_info(self._h, ctypes.byref(tp), ctypes.byref(tw)))
        return tp.value, tw.value

    def set_projector_gradients(self, dbeta):
        """dbeta: per atom (d/dx, d/dy, d/dz) blocks of npts x width column-major, concatenated."""
        g = np.ascontiguousarray(dbeta, dtype=np.float64)
        _check(lib.qsb_ham_set_projector_gradients(self._h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def nonlocal_energy(self, psi, occupancies, is_complex=False, g=(0.0, 0.0, 0.0)):
        nb = self._nb(psi, is_complex)
        occ = np.ascontiguousarray(occupancies, dtype=np.float64)
        assert occ.size == nb
        e = ctypes.c_double()
        _check(lib.qsb_ham_nonlocal_energy(self._h, _dtype_code(psi), int(is_complex), nb, _dev_ptr(psi),
                                           occ.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _c_d(g[0]),
                                           _c_d(g[1]), _c_d(g[2]), ctypes.byref(e), _stream_ptr(psi)))
        return e.value

    def nonlocal_energy_force(self, psi, occupancies, n_atoms, is_complex=False, g=(0.0, 0.0, 0.0)):
        """(energy, forces[n_atoms, 3]) of the nonlocal part."""
        nb = self._nb(psi, is_complex)
        occ = np.ascontiguousarray(occupancies, dtype=np.float64)
        assert occ.size == nb
        f = np.zeros((n_atoms, 3))
        e = ctypes.c_double()
        _check(lib.qsb_ham_nonlocal_energy_force(self._h, _dtype_code(psi), int(is_complex), nb, _dev_ptr(psi),
                                                 occ.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _c_d(g[0]),
                                                 _c_d(g[1]), _c_d(g[2]), ctypes.byref(e),
                                                 f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream_ptr(psi)))
        return e.value, f

    def set_timing(self, enable=True):
        _check(lib.qsb_ham_set_timing(self._h, int(bool(enable))))

    def get_timing(self):
        """(projection_ms, stencil_ms, expansion_ms, applies, kernel_launches) since the last call."""
        pm, sm, em = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n, k = ctypes.c_int(), ctypes.c_int()
        _check(lib.qsb_ham_get_timing(self._h, ctypes.byref(pm), ctypes.byref(sm), ctypes.byref(em), ctypes.byref(n),
                                      ctypes.byref(k)))
        return pm.value, sm.value, em.value, n.value, k.value

    def _nb(self, psi, is_complex):
        return psi.numel() // ((2 if is_complex else 1) * self.N)

    def apply(self, psi, hpsi, is_complex=False, g=(0.0, 0.0, 0.0)):
        """hpsi = H psi."""
        nb = self._nb(psi, is_complex)
        assert hpsi.dtype == psi.dtype and hpsi.numel() == psi.numel()
        _check(lib.qsb_ham_apply(self._h, _dtype_code(psi), int(is_complex), nb, _dev_ptr(psi), _dev_ptr(hpsi),
                                 _c_d(g[0]), _c_d(g[1]), _c_d(g[2]), _stream_ptr(psi)))
        return hpsi

    def set_kinetic(self, algorithm):
        """0: FD8 Laplacian (default); 1: FFT kinetic (the reference's default operator)."""
        _check(lib.qsb_ham_set_kinetic(self._h, int(algorithm)))

    def apply_host(self, psi, hpsi, is_complex=False, g=(0.0, 0.0, 0.0), chunk_bands=0):
        """hpsi = H psi for contiguous CPU tensors (pinned ones let the copies
        overlap), chunked through the device on the current CUDA stream;
        hpsi is complete once that stream is synchronized."""
        torch = _torch()
        if psi.is_cuda or hpsi.is_cuda or not (psi.is_contiguous() and hpsi.is_contiguous()):
            raise ValueError("expected contiguous CPU tensors")
        assert hpsi.dtype == psi.dtype and hpsi.numel() == psi.numel()
        nb = self._nb(psi, is_complex)
        _check(lib.qsb_ham_apply_host(self._h, _dtype_code(psi), int(is_complex), nb, _vp(psi.data_ptr()),
                                      _vp(hpsi.data_ptr()), _c_d(g[0]), _c_d(g[1]), _c_d(g[2]), int(chunk_bands),
                                      _vp(torch.cuda.current_stream().cuda_stream)))
        return hpsi

    def nonlocal_apply(self, psi, hpsi, is_complex=False, g=(0.0, 0.0, 0.0)):
        """hpsi += V_NL psi."""
        nb = self._nb(psi, is_complex)
        _check(lib.qsb_ham_nonlocal_apply(self._h, _dtype_code(psi), int(is_complex), nb, _dev_ptr(psi),
                                          _dev_ptr(hpsi), _c_d(g[0]), _c_d(g[1]), _c_d(g[2]), _stream_ptr(psi)))
        return hpsi

    def nonlocal_project(self, psi, is_complex=False, g=(0.0, 0.0, 0.0)):
        """<beta|psi> dV as a numpy [ncol, total_projectors] array."""
        nb = self._nb(psi, is_complex)
        _, P = self.projector_info()
        out = np.zeros(((2 if is_complex else 1) * nb, max(P, 1)))
        _check(lib.qsb_ham_nonlocal_project(self._h, _dtype_code(psi), int(is_complex), nb, _dev_ptr(psi),
                                            _c_d(g[0]), _c_d(g[1]), _c_d(g[2]),
                                            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _stream_ptr(psi)))
        return out[:, :P]


APPLY_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                            ctypes.c_void_p)


class EigenSolver:
    """Device block LOBPCG (qsb_lobpcg_z ~ LOBPCG::Eigen_z_multi_mpi, qsb_lobpcg_d ~
    EigenLOBPCG_d_multi) for bundles of up to n bands of N points."""

    PRECISIONS = {"fp64": 0, "mixed": 1}

    def __init__(self, N, n, is_complex, precision="fp64"):
        """precision "fp64" (the reference's arithmetic) or "mixed" (fp32 bundles
        and operator, tensor-core Gram / rotation products, fp64 pencil)."""
        h = ctypes.c_void_p()
        _check(lib.qsb_eigensolver_create_ex(ctypes.byref(h), ctypes.c_int64(N), n, int(bool(is_complex)),
                                             self.PRECISIONS[precision]))
        self._h = h
        self.N, self.n, self.is_complex, self.precision = N, n, bool(is_complex), precision
        self._cb = None

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsb_eigensolver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_hamiltonian(self, ham, g=(0.0, 0.0, 0.0)):
        self._ham = ham
        _check(lib.qsb_eigensolver_set_hamiltonian(self._h, ham._h, _c_d(g[0]), _c_d(g[1]), _c_d(g[2])))

    def set_operator(self, fn):
        """fn(nb, x_ptr, ax_ptr, stream_ptr) -> int, device pointers as ints."""
        def tramp(user, nb, x, ax, stream):
            try:
                return int(fn(nb, x, ax, stream))
            except Exception:
                return 4
        self._cb = APPLY_FN(tramp)
        _check(lib.qsb_eigensolver_set_operator(self._h, self._cb, None))

    def set_operator_f32(self, fn):
        """Mixed precision: fn(nb, x_ptr, ax_ptr, stream_ptr) -> int on fp32 bundles."""
        def tramp(user, nb, x, ax, stream):
            try:
                return int(fn(nb, x, ax, stream))
            except Exception:
                return 4
        self._cb = APPLY_FN(tramp)
        _check(lib.qsb_eigensolver_set_operator_f32(self._h, self._cb, None))

    def set_drop_tolerance(self, tol):
        _check(lib.qsb_eigensolver_set_drop_tolerance(self._h, _c_d(tol)))

    GRAM_KINDS = {"bf16x3": 3, "bf16x4": 4, "int8_ozaki": 8}

    def set_gram_kind(self, kind):
        """"bf16x3", "bf16x4" or "int8_ozaki" (the default) for the mixed-precision Gram products."""
        _check(lib.qsb_eigensolver_set_gram_kind(self._h, self.GRAM_KINDS[kind]))

    def solve_stats(self):
        """(Cholesky solves, overlap-basis fallbacks) of the last call (mixed precision)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib.qsb_eigensolver_solve_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def set_pencil_update(self, mode):
        """FP64 complex solver: 1 (default) the reference's steady-state pencil
        update between full recomputes every 6 iterations; 0 every block from
        the bundles in every iteration."""
        _check(lib.qsb_eigensolver_set_pencil_update(self._h, int(mode)))

    def pencil_stats(self):
        """(pencils formed in full, pencils formed by the steady-state update) of
        the last FP64 complex call."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib.qsb_eigensolver_pencil_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def overlap_stats(self):
        """(most directions dropped in one iteration, smallest kept overlap
        eigenvalue / largest, drop tolerance) of the last call (mixed precision)."""
        d, r, t = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        _check(lib.qsb_eigensolver_overlap_stats(self._h, ctypes.byref(d), ctypes.byref(r), ctypes.byref(t)))
        return d.value, r.value, t.value

    def last_stats(self):
        it, rb = ctypes.c_int(), ctypes.c_int()
        _check(lib.qsb_eigensolver_last_stats(self._h, ctypes.byref(it), ctypes.byref(rb)))
        return it.value, rb.value

    def lobpcg_z(self, dV, n, iter_max, eigen_values, X, keep, num_fix, residual_threshold, scf_step):
        """In place on X, keep (CUDA) and eigen_values (numpy float64); returns the new num_fix."""
        assert eigen_values.dtype == np.float64 and eigen_values.flags.c_contiguous
        nf = ctypes.c_int(int(num_fix))
        _check(lib.qsb_lobpcg_z(self._h, _c_d(dV), n, iter_max,
                                eigen_values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dev_ptr(X),
                                _dev_ptr(keep), ctypes.byref(nf), _c_d(residual_threshold), int(scf_step),
                                _stream_ptr(X)))
        return nf.value

    def lobpcg_d(self, dV, n, iter_max, eigen_values, X, keep, is_first_time):
        assert eigen_values.dtype == np.float64 and eigen_values.flags.c_contiguous
        _check(lib.qsb_lobpcg_d(self._h, _c_d(dV), n, iter_max,
                                eigen_values.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), _dev_ptr(X),
                                _dev_ptr(keep), int(bool(is_first_time)), _stream_ptr(X)))


def density(X, occupations, N):
    """rho = sum_n occ_n X_n^2 (qsb_density ~ SetDensityOne); X: [nb, N] fp64 CUDA."""
    torch = _torch()
    occ, occ_p = _f64(occupations)
    rho = torch.empty(N, dtype=torch.float64, device=X.device)
    _check(lib.qsb_density(ctypes.c_int64(N), len(occ), _dev_ptr(X), occ_p, _dev_ptr(rho), _stream_ptr(X)))
    return rho


class Upf:
    """A UPF (v2, ONCV) pseudopotential's radial data (qsb_upf_load)."""

    def __init__(self, path):
        h = ctypes.c_void_p()
        _check(lib.qsb_upf_load(ctypes.byref(h), os.fsencode(path)))
        self._h = h
        n, ng = ctypes.c_int(), ctypes.c_int()
        zv = ctypes.c_double()
        cut, cut_p = _f64(np.zeros(4))
        xi, xi_p = _f64(np.zeros(2))
        _check(lib.qsb_upf_info(h, ctypes.byref(n), ctypes.byref(zv), ctypes.byref(ng), cut_p, xi_p))
        self.n_projectors, self.z_valence, self.n_grid = n.value, zv.value, ng.value
        self.cutoff_l, self.xi = cut, xi
        r, r_p = _f64(np.zeros(ng.value))
        v, v_p = _f64(np.zeros(ng.value))
        l, l_p = _i32(np.zeros(max(n.value, 1), np.int32))
        e, e_p = _f64(np.zeros(max(n.value, 1)))
        pr, pr_p = _f64(np.zeros(max(n.value, 1) * ng.value))
        _check(lib.qsb_upf_radial(h, r_p, v_p, l_p, e_p, pr_p))
        self.radius, self.v_local = r, v
        self.l, self.energy = l[:n.value].copy(), e[:n.value].copy()
        self.projectors = pr[: n.value * ng.value].reshape(n.value, ng.value)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsb_upf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radial_local_table(radius, v, z, n_g, dg, sigma=0.5):
    """v(G) on G = j dg of a radial local potential with tail -z/r (qsb_radial_local_table)."""
    r, r_p = _f64(np.asarray(radius, np.float64).ravel())
    vv, v_p = _f64(np.asarray(v, np.float64).ravel())
    assert r.size == vv.size
    t, t_p = _f64(np.zeros(int(n_g)))
    _check(lib.qsb_radial_local_table(r.size, r_p, v_p, _c_d(z), _c_d(sigma), int(n_g), _c_d(dg), t_p))
    return t


def upf_grid_tables(upfs, pos, species, spacing, gradients=True):
    """Projector tables of atoms at pos [n, 3] (species index into upfs) on a grid
    of the given spacing (qsb_upf_grid_tables): (entry_atom, (npts, widths,
    coords, beta, energy), dbeta or None) -- the tables as
    Hamiltonian.set_projectors takes them."""
    arr = (ctypes.c_void_p * len(upfs))(*[u._h.value for u in upfs])
    p, p_p = _f64(np.asarray(pos, np.float64).reshape(-1, 3))
    sp, sp_p = _i32(np.asarray(species, np.int32).ravel())
    ne, npt, nv = ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
    dx, dy, dz = spacing
    args = (arr, len(upfs), len(p), p_p, sp_p, _c_d(dx), _c_d(dy), _c_d(dz), ctypes.byref(ne), ctypes.byref(npt),
            ctypes.byref(nv))
    _check(lib.qsb_upf_grid_tables(*args, None, None, None, None, None, None, None))
    ea, ea_p = _i32(np.zeros(max(ne.value, 1), np.int32))
    npts, npts_p = _i32(np.zeros(max(ne.value, 1), np.int32))
    w, w_p = _i32(np.zeros(max(ne.value, 1), np.int32))
    c, c_p = _i32(np.zeros(max(3 * npt.value, 1), np.int32))
    b, b_p = _f64(np.zeros(max(nv.value, 1)))
    e, e_p = _f64(np.zeros(max(16 * ne.value, 1)))
    g, g_p = (_f64(np.zeros(max(3 * nv.value, 1))) if gradients else (None, None))
    _check(lib.qsb_upf_grid_tables(*args, ea_p, npts_p, w_p, c_p, b_p, e_p, g_p))
    n = ne.value
    tables = (npts[:n].copy(), w[:n].copy(), c[: 3 * npt.value].copy(), b[: nv.value].copy(),
              e[: int(w[:n].sum())].copy())
    return ea[:n].copy(), tables, (g[: 3 * nv.value].copy() if gradients else None)


def cube_write(path, field, grid, axis, origin=(0.0, 0.0, 0.0), Z=(), pos=(), comment=""):
    """Writes field (nx*ny*nz values, x fastest) as a cube file in the
    reference's dialect (qsb_cube_write).  axis: the three box edge vectors."""
    nx, ny, nz = (int(v) for v in grid)
    f, f_p = _f64(np.asarray(field, np.float64).ravel())
    assert f.size == nx * ny * nz
    ax, ax_p = _f64(np.asarray(axis, np.float64).ravel())
    org, org_p = _f64(np.asarray(origin, np.float64).ravel())
    z, z_p = _i32(np.asarray(Z, np.int32).ravel())
    p, p_p = _f64(np.asarray(pos, np.float64).ravel())
    assert ax.size == 9 and org.size == 3 and p.size == 3 * z.size
    _check(lib.qsb_cube_write(os.fsencode(path), comment.encode(), nx, ny, nz, ax_p, org_p, int(z.size),
                              z_p if z.size else None, p_p if z.size else None, f_p))


def cube_read(path):
    """(field [nx*ny*nz], x fastest; dict with grid, axis [3, 3], origin, Z, pos [n, 3])."""
    grid = (ctypes.c_int * 3)()
    ax, ax_p = _f64(np.zeros(9))
    org, org_p = _f64(np.zeros(3))
    na = ctypes.c_int()
    _check(lib.qsb_cube_read_header(os.fsencode(path), grid, ax_p, org_p, ctypes.byref(na)))
    g = tuple(grid)
    f, f_p = _f64(np.zeros(g[0] * g[1] * g[2]))
    z, z_p = _i32(np.zeros(max(na.value, 1), np.int32))
    p, p_p = _f64(np.zeros(3 * max(na.value, 1)))
    _check(lib.qsb_cube_read(os.fsencode(path), f_p, z_p, p_p))
    n = na.value
    return f, {"grid": g, "axis": ax.reshape(3, 3), "origin": org, "Z": z[:n].copy(), "pos": p[:3 * n].reshape(n, 3)}


def write_states(directory, header, bundle, eigen_values, grid, box, Z=(), pos=(), is_complex=True, sk=0,
                 n_kpoints=1, kpoint=(0, 1, 0, 1, 0, 1), list_name=None):
    """Writes a band bundle (host array: complex SoA [n, 2, N] or real [n, N])
    as the reference's state files (its Output.StateVector writer,
    source/qumasun_base1.output.h:250-365): per band n the cube files
    {header}_{up|down}_k{k}_n{n}_re.cube and _im.cube with the comment
    "eigenvalue=..., kpoint=kx/nx,ky/ny,kz/nz", box axes on the diagonal, origin
    0; sk < n_kpoints is spin up.  Real bands get a zero imaginary file.  With
    list_name, also the list of file names (re, im per band) the reference's
    Initial.State reads.  Returns the file names."""
    nx, ny, nz = (int(v) for v in grid)
    N = nx * ny * nz
    b = np.asarray(bundle, np.float64).reshape(-1, 2, N) if is_complex else \
        np.asarray(bundle, np.float64).reshape(-1, N)
    axis = np.diag(np.asarray(box, np.float64))
    tag = ("_up" if sk < n_kpoints else "_down") + "_k%d" % (sk % n_kpoints)
    names = []
    for n in range(b.shape[0]):
        comment = "eigenvalue=%.10f, kpoint=%d/%d,%d/%d,%d/%d" % ((float(eigen_values[n]),) + tuple(kpoint))
        re = b[n, 0] if is_complex else b[n]
        im = b[n, 1] if is_complex else np.zeros(N)
        for part, field in (("_re", re), ("_im", im)):
            name = "%s%s_n%d%s.cube" % (header, tag, n, part)
            cube_write(os.path.join(directory, name), field, (nx, ny, nz), axis, (0.0, 0.0, 0.0), Z, pos, comment)
            names.append(name)
    if list_name:
        with open(os.path.join(directory, list_name), "w") as f:
            f.writelines(n + "\n" for n in names)
    return names


def read_states(list_path, directory=None):
    """Reads the state files a list names (re, im per band, the order of the
    reference's Initial.State lists, source/qumasun_base1.initialize.h:455-540):
    returns (bundle [n, 2, N] complex SoA, eigen_values [n] from each re file's
    "eigenvalue=" comment, header of the first file).  Relative names resolve
    against directory (default: the list's folder)."""
    base = directory if directory is not None else os.path.dirname(os.path.abspath(list_path))
    with open(list_path) as f:
        names = [l.strip() for l in f if l.strip()]
    if len(names) % 2:
        raise ValueError("state list: re and im files come in pairs")
    bands, evs, hdr0 = [], [], None
    for i in range(0, len(names), 2):
        pair = []
        for name in names[i:i + 2]:
            if name.startswith("["):
                raise ValueError("state list: operation keys ([...]) are not supported: " + name)
            path = name if os.path.isabs(name) else os.path.join(base, name)
            field, hdr = cube_read(path)
            if hdr0 is None:
                hdr0 = hdr
            elif hdr["grid"] != hdr0["grid"]:
                raise ValueError("state list: grids differ between files")
            pair.append(field)
            if len(pair) == 1:
                with open(path) as f:
                    f.readline()
                    comment = f.readline()
                k = comment.find("eigenvalue=")
                evs.append(float(comment[k + 11:].split(",")[0]) if k >= 0 else 0.0)
        bands.append(np.stack(pair))
    return np.stack(bands), np.array(evs), hdr0


def ewald(pos, charge, cell):
    """(energy, forces [n_atoms, 3]) of point charges in an orthorhombic cell
    with a neutralising background (qsb_ewald; host code)."""
    p, p_p = _f64(np.asarray(pos, np.float64).reshape(-1, 3))
    q, q_p = _f64(np.asarray(charge, np.float64).ravel())
    c, c_p = _f64(np.asarray(cell, np.float64).ravel())
    assert len(q) == len(p) and len(c) == 3
    f, f_p = _f64(np.zeros(3 * len(p)))
    e = ctypes.c_double()
    _check(lib.qsb_ewald(len(p), p_p, q_p, c_p, ctypes.byref(e), f_p))
    return e.value, f.reshape(len(p), 3)


def gga_pbe(rho, grid):
    """(energy density, v_xc) of spin-unpolarised GGA-PBE on a periodic grid
    (qsb_gga_pbe ~ the GGA branch of mSetPotentialVxc); grid = (nx, ny, nz, dx, dy, dz)."""
    torch = _torch()
    nx, ny, nz, dx, dy, dz = grid
    assert rho.numel() == nx * ny * nz
    exc, vxc = torch.empty_like(rho), torch.empty_like(rho)
    _check(lib.qsb_gga_pbe(int(nx), int(ny), int(nz), _c_d(dx), _c_d(dy), _c_d(dz), _dev_ptr(rho), _dev_ptr(exc),
                           _dev_ptr(vxc), _stream_ptr(rho)))
    return exc, vxc


def lda_pz(rho):
    """(rho eps_xc, v_xc) of the Perdew-Zunger LDA (qsb_lda_pz ~ Calc_XC_LDA)."""
    torch = _torch()
    exc, vxc = torch.empty_like(rho), torch.empty_like(rho)
    _check(lib.qsb_lda_pz(ctypes.c_int64(rho.numel()), _dev_ptr(rho), _dev_ptr(exc), _dev_ptr(vxc),
                          _stream_ptr(rho)))
    return exc, vxc


class SCF:
    """Device SCF loop (qsb_scf_* ~ QUMASUN_KPOINT::Execute with the LOBPCG
    solver): Gamma point, LDA, GTH local part, Fermi smearing, Kerker-DIIS."""

    def __init__(self, ham, solver, nb, num_electrons):
        h = ctypes.c_void_p()
        _check(lib.qsb_scf_create(ctypes.byref(h), ham._h, solver._h, nb, _c_d(num_electrons)))
        self._h, self._ham, self._es, self.nb = h, ham, solver, nb
        self.N = solver.N

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.qsb_scf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_gth_local(self, pos, species, zion, rloc, c1, c2):
        pos, pos_p = _f64(np.asarray(pos, np.float64).reshape(-1, 3))
        self._n_atoms = len(pos)
        sp, sp_p = _i32(species)
        arrs = [_f64(v) for v in (zion, rloc, c1, c2)]
        _check(lib.qsb_scf_set_gth_local(self._h, len(pos), pos_p, sp_p, len(arrs[0][0]),
                                         *[p for _, p in arrs]))

    def set_radial_local(self, pos, species, z, sigma, dg, tables):
        """Local parts from radial tables (qsb_scf_set_radial_local): tables
        [n_species, n_g] of radial_local_table(radius, v, z[k], n_g, dg, sigma[k])."""
        pos, pos_p = _f64(np.asarray(pos, np.float64).reshape(-1, 3))
        self._n_atoms = len(pos)
        sp, sp_p = _i32(species)
        zz, z_p = _f64(np.asarray(z, np.float64).ravel())
        ss, s_p = _f64(np.asarray(sigma, np.float64).ravel())
        tab = np.ascontiguousarray(np.asarray(tables, np.float64).reshape(len(zz), -1))
        t, t_p = _f64(tab.ravel())
        _check(lib.qsb_scf_set_radial_local(self._h, len(pos), pos_p, sp_p, len(zz), z_p, s_p, tab.shape[1],
                                            _c_d(dg), t_p))

    def set_mixing(self, amplitude=0.5, q0=0.8, depth=6):
        _check(lib.qsb_scf_set_mixing(self._h, _c_d(amplitude), _c_d(q0), depth))

    def set_density_tolerance(self, rho_tol):
        _check(lib.qsb_scf_set_density_tolerance(self._h, _c_d(rho_tol)))

    def set_smearing(self, kbt):
        _check(lib.qsb_scf_set_smearing(self._h, _c_d(kbt)))

    def set_xc(self, pz_variant=0, rho_min=1e-8):
        """XC form (qsb_scf_set_xc): 0 the reference's LDA-PZ, 1 PZ continuous at
        rs = 1 (cut rho_min), 2 GGA-PBE."""
        _check(lib.qsb_scf_set_xc(self._h, int(pz_variant), _c_d(rho_min)))

    def set_polish(self, solver_fp64, max_steps=10, tol_per_atom=0.0, rho_tol=0.0):
        """FP64 polish of a mixed run (qsb_scf_set_polish); solver_fp64=None switches it off."""
        self._polish = solver_fp64
        _check(lib.qsb_scf_set_polish(self._h, solver_fp64._h if solver_fp64 is not None else None,
                                      max_steps if solver_fp64 is not None else 0, _c_d(tol_per_atom),
                                      _c_d(rho_tol)))

    def polish_stats(self):
        """(first polish step or -1, polish steps) of the last run."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib.qsb_scf_polish_stats(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def run(self, X, keep, lobpcg_iters=4, max_steps=60, tol_per_atom=1e-6):
        """Runs to |dE|/atom < tol; X, keep: [nb, N] fp64 CUDA (updated in place).
        Returns (energies per step, final Rayleigh quotients, occupations)."""
        e, e_p = _f64(np.zeros(max_steps))
        ev, ev_p = _f64(np.zeros(self.nb))
        occ, occ_p = _f64(np.zeros(self.nb))
        steps = ctypes.c_int()
        _check(lib.qsb_scf_run(self._h, _dev_ptr(X), _dev_ptr(keep), lobpcg_iters, max_steps, _c_d(tol_per_atom),
                               e_p, ctypes.byref(steps), ev_p, occ_p, _stream_ptr(X)))
        return e[:steps.value].copy(), ev, occ

    _REDUCE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64)

    def set_kpoints(self, kvec, weights, owned=None):
        """k-points of a complex-band SCF (qsb_scf_set_kpoints): kvec [n_k, 3] bohr^-1,
        weights [n_k] summing to 1, owned [n_k] flags of the k-points this context computes."""
        kv, kv_p = _f64(np.asarray(kvec, np.float64).reshape(-1, 3))
        w, w_p = _f64(np.asarray(weights, np.float64).ravel())
        self.n_k = len(w)
        if owned is not None:
            ow, ow_p = _i32(np.asarray(owned, np.int32).ravel())
        else:
            ow, ow_p = None, None
        self._owned = [True] * self.n_k if owned is None else [bool(o) for o in np.asarray(owned).ravel()]
        _check(lib.qsb_scf_set_kpoints(self._h, self.n_k, kv_p, w_p, ow_p))

    def set_reduce(self, fn):
        """fn(array) must replace the float64 numpy array (host) by its sum over the
        contexts sharing the k-points (an allreduce); None: a single context."""
        if fn is None:
            self._reduce_cb = None
            _check(lib.qsb_scf_set_reduce(self._h, None, None))
            return

        def cb(user, buf, count):
            try:
                fn(np.ctypeslib.as_array(buf, shape=(count,)))
                return 0
            except Exception:
                return 1
        self._reduce_cb = self._REDUCE(cb)         # kept alive with the context
        _check(lib.qsb_scf_set_reduce(self._h, self._reduce_cb, None))

    def run_kpoints(self, Xs, keeps, lobpcg_iters=4, max_steps=60, tol_per_atom=1e-6):
        """k-point SCF (qsb_scf_run_kpoints); Xs, keeps: per k-point [nb, 2, N] fp64 CUDA
        bundles (None for k-points owned elsewhere), updated in place.  Returns
        (energies per step, levels [n_k, nb], occupations [n_k, nb])."""
        nk = self.n_k
        ptrs = (ctypes.c_void_p * nk)(*[_dev_ptr(x).value if x is not None else None for x in Xs])
        kptrs = (ctypes.c_void_p * nk)(*[_dev_ptr(x).value if x is not None else None for x in keeps])
        e, e_p = _f64(np.zeros(max_steps))
        ev, ev_p = _f64(np.zeros(nk * self.nb))
        occ, occ_p = _f64(np.zeros(nk * self.nb))
        steps = ctypes.c_int()
        ref = next(x for x in Xs if x is not None)
        _check(lib.qsb_scf_run_kpoints(self._h, ptrs, kptrs, lobpcg_iters, max_steps, _c_d(tol_per_atom), e_p,
                                       ctypes.byref(steps), ev_p, occ_p, _stream_ptr(ref)))
        return e[:steps.value].copy(), ev.reshape(nk, self.nb), occ.reshape(nk, self.nb)

    def local_forces(self, rho=None, n_atoms=None):
        """Forces of the GTH local parts, [n_atoms, 3], from the last output
        density (or a given fp64 CUDA density)."""
        na = n_atoms if n_atoms is not None else self._n_atoms
        f, f_p = _f64(np.zeros(3 * na))
        _check(lib.qsb_scf_local_forces(self._h, _dev_ptr(rho) if rho is not None else None, f_p))
        return f.reshape(na, 3)

    def step_residuals(self):
        """int |rho_out - rho_in| dV / N_e of each step of the last run."""
        buf, buf_p = _f64(np.zeros(4096))
        n = ctypes.c_int()
        _check(lib.qsb_scf_step_residuals(self._h, buf_p, len(buf), ctypes.byref(n)))
        return buf[:n.value].copy()

    def step_seconds(self):
        """Wall seconds of each step of the last run."""
        buf, buf_p = _f64(np.zeros(1024))
        n = ctypes.c_int()
        _check(lib.qsb_scf_step_seconds(self._h, buf_p, len(buf), ctypes.byref(n)))
        return buf[:n.value].copy()

    def relax(self, X, keep, pos, species, projectors, local, fixed=None, lobpcg_iters=4, scf_max_steps=60,
              scf_tol=1e-8, max_iter=50, fmax=1e-4, max_step=0.2, history=5):
        """LBFGS relaxation (qsb_relax_lbfgs) of the atoms at pos [n_atoms, 3];
        projectors = (nl, r_l, h_l, rcut_factor) as set_gth_projectors takes
        them, local = (zion, rloc, c1, c2) as set_gth_local.  X, keep: [nb, N]
        fp64 CUDA, warm states (updated).  Returns (positions, energies per
        step, forces [n_atoms, 3])."""
        p, p_p = _f64(np.asarray(pos, np.float64).reshape(-1, 3).copy())
        na = len(p)
        self._n_atoms = na
        sp, sp_p = _i32(species)
        nl, r_l, h_l, rcut = projectors
        n, n_p = _i32(nl)
        r, r_p = _f64(np.asarray(r_l, np.float64).ravel())
        hh, h_p = _f64(np.asarray(h_l, np.float64).ravel())
        loc = [_f64(v) for v in local]
        fx, fx_p = _i32(np.asarray(fixed, np.int32).ravel()) if fixed is not None else (None, None)
        assert fx is None or len(fx) == na
        e, e_p = _f64(np.zeros(max_iter + 1))
        f, f_p = _f64(np.zeros(3 * na))
        it = ctypes.c_int()
        _check(lib.qsb_relax_lbfgs(self._h, na, p_p, sp_p, len(n), n_p, r_p, h_p, _c_d(rcut),
                                   *[q for _, q in loc], fx_p, _dev_ptr(X), _dev_ptr(keep), lobpcg_iters,
                                   scf_max_steps, _c_d(scf_tol), max_iter, _c_d(fmax), _c_d(max_step), history, e_p,
                                   ctypes.byref(it), f_p, _stream_ptr(X)))
        return p.reshape(na, 3).copy(), e[:it.value + 1].copy(), f.reshape(na, 3)

    def field(self, which):
        """0: output density, 1: V_loc, 2: V_eff, 3: mixed input density."""
        torch = _torch()
        out = torch.empty(self.N, dtype=torch.float64, device="cuda")
        _check(lib.qsb_scf_get_field(self._h, which, _dev_ptr(out)))
        return out
