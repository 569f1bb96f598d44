"""UPF (v2, ONCV) input path on the CPU: qsb_upf_load against the reference's
own LoadUPF_ONCV (source/upf_oncv_loader.h:353-1050, compiled into oracle/_ref)
on the pseudopotentials the reference ships, and properties of the grid
projector tables qsb_upf_grid_tables builds from them.

Bars: log grid, channels, KB energies (D_kk / 2) and cutoffs equal the
reference's exactly; resampled projectors and the tail-corrected local
potential equal its values to 1e-14 relative (the same interpolant); on the grid, each column's norm sum beta^2 dV matches
the radial integral to 2e-3 at h = 0.15 bohr, different m of a channel are
orthogonal to 1e-3, and the gradient tables equal central differences of the
tables under an atom shift to 1e-6."""
import os

import numpy as np
import pytest

import oracle as O

PP_DIR = os.path.join(O.REFERENCE_ROOT, "PP", "nc-sr-05_pbe_standard_upf")
needs_pp = pytest.mark.skipif(not (O.ref_available() and os.path.isdir(PP_DIR)),
                              reason="needs the reference's UPF files and oracle/_ref")
SPECIES = ["C", "Al", "Au", "Bi", "Ba", "O", "Si"]


def _path(el):
    return os.path.join(PP_DIR, el + ".upf")


@needs_pp
@pytest.mark.parametrize("el", SPECIES)
def test_radial_data_equals_the_reference_loader(qsb_host, el):
    if not os.path.exists(_path(el)):
        pytest.skip("no %s.upf" % el)
    u = qsb_host.Upf(_path(el))
    r = O.ref_upf_load(_path(el))
    assert u.n_projectors == r["n_projectors"] and int(u.z_valence) == r["z_valence"]
    assert u.n_grid == r["n_grid"]
    assert np.array_equal(u.l, r["l"])
    assert np.array_equal(u.energy, r["energy"])
    assert np.array_equal(u.cutoff_l, r["cutoff_l"])
    assert np.array_equal(u.xi, r["xi"])
    assert np.array_equal(u.radius, r["radius"])
    scale = np.abs(r["projectors"]).max()
    assert np.abs(u.projectors - r["projectors"]).max() <= 1e-14 * scale
    # the local potential after the reference's tail correction
    assert np.abs(u.v_local - r["v_local"]).max() <= 1e-14 * np.abs(r["v_local"]).max()


def _load(qsb_host, el):
    if not os.path.exists(_path(el)):
        pytest.skip("no %s.upf" % el)
    return qsb_host.Upf(_path(el))


@needs_pp
@pytest.mark.parametrize("el", ["C", "Al", "Au"])
def test_grid_tables_norms_and_orthogonality(qsb_host, el):
    u = _load(qsb_host, el)
    h = 0.15
    pos = np.array([[3.01, 2.97, 3.05]])
    ea, (npts, widths, coords, beta, energy), _ = qsb_host.upf_grid_tables([u], pos, [0], (h, h, h), False)
    assert np.all(ea == 0) and widths.sum() == sum(2 * l + 1 for l in u.l) and np.all(widths <= 16)
    # radial norms int beta_k^2 r^2 dr on the log grid (r^3 dxi)
    rad = (u.projectors ** 2 * u.radius[None, :] ** 3).sum(axis=1) * u.xi[1]
    off = 0
    col = 0
    ks = [k for k in range(u.n_projectors) for _ in range(2 * u.l[k] + 1)]
    for e, (n, w) in enumerate(zip(npts, widths)):
        B = beta[off: off + n * w].reshape(w, n)
        G = B @ B.T * h ** 3
        for i in range(w):
            k = ks[col + i]
            assert abs(G[i, i] - rad[k]) <= 2e-3 * rad[k], (el, k, G[i, i], rad[k])
        # columns of one channel (same k, different m) are orthogonal
        for i in range(w):
            for j in range(w):
                if i != j and ks[col + i] == ks[col + j]:
                    assert abs(G[i, j]) <= 1e-3 * np.sqrt(G[i, i] * G[j, j])
        off += n * w
        col += w
    assert np.array_equal(energy, np.array([u.energy[k] for k in ks]))


@needs_pp
def test_wide_species_are_split_into_entries_of_at_most_16(qsb_host):
    u = _load(qsb_host, "Ba")            # s2 p2 d2 f2: 32 columns
    ea, (npts, widths, *_), _ = qsb_host.upf_grid_tables([u, u], np.array([[1.0, 1.0, 1.0], [4.0, 4.0, 4.0]]),
                                                        [0, 1], (0.3, 0.3, 0.3), False)
    assert widths.sum() == 2 * 32 and np.all(widths <= 16)
    assert list(ea) == sorted(ea) and set(ea) == {0, 1}
    assert widths[ea == 0].sum() == 32


@needs_pp
def test_gradient_tables_are_derivatives_of_the_tables(qsb_host):
    u = _load(qsb_host, "Al")
    h, d = 0.2, 1e-5
    R = np.array([[2.03, 1.96, 2.11]])

    def tab(pos):
        ea, (npts, widths, coords, beta, energy), g = qsb_host.upf_grid_tables([u], pos, [0], (h, h, h), True)
        # per entry: point -> column index, the value table and the gradient blocks
        res, voff, poff = [], 0, 0
        for n, w in zip(npts, widths):
            pts = [tuple(p) for p in coords[3 * poff: 3 * (poff + n)].reshape(n, 3)]
            B = beta[voff: voff + n * w].reshape(w, n)
            Gd = g[3 * voff: 3 * (voff + n * w)].reshape(3, w, n) if g is not None else None
            res.append((dict(zip(pts, range(n))), B, Gd))
            voff += n * w
            poff += n
        return res

    base = tab(R)
    for k in range(3):
        rp, rm = R.copy(), R.copy()
        rp[0, k] += d
        rm[0, k] -= d
        tp, tm = tab(rp), tab(rm)
        for (idx0, B0, G0), (idxp, Bp, _), (idxm, Bm, _) in zip(base, tp, tm):
            common = [p for p in idx0 if p in idxp and p in idxm]
            i0 = np.array([idx0[p] for p in common])
            fd = -(Bp[:, [idxp[p] for p in common]] - Bm[:, [idxm[p] for p in common]]) / (2 * d)
            scale = np.abs(G0[k]).max()
            assert np.abs(G0[k][:, i0] - fd).max() <= 1e-6 * scale


def test_missing_file_is_reported(qsb_host, tmp_path):
    with pytest.raises(qsb_host.QsbError, match="cannot open"):
        qsb_host.Upf(str(tmp_path / "none.upf"))
    bad = tmp_path / "bad.upf"
    bad.write_text("<UPF version=\"2.0.1\"><PP_INFO/></UPF>")
    with pytest.raises(qsb_host.QsbError, match="PP_HEADER"):
        qsb_host.Upf(str(bad))


def test_local_table_equals_the_analytic_gth_transform(qsb_host):
    """qsb_radial_local_table on a GTH-form local potential (Z 6, r_loc 0.45,
    C1 -4, C2 0.6) tabulated on a log grid equals the analytic GTH transform the
    SCF driver uses (-4 pi Z e^{-G^2 r^2/2} / G^2 + (2 pi)^{3/2} r^3 e^{-G^2 r^2/2}
    (C1 + C2 (3 - G^2 r^2)); 2 pi Z r^2 + ... at G = 0) to 1e-9 absolute for
    G < 20 bohr^-1, whatever the splitting width sigma."""
    import math
    from scipy.special import erf
    Z, rl, c1, c2 = 6.0, 0.45, -4.0, 0.6
    r = np.exp(-9 + np.arange(2000) * (math.log(15.0) + 9) / 2000)
    x = r / rl
    V = -Z * erf(r / (math.sqrt(2) * rl)) / r + np.exp(-0.5 * x * x) * (c1 + c2 * x * x)
    G = np.arange(400) * 0.05
    g2 = G * G
    e = np.exp(-0.5 * g2 * rl * rl)
    coul = np.where(G > 0, -4 * math.pi * Z * e / np.where(G > 0, g2, 1.0), 2 * math.pi * Z * rl * rl)
    ana = coul + (2 * math.pi) ** 1.5 * rl ** 3 * e * (c1 + c2 * (3 - g2 * rl * rl))
    for sigma in (0.3, 0.45, 0.8):
        t = qsb_host.radial_local_table(r, V, Z, 400, 0.05, sigma)
        assert np.abs(t - ana).max() <= 1e-9, sigma


def test_local_table_rejects_a_grid_that_does_not_start_above_zero_and_increase(qsb_host):
    """A decreasing radius would flip the sign of the Simpson sums and a
    radius <= 0 has no logarithm: both are argument errors."""
    r = np.exp(-9 + np.arange(200) * 0.05)
    V = -1.0 / r
    with pytest.raises(qsb_host.QsbError, match="increase"):
        qsb_host.radial_local_table(r[::-1].copy(), V[::-1].copy(), 1.0, 10, 0.1, 0.5)
    r0 = r.copy()
    r0[0] = 0.0
    with pytest.raises(qsb_host.QsbError, match="increase"):
        qsb_host.radial_local_table(r0, V, 1.0, 10, 0.1, 0.5)
    r0[0] = -r[0]
    with pytest.raises(qsb_host.QsbError, match="increase"):
        qsb_host.radial_local_table(r0, V, 1.0, 10, 0.1, 0.5)


@needs_pp
@pytest.mark.parametrize("el", ["C", "Al"])
def test_local_table_of_a_upf_does_not_depend_on_the_splitting(qsb_host, el):
    u = _load(qsb_host, el)
    t1 = qsb_host.radial_local_table(u.radius, u.v_local, float(int(u.z_valence)), 300, 0.05, 0.4)
    t2 = qsb_host.radial_local_table(u.radius, u.v_local, float(int(u.z_valence)), 300, 0.05, 0.7)
    assert np.abs(t1 - t2).max() <= 1e-6 * np.abs(t1[1:]).max()
