"""Seeded synthetic fields and QPhiX host-layout packers.

Everything here is host-side numpy: it builds the inputs a QPhiX caller would
hand to the library (gauge links, clover terms, sources) and converts between
the canonical site-major layout and QPhiX's blocked structure-of-arrays host
layout.  None of it is on the timed GPU path.

Canonical layouts (one checkerboard = Vh = Nx*Ny*Nz*Nt/2 sites):
  cb-site index   s = ((t*Nz + z)*Ny + y)*Nxh + xh,  x = 2*xh + ((y+z+t+cb)&1)
                  (include/qphix/qdp_packer_parscalar.h:80-90)
  spinor          complex128[Vh, 4 spin, 3 colour]
  gauge           complex128[2 cb, 4 mu, Vh, 3, 3]   U_mu(x) for x in cb
  clover (packed) float64[Vh, 2 block, 36] = diag[6], offd[15] (re, im)
  full clover     complex128[Vh, 2 block, 6, 6]
"""
from __future__ import annotations

import numpy as np

# ----------------------------------------------------------------------------
# lattice index helpers
# ----------------------------------------------------------------------------


def vh(dims):
    nx, ny, nz, nt = dims
    assert nx % 2 == 0, "Nx must be even for checkerboarding"
    return nx // 2 * ny * nz * nt


def cb_coords(dims, cb):
    """Full coordinates (x, y, z, t) of every site of checkerboard cb."""
    nx, ny, nz, nt = dims
    nxh = nx // 2
    s = np.arange(vh(dims))
    xh = s % nxh
    r = s // nxh
    y = r % ny
    r //= ny
    z = r % nz
    t = r // nz
    x = 2 * xh + ((y + z + t + cb) & 1)
    return x, y, z, t


def lex_to_cb(dims):
    """For every lexicographic site (t, z, y, x order), its (cb, cb-index)."""
    nx, ny, nz, nt = dims
    t, z, y, x = np.meshgrid(np.arange(nt), np.arange(nz), np.arange(ny),
                             np.arange(nx), indexing="ij")
    cb = (x + y + z + t) & 1
    s = ((t * nz + z) * ny + y) * (nx // 2) + x // 2
    return cb, s


# ----------------------------------------------------------------------------
# SU(3) generators
# ----------------------------------------------------------------------------


def _cross_conj(a, b):
    """conj(a x b) for batches of complex 3-vectors."""
    return np.conj(np.cross(a, b))


def reunitarize(m):
    """Gram-Schmidt on rows 0 and 1, row 2 = conj(row0 x row1): an SU(3)
    matrix (det = 1), so the 12-real compressed form reconstructs it."""
    m = np.array(m, dtype=np.complex128, copy=True)
    r0 = m[..., 0, :]
    r0 = r0 / np.linalg.norm(r0, axis=-1, keepdims=True)
    r1 = m[..., 1, :]
    r1 = r1 - np.sum(np.conj(r0) * r1, axis=-1, keepdims=True) * r0
    r1 = r1 / np.linalg.norm(r1, axis=-1, keepdims=True)
    r2 = _cross_conj(r0, r1)
    return np.stack([r0, r1, r2], axis=-2)


def gaussian_complex(rng, shape):
    """Complex Gaussian with unit variance per complex entry."""
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2.0)


def random_su3_gaussian(rng, n):
    """3x3 complex Gaussian matrices reunitarised by Gram-Schmidt."""
    return reunitarize(gaussian_complex(rng, (n, 3, 3)))


def random_su3_exp(rng, n, eps):
    """exp(i eps H), H a random traceless Hermitian 3x3 matrix.

    H is drawn from the Gaussian unitary ensemble (density ~ exp(-tr H^2 / 2):
    unit-variance diagonal, E|H_ij|^2 = 1 off the diagonal) and projected
    traceless.  The exponential is taken through the spectral decomposition
    of the Hermitian matrix (H = V diag(l) V^+, exp(i eps H) =
    V diag(e^{i eps l}) V^+), which is exactly unitary up to rounding;
    det = e^{i eps tr H} = 1.  A final reunitarisation pins det = 1 to the
    last bit for the 12-real form."""
    a = gaussian_complex(rng, (n, 3, 3))

    def expm(lo, hi):
        b = a[lo:hi]
        h = (b + np.conj(np.swapaxes(b, -1, -2))) / np.sqrt(2.0)
        tr = np.trace(h, axis1=-2, axis2=-1) / 3.0
        h = h - tr[:, None, None] * np.eye(3)
        lam, vec = np.linalg.eigh(h)
        ph = np.exp(1j * eps * lam)
        return reunitarize(np.einsum("nij,nj,nkj->nik", vec, ph, np.conj(vec)))

    # the matrices are independent: chunks in threads (numpy releases the GIL
    # in eigh / einsum), results identical to one pass
    chunk = 1 << 18
    if n <= chunk:
        return expm(0, n)
    import concurrent.futures as cf
    import os
    out = np.empty((n, 3, 3), dtype=np.complex128)
    bounds = [(lo, min(n, lo + chunk)) for lo in range(0, n, chunk)]
    with cf.ThreadPoolExecutor(max_workers=min(len(bounds), os.cpu_count() or 1)) as ex:
        for (lo, hi), u in zip(bounds, ex.map(lambda b: expm(*b), bounds)):
            out[lo:hi] = u
    return out


def random_weak_su3(rng, n, factor):
    """1 + factor * Gaussian, reunitarised (the reference tests' random gauge,
    tests/RandomGauge.h:162-172)."""
    m = np.eye(3)[None, :, :] + factor * gaussian_complex(rng, (n, 3, 3))
    return reunitarize(m)


def make_gauge(dims, seed, kind="gaussian", eps=0.3, factor=0.08):
    """Canonical gauge field complex128[2, 4, Vh, 3, 3]."""
    rng = np.random.default_rng(seed)
    n = 2 * 4 * vh(dims)
    if kind == "gaussian":
        u = random_su3_gaussian(rng, n)
    elif kind == "exp":
        u = random_su3_exp(rng, n, eps)
    elif kind == "weak":
        u = random_weak_su3(rng, n, factor)
    elif kind == "unit":
        u = np.broadcast_to(np.eye(3, dtype=np.complex128), (n, 3, 3)).copy()
    else:
        raise ValueError(kind)
    return u.reshape(2, 4, vh(dims), 3, 3)


def gaussian_spinor(dims, seed):
    """Unit-variance complex Gaussian spinor on one checkerboard."""
    rng = np.random.default_rng(seed)
    return gaussian_complex(rng, (vh(dims), 4, 3))


def point_source(dims, spin, colour, cb=1):
    """Unit point source at the origin (if the origin is on cb, else on the
    first site of cb): tests/RandomGauge.h:222-235."""
    f = np.zeros((vh(dims), 4, 3), dtype=np.complex128)
    f[0, spin, colour] = 1.0
    return f


def z2_noise(dims, seed):
    """Entries (+-1 +- i)/sqrt(2)."""
    rng = np.random.default_rng(seed)
    re = rng.integers(0, 2, size=(vh(dims), 4, 3)) * 2 - 1
    im = rng.integers(0, 2, size=(vh(dims), 4, 3)) * 2 - 1
    return (re + 1j * im) / np.sqrt(2.0)


# ----------------------------------------------------------------------------
# clover term (clover-leaf field strength, Chroma normalisation)
# ----------------------------------------------------------------------------

# axis of the (t, z, y, x) full-lattice array for direction mu
_AX = {0: 3, 1: 2, 2: 1, 3: 0}


def gauge_to_full(dims, gauge):
    """canonical [2,4,Vh,3,3] -> full lattice [4, Nt, Nz, Ny, Nx, 3, 3]."""
    nx, ny, nz, nt = dims
    cbm, sm = lex_to_cb(dims)
    full = np.empty((4, nt, nz, ny, nx, 3, 3), dtype=np.complex128)
    for mu in range(4):
        full[mu] = gauge[cbm, mu, sm]
    return full


def _fwd(f, mu):  # f(x + mu)
    return np.roll(f, -1, axis=_AX[mu])


def _bwd(f, mu):  # f(x - mu)
    return np.roll(f, 1, axis=_AX[mu])


def _mm(a, b):
    return np.einsum("...ij,...jk->...ik", a, b)


def _dag(a):
    return np.conj(np.swapaxes(a, -1, -2))


def field_strength(full):
    """Clover-leaf F_{mu nu} = (Q - Q^+)/8 with Q the sum of the four
    plaquette leaves around x (tests/mesfield.cc:25-64): returns the six
    planes (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)."""
    out = []
    for mu in range(3):
        for nu in range(mu + 1, 4):
            umu, unu = full[mu], full[nu]
            unu_xpmu = _fwd(unu, mu)
            umu_xpnu = _fwd(umu, nu)
            # leaf 1: U_mu(x) U_nu(x+mu) U_mu^+(x+nu) U_nu^+(x)
            q = _mm(_mm(umu, unu_xpmu), _mm(_dag(umu_xpnu), _dag(unu)))
            # leaf 2: U_nu(x) U_mu^+(x-mu+nu) U_nu^+(x-mu) U_mu(x-mu)
            umu_m = _bwd(umu, mu)
            unu_m = _bwd(unu, mu)
            umu_mpn = _bwd(umu_xpnu, mu)
            q += _mm(_mm(unu, _dag(umu_mpn)), _mm(_dag(unu_m), umu_m))
            # leaf 3: U_mu^+(x-mu) U_nu^+(x-mu-nu) U_mu(x-mu-nu) U_nu(x-nu)
            umu_mm = _bwd(umu_m, nu)
            unu_mm = _bwd(unu_m, nu)
            unu_n = _bwd(unu, nu)
            q += _mm(_mm(_dag(umu_m), _dag(unu_mm)), _mm(umu_mm, unu_n))
            # leaf 4: U_nu^+(x-nu) U_mu(x-nu) U_nu(x-nu+mu) U_mu^+(x)
            umu_n = _bwd(umu, nu)
            unu_pmn = _bwd(unu_xpmu, nu)
            q += _mm(_mm(_dag(unu_n), umu_n), _mm(unu_pmn, _dag(umu)))
            out.append((q - _dag(q)) * 0.125)
    return out


def clover_tri(f, diag_mass, coeff_r, coeff_t):
    """Pack the clover term 1*diag_mass + sigma.F into two 6x6 Hermitian
    blocks (diag[6], lower-triangle offd[15]) following the tri construction
    of tests/clover_term_qdp_w.h:325-442.  coeff_r / coeff_t are the clover
    coefficients already multiplied by 1/2 (:133-137)."""
    c = [coeff_r, coeff_r, coeff_t, coeff_r, coeff_t, coeff_t]
    f0, f1, f2, f3, f4, f5 = [fi * ci for fi, ci in zip(f, c)]
    shp = f0.shape[:-2]
    diag = np.full(shp + (2, 6), diag_mass, dtype=np.float64)
    offd = np.zeros(shp + (2, 15), dtype=np.complex128)
    for i in range(3):
        r0 = np.imag(f5[..., i, i] - f0[..., i, i])
        diag[..., 0, i] += r0
        diag[..., 0, i + 3] -= r0
        r1 = np.imag(f5[..., i, i] + f0[..., i, i])
        diag[..., 1, i] -= r1
        diag[..., 1, i + 3] += r1
    for i in range(1, 3):
        for j in range(i):
            eij = i * (i - 1) // 2 + j
            etmp = (i + 3) * (i + 2) // 2 + j + 3
            offd[..., 0, eij] = 1j * (f0[..., i, j] - f5[..., i, j])
            offd[..., 0, etmp] = -offd[..., 0, eij]
            offd[..., 1, eij] = 1j * (f5[..., i, j] + f0[..., i, j])
            offd[..., 1, etmp] = -offd[..., 1, eij]
    for i in range(3):
        for j in range(3):
            e = (i + 3) * (i + 2) // 2 + j
            e_minus = 1j * f2[..., i, j] + f4[..., i, j]
            b_minus = 1j * f3[..., i, j] - f1[..., i, j]
            offd[..., 0, e] = b_minus - e_minus
            offd[..., 1, e] = e_minus + b_minus
    packed = np.empty(shp + (2, 36), dtype=np.float64)
    packed[..., :6] = diag
    packed[..., 6::2] = offd.real
    packed[..., 7::2] = offd.imag
    return packed


def make_clover(dims, gauge, mass, csw, csw_t=None):
    """Packed clover term float64[2 cb, Vh, 2, 36] for isotropic Wilson-clover
    with bare mass `mass` (diag = 4 + mass) and coefficient csw."""
    if csw_t is None:
        csw_t = csw
    full = gauge_to_full(dims, gauge)
    f = field_strength(full)
    tri = clover_tri(f, 4.0 + mass, 0.5 * csw, 0.5 * csw_t)
    out = np.empty((2, vh(dims), 2, 36))
    for cb in range(2):
        x, y, z, t = cb_coords(dims, cb)
        out[cb] = tri[t, z, y, x]
    return out


def packed_to_blocks(packed):
    """[..., 2, 36] -> Hermitian complex [..., 2, 6, 6]."""
    shp = packed.shape[:-1]
    a = np.zeros(shp + (6, 6), dtype=np.complex128)
    idx = np.arange(6)
    a[..., idx, idx] = packed[..., :6]
    od = packed[..., 6::2] + 1j * packed[..., 7::2]
    k = 0
    for i in range(1, 6):
        for j in range(i):
            a[..., i, j] = od[..., k]
            a[..., j, i] = np.conj(od[..., k])
            k += 1
    return a


def blocks_to_packed(a):
    shp = a.shape[:-2]
    out = np.empty(shp + (36,))
    idx = np.arange(6)
    out[..., :6] = a[..., idx, idx].real
    k = 0
    for i in range(1, 6):
        for j in range(i):
            out[..., 6 + 2 * k] = a[..., i, j].real
            out[..., 7 + 2 * k] = a[..., i, j].imag
            k += 1
    return out


def invert_clover(packed):
    """Packed A^-1 (exact 6x6 Hermitian inverse per block)."""
    return blocks_to_packed(np.linalg.inv(packed_to_blocks(packed)))


def twisted_full_inverse(packed, mu):
    """(A + i mu g5)^-1 and (A - i mu g5)^-1 as full 6x6 blocks; g5 = +1 on
    block 0 (spins 0,1) and -1 on block 1 (spins 2,3)."""
    a = packed_to_blocks(packed)
    eye = np.eye(6)
    res = []
    for sgn in (1.0, -1.0):
        m = a.copy()
        m[..., 0, :, :] += 1j * sgn * mu * eye
        m[..., 1, :, :] -= 1j * sgn * mu * eye
        res.append(np.linalg.inv(m))
    return res


def ndtm_clover_inverses(packed, mu, eps):
    """Inverse of the two-flavour block [[A + i mu g5, -eps], [-eps, A - i mu g5]]:
    (Q (A - i mu g5), Q (A + i mu g5)) as full 6x6 blocks and eps Q packed,
    Q = (A^2 + mu^2 - eps^2)^-1 (g5 = +1 on block 0, -1 on block 1)."""
    a = packed_to_blocks(packed)
    eye = np.eye(6)
    q = np.linalg.inv(a @ a + (mu * mu - eps * eps) * eye)
    g5 = np.array([1.0, -1.0])[:, None, None]
    qa = q @ a
    return qa - 1j * mu * g5 * q, qa + 1j * mu * g5 * q, blocks_to_packed(eps * q)


def full_from_packed(packed):
    return packed_to_blocks(packed)


# ----------------------------------------------------------------------------
# QPhiX blocked host layout (include/qphix/geometry.h:115-396,
# include/qphix_codegen/decl_common.h:9-62, qdp_packer_parscalar.h)
# ----------------------------------------------------------------------------


class QPhiXLayout:
    """Index arithmetic of QPhiX's blocked SoA host layout for one
    (V, S, compress12, PadXY, PadXYZ) choice."""

    def __init__(self, dims, veclen, soalen, compress12, pad_xy=0, pad_xyz=0):
        nx, ny, nz, nt = dims
        self.dims = dims
        self.V, self.S, self.c12 = veclen, soalen, compress12
        nxh = nx // 2
        if nxh % soalen:
            raise ValueError("Nx/2 must be divisible by soalen")
        self.nvecs = nxh // soalen
        self.ngy = veclen // soalen
        if ny % self.ngy:
            raise ValueError("Ny must be divisible by veclen/soalen")
        self.pxy = self.nvecs * ny + pad_xy
        self.pxyz = self.pxy * nz + pad_xyz
        self.n_spinor_blocks = self.pxyz * nt + 1  # one leading pad block
        self.n_gauge_blocks = (self.pxyz * nt * soalen) // veclen
        s = np.arange(vh(dims))
        xh = s % nxh
        r = s // nxh
        y = r % ny
        r //= ny
        z = r % nz
        t = r // nz
        # spinor: block t*Pxyz + z*Pxy + y*nvecs + xh/S (+1 for the pad block)
        self.sp_block = t * self.pxyz + z * self.pxy + y * self.nvecs + xh // soalen + 1
        self.sp_lane = xh % soalen
        # gauge / clover: block (t*Pxyz + z*Pxy)/ngy + (y/ngy)*nvecs + xh/S
        self.g_block = (t * self.pxyz + z * self.pxy) // self.ngy + (y // self.ngy) * self.nvecs + xh // soalen
        self.g_lane = (y % self.ngy) * soalen + xh % soalen

    # spinor: T[3 col][4 spin][2][S]
    def pack_spinor(self, f, dtype=np.float64):
        out = np.zeros((self.n_spinor_blocks, 3, 4, 2, self.S), dtype=dtype)
        v = np.transpose(f, (0, 2, 1))  # site, col, spin
        out[self.sp_block, :, :, 0, self.sp_lane] = v.real
        out[self.sp_block, :, :, 1, self.sp_lane] = v.imag
        return out

    def unpack_spinor(self, a):
        a = np.asarray(a, dtype=np.float64)
        re = a[self.sp_block, :, :, 0, self.sp_lane]
        im = a[self.sp_block, :, :, 1, self.sp_lane]
        return np.transpose(re + 1j * im, (0, 2, 1))

    # gauge: T[8][2|3][3][2][V]; slot 2mu = U_mu(x-mu), 2mu+1 = U_mu(x);
    # stored element [c][c2] = U(c2, c) (qdp_packer_parscalar.h:94-129)
    def pack_gauge(self, gauge, cb, dtype=np.float64):
        nc = 2 if self.c12 else 3
        out = np.zeros((self.n_gauge_blocks, 8, nc, 3, 2, self.V), dtype=dtype)
        dims = self.dims
        x, y, z, t = cb_coords(dims, cb)
        nx, ny, nz, nt = dims
        for mu in range(4):
            fwd = gauge[cb, mu]
            c = [x, y, z, t]
            c[mu] = (c[mu] - 1) % dims[mu]
            sb = ((c[3] * nz + c[2]) * ny + c[1]) * (nx // 2) + c[0] // 2
            back = gauge[1 - cb, mu, sb]
            for slot, m in ((2 * mu, back), (2 * mu + 1, fwd)):
                mt = np.swapaxes(m, -1, -2)[:, :nc, :]  # [site][c][c2] = U(c2, c)
                out[self.g_block, slot, :, :, 0, self.g_lane] = mt.real
                out[self.g_block, slot, :, :, 1, self.g_lane] = mt.imag
        return out

    def unpack_gauge(self, blocks):
        """Forward links U_mu(x) [4, Vh, 3, 3] of a checkerboard from its
        blocked array (slots 2mu + 1); with 12-real storage the third row of
        U^T (the third column stored) is rebuilt as conj(row0 x row1) of the
        transposed matrix, as the kernels do (codegen/dslash_common.cc:1895-1913)."""
        a = np.asarray(blocks, dtype=np.float64)
        nc = 2 if self.c12 else 3
        out = np.empty((4, vh(self.dims), 3, 3), dtype=np.complex128)
        for mu in range(4):
            mt = a[self.g_block, 2 * mu + 1, :, :, 0, self.g_lane] + 1j * a[self.g_block, 2 * mu + 1, :, :, 1,
                                                                             self.g_lane]
            full = np.empty((mt.shape[0], 3, 3), dtype=np.complex128)
            full[:, :nc] = mt
            if nc == 2:
                full[:, 2] = np.conj(np.cross(mt[:, 0], mt[:, 1]))
            out[mu] = np.swapaxes(full, -1, -2)
        return out

    def unpack_back_gauge(self, blocks):
        """Backward links [4, Vh, 3, 3] stored with a checkerboard (slots 2mu):
        entry mu of site x is U_mu(x - mu), a link of the other checkerboard."""
        a = np.asarray(blocks, dtype=np.float64)
        nc = 2 if self.c12 else 3
        out = np.empty((4, vh(self.dims), 3, 3), dtype=np.complex128)
        for mu in range(4):
            mt = a[self.g_block, 2 * mu, :, :, 0, self.g_lane] + 1j * a[self.g_block, 2 * mu, :, :, 1, self.g_lane]
            full = np.empty((mt.shape[0], 3, 3), dtype=np.complex128)
            full[:, :nc] = mt
            if nc == 2:
                full[:, 2] = np.conj(np.cross(mt[:, 0], mt[:, 1]))
            out[mu] = np.swapaxes(full, -1, -2)
        return out

    # clover: struct {diag1[6][V], off_diag1[15][2][V], diag2[6][V], off_diag2[15][2][V]}
    def pack_clover(self, packed, dtype=np.float64):
        out = np.zeros((self.n_gauge_blocks, 72, self.V), dtype=dtype)
        for b in range(2):
            base = b * 36
            out[self.g_block, base:base + 6, self.g_lane] = packed[:, b, :6]
            out[self.g_block, base + 6:base + 36, self.g_lane] = packed[:, b, 6:]
        return out

    def unpack_clover(self, a):
        a = np.asarray(a, dtype=np.float64)
        out = np.empty((vh(self.dims), 2, 36))
        for b in range(2):
            out[:, b, :] = a[self.g_block, b * 36:(b + 1) * 36, self.g_lane]
        return out

    # full clover: block1[6][6][2][V], block2[6][6][2][V]
    def pack_full_clover(self, full, dtype=np.float64):
        out = np.zeros((self.n_gauge_blocks, 2, 6, 6, 2, self.V), dtype=dtype)
        out[self.g_block, :, :, :, 0, self.g_lane] = full.real
        out[self.g_block, :, :, :, 1, self.g_lane] = full.imag
        return out


# ----------------------------------------------------------------------------
# canonical <-> flat float64 arrays for the oracle
# ----------------------------------------------------------------------------


def spinor_to_real(f):
    return np.ascontiguousarray(np.stack([f.real, f.imag], axis=-1)).reshape(-1)


def real_to_spinor(a, dims):
    a = np.asarray(a).reshape(vh(dims), 4, 3, 2)
    return a[..., 0] + 1j * a[..., 1]


def gauge_to_real(g):
    return np.ascontiguousarray(np.stack([g.real, g.imag], axis=-1)).reshape(-1)


def full_clover_to_real(fc):
    return np.ascontiguousarray(np.stack([fc.real, fc.imag], axis=-1)).reshape(-1)


# ----------------------------------------------------------------------------
# QDP++ / Chroma CB2 full-lattice arrays (site = cb * Vh + cb index, the order
# include/qphix/qdp_packer_parscalar.h:94-110 reads)
# ----------------------------------------------------------------------------


def qdp_spinor(even, odd):
    """full-lattice LatticeFermion [(nrhs,) V, 4, 3] from the two checkerboards"""
    return np.ascontiguousarray(np.concatenate([even, odd], axis=-3))


def qdp_spinor_cb(full, cb):
    """checkerboard cb of a full-lattice spinor (a view)"""
    vhalf = full.shape[-3] // 2
    return full[..., cb * vhalf:(cb + 1) * vhalf, :, :]


def qdp_gauge(gauge):
    """multi1d<LatticeColorMatrix> [4, V, 3, 3] from the canonical [2, 4, Vh, 3, 3]"""
    return np.ascontiguousarray(np.transpose(gauge, (1, 0, 2, 3, 4)).reshape(4, -1, 3, 3))


def qdp_clover(packed):
    """Chroma's clover triangles [V, 72] (diag[2][6], offd[2][15][2] per site)
    from the packed canonical [2 cb, Vh, 2, 36]"""
    p = packed.reshape(-1, 2, 36)
    out = np.empty((p.shape[0], 72))
    for b in range(2):
        out[:, b * 6:(b + 1) * 6] = p[:, b, :6]
        out[:, 12 + b * 30:12 + (b + 1) * 30] = p[:, b, 6:]
    return out


def kappa_to_mass(kappa):
    """M = (4 + m) - D/2 normalisation: kappa = 1/(2(4+m))."""
    return 1.0 / (2.0 * kappa) - 4.0
