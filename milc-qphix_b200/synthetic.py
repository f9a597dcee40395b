"""Seeded synthetic lattice fields in MILC's raw even-first layout.

Inputs for the tests and the benchmark; nothing here is on the solver path.

Raw layout (what MILC hands to ``QPHIX_*_create_*_from_raw``, read by the
reference at qphix_f3.cpp:93-121 and :980-1018):

* sites are split by parity, even block first; inside a block the index is
  ``i = ((t*Nz + z)*Ny + y)*Nxh + x//2`` (qphix_f3.cpp:95-100), the odd block
  starts at ``V/2``;
* a colour vector is 6 reals per site: ``v[6*i + 2*c + ri]``;
* a link field is 72 reals per site: ``u[72*i + 18*dir + 6*row + 2*col + ri]``
  with ``dir`` = x, y, z, t;
* ``fatback``/``lngback`` at site x hold the forward link of x-mu (x-3mu for
  the Naik term) shifted to x without taking the adjoint (the convention of
  MILC's QPhiX glue); the stencil applies the adjoint and the minus sign.

Gauge fields follow the recipe of the benchmark configurations: random SU(3)
``exp(i*eps*H)`` with ``H`` Gaussian traceless Hermitian (exact exponential by
eigendecomposition in FP64, then re-unitarised), fat links scaled by 0.9, Naik
links by -1/24, MILC staggered phases folded in (x: (-1)^t, y: (-1)^(t+x),
z: (-1)^(t+x+y), t: 1; same sign rule as qphix_f3.cpp:1079), periodic
boundaries.  Random draws come from numpy ``Generator(PCG64(seed))``; the
eigendecomposition runs in torch FP64 on the requested device, so the same
seed gives the same field (to rounding) on CPU and GPU.

``ubench_fields`` restates the reference's analytic micro-benchmark
initialisers (ubench_helper.h:256-364) and ``ubench_checksum`` its weighted
spinor checksum (ubench_helper.h:451-487), expressed in raw layout.
"""
from __future__ import annotations

import numpy as np

DIRS = 4
NAIK = -1.0 / 24.0


class Lattice:
    """Global lattice ``[Nx, Ny, Nz, Nt]`` (MILC ``latsize`` order)."""

    def __init__(self, dims):
        self.dims = tuple(int(d) for d in dims)
        nx, ny, nz, nt = self.dims
        if nx % 2:
            raise ValueError("Nx must be even for even-odd preconditioning")
        self.nx, self.ny, self.nz, self.nt = nx, ny, nz, nt
        self.nxh = nx // 2
        self.V = nx * ny * nz * nt
        self.Vh = self.V // 2

    def raw_coords(self):
        """Coordinates (x, y, z, t) of every raw site index 0..V-1."""
        i = np.arange(self.Vh, dtype=np.int64)
        xh = i % self.nxh
        r = i // self.nxh
        y = r % self.ny
        r //= self.ny
        z = r % self.nz
        t = r // self.nz
        out = []
        for par in (0, 1):
            x = 2 * xh + ((y + z + t + par) & 1)
            out.append((x, y, z, t))
        return tuple(np.concatenate([out[0][k], out[1][k]]) for k in range(4))

    def raw_index(self, x, y, z, t):
        """Raw index of full-lattice coordinates (arrays allowed)."""
        x = np.asarray(x) % self.nx
        y = np.asarray(y) % self.ny
        z = np.asarray(z) % self.nz
        t = np.asarray(t) % self.nt
        par = (x + y + z + t) & 1
        return (((t * self.nz + z) * self.ny + y) * self.nxh + x // 2) + par * self.Vh

    def lex_of_raw(self):
        """Lexicographic index (x fastest) of each raw site."""
        x, y, z, t = self.raw_coords()
        return ((t * self.nz + z) * self.ny + y) * self.nx + x


def _torch_device(device):
    import torch

    if device is None:
        device = "cpu"
    return torch, torch.device(device)


def random_su3(n, eps, rng, device=None):
    """``n`` SU(3) matrices ``exp(i*eps*H)`` as complex128 numpy (n,3,3).

    On the CPU the exponential is formed from the eigendecomposition of H; on
    a GPU with ``torch.linalg.matrix_exp`` (both exact to FP64 rounding), then
    re-unitarised.  The Gaussian draws are the same either way."""
    torch, dev = _torch_device(device)
    a = rng.standard_normal((n, 3, 3)) + 1j * rng.standard_normal((n, 3, 3))
    out = np.empty((n, 3, 3), dtype=np.complex128)
    on_gpu = str(dev).startswith("cuda")
    chunk = 1 << 20 if on_gpu else 1 << 21
    for s in range(0, n, chunk):
        A = torch.from_numpy(a[s:s + chunk]).to(dev)
        H = 0.5 * (A + A.mH)
        tr = torch.diagonal(H, dim1=-2, dim2=-1).sum(-1) / 3.0
        H = H - tr[:, None, None] * torch.eye(3, dtype=H.dtype, device=dev)
        if on_gpu:
            U = torch.linalg.matrix_exp(1j * eps * H)
        else:
            w, Q = torch.linalg.eigh(H)
            ph = torch.exp(1j * eps * w.to(torch.complex128))
            U = (Q * ph[:, None, :]) @ Q.mH
        out[s:s + chunk] = _reunitarize(torch, U).cpu().numpy()
    return out


def _reunitarize(torch, U):
    """Gram-Schmidt on rows 0,1; row 2 = conj(row0 x row1): exact SU(3)."""
    r0 = U[:, 0, :]
    r0 = r0 / torch.linalg.vector_norm(r0, dim=-1, keepdim=True)
    r1 = U[:, 1, :]
    r1 = r1 - (r0.conj() * r1).sum(-1, keepdim=True) * r0
    r1 = r1 / torch.linalg.vector_norm(r1, dim=-1, keepdim=True)
    r2 = torch.linalg.cross(r0, r1, dim=-1).conj()
    return torch.stack([r0, r1, r2], dim=1)


def _phases(lat):
    """MILC staggered phases eta_mu(x) on the lexicographic lattice (T,Z,Y,X,4)."""
    t, z, y, x = np.meshgrid(np.arange(lat.nt), np.arange(lat.nz), np.arange(lat.ny),
                             np.arange(lat.nx), indexing="ij")
    eta = np.ones((lat.nt, lat.nz, lat.ny, lat.nx, 4))
    eta[..., 0] = np.where(t & 1, -1.0, 1.0)
    eta[..., 1] = np.where((t + x) & 1, -1.0, 1.0)
    eta[..., 2] = np.where((t + x + y) & 1, -1.0, 1.0)
    return eta


def _roll_axis(mu):
    # lexicographic arrays are indexed [t, z, y, x]
    return 3 - mu


def _shift(a, mu, k):
    """Field value at x + k*mu, i.e. np.roll by -k along the mu axis."""
    return np.roll(a, -k, axis=_roll_axis(mu))


def _smear3(lat, U):
    """One 3-staple smear of thin links U (T,Z,Y,X,4,3,3)."""
    out = U.copy()
    w = 1.0 / 8.0
    for mu in range(4):
        acc = np.zeros_like(U[..., mu, :, :])
        for nu in range(4):
            if nu == mu:
                continue
            Unu = U[..., nu, :, :]
            Umu_xnu = _shift(U[..., mu, :, :], nu, 1)
            Unu_xmu = _shift(Unu, mu, 1)
            acc += Unu @ Umu_xnu @ np.conj(np.swapaxes(Unu_xmu, -1, -2))
            Unu_mnu = _shift(Unu, nu, -1)
            Umu_mnu = _shift(U[..., mu, :, :], nu, -1)
            Unu_mnu_pmu = _shift(Unu_mnu, mu, 1)
            acc += np.conj(np.swapaxes(Unu_mnu, -1, -2)) @ Umu_mnu @ Unu_mnu_pmu
        out[..., mu, :, :] = U[..., mu, :, :] + w * acc
    return out


def _smear3_torch(U, dev):
    """_smear3 on a torch device (same arithmetic; used for large lattices)."""
    import torch
    T = torch.from_numpy(U).to(dev)
    ax = lambda mu: 3 - mu  # noqa: E731  (axis of direction mu in (T,Z,Y,X))
    sh = lambda a, mu, k: torch.roll(a, -k, dims=ax(mu))  # noqa: E731
    adj = lambda a: a.mH  # noqa: E731
    out = T.clone()
    for mu in range(4):
        Umu = T[..., mu, :, :]
        acc = torch.zeros_like(Umu)
        for nu in range(4):
            if nu == mu:
                continue
            Unu = T[..., nu, :, :]
            acc += Unu @ sh(Umu, nu, 1) @ adj(sh(Unu, mu, 1))
            Unu_mnu = sh(Unu, nu, -1)
            acc += adj(Unu_mnu) @ sh(Umu, nu, -1) @ sh(Unu_mnu, mu, 1)
        out[..., mu, :, :] = Umu + acc / 8.0
    return out.cpu().numpy()


def _to_raw_links(lat, Ulex):
    """(T,Z,Y,X,4,3,3) complex -> raw float64 (V*72,)."""
    lex = lat.lex_of_raw()
    flat = Ulex.reshape(lat.V, 4, 3, 3)[lex]
    raw = np.empty((lat.V, 4, 3, 3, 2))
    raw[..., 0] = flat.real
    raw[..., 1] = flat.imag
    return raw.reshape(-1)


def _backlinks(lat, Ulex, hop):
    """Forward link of x - hop*mu placed at x (no adjoint)."""
    out = np.empty_like(Ulex)
    for mu in range(4):
        out[..., mu, :, :] = _shift(Ulex[..., mu, :, :], mu, -hop)
    return out


def links_raw_to_lex(dims, raw):
    """Raw MILC link array (V*72 reals) -> complex (T,Z,Y,X,4,3,3)."""
    lat = Lattice(dims)
    a = np.asarray(raw, dtype=np.float64).reshape(lat.V, 4, 3, 3, 2)
    U = np.empty((lat.V, 4, 3, 3), dtype=np.complex128)
    U[lat.lex_of_raw()] = a[..., 0] + 1j * a[..., 1]
    return U.reshape(lat.nt, lat.nz, lat.ny, lat.nx, 4, 3, 3)


def backlinks_raw(dims, raw, hop):
    """The backward-link array MILC passes beside a forward one: the forward
    link of x - hop*mu placed at x (no adjoint), raw layout."""
    lat = Lattice(dims)
    return _to_raw_links(lat, _backlinks(lat, links_raw_to_lex(dims, raw), hop))


def asqtad_links(dims, seed=1001, eps_fat=0.3, eps_long=0.3, fat_scale=0.9,
                 smear=False, device=None):
    """Random asqtad/HISQ-shaped links in raw layout.

    Returns a dict of float64 arrays ``fat, lng, fatback, lngback`` (V*72 each).
    ``smear=True`` gives the "HISQ-shaped" fat links of the 32^3x64 benchmark:
    one 3-staple smear of eps_fat SU(3) links with staple weight 1/8, then a
    global rescale so the mean of ||F||_Frobenius/sqrt(3) equals ``fat_scale``.
    """
    lat = Lattice(dims)
    rng = np.random.Generator(np.random.PCG64(seed))
    shape = (lat.nt, lat.nz, lat.ny, lat.nx, 4, 3, 3)
    Uf = random_su3(lat.V * 4, eps_fat, rng, device).reshape(shape)
    Ul = random_su3(lat.V * 4, eps_long, rng, device).reshape(shape)
    if smear:
        torch, dev = _torch_device(device)
        Uf = _smear3_torch(Uf, dev) if str(dev).startswith("cuda") else _smear3(lat, Uf)
        norm = np.mean(np.sqrt(np.sum(np.abs(Uf) ** 2, axis=(-1, -2)) / 3.0))
        Uf = Uf * (fat_scale / norm)
    else:
        Uf = Uf * fat_scale
    Ul = Ul * NAIK
    eta = _phases(lat)[..., None, None]
    Uf = Uf * eta
    Ul = Ul * eta
    return {
        "fat": _to_raw_links(lat, Uf),
        "lng": _to_raw_links(lat, Ul),
        "fatback": _to_raw_links(lat, _backlinks(lat, Uf, 1)),
        "lngback": _to_raw_links(lat, _backlinks(lat, Ul, 3)),
    }


def gaussian_source(dims, seed=2002, parity="even"):
    """Gaussian complex colour vector (unit variance per real) in raw layout.

    ``parity`` in {"even", "odd", "evenodd"}; the other block is zero.
    """
    lat = Lattice(dims)
    rng = np.random.Generator(np.random.PCG64(seed))
    v = np.zeros(lat.V * 6)
    if parity in ("even", "evenodd"):
        v[:lat.Vh * 6] = rng.standard_normal(lat.Vh * 6)
    if parity in ("odd", "evenodd"):
        v[lat.Vh * 6:] = rng.standard_normal(lat.Vh * 6)
    return v


def unit_links(dims, naik=NAIK, phases=True):
    """Free-field links: identity fat links, naik*identity long links."""
    lat = Lattice(dims)
    eye = np.broadcast_to(np.eye(3, dtype=np.complex128),
                          (lat.nt, lat.nz, lat.ny, lat.nx, 4, 3, 3)).copy()
    eta = _phases(lat)[..., None, None] if phases else 1.0
    Uf = eye * eta
    Ul = eye * naik * eta
    return {
        "fat": _to_raw_links(lat, Uf),
        "lng": _to_raw_links(lat, Ul),
        "fatback": _to_raw_links(lat, _backlinks(lat, Uf, 1)),
        "lngback": _to_raw_links(lat, _backlinks(lat, Ul, 3)),
    }


def ubench_fields(dims):
    """Analytic inputs of the reference micro-benchmark, in raw layout.

    Spinor (both parity blocks): ubench_helper.h:256-288; fat links (all 8
    internal slots, forward slots -> ``fat``, backward -> ``fatback``):
    init_gauge18 ubench_helper.h:328-364 (scale 9e-3); long links: init_gauge
    :290-326 (scale 4e-3).  Coordinates are the checkerboarded ones the
    reference loops over (t, z, y, xh) at VECLEN=1.
    """
    lat = Lattice(dims)
    i = np.arange(lat.Vh)
    xh = i % lat.nxh
    r = i // lat.nxh
    y = r % lat.ny
    r //= lat.ny
    z = r % lat.nz
    t = r // lat.nz
    c = np.arange(3)[None, :]
    re = t[:, None] * 0.1 + z[:, None] * 0.2 - y[:, None] * 0.3 + xh[:, None] * 0.4 + c * 0.2 - 0.3
    im = -(t[:, None] * 0.1 - z[:, None] * 0.2 + y[:, None] * 0.3 - xh[:, None] * 0.4 - c * 0.2 + 0.4)
    half = np.stack([re, im], axis=-1).reshape(-1)
    spinor = np.concatenate([half, half])

    def gauge(scale):
        d = np.arange(8)[None, :, None, None]
        rr = np.arange(3)[None, None, :, None]
        cc = np.arange(3)[None, None, None, :]
        T = t[:, None, None, None]
        Z = z[:, None, None, None]
        Y = y[:, None, None, None]
        X = xh[:, None, None, None]
        gre = scale * (T * 0.1 - Z * 0.2 + Y * 0.3 - X * 0.4 + rr * 0.1 - cc * 0.2 + 0.3 * d - 0.5)
        gim = -scale * (T * 0.1 + Z * 0.2 - Y * 0.3 + X * 0.4 - rr * 0.1 + cc * 0.2 - 0.3 * d + 0.4)
        g = np.stack([gre, gim], axis=-1)  # (Vh, 8, 3, 3, 2)
        fwd = g[:, 1::2].reshape(lat.Vh, -1)
        bwd = g[:, 0::2].reshape(lat.Vh, -1)
        return np.concatenate([fwd, fwd]).reshape(-1), np.concatenate([bwd, bwd]).reshape(-1)

    fat, fatback = gauge(9.0e-3)
    lng, lngback = gauge(4.0e-3)
    return {"fat": fat, "lng": lng, "fatback": fatback, "lngback": lngback, "spinor": spinor}


def ubench_checksum(dims, v_raw, parity):
    """Weighted spinor checksum of ubench_helper.h:451-487 on one parity block."""
    lat = Lattice(dims)
    i = np.arange(lat.Vh)
    xh = i % lat.nxh
    r = i // lat.nxh
    y = r % lat.ny
    r //= lat.ny
    z = r % lat.nz
    t = r // lat.nz
    c = np.arange(3)[None, :]
    wre = t[:, None] * 0.1 + z[:, None] * 0.2 - y[:, None] * 0.3 + xh[:, None] * 0.4 + c * 0.2 - 0.3
    wim = t[:, None] * 0.1 - z[:, None] * 0.2 + y[:, None] * 0.3 - xh[:, None] * 0.4 - c * 0.2 + 0.4
    blk = np.asarray(v_raw, dtype=np.float64).reshape(2, lat.Vh, 3, 2)[parity]
    return float(np.sum(blk[..., 0] * wre) + np.sum(blk[..., 1] * wim))
