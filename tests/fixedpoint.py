"""Test helpers: the library's 16-bit storage formats restated in numpy, and
field variants used by the inner-operator parity tests.

The 16-bit inner solves store
  * links as 16-bit fixed point, q = rint(fp32(x) * (32767 / link_max)) in
    FP32 arithmetic, one link_max = max |FP32 real| over the fat and
    backward fat links and one over the Naik links; the Dslash uses
    q * (link_max / 32767);
  * colour vectors with a per-site norm m = max |FP32 component| of the
    site, q = rint(fp32(v) * (32767 / m)), value q * (m / 32767).
Applying the FP64 oracle Dslash to these rounded inputs isolates the
kernel's own arithmetic (FP32, so ~1e-7 relative) from the storage
rounding.

Storage error bound, for the direct comparison with the FP64 oracle.  Each
real of a link is off by at most Delta_U / 2 (Delta_U = link_max / 32767)
and each vector component by at most Delta_v / 2 (Delta_v = m / 32767 of
its site).  One real of U v then moves by at most 3 Delta_U |v|_max +
3 u_max Delta_v ~ 6 u_max |v|_max / 32767, and the 16 terms of the
Dslash by at most 48 (u_fat + u_naik) |v|_max / 32767: about 5e-4 of
max |D v| for the benchmark fields.  Rounding errors are independent and
of both signs, so the measured error is far below that worst case: 2-3e-5
of max |D v| on 8^4 .. 16x8^3 fields in this emulation, growing slowly
(as the largest of many Gaussian-like errors) with the volume.
"""
from __future__ import annotations

import numpy as np

from conftest import synthetic

F32 = np.float32
Q = F32(32767.0)


def quantize_links(links):
    """Raw links (dict of fat, lng, fatback, lngback) as the 16-bit link
    copy represents them, in float64."""
    f32 = {k: np.asarray(links[k], dtype=np.float32) for k in ("fat", "fatback", "lng", "lngback")}
    m_fat = F32(max(np.abs(f32["fat"]).max(), np.abs(f32["fatback"]).max()))
    m_naik = F32(max(np.abs(f32["lng"]).max(), np.abs(f32["lngback"]).max()))
    out = {}
    for k, m in (("fat", m_fat), ("fatback", m_fat), ("lng", m_naik), ("lngback", m_naik)):
        inv = Q / m
        q = np.rint((f32[k] * inv).astype(np.float32))
        out[k] = q.astype(np.float64) * float(F32(m / Q))
    return out, float(m_fat), float(m_naik)


def quantize_vec(raw):
    """Raw colour vector (6 reals per site) as the 16-bit vector format
    represents it, in float64; also returns the per-site norms."""
    v = np.asarray(raw, dtype=np.float32).reshape(-1, 6)
    m = np.abs(v).max(axis=1)
    safe = np.where(m > 0, m, F32(1.0)).astype(np.float32)
    inv = np.where(m > 0, Q / safe, F32(0.0)).astype(np.float32)
    q = np.rint((v * inv[:, None]).astype(np.float32))
    n = (m * F32(1.0 / 32767.0)).astype(np.float32)
    return (q * n[:, None]).astype(np.float32).astype(np.float64).reshape(-1), m.astype(np.float64)


def storage_bound(links, vin, ref_out):
    """Worst-case relative (max-norm) error of the 16-bit storage (module
    docstring)."""
    u_fat = max(np.abs(links["fat"]).max(), np.abs(links["fatback"]).max())
    u_naik = max(np.abs(links["lng"]).max(), np.abs(links["lngback"]).max())
    return 48.0 * (u_fat + u_naik) * np.abs(vin).max() / 32767.0 / np.abs(ref_out).max()


def naik_phased(dims, links, seed=5):
    """The same links with every Naik link times a random U(1) phase: U(3)
    Naik links times the Naik coefficient, the form of HISQ Naik links
    built from unitarised links (13-real, not 12-real)."""
    V = int(np.prod(dims))
    rng = np.random.default_rng(seed)
    lng = np.asarray(links["lng"]).reshape(V, 4, 9, 2)
    z = lng[..., 0] + 1j * lng[..., 1]
    z = z * np.exp(1j * rng.uniform(-np.pi, np.pi, (V, 4)))[:, :, None]
    out = dict(links)
    out["lng"] = np.stack([z.real, z.imag], axis=-1).reshape(-1)
    out["lngback"] = synthetic.backlinks_raw(dims, out["lng"], 3)
    return out
