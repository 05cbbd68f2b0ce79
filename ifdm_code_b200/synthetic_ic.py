"""Seeded synthetic initial conditions in the reference's Gadget-1 chunk format.

The reference reads MUSIC/Gadget particle files ``<icpath>.0`` .. ``<icpath>.3``
(``src/gadget_IC.h:259-353``, ``tot_chunks = 4`` at ``src/gadget_IC.h:610``).
Those files are not distributed with the reference, so runs here start from a
lattice of N^3 particles displaced by the Zel'dovich approximation of a seeded
Gaussian random field:

* power spectrum P(k) ~ k^-2.5, normalised to an rms density contrast of 0.02
  on the grid (at a = 1/51, z = 50, by default);
* displacement s(k) = i k / k^2 delta(k), so delta = -div s;
* peculiar velocity v = a H(a) f(a) s with f = Omega_m(a)^0.55, written in the
  Gadget convention v / sqrt(a) in km/s;
* positions in kpc/h in [0, BoxSize), BoxSize = 2 * xmax * 1000 kpc/h, which
  is the box the reference checks against (``src/gadget_IC.h:309``);
* particle mass chosen so the reference's mean density
  ``4 * npart * mass / Box^3 * 1e9 * h^2`` (``src/gadget_IC.h:319``) equals
  rho_c = 3.51059e10 Msun/Mpc^3 (``src/Cosmoinput3D.h:10``);
* particles sorted by x and split into four equal chunks, which is the order
  the reference's slab distribution assumes (``src/gadget_IC.h:412-473``).
"""

from __future__ import annotations

import os
import struct

import numpy as np

H_LITTLE = 0.677
OMEGA_M0 = 0.276
RHOC = 3.51059e10
N_CHUNKS = 4


def gadget_header(npart_chunk: int, npart_total: int, mass_1e10: float, a: float, box: float) -> bytes:
    """The 256-byte ``io_header`` of ``src/gadget_IC.h:17-33`` (type-1 particles only)."""
    npart = [0, npart_chunk, 0, 0, 0, 0]
    mass = [0.0, mass_1e10, 0.0, 0.0, 0.0, 0.0]
    tot = [0, npart_total, 0, 0, 0, 0]
    body = struct.pack("<6i6d2d2i6i2i4d", *npart, *mass, a, 1.0 / a - 1.0, 0, 0, *tot, 0, N_CHUNKS,
                       box, OMEGA_M0, 1.0 - OMEGA_M0, H_LITTLE)
    return body + b"\0" * (256 - len(body))


def write_gadget_chunks(prefix: str, pos: np.ndarray, vel: np.ndarray, mass_1e10: float, a: float,
                        box: float) -> list[str]:
    """Write x-sorted particles as four Gadget-1 files ``prefix.0`` .. ``prefix.3``."""
    n = pos.shape[0]
    if n % N_CHUNKS:
        raise ValueError("particle count must split into 4 equal chunks")
    m = n // N_CHUNKS
    paths = []
    d = os.path.dirname(prefix)
    if d:
        os.makedirs(d, exist_ok=True)
    for c in range(N_CHUNKS):
        p = np.ascontiguousarray(pos[c * m:(c + 1) * m], dtype="<f4")
        v = np.ascontiguousarray(vel[c * m:(c + 1) * m], dtype="<f4")
        ids = np.arange(c * m, (c + 1) * m, dtype="<i4")
        path = f"{prefix}.{c}"
        with open(path, "wb") as f:
            f.write(struct.pack("<i", 256))
            f.write(gadget_header(m, n, mass_1e10, a, box))
            f.write(struct.pack("<i", 256))
            for blk in (p, v):
                f.write(struct.pack("<i", blk.nbytes))
                f.write(blk.tobytes())
                f.write(struct.pack("<i", blk.nbytes))
            f.write(struct.pack("<i", ids.nbytes))
            f.write(ids.tobytes())
            f.write(struct.pack("<i", ids.nbytes))
        paths.append(path)
    return paths


def zeldovich_particles(N: int, xmax: float = 5.0, seed: int = 0, a: float = 1.0 / 51.0,
                        rms_delta: float = 0.02, slope: float = -2.5):
    """Particles (pos kpc/h float32 [N^3,3], vel km/s float32 [N^3,3]), x-sorted,
    plus (mass_1e10, a, box)."""
    box = 2.0 * xmax * 1e3
    Lg = box / N
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((N, N, N))
    wk = np.fft.rfftn(white)
    kf = 2.0 * np.pi * np.fft.fftfreq(N, d=Lg)
    kr = 2.0 * np.pi * np.fft.rfftfreq(N, d=Lg)
    kx = kf[:, None, None]
    ky = kf[None, :, None]
    kz = kr[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (slope / 4.0)
    amp[0, 0, 0] = 0.0
    dk = wk * amp
    delta = np.fft.irfftn(dk, s=(N, N, N), axes=(0, 1, 2))
    dk *= rms_delta / delta.std()
    disp = []
    for kc in (kx, ky, kz):
        disp.append(np.fft.irfftn(1j * kc / k2 * dk, s=(N, N, N), axes=(0, 1, 2)))
    q = (np.arange(N) + 0.5) * Lg
    qx, qy, qz = np.meshgrid(q, q, q, indexing="ij")
    E = np.sqrt(OMEGA_M0 / a**3 + 1.0 - OMEGA_M0)
    f = (OMEGA_M0 / a**3 / E**2) ** 0.55
    # v_pec [km/s] = a * 100 h E f * s[Mpc], s[Mpc] = s[kpc/h] / 1000 / h; Gadget stores v_pec / sqrt(a)
    vfac = np.sqrt(a) * 100.0 * E * f / 1000.0
    pos = np.stack([(qx + disp[0]) % box, (qy + disp[1]) % box, (qz + disp[2]) % box], axis=-1).reshape(-1, 3)
    vel = np.stack([vfac * disp[0], vfac * disp[1], vfac * disp[2]], axis=-1).reshape(-1, 3)
    pos = pos.astype(np.float32)
    pos[pos >= np.float32(box)] = 0.0
    vel = vel.astype(np.float32)
    order = np.argsort(pos[:, 0], kind="stable")
    pos = pos[order]
    vel = vel[order]
    npart_chunk = N**3 // N_CHUNKS
    mass_1e10 = RHOC * box**3 / (N_CHUNKS * npart_chunk * 1e10 * 1e9 * H_LITTLE**2)
    return pos, vel, mass_1e10, a, box


def zeldovich_particles_device(N: int, xmax: float = 5.0, seed: int = 0, a: float = 1.0 / 51.0,
                               rms_delta: float = 0.02, slope: float = -2.5, device: int = 0):
    """The same model as ``zeldovich_particles`` generated on a CUDA device
    with torch (its own random stream, so not the same particles for a given
    seed): large test inputs (512^3 particles) in seconds instead of minutes.
    Returns host numpy arrays like ``zeldovich_particles``."""
    import torch

    dev = torch.device("cuda", device)
    box = 2.0 * xmax * 1e3
    Lg = box / N
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    white = torch.randn((N, N, N), generator=gen, device=dev, dtype=torch.float64)
    dk = torch.fft.rfftn(white)
    del white
    kf = 2.0 * np.pi * torch.fft.fftfreq(N, d=Lg, device=dev, dtype=torch.float64)
    kr = 2.0 * np.pi * torch.fft.rfftfreq(N, d=Lg, device=dev, dtype=torch.float64)
    kx, ky, kz = kf[:, None, None], kf[None, :, None], kr[None, None, :]
    k2 = kx * kx + ky * ky + kz * kz
    k2[0, 0, 0] = 1.0
    amp = k2 ** (slope / 4.0)
    amp[0, 0, 0] = 0.0
    dk *= amp
    del amp
    dk *= rms_delta / torch.fft.irfftn(dk, s=(N, N, N)).std()
    E = np.sqrt(OMEGA_M0 / a**3 + 1.0 - OMEGA_M0)
    f = (OMEGA_M0 / a**3 / E**2) ** 0.55
    vfac = np.sqrt(a) * 100.0 * E * f / 1000.0
    q = (torch.arange(N, device=dev, dtype=torch.float64) + 0.5) * Lg
    pos = torch.empty((N, N, N, 3), device=dev, dtype=torch.float32)
    vel = torch.empty((N, N, N, 3), device=dev, dtype=torch.float32)
    qs = (q[:, None, None], q[None, :, None], q[None, None, :])
    for c, kc in enumerate((kx, ky, kz)):
        s = torch.fft.irfftn(1j * kc / k2 * dk, s=(N, N, N))
        pos[..., c] = ((qs[c] + s) % box).to(torch.float32)
        vel[..., c] = (vfac * s).to(torch.float32)
        del s
    pos = pos.reshape(-1, 3)
    vel = vel.reshape(-1, 3)
    pos[pos >= np.float32(box)] = 0.0
    order = torch.sort(pos[:, 0], stable=True).indices
    pos = pos[order].cpu().numpy()
    vel = vel[order].cpu().numpy()
    npart_chunk = N**3 // N_CHUNKS
    mass_1e10 = RHOC * box**3 / (N_CHUNKS * npart_chunk * 1e10 * 1e9 * H_LITTLE**2)
    return pos, vel, mass_1e10, a, box


def make_ic(prefix: str, N: int, xmax: float = 5.0, seed: int = 0, a: float = 1.0 / 51.0,
            rms_delta: float = 0.02) -> list[str]:
    """Generate and write the four chunk files for an N^3 run; returns their paths."""
    pos, vel, mass, a, box = zeldovich_particles(N, xmax=xmax, seed=seed, a=a, rms_delta=rms_delta)
    return write_gadget_chunks(prefix, pos, vel, mass, a, box)


def read_gadget_chunk(path: str):
    """Read one chunk written in the reference's layout (header dict, pos, vel)."""
    with open(path, "rb") as f:
        raw = f.read()
    (b0,) = struct.unpack_from("<i", raw, 0)
    if b0 != 256:
        raise ValueError("not a Gadget-1 file")
    vals = struct.unpack_from("<6i6d2d2i6i2i4d", raw, 4)
    hdr = dict(npart=vals[0:6], mass=vals[6:12], time=vals[12], redshift=vals[13], npartTotal=vals[16:22],
               num_files=vals[23], BoxSize=vals[24], Omega0=vals[25], OmegaLambda=vals[26],
               HubbleParam=vals[27])
    n = hdr["npart"][1]
    off = 4 + 256 + 4
    pos = np.frombuffer(raw, dtype="<f4", count=3 * n, offset=off + 4).reshape(n, 3)
    off += 8 + 12 * n
    vel = np.frombuffer(raw, dtype="<f4", count=3 * n, offset=off + 4).reshape(n, 3)
    return hdr, pos, vel


def zeldovich_psi(N: int, xmax: float = 5.0, seed: int = 0, a: float = 1.0 / 51.0, rms_delta: float = 0.02,
                  mfdm: float = 2.5e-24, slope: float = -2.5, workers: int = -1) -> np.ndarray:
    """psi at the IC in the reference's units, built on the grid directly.

    Field-level form of the particle recipe above, for grids where writing
    N^3 particles is impractical (the benchmark's 512^3): the CIC density of
    the Zel'dovich lattice is rho = rho_c (1 + delta) to first order, and the
    reference's phase solve (src/gadget_IC.h:157-247) turns the linear
    velocity v = vfac s into theta = a^{3/2} uc vfac/(1000 h) grad^-2 delta
    (kpc/h gradients).  psi = 1.225 sqrt(rho / m_solar) exp(i m/(c^2 hbar) theta)
    as in src/gadget_IC.h:666, rho in Msun/Mpc^3.
    """
    import scipy.fft as sfft

    box = 2.0 * xmax * 1e3
    Lg = box / N
    rng = np.random.default_rng(seed)
    wk = sfft.rfftn(rng.standard_normal((N, N, N), dtype=np.float64), workers=workers)
    kf = (2.0 * np.pi * np.fft.fftfreq(N, d=Lg)).astype(np.float64)
    kr = (2.0 * np.pi * np.fft.rfftfreq(N, d=Lg)).astype(np.float64)
    k2 = kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + kr[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    wk *= k2 ** (slope / 4.0)
    wk[0, 0, 0] = 0.0
    delta = sfft.irfftn(wk, s=(N, N, N), workers=workers)
    scale = rms_delta / delta.std()
    delta *= scale
    wk *= -scale / k2
    pot = sfft.irfftn(wk, s=(N, N, N), workers=workers)  # grad^-2 delta, (kpc/h)^2
    del wk, k2
    E = np.sqrt(OMEGA_M0 / a**3 + 1.0 - OMEGA_M0)
    f = (OMEGA_M0 / a**3 / E**2) ** 0.55
    vfac = np.sqrt(a) * 100.0 * E * f / 1000.0
    m2Mpc, s2Myr = 3.086e22, 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    uc = 1e3 / m2Mpc * s2Myr
    hbar = 6.58211928e-16 / s2Myr
    c = 2.99792458e8 / m2Mpc * s2Myr
    mfdm_solar = mfdm * 1.783e-36 / 1.989e30
    theta = a**1.5 * uc * vfac / (1000.0 * H_LITTLE) * pot
    phase = (mfdm / c**2 / hbar) * theta
    amp = 1.225 * np.sqrt(np.maximum(RHOC * (1.0 + delta), 0.0) / mfdm_solar)
    return (amp * np.exp(1j * phase)).astype(np.complex128)


def zeldovich_psi_device(N: int, xmax: float = 5.0, seed: int = 0, a: float = 1.0 / 51.0, rms_delta: float = 0.02,
                         mfdm: float = 2.5e-24, slope: float = -2.5, device: int = 0):
    """The field-level psi of ``zeldovich_psi`` generated on a CUDA device with
    torch (its own random stream, so not the same field for a given seed), for
    grids whose host generation would need tens of GB (1024^3).  Returns a
    complex128 CUDA tensor of shape (N, N, N) in the reference's units."""
    import torch

    dev = torch.device("cuda", device)
    box = 2.0 * xmax * 1e3
    Lg = box / N
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    wk = torch.fft.rfftn(torch.randn((N, N, N), generator=gen, device=dev, dtype=torch.float64))
    kf = 2.0 * np.pi * torch.fft.fftfreq(N, d=Lg, device=dev, dtype=torch.float64)
    kr = 2.0 * np.pi * torch.fft.rfftfreq(N, d=Lg, device=dev, dtype=torch.float64)
    k2 = kf[:, None, None] ** 2 + kf[None, :, None] ** 2 + kr[None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    wk *= k2 ** (slope / 4.0)
    wk[0, 0, 0] = 0.0
    delta = torch.fft.irfftn(wk, s=(N, N, N))
    scale = rms_delta / float(delta.std())
    delta *= scale
    wk *= -scale / k2
    del k2
    pot = torch.fft.irfftn(wk, s=(N, N, N))
    del wk
    E = np.sqrt(OMEGA_M0 / a**3 + 1.0 - OMEGA_M0)
    f = (OMEGA_M0 / a**3 / E**2) ** 0.55
    vfac = np.sqrt(a) * 100.0 * E * f / 1000.0
    m2Mpc, s2Myr = 3.086e22, 60.0 * 60.0 * 24.0 * 365.0 * 1e6
    uc = 1e3 / m2Mpc * s2Myr
    hbar = 6.58211928e-16 / s2Myr
    c = 2.99792458e8 / m2Mpc * s2Myr
    mfdm_solar = mfdm * 1.783e-36 / 1.989e30
    pot *= (mfdm / c**2 / hbar) * a**1.5 * uc * vfac / (1000.0 * H_LITTLE)  # the phase
    delta += 1.0
    delta.clamp_(min=0.0)
    delta *= RHOC / mfdm_solar
    amp = delta.sqrt_().mul_(1.225)
    psi = torch.polar(amp, pot)
    del amp, pot
    return psi
