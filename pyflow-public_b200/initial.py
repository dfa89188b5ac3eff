"""Seeded, discretely divergence-free initial velocity fields on the staggered grid.

The reference has no spectral initial condition (it starts from NGA restart
files, src/data/initial_conditions.py:57-77); this generator produces the
decaying-turbulence fields the benchmarks use and writes them through the same
restart path.  Host-side numpy FP64; it is input generation, not hot path.

Recipe (per seed):
  1. white Gaussian noise per component, ``np.random.default_rng(seed)``;
  2. shape its DFT to the 3-D energy spectrum E(k) ~ k^4 exp(-2 (k/k0)^2), i.e.
     amplitude sqrt(E(k) / (4 pi k^2)), zero mean;
  3. project onto the kernel of the staggered divergence
     D = sum_d (U_d[i+e_d] - U_d[i]) / h_d, exactly in DFT space:
     U_d <- U_d - conj(g_d) (sum_e g_e U_e) / sum_e |g_e|^2, g_d = (e^{i theta_d} - 1)/h_d,
     so the discrete divergence (src/metric/metric_staggered.py:438-453) is zero
     to round-off;
  4. rescale so <u^2 + v^2 + w^2>/3 = urms^2.
"""
import numpy as np


def spectral_velocity(shape, lengths=(2 * np.pi,) * 3, k0=4.0, urms=1.0,
                      seed=0):
    """Return (u, v, w) float64 arrays of ``shape`` = (nx, ny, nz), layout
    [x][y][z] with z contiguous; u on x-faces, v on y-faces, w on z-faces."""
    nx, ny, nz = (int(n) for n in shape)
    rng = np.random.default_rng(seed)
    noise = [rng.standard_normal((nx, ny, nz)) for _ in range(3)]
    h = [lengths[d] / shape[d] for d in range(3)]
    # physical wavenumbers (integers for a 2*pi box)
    kax = [np.fft.fftfreq(shape[d], d=h[d]) * 2 * np.pi for d in range(3)]
    KX, KY, KZ = np.meshgrid(*kax, indexing="ij")
    kmag = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        ek = kmag ** 4 * np.exp(-2.0 * (kmag / k0) ** 2)
        amp = np.where(kmag > 0, np.sqrt(ek / (4 * np.pi * kmag ** 2)), 0.0)
    hat = [np.fft.fftn(n) * amp for n in noise]
    # exact staggered projection
    th = [2 * np.pi * np.fft.fftfreq(shape[d]) for d in range(3)]
    TX, TY, TZ = np.meshgrid(*th, indexing="ij")
    g = [(np.exp(1j * T) - 1.0) / h[d] for d, T in enumerate((TX, TY, TZ))]
    div = g[0] * hat[0] + g[1] * hat[1] + g[2] * hat[2]
    g2 = (np.abs(g[0]) ** 2 + np.abs(g[1]) ** 2 + np.abs(g[2]) ** 2)
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(g2 > 0, div / g2, 0.0)
    hat = [hat[d] - np.conj(g[d]) * phi for d in range(3)]
    vel = [np.real(np.fft.ifftn(a)) for a in hat]
    e = (np.mean(vel[0] ** 2) + np.mean(vel[1] ** 2) + np.mean(vel[2] ** 2)) / 3
    s = urms / np.sqrt(e) if e > 0 else 0.0
    return tuple(np.ascontiguousarray(a * s) for a in vel)


def box_lengths(shape, lengths=None):
    """Periodic box lengths; default is [0, 2*pi]^3."""
    return tuple(lengths) if lengths is not None else (2 * np.pi,) * 3


def spectral_velocity_device(shape, lengths=(2 * np.pi,) * 3, k0=4.0, urms=1.0,
                             seed=0, device="cuda", noise="host"):
    """Same recipe as :func:`spectral_velocity`, with the FFTs done by torch
    on ``device``; for large grids.  noise='host' draws the same noise as
    spectral_velocity from the same seed (numpy, on the host); noise='device'
    draws it on the device from a torch generator seeded with ``seed`` (a
    different field with the same spectrum, without the host cost).
    Returns FP64 torch tensors."""
    import torch
    nx, ny, nz = (int(n) for n in shape)
    rng = np.random.default_rng(seed)
    gen = None
    if noise == "device":
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed))
    h = [lengths[d] / shape[d] for d in range(3)]
    kax = [torch.tensor(np.fft.fftfreq(shape[d], d=h[d]) * 2 * np.pi,
                        device=device) for d in range(3)]
    th = [torch.tensor(2 * np.pi * np.fft.fftfreq(shape[d]), device=device)
          for d in range(3)]
    KX, KY, KZ = kax[0][:, None, None], kax[1][None, :, None], kax[2][None, None, :]
    kmag = torch.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    ek = kmag ** 4 * torch.exp(-2.0 * (kmag / k0) ** 2)
    amp = torch.where(kmag > 0, torch.sqrt(ek / (4 * np.pi * kmag.clamp_min(1e-300) ** 2)),
                      torch.zeros_like(kmag))
    del ek, kmag
    hat = []
    for _ in range(3):
        if gen is not None:
            nz_ = torch.randn((nx, ny, nz), generator=gen, dtype=torch.float64, device=device)
        else:
            nz_ = torch.from_numpy(rng.standard_normal((nx, ny, nz))).to(device)
        hat.append(torch.fft.fftn(nz_) * amp)
        del nz_
    g = [(torch.exp(1j * th[0]) - 1.0)[:, None, None] / h[0],
         (torch.exp(1j * th[1]) - 1.0)[None, :, None] / h[1],
         (torch.exp(1j * th[2]) - 1.0)[None, None, :] / h[2]]
    div = g[0] * hat[0] + g[1] * hat[1] + g[2] * hat[2]
    g2 = (g[0].abs() ** 2 + g[1].abs() ** 2 + g[2].abs() ** 2)
    phi = torch.where(g2 > 0, div / torch.where(g2 > 0, g2, torch.ones_like(g2)),
                      torch.zeros_like(div))
    del div, g2
    vel = []
    for d in range(3):
        a = hat[d] - torch.conj(g[d]) * phi
        hat[d] = None
        vel.append(torch.fft.ifftn(a).real.contiguous())
        del a
    e = sum(float((v * v).mean()) for v in vel) / 3
    s = urms / np.sqrt(e) if e > 0 else 0.0
    return tuple(v * s for v in vel)
