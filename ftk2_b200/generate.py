"""Device-side synthetic fields for full-size runs (bench, large tests).

Same definitions as ftk2_b200.synthetic (blob parameters drawn from the same
seeded numpy generator), evaluated on the GPU with torch so that 10^8-vertex
fields take milliseconds instead of minutes.  Values agree with the numpy
version to rounding; tests that compare against the oracle copy the device
field back to the host, so both sides always read identical bytes.
"""
from __future__ import annotations

import numpy as np

from .synthetic import gaussian_blobs


def gaussian_field_device(dims, nt: int, seed: int = 1234, n_blobs: int = 32, dtype=None,
                          noise: float = 0.0, noise_seed: int | None = None, sigma=(4.0, 12.0),
                          drift: float = 0.5, scale: float = 1.0, device: str = "cuda", t0: int = 0):
    """Analytic gradient of a drifting Gaussian sum, shape (nt, [nz,] ny, nx, ndim),
    timesteps t0 .. t0 + nt - 1 (t0 > 0 only without noise),
    multiplied by ``scale`` (e.g. the box side for gradients per box length),
    plus ``noise`` * N(0,1)."""
    import torch
    dtype = dtype or torch.float64
    ndim = len(dims)
    blobs = gaussian_blobs(seed, n_blobs, dims, sigma, drift)
    axes = [torch.arange(n, dtype=torch.float64, device=device) for n in dims]
    shape = tuple(dims[::-1])
    out = torch.empty((nt,) + shape + (ndim,), dtype=dtype, device=device)
    gen = None
    if noise:
        gen = torch.Generator(device=device)
        gen.manual_seed(int(seed + 1 if noise_seed is None else noise_seed))
    for k in range(nt):
        acc = torch.zeros(shape + (ndim,), dtype=torch.float64, device=device)
        for b in range(n_blobs):
            c = blobs["centers"][b] + blobs["vel"][b] * (k + t0)
            s2 = float(blobs["sigma"][b]) ** 2
            d = []
            for i in range(ndim):
                view = [1] * ndim
                view[ndim - 1 - i] = dims[i]
                d.append((axes[i] - float(c[i])).view(view))
            r2 = d[0] * d[0]
            for i in range(1, ndim):
                r2 = r2 + d[i] * d[i]
            e = float(blobs["amps"][b]) * torch.exp(-r2 / (2.0 * s2)) / s2
            for i in range(ndim):
                acc[..., i] -= (e * d[i]).expand(shape)
        if scale != 1.0:
            acc *= scale
        if noise:
            acc += noise * torch.randn(acc.shape, dtype=torch.float64, device=device, generator=gen)
        out[k] = acc.to(dtype)
    return out


def gaussian_potential_device(dims, nt: int, seed: int = 1234, n_blobs: int = 32, sigma=(4.0, 12.0),
                              drift: float = 0.5, device: str = "cuda"):
    """The drifting Gaussian sum itself, sum_b A_b exp(-|p - c_b(t)|^2 / (2 s_b^2)),
    float64, shape (nt, [nz,] ny, nx): the scalar whose gradient
    gaussian_field_device returns (same blob draws), for level sets."""
    import torch
    ndim = len(dims)
    blobs = gaussian_blobs(seed, n_blobs, dims, sigma, drift)
    axes = [torch.arange(n, dtype=torch.float64, device=device) for n in dims]
    shape = tuple(dims[::-1])
    out = torch.empty((nt,) + shape, dtype=torch.float64, device=device)
    for k in range(nt):
        acc = torch.zeros(shape, dtype=torch.float64, device=device)
        for b in range(n_blobs):
            c = blobs["centers"][b] + blobs["vel"][b] * k
            s2 = float(blobs["sigma"][b]) ** 2
            r2 = None
            for i in range(ndim):
                view = [1] * ndim
                view[ndim - 1 - i] = dims[i]
                d = ((axes[i] - float(c[i])) ** 2).view(view)
                r2 = d if r2 is None else r2 + d
            acc += float(blobs["amps"][b]) * torch.exp(-r2 / (2.0 * s2))
        out[k] = acc
    return out


def c2_field(device: str = "cuda"):
    """3D flow critical points, plain drop-in: 128^3 x 16, 32 blobs, float64."""
    import torch
    return gaussian_field_device((128, 128, 128), 16, seed=1234, n_blobs=32, dtype=torch.float64,
                                 device=device)


def c4_field(device: str = "cuda"):
    """Precision workload: 256^3 x 8 float32, 64 blobs of width U[16,48] voxels,
    gradient per box length (x256) plus 1e-3 N(0,1) noise."""
    import torch
    return gaussian_field_device((256, 256, 256), 8, seed=4321, n_blobs=64, dtype=torch.float32,
                                 noise=1e-3, sigma=(16.0, 48.0), scale=256.0, device=device)


def gaussian_at_device(points, nt: int, seed: int = 1234, n_blobs: int = 32, dtype=None, box=None,
                       sigma=(4.0, 12.0), drift: float = 0.5, t0: int = 0, device: str = "cuda"):
    """The drifting Gaussian-sum gradient at arbitrary points (nv, ndim), on the
    device: one per-vertex array per component of length nt * nv (vertex id =
    spatial id + t * nv), as ftk2_b200.synthetic.gaussian_sum_gradient_at
    defines it; ``t0`` shifts the time of the first step."""
    import torch
    dtype = dtype or torch.float64
    P = torch.as_tensor(np.asarray(points, dtype=np.float64), device=device)
    nv, ndim = P.shape
    if box is None:
        box = (P.max(dim=0).values + 1.0).cpu().numpy()
    blobs = gaussian_blobs(seed, n_blobs, box, sigma, drift)
    out = torch.zeros((ndim, nt, nv), dtype=torch.float64, device=device)
    for k in range(nt):
        for b in range(n_blobs):
            c = torch.as_tensor(blobs["centers"][b] + blobs["vel"][b] * (k + t0), device=device)
            s2 = float(blobs["sigma"][b]) ** 2
            d = P - c
            e = float(blobs["amps"][b]) * torch.exp(-(d * d).sum(1) / (2.0 * s2))
            out[:, k, :] -= (e[:, None] * d / s2).T
    return out.reshape(ndim, nt * nv).to(dtype)


def batch_specs(n: int = 256, seed: int = 2024, sides2=(32, 512), sides3=(16, 96), nt=(2, 8), blobs=(8, 64)):
    """Seeded shapes of a batch of independent fields: each field is 2D or 3D
    with probability 1/2, sides U[sides2] (2D) or U[sides3] (3D) per axis,
    nt U[nt] timesteps and U[blobs] Gaussians; returns a list of
    (spatial dims, nt, n_blobs, field seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        three = bool(rng.integers(0, 2))
        lo, hi = sides3 if three else sides2
        dims = tuple(int(v) for v in rng.integers(lo, hi + 1, size=3 if three else 2))
        out.append((dims, int(rng.integers(nt[0], nt[1] + 1)), int(rng.integers(blobs[0], blobs[1] + 1)),
                    int(seed * 1000 + i)))
    return out


def gaussian_field_fast(dims, nt: int, seed: int, n_blobs: int, dtype=None, sigma=(4.0, 12.0), drift: float = 0.5,
                        device: str = "cuda", chunk: int = 16):
    """The drifting Gaussian-sum gradient of gaussian_field_device with the
    blobs evaluated ``chunk`` at a time (same blob parameters; the sum is
    accumulated in another order, so values may differ in the last bits)."""
    import torch
    dtype = dtype or torch.float32
    ndim = len(dims)
    b = gaussian_blobs(seed, n_blobs, dims, sigma, drift)
    shape = tuple(dims[::-1])
    axes = []
    for i in range(ndim):
        view = [1] * (ndim + 1)
        view[ndim - i] = dims[i]
        axes.append(torch.arange(dims[i], dtype=torch.float64, device=device).view(view))
    out = torch.empty((nt,) + shape + (ndim,), dtype=dtype, device=device)
    cen = torch.as_tensor(b["centers"], device=device)
    vel = torch.as_tensor(b["vel"], device=device)
    amp = torch.as_tensor(b["amps"], device=device)
    s2 = torch.as_tensor(b["sigma"], device=device) ** 2
    bview = [-1] + [1] * ndim
    for k in range(nt):
        acc = torch.zeros(shape + (ndim,), dtype=torch.float64, device=device)
        for c0 in range(0, n_blobs, chunk):
            c1 = min(n_blobs, c0 + chunk)
            c = cen[c0:c1] + vel[c0:c1] * k
            d = [axes[i] - c[:, i].view(bview) for i in range(ndim)]
            r2 = d[0] * d[0]
            for i in range(1, ndim):
                r2 = r2 + d[i] * d[i]
            e = amp[c0:c1].view(bview) * torch.exp(-r2 / (2.0 * s2[c0:c1].view(bview))) / s2[c0:c1].view(bview)
            for i in range(ndim):
                acc[..., i] -= (e * d[i]).sum(0)
        out[k] = acc.to(dtype)
    return out


def c3_batch(n: int = 256, seed: int = 2024, device: str = "cuda"):
    """Batched workload: n independent float32 fields (2D sides U[32,512] or
    3D sides U[16,96], nt U[2,8], 8-64 blobs each) as a list of
    (mesh dims incl. time, ncomp, device tensor (nt, [nz,] ny, nx, ncomp))."""
    import torch
    out = []
    for dims, nt, nb, fs in batch_specs(n, seed):
        f = gaussian_field_fast(dims, nt, fs, nb, dtype=torch.float32, device=device)
        out.append((list(dims) + [nt], len(dims), f))
    return out
