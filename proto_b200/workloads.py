"""Seeded synthetic inputs for the structured-grid workloads (no datasets are involved).

Every generator is deterministic in its seed (numpy PCG64 via default_rng) and returns float64
arrays in BoxData order: x fastest, shaped (z, y, x).
"""
import numpy as np


def uniform_box(shape_zyx, seed, lo=-1.0, hi=1.0):
    """uniform[lo, hi] values over a box, filled in BoxData linear order."""
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape_zyx))
    return rng.uniform(lo, hi, size=n).reshape(shape_zyx)


def plain_input(n=64, seed=0):
    """The small plain-method case: u on [-1, n]^3 (one ghost layer) ~ uniform[-1, 1]."""
    return uniform_box((n + 2,) * 3, seed)


def sine_modes_rhs(n, seed=1, modes=8, kmax=8, amplitudes=None):
    """f = sum_m A_m sin(2 pi (k_m . x)) at the cell centres of a periodic n^3 grid on [0,1]^3,
    integer wave vectors k_m in [1, kmax]^3, A_m ~ N(0, 1); the mean is removed."""
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, kmax + 1, size=(modes, 3))
    amps = rng.standard_normal(modes) if amplitudes is None else np.asarray(amplitudes, dtype=np.float64)
    x = (np.arange(n) + 0.5) / n
    f = np.zeros((n, n, n))
    # separable evaluation: sin(a+b+c) through angle sums keeps this O(n^3) per mode
    for (kx, ky, kz), a in zip(ks, amps):
        sx, cx = np.sin(2 * np.pi * kx * x), np.cos(2 * np.pi * kx * x)
        sy, cy = np.sin(2 * np.pi * ky * x), np.cos(2 * np.pi * ky * x)
        sz, cz = np.sin(2 * np.pi * kz * x), np.cos(2 * np.pi * kz * x)
        sxy = sx[None, :] * cy[:, None] + cx[None, :] * sy[:, None]      # (y, x)
        cxy = cx[None, :] * cy[:, None] - sx[None, :] * sy[:, None]
        f += a * (sxy[None, :, :] * cz[:, None, None] + cxy[None, :, :] * sz[:, None, None])
    f -= f.mean()
    return f


def sine_modes_rhs_device(n, seed, modes=4, kmax=8, device="cuda"):
    """sine_modes_rhs evaluated in FP64 on a torch device (the same wave vectors and amplitudes from
    the same seeded generator; the sums run on the device, so the last bits may differ from the
    numpy evaluation). Used to make many large right-hand sides quickly."""
    import torch
    rng = np.random.default_rng(seed)
    ks = rng.integers(1, kmax + 1, size=(modes, 3))
    amps = rng.standard_normal(modes)
    x = (torch.arange(n, dtype=torch.float64, device=device) + 0.5) / n
    f = torch.zeros((n, n, n), dtype=torch.float64, device=device)
    for (kx, ky, kz), a in zip(ks, amps):
        sx, cx = torch.sin(2 * np.pi * int(kx) * x), torch.cos(2 * np.pi * int(kx) * x)
        sy, cy = torch.sin(2 * np.pi * int(ky) * x), torch.cos(2 * np.pi * int(ky) * x)
        sz, cz = torch.sin(2 * np.pi * int(kz) * x), torch.cos(2 * np.pi * int(kz) * x)
        sxy = sx[None, :] * cy[:, None] + cx[None, :] * sy[:, None]
        cxy = cx[None, :] * cy[:, None] - sx[None, :] * sy[:, None]
        f += float(a) * (sxy[None, :, :] * cz[:, None, None] + cxy[None, :, :] * sz[:, None, None])
    f -= f.mean()
    return f


def poisson_rho(n, seed=1, modes=8):
    """Right-hand side in the reference multigrid's sign convention (L_h phi = rho) for -Lap u = f."""
    return -sine_modes_rhs(n, seed=seed, modes=modes)


def helmholtz_alpha(n, seed=3, lo=0.1, hi=1.0):
    return uniform_box((n, n, n), seed, lo, hi)


def amr_widths(seed=2, per_axis=8, choices=(16, 24, 32, 48, 64)):
    """Per-axis patch widths of the uneven AMR-level tiling (a tensor product of the draws)."""
    rng = np.random.default_rng(seed)
    return [list(int(v) for v in rng.choice(np.asarray(choices), size=per_axis)) for _ in range(3)]


def amr_patches(widths):
    """Boxes (lo, hi) of the tensor-product tiling, patch order x fastest; and the domain extents."""
    boxes = []
    z0 = 0
    for wz in widths[2]:
        y0 = 0
        for wy in widths[1]:
            x0 = 0
            for wx in widths[0]:
                boxes.append(((x0, y0, z0), (x0 + wx - 1, y0 + wy - 1, z0 + wz - 1)))
                x0 += wx
            y0 += wy
        z0 += wz
    return boxes, [sum(w) for w in widths]
