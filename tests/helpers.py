"""Seeded synthetic inputs shared by the tests (test infrastructure)."""
import numpy as np


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def viscosity_field(m, seed=0, contrast=1e4, blobs=6):
    """k = exp(ln(contrast) (0.5 radial ramp + 0.5 Gaussian-blob field)), clamped to [1, contrast]."""
    rng = np.random.default_rng(seed)
    x = m.coords[:, :, :, None, :] * m.radii[:, None, None, :, None]
    rho = (m.radii - m.radii.min()) / (m.radii.max() - m.radii.min())
    ramp = np.broadcast_to(rho[:, None, None, :], m.shape)
    field = np.zeros(m.shape)
    for _ in range(blobs):
        c = rng.normal(size=3)
        c = c / np.linalg.norm(c) * rng.uniform(m.radii.min(), m.radii.max())
        w = rng.uniform(0.1, 0.3)
        field += np.exp(-np.sum((x - c) ** 2, axis=-1) / (2 * w * w))
    field = (field - field.min()) / (field.max() - field.min() + 1e-300)
    k = np.exp(np.log(contrast) * (0.5 * ramp + 0.5 * field))
    return np.clip(k, 1.0, contrast)


def random_vector(m, seed, ncomp=3):
    rng = np.random.default_rng(seed)
    shape = ((ncomp,) if ncomp > 1 else ()) + m.shape
    return m.make_consistent(rng.normal(size=shape)).reshape(shape)
