"""Seeded synthetic systems of the benchmark configurations.

The reference quotes no public data set for this path; these generators stand
in for it.  Matrices come from the platform's Q1 assembler (lexicographic
DoFs, Dirichlet rows set to identity, structure kept), right-hand sides from
the splitmix64 stream (uniform[-1, 1) on interior DoFs, 0 on the boundary).

Gaussian random field (the variable coefficient k = exp(g) of the 3-D
128^3 system): squared-exponential covariance C(r) = sigma^2 exp(-r^2 / (2 l^2))
sampled at the cell centres by circulant embedding -- the grid is embedded in a
periodic box of twice its size, the covariance's eigenvalues on that torus
come from one FFT (negative round-off clipped to 0), and
g = IFFT(sqrt(lambda) * FFT(white noise)) restricted to the original cells has
exactly the stated covariance.  numpy's PCG64 generator with the given seed
supplies the white noise.
"""
import numpy as np


def grf_cells(N, dim=3, sigma=1.0, ell=0.1, seed=2024):
    """Gaussian random field on the N^dim cell centres of the unit cube (x fastest)."""
    M = 2 * N
    h = 1.0 / N
    d = np.minimum(np.arange(M), M - np.arange(M)) * h        # periodic distance per axis
    r2 = np.zeros((M,) * dim)
    for ax in range(dim):
        shape = [1] * dim
        shape[ax] = M
        r2 = r2 + (d ** 2).reshape(shape)
    c = sigma ** 2 * np.exp(-r2 / (2.0 * ell ** 2))
    lam = np.fft.rfftn(c).real
    lam = np.maximum(lam, 0.0)
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((M,) * dim)
    g = np.fft.irfftn(np.sqrt(lam) * np.fft.rfftn(white), s=(M,) * dim, axes=tuple(range(dim)))
    g = g[(slice(0, N),) * dim]
    # array axes are (z, y, x) so that flattening gives x fastest
    return np.ascontiguousarray(g).reshape(-1)


def kcell_lognormal(N, dim, sigma, seed):
    """Cell-wise log-normal coefficient exp(sigma * xi), xi i.i.d. N(0, 1)."""
    rng = np.random.default_rng(seed)
    return np.exp(sigma * rng.standard_normal(N ** dim))


CONFIGS = {
    "c1": dict(desc="2D Q1 Poisson 256x256 cells, Jacobi-CG to 1e-10", dim=2, N=256, kind=0, tol=1e-10),
    "c2": dict(desc="3D Q1 Poisson 128^3 cells, 8-colour MC-SGS CG to 1e-8", dim=3, N=128, kind=0, tol=1e-8),
    "c3": dict(desc="3D Q1 128^3 cells, k = exp(GRF sigma=1, l=0.1), FP32 Jacobi-CG (1e-4) inside FP64 "
                    "defect correction to 1e-10", dim=3, N=128, kind=0, tol=1e-10, grf=True),
    "c4": dict(desc="2D Q1 convection-diffusion 512x512, nu=1e-3, beta=(1,0.5), GMRES(30)+ILU(0) level-scheduled "
                    "to 1e-9", dim=2, N=512, kind=1, tol=1e-9, nu=1e-3, beta=(1.0, 0.5)),
}


def system(b200, name, seed=42, N=None):
    """(row, col, val, b, kcell) of a configuration, optionally at another size."""
    cfg = CONFIGS[name]
    n_cells = N or cfg["N"]
    kc = np.exp(grf_cells(n_cells, cfg["dim"])) if cfg.get("grf") else None
    row, col, val = b200.q1_assemble(cfg["dim"], n_cells, cfg["kind"], kc, cfg.get("nu", 1.0),
                                     cfg.get("beta", (0.0, 0.0, 0.0)))
    b = b200.q1_rhs(seed, cfg["dim"], n_cells)
    return row, col, val, b, kc
