"""numpy restatement of PoissonDirichlet::poisson_solve
(src/poissonDirichlet.cpp:23-98).

ORACLE ONLY (test infrastructure): tests/ use it as a checker of the GPU
solve; the product never imports this module.

Each radial row of rho gets the sine transform along z of
Fourier::fast_sine_transform (src/math/fourier.cpp:17-51),
    S[k] = sum_j a[j] sin(pi (j+1)(k+1) / (N+1)),  N = n_grid_z,
(here through numpy's FFT of the odd extension of length 2N + 2); per mode k
the radial recurrence alpha/beta with b = 2 (1 - dr^2/dz^2 (cos(pi (k+1) /
(N+1)) - 1)), a = 1 - 1/(2i), c = 1 + 1/(2i), d = dr^2 S[i][k] / EPSILON0,
alpha[1] = 4 / (2 + b), beta[1] = d[0] / (2 + b), then phi[i] = beta[i+1] +
alpha[i+1] phi[i+1] down from phi[n_grid_r-1] = 0 (EField::set_fi_on_z); the
inverse transform is the same sum times 2 / (N+1); E_r = (phi_i - phi_i+1)
/ dr for i < n_grid_r-1, E_z = (phi_k - phi_k+1) / dz for k < n_grid_z-1.
"""
import numpy as np

PI = 3.1415926535897932  # include/constant.h:10
EPSILON0 = 8.85e-12  # include/constant.h:12


def sine_transform(a):
    """S[..., k] = sum_j a[..., j] sin(pi (j+1)(k+1) / (N+1))."""
    n = a.shape[-1]
    ext = np.zeros(a.shape[:-1] + (2 * n + 2,))
    ext[..., 1:n + 1] = a
    ext[..., n + 2:] = -a[..., ::-1]
    return -0.5 * np.fft.fft(ext, axis=-1).imag[..., 1:n + 1]


def poisson_dirichlet(rho, dr, dz, er=None, ez=None):
    """(phi, E_r, E_z); er, ez: the E grids before the solve (their last
    row / column are kept), zeros when not given."""
    rho = np.asarray(rho, dtype=np.float64)
    nr, nz = rho.shape
    t = sine_transform(rho)
    k = np.arange(nz)
    b = 2. * (1. - dr * dr / (dz * dz) * (np.cos(PI * (k + 1) / (nz + 1)) - 1))
    alpha = np.zeros((nr, nz))
    beta = np.zeros((nr, nz))
    d = dr * dr * t[0] / EPSILON0
    alpha[1] = 4. / (2. + b)
    beta[1] = d / (2. + b)
    for i in range(1, nr - 1):
        a = 1. - 1. / (2. * i)
        c = 1. + 1. / (2. * i)
        d = dr * dr * t[i] / EPSILON0
        alpha[i + 1] = c / (b - alpha[i] * a)
        beta[i + 1] = (d + beta[i] * a) / (b - alpha[i] * a)
    fi = np.zeros((nr, nz))
    for i in range(nr - 2, -1, -1):
        fi[i] = beta[i + 1] + alpha[i + 1] * fi[i + 1]
    fi = sine_transform(fi) * 2.0 / (nz + 1)
    er = np.zeros((nr, nz)) if er is None else np.array(er, dtype=np.float64)
    ez = np.zeros((nr, nz)) if ez is None else np.array(ez, dtype=np.float64)
    er[:-1] = (fi[:-1] - fi[1:]) / dr
    ez[:, :-1] = (fi[:, :-1] - fi[:, 1:]) / dz
    return fi, er, ez
