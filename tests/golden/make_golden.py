"""Generate the golden vectors that pin the CPU oracle.

The reference ships no tests and cannot be built here, so the oracle is
pinned by independent implementations run in this container: numpy.fft for
the transforms, scipy.special for erf, and closed-form known answers.  Run:
    python tests/golden/make_golden.py
Outputs small .npz files next to this script.
"""
import os

import numpy as np
from scipy.special import erf

HERE = os.path.dirname(os.path.abspath(__file__))
rng = np.random.default_rng(20261203)

# 1. unnormalised DFTs (numpy.fft) of seeded complex fields
fft = {}
for dim, s in [(3, 8), (3, 12), (2, 12), (2, 16)]:
    x = rng.standard_normal((s,) * dim) + 1j * rng.standard_normal((s,) * dim)
    fft["in_%dd_%d" % (dim, s)] = x.reshape(-1)
    fft["fwd_%dd_%d" % (dim, s)] = np.fft.fftn(x).reshape(-1)
    fft["bwd_%dd_%d" % (dim, s)] = (np.fft.ifftn(x) * x.size).reshape(-1)
np.savez_compressed(os.path.join(HERE, "fft_numpy.npz"), **fft)

# 2. centred transform with the reference's conventions (fftParallel):
#    f~(k_m) = dx^D sum_n f(x_n) exp(-i k_m x_n), x_n = -L/2 + n dx,
#    k_m = -pi/dx + m dk; evaluated by direct summation along each axis.
def centred_dft_1d(f, L, sign):
    s = f.shape[0]
    dx = L / s
    x = -L / 2 + dx * np.arange(s)
    k = -np.pi / dx + (2 * np.pi / L) * np.arange(s)
    if sign < 0:
        return dx * np.exp(-1j * np.outer(k, x))
    return (1.0 / L) * np.exp(1j * np.outer(x, k))


cent = {}
for dim, s, L in [(3, 8, 6.0), (2, 12, 8.0)]:
    f = rng.standard_normal((s,) * dim) + 1j * rng.standard_normal((s,) * dim)
    Mf = centred_dft_1d(f, L, -1)
    Mb = centred_dft_1d(f, L, +1)
    g = f.copy()
    h = f.copy()
    for ax in range(dim):
        g = np.moveaxis(np.tensordot(Mf, np.moveaxis(g, ax, 0), axes=1), 0, ax)
        h = np.moveaxis(np.tensordot(Mb, np.moveaxis(h, ax, 0), axes=1), 0, ax)
    cent["in_%dd" % dim] = f.reshape(-1)
    cent["fwd_%dd" % dim] = g.reshape(-1)
    cent["bwd_%dd" % dim] = h.reshape(-1)
    cent["L_%dd" % dim] = L
    cent["s_%dd" % dim] = s
np.savez_compressed(os.path.join(HERE, "fft_centred.npz"), **cent)

# 3. Poisson known answer: potential of a Gaussian charge (scipy erf)
s, L, sig, Q = 32, 16.0, 0.8, 2.0
dx = L / s
x = -L / 2 + dx * np.arange(s)
X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
r = np.sqrt(X * X + Y * Y + Z * Z)
rho = Q * np.exp(-r * r / (2 * sig * sig)) / (2 * np.pi * sig * sig) ** 1.5
with np.errstate(invalid="ignore", divide="ignore"):
    pot = np.where(r > 0, Q * erf(r / (np.sqrt(2) * sig)) / r, Q * np.sqrt(2 / np.pi) / sig)
np.savez_compressed(os.path.join(HERE, "poisson_gauss.npz"), rho=rho.reshape(-1), pot=pot.reshape(-1),
                    r=r.reshape(-1), s=s, L=L, sig=sig, Q=Q)
print("golden vectors written to", HERE)
