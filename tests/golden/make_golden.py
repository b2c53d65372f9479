"""Generate the golden direct-sum fixtures (run once; output committed).

Independent of both the oracle and the CUDA library: the sums are evaluated
in 40-digit arithmetic with mpmath from the kernel definitions the reference
implements (src/laplace/cauchykernels2d.f, lapkernels2d.f):
  Cauchy : pot = sum q log|z| + d/z, grad = q/z - d/z^2, hess = -q/z^2 + 2d/z^3
  Laplace: pot = sum q log r - d v.(x-y)/r^2, gradient, Hessian (xx, xy, yy)
with z = x - y.  Usage: python tests/golden/make_golden.py
"""
import os

import mpmath as mp
import numpy as np

mp.mp.dps = 40
HERE = os.path.dirname(os.path.abspath(__file__))


def cauchy(src, trg, q, d):
    nt = trg.shape[1]
    pot = np.zeros(nt, complex)
    grad = np.zeros(nt, complex)
    hess = np.zeros(nt, complex)
    for j in range(nt):
        P = G = H = mp.mpc(0)
        for i in range(src.shape[1]):
            z = mp.mpc(mp.mpf(trg[0, j]) - mp.mpf(src[0, i]), mp.mpf(trg[1, j]) - mp.mpf(src[1, i]))
            qi = mp.mpc(q[i].real, q[i].imag)
            di = mp.mpc(d[i].real, d[i].imag)
            P += qi * mp.log(abs(z)) + di / z
            G += qi / z - di / z**2
            H += -qi / z**2 + 2 * di / z**3
        pot[j], grad[j], hess[j] = complex(P), complex(G), complex(H)
    return pot, grad, hess


def laplace(src, trg, q, d, v):
    nt = trg.shape[1]
    pot = np.zeros(nt, complex)
    grad = np.zeros((2, nt), complex)
    hess = np.zeros((3, nt), complex)
    for j in range(nt):
        acc = [mp.mpc(0)] * 6
        for i in range(src.shape[1]):
            x = mp.mpf(trg[0, j]) - mp.mpf(src[0, i])
            y = mp.mpf(trg[1, j]) - mp.mpf(src[1, i])
            rr = x * x + y * y
            qi = mp.mpc(q[i].real, q[i].imag)
            di = mp.mpc(d[i].real, d[i].imag)
            v1, v2 = mp.mpf(v[0, i]), mp.mpf(v[1, i])
            gx, gy = x / rr, y / rr
            hxx, hxy, hyy = (rr - 2 * x * x) / rr**2, -2 * x * y / rr**2, (rr - 2 * y * y) / rr**2
            txxx = (-6 * x * rr + 8 * x**3) / rr**3
            txxy = (-2 * y * rr + 8 * x * x * y) / rr**3
            txyy = (-2 * x * rr + 8 * x * y * y) / rr**3
            tyyy = (-6 * y * rr + 8 * y**3) / rr**3
            d1, d2 = di * v1, di * v2
            acc[0] += qi * mp.log(rr) / 2 - (d1 * gx + d2 * gy)
            acc[1] += qi * gx - (d1 * hxx + d2 * hxy)
            acc[2] += qi * gy - (d1 * hxy + d2 * hyy)
            acc[3] += qi * hxx - (d1 * txxx + d2 * txxy)
            acc[4] += qi * hxy - (d1 * txxy + d2 * txyy)
            acc[5] += qi * hyy - (d1 * txyy + d2 * tyyy)
        pot[j] = complex(acc[0])
        grad[:, j] = [complex(acc[1]), complex(acc[2])]
        hess[:, j] = [complex(acc[3]), complex(acc[4]), complex(acc[5])]
    return pot, grad, hess


def main():
    rng = np.random.default_rng(20261203)
    ns, nt = 60, 16
    src = rng.uniform(0, 1, (2, ns))
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    d = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    v = rng.uniform(-1, 1, (2, ns))
    qr = rng.normal(size=ns)
    dr = rng.normal(size=ns)
    cp, cg, ch = cauchy(src, trg, q, d)
    lp, lg, lh = laplace(src, trg, q, d, v)
    rp, rg, rh = laplace(src, trg, qr + 0j, dr + 0j, v)
    np.savez(os.path.join(HERE, "laplace_direct.npz"), src=src, trg=trg, q=q, d=d, v=v, qr=qr,
             dr=dr, cpot=cp, cgrad=cg, chess=ch, lpot=lp, lgrad=lg, lhess=lh, rpot=rp.real,
             rgrad=rg.real, rhess=rh.real)


if __name__ == "__main__":
    main()
