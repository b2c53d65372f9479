"""Generate the golden Helmholtz fixtures (run once; output committed).

Independent of both the oracle and the CUDA library: mpmath values (60
digits for the special functions, 30 for the sums) of
  * H0, H1 of the first kind (hank103, src/common/hank103.f:116) on real and
    complex arguments covering every evaluation region;
  * the scaled sequences J_n(z)/rs^n (jbessel2d, src/common/cdjseval2d.f:5)
    and H_n(z) rs^n (h2dall, src/helmholtz/h2dcommon.f:71);
  * direct sums of the Helmholtz kernel of src/helmholtz/helmkernels2d.f,
      pot(x) = sum_j q_j G(x - y_j) - d_j v_j . grad_x G(x - y_j),
      G(r) = (i/4) H0(k |r|),
    with gradients and Hessians obtained by numerical differentiation of
    that definition (mpmath.diff), not from the closed forms the
    implementations use.
Usage: python tests/golden/make_golden_helm.py
"""
import os

import mpmath as mp
import numpy as np

mp.mp.dps = 30
HERE = os.path.dirname(os.path.abspath(__file__))

HANKEL_Z = [1e-3, 0.5, 2.0, 3.99, 4.01, 7.5, 12.7, 19.9, 20.1, 35.0, 60.0, 3 + 0.5j, 10 + 1j,
            15 + 1.5j, 0.5 + 0.1j, 25 + 2j, 1e-4 + 1e-5j, 6 - 0.5j]
SEQ_CASES = [(3.7 + 0.2j, 0.8, 40), (0.01, 0.01, 30), (28.0, 1.0, 60), (45 + 0.5j, 1.0, 60),
             (5.0, 1.0, 40), (0.3, 0.05, 30)]


def mpc(z):
    z = complex(z)
    return mp.mpc(z.real, z.imag)


def mparg(z):
    # real arguments stay real: mpmath's complex Bessel routines lose digits
    # at high order and small |z| (J_19(0.01) is wrong in the 6th digit at
    # 30 digits)
    z = complex(z)
    return mp.mpf(z.real) if z.imag == 0 else mp.mpc(z.real, z.imag)


def special():
    mp.mp.dps = 60
    h = np.array([[complex(mp.hankel1(0, mparg(z))), complex(mp.hankel1(1, mparg(z)))]
                  for z in HANKEL_Z])
    seq_j, seq_h = [], []
    for z, rs, n in SEQ_CASES:
        zz, r = mparg(z), mp.mpf(rs)
        seq_j.append([complex(mp.besselj(k, zz) / r**k) for k in range(n + 1)] + [0j] * (60 - n))
        seq_h.append([complex(mp.hankel1(k, zz) * r**k) for k in range(n + 1)] + [0j] * (60 - n))
    mp.mp.dps = 30
    return h, np.array(seq_j), np.array(seq_h)


def direct(zk, src, trg, q, d, v):
    k = mparg(zk)
    nt, ns = trg.shape[1], src.shape[1]
    out = np.zeros((6, nt), complex)
    for j in range(nt):
        acc = [mp.mpc(0)] * 6
        for i in range(ns):
            y1, y2 = mp.mpf(src[0, i]), mp.mpf(src[1, i])
            qi, di = mpc(q[i]), mpc(d[i])
            v1, v2 = mp.mpf(v[0, i]), mp.mpf(v[1, i])

            def G(x1, x2):
                return mp.mpc(0, 0.25) * mp.hankel1(0, k * mp.sqrt((x1 - y1)**2 + (x2 - y2)**2))

            x = (mp.mpf(trg[0, j]), mp.mpf(trg[1, j]))

            def D(a, b):
                return mp.diff(G, x, (a, b))

            acc[0] += qi * G(*x) - di * (v1 * D(1, 0) + v2 * D(0, 1))
            acc[1] += qi * D(1, 0) - di * (v1 * D(2, 0) + v2 * D(1, 1))
            acc[2] += qi * D(0, 1) - di * (v1 * D(1, 1) + v2 * D(0, 2))
            acc[3] += qi * D(2, 0) - di * (v1 * D(3, 0) + v2 * D(2, 1))
            acc[4] += qi * D(1, 1) - di * (v1 * D(2, 1) + v2 * D(1, 2))
            acc[5] += qi * D(0, 2) - di * (v1 * D(1, 2) + v2 * D(0, 3))
        out[:, j] = [complex(a) for a in acc]
    return out


def main():
    h, sj, sh = special()
    rng = np.random.default_rng(20261204)
    ns, nt = 24, 8
    src = rng.uniform(0, 1, (2, ns))
    trg = rng.uniform(0, 1, (2, nt))
    q = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    d = rng.normal(size=ns) + 1j * rng.normal(size=ns)
    v = rng.uniform(-1, 1, (2, ns))
    res = {}
    for name, zk in (("k10", 10.0), ("kc", 3 + 0.5j)):
        res["dir_" + name] = direct(zk, src, trg, q, d, v)
    np.savez_compressed(
        os.path.join(HERE, "helm_golden.npz"), hankel_z=np.array(HANKEL_Z, complex), hankel=h,
        seq_z=np.array([c[0] for c in SEQ_CASES], complex),
        seq_rs=np.array([c[1] for c in SEQ_CASES]), seq_n=np.array([c[2] for c in SEQ_CASES]),
        seq_j=sj, seq_h=sh, src=src, trg=trg, q=q, d=d, v=v, zk=np.array([10.0, 3 + 0.5j]),
        **res)


if __name__ == "__main__":
    main()
