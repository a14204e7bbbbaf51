"""Generate the golden fixtures in this directory with numpy alone.

The reference (Fortran) ships no golden vectors and cannot be compiled here,
so these fixtures come from a second, independent restatement of the same
formulas written directly in vectorised numpy (float64), without the C++
oracle.  The oracle and the GPU kernels are both checked against them.

  python tests/golden/make_golden.py      # rewrites *.npz next to this file

Cases (N = 16 grid, seeded inputs):
  cic      DENSIT weights (PMP2mod_density.f90:235-281), cell keys, cell counts
  poisson  POTENTfft5 eigenvalue division (PMP2main.f90:736-816)
  power    POWERfft5 NGP binning, linear and log bins (PMP2mod_power.f90:355-456)
  move     MOVE gradient/kick/drift (PMP2main.f90:488-676)
  fr_relax one red + one black f(R) n=1 sweep and the level-0 residual RMS
           (PMP2MGsolver_fR.f90:143-182, 433-462)
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
N = 16
NP = 600


def particles(seed):
    rng = np.random.default_rng(seed)
    pos = (1.0 + rng.random((3, NP)) * N).astype(np.float32)
    pos[:, :8] = np.float32(N + 1) - np.float32(1e-3)      # upper edge
    pos[:, 8:16] = np.float32(1.0)                           # lower edge
    vel = (0.3 * rng.standard_normal((3, NP))).astype(np.float32)
    return pos, vel


def cic(pos):
    X = pos.astype(np.float64)
    I = np.floor(X).astype(np.int64)           # 1-based cell
    D = X - I
    T = 1.0 - D
    wpar = np.float64(np.float32(float(N) ** 3 / float(np.float32(NP))))
    fi = np.full((N, N, N), -1.0)              # [k][j][i]
    i0, j0, k0 = I[0] - 1, I[1] - 1, I[2] - 1
    i1, j1, k1 = i0 + 1, j0 + 1, k0 + 1
    i1[i1 == N] = 0
    j1[j1 == N] = 0
    k1[k1 == N] = 0
    for (kk, wz) in ((k0, T[2]), (k1, D[2])):
        for (jj, wy) in ((j0, T[1]), (j1, D[1])):
            for (ii, wx) in ((i0, T[0]), (i1, D[0])):
                np.add.at(fi, (kk, jj, ii), wz * wx * (wy * wpar))
    key = i0 + N * (j0 + N * k0)
    counts = np.bincount(key, minlength=N ** 3)
    return fi.reshape(-1), key.astype(np.int64), counts.astype(np.int64)


def greens():
    P16 = 6.28318530718
    k = np.arange(N)
    m = np.minimum(k, N - k)
    g = 2.0 * np.cos(P16 * m / N)
    g[0] = 2.0
    g[N // 2] = -2.0
    return g


def poisson(delta, a, om):
    trfi = float(np.float32(np.float32(1.5) * np.float32(om) / np.float32(a)))
    F = np.fft.fftn(delta.reshape(N, N, N))
    g = greens()
    A = g[:, None, None] + g[None, :, None] + g[None, None, :] - 6.0
    A[0, 0, 0] = 1.0
    return np.real(np.fft.ifftn(F * trfi / A)).reshape(-1)


def power(delta, box):
    F = np.fft.fftn(delta.reshape(N, N, N)) / N ** 3
    amp = np.abs(F) ** 2
    k = np.arange(N)
    m = np.minimum(k, N - k)
    m2 = m[:, None, None] ** 2 + m[None, :, None] ** 2 + m[None, None, :] ** 2
    rk = np.sqrt(m2.astype(np.float32))
    mp = np.maximum((rk + np.float32(0.5)).astype(np.int64), 1)
    with np.errstate(divide="ignore", invalid="ignore"):
        ml = (np.log10(rk) / np.float32(0.02) + np.float32(1000.0)).astype(np.int64) - 1000
    ml = np.clip(ml, 1, N)
    sel = m2 > 0
    nb = N // 2
    out = {}
    for name, idx in (("lin", mp), ("log", ml)):
        P = np.bincount(idx[sel], weights=amp[sel], minlength=N + 1)
        C = np.bincount(idx[sel], minlength=N + 1).astype(np.float64)
        K = np.bincount(idx[sel], weights=rk[sel].astype(np.float64), minlength=N + 1)
        with np.errstate(invalid="ignore", divide="ignore"):
            out["pk_" + name] = np.where(C[1:nb + 1] > 0, box ** 3 * P[1:nb + 1] / C[1:nb + 1], 0.0)
            out["k_" + name] = np.where(C[1:nb + 1] > 0, K[1:nb + 1] / C[1:nb + 1] * (2 * np.float32(3.141592653) / box), 0.0)
        out["n_" + name] = C[1:nb + 1]
    return out


def move(phi, pos, vel, a, da, fv, om, oml):
    f32 = np.float32
    a, da, fv, om, oml = f32(a), f32(da), f32(fv), f32(om), f32(oml)
    pconst = float(-np.sqrt(a / (om + oml * a * a * a)) * da * f32(0.5) / fv)
    ah = a + da / f32(2.0)
    xconst = float(da / np.sqrt(ah * (om + oml * ah * ah * ah)) / ah)
    F = phi.reshape(N, N, N).astype(np.float32)        # [k][j][i]
    X = pos.astype(np.float64)
    I = np.floor(X).astype(np.int64) - 1
    D = X - (I + 1)
    T = 1.0 - D
    w = lambda o, ax: (I[ax] + o) % N

    def f(oi, oj, ok):
        return F[w(ok, 2), w(oj, 1), w(oi, 0)]

    G = np.zeros((3, NP))
    for ax in range(3):
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    o = [di, dj, dk]
                    up = list(o)
                    lo = list(o)
                    up[ax] += 1
                    lo[ax] -= 1
                    g = (f(*up) - f(*lo)).astype(np.float64)    # Real*4 difference
                    wgt = (D[0] if di else T[0]) * (D[1] if dj else T[1]) * (D[2] if dk else T[2])
                    G[ax] += wgt * g
    V = vel.astype(np.float64) + pconst * G
    Xn = X + V * xconst
    xn = float(f32(N) + f32(1.0) - f32(1e-8))
    Xn = np.where(Xn < 1.0, Xn + N, Xn)
    Xn = np.where(Xn >= xn, Xn - N, Xn)
    wpar = float(np.float32(float(N) ** 3 / float(np.float32(NP))))
    svel = np.sum(V ** 2) * wpar
    enkin = float(np.float32(svel / 2.0 / float(ah * ah)))
    return Xn.astype(np.float32), V.astype(np.float32), enkin


def fr_consts(a, box, fr0=-1e-5, om=0.3089, oml=0.6911, n=1):
    f32 = np.float32
    a32 = f32(a)
    R = 3.0 * (float(f32(om) / (a32 * a32 * a32)) + 4.0 * float(f32(oml)))
    R0 = 3.0 * (float(f32(om)) + 4.0 * float(f32(oml)))
    fR = fr0 * (R0 / R) ** (n + 1)
    ctl = 2.99792458e3 * N / box
    fct2 = 1.0 / (ctl * ctl * np.sign(fR)) / 6.0
    fct1 = -(float(f32(om) / a32) * fct2)
    Q2 = R * float(a32 * a32) * fct2 / 3.0
    Q = Q2 * abs(fR) ** 0.5
    return dict(fR=fR, ctl=ctl, fct1=fct1, fct2=fct2, Q2=Q2, Q=Q, R=R,
                r1=float(f32(om) / a32), r2=-R * float(a32 * a32) / 3.0, r3=ctl * ctl * np.sign(fR))


def fr_sweeps(delta, u, a, box):
    c = fr_consts(a, box)
    d = delta.reshape(N, N, N)
    u = u.reshape(N, N, N).astype(np.float32).copy()
    K, J, I = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    for colour in (0, 1):                      # red: (i+j+k) even, 0-based
        mask = ((I + J + K) % 2) == colour
        s = np.zeros_like(u, dtype=np.float32)
        for ax in (0, 1, 2):
            for sh in (1, -1):
                nb = np.roll(u, sh, axis=ax)
                s = (s + nb * nb).astype(np.float32)
        P = c["fct1"] * d - c["Q2"] - s.astype(np.float64) / 6.0
        D10 = -3.0 * P
        D11 = 27.0 * c["Q"]
        CC = D11 * D11 - 4.0 * D10 ** 3
        sq = np.sqrt(np.maximum(D10, 0.0))
        with np.errstate(invalid="ignore", divide="ignore"):
            S = np.arccos(np.clip(0.5 * D11 / sq ** 3, -1, 1))
            trig = -(2.0 / 3.0) * sq * np.cos(S / 3.0 + 2.0 / 3.0 * np.pi)
            t1 = 0.5 * (np.sqrt(np.maximum(CC, 0.0)) + D11)
            t2 = t1 - D11
            card = -(np.cbrt(t1) - np.cbrt(t2)) / 3.0
        val = np.where(CC >= 0.0, card, trig)
        u = np.where(mask, val.astype(np.float32), u)
    # residual RMS (level 0)
    s = np.zeros_like(u, dtype=np.float32)
    for ax in (0, 1, 2):
        for sh in (1, -1):
            nb = np.roll(u, sh, axis=ax)
            s = (s + nb * nb).astype(np.float32)
    op = (s.astype(np.float64) - (u * u).astype(np.float64) * 6.0) * c["r3"]
    op = op + c["r1"] * d + c["r2"] * (abs(c["fR"]) ** 0.5 / u.astype(np.float64) - 1.0)
    res = np.sqrt(np.sum(op * op) / N ** 3)
    return u.reshape(-1), res


def main():
    pos, vel = particles(2024)
    fi, key, counts = cic(pos)
    np.savez_compressed(os.path.join(HERE, "cic.npz"), pos=pos, fi=fi, key=key, counts=counts)
    rng = np.random.default_rng(7)
    delta = rng.standard_normal(N ** 3)
    delta -= delta.mean()
    delta32 = delta.astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "poisson.npz"), delta=delta32,
                        phi=poisson(delta32.astype(np.float64), 0.4, 0.3089), a=0.4, om=0.3089)
    pk = power(fi, 64.0)
    np.savez_compressed(os.path.join(HERE, "power.npz"), delta=fi.astype(np.float32), box=64.0,
                        **{k: v for k, v in pk.items()})
    phi = rng.standard_normal(N ** 3).astype(np.float32)
    xn, vn, ek = move(phi, pos, vel, 0.3, 0.01, 1.2, 0.3089, 0.6911)
    np.savez_compressed(os.path.join(HERE, "move.npz"), phi=phi, pos=pos, vel=vel, pos_out=xn, vel_out=vn,
                        enkin=ek, a=0.3, da=0.01, fv=1.2)
    a = 0.7
    c = fr_consts(a, 16.0)
    u0 = np.full(N ** 3, abs(c["fR"]) ** 0.5, np.float32)
    u1, res = fr_sweeps(fi, u0, a, 16.0)
    np.savez_compressed(os.path.join(HERE, "fr_relax.npz"), delta=fi.astype(np.float32), u0=u0, u1=u1, res=res,
                        a=a, box=16.0)


if __name__ == "__main__":
    main()
