"""Generates the golden fixtures of the free-propagation known answer.

With cold links (U = 1, E = 0; ColdInit, src/gaugeconfiguration_su3.f90:363-378)
and a point source 1_6/sqrt(6) at the origin (InitSinglePoint,
src/nrqcd.f90:324-350) every block of the assembled CN operator is a
multiple of the identity, so the n-step propagators are known exactly:

  psi_q(x, n) = (1_6/sqrt 6) (1/V) sum_p e^{ipx} R(p)^n,
  R(p) = (1 - i tau eps(p)) / (1 + i tau eps(p)),  tau = a0 dt / 2,
  eps(p) = (2 c1 / M) sum_i sin^2(theta_i / 2) / a_i^2,  theta_i = 2 pi k_i / N_i,

and the antiquark (M -> -M) has conj(R).  The O1(1S0) correlator is
i (1/V) sum_p R(p)^{2n}.  The fixture stores the diagonal amplitude of both
propagators and the four correlators after each step.

Run:  python tests/golden/make_golden.py
"""
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def free_kat(n, a, mass, c1, nsteps, dt=1.0):
    nx, ny, nz = n
    tau = a[0] * dt / 2
    px = 2 * np.pi * np.fft.fftfreq(nx)
    py = 2 * np.pi * np.fft.fftfreq(ny)
    pz = 2 * np.pi * np.fft.fftfreq(nz)
    PZ, PY, PX = np.meshgrid(pz, py, px, indexing="ij")  # array [z, y, x]
    eps = (2 * c1 / mass) * (np.sin(PX / 2) ** 2 / a[1] ** 2 + np.sin(PY / 2) ** 2 / a[2] ** 2
                             + np.sin(PZ / 2) ** 2 / a[3] ** 2)
    R = (1 - 1j * tau * eps) / (1 + 1j * tau * eps)
    amp_q, amp_a, corr = [], [], []
    for s in range(1, nsteps + 1):
        fq = np.fft.ifftn(R ** s).reshape(-1) / np.sqrt(6)   # site order x fastest
        fa = np.fft.ifftn(np.conj(R) ** s).reshape(-1) / np.sqrt(6)
        amp_q.append(fq)
        amp_a.append(fa)
        corr.append(1j * np.mean(R ** (2 * s)))
    return np.array(amp_q), np.array(amp_a), np.array(corr)


def main():
    cases = {
        "free_kat_8x8x8_M1": dict(n=(8, 8, 8), a=(0.05, 1.0, 1.0, 1.0), mass=1.0, c1=1.0, nsteps=5),
        "free_kat_6x4x10_M2": dict(n=(6, 4, 10), a=(0.1, 1.0, 1.5, 0.8), mass=2.0, c1=1.0, nsteps=4),
    }
    for name, p in cases.items():
        q, an, corr = free_kat(p["n"], p["a"], p["mass"], p["c1"], p["nsteps"])
        np.savez_compressed(os.path.join(HERE, name + ".npz"), amp_q=q, amp_a=an, o1_1s0=corr,
                            n=np.array(p["n"]), a=np.array(p["a"]), mass=p["mass"], c1=p["c1"],
                            nsteps=p["nsteps"])
        print("wrote", name)


if __name__ == "__main__":
    main()
