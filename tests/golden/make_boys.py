"""Reference Boys values F_m(T), m = 0..8, from mpmath at 40 digits.

    python tests/golden/make_boys.py    # writes tests/golden/boys_mpmath.npz

F_m(T) = 1F1(m + 1/2; m + 3/2; -T) / (2m + 1).  scipy's hyp1f1 loses ~2
digits near T = 45, so the GPU Boys test reads these instead."""
import os

import mpmath
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    mpmath.mp.dps = 40
    T = np.concatenate([np.linspace(0, 60, 2401), [1e-16, 1e-8, 49.95, 49.999, 50.0, 50.05, 80.0, 700.0]])
    F = np.array([[float(mpmath.hyp1f1(m + 0.5, m + 1.5, -mpmath.mpf(float(t))) / (2 * m + 1)) for m in range(9)]
                  for t in T])
    T32 = T.astype(np.float32)
    F32 = np.array([[float(mpmath.hyp1f1(m + 0.5, m + 1.5, -mpmath.mpf(float(t))) / (2 * m + 1)) for m in range(9)]
                    for t in T32])
    np.savez_compressed(os.path.join(HERE, "boys_mpmath.npz"), T=T, F=F, T32=T32, F32=F32)


if __name__ == "__main__":
    main()
