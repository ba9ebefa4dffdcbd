"""Generates golden fixtures for the CPU oracle from independent sources.

    python tests/golden/make_golden.py

* transforms.npz: random vectors and scipy.fft's DCT-II / DCT-III / DST-III
  of them.  scipy's unnormalised transforms are exactly twice rustdct's
  (the crate the reference calls, density.rs:211-275), so the oracle's
  transforms must equal these / 2.
* rng.json: the first outputs of xorshift64 (context/rng.rs:19-31) and a
  Fisher-Yates shuffle (rng.rs:52-61), computed here with Python integers --
  an independent restatement of the reference RNG.
* wa.json: WA values and analytic gradients of the reference's own unit-test
  inputs (solver/wa.rs:120-230) computed with numpy in FP64 from the
  formulas, plus their central finite differences.
"""

import json
import os

import numpy as np
import scipy.fft as sf

HERE = os.path.dirname(os.path.abspath(__file__))
MASK = (1 << 64) - 1


def xorshift64(seed, n):
    s = max(seed, 1)
    out = []
    for _ in range(n):
        s ^= (s << 13) & MASK
        s ^= s >> 7
        s ^= (s << 17) & MASK
        out.append(s)
    return out


def shuffle(seed, values):
    s = [max(seed, 1)]
    a = list(values)

    def nxt():
        v = s[0]
        v ^= (v << 13) & MASK
        v ^= v >> 7
        v ^= (v << 17) & MASK
        s[0] = v
        return v

    for i in range(len(a) - 1, 0, -1):
        j = (nxt() & 0xFFFFFFFF) % (i + 1)
        a[i], a[j] = a[j], a[i]
    return a


def wa_value(c, g):
    c = np.asarray(c, np.float64)
    if c.size < 2:
        return 0.0
    m = c.mean()
    ea = np.exp(np.maximum(g * (c - m), -3000.0))
    eb = np.exp(np.maximum(g * (m - c), -3000.0))
    return float((c * ea).sum() / ea.sum() - (c * eb).sum() / eb.sum())


def wa_grad(c, g):
    c = np.asarray(c, np.float64)
    m = c.mean()
    ea = np.exp(np.maximum(g * (c - m), -3000.0))
    eb = np.exp(np.maximum(g * (m - c), -3000.0))
    sa, sb, xa, xb = ea.sum(), eb.sum(), (c * ea).sum(), (c * eb).sum()
    dmax = ea / sa + g * ea * (c * sa - xa) / sa**2
    dmin = eb / sb - g * eb * (c * sb - xb) / sb**2
    return (dmax - dmin).tolist()


def main():
    rng = np.random.default_rng(20261203)
    arrays = {}
    for n in (1, 2, 3, 4, 5, 8, 16, 31, 64, 128, 512):
        v = rng.standard_normal(n)
        arrays["x_%d" % n] = v
        arrays["dct2_%d" % n] = sf.dct(v, type=2)
        arrays["dct3_%d" % n] = sf.dct(v, type=3)
        arrays["dst3_%d" % n] = sf.dst(v, type=3)
    np.savez_compressed(os.path.join(HERE, "transforms.npz"), **arrays)

    rngd = {
        "seeds": {str(s): [str(v) for v in xorshift64(s, 8)] for s in (0, 1, 42, 99, 123, 2**63 + 5)},
        "shuffle_seed_7_range_10": shuffle(7, range(10)),
        "shuffle_seed_1_range_33": shuffle(1, range(33)),
    }
    with open(os.path.join(HERE, "rng.json"), "w") as f:
        json.dump(rngd, f, indent=1)

    cases = [([1.0, 4.0, 2.0, 6.0], 0.5), ([1.0, 4.0, 2.0], 0.5), ([2.0, 1.0, 5.0], 0.5), ([0.0, 3.0], 0.5),
             ([0.0, 3.0], 5.0), ([0.0, 5.0, 2.0], 0.1), ([0.0, 5.0, 2.0], 2.0), ([10.5, 11.25, 9.0, 30.0, 2.0], 1.3)]
    wa = []
    for c, g in cases:
        eps = 1e-6
        fd = []
        for i in range(len(c)):
            cp = list(c)
            cm = list(c)
            cp[i] += eps
            cm[i] -= eps
            fd.append((wa_value(cp, g) - wa_value(cm, g)) / (2 * eps))
        wa.append({"coords": c, "coeff": g, "value": wa_value(c, g), "grad": wa_grad(c, g), "fd": fd})
    with open(os.path.join(HERE, "wa.json"), "w") as f:
        json.dump(wa, f, indent=1)


if __name__ == "__main__":
    main()
