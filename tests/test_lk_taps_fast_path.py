"""CPU restatement of make_taps (lk_common.cuh) in FP32: the warp-uniform fast path (taken when xmin
and xmin + 8, and ymin and ymin + 8, share an FP32 exponent) must give what the general per-lane path
gives: uniform taps, and every lane's texel index, fraction and quantised fraction."""

import numpy as np

F = np.float32


def general(xmin, ymin):
    """Per lane (base, fr, q) and the uniformity vote of the general path."""
    base, fr, q = [], [], []
    for lane in range(32):
        if lane < 9:
            p = F(F(xmin) + F(lane))
        elif 16 <= lane < 25:
            p = F(F(ymin) + F(lane - 16))
        else:
            p = F(F(ymin) + F(0))
        pb = F(p - F(0.5))
        fl = F(np.floor(pb))
        f = F(pb - fl)
        base.append(int(fl))
        fr.append(f)
        q.append(int(np.floor(F(F(f * F(256)) + F(0.5)))))
    ok = all(base[i] == base[0] + i and q[i] == q[0] for i in range(9))
    ok = ok and all(base[16 + j] == base[16] + j and q[16 + j] == q[16] for j in range(9))
    return base, fr, q, ok


def fast_applies(xmin, ymin):
    bits = lambda v: int(np.array(F(v)).view(np.uint32))
    return ((bits(xmin) ^ bits(F(F(xmin) + F(8)))) | (bits(ymin) ^ bits(F(F(ymin) + F(8))))) >> 23 == 0


def fast(xmin, ymin):
    pbx, pby = F(F(xmin) - F(0.5)), F(F(ymin) - F(0.5))
    flx, fly = F(np.floor(pbx)), F(np.floor(pby))
    frx, fry = F(pbx - flx), F(pby - fly)
    qx = int(np.floor(F(F(frx * F(256)) + F(0.5))))
    qy = int(np.floor(F(F(fry * F(256)) + F(0.5))))
    base = [int(flx) + l if l < 9 else (int(fly) + l - 16 if 16 <= l < 25 else int(fly)) for l in range(32)]
    fr = [frx if l < 9 else fry for l in range(32)]
    q = [qx if l < 9 else qy for l in range(32)]
    return base, fr, q


def test_fast_path_equals_general_path():
    rng = np.random.default_rng(7)
    vals = list(rng.uniform(0, 4096, 3000).astype(F)) + list(rng.uniform(0, 40, 2000).astype(F))
    for k in [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048]:
        for d in np.linspace(-9, 1, 41):
            vals.append(F(k + d))
    vals = [v for v in vals if v >= 0]
    taken = 0
    for i, xmin in enumerate(vals):
        ymin = vals[(i * 7919) % len(vals)]
        if not fast_applies(xmin, ymin):
            continue
        taken += 1
        gb, gf, gq, ok = general(xmin, ymin)
        fb, ff, fq = fast(xmin, ymin)
        assert ok, (float(xmin), float(ymin))
        assert gb == fb and gq == fq and all(a == b for a, b in zip(gf, ff)), (float(xmin), float(ymin))
    assert taken > 1000
