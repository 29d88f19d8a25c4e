"""Literal pure-Python transcription of the reference pair loop, for tiny inputs.

An independent second restatement used to check the C oracle: it follows
XiEstimator::skybin_xi_task / accumulate_pixel_pairs (XiEstimator.cc:121-296)
and XiBin::accumulate_pair (types.h:77-87) statement by statement, with
numpy float32 scalars wherever the reference computes in float and Python
floats (IEEE double) elsewhere.  No sky index: every j > i is a candidate.
"""
import math

import numpy as np

f32 = np.float32
M32 = 0xFFFFFFFF


def ref_u32(x: float) -> int:
    """static_cast<unsigned>(double) as x86-64 code computes it (cvttsd2si r64, low 32 bits)."""
    if not (x > -9.223372036854775808e18 and x < 9.223372036854775808e18):
        return 0
    return int(math.trunc(x)) & M32


def _grid(coord, axes, scale):
    a = np.asarray(axes, dtype=np.float64).reshape(3, 3)
    w = [(a[k, 1] - a[k, 0]) / a[k, 2] for k in range(3)]
    hi = [a[k, 0] + a[k, 2] * w[k] for k in range(3)]
    g = dict(min0=a[0, 0], inv0=1.0 / w[0], min1=a[1, 0], inv1=1.0 / w[1], min2=a[2, 0],
             invn2=1.0 / a[2, 2], n0=int(a[0, 2]), n1=int(a[1, 2]), n2=int(a[2, 2]))
    g["ntotal"] = g["n0"] * g["n1"] * g["n2"]
    if coord == 1:
        g["max_ang"] = hi[1] / scale
    elif coord == 0:
        g["max_ang"] = hi[0] * math.sqrt(1.0 - a[1, 0] * a[1, 0]) / scale
    else:
        g["max_ang"] = hi[1]
    return g


def _accumulate(b, p1, p2, mode):
    v1, l1, w1 = p1[0], p1[1], p1[2]
    v2, l2, w2 = p2[0], p2[1], p2[2]
    if mode == 0:
        wdi, wdj = f32(w1 * v1), f32(w2 * v2)
        b[0] += float(wdi * wdj)
        b[1] += float(wdi)
        b[2] += float(wdj)
        b[3] += float(w1 * w2)
        b[4] += float(w1)
        b[5] += float(w2)
        b[6] += 0.5 * float(l1 + l2)
    else:
        wdi, wdj = float(w1) * float(v1), float(w2) * float(v2)
        b[0] += wdi * wdj
        b[1] += wdi
        b[2] += wdj
        b[3] += float(w1) * float(w2)
        b[4] += float(w1)
        b[5] += float(w2)
        b[6] += 0.5 * (float(l1) + float(l2))
    b[7] += 1


def xi(sightlines, pixels, coord, axes, scale, mode=1):
    """Returns (sums [ntotal, 8] float64 with count in column 7, stats)."""
    g = _grid(coord, axes, scale)
    cos_max = math.cos(g["max_ang"])
    out = np.zeros((g["ntotal"], 8))
    n = len(sightlines)
    trig = [(math.sin(s["dec"]), math.cos(s["dec"]), math.sin(s["ra"]), math.cos(s["ra"])) for s in sightlines]
    px = [[(f32(p["value"]), f32(p["loglam"]), f32(p["weight"]), f32(p["distance"]))
           for p in pixels[int(s["pixel_offset"]):int(s["pixel_offset"]) + int(s["num_pixels"])]]
          for s in sightlines]
    used_pairs = pix_pairs = pix_used = 0
    for i in range(n):
        for j in range(i + 1, n):
            a, b = trig[i], trig[j]
            c = a[0] * b[0] + a[1] * b[1] * (a[2] * b[2] + a[3] * b[3])
            if c <= cos_max:
                continue
            used_pairs += 1
            pix_pairs += len(px[i]) * len(px[j])
            sep = math.acos(c)
            for p1 in px[i]:
                d1, l1 = p1[3], p1[1]
                r1_sq = float(d1 * d1)
                two_r1_cos12 = float(f32(2) * d1) * c
                for p2 in px[j]:
                    d2, l2 = p2[3], p2[1]
                    if coord == 0:
                        r_sq = r1_sq + (float(d2) - two_r1_cos12) * float(d2)
                        r = math.sqrt(r_sq) if r_sq >= 0 else float("nan")
                        idx = ref_u32((r - g["min0"]) * g["inv0"])
                        if idx >= g["n0"]:
                            continue
                        if r == 0:
                            continue
                        mu = float(abs(d1 - d2)) / r
                        mb = ref_u32((mu - g["min1"]) * g["inv1"])
                        if mb >= g["n1"]:
                            continue
                        idx = (mb + idx * g["n1"]) & M32
                    elif coord == 1:
                        r_para = float(abs(d1 - d2))
                        idx = ref_u32((r_para - g["min0"]) * g["inv0"])
                        if idx >= g["n0"]:
                            continue
                        r_sq = r1_sq + (float(d2) - two_r1_cos12) * float(d2)
                        pb = ref_u32((math.sqrt(abs(r_sq - r_para * r_para)) - g["min1"]) * g["inv1"])
                        if pb >= g["n1"]:
                            continue
                        idx = (pb + idx * g["n1"]) & M32
                    else:
                        sb = ref_u32((sep - g["min1"]) * g["inv1"])
                        idx = ref_u32((float(abs(l1 - l2)) - g["min0"]) * g["inv0"])
                        if idx >= g["n0"]:
                            continue
                        idx = (sb + idx * g["n1"]) & M32
                    lz = 0.5 * float(l1 + l2)
                    zb = ref_u32((lz - g["min2"]) * g["invn2"])
                    idx = (zb + idx * g["n2"]) & M32
                    pix_used += 1
                    if idx >= g["ntotal"]:
                        continue
                    _accumulate(out[idx], p1, p2, mode)
    stats = dict(num_sightline_pairs_used=used_pairs, num_pixel_pairs=pix_pairs, num_pixel_pairs_used=pix_used)
    return out, stats
