"""The benchmark configurations as parity workloads: the generator images, the
quality -> qindex, QM and lambda laws of the library, and the default decision
CDF snapshot of the frame's coefficient q context.

  C1     512x512, seed 1, sigma 4, 4:4:4, quality 60 (qindex 70)
  C2q40  1920x1080, seed 2, sigma 4 + texture band + gradient quadrant, 4:2:0,
         quality 40 (qindex 116)
  C2q60  the same at seed 3, quality 60 (qindex 70)
  C2q80  the same at seed 4, quality 80 (qindex 35)
  C3     4096x4096, seed 5, sigma 8 noise on the left half, piecewise-constant
         cells on the right half, 4:4:4, quality 60 (qindex 70): two tiles
         (the whole-frame encode only)

The reconstruction snapshot the candidates predict from is the source plus a
seeded +-3 coding error (the decision engine that would supply the real one
is not part of this library)."""
import functools
import os
import types

import numpy as np

from maroontree_b200 import synth

CONFIGS = {
    "C1": dict(w=512, h=512, seed=1, variant="plain", quality=60, sub=0),
    "C2q40": dict(w=1920, h=1080, seed=2, variant="1080p", quality=40, sub=2),
    "C2q60": dict(w=1920, h=1080, seed=3, variant="1080p", quality=60, sub=2),
    "C2q80": dict(w=1920, h=1080, seed=4, variant="1080p", quality=80, sub=2),
    "C3": dict(w=4096, h=4096, seed=5, variant="large", quality=60, sub=0, sigma=8.0),
}
NAMES = ["C1", "C2q40", "C2q60", "C2q80"]  # the kernel-family parity workloads
THREADS = os.cpu_count() or 1


@functools.lru_cache(maxsize=None)
def workload(name):
    import maroontree_b200 as mt

    c = CONFIGS[name]
    rgb = synth.generate_rgb(c["w"], c["h"], c["seed"], sigma=c.get("sigma", 4.0), variant=c["variant"])
    src = synth.rgb_to_luma(rgb)
    rec = synth.synthetic_recon(src, c["seed"] + 1000)
    qidx = mt.quality_to_q(c["quality"])
    qm_y, qm_uv = mt.qm_levels(qidx, c["sub"])
    q = mt.quant_new(qidx, 8, qm_y)
    lam = mt.rd_lambdas(qidx, q.dc_q, c["sub"])
    return types.SimpleNamespace(name=name, w=c["w"], h=c["h"], sub=c["sub"], rgb=rgb, src=src, rec=rec, qidx=qidx,
                                 qm_level=qm_y, qm_uv=qm_uv, q=q, lam=lam, qctx=mt.qcat(qidx))


def qm(mt, wl, n):
    return mt.qm_row(wl.qm_level, 0, n) if wl.qm_level < 15 else None


def cdfs(mt, wl, n, plane=0):
    return mt.coef_cdfs_default(wl.qctx, n, n, plane)
