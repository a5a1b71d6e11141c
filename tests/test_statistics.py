"""Statistical parity: the GPU painter in single precision against the
reference painter in double precision, on independent random streams, for
both integrators (BPT and PT).

Each side renders K one-pass images with different seeds; per pixel the two
means are compared with the z-score

    z = (mean_gpu - mean_ref) / sqrt(var_gpu / K + var_ref / K)

from the pass-to-pass variances.  An unbiased match leaves |z| > 3 on about
0.27 % of the pixels and |z| > 6 on none; the bar here is at most 0.5 % of
the pixels above 3 and none above 6, and the relative RMSE of the two means
is reported against the noise it should have.  Both sides are seeded, so the
outcome is reproducible.
"""

from __future__ import annotations

import numpy as np
import pytest

from math_b200 import painter as P
from math_b200 import scenes

K = 48

CASES = {
    "cornell3d": (lambda: scenes.cornell_3d(size=(32, 32), subdivisions=3), False, 16, 5, "bpt"),
    "cornell4d": (lambda: scenes.cornell_4d(size=(10, 10, 10), points=600), True, 8, 6, "bpt"),
    "cornell3d_pt": (lambda: scenes.cornell_3d(size=(32, 32), subdivisions=3), False, 16, 5, "pt"),
}


def luminance(rgb: np.ndarray) -> np.ndarray:
    return rgb.astype(np.float64) @ np.array([0.2126, 0.7152, 0.0722])


def z_scores(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """a, b: [K, pixels] per-pass values."""
    ma, mb = a.mean(axis=0), b.mean(axis=0)
    va, vb = a.var(axis=0, ddof=1), b.var(axis=0, ddof=1)
    se = np.sqrt(va / len(a) + vb / len(b))
    z = np.zeros_like(ma)
    nz = se > 0
    z[nz] = (ma[nz] - mb[nz]) / se[nz]
    z[~nz & (ma != mb)] = np.inf
    return z


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_float_gpu_matches_double_reference_statistically(painter, oracle_lib, name):
    make, spectrum, spp, depth, integrator = CASES[name]
    desc = make()
    scene = P.Scene(desc, "float", spectrum)
    gpu = []
    for k in range(K):
        p = scene.painter(spp, depth, seed=1000 + k, integrator=integrator)
        p.run(1)
        gpu.append(luminance(p.images()[0]))
        p.close()
    ref_scene = oracle_lib.Scene(desc, "double", spectrum)
    ref_scene.set_integrator(integrator)
    ref = [luminance(ref_scene.render_image(spp, depth, seed=5000 + k)[0]) for k in range(K)]
    gpu = np.array(gpu)
    ref = np.array(ref)
    z = np.abs(z_scores(gpu, ref))
    share = float((z > 3).mean())
    rmse = float(np.sqrt(((gpu.mean(0) - ref.mean(0)) ** 2).sum() / (ref.mean(0) ** 2).sum()))
    noise = float(np.sqrt((ref.var(0, ddof=1) / K * 2).sum() / (ref.mean(0) ** 2).sum()))
    print(f"{name}: |z|>3 share {share:.4f}, max |z| {z.max():.2f}, rel RMSE of means {rmse:.4f} "
          f"(expected from noise {noise:.4f})")
    assert share <= 0.005
    assert z.max() < 6
    assert rmse < 2 * noise + 1e-3
