"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is involved: every workload is generated from
numpy.random.Generator(PCG64(seed)), seed = 20261203 + config index.

  C1  plain 2D, 10,000 Diracs uniform in [0,1]^2, w = 0, unit box, density 1
  C2  2D at scale: 1,000,000 Diracs, 50% uniform + 50% from 20 isotropic
      Gaussian clusters (centres uniform, sigma 0.02, clamped to the box),
      weights uniform in [-1e-6, 1e-6], unit box, density 1
  C3  2D partial OT: 500,000 Diracs uniform, w = (0.5/sqrt(n))^2, 512x512
      image 1 + 0.5 sin(6 pi x) cos(4 pi y) scaled to total mass 0.8, disc clip
  C4  3D: 200,000 Diracs, 70% uniform + 30% jittered lattice (+-0.1 spacing),
      w = 0, unit cube, density 1 + 0.3 x y z (normalised)
  C5  serving stream: Poisson arrivals, 80% 2D / 20% 3D, n log-uniform in
      [1e3, 2e5], uniform or clustered points (50/50)
"""
import numpy as np

SEED0 = 20261203


def rng_for(config_index, salt=0):
    return np.random.Generator(np.random.PCG64(SEED0 + config_index + 1000 * salt))


def uniform_points(n, dim, rng):
    return rng.random((n, dim))


def clustered_points(n, dim, rng, nb_clusters=20, sigma=0.02, boundary="clamp"):
    """Isotropic Gaussian clusters (centres uniform); points leaving the unit
    box are clamped to it (boundary="clamp", the C2 definition) or mirrored
    back into it (boundary="reflect": no two points coincide)."""
    centres = rng.random((nb_clusters, dim))
    k = np.arange(n) % nb_clusters
    p = centres[k] + sigma * rng.standard_normal((n, dim))
    if boundary == "reflect":
        p = np.abs(p)
        return np.where(p > 1.0, 2.0 - p, p)
    return np.clip(p, 0.0, 1.0)


def config1(n=10_000):
    rng = rng_for(1)
    return {"positions": uniform_points(n, 2, rng), "weights": np.zeros(n), "domain": "unit_box",
            "target": np.full(n, 1.0 / n)}


def config2(n=1_000_000):
    rng = rng_for(2)
    nu = n // 2
    p = np.concatenate([uniform_points(nu, 2, rng), clustered_points(n - nu, 2, rng)])
    w = rng.uniform(-1e-6, 1e-6, n)
    return {"positions": p, "weights": w, "domain": "unit_box", "target": np.full(n, 1.0 / n)}


def c3_image(res=512, total=0.8):
    x = (np.arange(res) + 0.5) / res
    X, Y = np.meshgrid(x, x)          # image[iy, ix]: last axis is x
    img = 1 + 0.5 * np.sin(6 * np.pi * X) * np.cos(4 * np.pi * Y)
    # ScaledImage::measure = mean * area (area 1 here)
    return img * (total / img.mean())


def config3(n=500_000, res=512):
    rng = rng_for(3)
    p = uniform_points(n, 2, rng)
    w = np.full(n, (0.5 / np.sqrt(n)) ** 2)
    return {"positions": p, "weights": w, "image": c3_image(res), "target": np.full(n, 0.8 / n)}


def config4(n=200_000):
    rng = rng_for(4)
    nu = int(round(0.7 * n))
    nl = n - nu
    m = int(np.ceil(nl ** (1.0 / 3.0)))
    g = (np.arange(m) + 0.5) / m
    L = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)[:nl]
    L = L + rng.uniform(-0.1 / m, 0.1 / m, L.shape)
    p = np.concatenate([uniform_points(nu, 3, rng), L])
    return {"positions": p, "weights": np.zeros(n), "domain": "unit_cube", "target": np.full(n, 1.0 / n),
            "density": C4_DENSITY}


# 1 + 0.3 xyz in the multilinear basis (1, x, y, z, xy, xz, yz, xyz),
# normalised to unit mass on the unit cube (its integral there is 1 + 0.3/8)
C4_DENSITY = np.array([1.0, 0, 0, 0, 0, 0, 0, 0.3]) / (1.0 + 0.3 / 8)


def serving_requests(count=2000, rate_hz=50.0, seed_salt=0):
    """Poisson stream of solve requests (C5).  Clustered requests mirror
    their points at the box faces instead of clamping them: clamping makes
    coincident Diracs (in 3D, at the box corners), for which no weights
    reach the target masses."""
    rng = rng_for(5, seed_salt)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, count))
    reqs = []
    for k in range(count):
        dim = 2 if rng.random() < 0.8 else 3
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        clustered = rng.random() < 0.5
        r = np.random.Generator(np.random.PCG64(SEED0 + 5 + 7919 * (k + 1)))
        p = clustered_points(n, dim, r, boundary="reflect") if clustered else uniform_points(n, dim, r)
        reqs.append({"arrival_s": float(t[k]), "dim": dim, "n": n, "clustered": bool(clustered), "positions": p})
    return reqs
