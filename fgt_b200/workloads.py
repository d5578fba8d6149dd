"""Seeded synthetic point sets of the benchmark configurations.

No public dataset is involved: the point clouds are regenerated from their
stated distributions with numpy PCG64 (seed = 20261203 + config index).
"""
import numpy as np

SEED0 = 20261203


def rng_for(config_index):
    return np.random.Generator(np.random.PCG64(SEED0 + config_index))


def uniform(rng, n, dim):
    return rng.uniform(-0.5, 0.5, size=(n, dim))


def gaussian_clusters(rng, n, dim, ncl=64):
    """n points from ncl isotropic Gaussians: centres uniform in the box,
    sigma log-uniform in [1e-3, 5e-2], equal weights, clipped to the box."""
    cen = rng.uniform(-0.5, 0.5, size=(ncl, dim))
    sig = np.exp(rng.uniform(np.log(1e-3), np.log(5e-2), size=ncl))
    counts = rng.multinomial(n, np.full(ncl, 1.0 / ncl))
    lab = np.repeat(np.arange(ncl), counts)
    pts = cen[lab] + rng.standard_normal((n, dim)) * sig[lab, None]
    return np.clip(pts, -0.5, 0.5)


def sphere_surface(rng, n, radius=0.4, centre=0.0):
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return centre + radius * v


def sphere_with_background(rng, n, frac_bg=0.01, radius=0.4):
    """99% uniform on the sphere of radius 0.4 centred at 0, 1% uniform in
    [-0.5,0.5]^3 (highly non-uniform precision-sweep workload)."""
    nbg = int(round(n * frac_bg))
    pts = np.concatenate([sphere_surface(rng, n - nbg, radius), uniform(rng, nbg, 3)])
    return pts[rng.permutation(n)]


def wiggly_curve(rng, n, dim, rin=0.3, rwig=0.12, nwig=6):
    """Non-uniform point set of the reference test driver
    (test/pfgt/test_pfgt_all.f:146-166): r = rin + rwig*cos(nwig*theta),
    centred at 0.5, plus its three special sources (:188-206)."""
    theta = rng.uniform(0, np.pi, n)
    phi = rng.uniform(0, 2 * np.pi, n)
    rr = rin + rwig * np.cos(nwig * theta)
    if dim == 3:
        pts = np.stack([rr * np.sin(theta) * np.cos(phi) + 0.5,
                        rr * np.sin(theta) * np.sin(phi) + 0.5,
                        rr * np.cos(theta) + 0.5], axis=1)
    elif dim == 2:
        pts = np.stack([rr * np.cos(phi) + 0.5, rr * np.sin(phi) + 0.5], axis=1)
    else:
        i = np.arange(1, n + 1)
        pts = ((np.cos(i * np.pi / (n + 1)) + 1) / 2)[:, None]
    pts[0, :] = 0.0
    pts[1, :] = 1.0
    pts[2, :] = 0.05
    return pts


def config(index, scale=1.0, delta=None, eps=None):
    """Inputs of configuration `index` (1..5 as in the benchmark list).

    scale < 1 shrinks N (for tests); delta/eps override the cell of config 5.
    Returns a dict of pfgt arguments.
    """
    rng = rng_for(index)
    if index == 1:
        n = int(1e5 * scale)
        src = uniform(rng, n, 3)
        return dict(nd=1, dim=3, delta=1e-4, eps=1e-6, iperiod=0, sources=src,
                    charge=rng.uniform(-1, 1, (n, 1)), ifpgh=1, targets=None, ifpghtarg=0,
                    name="3D uniform N=1e5 sources=targets delta=1e-4 eps=1e-6 pot")
    if index == 2:
        n = int(2e6 * scale)
        src = gaussian_clusters(rng, n, 3)
        trg = uniform(rng, n, 3)
        return dict(nd=1, dim=3, delta=1e-5, eps=1e-9, iperiod=0, sources=src,
                    charge=rng.standard_normal((n, 1)), ifpgh=2, targets=trg, ifpghtarg=2,
                    name="3D 64-Gaussian clusters N=M=2e6 delta=1e-5 eps=1e-9 pot+grad")
    if index == 3:
        n = int(1e7 * scale)
        src = uniform(rng, n, 2)
        return dict(nd=4, dim=2, delta=1e-6, eps=1e-6, iperiod=1, sources=src,
                    charge=rng.uniform(-1, 1, (n, 4)), ifpgh=2, targets=None, ifpghtarg=0,
                    bs0=1.0, cen0=[0.0, 0.0],
                    name="2D periodic uniform N=1e7 nd=4 delta=1e-6 eps=1e-6 pot+grad")
    if index == 5:
        n = int(1e7 * scale)
        src = sphere_with_background(rng, n)
        return dict(nd=1, dim=3, delta=1e-4 if delta is None else delta,
                    eps=1e-6 if eps is None else eps, iperiod=0, sources=src,
                    charge=rng.standard_normal((n, 1)), ifpgh=2, targets=src.copy(),
                    ifpghtarg=2,
                    name="3D sphere+1% background N=M=1e7 pot+grad")
    raise ValueError(index)


def batch_instances(count=512, seed_index=4, nmin=1e3, nmax=1e5):
    """Batched workload: independent 3D free-space instances."""
    rng = rng_for(seed_index)
    out = []
    for _ in range(count):
        n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
        if rng.uniform() < 0.5:
            src = uniform(rng, n, 3)
        else:
            src = sphere_surface(rng, n, radius=rng.uniform(0.3, 0.45))
        delta = float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-2))))
        eps = float(rng.choice([1e-3, 1e-6]))
        out.append(dict(nd=1, dim=3, delta=delta, eps=eps, iperiod=0, sources=src,
                        charge=rng.uniform(-1, 1, (n, 1)), ifpgh=1))
    return out
