"""Seeded synthetic microstructures (uint8 voxel images, numpy (z, y, x) arrays).

They stand in for the digital-rock datasets that chfem's example scripts download
(examples/scripts/run_drp_benchmarks.py:27-43), which are not available offline:
  * spheres(): non-overlapping balls (periodic distance) placed by seeded rejection until a
    target volume fraction is reached -- thermal two-phase inclusions;
  * grf(): periodic Gaussian random field (white noise smoothed by a Gaussian kernel in
    Fourier space) thresholded at a quantile -- two-phase elastic media;
  * pore_grf(): thresholded field whose pore phase (code 0) keeps only the clusters that
    percolate along the flow axis (26-connectivity, periodic) -- Stokes permeability.
Seeds follow seed = 1000*config + sample_index in the benchmarks.
"""
import numpy as np


def spheres(shape=(64, 64, 64), vf=0.30, rmin=4, rmax=8, seed=1000, codes=(0, 255), max_tries=200000, overlap=False):
    """Balls of integer radius uniform in [rmin, rmax] (code codes[1]) in a matrix (codes[0]),
    placed at uniform random centres (periodic) until the volume fraction reaches vf.  Without
    overlap a ball that would come within one voxel of an earlier one is rejected (random
    sequential addition, which jams near vf 0.38); with overlap every ball is kept."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    dims = np.array(shape, dtype=float)
    img = np.full(shape, codes[0], dtype=np.uint8)
    centers = np.zeros((0, 3))
    radii = np.zeros(0)
    target = vf * img.size
    filled = 0
    tries = 0
    while filled < target and tries < max_tries:
        tries += 1
        r = int(rng.integers(rmin, rmax + 1))
        c = np.array([rng.uniform(0, nz), rng.uniform(0, ny), rng.uniform(0, nx)])
        if not overlap and len(radii):
            d = np.abs(centers - c)
            d = np.minimum(d, dims - d)
            if np.any(np.sqrt((d ** 2).sum(axis=1)) < r + radii + 1):
                continue
        centers = np.vstack([centers, c])
        radii = np.append(radii, r)
        # paint the ball inside its periodic bounding box
        idx = []
        dist2 = 0.0
        for ax, n in enumerate(shape):
            lo, hi = int(np.floor(c[ax] - r)), int(np.ceil(c[ax] + r))
            pos = np.arange(lo, hi + 1)
            dd = np.abs(pos - c[ax])
            dd = np.minimum(dd, n - dd)
            idx.append(np.unique(np.mod(pos, n), return_index=True))
            dist2 = dist2 + (dd[idx[-1][1]] ** 2).reshape([-1 if a == ax else 1 for a in range(3)])
        box = np.ix_(idx[0][0], idx[1][0], idx[2][0])
        inside = dist2 <= r * r
        sub = img[box]
        filled += int(np.count_nonzero(inside & (sub == codes[0])))
        sub[inside] = codes[1]
        img[box] = sub
    return img


def _smooth_field(shape, corr, rng):
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(n) for n in shape]
    kz, ky, kx = np.meshgrid(*k, indexing="ij")
    g = np.exp(-2.0 * (np.pi * corr) ** 2 * (kz ** 2 + ky ** 2 + kx ** 2))
    return np.real(np.fft.ifftn(np.fft.fftn(noise) * g))


def grf(shape=(128, 128, 128), corr=6.0, fraction=0.40, seed=2000, codes=(0, 255)):
    """Two phases from a thresholded periodic GRF; codes[1] occupies `fraction` of the voxels."""
    rng = np.random.default_rng(seed)
    f = _smooth_field(shape, corr, rng)
    thr = np.quantile(f, 1.0 - fraction)
    return np.where(f > thr, codes[1], codes[0]).astype(np.uint8)


def _label_periodic(mask):
    from scipy import ndimage
    lab, n = ndimage.label(mask, structure=np.ones((3, 3, 3), dtype=bool))
    parent = np.arange(n + 1)

    def find(a):
        while parent[a] != a:
            parent[a] = parent[parent[a]]
            a = parent[a]
        return a

    def union(a, b):
        ra, rb = find(a), find(b)
        if ra != rb:
            parent[max(ra, rb)] = min(ra, rb)

    # 26-neighbour links across each periodic face
    for ax in range(3):
        a = np.take(lab, 0, axis=ax)
        b = np.take(lab, -1, axis=ax)
        for s0 in (-1, 0, 1):
            for s1 in (-1, 0, 1):
                bb = np.roll(np.roll(b, s0, axis=0), s1, axis=1)
                m = (a > 0) & (bb > 0)
                for u, v in zip(a[m].tolist(), bb[m].tolist()):
                    union(u, v)
    roots = np.array([find(i) for i in range(n + 1)])
    return roots[lab], n


def pore_grf(shape=(128, 128, 128), corr=8.0, porosity=0.35, seed=3000, axis=None, pore=0, solid=255):
    """Pore space (code `pore`) = lowest `porosity` fraction of a GRF, keeping only the
    clusters that touch both faces of the flow axis (all three axes when axis is None)."""
    rng = np.random.default_rng(seed)
    f = _smooth_field(shape, corr, rng)
    mask = f < np.quantile(f, porosity)
    lab, _ = _label_periodic(mask)
    keep = None
    axes = range(3) if axis is None else [axis]
    for ax in axes:
        a = set(np.unique(np.take(lab, 0, axis=ax)).tolist()) - {0}
        b = set(np.unique(np.take(lab, -1, axis=ax)).tolist()) - {0}
        both = a & b
        keep = both if keep is None else keep | both
    keep_mask = np.isin(lab, np.array(sorted(keep), dtype=lab.dtype)) if keep else np.zeros_like(mask)
    return np.where(keep_mask, pore, solid).astype(np.uint8)


def write_case(prefix, img, analysis, mat_props=None, tol=1e-6, maxit=10000, solver=0, voxel=1.0, refinement=1):
    """Write <prefix>.nf and <prefix>.raw for the CLI (chfem .nf grammar)."""
    from .io import export_for_chfem
    export_for_chfem(prefix + ".raw", img, analysis, mat_props=mat_props, voxel_size=voxel, solver_type=solver,
                     refinement=refinement, export_raw=True, export_nf=True, solver_tolerance=tol,
                     solver_maxiter=maxit)
    return prefix + ".nf", prefix + ".raw"
